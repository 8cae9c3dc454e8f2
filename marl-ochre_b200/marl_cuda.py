"""Python binding of libmarl_cuda.so (ctypes over the C ABI in include/marl_cuda.h).

This is the host-side mirror of the reference's plugin seam for the per-tick
field-and-cell path:

* ``Context`` — device-resident field, light, occupancy and cell table, with
  per-phase calls.  ``Context.diffuse_tick_with_cells`` is the counterpart of
  ``GpuFieldDiffuser::diffuse_tick_with_cells``
  (crates/marl-gpu/src/field_diffusion.rs:158-268): same arguments (a host
  field, a host occupancy of one bool per voxel, the simulation config) and
  the same error behaviour (invalid sizes -> ``MarlError`` with status
  INVALID_INPUT, ``diffusion_substeps == 0`` -> no work).
* ``Engine`` — the tick loop of ``marl_sim::run`` (crates/marl-sim/src/lib.rs:
  160-277) with fate, division and mutation on the host.

There is no CPU fallback: if the shared library or a CUDA device is missing,
the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int32, c_uint8, c_uint32, c_uint64, c_void_p

import numpy as np

S_EXT = 12
M_INT = 16
R_MAX = 16
NO_COFACTOR = 0xFF

EVENT_NONE, EVENT_DIVISION, EVENT_DEATH, EVENT_QUIESCENCE = 0, 1, 2, 3
SOURCES_ADDITIVE, SOURCES_DIRICHLET = 0, 1

STATUS_NAMES = {
    0: "OK",
    1: "INVALID_INPUT",
    2: "NO_DEVICE",
    3: "CUDA",
    4: "OUT_OF_MEMORY",
    5: "TIMEOUT",
    6: "CAPACITY",
    7: "STATE",
}

# ---- plain-data layouts (must match include/marl_cuda.h) --------------------
RECEPTOR_DTYPE = np.dtype([("k_half", "<f4"), ("n_hill", "<f4"), ("gain", "<f4")])
TRANSPORT_DTYPE = np.dtype(
    [("uptake_rate", "<f4"), ("secrete_rate", "<f4"), ("ext_species", "u1"), ("int_species", "u1"), ("_pad", "u1", (2,))]
)
REACTION_DTYPE = np.dtype(
    [("substrate", "u1"), ("product", "u1"), ("catalyst", "u1"), ("cofactor", "u1"),
     ("k_m", "<f4"), ("v_max", "<f4"), ("k_cat", "<f4")]
)
EFFECTOR_DTYPE = np.dtype(
    [("threshold", "<f4"), ("rate", "<f4"), ("int_species", "u1"), ("ext_species", "u1"), ("_pad", "u1", (2,))]
)
FATE_DTYPE = np.dtype(
    [("division_energy", "<f4"), ("death_energy", "<f4"), ("quiescence_energy", "<f4"), ("division_prep_ticks", "<f4")]
)
RULESET_DTYPE = np.dtype(
    [("receptors", RECEPTOR_DTYPE, (8,)), ("transport", TRANSPORT_DTYPE, (8,)), ("reactions", REACTION_DTYPE, (16,)),
     ("effectors", EFFECTOR_DTYPE, (8,)), ("fate", FATE_DTYPE), ("hgt_propensity", "<f4"), ("mutation_rate", "<f4")]
)
CELL_DTYPE = np.dtype(
    [("pos", "<u2", (3,)), ("quiescent", "u1"), ("starter_type", "u1"), ("age", "<u4"), ("prep_remaining", "<u2"),
     ("_pad0", "<u2"), ("lineage_id", "<u8"), ("internal", "<f4", (16,)), ("ruleset", RULESET_DTYPE)]
)
CHANGE_DTYPE = np.dtype(
    [("cell", "<u4"), ("event", "u1"), ("quiescent", "u1"), ("_pad", "<u2"), ("internal", "<f4", (16,))]
)
assert RULESET_DTYPE.itemsize == 568 and CELL_DTYPE.itemsize == 656 and CHANGE_DTYPE.itemsize == 72


class SimParams(ctypes.Structure):
    """marl_sim_params == SimulationConfig (crates/marl-config/src/lib.rs:41-106)."""

    _fields_ = [
        ("dx", c_float), ("dt", c_float), ("diffusion_substeps", c_uint32),
        ("d_voxel", c_float * S_EXT), ("lambda_decay", c_float * S_EXT),
        ("source_rate_oxidant", c_float), ("source_rate_carbon", c_float), ("source_rate_reductant", c_float),
        ("epsilon", c_float), ("c_max", c_float), ("lambda_maintenance", c_float), ("hard_death_floor", c_float),
        ("reaction_maintenance", c_float), ("base_division_prep", c_float), ("prep_maintenance_multiplier", c_float),
        ("rush_penalty_rate", c_float), ("alpha_eps", c_float), ("k_eps", c_float), ("light_efficiency", c_float),
        ("surface_intensity", c_float), ("cell_absorption", c_float), ("chemical_absorption", c_float),
        ("light_floor", c_float), ("mutation_stddev", c_float), ("structural_mutation_rate_mult", c_float),
        ("meta_mutation_rate", c_float), ("meta_mutation_clamp_low", c_float), ("meta_mutation_clamp_high", c_float),
        ("hill_exponent_clamp_low", c_float), ("hill_exponent_clamp_high", c_float),
        ("active_reaction_threshold", c_float), ("seed_margin", c_uint32), ("phototroph_z_lo", c_float),
        ("phototroph_z_hi", c_float), ("chemolithotroph_z_lo", c_float), ("chemolithotroph_z_hi", c_float),
        ("anaerobe_z_lo", c_float), ("anaerobe_z_hi", c_float), ("division_neighbor_distance", c_uint32),
        ("boundary_prime_layers", c_uint32), ("boundary_prime_oxidant", c_float),
        ("boundary_prime_carbon", c_float), ("boundary_prime_reductant", c_float), ("source_mode", c_uint32),
    ]

    def copy(self) -> "SimParams":
        out = SimParams()
        ctypes.memmove(ctypes.byref(out), ctypes.byref(self), ctypes.sizeof(SimParams))
        return out


class EngineStats(ctypes.Structure):
    _fields_ = [(name, c_uint64) for name in (
        "tick", "population", "total_divisions", "total_deaths", "tick_divisions", "tick_deaths",
        "h2d_bytes_last_tick", "d2h_bytes_last_tick")]


class Counters(ctypes.Structure):
    _fields_ = [("h2d_bytes", c_uint64), ("d2h_bytes", c_uint64), ("kernel_launches", c_uint64), ("ticks", c_uint64),
                ("device_us", c_double)]


class EditList(ctypes.Structure):
    _fields_ = [
        ("n_halve", c_uint32), ("halve", POINTER(c_uint32)),
        ("n_deaths", c_uint32), ("deaths", POINTER(c_uint32)),
        ("n_moves", c_uint32), ("move_dst", POINTER(c_uint32)), ("move_src", POINTER(c_uint32)),
        ("n_after_deaths", c_uint32),
        ("n_births", c_uint32), ("births", c_void_p),
    ]


class RunSpec(ctypes.Structure):
    _fields_ = [("gx", c_int32), ("gy", c_int32), ("gz", c_int32), ("seed_count", c_uint32), ("rng_seed", c_uint64),
                ("cell_capacity", c_uint32), ("_pad", c_uint32)]


class MarlError(RuntimeError):
    def __init__(self, status: int, where: str, message: str = ""):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{where}: {self.status_name} ({status}) {message}".strip())


class SurrogateConfig(ctypes.Structure):
    _fields_ = [("max_pairs", c_uint32), ("batch", c_uint32), ("lr", c_float), ("beta1", c_float),
                ("beta2", c_float), ("adam_eps", c_float), ("seed", c_uint64)]


class SurrogateEval(ctypes.Structure):
    _fields_ = [("rows", c_uint32), ("accepted", c_uint32), ("max_err", c_float), ("mean_err", c_float),
                ("mse_normalised", c_float)]


class SurrogateCounters(ctypes.Structure):
    _fields_ = [("cells", c_uint64), ("speculated", c_uint64), ("accepted", c_uint64), ("rejected", c_uint64),
                ("max_err", c_float)]


class Stats(ctypes.Structure):
    _fields_ = [("population", c_uint64), ("top", c_uint64), ("middle", c_uint64), ("bottom", c_uint64),
                ("avg_energy", ctypes.c_double), ("avg_enzyme", ctypes.c_double),
                ("avg_enzyme_b", ctypes.c_double),
                ("avg_active_reactions", ctypes.c_double), ("oxidant_top", c_float), ("oxidant_middle", c_float),
                ("reductant_bottom", c_float), ("organic_middle", c_float)]


class FateStats(ctypes.Structure):
    _fields_ = [(name, c_uint64) for name in (
        "tick", "population", "total_divisions", "total_deaths", "tick_divisions", "tick_deaths", "tick_births",
        "tick_moves")]


VIEWER_CELL_DTYPE = np.dtype([("pos", "<f4", (3,)), ("lineage_id", "<u8"), ("starter_type", "u1"),
                              ("energy", "<f4")])  # packed, 25 bytes
assert VIEWER_CELL_DTYPE.itemsize == 25


def viewer_cells(ctx_handle, n: int) -> np.ndarray:
    """marl_ctx_viewer_cells: the packed 25-byte viewer records of a context's cells."""
    lib = load()
    out = np.zeros(max(n, 1), VIEWER_CELL_DTYPE)
    got = c_uint32()
    _check(lib.marl_ctx_viewer_cells(ctx_handle, _ptr(out), out.nbytes, ctypes.byref(got)), "marl_ctx_viewer_cells")
    return out[: got.value]


def write_dump(directory: str, tick: int, dims, field: np.ndarray | None, cells: np.ndarray | None) -> None:
    """marl_write_dump: run_meta.json and tick_<tick>.{field,cells}.bin under `directory`."""
    lib = load()
    X, Y, Z = dims
    f = None if field is None else _as_field(np.ascontiguousarray(field, np.float32), dims)
    c = None if cells is None else np.ascontiguousarray(cells, VIEWER_CELL_DTYPE)
    _check(lib.marl_write_dump(os.fsencode(directory), tick, X, Y, Z, _ptr(f) if f is not None else None,
                               _ptr(c) if c is not None and c.size else (None if c is None else
                                                                          _ptr(np.zeros(1, np.uint8))),
                               0 if c is None else c.size), "marl_write_dump")


RULESETS_LAYERS, RULESETS_FULL, RULESETS_BOTH = 1, 2, 3


def ctx_write_ruleset_dumps(ctx_handle, directory: str, tick: int, mode: int = RULESETS_BOTH) -> None:
    """marl_ctx_write_ruleset_dumps: ruleset sidecars of a context's cells (device reductions)."""
    _check(load().marl_ctx_write_ruleset_dumps(ctx_handle, os.fsencode(directory), tick, mode),
           "marl_ctx_write_ruleset_dumps")


def write_ruleset_dumps(directory: str, tick: int, dims, cells: np.ndarray, mode: int = RULESETS_BOTH) -> None:
    """marl_write_ruleset_dumps: the same sidecars from host cells (CELL_DTYPE records)."""
    X, Y, Z = dims
    c = np.ascontiguousarray(cells, CELL_DTYPE)
    _check(load().marl_write_ruleset_dumps(os.fsencode(directory), tick, X, Y, Z, _ptr(c) if c.size else None,
                                           c.size, mode), "marl_write_ruleset_dumps")


SURR_FEATURES = 93
SURR_RAW_STRIDE = 112
SURR_PARAMS = 256 * 128 + 256 + 256 * 256 + 256 + 16 * 256 + 16
SURR_NORM = 93 + 93 + 16 + 16
SURR_OFF, SURR_CAPTURE, SURR_GATED, SURR_TRUSTED = 0, 1, 2, 3

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmarl_cuda.so")

# Every symbol declared in include/marl_cuda.h (checked by tests against the header).
EXPORTED = [
    "marl_sim_params_default", "marl_last_error", "marl_abi_version",
    "marl_ctx_create", "marl_ctx_destroy", "marl_ctx_set_stream", "marl_ctx_set_params", "marl_ctx_synchronize",
    "marl_ctx_set_tile", "marl_ctx_get_tile", "marl_ctx_set_cell_lanes", "marl_ctx_set_wait_limit",
    "marl_ctx_test_hold_dependency", "marl_ctx_set_receptor_output", "marl_ctx_download_receptor_activations",
    "marl_ctx_hgt", "marl_ctx_autotune", "marl_ctx_counters",
    "marl_upload_field", "marl_download_field", "marl_upload_light", "marl_download_light",
    "marl_upload_cells", "marl_download_cells", "marl_cell_count", "marl_download_occupancy",
    "marl_apply_boundary_sources", "marl_diffuse", "marl_light_update", "marl_cell_phase", "marl_tick",
    "marl_apply_edits", "marl_mass_f64", "marl_diffuse_tick_with_cells", "marl_diffuse_device",
    "marl_diffuse_device_noalloc",
    "marl_ruleset_pack_canonical", "marl_ruleset_unpack_canonical",
    "marl_engine_create", "marl_engine_create_from_state", "marl_engine_destroy", "marl_engine_set_stream",
    "marl_engine_step", "marl_engine_stats_get", "marl_engine_get_cells", "marl_engine_get_field",
    "marl_engine_get_light", "marl_engine_ctx",
    "marl_batch_create", "marl_batch_destroy", "marl_batch_set_stream", "marl_batch_set_host_threads",
    "marl_batch_set_tile", "marl_batch_get_tile", "marl_batch_autotune", "marl_batch_set_graph", "marl_batch_step",
    "marl_batch_run_count", "marl_batch_stats_get", "marl_batch_get_cells", "marl_batch_get_field",
    "marl_batch_get_light", "marl_batch_counters",
    "marl_surrogate_config_default", "marl_surrogate_create", "marl_surrogate_destroy", "marl_surrogate_set_stream",
    "marl_surrogate_pair_count", "marl_surrogate_download_pairs", "marl_surrogate_upload_pairs",
    "marl_surrogate_prepare", "marl_surrogate_set_lr", "marl_surrogate_train", "marl_surrogate_evaluate",
    "marl_surrogate_get_weights", "marl_surrogate_set_weights", "marl_surrogate_gradients",
    "marl_surrogate_infer_device", "marl_ctx_set_surrogate", "marl_ctx_surrogate_counters",
    "marl_batch_set_surrogate", "marl_batch_surrogate_counters", "marl_surrogate_set_inference",
    "marl_ctx_stats", "marl_ctx_viewer_cells", "marl_write_dump", "marl_ctx_write_ruleset_dumps",
    "marl_write_ruleset_dumps",
    "marl_ctx_fate_init", "marl_ctx_fate", "marl_ctx_fate_stats", "marl_ctx_set_events", "marl_ctx_run_ticks",
    "marl_fate_stream_probe", "marl_fate_stream_ln", "marl_engine_set_device_fate", "marl_batch_set_device_fate",
    "marl_selftest_small_division",
]

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libmarl_cuda.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built; run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    P = c_void_p
    sig = {
        "marl_sim_params_default": (c_int32, [POINTER(SimParams)]),
        "marl_last_error": (c_char_p, []),
        "marl_abi_version": (c_uint32, []),
        "marl_ctx_create": (c_int32, [c_int32, c_int32, c_int32, POINTER(SimParams), c_uint32, POINTER(c_void_p)]),
        "marl_ctx_destroy": (None, [P]),
        "marl_ctx_set_stream": (c_int32, [P, P]),
        "marl_ctx_set_params": (c_int32, [P, POINTER(SimParams)]),
        "marl_ctx_synchronize": (c_int32, [P]),
        "marl_ctx_set_tile": (c_int32, [P, c_int32, c_int32]),
        "marl_ctx_get_tile": (c_int32, [P, POINTER(c_int32), POINTER(c_int32)]),
        "marl_ctx_set_cell_lanes": (c_int32, [P, c_uint32]),
        "marl_ctx_set_wait_limit": (c_int32, [P, c_uint32]),
        "marl_ctx_test_hold_dependency": (c_int32, [P, c_uint32, c_uint32, c_uint32]),
        "marl_ctx_set_receptor_output": (c_int32, [P, c_int32]),
        "marl_ctx_download_receptor_activations": (c_int32, [P, P, c_uint32, POINTER(c_uint32)]),
        "marl_ctx_hgt": (c_int32, [P, P, P, c_uint32, c_uint64, c_uint64]),
        "marl_ctx_autotune": (c_int32, [P, c_int32, POINTER(c_float)]),
        "marl_ctx_counters": (c_int32, [P, POINTER(Counters)]),
        "marl_upload_field": (c_int32, [P, P]),
        "marl_download_field": (c_int32, [P, P]),
        "marl_upload_light": (c_int32, [P, P]),
        "marl_download_light": (c_int32, [P, P]),
        "marl_upload_cells": (c_int32, [P, P, c_uint32]),
        "marl_download_cells": (c_int32, [P, P, c_uint32, POINTER(c_uint32)]),
        "marl_cell_count": (c_int32, [P, POINTER(c_uint32)]),
        "marl_download_occupancy": (c_int32, [P, P]),
        "marl_apply_boundary_sources": (c_int32, [P]),
        "marl_diffuse": (c_int32, [P, c_uint32, c_int32]),
        "marl_light_update": (c_int32, [P]),
        "marl_cell_phase": (c_int32, [P, P]),
        "marl_tick": (c_int32, [P, P, c_uint32, POINTER(c_uint32)]),
        "marl_apply_edits": (c_int32, [P, POINTER(EditList)]),
        "marl_mass_f64": (c_int32, [P, P]),
        "marl_diffuse_tick_with_cells": (c_int32, [P, P, P]),
        "marl_diffuse_device": (c_int32, [P, P, P, c_int32, c_int32, c_int32, POINTER(SimParams), c_uint32, P]),
        "marl_diffuse_device_noalloc": (c_int32, [P, P, c_int32, c_int32, c_int32, POINTER(SimParams), c_uint32, P]),
        "marl_ruleset_pack_canonical": (c_int32, [P, P]),
        "marl_ruleset_unpack_canonical": (c_int32, [P, P]),
        "marl_engine_create": (c_int32, [c_int32, c_int32, c_int32, POINTER(SimParams), c_uint64, c_uint32, c_uint32,
                                         POINTER(c_void_p)]),
        "marl_engine_create_from_state": (c_int32, [c_int32, c_int32, c_int32, POINTER(SimParams), c_uint64, P, P,
                                                    c_uint32, c_uint32, POINTER(c_void_p)]),
        "marl_engine_destroy": (None, [P]),
        "marl_engine_set_stream": (c_int32, [P, P]),
        "marl_engine_step": (c_int32, [P, c_uint32]),
        "marl_engine_stats_get": (c_int32, [P, POINTER(EngineStats)]),
        "marl_engine_get_cells": (c_int32, [P, P, c_uint32, POINTER(c_uint32)]),
        "marl_engine_get_field": (c_int32, [P, P]),
        "marl_engine_get_light": (c_int32, [P, P]),
        "marl_engine_ctx": (c_void_p, [P]),
        "marl_batch_create": (c_int32, [POINTER(RunSpec), c_uint32, POINTER(SimParams), POINTER(c_void_p)]),
        "marl_batch_destroy": (None, [P]),
        "marl_batch_set_stream": (c_int32, [P, P]),
        "marl_batch_set_host_threads": (c_int32, [P, c_int32]),
        "marl_batch_set_tile": (c_int32, [P, c_int32, c_int32]),
        "marl_batch_get_tile": (c_int32, [P, POINTER(c_int32), POINTER(c_int32)]),
        "marl_batch_autotune": (c_int32, [P, c_int32, POINTER(c_float)]),
        "marl_batch_set_graph": (c_int32, [P, c_int32]),
        "marl_batch_step": (c_int32, [P, c_uint32]),
        "marl_batch_run_count": (c_int32, [P, POINTER(c_uint32)]),
        "marl_batch_stats_get": (c_int32, [P, c_uint32, POINTER(EngineStats)]),
        "marl_batch_get_cells": (c_int32, [P, c_uint32, P, c_uint32, POINTER(c_uint32)]),
        "marl_batch_get_field": (c_int32, [P, c_uint32, P]),
        "marl_batch_get_light": (c_int32, [P, c_uint32, P]),
        "marl_batch_counters": (c_int32, [P, POINTER(Counters)]),
        "marl_surrogate_config_default": (c_int32, [POINTER(SurrogateConfig)]),
        "marl_surrogate_create": (c_int32, [POINTER(SurrogateConfig), POINTER(c_void_p)]),
        "marl_surrogate_destroy": (None, [P]),
        "marl_surrogate_set_stream": (c_int32, [P, P]),
        "marl_surrogate_pair_count": (c_int32, [P, POINTER(c_uint32)]),
        "marl_surrogate_download_pairs": (c_int32, [P, c_uint32, c_uint32, P]),
        "marl_surrogate_upload_pairs": (c_int32, [P, P, c_uint32]),
        "marl_surrogate_prepare": (c_int32, [P, c_uint32]),
        "marl_surrogate_set_lr": (c_int32, [P, c_float]),
        "marl_surrogate_train": (c_int32, [P, c_uint32, P]),
        "marl_surrogate_evaluate": (c_int32, [P, c_uint32, c_uint32, c_float, POINTER(SurrogateEval), P]),
        "marl_surrogate_get_weights": (c_int32, [P, P, P]),
        "marl_surrogate_set_weights": (c_int32, [P, P, P]),
        "marl_surrogate_gradients": (c_int32, [P, P, P, c_uint32, P, POINTER(c_float), P]),
        "marl_surrogate_infer_device": (c_int32, [P, P, c_uint32, P, c_uint32]),
        "marl_ctx_set_surrogate": (c_int32, [P, P, c_int32, c_float]),
        "marl_ctx_surrogate_counters": (c_int32, [P, POINTER(SurrogateCounters)]),
        "marl_batch_set_surrogate": (c_int32, [P, P, c_int32, c_float]),
        "marl_batch_surrogate_counters": (c_int32, [P, POINTER(SurrogateCounters)]),
        "marl_surrogate_set_inference": (c_int32, [P, c_int32]),
        "marl_ctx_stats": (c_int32, [P, POINTER(Stats), P, P]),
        "marl_ctx_viewer_cells": (c_int32, [P, P, c_uint64, POINTER(c_uint32)]),
        "marl_write_dump": (c_int32, [c_char_p, c_uint64, c_int32, c_int32, c_int32, P, P, c_uint32]),
        "marl_ctx_write_ruleset_dumps": (c_int32, [P, c_char_p, c_uint64, c_int32]),
        "marl_write_ruleset_dumps": (c_int32, [c_char_p, c_uint64, c_int32, c_int32, c_int32, P, c_uint32, c_int32]),
        "marl_ctx_fate_init": (c_int32, [P, c_uint64, c_uint64, c_uint64, c_uint64]),
        "marl_ctx_fate": (c_int32, [P]),
        "marl_ctx_fate_stats": (c_int32, [P, POINTER(FateStats)]),
        "marl_ctx_set_events": (c_int32, [P, P, c_uint32]),
        "marl_ctx_run_ticks": (c_int32, [P, c_uint32]),
        "marl_fate_stream_probe": (c_int32, [c_uint64, c_uint64, c_uint32, c_uint32, c_float, P, P]),
        "marl_fate_stream_ln": (c_int32, [P, c_uint32, P]),
        "marl_selftest_small_division": (c_int32, [P]),
        "marl_engine_set_device_fate": (c_int32, [P, c_int32]),
        "marl_batch_set_device_fate": (c_int32, [P, c_int32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int, where: str) -> None:
    if status != 0:
        msg = _lib.marl_last_error().decode(errors="replace") if _lib is not None else ""
        raise MarlError(status, where, msg)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def default_params() -> SimParams:
    """SimulationConfig::default() (crates/marl-config/src/lib.rs:108-168)."""
    lib = load()
    p = SimParams()
    _check(lib.marl_sim_params_default(ctypes.byref(p)), "marl_sim_params_default")
    return p


def _as_field(field: np.ndarray, dims) -> np.ndarray:
    X, Y, Z = dims
    if field.dtype != np.float32 or field.size != X * Y * Z * S_EXT or not field.flags.c_contiguous:
        raise MarlError(1, "field", f"expected contiguous float32 with {X * Y * Z * S_EXT} values")
    return field


class Context:
    """Device-resident state for one grid (marl_ctx)."""

    def __init__(self, dims, params: SimParams | None = None, cell_capacity: int = 1 << 16):
        self.lib = load()
        self.dims = tuple(int(d) for d in dims)
        self.params = (params or default_params()).copy()
        h = c_void_p()
        X, Y, Z = self.dims
        _check(self.lib.marl_ctx_create(X, Y, Z, ctypes.byref(self.params), cell_capacity, ctypes.byref(h)),
               "marl_ctx_create")
        self.h = h
        self.cell_capacity = cell_capacity

    # lifetime
    def close(self):
        if getattr(self, "h", None):
            self.lib.marl_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def voxels(self) -> int:
        X, Y, Z = self.dims
        return X * Y * Z

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib.marl_ctx_set_stream(self.h, c_void_p(stream_ptr)), "marl_ctx_set_stream")

    def set_params(self, params: SimParams) -> None:
        self.params = params.copy()
        _check(self.lib.marl_ctx_set_params(self.h, ctypes.byref(self.params)), "marl_ctx_set_params")

    def synchronize(self) -> None:
        _check(self.lib.marl_ctx_synchronize(self.h), "marl_ctx_synchronize")

    def set_tile(self, tile: int, zc: int) -> None:
        _check(self.lib.marl_ctx_set_tile(self.h, tile, zc), "marl_ctx_set_tile")

    def set_receptor_output(self, enable: bool = True) -> None:
        """Phase 1 (receptor activations) as an output of every later cell phase."""
        _check(self.lib.marl_ctx_set_receptor_output(self.h, 1 if enable else 0), "marl_ctx_set_receptor_output")

    def receptor_activations(self) -> np.ndarray:
        """The last cell phase's receptor activations, [n][8]."""
        n = self.cell_count()
        out = np.zeros((max(n, 1), 8), np.float32)
        got = c_uint32()
        _check(self.lib.marl_ctx_download_receptor_activations(self.h, _ptr(out), out.shape[0], ctypes.byref(got)),
               "marl_ctx_download_receptor_activations")
        return out[: got.value]

    def hgt(self, donors, recipients, seed: int, tick: int) -> None:
        """transfer_reaction for each (donor, recipient) pair, in order."""
        d = np.ascontiguousarray(donors, np.uint32)
        r = np.ascontiguousarray(recipients, np.uint32)
        if d.shape != r.shape:
            raise ValueError("donors and recipients differ in length")
        _check(self.lib.marl_ctx_hgt(self.h, _ptr(d) if d.size else None, _ptr(r) if r.size else None, d.size,
                                     seed, tick), "marl_ctx_hgt")

    def set_wait_limit(self, polls: int) -> None:
        """Polls of an unfinished dependency before a cell gives up (0: default)."""
        _check(self.lib.marl_ctx_set_wait_limit(self.h, polls), "marl_ctx_set_wait_limit")

    def test_hold_dependency(self, cell: int, face: int, slot: int) -> None:
        """Failure injection for the next cell phase: `cell` also waits, through
        empty face `face`, for slot `slot` (population <= slot < capacity),
        which no cell completes; the phase then reports TIMEOUT."""
        _check(self.lib.marl_ctx_test_hold_dependency(self.h, cell, face, slot), "marl_ctx_test_hold_dependency")

    def get_tile(self) -> tuple[int, int]:
        t, z = c_int32(), c_int32()
        _check(self.lib.marl_ctx_get_tile(self.h, ctypes.byref(t), ctypes.byref(z)), "marl_ctx_get_tile")
        return t.value, z.value

    def autotune(self, reps: int = 5) -> float:
        """Pick the fastest diffusion tile shape / z-chunk; returns us per substep."""
        us = c_float()
        _check(self.lib.marl_ctx_autotune(self.h, reps, ctypes.byref(us)), "marl_ctx_autotune")
        return us.value

    def counters(self) -> dict:
        c = Counters()
        _check(self.lib.marl_ctx_counters(self.h, ctypes.byref(c)), "marl_ctx_counters")
        return {name: getattr(c, name) for name, _ in Counters._fields_}

    # state transfer
    def upload_field(self, field: np.ndarray) -> None:
        f = _as_field(np.ascontiguousarray(field, dtype=np.float32), self.dims)
        _check(self.lib.marl_upload_field(self.h, _ptr(f)), "marl_upload_field")

    def download_field(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X, S_EXT), np.float32)
        _check(self.lib.marl_download_field(self.h, _ptr(out)), "marl_download_field")
        return out

    def upload_light(self, light: np.ndarray) -> None:
        l = np.ascontiguousarray(light, dtype=np.float32)
        if l.size != self.voxels:
            raise MarlError(1, "upload_light", "size mismatch")
        _check(self.lib.marl_upload_light(self.h, _ptr(l)), "marl_upload_light")

    def download_light(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X), np.float32)
        _check(self.lib.marl_download_light(self.h, _ptr(out)), "marl_download_light")
        return out

    def upload_cells(self, cells: np.ndarray) -> None:
        c = np.ascontiguousarray(cells, dtype=CELL_DTYPE)
        _check(self.lib.marl_upload_cells(self.h, _ptr(c) if c.size else None, c.size), "marl_upload_cells")

    def cell_count(self) -> int:
        n = c_uint32()
        _check(self.lib.marl_cell_count(self.h, ctypes.byref(n)), "marl_cell_count")
        return n.value

    def download_cells(self) -> np.ndarray:
        n = self.cell_count()
        out = np.zeros(max(n, 1), CELL_DTYPE)
        got = c_uint32()
        _check(self.lib.marl_download_cells(self.h, _ptr(out), out.size, ctypes.byref(got)), "marl_download_cells")
        return out[: got.value]

    def download_occupancy(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X), np.uint8)
        _check(self.lib.marl_download_occupancy(self.h, _ptr(out)), "marl_download_occupancy")
        return out

    # phases
    def apply_boundary_sources(self) -> None:
        _check(self.lib.marl_apply_boundary_sources(self.h), "marl_apply_boundary_sources")

    def diffuse(self, substeps: int | None = None, fuse_sources: bool = False) -> None:
        s = self.params.diffusion_substeps if substeps is None else substeps
        _check(self.lib.marl_diffuse(self.h, s, 1 if fuse_sources else 0), "marl_diffuse")

    def light_update(self) -> None:
        _check(self.lib.marl_light_update(self.h), "marl_light_update")

    def cell_phase(self) -> np.ndarray:
        n = self.cell_count()
        ev = np.zeros(max(n, 1), np.uint8)
        _check(self.lib.marl_cell_phase(self.h, _ptr(ev)), "marl_cell_phase")
        return ev[:n]

    def tick(self, cap: int | None = None) -> np.ndarray:
        cap = self.cell_capacity if cap is None else cap
        out = np.zeros(max(cap, 1), CHANGE_DTYPE)
        n = c_uint32()
        _check(self.lib.marl_tick(self.h, _ptr(out), cap, ctypes.byref(n)), "marl_tick")
        return out[: n.value]

    def apply_edits(self, halve=(), deaths=(), moves=(), n_after_deaths=None, births=None) -> None:
        halve = np.ascontiguousarray(halve, np.uint32)
        deaths = np.ascontiguousarray(deaths, np.uint32)
        moves = np.asarray(moves, np.uint32).reshape(-1, 2)
        dst = np.ascontiguousarray(moves[:, 0])
        src = np.ascontiguousarray(moves[:, 1])
        births = np.zeros(0, CELL_DTYPE) if births is None else np.ascontiguousarray(births, CELL_DTYPE)
        if n_after_deaths is None:
            n_after_deaths = self.cell_count() - deaths.size
        u32p = POINTER(c_uint32)
        e = EditList(
            halve.size, halve.ctypes.data_as(u32p), deaths.size, deaths.ctypes.data_as(u32p),
            dst.size, dst.ctypes.data_as(u32p), src.ctypes.data_as(u32p), int(n_after_deaths),
            births.size, births.ctypes.data if births.size else None,
        )
        _check(self.lib.marl_apply_edits(self.h, ctypes.byref(e)), "marl_apply_edits")

    def mass_f64(self) -> np.ndarray:
        out = np.zeros(S_EXT, np.float64)
        _check(self.lib.marl_mass_f64(self.h, _ptr(out)), "marl_mass_f64")
        return out

    def stats(self):
        """print_stats / print_z_profile quantities (marl_ctx_stats): (dict,
        cells per z, centre column [5][Z] = light, species 1-4)."""
        st = Stats()
        Z = self.dims[2]
        per_z = np.zeros(Z, np.uint32)
        col = np.zeros((5, Z), np.float32)
        _check(self.lib.marl_ctx_stats(self.h, ctypes.byref(st), _ptr(per_z), _ptr(col)), "marl_ctx_stats")
        return {name: getattr(st, name) for name, _ in Stats._fields_}, per_z, col

    # device fate
    def fate_init(self, seed: int, tick: int = 0, total_divisions: int = 0, total_deaths: int = 0) -> None:
        _check(self.lib.marl_ctx_fate_init(self.h, seed, tick, total_divisions, total_deaths), "marl_ctx_fate_init")

    def fate(self) -> None:
        """Enqueue one device fate step over the current events."""
        _check(self.lib.marl_ctx_fate(self.h), "marl_ctx_fate")

    def fate_stats(self) -> dict:
        st = FateStats()
        _check(self.lib.marl_ctx_fate_stats(self.h, ctypes.byref(st)), "marl_ctx_fate_stats")
        return {name: getattr(st, name) for name, _ in FateStats._fields_}

    def set_events(self, events: np.ndarray) -> None:
        ev = np.ascontiguousarray(events, np.uint8)
        _check(self.lib.marl_ctx_set_events(self.h, _ptr(ev) if ev.size else None, ev.size), "marl_ctx_set_events")

    def run_ticks(self, ticks: int = 1) -> None:
        """Whole ticks with device fate, enqueued without synchronising."""
        _check(self.lib.marl_ctx_run_ticks(self.h, ticks), "marl_ctx_run_ticks")

    def diffuse_tick_with_cells(self, field: np.ndarray, occupancy: np.ndarray) -> None:
        """GpuFieldDiffuser::diffuse_tick_with_cells: `field` is updated in place."""
        X, Y, Z = self.dims
        if field.dtype != np.float32 or field.size != X * Y * Z * S_EXT or not field.flags.c_contiguous:
            raise MarlError(1, "diffuse_tick_with_cells",
                            f"field has {field.size} floats, expected {X * Y * Z * S_EXT}")
        occ = np.ascontiguousarray(occupancy).astype(np.uint8, copy=False)
        if occ.size != X * Y * Z:
            raise MarlError(1, "diffuse_tick_with_cells", f"occupancy has {occ.size} voxels, expected {X * Y * Z}")
        _check(self.lib.marl_diffuse_tick_with_cells(self.h, _ptr(field), _ptr(occ)), "marl_diffuse_tick_with_cells")


def fate_stream_probe(seed: int, tick: int, parent: int, count: int, stddev: float = 1.0):
    """marl_fate_stream_probe: `count` u64 draws and `count` normals of the
    device-fate stream keyed by (seed, tick, parent), computed on the GPU."""
    lib = load()
    u = np.zeros(max(count, 1), np.uint64)
    z = np.zeros(max(count, 1), np.float32)
    _check(lib.marl_fate_stream_probe(seed, tick, parent, count, stddev, _ptr(u), _ptr(z)), "marl_fate_stream_probe")
    return u[:count], z[:count]


def fate_stream_ln(x: np.ndarray) -> np.ndarray:
    """marl_fate_stream_ln: the device-fate streams' logarithm, on the GPU."""
    lib = load()
    xs = np.ascontiguousarray(x, np.float64)
    out = np.zeros(max(xs.size, 1), np.float64)
    _check(lib.marl_fate_stream_ln(_ptr(xs), xs.size, _ptr(out)), "marl_fate_stream_ln")
    return out[:xs.size]


def selftest_small_division() -> int:
    """marl_selftest_small_division: differences between the cell loop's
    division by 3, 5 or 6 and the IEEE division over every finite float."""
    lib = load()
    out = np.zeros(1, np.uint64)
    _check(lib.marl_selftest_small_division(_ptr(out)), "marl_selftest_small_division")
    return int(out[0])


def diffuse_device(field_ptr: int, scratch_ptr: int, occ_ptr: int, dims, params: SimParams, substeps: int,
                   stream_ptr: int = 0) -> None:
    """marl_diffuse_device on caller-owned device buffers (raw pointers)."""
    lib = load()
    X, Y, Z = dims
    _check(lib.marl_diffuse_device(c_void_p(field_ptr), c_void_p(scratch_ptr), c_void_p(occ_ptr), X, Y, Z,
                                   ctypes.byref(params), substeps, c_void_p(stream_ptr)), "marl_diffuse_device")


def diffuse_device_noalloc(field_ptr: int, occ_ptr: int, dims, params: SimParams, substeps: int,
                           stream_ptr: int = 0) -> None:
    """marl_diffuse_device_noalloc: like diffuse_device, but with no device allocation at all.

    For callers that must not allocate device memory while they run.  Its
    scratch (about 13 MiB) is a static device array shared by every call, so
    calls must not overlap on the GPU; grids are limited to 262,144 voxels.
    """
    lib = load()
    X, Y, Z = dims
    _check(lib.marl_diffuse_device_noalloc(c_void_p(field_ptr), c_void_p(occ_ptr), X, Y, Z, ctypes.byref(params),
                                           substeps, c_void_p(stream_ptr)), "marl_diffuse_device_noalloc")


def pack_ruleset(rs: np.ndarray) -> bytes:
    lib = load()
    r = np.ascontiguousarray(rs, RULESET_DTYPE).reshape(1)
    out = np.zeros(536, np.uint8)
    _check(lib.marl_ruleset_pack_canonical(_ptr(r), _ptr(out)), "marl_ruleset_pack_canonical")
    return out.tobytes()


def unpack_ruleset(payload: bytes) -> np.ndarray:
    lib = load()
    buf = np.frombuffer(payload, np.uint8).copy()
    if buf.size != 536:
        raise MarlError(1, "unpack_ruleset", "payload must be 536 bytes")
    out = np.zeros(1, RULESET_DTYPE)
    _check(lib.marl_ruleset_unpack_canonical(_ptr(buf), _ptr(out)), "marl_ruleset_unpack_canonical")
    return out[0]


class Engine:
    """marl_sim::run's tick loop (seeding, device tick, host fate) — marl_engine."""

    def __init__(self, dims, params: SimParams | None = None, rng_seed: int = 42, seed_count: int = 30,
                 cell_capacity: int = 1 << 18, field: np.ndarray | None = None, cells: np.ndarray | None = None):
        self.lib = load()
        self.dims = tuple(int(d) for d in dims)
        self.params = (params or default_params()).copy()
        X, Y, Z = self.dims
        h = c_void_p()
        if field is None:
            _check(self.lib.marl_engine_create(X, Y, Z, ctypes.byref(self.params), rng_seed, seed_count,
                                               cell_capacity, ctypes.byref(h)), "marl_engine_create")
        else:
            f = _as_field(np.ascontiguousarray(field, np.float32), self.dims)
            c = np.ascontiguousarray(cells if cells is not None else np.zeros(0, CELL_DTYPE), CELL_DTYPE)
            _check(self.lib.marl_engine_create_from_state(X, Y, Z, ctypes.byref(self.params), rng_seed, _ptr(f),
                                                          _ptr(c) if c.size else None, c.size, cell_capacity,
                                                          ctypes.byref(h)), "marl_engine_create_from_state")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.marl_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib.marl_engine_set_stream(self.h, c_void_p(stream_ptr)), "marl_engine_set_stream")

    def counters(self) -> dict:
        c = Counters()
        _check(self.lib.marl_ctx_counters(self.lib.marl_engine_ctx(self.h), ctypes.byref(c)), "marl_ctx_counters")
        return {name: getattr(c, name) for name, _ in Counters._fields_}

    def autotune(self, reps: int = 5) -> float:
        us = c_float()
        _check(self.lib.marl_ctx_autotune(self.lib.marl_engine_ctx(self.h), reps, ctypes.byref(us)),
               "marl_ctx_autotune")
        return us.value

    def step(self, ticks: int = 1) -> None:
        _check(self.lib.marl_engine_step(self.h, ticks), "marl_engine_step")

    def set_device_fate(self, enable: bool = True) -> None:
        """Fate on the device (per-division streams keyed by rng_seed) or on the host."""
        _check(self.lib.marl_engine_set_device_fate(self.h, 1 if enable else 0), "marl_engine_set_device_fate")

    def device_stats(self):
        """marl_ctx_stats on the engine's context: (dict, cells per z, centre column [5][Z])."""
        st = Stats()
        Z = self.dims[2]
        per_z = np.zeros(Z, np.uint32)
        col = np.zeros((5, Z), np.float32)
        _check(self.lib.marl_ctx_stats(self.lib.marl_engine_ctx(self.h), ctypes.byref(st), _ptr(per_z), _ptr(col)),
               "marl_ctx_stats")
        return {name: getattr(st, name) for name, _ in Stats._fields_}, per_z, col

    def stats(self) -> dict:
        s = EngineStats()
        _check(self.lib.marl_engine_stats_get(self.h, ctypes.byref(s)), "marl_engine_stats_get")
        return {name: getattr(s, name) for name, _ in EngineStats._fields_}

    def cells(self) -> np.ndarray:
        n = self.stats()["population"]
        out = np.zeros(max(int(n), 1), CELL_DTYPE)
        got = c_uint32()
        _check(self.lib.marl_engine_get_cells(self.h, _ptr(out), out.size, ctypes.byref(got)), "marl_engine_get_cells")
        return out[: got.value]

    def field(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X, S_EXT), np.float32)
        _check(self.lib.marl_engine_get_field(self.h, _ptr(out)), "marl_engine_get_field")
        return out

    def light(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X), np.float32)
        _check(self.lib.marl_engine_get_light(self.h, _ptr(out)), "marl_engine_get_light")
        return out


class Batch:
    """Many independent runs advanced together — marl_batch.

    `runs` is a list of (dims, rng_seed) or (dims, rng_seed, seed_count,
    cell_capacity); run r behaves exactly like Engine(dims, params, rng_seed,
    seed_count, cell_capacity)."""

    def __init__(self, runs, params: SimParams | None = None, seed_count: int = 30, cell_capacity: int = 0):
        self.lib = load()
        self.params = (params or default_params()).copy()
        specs = (RunSpec * len(runs))()
        self.dims = []
        for i, r in enumerate(runs):
            dims, seed = r[0], r[1]
            sc = r[2] if len(r) > 2 else seed_count
            cap = r[3] if len(r) > 3 else cell_capacity
            X, Y, Z = (int(d) for d in dims)
            specs[i] = RunSpec(X, Y, Z, sc, seed, cap, 0)
            self.dims.append((X, Y, Z))
        h = c_void_p()
        _check(self.lib.marl_batch_create(specs, len(runs), ctypes.byref(self.params), ctypes.byref(h)),
               "marl_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.marl_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.dims)

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib.marl_batch_set_stream(self.h, c_void_p(stream_ptr)), "marl_batch_set_stream")

    def set_host_threads(self, threads: int) -> None:
        _check(self.lib.marl_batch_set_host_threads(self.h, threads), "marl_batch_set_host_threads")

    def set_tile(self, tile: int, zc: int) -> None:
        _check(self.lib.marl_batch_set_tile(self.h, tile, zc), "marl_batch_set_tile")

    def get_tile(self) -> tuple[int, int]:
        t, z = c_int32(), c_int32()
        _check(self.lib.marl_batch_get_tile(self.h, ctypes.byref(t), ctypes.byref(z)), "marl_batch_get_tile")
        return t.value, z.value

    def autotune(self, reps: int = 5) -> float:
        us = c_float()
        _check(self.lib.marl_batch_autotune(self.h, reps, ctypes.byref(us)), "marl_batch_autotune")
        return us.value

    def set_graph(self, use_graph: bool) -> None:
        _check(self.lib.marl_batch_set_graph(self.h, 1 if use_graph else 0), "marl_batch_set_graph")

    def step(self, ticks: int = 1) -> None:
        _check(self.lib.marl_batch_step(self.h, ticks), "marl_batch_step")

    def set_device_fate(self, enable: bool = True) -> None:
        """Fate of every run on the device (per-division streams keyed by each run's seed) or on the host."""
        _check(self.lib.marl_batch_set_device_fate(self.h, 1 if enable else 0), "marl_batch_set_device_fate")

    def set_surrogate(self, surrogate: "Surrogate | None", mode: int, tol: float = 1e-3) -> None:
        _check(self.lib.marl_batch_set_surrogate(self.h, surrogate.h if surrogate is not None else None, mode, tol),
               "marl_batch_set_surrogate")

    def surrogate_counters(self) -> dict:
        c = SurrogateCounters()
        _check(self.lib.marl_batch_surrogate_counters(self.h, ctypes.byref(c)), "marl_batch_surrogate_counters")
        return {name: getattr(c, name) for name, _ in SurrogateCounters._fields_}

    def counters(self) -> dict:
        c = Counters()
        _check(self.lib.marl_batch_counters(self.h, ctypes.byref(c)), "marl_batch_counters")
        return {name: getattr(c, name) for name, _ in Counters._fields_}

    def stats(self, run: int) -> dict:
        s = EngineStats()
        _check(self.lib.marl_batch_stats_get(self.h, run, ctypes.byref(s)), "marl_batch_stats_get")
        return {name: getattr(s, name) for name, _ in EngineStats._fields_}

    def cells(self, run: int) -> np.ndarray:
        n = self.stats(run)["population"]
        out = np.zeros(max(int(n), 1), CELL_DTYPE)
        got = c_uint32()
        _check(self.lib.marl_batch_get_cells(self.h, run, _ptr(out), out.size, ctypes.byref(got)),
               "marl_batch_get_cells")
        return out[: got.value]

    def field(self, run: int) -> np.ndarray:
        X, Y, Z = self.dims[run]
        out = np.empty((Z, Y, X, S_EXT), np.float32)
        _check(self.lib.marl_batch_get_field(self.h, run, _ptr(out)), "marl_batch_get_field")
        return out

    def light(self, run: int) -> np.ndarray:
        X, Y, Z = self.dims[run]
        out = np.empty((Z, Y, X), np.float32)
        _check(self.lib.marl_batch_get_light(self.h, run, _ptr(out)), "marl_batch_get_light")
        return out


class Surrogate:
    """Learned reaction surrogate (marl_surrogate): pair store, training on the
    GPU, evaluation and inference.  See include/marl_cuda.h for the features."""

    def __init__(self, max_pairs: int | None = None, batch: int | None = None, lr: float | None = None,
                 seed: int | None = None):
        self.lib = load()
        cfg = SurrogateConfig()
        _check(self.lib.marl_surrogate_config_default(ctypes.byref(cfg)), "marl_surrogate_config_default")
        if max_pairs is not None:
            cfg.max_pairs = max_pairs
        if batch is not None:
            cfg.batch = batch
        if lr is not None:
            cfg.lr = lr
        if seed is not None:
            cfg.seed = seed
        self.cfg = cfg
        h = c_void_p()
        _check(self.lib.marl_surrogate_create(ctypes.byref(cfg), ctypes.byref(h)), "marl_surrogate_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.marl_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib.marl_surrogate_set_stream(self.h, c_void_p(stream_ptr)), "marl_surrogate_set_stream")

    def pair_count(self) -> int:
        n = c_uint32()
        _check(self.lib.marl_surrogate_pair_count(self.h, ctypes.byref(n)), "marl_surrogate_pair_count")
        return n.value

    def download_pairs(self, row0: int = 0, n: int | None = None) -> np.ndarray:
        n = self.pair_count() - row0 if n is None else n
        out = np.zeros((max(n, 1), SURR_RAW_STRIDE), np.float32)
        _check(self.lib.marl_surrogate_download_pairs(self.h, row0, n, _ptr(out)), "marl_surrogate_download_pairs")
        return out[:n]

    def upload_pairs(self, rows: np.ndarray) -> None:
        r = np.ascontiguousarray(rows, np.float32).reshape(-1, SURR_RAW_STRIDE)
        _check(self.lib.marl_surrogate_upload_pairs(self.h, _ptr(r), r.shape[0]), "marl_surrogate_upload_pairs")

    def prepare(self, n_train: int) -> None:
        _check(self.lib.marl_surrogate_prepare(self.h, n_train), "marl_surrogate_prepare")

    def set_lr(self, lr: float) -> None:
        _check(self.lib.marl_surrogate_set_lr(self.h, lr), "marl_surrogate_set_lr")

    def train(self, steps: int) -> np.ndarray:
        loss = np.zeros(max(steps, 1), np.float32)
        _check(self.lib.marl_surrogate_train(self.h, steps, _ptr(loss)), "marl_surrogate_train")
        return loss[:steps]

    def evaluate(self, row0: int, n: int, tol: float = 1e-3, per_row: bool = False):
        ev = SurrogateEval()
        errs = np.zeros(n, np.float32) if per_row else None
        _check(self.lib.marl_surrogate_evaluate(self.h, row0, n, tol, ctypes.byref(ev),
                                                _ptr(errs) if per_row else None), "marl_surrogate_evaluate")
        out = {name: getattr(ev, name) for name, _ in SurrogateEval._fields_}
        if per_row:
            out["row_err"] = errs
        return out

    def get_weights(self) -> tuple[np.ndarray, np.ndarray]:
        p = np.zeros(SURR_PARAMS, np.float32)
        nrm = np.zeros(SURR_NORM, np.float32)
        _check(self.lib.marl_surrogate_get_weights(self.h, _ptr(p), _ptr(nrm)), "marl_surrogate_get_weights")
        return p, nrm

    def set_weights(self, params: np.ndarray | None = None, norm: np.ndarray | None = None) -> None:
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        nrm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        _check(self.lib.marl_surrogate_set_weights(self.h, _ptr(p) if p is not None else None,
                                                   _ptr(nrm) if nrm is not None else None),
               "marl_surrogate_set_weights")

    def gradients(self, x_bf16: np.ndarray, t: np.ndarray):
        """One forward + backward without an update: (grads, loss, y)."""
        x = np.ascontiguousarray(x_bf16, np.uint16)
        tt = np.ascontiguousarray(t, np.float32)
        B = x.shape[0]
        g = np.zeros(SURR_PARAMS, np.float32)
        y = np.zeros((B, 16), np.float32)
        loss = c_float()
        _check(self.lib.marl_surrogate_gradients(self.h, _ptr(x), _ptr(tt), B, _ptr(g), ctypes.byref(loss), _ptr(y)),
               "marl_surrogate_gradients")
        return g, loss.value, y

    def set_inference(self, fused: bool) -> None:
        _check(self.lib.marl_surrogate_set_inference(self.h, 1 if fused else 0), "marl_surrogate_set_inference")

    def infer_device(self, x_ptr: int, n: int, y_ptr: int, ldy: int) -> None:
        _check(self.lib.marl_surrogate_infer_device(self.h, c_void_p(x_ptr), n, c_void_p(y_ptr), ldy),
               "marl_surrogate_infer_device")


def ctx_set_surrogate(ctx_handle, surrogate: "Surrogate | None", mode: int, tol: float = 1e-3) -> None:
    """marl_ctx_set_surrogate on a context handle (Context.h or marl_engine_ctx)."""
    lib = load()
    _check(lib.marl_ctx_set_surrogate(ctx_handle, surrogate.h if surrogate is not None else None, mode, tol),
           "marl_ctx_set_surrogate")


def ctx_surrogate_counters(ctx_handle) -> dict:
    lib = load()
    c = SurrogateCounters()
    _check(lib.marl_ctx_surrogate_counters(ctx_handle, ctypes.byref(c)), "marl_ctx_surrogate_counters")
    return {name: getattr(c, name) for name, _ in SurrogateCounters._fields_}
