"""TEST INFRASTRUCTURE ONLY — ctypes wrapper over oracle/liboracle.so.

The C++ oracle (oracle/oracle.cpp) restates the reference MARL-OCHRE hot path
on the CPU.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg may import this module; the product never does.  See oracle.cpp's header
for the parity pin status of each part.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from ctypes import POINTER, c_float, c_int, c_int32, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "marl-ochre_b200"))
from marl_cuda import CELL_DTYPE, RULESET_DTYPE, SimParams  # noqa: E402  (plain-data layouts only)

LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = ctypes.CDLL(LIB_PATH)
    P = c_void_p
    sp = POINTER(SimParams)
    sig = {
        "oracle_default_params": (None, [sp]),
        "oracle_struct_layout": (None, [P]),
        "oracle_set_threads": (None, [c_int]),
        "oracle_max_threads": (c_int, []),
        "oracle_sources_f32": (None, [P, c_int, c_int, c_int, sp]),
        "oracle_diffuse_f32": (None, [P, P, c_int, c_int, c_int, sp, c_uint32]),
        "oracle_diffuse_f64": (None, [P, P, P, c_int, c_int, c_int, sp, c_uint32, c_int]),
        "oracle_light_f32": (None, [P, P, P, c_int, c_int, c_int, sp]),
        "oracle_light_f64": (None, [P, P, P, c_int, c_int, c_int, sp]),
        "oracle_cell_tick": (c_int, [P, P, c_float, sp, P]),
        "oracle_cell_phase_f32": (None, [P, P, P, c_uint32, c_int, c_int, c_int, sp, P]),
        "oracle_cell_phase_f64": (None, [P, P, P, c_uint32, c_int, c_int, c_int, sp, P]),
        "oracle_cell_phase_act_f32": (None, [P, P, P, c_uint32, c_int, c_int, c_int, sp, P, P]),
        "oracle_hgt": (None, [P, c_uint32, P, P, c_uint32, c_uint64, c_uint64]),
        "oracle_mutate": (None, [P, P, sp]),
        "oracle_rng_seed": (None, [c_uint64, P]),
        "oracle_rng_next_u64": (c_uint64, [P]),
        "oracle_make_starter": (None, [c_int, P, c_uint64, P]),
        "oracle_world_create": (c_void_p, [c_int, c_int, c_int, sp, c_uint64, c_uint32]),
        "oracle_world_create_empty": (c_void_p, [c_int, c_int, c_int, sp, c_uint64]),
        "oracle_world_destroy": (None, [P]),
        "oracle_world_set_field": (None, [P, P]),
        "oracle_world_get_field": (None, [P, P]),
        "oracle_world_set_light": (None, [P, P]),
        "oracle_world_get_light": (None, [P, P]),
        "oracle_world_set_cells": (None, [P, P, c_uint32]),
        "oracle_world_cell_count": (c_uint32, [P]),
        "oracle_world_get_cells": (c_uint32, [P, P, c_uint32]),
        "oracle_world_get_occupancy": (None, [P, P]),
        "oracle_world_get_rng": (None, [P, P]),
        "oracle_world_sources": (None, [P]),
        "oracle_world_diffuse": (None, [P, c_uint32]),
        "oracle_world_light": (None, [P]),
        "oracle_world_cell_phase": (None, [P, P]),
        "oracle_world_fate": (None, [P, P, c_uint32]),
        "oracle_world_tick": (None, [P, c_uint32]),
        "oracle_world_stats": (None, [P, P]),
        "oracle_world_set_fate_mode": (None, [P, c_int]),
        "oracle_world_set_tick": (None, [P, c_uint64]),
        "oracle_fate_stream": (None, [c_uint64, c_uint64, c_uint32, c_uint32, c_float, P, P]),
        "oracle_fate_log": (None, [P, c_uint32, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _p(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


def default_params() -> SimParams:
    p = SimParams()
    lib().oracle_default_params(ctypes.byref(p))
    return p


def struct_layout() -> np.ndarray:
    out = np.zeros(10, np.uint64)
    lib().oracle_struct_layout(_p(out))
    return out


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def sources(field: np.ndarray, dims, params: SimParams) -> None:
    X, Y, Z = dims
    lib().oracle_sources_f32(_p(field), X, Y, Z, ctypes.byref(params))


def diffuse(field: np.ndarray, occ: np.ndarray | None, dims, params: SimParams, substeps: int) -> None:
    """In-place Field::diffuse_tick_with_cells (occ=None: Field::diffuse_tick)."""
    X, Y, Z = dims
    keep = None if occ is None else np.ascontiguousarray(occ, np.uint8)
    o = None if keep is None else _p(keep)
    lib().oracle_diffuse_f32(_p(field), o, X, Y, Z, ctypes.byref(params), substeps)


def diffuse_f64(field: np.ndarray, occ: np.ndarray, dims, params: SimParams, substeps: int,
                apply_sources: bool = False) -> np.ndarray:
    X, Y, Z = dims
    f = np.ascontiguousarray(field, np.float32)
    out = np.empty(f.shape, np.float64)
    o = np.ascontiguousarray(occ, np.uint8)
    lib().oracle_diffuse_f64(_p(f), _p(out), _p(o), X, Y, Z, ctypes.byref(params), substeps, int(apply_sources))
    return out


def light(field: np.ndarray, occ: np.ndarray, dims, params: SimParams) -> np.ndarray:
    X, Y, Z = dims
    out = np.empty((Z, Y, X), np.float32)
    f = np.ascontiguousarray(field, np.float32)
    o = np.ascontiguousarray(occ, np.uint8)
    lib().oracle_light_f32(_p(out), _p(f), _p(o), X, Y, Z, ctypes.byref(params))
    return out


def light_f64(field: np.ndarray, occ: np.ndarray, dims, params: SimParams) -> np.ndarray:
    X, Y, Z = dims
    out = np.empty((Z, Y, X), np.float64)
    f = np.ascontiguousarray(field, np.float32)
    o = np.ascontiguousarray(occ, np.uint8)
    lib().oracle_light_f64(_p(out), _p(f), _p(o), X, Y, Z, ctypes.byref(params))
    return out


def cell_tick(cell: np.ndarray, ext, light_value: float, params: SimParams):
    """One CellState::tick; returns (updated cell, deltas[12], event)."""
    c = np.array(cell, CELL_DTYPE).reshape(1).copy()
    e = np.ascontiguousarray(ext, np.float32)
    d = np.zeros(12, np.float32)
    ev = lib().oracle_cell_tick(_p(c), _p(e), c_float(light_value), ctypes.byref(params), _p(d))
    return c[0], d, ev


def cell_phase(field: np.ndarray, light_arr: np.ndarray, cells: np.ndarray, dims, params: SimParams):
    """The sequential cell loop; returns (field, cells, events) as new arrays."""
    X, Y, Z = dims
    f = np.ascontiguousarray(field, np.float32).copy()
    l = np.ascontiguousarray(light_arr, np.float32)
    c = np.ascontiguousarray(cells, CELL_DTYPE).copy()
    ev = np.zeros(max(c.size, 1), np.int32)
    lib().oracle_cell_phase_f32(_p(f), _p(l), _p(c) if c.size else None, c.size, X, Y, Z, ctypes.byref(params),
                                _p(ev))
    return f, c, ev[: c.size]


def cell_phase_act(field: np.ndarray, light_arr: np.ndarray, cells: np.ndarray, dims, params: SimParams):
    """The sequential cell loop plus each cell's receptor activations (cell.rs:206-220);
    returns (field, cells, events, activations [n][8])."""
    X, Y, Z = dims
    f = np.ascontiguousarray(field, np.float32).copy()
    l = np.ascontiguousarray(light_arr, np.float32)
    c = np.ascontiguousarray(cells, CELL_DTYPE).copy()
    ev = np.zeros(max(c.size, 1), np.int32)
    act = np.zeros((max(c.size, 1), 8), np.float32)
    lib().oracle_cell_phase_act_f32(_p(f), _p(l), _p(c) if c.size else None, c.size, X, Y, Z, ctypes.byref(params),
                                    _p(ev), _p(act))
    return f, c, ev[: c.size], act[: c.size]


def hgt(cells: np.ndarray, donors, recipients, seed: int, tick: int) -> np.ndarray:
    """transfer_reaction (crates/marl-cell/src/hgt.rs:7-27) for each (donor, recipient) pair in order."""
    c = np.ascontiguousarray(cells, CELL_DTYPE).copy()
    d = np.ascontiguousarray(donors, np.uint32)
    r = np.ascontiguousarray(recipients, np.uint32)
    lib().oracle_hgt(_p(c), c.size, _p(d) if d.size else None, _p(r) if r.size else None, d.size, seed, tick)
    return c


def cell_phase_f64(field: np.ndarray, light_arr: np.ndarray, cells: np.ndarray, dims, params: SimParams):
    """FP64 cell loop: returns (field f64, internal f64 [n,16])."""
    X, Y, Z = dims
    f = np.ascontiguousarray(field, np.float64).copy()
    l = np.ascontiguousarray(light_arr, np.float64)
    c = np.ascontiguousarray(cells, CELL_DTYPE).copy()
    internal = np.zeros((max(c.size, 1), 16), np.float64)
    lib().oracle_cell_phase_f64(_p(f), _p(l), _p(c) if c.size else None, c.size, X, Y, Z, ctypes.byref(params),
                                _p(internal))
    return f, internal[: c.size]


def make_starter(kind: int, pos, lineage: int) -> np.ndarray:
    out = np.zeros(1, CELL_DTYPE)
    p = np.ascontiguousarray(pos, np.uint16)
    lib().oracle_make_starter(kind, _p(p), lineage, _p(out))
    return out[0]


def rng_seed(seed: int) -> np.ndarray:
    s = np.zeros(4, np.uint64)
    lib().oracle_rng_seed(seed, _p(s))
    return s


def rng_next_u64(state: np.ndarray) -> int:
    return int(lib().oracle_rng_next_u64(_p(state)))


def mutate(ruleset: np.ndarray, rng_state: np.ndarray, params: SimParams) -> np.ndarray:
    r = np.array(ruleset, RULESET_DTYPE).reshape(1).copy()
    lib().oracle_mutate(_p(r), _p(rng_state), ctypes.byref(params))
    return r[0]


def fate_stream(seed: int, tick: int, parent: int, count: int, stddev: float = 1.0):
    """Device-fate stream keyed by (seed, tick, parent): `count` u64 draws and
    `count` normals(stddev) of a fresh stream with the same key."""
    u = np.zeros(max(count, 1), np.uint64)
    z = np.zeros(max(count, 1), np.float32)
    lib().oracle_fate_stream(seed, tick, parent, count, stddev, _p(u), _p(z))
    return u[:count], z[:count]


def fate_log(x: np.ndarray) -> np.ndarray:
    """The device-fate streams' logarithm of x in (0, 1)."""
    xs = np.ascontiguousarray(x, np.float64)
    out = np.zeros(max(xs.size, 1), np.float64)
    lib().oracle_fate_log(_p(xs), xs.size, _p(out))
    return out[:xs.size]


class World:
    """Stateful restatement of marl_sim::run's state (field, light, cells, cell_map, rng)."""

    def __init__(self, dims, params: SimParams | None = None, seed: int = 42, seed_count: int | None = 30):
        self.dims = tuple(int(d) for d in dims)
        self.params = (params or default_params()).copy()
        X, Y, Z = self.dims
        L = lib()
        if seed_count is None:
            self.h = L.oracle_world_create_empty(X, Y, Z, ctypes.byref(self.params), seed)
        else:
            self.h = L.oracle_world_create(X, Y, Z, ctypes.byref(self.params), seed, seed_count)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_world_destroy(self.h)
            self.h = None

    @property
    def voxels(self) -> int:
        X, Y, Z = self.dims
        return X * Y * Z

    def field(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X, 12), np.float32)
        lib().oracle_world_get_field(self.h, _p(out))
        return out

    def set_field(self, f: np.ndarray) -> None:
        lib().oracle_world_set_field(self.h, _p(np.ascontiguousarray(f, np.float32)))

    def light(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X), np.float32)
        lib().oracle_world_get_light(self.h, _p(out))
        return out

    def set_light(self, l: np.ndarray) -> None:
        lib().oracle_world_set_light(self.h, _p(np.ascontiguousarray(l, np.float32)))

    def cells(self) -> np.ndarray:
        n = lib().oracle_world_cell_count(self.h)
        out = np.zeros(max(n, 1), CELL_DTYPE)
        lib().oracle_world_get_cells(self.h, _p(out), out.size)
        return out[:n]

    def set_cells(self, c: np.ndarray) -> None:
        arr = np.ascontiguousarray(c, CELL_DTYPE)
        lib().oracle_world_set_cells(self.h, _p(arr) if arr.size else None, arr.size)

    def occupancy(self) -> np.ndarray:
        X, Y, Z = self.dims
        out = np.empty((Z, Y, X), np.uint8)
        lib().oracle_world_get_occupancy(self.h, _p(out))
        return out

    def rng_state(self) -> np.ndarray:
        s = np.zeros(4, np.uint64)
        lib().oracle_world_get_rng(self.h, _p(s))
        return s

    def sources(self):
        lib().oracle_world_sources(self.h)

    def diffuse(self, substeps: int | None = None):
        lib().oracle_world_diffuse(self.h, self.params.diffusion_substeps if substeps is None else substeps)

    def update_light(self):
        lib().oracle_world_light(self.h)

    def cell_phase(self) -> np.ndarray:
        n = lib().oracle_world_cell_count(self.h)
        ev = np.zeros(max(n, 1), np.int32)
        lib().oracle_world_cell_phase(self.h, _p(ev))
        return ev[:n]

    def fate(self, events: np.ndarray) -> None:
        ev = np.ascontiguousarray(events, np.int32)
        lib().oracle_world_fate(self.h, _p(ev) if ev.size else None, ev.size)

    def tick(self, n: int = 1) -> None:
        lib().oracle_world_tick(self.h, n)

    def set_fate_mode(self, mode: int) -> None:
        """0: fate draws from the run's one sequential stream (host engine);
        1: one stream per division keyed by (seed, tick, parent) (device fate)."""
        lib().oracle_world_set_fate_mode(self.h, mode)

    def set_tick(self, tick: int) -> None:
        lib().oracle_world_set_tick(self.h, tick)

    def stats(self) -> dict:
        out = np.zeros(6, np.uint64)
        lib().oracle_world_stats(self.h, _p(out))
        keys = ("tick", "population", "total_divisions", "total_deaths", "tick_divisions", "tick_deaths")
        return {k: int(v) for k, v in zip(keys, out)}
