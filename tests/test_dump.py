"""Binary snapshot output (marl_write_dump, marl_ctx_viewer_cells) in the
reference's dump format: run_meta.json plus tick_<T>.field.bin and
tick_<T>.cells.bin (crates/marl-output/src/binary_dump.rs:109-120,
crates/marl-format/src/lib.rs:130-218, 351-364).

Ruleset sidecars (binary_dump.rs:121-350): tick_<T>.ruleset_layers.bin
(per-layer f64-summed averages of the 110 float ruleset fields) and the
deduplicated "MRSF" tick_<T>.rulesets.bin.

CPU: the host writers' files read back exactly and match a numpy restatement
of the reference's layer averaging and first-occurrence deduplication; the
reference's own checkers (scripts/check_binary_dump.py, inspect_rulesets.py,
run from a reference checkout named by MARL_REF_SCRIPTS) accept them.  GPU:
the device-packed viewer records and the device-written ruleset files equal
the ones written on the host from the same cells, byte for byte.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

# The reference's scripts directory (check_binary_dump.py, inspect_rulesets.py
# of a reference checkout), named by an environment variable; the tests that
# run them skip when it is unset.
REF_SCRIPTS = os.environ.get("MARL_REF_SCRIPTS", "")
REF_CHECKER = os.path.join(REF_SCRIPTS, "check_binary_dump.py") if REF_SCRIPTS else ""
REF_INSPECTOR = os.path.join(REF_SCRIPTS, "inspect_rulesets.py") if REF_SCRIPTS else ""


def host_viewer(marl, cells):
    v = np.zeros(len(cells), marl.VIEWER_CELL_DTYPE)
    v["pos"] = cells["pos"].astype(np.float32)
    v["lineage_id"] = cells["lineage_id"]
    v["starter_type"] = cells["starter_type"]
    v["energy"] = cells["internal"][:, 0]
    return v


def write_sample_dump(marl, path):
    dims = (24, 20, 12)
    X, Y, Z = dims
    rng = np.random.default_rng(1)
    field = rng.random((Z, Y, X, 12), dtype=np.float32)
    v = np.zeros(57, marl.VIEWER_CELL_DTYPE)
    v["pos"] = rng.integers(0, 12, (57, 3)).astype(np.float32)
    v["lineage_id"] = rng.integers(0, 2**63, 57, dtype=np.int64).astype(np.uint64)
    v["starter_type"] = rng.integers(0, 3, 57)
    v["energy"] = rng.random(57, dtype=np.float32)
    marl.write_dump(str(path), 42, dims, field, v)
    return dims, field, v


def test_write_dump_round_trip(marl, tmp_path):
    dims, field, v = write_sample_dump(marl, tmp_path)
    meta = json.loads((tmp_path / "run_meta.json").read_text())
    assert (meta["grid_x"], meta["grid_y"], meta["grid_z"]) == dims
    assert meta["field_byte_len"] == field.nbytes and meta["cell_record_stride"] == 25
    assert meta["field_layout"] == "z_y_x_species" and meta["endianness"] == "little"
    assert (tmp_path / "tick_42.field.bin").read_bytes() == field.tobytes()
    assert (tmp_path / "tick_42.cells.bin").read_bytes() == v.tobytes()
    assert not any(p.name.endswith(".tmp") for p in tmp_path.iterdir())


@pytest.mark.skipif(not REF_SCRIPTS, reason="MARL_REF_SCRIPTS (the reference's scripts directory) not set")
def test_reference_checker_accepts_dump(marl, tmp_path):
    write_sample_dump(marl, tmp_path)
    out = subprocess.run([sys.executable, REF_CHECKER, str(tmp_path), "42"], capture_output=True, text=True,
                         timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "cell_count=57" in out.stdout


def test_write_dump_errors(marl, tmp_path):
    with pytest.raises(marl.MarlError):
        marl.write_dump(str(tmp_path / "missing" / "dir"), 1, (8, 8, 8), np.zeros((8, 8, 8, 12), np.float32), None)
    with pytest.raises(marl.MarlError):
        marl.write_dump(str(tmp_path), 1, (0, 8, 8), np.zeros(0, np.float32), None)


@pytest.mark.gpu
def test_device_viewer_records_match_host(marl, tmp_path):
    dims = (48, 40, 32)
    e = marl.Engine(dims, marl.default_params(), rng_seed=9, seed_count=30, cell_capacity=1 << 14)
    e.step(40)
    cells = e.cells()
    got = marl.viewer_cells(e.lib.marl_engine_ctx(e.h), len(cells))
    assert got.tobytes() == host_viewer(marl, cells).tobytes()
    marl.write_dump(str(tmp_path), 40, dims, e.field(), got)
    assert (tmp_path / "tick_40.cells.bin").stat().st_size == 25 * len(cells)
    assert (tmp_path / "tick_40.field.bin").read_bytes() == e.field().tobytes()


def ruleset_cells(marl, dims, n, seed):
    from helpers import random_cells

    rng = np.random.default_rng(seed)
    cells = random_cells(dims, n, rng)
    # duplicated rulesets, so the dictionary is smaller than the cell count
    for j in range(1, n, 3):
        cells["ruleset"][j] = cells["ruleset"][j - 1]
    return cells


def numpy_layers(cells, Z):
    """binary_dump.rs:121-186: per layer, f64 sums in cell order, (sum / count) as f32."""
    rs = cells["ruleset"]
    vals = np.concatenate([
        np.stack([rs["receptors"]["k_half"], rs["receptors"]["n_hill"], rs["receptors"]["gain"]], 2).reshape(-1, 24),
        np.stack([rs["transport"]["uptake_rate"], rs["transport"]["secrete_rate"]], 2).reshape(-1, 16),
        np.stack([rs["reactions"]["k_m"], rs["reactions"]["v_max"], rs["reactions"]["k_cat"]], 2).reshape(-1, 48),
        np.stack([rs["effectors"]["threshold"], rs["effectors"]["rate"]], 2).reshape(-1, 16),
        np.stack([rs["fate"][k] for k in ("division_energy", "death_energy", "quiescence_energy",
                                          "division_prep_ticks")], 1),
        rs["hgt_propensity"][:, None], rs["mutation_rate"][:, None]], 1).astype(np.float64)
    out = bytearray()
    z = cells["pos"][:, 2]
    for layer in range(Z):
        sel = vals[z == layer]
        acc = np.zeros(110, np.float64)
        for row in sel:  # sequential f64 sums in cell order
            acc = acc + row
        cnt = len(sel)
        avg = (acc / cnt).astype(np.float32) if cnt else np.zeros(110, np.float32)
        out += np.uint16(layer).tobytes() + b"\0\0" + np.uint32(cnt).tobytes() + avg.tobytes()
    return bytes(out)


def numpy_full(marl, cells):
    """binary_dump.rs:272-350: MRSF v1 with the dictionary in first-occurrence order."""
    dict_ids, entries, refs = {}, [], bytearray()
    for c in cells:
        key = marl.pack_ruleset(c["ruleset"])
        if key not in dict_ids:
            dict_ids[key] = len(entries)
            entries.append(key)
        refs += np.asarray(c["pos"], np.uint16).tobytes() + np.uint32(dict_ids[key]).tobytes()
    head = b"MRSF" + np.array([1, 0, len(entries), len(cells), 536], np.uint32).tobytes()
    return head + b"".join(entries) + bytes(refs)


def test_host_ruleset_dumps_match_restatement(marl, tmp_path):
    dims = (20, 16, 12)
    cells = ruleset_cells(marl, dims, 301, 4)
    marl.write_ruleset_dumps(str(tmp_path), 7, dims, cells, marl.RULESETS_BOTH)
    assert (tmp_path / "tick_7.ruleset_layers.bin").read_bytes() == numpy_layers(cells, dims[2])
    full = (tmp_path / "tick_7.rulesets.bin").read_bytes()
    assert full == numpy_full(marl, cells)
    assert int.from_bytes(full[12:16], "little") == 201  # 301 cells, every third a repeat of its predecessor
    meta = json.loads((tmp_path / "run_meta.json").read_text())
    assert meta["ruleset_output_mode"] == "both" and meta["ruleset_layer_record_stride"] == 448
    assert meta["ruleset_full_ruleset_byte_size"] == 536 and meta["ruleset_full_magic_ascii"] == "MRSF"
    marl.write_ruleset_dumps(str(tmp_path), 8, dims, cells[:0], marl.RULESETS_BOTH)  # no cells
    assert (tmp_path / "tick_8.rulesets.bin").read_bytes() == numpy_full(marl, cells[:0])
    with pytest.raises(marl.MarlError):
        marl.write_ruleset_dumps(str(tmp_path), 9, dims, cells, 0)


@pytest.mark.skipif(not REF_SCRIPTS, reason="MARL_REF_SCRIPTS (the reference's scripts directory) not set")
def test_reference_checkers_accept_ruleset_dumps(marl, tmp_path):
    dims, field, v = write_sample_dump(marl, tmp_path)
    cells = ruleset_cells(marl, dims, 57, 5)
    marl.write_ruleset_dumps(str(tmp_path), 42, dims, cells, marl.RULESETS_BOTH)
    out = subprocess.run([sys.executable, REF_CHECKER, str(tmp_path), "42", "--require-rulesets",
                          "--require-full-rulesets"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "rulesets: OK" in out.stdout
    out = subprocess.run([sys.executable, REF_INSPECTOR, str(tmp_path / "tick_42.rulesets.bin")],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2, 3])
def test_device_ruleset_dumps_match_host(marl, tmp_path, mode):
    dims = (48, 40, 32)
    e = marl.Engine(dims, marl.default_params(), rng_seed=11, seed_count=30, cell_capacity=1 << 14)
    e.step(60)
    cells = e.cells()
    dev, host = tmp_path / "dev", tmp_path / "host"
    dev.mkdir()
    host.mkdir()
    marl.ctx_write_ruleset_dumps(e.lib.marl_engine_ctx(e.h), str(dev), 60, mode)
    marl.write_ruleset_dumps(str(host), 60, dims, cells, mode)
    names = sorted(p.name for p in host.iterdir())
    assert names == sorted(p.name for p in dev.iterdir())
    for name in names:
        assert (dev / name).read_bytes() == (host / name).read_bytes(), name
    if mode & 1:
        assert (host / "tick_60.ruleset_layers.bin").read_bytes() == numpy_layers(cells, dims[2])
