"""Binary snapshot output (marl_write_dump, marl_ctx_viewer_cells) in the
reference's dump format: run_meta.json plus tick_<T>.field.bin and
tick_<T>.cells.bin (crates/marl-output/src/binary_dump.rs:109-120,
crates/marl-format/src/lib.rs:130-218, 351-364).

CPU: the host writer's files read back exactly, and the reference's own
checker (scripts/check_binary_dump.py, run from the reference checkout when
it is present on this machine) accepts them.  GPU: the device-packed viewer
records of an engine equal the records packed on the host from its cells.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

# The reference's dump checker (scripts/check_binary_dump.py of a reference
# checkout), named by an environment variable; its test skips when unset.
REF_CHECKER = os.environ.get("MARL_REF_DUMP_CHECKER", "")


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


@pytest.mark.skipif(not REF_CHECKER, reason="MARL_REF_DUMP_CHECKER (the reference's check_binary_dump.py) not set")
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
