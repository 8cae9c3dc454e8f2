"""The cell loop's bounded dependency wait, driven to expiry on purpose.

A cell of the dependency-ordered loop starts only after the cells it depends
on have published their completion flag.  Every such wait is bounded: after
`wait_limit` polls the cell gives up, is left un-updated, and the phase
reports MARL_ERR_TIMEOUT instead of hanging.  Here one cell is made to wait
for a slot past the population, whose flag no cell sets in that phase
(marl_ctx_test_hold_dependency), with a short limit.  This is a software flag
wait that ends on its own: no fault, trap or hang.  The context must stay
usable: the next phase is bit-identical to the oracle's sequential loop.
"""
import numpy as np
import pytest

from helpers import random_cells, random_field

pytestmark = pytest.mark.gpu


def two_isolated_cells(dims):
    X, Y, Z = dims
    cells = random_cells(dims, 2, np.random.default_rng(5))
    cells["pos"][0] = (X // 4, Y // 2, Z // 2)      # all six faces empty, in the grid
    cells["pos"][1] = (3 * X // 4, Y // 2, Z // 2)  # far from cell 0: no shared neighbour voxel
    return cells


def test_dependency_wait_times_out_and_context_recovers(marl, oracle_mod):
    dims = (16, 12, 10)
    X, Y, Z = dims
    rng = np.random.default_rng(11)
    f = random_field(dims, rng)
    light = rng.random((Z, Y, X), dtype=np.float32)
    cells = two_isolated_cells(dims)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=4)
    ctx.upload_field(f)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    ctx.set_wait_limit(2000)  # polls of >= 64 ns: the wait gives up within milliseconds

    ctx.test_hold_dependency(cell=1, face=0, slot=3)  # slot 3 >= population 2: never completed
    with pytest.raises(marl.MarlError) as e:
        ctx.cell_phase()
    assert e.value.status_name == "TIMEOUT"

    # Cell 0 was not held: it was updated exactly as the oracle updates it.
    # Cell 1 gave up before touching anything: its state is unchanged.
    got = ctx.download_cells()
    cf, cc, _ = oracle_mod.cell_phase(f, light, cells[:1], dims, p)
    np.testing.assert_array_equal(got["internal"][0], cc["internal"][0])
    np.testing.assert_array_equal(got["internal"][1], cells["internal"][1])
    assert got["age"][1] == cells["age"][1]

    # The context still works: the hold was for one phase only.  From a fresh
    # upload of the same state the next phase matches the oracle bit for bit.
    ctx.set_wait_limit(0)
    ctx.upload_field(f)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    ev = ctx.cell_phase()
    cf, cc, ce = oracle_mod.cell_phase(f, light, cells, dims, p)
    np.testing.assert_array_equal(ctx.download_field(), cf)
    np.testing.assert_array_equal(ctx.download_cells()["internal"], cc["internal"])
    np.testing.assert_array_equal(ev.astype(np.int32), ce)
    ctx.close()


def test_hold_rejects_bad_arguments(marl):
    dims = (16, 12, 10)
    ctx = marl.Context(dims, marl.default_params(), cell_capacity=4)
    ctx.upload_cells(two_isolated_cells(dims))
    for cell, face, slot in ((2, 0, 3), (0, 6, 3), (0, 0, 1), (0, 0, 4)):  # cell >= n, face >= 6, slot < n, slot >= cap
        with pytest.raises(marl.MarlError) as e:
            ctx.test_hold_dependency(cell, face, slot)
        assert e.value.status_name == "INVALID_INPUT"
    ctx.close()


def test_hold_through_occupied_face_is_reported(marl):
    """A face that is not an empty in-grid voxel has no dependency to hold."""
    dims = (16, 12, 10)
    X, Y, Z = dims
    cells = random_cells(dims, 2, np.random.default_rng(6))
    cells["pos"][0] = (0, Y // 2, Z // 2)          # face 1 (-x) lies outside the grid
    cells["pos"][1] = (X // 2, Y // 2, Z // 2)
    ctx = marl.Context(dims, marl.default_params(), cell_capacity=4)
    ctx.upload_field(random_field(dims, np.random.default_rng(1)))
    ctx.upload_cells(cells)
    ctx.test_hold_dependency(cell=0, face=1, slot=3)
    with pytest.raises(marl.MarlError) as e:
        ctx.cell_phase()
    assert e.value.status_name == "INVALID_INPUT"
    ctx.close()


def lattice_cells(dims, spacing):
    """Cells on a lattice: no two share a neighbour voxel, all faces empty."""
    X, Y, Z = dims
    g = np.stack(np.meshgrid(np.arange(1, X - 1, spacing), np.arange(1, Y - 1, spacing),
                             np.arange(1, Z - 1, spacing), indexing="ij"), -1).reshape(-1, 3)
    cells = random_cells(dims, len(g), np.random.default_rng(8))
    cells["pos"] = g.astype(np.uint16)
    return cells


def test_dependency_wait_times_out_under_lane_refill(marl, oracle_mod):
    """The same bounded wait with more cells than lanes (one cell per warp
    ticket), where a waiting lane stays put while the warp's other lanes take
    new cells: the held cell gives up, every other cell is updated."""
    dims = (62, 62, 14)
    rng = np.random.default_rng(12)
    f = random_field(dims, rng)
    X, Y, Z = dims
    light = rng.random((Z, Y, X), dtype=np.float32)
    cells = lattice_cells(dims, 3)
    n = len(cells)
    assert n > 1184  # more than the lanes of a full grid at one cell per warp
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=n + 2)
    marl._check(marl.load().marl_ctx_set_cell_lanes(ctx.h, 1), "marl_ctx_set_cell_lanes")
    ctx.upload_field(f)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    ctx.set_wait_limit(2000)
    held = n // 3
    ctx.test_hold_dependency(cell=held, face=0, slot=n + 1)
    with pytest.raises(marl.MarlError) as e:
        ctx.cell_phase()
    assert e.value.status_name == "TIMEOUT"
    got = ctx.download_cells()
    others = np.ones(n, bool)
    others[held] = False
    _, cc, _ = oracle_mod.cell_phase(f, light, cells[others], dims, p)
    np.testing.assert_array_equal(got["internal"][others], cc["internal"])
    np.testing.assert_array_equal(got["internal"][held], cells["internal"][held])
    ctx.close()
