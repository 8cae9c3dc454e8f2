"""GPU parity of the cell loop (gather -> tick -> scatter in the reference's
sequential order), the change list and the edit list, against the CPU oracle.

With the same light field, the cell phase is bit-identical to the oracle's
sequential loop (crates/marl-sim/src/lib.rs:206-217) — field, internals,
fate state and events — for sparse, clustered and dense populations.
"""
import numpy as np
import pytest

from helpers import clustered_positions, random_cells, random_field

pytestmark = pytest.mark.gpu


def run_cell_phase(marl, oracle_mod, dims, cells, seed, lanes=32):
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    f = random_field(dims, rng)
    light = rng.random((Z, Y, X), dtype=np.float32)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=max(len(cells), 1))
    marl._check(marl.load().marl_ctx_set_cell_lanes(ctx.h, lanes), "marl_ctx_set_cell_lanes")
    ctx.upload_field(f)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    ev = ctx.cell_phase()
    gf, gc = ctx.download_field(), ctx.download_cells()
    cf, cc, ce = oracle_mod.cell_phase(f, light, cells, dims, p)
    return (gf, gc, ev), (cf, cc, ce)


def assert_same(gpu, cpu):
    (gf, gc, ge), (cf, cc, ce) = gpu, cpu
    np.testing.assert_array_equal(gf, cf)
    np.testing.assert_array_equal(gc["internal"], cc["internal"])
    np.testing.assert_array_equal(gc["prep_remaining"], cc["prep_remaining"])
    np.testing.assert_array_equal(gc["quiescent"], cc["quiescent"])
    np.testing.assert_array_equal(gc["age"], cc["age"])
    np.testing.assert_array_equal(ge.astype(np.int32), ce)
    # cold data travels unchanged
    np.testing.assert_array_equal(gc["lineage_id"], cc["lineage_id"])
    assert gc["ruleset"].tobytes() == cc["ruleset"].tobytes()


@pytest.mark.parametrize("n", [1, 7, 300])
def test_cell_phase_sparse(marl, oracle_mod, n):
    dims = (32, 24, 16)
    cells = random_cells(dims, n, np.random.default_rng(n))
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, n)
    assert_same(gpu, cpu)


@pytest.mark.parametrize("lanes", [1, 5, 8, 16])
def test_cell_phase_cells_per_warp(marl, oracle_mod, lanes):
    """Fewer cells per warp ticket (marl_ctx_set_cell_lanes) leave the result
    unchanged: dense blobs, long dependency chains."""
    dims = (24, 20, 16)
    rng = np.random.default_rng(31)
    pos = clustered_positions(dims, 0.5, rng, 1, 3)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, 78, lanes=lanes)
    assert_same(gpu, cpu)


@pytest.mark.parametrize("lanes,frac", [(1, 0.3), (1, 0.7), (4, 0.5), (32, 0.5)])
def test_cell_phase_lane_refill(marl, oracle_mod, lanes, frac):
    """More cells than the grid has lanes: warps hand finished lanes the next
    cells while other lanes wait on dependencies (lane refill).  With one or
    four cells per warp this happens at a few thousand cells; with 32 the
    grid covers every cell of this population at once (warp tickets)."""
    dims = (40, 32, 24)
    rng = np.random.default_rng(int(frac * 10) + lanes)
    pos = clustered_positions(dims, frac, rng, 1, 3)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, 90 + lanes, lanes=lanes)
    assert_same(gpu, cpu)


def test_cell_lanes_rejects_out_of_range(marl):
    ctx = marl.Context((8, 8, 8), marl.default_params(), cell_capacity=8)
    lib = marl.load()
    assert lib.marl_ctx_set_cell_lanes(ctx.h, 0) != 0
    assert lib.marl_ctx_set_cell_lanes(ctx.h, 33) != 0
    assert lib.marl_ctx_set_cell_lanes(ctx.h, 32) == 0


@pytest.mark.parametrize("frac", [0.05, 0.3, 0.7])
def test_cell_phase_clustered(marl, oracle_mod, frac):
    """Clustered blobs: many cells share empty voxels, long dependency chains."""
    dims = (24, 20, 16)
    rng = np.random.default_rng(int(frac * 100))
    pos = clustered_positions(dims, frac, rng, 1, 3)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, 77)
    assert_same(gpu, cpu)


def test_cell_phase_chain_order(marl, oracle_mod):
    """Cells in a line with one-voxel gaps: every cell depends on its predecessor."""
    dims = (64, 1, 1)
    xs = np.arange(0, 64, 2)
    rng = np.random.default_rng(1)
    order = rng.permutation(len(xs))  # scrambled Vec order
    pos = np.stack([xs[order], np.zeros_like(xs), np.zeros_like(xs)], 1)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, 5)
    assert_same(gpu, cpu)


def test_cell_phase_many_cells(marl, oracle_mod):
    """Cell-kinetics microbenchmark shape at reduced size: 11.9% random occupancy."""
    dims = (64, 64, 48)
    n = int(0.119 * 64 * 64 * 48)
    cells = random_cells(dims, n, np.random.default_rng(2024))
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, 2024)
    assert_same(gpu, cpu)


@pytest.mark.parametrize("seed", [31, 32, 33])
def test_cell_phase_edge_rulesets(marl, oracle_mod, seed):
    """Rulesets that take every branch of the transport, reaction and effector
    order: transporters and effectors sharing a species, invalid indices
    (species out of range skip the slot), reactions whose cofactor is their
    substrate or product, substrate equal to product, v_max exactly at the
    threshold (runs, not counted active), cofactor indices out of range, and
    cells dense enough to chain."""
    dims = (20, 16, 12)
    rng = np.random.default_rng(seed)
    pos = clustered_positions(dims, 0.3, rng, 1, 3)
    n = len(pos)
    cells = random_cells(dims, n, rng, positions=pos)
    rs = cells["ruleset"]
    tp, rx, ef = rs["transport"], rs["reactions"], rs["effectors"]
    tp["int_species"] = rng.integers(0, 4, (n, 8))          # few species: many transporters share one
    tp["ext_species"] = rng.integers(0, 3, (n, 8))
    bad = rng.random((n, 8)) < 0.15
    tp["ext_species"][bad] = rng.integers(12, 256, bad.sum())
    bad = rng.random((n, 8)) < 0.15
    tp["int_species"][bad] = rng.integers(16, 256, bad.sum())
    ef["int_species"] = rng.integers(0, 4, (n, 8))
    ef["ext_species"] = rng.integers(0, 3, (n, 8))
    ef["threshold"] = (0.3 * rng.random((n, 8))).astype(np.float32)
    bad = rng.random((n, 8)) < 0.15
    ef["int_species"][bad] = rng.integers(16, 256, bad.sum())
    bad = rng.random((n, 8)) < 0.15
    ef["ext_species"][bad] = rng.integers(12, 256, bad.sum())
    rx["substrate"] = rng.integers(0, 5, (n, 16))
    rx["product"] = rng.integers(0, 5, (n, 16))
    rx["catalyst"] = rng.integers(0, 6, (n, 16))
    cof = rng.integers(0, 5, (n, 16))
    pick = rng.random((n, 16))
    cof[pick < 0.2] = rx["substrate"][pick < 0.2]                       # cofactor = substrate
    cof[(pick >= 0.2) & (pick < 0.4)] = rx["product"][(pick >= 0.2) & (pick < 0.4)]  # cofactor = product
    cof[pick > 0.8] = 0xFF
    cof[(pick > 0.75) & (pick <= 0.8)] = rng.integers(16, 255, ((pick > 0.75) & (pick <= 0.8)).sum())
    rx["cofactor"] = cof
    thr = marl.default_params().active_reaction_threshold
    vm = rx["v_max"]
    vm[rng.random((n, 16)) < 0.1] = np.float32(thr)
    vm[rng.random((n, 16)) < 0.1] = np.float32(-thr)
    vm[rng.random((n, 16)) < 0.1] = 0.0
    bad = rng.random((n, 16)) < 0.05
    rx["catalyst"][bad] = rng.integers(16, 256, bad.sum())
    gpu, cpu = run_cell_phase(marl, oracle_mod, dims, cells, seed)
    assert_same(gpu, cpu)


def test_cell_phase_repeated(marl, oracle_mod):
    """Several phases in a row on the same table (schedule reused, epochs advance)."""
    dims = (20, 20, 12)
    rng = np.random.default_rng(3)
    pos = clustered_positions(dims, 0.25, rng)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    f = random_field(dims, rng)
    light = rng.random((12, 20, 20), dtype=np.float32)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=len(cells))
    ctx.upload_field(f)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    cf, cc = f, cells
    for _ in range(5):
        ev = ctx.cell_phase()
        cf, cc, ce = oracle_mod.cell_phase(cf, light, cc, dims, p)
        np.testing.assert_array_equal(ev.astype(np.int32), ce)
    np.testing.assert_array_equal(ctx.download_field(), cf)
    np.testing.assert_array_equal(ctx.download_cells()["internal"], cc["internal"])


def test_tick_change_list(marl, oracle_mod):
    """marl_tick = sources + diffusion + light + cell loop, then the ordered change list."""
    dims = (40, 36, 24)
    rng = np.random.default_rng(10)
    pos = clustered_positions(dims, 0.1, rng)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    cells["internal"][:, 0] = rng.random(len(cells)).astype(np.float32) * 2  # some die, some divide
    cells["prep_remaining"] = np.where(rng.random(len(cells)) < 0.3, 1, 0)
    f = random_field(dims, rng)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=len(cells))
    ctx.upload_field(f)
    ctx.upload_cells(cells)
    changes = ctx.tick()
    w = oracle_mod.World(dims, p, seed=0, seed_count=None)
    w.set_field(f)
    w.set_cells(cells)
    w.sources()
    w.diffuse()
    w.update_light()
    np.testing.assert_allclose(ctx.download_light(), w.light(), rtol=1e-5, atol=1e-6)
    ctx.upload_light(w.light())  # same light for a bit-exact cell-phase check below
    ev = w.cell_phase()
    want = [(i, e) for i, e in enumerate(ev) if e in (1, 2)]
    assert [(int(c["cell"]), int(c["event"])) for c in changes] == want
    assert len(want) > 0
    wc = w.cells()
    for c in changes:
        if c["event"] == 1:
            np.testing.assert_allclose(c["internal"], wc[c["cell"]]["internal"], rtol=1e-5, atol=1e-6)
            assert c["quiescent"] == wc[c["cell"]]["quiescent"]


def test_apply_edits_matches_swap_remove(marl, oracle_mod):
    dims = (16, 16, 16)
    rng = np.random.default_rng(6)
    cells = random_cells(dims, 10, rng)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=32)
    ctx.upload_cells(cells)
    births = random_cells(dims, 3, rng, positions=np.array([[0, 0, 0], [15, 15, 15], [7, 0, 3]]))
    occupied = {tuple(c["pos"]) for c in cells}
    births = births[[tuple(b["pos"]) not in occupied for b in births]]
    # deaths 2, 5, 9 of 10: swap_remove(9) -> pop; swap_remove(5) <- 8; swap_remove(2) <- 7
    ctx.apply_edits(halve=[0, 4], deaths=[2, 5, 9], moves=[(2, 7), (5, 8)], n_after_deaths=7, births=births)
    out = ctx.download_cells()
    expect = [cells[i].copy() for i in (0, 1, 7, 3, 4, 8, 6)] + list(births)
    expect[0]["internal"] = expect[0]["internal"] * np.float32(0.5)
    expect[4]["internal"] = expect[4]["internal"] * np.float32(0.5)
    assert len(out) == len(expect)
    for a, b in zip(out, expect):
        assert tuple(a["pos"]) == tuple(b["pos"])
        np.testing.assert_array_equal(a["internal"], b["internal"])
        assert a["ruleset"].tobytes() == b["ruleset"].tobytes() and a["lineage_id"] == b["lineage_id"]
    occ = ctx.download_occupancy()
    want = np.zeros((16, 16, 16), np.uint8)
    for c in expect:
        want[c["pos"][2], c["pos"][1], c["pos"][0]] = 1
    np.testing.assert_array_equal(occ, want)
