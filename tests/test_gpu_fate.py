"""Device fate processing against the oracle's stream fate mode, bit for bit:
the stream specification itself (u64 draws, normals, logarithm), single fate
steps driven by random events (collisions, blocked divisions, mass deaths,
empty steps, full tables), consecutive steps, and whole engine runs with
device fate, including switches between host and device fate."""
import numpy as np
import pytest

from helpers import random_cells

pytestmark = pytest.mark.gpu

DIV, DEATH, QUIESCENT = 1, 2, 3


def mutable_cells(dims, n, rng):
    """Cells whose rulesets exercise every branch of Ruleset::mutate."""
    cells = random_cells(dims, n, rng)
    rs = cells["ruleset"]
    rs["mutation_rate"] = rng.choice([0.0, 0.05, 0.5, 1.0], size=n).astype(np.float32)
    rx = rs["reactions"]
    rx["v_max"][rng.random(rx["v_max"].shape) < 0.4] = 0.0  # inactive reactions: donors vary
    return cells


def mutation_params(marl):
    p = marl.default_params()
    p.structural_mutation_rate_mult = 1.0
    p.meta_mutation_rate = 0.5
    return p


def device_step(marl, dims, p, cells, events, seed, tick, cap=None):
    ctx = marl.Context(dims, p, cell_capacity=cap or max(4 * cells.size, 64))
    ctx.upload_cells(cells)
    ctx.fate_init(seed, tick)
    ctx.set_events(events)
    ctx.fate()
    st = ctx.fate_stats()
    return ctx, ctx.download_cells(), ctx.download_occupancy(), st


def oracle_step(oracle_mod, dims, p, cells, events, seed, tick):
    w = oracle_mod.World(dims, p, seed=seed, seed_count=None)
    w.set_cells(cells)
    w.set_tick(tick)
    w.set_fate_mode(1)
    w.fate(np.asarray(events, np.int32))
    return w, w.cells(), w.occupancy(), w.stats()


def assert_same_cells(got, want):
    assert got.size == want.size
    for name in ("pos", "lineage_id", "age", "prep_remaining", "quiescent", "starter_type"):
        np.testing.assert_array_equal(got[name], want[name], err_msg=name)
    assert got["internal"].tobytes() == want["internal"].tobytes()
    assert got["ruleset"].tobytes() == want["ruleset"].tobytes()


def test_stream_probe_matches_oracle(marl, oracle_mod):
    for seed, tick, parent in [(0, 0, 0), (42, 7, 1234), (2**64 - 1, 2**40 + 3, 2**32 - 1), (5, 999, 17)]:
        du, dz = marl.fate_stream_probe(seed, tick, parent, 4000, 0.1)
        ou, oz = oracle_mod.fate_stream(seed, tick, parent, 4000, 0.1)
        np.testing.assert_array_equal(du, ou)
        assert dz.tobytes() == oz.tobytes()


def test_stream_ln_matches_oracle(marl, oracle_mod):
    rng = np.random.default_rng(4)
    x = np.concatenate([rng.random(100000), np.ldexp(rng.random(1000) + 0.5, -rng.integers(1, 100, 1000))])
    x = x[(x > 0) & (x < 1)]
    assert marl.fate_stream_ln(x).tobytes() == oracle_mod.fate_log(x).tobytes()


@pytest.mark.parametrize("dims,n,probs,seed,tick", [
    ((16, 16, 16), 1800, (0.4, 0.3, 0.2, 0.1), 7, 0),        # ~44% occupied: collisions, blocked divisions
    ((24, 20, 12), 600, (0.5, 0.3, 0.15, 0.05), 99, 12345),  # sparse
    ((12, 12, 12), 1700, (0.0, 1.0, 0.0, 0.0), 3, 5),        # every cell divides in a nearly full grid
    ((20, 20, 20), 3000, (0.0, 0.0, 1.0, 0.0), 1, 1),        # every cell dies
    ((20, 20, 20), 3000, (0.3, 0.0, 0.7, 0.0), 2, 2),        # mass death: long swap_remove chains
    ((20, 20, 20), 3000, (1.0, 0.0, 0.0, 0.0), 2, 3),        # no events
    ((64, 64, 48), 60000, (0.6, 0.2, 0.15, 0.05), 11, 77),   # several fate blocks
])
def test_fate_step_matches_oracle(marl, oracle_mod, dims, n, probs, seed, tick):
    rng = np.random.default_rng(seed * 1000 + n)
    cells = mutable_cells(dims, n, rng)
    events = rng.choice([0, DIV, DEATH, QUIESCENT], size=n, p=probs).astype(np.uint8)
    p = mutation_params(marl)
    _, gc, gocc, gs = device_step(marl, dims, p, cells, events, seed, tick)
    _, wc, wocc, ws = oracle_step(oracle_mod, dims, p, cells, events, seed, tick)
    assert gs["tick_divisions"] == ws["tick_divisions"]
    assert gs["tick_deaths"] == ws["tick_deaths"] == int((events == DEATH).sum())
    assert gs["population"] == ws["population"] == wc.size
    assert gs["tick"] == tick + 1
    assert_same_cells(gc, wc)
    np.testing.assert_array_equal(gocc, wocc)


@pytest.mark.parametrize("dims,n,dist", [
    ((32, 32, 1), 300, 1),    # one plane: the z faces are off the grid
    ((20, 20, 20), 2000, 3),  # placement three voxels out
    ((7, 5, 3), 60, 2),       # ragged grid, more than half occupied
])
def test_fate_step_other_geometry(marl, oracle_mod, dims, n, dist):
    rng = np.random.default_rng(n + dist)
    cells = mutable_cells(dims, n, rng)
    events = rng.choice([0, DIV, DEATH, QUIESCENT], size=n, p=(0.4, 0.35, 0.2, 0.05)).astype(np.uint8)
    p = mutation_params(marl)
    p.division_neighbor_distance = dist
    _, gc, gocc, gs = device_step(marl, dims, p, cells, events, 17, 3)
    _, wc, wocc, ws = oracle_step(oracle_mod, dims, p, cells, events, 17, 3)
    assert (gs["tick_divisions"], gs["population"]) == (ws["tick_divisions"], ws["population"])
    assert_same_cells(gc, wc)
    np.testing.assert_array_equal(gocc, wocc)


def test_consecutive_fate_steps(marl, oracle_mod):
    dims = (24, 24, 24)
    rng = np.random.default_rng(5)
    cells = mutable_cells(dims, 4000, rng)
    p = mutation_params(marl)
    ctx = marl.Context(dims, p, cell_capacity=1 << 15)
    ctx.upload_cells(cells)
    ctx.fate_init(21, 100, 10, 20)
    w = oracle_mod.World(dims, p, seed=21, seed_count=None)
    w.set_cells(cells)
    w.set_fate_mode(1)
    total_div = total_death = 0
    for step in range(12):
        n = w.cells().size
        ev = rng.choice([0, DIV, DEATH, QUIESCENT], size=n, p=[0.5, 0.25, 0.2, 0.05]).astype(np.uint8)
        ctx.set_events(ev)
        ctx.fate()
        w.set_tick(100 + step)
        w.fate(ev.astype(np.int32))
        ws = w.stats()
        total_div += ws["tick_divisions"]
        total_death += ws["tick_deaths"]
    st = ctx.fate_stats()
    assert (st["tick"], st["total_divisions"], st["total_deaths"]) == (112, 10 + total_div, 20 + total_death)
    assert_same_cells(ctx.download_cells(), w.cells())
    np.testing.assert_array_equal(ctx.download_occupancy(), w.occupancy())


def test_full_table_reports_capacity(marl, oracle_mod):
    dims = (16, 16, 16)
    rng = np.random.default_rng(6)
    cells = mutable_cells(dims, 500, rng)
    events = np.full(500, DIV, np.uint8)
    p = mutation_params(marl)
    ctx = marl.Context(dims, p, cell_capacity=520)
    ctx.upload_cells(cells)
    ctx.set_events(events)
    ctx.fate()
    with pytest.raises(marl.MarlError) as e:
        ctx.fate_stats()
    assert e.value.status_name == "CAPACITY"
    got = ctx.download_cells()
    assert got.size == 520
    _, wc, _, _ = oracle_step(oracle_mod, dims, p, cells, events, 0, 0)
    assert_same_cells(got, wc[:520])  # the first daughters in division order are kept


def test_set_events_validates(marl):
    dims = (8, 8, 8)
    ctx = marl.Context(dims, marl.default_params(), cell_capacity=64)
    ctx.upload_cells(random_cells(dims, 10, np.random.default_rng(1)))
    with pytest.raises(marl.MarlError):
        ctx.set_events(np.zeros(9, np.uint8))
    with pytest.raises(marl.MarlError):
        ctx.set_events(np.full(10, 4, np.uint8))


def compare_device_fate_runs(marl, oracle_mod, dims, ticks, seed=42, switch=None):
    p = marl.default_params()
    eng = marl.Engine(dims, p, rng_seed=seed, seed_count=30, cell_capacity=1 << 16)
    w = oracle_mod.World(dims, p, seed=seed, seed_count=30)
    mode = 1
    eng.set_device_fate(True)
    w.set_fate_mode(1)
    pops = []
    for t in range(ticks):
        if switch and t in switch:
            mode ^= 1
            eng.set_device_fate(mode == 1)
            w.set_fate_mode(mode)
        eng.step(1)
        w.tick(1)
        es, ws = eng.stats(), w.stats()
        pops.append((es["population"], ws["population"]))
        assert (es["tick"], es["population"], es["total_divisions"], es["total_deaths"]) == (
            ws["tick"], ws["population"], ws["total_divisions"], ws["total_deaths"]), (t, es, ws)
        gc, wc = eng.cells(), w.cells()
        np.testing.assert_array_equal(gc["pos"], wc["pos"])
        np.testing.assert_array_equal(gc["lineage_id"], wc["lineage_id"])
        assert gc["ruleset"].tobytes() == wc["ruleset"].tobytes()
        np.testing.assert_allclose(gc["internal"], wc["internal"], rtol=1e-4, atol=1e-5)
    return eng, w, pops


def test_engine_device_fate_matches_oracle(marl, oracle_mod):
    eng, w, pops = compare_device_fate_runs(marl, oracle_mod, (48, 40, 64), 40)
    s = eng.stats()
    assert s["total_divisions"] > 0 and s["total_deaths"] > 0
    np.testing.assert_allclose(eng.field(), w.field(), rtol=1e-4, atol=1e-5)


def test_engine_switches_fate_modes(marl, oracle_mod):
    compare_device_fate_runs(marl, oracle_mod, (48, 40, 64), 36, switch={12, 24})


def test_run_ticks_batches_without_sync(marl, oracle_mod):
    """Many ticks enqueued by one call equal the same ticks one by one."""
    dims = (64, 64, 32)
    p = marl.default_params()
    a = marl.Engine(dims, p, rng_seed=3, seed_count=30, cell_capacity=1 << 16)
    b = marl.Engine(dims, p, rng_seed=3, seed_count=30, cell_capacity=1 << 16)
    a.set_device_fate(True)
    b.set_device_fate(True)
    a.step(30)
    for _ in range(30):
        b.step(1)
    sa, sb = a.stats(), b.stats()
    for k in ("tick", "population", "total_divisions", "total_deaths", "tick_divisions", "tick_deaths"):
        assert sa[k] == sb[k], k
    assert a.cells().tobytes() == b.cells().tobytes()
    np.testing.assert_array_equal(a.field(), b.field())


BATCH_RUNS = [((24, 24, 16), 3), ((32, 24, 24), 7), ((48, 40, 64), 42), ((40, 36, 32), 11)]


def device_fate_engines(marl, p, runs, ticks, switch_at=None):
    out = []
    for dims, seed in runs:
        e = marl.Engine(dims, p, rng_seed=seed, seed_count=30, cell_capacity=1 << 14)
        if switch_at is None:
            e.set_device_fate(True)
            e.step(ticks)
        else:
            e.step(switch_at)
            e.set_device_fate(True)
            e.step(ticks - switch_at)
        out.append(e)
    return out


def assert_batch_run_equal(batch, r, eng):
    bs, es = batch.stats(r), eng.stats()
    for k in ("tick", "population", "total_divisions", "total_deaths", "tick_divisions", "tick_deaths"):
        assert bs[k] == es[k], (r, k, bs[k], es[k])
    assert batch.cells(r).tobytes() == eng.cells().tobytes(), r
    assert np.array_equal(batch.field(r).view(np.uint32), eng.field().view(np.uint32)), r
    assert np.array_equal(batch.light(r).view(np.uint32), eng.light().view(np.uint32)), r


@pytest.mark.parametrize("substeps,graph", [(10, True), (3, True), (10, False)])
def test_batch_device_fate_matches_engines(marl, substeps, graph):
    """Each run of a batch with device fate equals a single engine with device
    fate, bit for bit (odd substep counts alternate the two captured graphs)."""
    p = marl.default_params()
    p.diffusion_substeps = substeps
    b = marl.Batch(BATCH_RUNS, p, cell_capacity=1 << 14)
    b.set_graph(graph)
    b.set_device_fate(True)
    b.step(25)
    b.step(15)
    refs = device_fate_engines(marl, p, BATCH_RUNS, 40)
    events = 0
    for r, eng in enumerate(refs):
        assert_batch_run_equal(b, r, eng)
        events += b.stats(r)["total_divisions"]
    assert events > 0


def test_batch_switches_fate_modes(marl):
    """Host fate for 10 ticks, device fate for 20, host fate again: every run
    equals an engine that switched at the same ticks."""
    p = marl.default_params()
    b = marl.Batch(BATCH_RUNS, p, cell_capacity=1 << 14)
    b.step(10)
    b.set_device_fate(True)
    b.step(20)
    b.set_device_fate(False)
    b.step(10)
    for r, (dims, seed) in enumerate(BATCH_RUNS):
        e = marl.Engine(dims, p, rng_seed=seed, seed_count=30, cell_capacity=1 << 14)
        e.step(10)
        e.set_device_fate(True)
        e.step(20)
        e.set_device_fate(False)
        e.step(10)
        assert_batch_run_equal(b, r, e)


def test_device_fate_under_lane_refill(marl):
    """Device fate with one cell per warp ticket: the grid has 1,184 lanes,
    fewer than the ~3,000 seeded cells, so every tick's cell loop (reading its
    cell count on the device) runs by lane refill.  It must equal the same
    run with 32 cells per ticket (warp tickets) bit for bit."""
    dims = (96, 96, 48)
    p = marl.default_params()
    runs = []
    for lanes in (32, 1):
        e = marl.Engine(dims, p, rng_seed=5, seed_count=1000, cell_capacity=1 << 15)
        marl._check(e.lib.marl_ctx_set_cell_lanes(e.lib.marl_engine_ctx(e.h), lanes), "marl_ctx_set_cell_lanes")
        e.set_device_fate(True)
        e.step(12)
        runs.append(e)
    a, b = runs
    assert a.stats()["population"] > 1184
    for k in ("tick", "population", "total_divisions", "total_deaths"):
        assert a.stats()[k] == b.stats()[k], k
    assert a.cells().tobytes() == b.cells().tobytes()
    np.testing.assert_array_equal(a.field().view(np.uint32), b.field().view(np.uint32))
