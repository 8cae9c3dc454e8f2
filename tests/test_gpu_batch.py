"""The batched ensemble (marl_batch): every run of a batch must equal, bit for
bit, a single-run engine created with the same grid, parameters, seed and
seed count, whatever the batch's tile choice, graph use or host thread count."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RUNS = [((24, 24, 16), 3), ((32, 24, 24), 7), ((48, 40, 64), 42), ((40, 36, 32), 11)]


def engines(marl, params, runs, ticks, seed_count=30):
    out = []
    for dims, seed in runs:
        e = marl.Engine(dims, params, rng_seed=seed, seed_count=seed_count, cell_capacity=1 << 14)
        e.step(ticks)
        out.append(e)
    return out


def assert_run_equal(batch, r, eng):
    bs, es = batch.stats(r), eng.stats()
    for k in ("tick", "population", "total_divisions", "total_deaths"):
        assert bs[k] == es[k], (r, k, bs[k], es[k])
    assert batch.cells(r).tobytes() == eng.cells().tobytes(), r
    assert np.array_equal(batch.field(r).view(np.uint32), eng.field().view(np.uint32)), r
    assert np.array_equal(batch.light(r).view(np.uint32), eng.light().view(np.uint32)), r


@pytest.mark.parametrize("substeps", [10, 3])
def test_batch_matches_single_engines(marl, substeps):
    """Uneven grids; odd substep counts flip the ping-pong parity every tick
    (two captured graphs)."""
    p = marl.default_params()
    p.diffusion_substeps = substeps
    ticks = 60
    b = marl.Batch(RUNS, p, cell_capacity=1 << 14)
    b.step(ticks)
    refs = engines(marl, p, RUNS, ticks)
    events = 0
    for r, eng in enumerate(refs):
        assert_run_equal(b, r, eng)
        s = b.stats(r)
        events += s["total_divisions"] + s["total_deaths"]
    assert events > 0, "no fate events: the edit path was not exercised"
    c = b.counters()
    assert c["ticks"] == ticks and c["device_us"] > 0 and c["kernel_launches"] >= ticks * (substeps + 5)


def test_batch_graph_tile_threads_invariance(marl):
    """Graph replay vs direct launches, a tile change mid-run, one vs many host
    threads: identical results."""
    p = marl.default_params()
    runs = RUNS[:3]
    a = marl.Batch(runs, p, cell_capacity=1 << 14)
    a.set_graph(False)
    a.set_host_threads(1)
    a.step(25)
    b = marl.Batch(runs, p, cell_capacity=1 << 14)
    b.set_host_threads(0)
    b.step(10)
    b.set_tile(5, 8)
    assert b.get_tile() == (5, 8)
    b.step(10)
    b.autotune(reps=2)
    b.step(5)
    for r in range(len(runs)):
        assert a.cells(r).tobytes() == b.cells(r).tobytes(), r
        assert np.array_equal(a.field(r).view(np.uint32), b.field(r).view(np.uint32)), r


def test_batch_errors(marl):
    p = marl.default_params()
    with pytest.raises(marl.MarlError):
        marl.Batch([], p)
    with pytest.raises(marl.MarlError):
        marl.Batch([((8, 8, 8), 1)], p)  # grid too small for the seeding margin
    b = marl.Batch([((24, 24, 16), 1)], p)
    with pytest.raises(marl.MarlError):
        b.stats(1)
    with pytest.raises(marl.MarlError):
        b.set_tile(99, 16)
    b.step(2)
    assert b.stats(0)["tick"] == 2


def captured_surrogate(marl, p, seed=3):
    """A surrogate standardised on pairs captured from one single-run engine
    (untrained weights: the modes' bookkeeping does not need a good network)."""
    e = marl.Engine((32, 24, 24), p, rng_seed=seed, seed_count=30, cell_capacity=1 << 14)
    s = marl.Surrogate(max_pairs=200_000, batch=128, seed=seed)
    e.step(10)
    marl.ctx_set_surrogate(e.lib.marl_engine_ctx(e.h), s, marl.SURR_CAPTURE)
    e.step(15)
    marl.ctx_set_surrogate(e.lib.marl_engine_ctx(e.h), None, marl.SURR_OFF)
    s.prepare(s.pair_count())
    return s


def test_batch_surrogate_gated_zero_tolerance_is_plain(marl):
    """The batched surrogate path at tolerance 0 reproduces the plain batch bit
    for bit (a prediction is kept only when it equals the plain result)."""
    p = marl.default_params()
    runs = RUNS[:3]
    s = captured_surrogate(marl, p)
    plain = marl.Batch(runs, p, cell_capacity=1 << 14)
    plain.step(30)
    gated = marl.Batch(runs, p, cell_capacity=1 << 14)
    gated.step(5)
    gated.set_surrogate(s, marl.SURR_GATED, 0.0)
    gated.step(25)
    c = gated.surrogate_counters()
    assert c["cells"] > 0 and c["accepted"] + c["rejected"] == c["speculated"] <= c["cells"]
    assert c["max_err"] == 0.0
    for r in range(len(runs)):
        assert plain.cells(r).tobytes() == gated.cells(r).tobytes(), r
        assert np.array_equal(plain.field(r).view(np.uint32), gated.field(r).view(np.uint32)), r
    gated.set_surrogate(None, marl.SURR_OFF)
    gated.step(2)  # back to the captured-graph plain tick
    s.close()


def test_batch_surrogate_trusted_runs(marl):
    p = marl.default_params()
    s = captured_surrogate(marl, p, seed=8)
    b = marl.Batch(RUNS, p, cell_capacity=1 << 14)
    b.set_surrogate(s, marl.SURR_TRUSTED)
    b.step(20)
    c = b.surrogate_counters()
    assert c["rejected"] == 0 and c["accepted"] == c["speculated"] > 0
    for r in range(len(RUNS)):
        x = b.cells(r)["internal"]
        assert np.all(np.isfinite(x)) and np.all(x >= 0)
    with pytest.raises(marl.MarlError):
        b.set_surrogate(s, marl.SURR_CAPTURE)
    s.close()


# Five runs of ~9,000 seeded cells each: together more cells than the batched
# cell kernel's grid has lanes (2 resident blocks x 148 SMs x 128 = 37,888),
# so the batch advances them by lane refill, while each single-run engine
# (9,000 cells, one lane each) uses warp tickets.
BIG_RUNS = [((96, 96, 48), seed, 3000, 1 << 15) for seed in (21, 22, 23, 24, 25)]


def test_batch_lane_refill_matches_single_engines(marl):
    p = marl.default_params()
    ticks = 8
    b = marl.Batch(BIG_RUNS, p)
    total = sum(b.stats(r)["population"] for r in range(len(BIG_RUNS)))
    assert total > 37_888, total
    b.step(ticks)
    for r, (dims, seed, seed_count, cap) in enumerate(BIG_RUNS):
        e = marl.Engine(dims, p, rng_seed=seed, seed_count=seed_count, cell_capacity=cap)
        e.step(ticks)
        assert_run_equal(b, r, e)
        e.close()


def test_batch_surrogate_gated_zero_tolerance_under_lane_refill(marl):
    """Gated at tolerance 0 through the lane-refill form of the batched loop
    reproduces the plain batch bit for bit."""
    p = marl.default_params()
    s = captured_surrogate(marl, p, seed=9)
    plain = marl.Batch(BIG_RUNS, p)
    plain.step(6)
    gated = marl.Batch(BIG_RUNS, p)
    gated.step(2)
    gated.set_surrogate(s, marl.SURR_GATED, 0.0)
    gated.step(4)
    c = gated.surrogate_counters()
    assert c["cells"] > 37_888 and c["max_err"] == 0.0
    for r in range(len(BIG_RUNS)):
        assert plain.cells(r).tobytes() == gated.cells(r).tobytes(), r
        assert np.array_equal(plain.field(r).view(np.uint32), gated.field(r).view(np.uint32)), r
    gated.set_surrogate(None, marl.SURR_OFF)
    s.close()
