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
