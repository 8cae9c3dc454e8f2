"""Whole runs: the device engine (marl_sim::run's tick loop with host fate
processing) against the oracle's sequential restatement with the same seeded
RNG, and the C-ABI error paths."""
import numpy as np
import pytest

from helpers import random_cells

pytestmark = pytest.mark.gpu


def compare_runs(marl, oracle_mod, dims, ticks, seed=42, seed_count=30):
    p = marl.default_params()
    eng = marl.Engine(dims, p, rng_seed=seed, seed_count=seed_count, cell_capacity=1 << 16)
    w = oracle_mod.World(dims, p, seed=seed, seed_count=seed_count)
    np.testing.assert_array_equal(eng.field(), w.field())
    c0 = eng.cells()
    assert c0.tobytes() == w.cells().tobytes()  # identical seeding (same RNG stream)
    report = []
    for t in range(ticks):
        eng.step(1)
        w.tick(1)
        es, ws = eng.stats(), w.stats()
        gc, wc = eng.cells(), w.cells()
        same_pop = es["population"] == ws["population"]
        report.append((t, es["population"], ws["population"]))
        if not same_pop:
            break
        np.testing.assert_array_equal(gc["pos"], wc["pos"])
        np.testing.assert_array_equal(gc["lineage_id"], wc["lineage_id"])
        np.testing.assert_allclose(gc["internal"], wc["internal"], rtol=1e-4, atol=1e-5)
    return eng, w, report


def test_engine_matches_oracle_small_grid(marl, oracle_mod):
    eng, w, rep = compare_runs(marl, oracle_mod, (48, 40, 64), 40)
    assert all(a == b for _, a, b in rep), rep
    np.testing.assert_allclose(eng.field(), w.field(), rtol=1e-4, atol=1e-5)
    s = eng.stats()
    assert s["tick"] == 40 and s["h2d_bytes_last_tick"] >= 0 and s["d2h_bytes_last_tick"] > 0


def test_engine_default_run_prefix(marl, oracle_mod):
    """Reference default run (128x128x64, 3 x 30 seeded cells), first ticks."""
    eng, w, rep = compare_runs(marl, oracle_mod, (128, 128, 64), 8)
    assert all(a == b for _, a, b in rep), rep
    np.testing.assert_allclose(eng.light(), w.light(), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(eng.field(), w.field(), rtol=1e-4, atol=1e-5)


def test_engine_divisions_and_deaths_tracked(marl, oracle_mod):
    """Dense energetic population: divisions and deaths in the first ticks."""
    dims = (24, 24, 16)
    rng = np.random.default_rng(31)
    cells = random_cells(dims, 400, rng)
    cells["prep_remaining"] = np.where(rng.random(400) < 0.5, 1, 0)
    cells["internal"][:, 0] = np.where(rng.random(400) < 0.3, 0.0, 2.0)
    f = rng.random((16, 24, 24, 12), dtype=np.float32)
    p = marl.default_params()
    eng = marl.Engine(dims, p, rng_seed=5, cell_capacity=4096, field=f, cells=cells)
    w = oracle_mod.World(dims, p, seed=5, seed_count=None)
    w.set_field(f)
    w.set_cells(cells)
    eng.step(1)
    w.tick(1)
    es, ws = eng.stats(), w.stats()
    assert es["tick_divisions"] > 0 and es["tick_deaths"] > 0
    assert (es["population"], es["tick_divisions"], es["tick_deaths"]) == (
        ws["population"], ws["tick_divisions"], ws["tick_deaths"])
    gc, wc = eng.cells(), w.cells()
    np.testing.assert_array_equal(gc["pos"], wc["pos"])
    np.testing.assert_array_equal(gc["lineage_id"], wc["lineage_id"])
    assert gc["ruleset"].tobytes() == wc["ruleset"].tobytes()  # mutation stream identical
    np.testing.assert_allclose(gc["internal"], wc["internal"], rtol=1e-4, atol=1e-5)


def test_errors_are_reported(marl):
    dims = (8, 8, 8)
    ctx = marl.Context(dims, cell_capacity=4)
    rng = np.random.default_rng(0)
    dup = random_cells(dims, 2, rng, positions=np.array([[1, 1, 1], [1, 1, 1]]))
    with pytest.raises(marl.MarlError) as e:
        ctx.upload_cells(dup)
    assert e.value.status_name == "INVALID_INPUT"
    out = random_cells(dims, 1, rng, positions=np.array([[1, 1, 1]]))
    out["pos"][0] = (8, 0, 0)
    with pytest.raises(marl.MarlError) as e:
        ctx.upload_cells(out)
    assert e.value.status_name == "INVALID_INPUT"
    with pytest.raises(marl.MarlError) as e:
        ctx.upload_cells(random_cells(dims, 5, rng))
    assert e.value.status_name == "CAPACITY"
    ctx.upload_cells(random_cells(dims, 3, rng))
    with pytest.raises(marl.MarlError) as e:  # n_after_deaths inconsistent
        ctx.apply_edits(deaths=[0], n_after_deaths=3)
    assert e.value.status_name == "INVALID_INPUT"
    with pytest.raises(marl.MarlError) as e:  # move source inside the kept range
        ctx.apply_edits(deaths=[0], moves=[(0, 1)], n_after_deaths=2)
    assert e.value.status_name == "INVALID_INPUT"
    with pytest.raises(marl.MarlError) as e:
        ctx.apply_edits(births=random_cells(dims, 2, rng))
    assert e.value.status_name == "CAPACITY"
    assert ctx.cell_count() == 3
