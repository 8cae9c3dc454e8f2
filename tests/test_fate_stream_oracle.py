"""The oracle's restatement of the device-fate random streams (CPU): the
series logarithm against numpy, the polar normals' distribution, and the
stream fate mode of the oracle's world against its sequential mode on the
parts that draw no random numbers (deaths, swap_remove order)."""
import numpy as np
import pytest

from helpers import random_cells


def test_fate_log_matches_numpy(oracle_mod):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.random(200000), np.ldexp(rng.random(2000) + 0.5, -rng.integers(1, 100, 2000)),
                        [0.5, np.nextafter(1.0, 0.0), 2.0 ** -104, np.sqrt(0.5), np.nextafter(np.sqrt(0.5), 0.0)]])
    x = x[(x > 0) & (x < 1)]
    got = oracle_mod.fate_log(x)
    ref = np.log(x)
    ulp = np.spacing(np.abs(ref))
    assert np.max(np.abs(got - ref) / ulp) <= 4.0


def test_fate_stream_normals_are_standard_normal(oracle_mod):
    from scipy import stats

    draws = np.concatenate([oracle_mod.fate_stream(11, t, p, 500)[1] for t in range(4) for p in range(50)])
    assert draws.size == 100000
    assert abs(draws.mean()) < 0.015 and abs(draws.std() - 1.0) < 0.01
    assert stats.kstest(draws.astype(np.float64), "norm").pvalue > 1e-3
    assert np.all(np.isfinite(draws))


def test_fate_stream_keys_are_distinct(oracle_mod):
    seen = set()
    for seed in (0, 1, 42):
        for tick in (0, 1, 2**40):
            for parent in (0, 1, 7, 2**31):
                u, _ = oracle_mod.fate_stream(seed, tick, parent, 2)
                seen.add(tuple(int(v) for v in u))
    assert len(seen) == 3 * 3 * 4


def test_stream_mode_keeps_deaths_and_order(oracle_mod):
    """Deaths and the swap_remove order draw nothing: the surviving parents
    and their order agree between the two fate modes."""
    dims = (20, 20, 12)
    rng = np.random.default_rng(8)
    cells = random_cells(dims, 1200, rng)
    ev = rng.choice([0, 1, 2, 3], size=cells.size, p=[0.45, 0.25, 0.2, 0.1]).astype(np.int32)
    p = oracle_mod.default_params()
    out = []
    for mode in (0, 1):
        w = oracle_mod.World(dims, p, seed=9, seed_count=None)
        w.set_cells(cells)
        w.set_fate_mode(mode)
        w.fate(ev)
        out.append((w.cells(), w.stats()))
    (c0, s0), (c1, s1) = out
    n1 = cells.size - int((ev == 2).sum())
    assert s0["tick_deaths"] == s1["tick_deaths"] == int((ev == 2).sum())
    np.testing.assert_array_equal(c0["lineage_id"][:n1], c1["lineage_id"][:n1])
    np.testing.assert_array_equal(c0["pos"][:n1], c1["pos"][:n1])
