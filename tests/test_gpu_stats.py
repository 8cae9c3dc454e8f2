"""Device statistics (marl_ctx_stats) against the quantities of
print_stats / print_z_profile (crates/marl-sim/src/stats.rs:9-103) computed
on the host from the downloaded cells, field and light: counts and
centre-column samples exactly, the averages as FP64 sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_stats(cells, field, light, dims):
    X, Y, Z = dims
    n = len(cells)
    z = cells["pos"][:, 2].astype(np.int64)
    zt = Z // 3
    vmax = cells["ruleset"]["reactions"]["v_max"]
    return {
        "population": n,
        "top": int((z < zt).sum()), "middle": int(((z >= zt) & (z < 2 * zt)).sum()), "bottom": int((z >= 2 * zt).sum()),
        "avg_energy": cells["internal"][:, 0].astype(np.float64).sum() / n,
        "avg_enzyme": cells["internal"][:, 5].astype(np.float64).sum() / n,
        "avg_enzyme_b": cells["internal"][:, 6].astype(np.float64).sum() / n,
        "avg_active_reactions": (np.abs(vmax) > np.float32(1e-9)).sum() / n,
        "oxidant_top": field[0, Y // 2, X // 2, 1], "oxidant_middle": field[Z // 2, Y // 2, X // 2, 1],
        "reductant_bottom": field[Z - 1, Y // 2, X // 2, 2], "organic_middle": field[Z // 2, Y // 2, X // 2, 4],
    }, np.bincount(z, minlength=Z), np.stack([light[:, Y // 2, X // 2]] +
                                            [field[:, Y // 2, X // 2, s] for s in (1, 2, 3, 4)])


@pytest.mark.parametrize("dims,ticks", [((48, 40, 32), 60), ((37, 21, 13), 25)])
def test_device_stats_match_host(marl, dims, ticks):
    e = marl.Engine(dims, marl.default_params(), rng_seed=3, seed_count=20 if dims[2] > 20 else 3,
                    cell_capacity=1 << 14)
    e.step(ticks)
    got, per_z, col = e.device_stats()
    want, want_z, want_col = host_stats(e.cells(), e.field(), e.light(), dims)
    assert got["population"] == want["population"] > 0
    for k in ("top", "middle", "bottom"):
        assert got[k] == want[k], k
    for k in ("avg_energy", "avg_enzyme", "avg_enzyme_b", "avg_active_reactions"):
        assert got[k] == pytest.approx(want[k], rel=1e-12, abs=1e-15), k
    for k in ("oxidant_top", "oxidant_middle", "reductant_bottom", "organic_middle"):
        assert np.float32(got[k]) == np.float32(want[k]), k
    np.testing.assert_array_equal(per_z, want_z)
    np.testing.assert_array_equal(col, want_col)
