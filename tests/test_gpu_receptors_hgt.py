"""Receptor activations (phase 1 of CellState::tick, crates/marl-cell/src/
cell.rs:206-220) and horizontal gene transfer (crates/marl-cell/src/hgt.rs:
7-27) on the GPU against the oracle.

- With the receptor output on, each cell's 8 activations, from the
  environment it gathered in the sequential loop, are within 1e-5 relative
  (absolute floor 1e-6) of the oracle's (CUDA powf against glibc powf), and
  the tick itself stays bit-identical to the oracle's.
- HGT over pair lists with repeated donors, chained transfers (a recipient
  that later donates, a donor that later receives) and self pairs gives
  rulesets byte-identical to the oracle's sequential transfers with the same
  per-pair streams.
"""
import numpy as np
import pytest

from helpers import clustered_positions, random_cells, random_field

pytestmark = pytest.mark.gpu


def state(dims, frac, seed):
    rng = np.random.default_rng(seed)
    pos = clustered_positions(dims, frac, rng, 1, 3)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    cells["ruleset"]["receptors"]["n_hill"] = rng.uniform(0.1, 10.0, (len(cells), 8)).astype(np.float32)
    cells["ruleset"]["receptors"]["gain"][:, ::3] = 0.0  # inactive receptors give 0
    X, Y, Z = dims
    return cells, random_field(dims, rng), rng.random((Z, Y, X), dtype=np.float32)


@pytest.mark.parametrize("dims,frac,seed", [((24, 20, 16), 0.2, 3), ((32, 24, 16), 0.05, 4)])
def test_receptor_activations_match_oracle(marl, oracle_mod, dims, frac, seed):
    cells, field, light = state(dims, frac, seed)
    p = marl.default_params()
    ctx = marl.Context(dims, p, cell_capacity=len(cells))
    ctx.upload_field(field)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    ctx.set_receptor_output(True)
    ev = ctx.cell_phase()
    act = ctx.receptor_activations()
    cf, cc, ce, want = oracle_mod.cell_phase_act(field, light, cells, dims, p)
    np.testing.assert_allclose(act, want, rtol=1e-5, atol=1e-6)
    assert np.all(act[:, ::3] == 0) and np.count_nonzero(act) > len(cells)
    # the output changes nothing in the tick
    np.testing.assert_array_equal(ctx.download_field(), cf)
    np.testing.assert_array_equal(ctx.download_cells()["internal"], cc["internal"])
    np.testing.assert_array_equal(ev.astype(np.int32), ce)
    ctx.set_receptor_output(False)
    with pytest.raises(marl.MarlError) as e:
        ctx.receptor_activations()
    assert e.value.status_name == "STATE"
    ctx.close()


def test_hgt_matches_oracle(marl, oracle_mod):
    dims = (24, 20, 16)
    rng = np.random.default_rng(8)
    cells = random_cells(dims, 400, rng)
    vmax = cells["ruleset"]["reactions"]["v_max"]
    vmax[rng.random(vmax.shape) < 0.3] = 0.0   # inactive slots (recipients fill the first one)
    vmax[:40] = 0.0                            # donors with no active reaction: no transfer
    vmax[40:80] = 1.0                          # recipients with every slot active: a random slot
    donors = rng.integers(0, 400, 3000)
    recipients = rng.integers(0, 400, 3000)
    donors[:50] = 7                            # one donor, many recipients
    recipients[50:60] = donors[60:70]          # recipients that donate next
    donors[70:80] = recipients[80:90]          # donors that receive next
    recipients[90:100] = donors[90:100]        # self transfers
    ctx = marl.Context(dims, marl.default_params(), cell_capacity=len(cells))
    ctx.upload_cells(cells)
    ctx.hgt(donors, recipients, seed=12345, tick=77)
    got = ctx.download_cells()
    want = oracle_mod.hgt(cells, donors, recipients, 12345, 77)
    assert got["ruleset"].tobytes() == want["ruleset"].tobytes()
    assert got["ruleset"].tobytes() != cells["ruleset"].tobytes()
    with pytest.raises(marl.MarlError) as e:
        ctx.hgt([0, 400], [1, 2], 1, 1)
    assert e.value.status_name == "INVALID_INPUT"
    ctx.close()
