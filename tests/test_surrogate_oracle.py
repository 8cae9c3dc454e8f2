"""CPU checks of the surrogate's oracle (oracle/mlp_ref.py), no GPU.

- The backward formulas are the derivative of the loss: with the BF16
  rounding switched off, the analytic gradient matches central differences.
- The vectorised reaction phase equals the C++ oracle's CellState::tick
  (crates/marl-cell/src/cell.rs:193-369) bit for bit on cells whose
  transport, maintenance and effectors are switched off, so that the tick's
  only change to the internal state is the reaction phase.
"""
import numpy as np
import pytest

import mlp_ref
from helpers import random_cells


@pytest.fixture
def exact_network():
    mlp_ref._ROUND = False
    yield
    mlp_ref._ROUND = True


def test_backward_is_the_derivative_of_the_loss(exact_network):
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, mlp_ref.N_PARAMS)
    p[:mlp_ref.OFF_B1].reshape(256, 128)[:, 93:] = 0
    x = rng.normal(0, 1, (8, 128))
    x[:, 93:] = 0
    t = rng.normal(0, 1, (8, 16))
    _, g, _ = mlp_ref.loss_and_gradients(p, x, t)
    idx = np.concatenate([rng.integers(a, b, 6) for a, b in (
        (mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
        (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.OFF_B3), (mlp_ref.OFF_B3, mlp_ref.N_PARAMS))])
    idx = [i for i in idx if not (i < mlp_ref.OFF_B1 and i % 128 >= 93)]
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        num = (mlp_ref.loss_and_gradients(pp, x, t)[0] - mlp_ref.loss_and_gradients(pm, x, t)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])


def test_reaction_phase_matches_the_cpp_oracle(oracle_mod):
    dims = (16, 16, 16)
    rng = np.random.default_rng(3)
    cells = random_cells(dims, 64, rng)
    rs = cells["ruleset"]
    rs["transport"]["ext_species"] = 0xFF  # no transporter acts
    rs["effectors"]["int_species"] = 0xFF
    cells["prep_remaining"] = 0
    p = oracle_mod.default_params()
    p.lambda_maintenance = 0.0
    p.reaction_maintenance = 0.0
    light = rng.random(len(cells)).astype(np.float32)
    ext = rng.random((len(cells), 12)).astype(np.float32)
    x = cells["internal"].copy()
    x[:, 15] = light
    got = mlp_ref.reaction_phase(x, rs["reactions"], p)
    for j in range(len(cells)):
        out = oracle_mod.cell_tick(cells[j], ext[j], float(light[j]), p)
        want = out[0]["internal"] if isinstance(out, tuple) else out["internal"]
        np.testing.assert_array_equal(got[j], want)
