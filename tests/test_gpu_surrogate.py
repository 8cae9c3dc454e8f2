"""The learned reaction surrogate on the GPU, through the C ABI.

- The tensor-core training kernels (forward + backward) against the CPU
  restatement of the network (oracle/mlp_ref.py), on the same BF16 inputs.
- Training pairs captured from the plain cell kernel: the capture mode leaves
  the tick bit-identical, and each captured delta is the reference reaction
  phase (crates/marl-cell/src/cell.rs:246-285) applied to the captured state.
- The gated mode at tolerance 0 is the plain tick, bit for bit; counters are
  consistent; the trusted mode runs.
- Gated at 1e-3 with a network trained in the test, every cell's final state
  (after maintenance and effectors, cell.rs:291-329) is within 1e-3 of the
  plain phase's, normwise relative over its 16 species.
- Training on captured pairs reduces the held-out error, and the trained
  network is within 1e-3 of the plain result on more held-out cells than the
  method without it (no reaction update at all) or the untrained network.
"""
import numpy as np
import pytest

import mlp_ref
from helpers import clustered_positions, random_cells, random_field

pytestmark = pytest.mark.gpu


def normwise(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def random_params(rng, scale=1.0) -> np.ndarray:
    p = np.zeros(mlp_ref.N_PARAMS, np.float32)
    w1 = rng.normal(0, scale / np.sqrt(93), (256, 128)).astype(np.float32)
    w1[:, 93:] = 0
    p[mlp_ref.OFF_W1:mlp_ref.OFF_B1] = w1.ravel()
    p[mlp_ref.OFF_B1:mlp_ref.OFF_W2] = rng.normal(0, 0.1, 256)
    p[mlp_ref.OFF_W2:mlp_ref.OFF_B2] = rng.normal(0, scale / 16, 256 * 256)
    p[mlp_ref.OFF_B2:mlp_ref.OFF_W3] = rng.normal(0, 0.1, 256)
    p[mlp_ref.OFF_W3:mlp_ref.OFF_B3] = rng.normal(0, scale / 16, 16 * 256)
    p[mlp_ref.OFF_B3:] = rng.normal(0, 0.1, 16)
    return p


def identity_norm() -> np.ndarray:
    n = np.zeros(mlp_ref.IN * 2 + 32, np.float32)
    n[93:186] = 1.0
    n[202:218] = 1.0
    return n


@pytest.mark.parametrize("batch", [128, 384, 1024])
def test_gradients_match_cpu_oracle(marl, batch):
    """Forward output, loss and every parameter gradient of one batch, GPU
    tcgen05 kernels against the float64 restatement with the same BF16
    rounding points; normwise relative error per tensor <= 2e-3."""
    rng = np.random.default_rng(batch)
    s = marl.Surrogate(max_pairs=1024, batch=128)
    params = random_params(rng)
    s.set_weights(params, identity_norm())
    x = rng.normal(0, 1, (batch, 128)).astype(np.float32)
    x[:, 93:] = 0
    xb = mlp_ref.bf16_bits(x)
    t = rng.normal(0, 1, (batch, 16)).astype(np.float32)
    g, loss, y = s.gradients(xb, t)
    loss_ref, g_ref, y_ref = mlp_ref.loss_and_gradients(params, xb, t)
    assert normwise(y, y_ref) < 2e-3
    assert abs(loss - loss_ref) <= 2e-3 * abs(loss_ref)
    sl = {"W1": (mlp_ref.OFF_W1, mlp_ref.OFF_B1), "b1": (mlp_ref.OFF_B1, mlp_ref.OFF_W2),
          "W2": (mlp_ref.OFF_W2, mlp_ref.OFF_B2), "b2": (mlp_ref.OFF_B2, mlp_ref.OFF_W3),
          "W3": (mlp_ref.OFF_W3, mlp_ref.OFF_B3), "b3": (mlp_ref.OFF_B3, mlp_ref.N_PARAMS)}
    for name, (a, b) in sl.items():
        err = normwise(g[a:b], g_ref[a:b])
        assert err < 2e-3, (name, err)
    # padded input columns of W1 get no gradient
    assert not np.any(g[:mlp_ref.OFF_B1].reshape(256, 128)[:, 93:])
    s.close()


def clustered_state(dims, frac, seed):
    rng = np.random.default_rng(seed)
    pos = clustered_positions(dims, frac, rng, 1, 3)
    cells = random_cells(dims, len(pos), rng, positions=pos)
    field = random_field(dims, rng)
    X, Y, Z = dims
    light = rng.random((Z, Y, X), dtype=np.float32)
    return cells, field, light


def make_ctx(marl, dims, cells, field, light, lanes=32):
    ctx = marl.Context(dims, marl.default_params(), cell_capacity=len(cells))
    marl._check(marl.load().marl_ctx_set_cell_lanes(ctx.h, lanes), "marl_ctx_set_cell_lanes")
    ctx.upload_field(field)
    ctx.upload_light(light)
    ctx.upload_cells(cells)
    return ctx


def test_capture_rows_are_the_plain_reaction_phase(marl):
    dims = (24, 20, 16)
    cells, field, light = clustered_state(dims, 0.2, 5)
    plain = make_ctx(marl, dims, cells, field, light)
    ev_plain = plain.cell_phase()
    cap = make_ctx(marl, dims, cells, field, light)
    s = marl.Surrogate(max_pairs=len(cells) + 10, batch=128)
    marl.ctx_set_surrogate(cap.h, s, marl.SURR_CAPTURE)
    ev_cap = cap.cell_phase()
    # capture changes nothing in the tick
    np.testing.assert_array_equal(ev_cap, ev_plain)
    np.testing.assert_array_equal(cap.download_field(), plain.download_field())
    assert cap.download_cells().tobytes() == plain.download_cells().tobytes()
    rows = s.download_pairs()
    n = len(cells)
    assert rows.shape == (n, marl.SURR_RAW_STRIDE)
    xt = rows[:, :16]
    np.testing.assert_array_equal(rows[:, 15], rows[:, 28])  # light in slot 15 (cell.rs:243)
    rx = cells["ruleset"]["reactions"]
    np.testing.assert_array_equal(rows[:, 29:93:4], rx["k_m"])
    np.testing.assert_array_equal(rows[:, 30:93:4], rx["v_max"])
    np.testing.assert_array_equal(rows[:, 31:93:4], rx["k_cat"])
    np.testing.assert_array_equal(rows[:, 32:93:4], (rx["cofactor"] != 0xFF).astype(np.float32))
    p = marl.default_params()
    xr = mlp_ref.reaction_phase(xt, rx, p)
    np.testing.assert_array_equal(rows[:, 93:109], (xr - xt).astype(np.float32))
    # a full store stops capturing
    cap2 = make_ctx(marl, dims, cells, field, light)
    marl.ctx_set_surrogate(cap2.h, s, marl.SURR_CAPTURE)
    cap2.cell_phase()
    assert s.pair_count() == n + 10
    s.close()


def independent_cells(cells, dims) -> int:
    """Cells none of whose empty face-neighbour voxels touches an earlier cell."""
    X, Y, Z = dims
    cmap = -np.ones((Z, Y, X), np.int64)
    pos = cells["pos"].astype(np.int64)
    cmap[pos[:, 2], pos[:, 1], pos[:, 0]] = np.arange(len(cells))
    faces = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    count = 0
    for j, (x, y, z) in enumerate(pos):
        dep = False
        for dx, dy, dz in faces:
            nx, ny, nz = x + dx, y + dy, z + dz
            if not (0 <= nx < X and 0 <= ny < Y and 0 <= nz < Z) or cmap[nz, ny, nx] >= 0:
                continue
            for ex, ey, ez in faces:
                ux, uy, uz = nx + ex, ny + ey, nz + ez
                if 0 <= ux < X and 0 <= uy < Y and 0 <= uz < Z and 0 <= cmap[uz, uy, ux] < j:
                    dep = True
        count += not dep
    return count


def prepared_surrogate(marl, dims, cells, field, light, seed=0):
    """A surrogate with standardisation from one captured phase (untrained)."""
    cap = make_ctx(marl, dims, cells, field, light)
    s = marl.Surrogate(max_pairs=4 * len(cells), batch=128, seed=seed)
    marl.ctx_set_surrogate(cap.h, s, marl.SURR_CAPTURE)
    cap.cell_phase()
    s.prepare(s.pair_count())
    cap.close()
    return s


def test_gated_zero_tolerance_is_the_plain_tick(marl):
    dims = (24, 20, 16)
    cells, field, light = clustered_state(dims, 0.15, 9)
    s = prepared_surrogate(marl, dims, cells, field, light)
    plain = make_ctx(marl, dims, cells, field, light)
    ev_plain = plain.cell_phase()
    gated = make_ctx(marl, dims, cells, field, light)
    marl.ctx_set_surrogate(gated.h, s, marl.SURR_GATED, 0.0)
    ev = gated.cell_phase()
    np.testing.assert_array_equal(ev, ev_plain)
    np.testing.assert_array_equal(gated.download_field(), plain.download_field())
    assert gated.download_cells().tobytes() == plain.download_cells().tobytes()
    c = marl.ctx_surrogate_counters(gated.h)
    assert c["cells"] == len(cells)
    assert c["accepted"] + c["rejected"] == c["speculated"] <= c["cells"]
    assert c["max_err"] == 0.0
    # the pre-pass is exact for every cell whose neighbourhood no earlier cell writes
    assert c["speculated"] >= independent_cells(cells, dims)
    s.close()


@pytest.mark.parametrize("mode", ["gated", "trusted"])
def test_surrogate_modes_under_lane_refill(marl, mode):
    """With one cell per warp ticket the grid has 1,184 lanes, fewer than the
    cells, so the surrogate modes run through the lane-refill loop.  Gated at
    tolerance 0 it equals the plain phase (run with warp tickets) bit for bit;
    trusted accepts every speculated cell."""
    dims = (40, 32, 24)
    cells, field, light = clustered_state(dims, 0.3, 12)
    assert len(cells) > 1184
    s = prepared_surrogate(marl, dims, cells, field, light, seed=4)
    plain = make_ctx(marl, dims, cells, field, light)
    ev_plain = plain.cell_phase()
    ctx = make_ctx(marl, dims, cells, field, light, lanes=1)
    m = marl.SURR_GATED if mode == "gated" else marl.SURR_TRUSTED
    marl.ctx_set_surrogate(ctx.h, s, m, 0.0)
    ev = ctx.cell_phase()
    c = marl.ctx_surrogate_counters(ctx.h)
    assert c["cells"] == len(cells)
    assert c["accepted"] + c["rejected"] == c["speculated"] <= c["cells"]
    if mode == "gated":
        assert c["max_err"] == 0.0
        np.testing.assert_array_equal(ev, ev_plain)
        np.testing.assert_array_equal(ctx.download_field(), plain.download_field())
        assert ctx.download_cells().tobytes() == plain.download_cells().tobytes()
    else:
        assert c["rejected"] == 0 and c["accepted"] == c["speculated"] > 0
    s.close()


@pytest.mark.parametrize("mode", ["gated", "trusted"])
def test_surrogate_modes_run_and_count(marl, mode):
    dims = (32, 24, 16)
    cells, field, light = clustered_state(dims, 0.1, 21)
    s = prepared_surrogate(marl, dims, cells, field, light, seed=3)
    ctx = make_ctx(marl, dims, cells, field, light)
    m = marl.SURR_GATED if mode == "gated" else marl.SURR_TRUSTED
    marl.ctx_set_surrogate(ctx.h, s, m, 1e-3)
    ctx.cell_phase()
    ctx.cell_phase()
    c = marl.ctx_surrogate_counters(ctx.h)
    assert c["cells"] == 2 * len(cells)
    assert c["accepted"] + c["rejected"] == c["speculated"] <= c["cells"]
    if mode == "gated":
        assert c["max_err"] <= 1e-3
    else:
        assert c["rejected"] == 0 and c["accepted"] == c["speculated"]
    out = ctx.download_cells()["internal"]
    assert np.all(np.isfinite(out)) and np.all(out >= 0)
    marl.ctx_set_surrogate(ctx.h, None, marl.SURR_OFF)
    ctx.cell_phase()  # back to the plain kernel
    s.close()


def test_training_gain_over_the_method_without_it(marl):
    """Pairs captured from a seeded run of the reference default set-up on a
    smaller grid; the last 10 % of rows (the latest ticks) are held out."""
    dims = (64, 64, 32)
    p = marl.default_params()
    eng = marl.Engine(dims, p, rng_seed=7, seed_count=30, cell_capacity=1 << 16)
    s = marl.Surrogate(max_pairs=400_000, batch=4096, lr=2e-3, seed=11)
    eng.step(20)
    marl.ctx_set_surrogate(eng.lib.marl_engine_ctx(eng.h), s, marl.SURR_CAPTURE)
    eng.step(160)
    n = s.pair_count()
    assert n > 20_000, n
    n_train = int(0.9 * n)
    s.prepare(n_train)
    held = (n_train, n - n_train)
    before = s.evaluate(*held, tol=1e-3)
    loss = s.train(1500)
    s.set_lr(5e-4)
    loss = np.concatenate([loss, s.train(1500)])
    after = s.evaluate(*held, tol=1e-3, per_row=True)
    s.set_inference(False)
    layer = s.evaluate(*held, tol=1e-3, per_row=True)
    s.set_inference(True)
    print(f"\nfused: accepted {after['accepted']} mean err {after['mean_err']:.3e}; "
          f"layerwise: accepted {layer['accepted']} mean err {layer['mean_err']:.3e}; "
          f"max row diff {np.abs(after['row_err'] - layer['row_err']).max():.3e}")
    np.testing.assert_array_equal(after["row_err"], layer["row_err"])
    raw = s.download_pairs(n_train, n - n_train)
    xt, d = raw[:, :16], raw[:, 93:109]
    plain = xt + d
    zero_err = np.abs(d).max(1) / np.maximum(np.abs(plain).max(1), 1e-6)  # no reaction update at all
    zero_accept = int((zero_err <= 1e-3).sum())
    print(f"\nheld-out rows {held[1]}: untrained accepts {before['accepted']}, zero-delta accepts {zero_accept}, "
          f"trained accepts {after['accepted']} ({after['accepted'] / held[1]:.3f}); "
          f"mse {before['mse_normalised']:.4f} -> {after['mse_normalised']:.5f}; "
          f"mean err {after['mean_err']:.2e}; loss {loss[:20].mean():.4f} -> {loss[-100:].mean():.5f}")
    assert np.all(np.isfinite(loss))
    assert loss[-100:].mean() < 0.2 * loss[:20].mean()
    assert after["mse_normalised"] < 0.2 * before["mse_normalised"]
    assert after["accepted"] > zero_accept
    assert after["accepted"] > before["accepted"]
    s.close()


@pytest.mark.parametrize("rows", [1, 127, 128, 1000, 40_000])
def test_fused_inference_matches_layerwise_and_oracle(marl, rows):
    """The persistent fused inference kernel against the one-GEMM-per-layer
    path (same hardware tanh) and against the CPU restatement (exact tanh):
    normwise relative error <= 1e-4 and <= 1e-2 (BF16 activations)."""
    import torch

    rng = np.random.default_rng(rows)
    s = marl.Surrogate(max_pairs=128, batch=128)
    # inputs and outputs are torch tensors: order the inference on torch's stream
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    params = random_params(rng)
    norm = identity_norm()
    norm[186:202] = rng.normal(0, 0.1, 16)          # output mean
    norm[202:218] = rng.uniform(0.5, 2.0, 16)        # output std
    s.set_weights(params, norm)
    x = rng.normal(0, 1, (rows, 128)).astype(np.float32)
    x[:, 93:] = 0
    bits = mlp_ref.bf16_bits(x)
    X = torch.from_numpy(bits.view(np.int16)).cuda()
    y_fused = torch.full((16, rows), float("nan"), device="cuda")
    y_layer = torch.full((16, rows), float("nan"), device="cuda")
    s.set_inference(True)
    s.infer_device(X.data_ptr(), rows, y_fused.data_ptr(), rows)
    s.set_inference(False)
    s.infer_device(X.data_ptr(), rows, y_layer.data_ptr(), rows)
    torch.cuda.synchronize()
    yf, yl = y_fused.cpu().numpy().T, y_layer.cpu().numpy().T
    assert np.all(np.isfinite(yf))
    ref = mlp_ref.forward(params, bits)[0].astype(np.float64) * norm[202:218] + norm[186:202]
    e_layer, e_ref = normwise(yf, yl), normwise(yf, ref)
    print(f"\nrows {rows}: fused vs layerwise {e_layer:.2e}, fused vs oracle {e_ref:.2e}")
    assert e_layer <= 1e-4
    assert e_ref <= 1e-2
    s.close()


def test_gated_final_state_within_tolerance(marl):
    """A network trained on pairs from a seeded 64x64x32 default run; from a
    later state of that run one plain and one gated (1e-3) cell phase.  The
    gate judges the cell's final state, so every cell, accepted or not, ends
    within 1e-3 of the plain phase (normwise relative, 16 species)."""
    dims = (64, 64, 32)
    p = marl.default_params()
    eng = marl.Engine(dims, p, rng_seed=7, seed_count=30, cell_capacity=1 << 16)
    s = marl.Surrogate(max_pairs=400_000, batch=4096, lr=2e-3, seed=11)
    eng.step(20)
    marl.ctx_set_surrogate(eng.lib.marl_engine_ctx(eng.h), s, marl.SURR_CAPTURE)
    eng.step(160)
    marl.ctx_set_surrogate(eng.lib.marl_engine_ctx(eng.h), None, marl.SURR_OFF)
    s.prepare(s.pair_count())
    s.train(1500)
    s.set_lr(5e-4)
    s.train(1500)
    eng.step(20)
    field, cells, light = eng.field(), eng.cells(), eng.light()
    eng.close()
    plain = make_ctx(marl, dims, cells, field, light)
    plain.cell_phase()
    want = plain.download_cells()["internal"]
    gated = make_ctx(marl, dims, cells, field, light)
    marl.ctx_set_surrogate(gated.h, s, marl.SURR_GATED, 1e-3)
    gated.cell_phase()
    got = gated.download_cells()["internal"]
    c = marl.ctx_surrogate_counters(gated.h)
    err = np.abs(got - want).max(1) / np.maximum(np.abs(want).max(1), 1e-6)
    print(f"\n{len(cells)} cells: speculated {c['speculated']}, accepted {c['accepted']}, "
          f"max accepted err {c['max_err']:.3e}, max cell err {err.max():.3e}")
    assert c["accepted"] > 0
    assert c["max_err"] <= 1e-3
    assert err.max() <= 1e-3
    s.close()
