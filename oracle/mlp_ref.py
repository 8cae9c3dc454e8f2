"""CPU restatement of the reaction surrogate's network, for tests only.

Test infrastructure: the parity tests compare the GPU training kernels
(forward, backward) against this file, and the surrogate's input features and
reaction deltas against `reaction_phase` below.  Nothing in the product path
imports it.

The network has no counterpart in the reference.  What it learns does: the
reaction phase of CellState::tick (crates/marl-cell/src/cell.rs:246-285),
restated here in float32 with the reference's operation order.

Network: 93 -> 256 -> 256 -> 16, tanh-form GELU, weights and activations
rounded to BF16 where the GPU stores them in BF16, products accumulated in
float64 here (FP32 on the GPU).  The rounding points follow the GPU kernels:
x, W1, W2, W3, h1, h2, dy, dz2, dz1 are BF16; pre-activations z1, z2, the
output y and all gradients are FP32.  Bias gradients are column sums of the
unrounded dy / dz.
"""
from __future__ import annotations

import numpy as np

IN, IN_PAD, HID, OUT = 93, 128, 256, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN_PAD
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
N_PARAMS = OFF_B3 + OUT
K0 = 0.7978845608028654
K1 = 0.044715


def bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> BF16 bit patterns, round to nearest even (finite inputs)."""
    b = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32)


_ROUND = True  # cleared only by the finite-difference check of the formulas


def bf16(a: np.ndarray) -> np.ndarray:
    if not _ROUND:
        return np.asarray(a)
    return bf16_value(bf16_bits(a))


def unpack(params: np.ndarray):
    p = np.asarray(params, np.float32 if _ROUND else np.float64)
    return (p[OFF_W1:OFF_B1].reshape(HID, IN_PAD), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(OUT, HID), p[OFF_B3:N_PARAMS])


def gelu(z: np.ndarray) -> np.ndarray:
    return 0.5 * z * (1.0 + np.tanh(K0 * (z + K1 * z ** 3)))


def gelu_grad(z: np.ndarray) -> np.ndarray:
    t = np.tanh(K0 * (z + K1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * K0 * (1.0 + 3.0 * K1 * z * z)


def forward(params: np.ndarray, x_bits: np.ndarray):
    """Returns (y, cache) for standardised BF16 inputs x_bits [B][128]."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    f = np.float32 if _ROUND else np.float64
    x = (bf16_value(x_bits) if x_bits.dtype == np.uint16 else x_bits).astype(np.float64)
    z1 = (x @ bf16(W1).astype(np.float64).T + b1).astype(f)
    h1 = bf16(gelu(z1.astype(np.float64)).astype(f)).astype(np.float64)
    z2 = (h1 @ bf16(W2).astype(np.float64).T + b2).astype(f)
    h2 = bf16(gelu(z2.astype(np.float64)).astype(f)).astype(np.float64)
    y = (h2 @ bf16(W3).astype(np.float64).T + b3).astype(f)
    return y, (x, z1, h1, z2, h2)


def loss_and_gradients(params: np.ndarray, x_bits: np.ndarray, t: np.ndarray):
    """Mean squared error over batch and outputs, and its gradient (flat,
    same layout as the parameters)."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    y, (x, z1, h1, z2, h2) = forward(params, x_bits)
    B = x.shape[0]
    e = y.astype(np.float64) - t
    loss = float((e * e).mean())
    f = np.float32 if _ROUND else np.float64
    dy = (2.0 * e / (B * OUT)).astype(f)
    dyb = bf16(dy).astype(np.float64)
    g = np.zeros(N_PARAMS, np.float64)
    g[OFF_B3:N_PARAMS] = dy.sum(0)
    g[OFF_W3:OFF_B3] = (dyb.T @ h2).ravel()
    dz2 = ((dyb @ bf16(W3).astype(np.float64)) * gelu_grad(z2.astype(np.float64))).astype(f)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz2b = bf16(dz2).astype(np.float64)
    g[OFF_W2:OFF_B2] = (dz2b.T @ h1).ravel()
    dz1 = ((dz2b @ bf16(W2).astype(np.float64)) * gelu_grad(z1.astype(np.float64))).astype(f)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    dz1b = bf16(dz1).astype(np.float64)
    g[OFF_W1:OFF_B1] = (dz1b.T @ x).ravel()
    return loss, g.astype(f), y


def feature_transform(raw: np.ndarray) -> np.ndarray:
    """log(|v| + 1e-3) for k_m, v_max and k_cat (features 29 + 4r + {0,1,2})."""
    f = np.array(raw[..., :IN], np.float32, copy=True)
    cols = [29 + 4 * r + k for r in range(16) for k in range(3)]
    f[..., cols] = np.log(np.abs(f[..., cols]) + np.float32(1e-3)).astype(np.float32)
    return f


def reaction_phase(x: np.ndarray, rx: np.ndarray, p) -> np.ndarray:
    """Phase 3 of CellState::tick (crates/marl-cell/src/cell.rs:246-285) for
    many cells at once, float32 in the reference's operation order.

    x: [n][16] internal state after transport (light in slot 15); rx: the
    cells' REACTION_DTYPE records [n][16].  Returns the state after the
    reactions."""
    f32 = np.float32
    x = np.array(x, np.float32, copy=True)
    n = x.shape[0]
    ar = np.arange(n)
    dt, cmax, thr, eps = f32(p.dt), f32(p.c_max), f32(p.active_reaction_threshold), f32(p.epsilon)
    feps = f32(np.finfo(np.float32).eps)
    one = f32(1.0)
    for r in range(16):
        q = rx[:, r]
        vmax = q["v_max"].astype(f32)
        si, pi, ci, fi = (q[k].astype(np.int64) for k in ("substrate", "product", "catalyst", "cofactor"))
        ok = (np.abs(vmax) >= thr) & (si != pi) & (si < 16) & (pi < 16) & (ci < 16)
        si0, pi0, ci0 = (np.where(ok, a, 0) for a in (si, pi, ci))
        s = x[ar, si0]
        cc = x[ar, ci0]
        st = (s / ((q["k_m"].astype(f32) + s) + feps)).astype(f32)
        ct = (eps + (cc / ((q["k_cat"].astype(f32) + cc) + feps)).astype(f32)).astype(f32)
        rate = ((vmax * st).astype(f32) * ct).astype(f32)
        has_cof = ok & (fi != 0xFF) & (fi < 16)
        fi0 = np.where(has_cof, fi, 0)
        cof = x[ar, fi0]
        rate = np.where(has_cof, (rate * (cof / (one + cof)).astype(f32)).astype(f32), rate)
        consumed = np.minimum(((f32(0.5) * rate).astype(f32) * dt).astype(f32), cof)
        x[ar[has_cof], fi0[has_cof]] = (cof - consumed)[has_cof]
        s = x[ar, si0]
        flux = np.minimum((rate * dt).astype(f32), s)
        x[ar[ok], si0[ok]] = (s - flux)[ok]
        pv = x[ar, pi0]
        x[ar[ok], pi0[ok]] = np.minimum((pv + flux).astype(f32), cmax)[ok]
    return x
