"""Single-kernel cases on synthetic inputs, for profiling one kernel in isolation.

    python marl-ochre_b200/kernel_cases.py diffusion [--dims 128 128 64] [--tile 6] [--zc 16] [--substeps 8]
    python marl-ochre_b200/kernel_cases.py cells [--dims 128 128 64] [--cells 90] [--reps 4]
    python marl-ochre_b200/kernel_cases.py light [--dims 128 128 64] [--reps 4]
    python marl-ochre_b200/kernel_cases.py mlp [--rows 300000] [--reps 4]
    python marl-ochre_b200/kernel_cases.py engine [--ticks 1000] [--device-fate]   (seed-42 default
        run; one k_cell_tick launch per tick, so `-k regex:k_cell_tick -s <ticks-1> -c 1` captures
        the last; with --device-fate the fate step runs on the GPU and all ticks are enqueued at once)

Each case builds a context, uploads seeded synthetic state and runs the kernel
a few times.  Under `ncu -k regex:<kernel> -s <n> -c 1` that captures one
launch with the earlier launches as warm-up.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import marl_cuda as marl  # noqa: E402


def clustered_cells(dims, frac: float, rng: np.random.Generator) -> np.ndarray:
    """Cells on random balls of radius 2-4 until `frac` of the voxels are covered."""
    X, Y, Z = dims
    occ = np.zeros((Z, Y, X), bool)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    while occ.sum() < frac * X * Y * Z:
        r = rng.integers(2, 5)
        cx, cy, cz = rng.integers(0, X), rng.integers(0, Y), rng.integers(0, Z)
        occ |= (xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2 <= r * r
    z, y, x = np.nonzero(occ)
    c = np.zeros(len(x), marl.CELL_DTYPE)
    c["pos"] = np.stack([x, y, z], 1)
    return c


def random_cells(dims, n: int, rng: np.random.Generator) -> np.ndarray:
    """n cells with random rulesets at unique random voxels."""
    X, Y, Z = dims
    flat = rng.choice(X * Y * Z, size=n, replace=False)
    z, rem = np.divmod(flat, X * Y)
    y, x = np.divmod(rem, X)
    c = np.zeros(n, marl.CELL_DTYPE)
    c["pos"] = np.stack([x, y, z], 1)
    c["internal"] = rng.random((n, 16), dtype=np.float32)
    rx = c["ruleset"]["reactions"]
    rx["substrate"] = rng.integers(0, 16, (n, 16))
    rx["product"] = rng.integers(0, 16, (n, 16))
    rx["catalyst"] = rng.integers(0, 16, (n, 16))
    rx["cofactor"] = 0xFF
    rx["k_m"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    rx["v_max"] = rng.lognormal(0.0, 1.0, (n, 16)).astype(np.float32)
    rx["k_cat"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    tp = c["ruleset"]["transport"]
    tp["uptake_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["secrete_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["ext_species"] = rng.integers(0, 12, (n, 8))
    tp["int_species"] = rng.integers(0, 16, (n, 8))
    c["ruleset"]["fate"]["division_energy"] = 10.0
    return c


def mlp_case(rows: int, reps: int, rng: np.random.Generator) -> int:
    """Surrogate inference (three tcgen05 GEMM launches) on `rows` random
    standardised feature rows, with random weights."""
    import torch

    s = marl.Surrogate(max_pairs=128, batch=128)
    s.set_stream(torch.cuda.current_stream().cuda_stream)  # inputs are torch tensors
    params = np.zeros(marl.SURR_PARAMS, np.float32)
    params[: 256 * 128] = rng.normal(0, 0.1, 256 * 128)
    params[256 * 128 + 256: 256 * 128 + 256 + 65536] = rng.normal(0, 0.06, 65536)
    params[-16 - 4096: -16] = rng.normal(0, 0.06, 4096)
    norm = np.zeros(marl.SURR_NORM, np.float32)
    norm[93:186] = 1.0
    norm[202:218] = 1.0
    s.set_weights(params, norm)
    x = torch.randn(rows, 128, device="cuda").to(torch.bfloat16)
    x[:, 93:] = 0
    y = torch.empty(16, rows, device="cuda")
    torch.cuda.synchronize()
    for _ in range(reps):
        s.infer_device(x.data_ptr(), rows, y.data_ptr(), rows)
    torch.cuda.synchronize()
    print(f"mlp ok: rows={rows} reps={reps} finite={bool(torch.isfinite(y).all())}")
    s.close()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["diffusion", "cells", "light", "mlp", "engine"])
    ap.add_argument("--ticks", type=int, default=1000, help="engine: ticks of the seed-42 default run")
    ap.add_argument("--device-fate", action="store_true", help="engine: fate on the device")
    ap.add_argument("--rows", type=int, default=300_000, help="mlp: rows (cells) per inference")
    ap.add_argument("--dims", type=int, nargs=3, default=[128, 128, 64])
    ap.add_argument("--tile", type=int, default=-1, help="diffusion tile index (-1: autotune)")
    ap.add_argument("--zc", type=int, default=16)
    ap.add_argument("--substeps", type=int, default=8)
    ap.add_argument("--cells", type=int, default=90)
    ap.add_argument("--reps", type=int, default=4)
    a = ap.parse_args()
    dims = tuple(a.dims)
    X, Y, Z = dims
    rng = np.random.default_rng(1)
    if a.case == "mlp":
        return mlp_case(a.rows, a.reps, rng)
    if a.case == "engine":
        e = marl.Engine(dims, marl.default_params(), rng_seed=42, seed_count=30, cell_capacity=1 << 20)
        if a.device_fate:
            e.set_device_fate(True)
        e.step(a.ticks)
        print(f"engine ok: dims={dims} ticks={a.ticks} stats={e.stats()}")
        return 0
    field = rng.random((Z, Y, X, 12), dtype=np.float32)
    if a.case == "cells":
        cells = random_cells(dims, a.cells, rng)
    else:
        cells = clustered_cells(dims, 0.05, rng)
    ctx = marl.Context(dims, cell_capacity=max(len(cells), 1))
    ctx.upload_field(field)
    ctx.upload_cells(cells)
    if a.case == "diffusion":
        if a.tile >= 0:
            ctx.set_tile(a.tile, a.zc)
        else:
            ctx.autotune(3)
        ctx.diffuse(a.substeps)
    elif a.case == "cells":
        ctx.upload_light(rng.random((Z, Y, X), dtype=np.float32))
        for _ in range(a.reps):
            ctx.cell_phase()
    else:
        for _ in range(a.reps):
            ctx.light_update()
    ctx.synchronize()
    print(f"{a.case} ok: dims={dims} cells={len(cells)} tile={ctx.get_tile()}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
