"""Seeded synthetic inputs of the field and cell microbenchmarks.

Field microbenchmark: a 256x256x128 grid, 12 species with values uniform in
[0, 1), 5 % of the voxels occupied as random balls of radius 2-4, and a
deposit slowdown factor f uniform in [0.5, 1].  The reference applies the
slowdown through the centre voxel's species 7 (crates/marl-field/src/field.rs:
nf = 1 - alpha * c7 / (k + c7), alpha = 0.8, k = 2), so species 7 is set to
c7 = k (1 - f) / (f - (1 - alpha)), which makes nf equal f.  Species 4
uniform in [0, 1) with chemical_absorption 0.05 gives a per-voxel absorbance
uniform in [0, 0.05] for the light scan.

Cell microbenchmark: 1,000,000 cells at unique random voxels of a 256x256x128
grid.  Each cell has 16 internal species uniform in [0, 1) and 16 reactions
with substrate, product and catalyst uniform over the 16 internal species
(catalyst forced to the light slot 15 on 25 % of reactions), v_max
lognormal(0, 1), k_m and k_cat uniform in [0.01, 1], no cofactor; 8
transporters and 8 effectors with random species and rates uniform in [0, 1).
"""
from __future__ import annotations

import numpy as np

import marl_cuda as marl

MICRO_DIMS = (256, 256, 128)


def clustered_occupancy(dims, frac: float, rng: np.random.Generator, rmin: int = 2, rmax: int = 4) -> np.ndarray:
    """u8 [z][y][x]: random balls of radius U{rmin..rmax} until `frac` of the grid is covered."""
    X, Y, Z = dims
    occ = np.zeros((Z, Y, X), np.uint8)
    target = int(frac * X * Y * Z)
    covered = 0
    offs = {}
    for r in range(rmin, rmax + 1):
        d = np.arange(-r, r + 1)
        dz, dy, dx = np.meshgrid(d, d, d, indexing="ij")
        keep = dx * dx + dy * dy + dz * dz <= r * r
        offs[r] = (dx[keep], dy[keep], dz[keep])
    while covered < target:
        r = int(rng.integers(rmin, rmax + 1))
        cx, cy, cz = (int(v) for v in rng.integers(0, (X, Y, Z)))
        dx, dy, dz = offs[r]
        x, y, z = cx + dx, cy + dy, cz + dz
        ok = (x >= 0) & (x < X) & (y >= 0) & (y < Y) & (z >= 0) & (z < Z)
        x, y, z = x[ok], y[ok], z[ok]
        covered += int((occ[z, y, x] == 0).sum())
        occ[z, y, x] = 1
    return occ


def field_microbench(seed: int = 42, dims=MICRO_DIMS):
    """(field [z][y][x][12] f32, occupancy [z][y][x] u8)."""
    X, Y, Z = dims
    rng = np.random.default_rng(seed)
    field = rng.random((Z, Y, X, 12), dtype=np.float32)
    f = (np.float32(0.5) + np.float32(0.5) * rng.random((Z, Y, X), dtype=np.float32)).astype(np.float32)
    field[..., 7] = (np.float32(2.0) * (np.float32(1.0) - f) / (f - np.float32(0.2))).astype(np.float32)
    occ = clustered_occupancy(dims, 0.05, rng)
    return field, occ


def cell_microbench(n: int = 1_000_000, seed: int = 42, dims=MICRO_DIMS) -> np.ndarray:
    """n cells (CELL_DTYPE) at unique random voxels with random rulesets."""
    X, Y, Z = dims
    rng = np.random.default_rng(seed + 1)
    flat = rng.choice(X * Y * Z, size=n, replace=False)
    z, rem = np.divmod(flat, X * Y)
    y, x = np.divmod(rem, X)
    c = np.zeros(n, marl.CELL_DTYPE)
    c["pos"] = np.stack([x, y, z], 1).astype(np.uint16)
    c["internal"] = rng.random((n, 16), dtype=np.float32)
    rs = c["ruleset"]
    rx = rs["reactions"]
    rx["substrate"] = rng.integers(0, 16, (n, 16))
    rx["product"] = rng.integers(0, 16, (n, 16))
    cat = rng.integers(0, 16, (n, 16))
    cat[rng.random((n, 16)) < 0.25] = 15
    rx["catalyst"] = cat
    rx["cofactor"] = 0xFF
    rx["k_m"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    rx["v_max"] = rng.lognormal(0.0, 1.0, (n, 16)).astype(np.float32)
    rx["k_cat"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    tp = rs["transport"]
    tp["uptake_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["secrete_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["ext_species"] = rng.integers(0, 12, (n, 8))
    tp["int_species"] = rng.integers(0, 16, (n, 8))
    ef = rs["effectors"]
    ef["threshold"] = rng.random((n, 8), dtype=np.float32)
    ef["rate"] = rng.random((n, 8), dtype=np.float32)
    ef["int_species"] = rng.integers(0, 16, (n, 8))
    ef["ext_species"] = rng.integers(0, 12, (n, 8))
    rs["fate"]["division_energy"] = 1e30  # no fate edits between phases
    rs["fate"]["death_energy"] = -1.0
    rs["fate"]["quiescence_energy"] = -1.0
    return c


def touched_voxels(cells: np.ndarray, dims) -> int:
    """Distinct empty in-grid face neighbours of the cells (the voxels the
    cell loop reads and writes)."""
    X, Y, Z = dims
    pos = cells["pos"].astype(np.int64)
    occ = np.zeros(X * Y * Z, bool)
    occ[(pos[:, 2] * Y + pos[:, 1]) * X + pos[:, 0]] = True
    seen = np.zeros(X * Y * Z, bool)
    for dx, dy, dz in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        x, y, z = pos[:, 0] + dx, pos[:, 1] + dy, pos[:, 2] + dz
        ok = (x >= 0) & (x < X) & (y >= 0) & (y < Y) & (z >= 0) & (z < Z)
        idx = (z[ok] * Y + y[ok]) * X + x[ok]
        seen[idx[~occ[idx]]] = True
    return int(seen.sum())
