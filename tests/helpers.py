"""Seeded synthetic inputs shared by the tests and the benchmark.

The generators follow the workload descriptions of the cell-kinetics and
field microbenchmarks (random species in [0,1), random reaction wiring over
16 internal species, Vmax lognormal(0,1), Km and Kcat uniform in [0.01,1],
light catalysis on 25% of reactions, clustered occupancy blobs).
"""
from __future__ import annotations

import numpy as np

from marl_cuda import CELL_DTYPE


def random_field(dims, rng: np.random.Generator, hi: float = 1.0) -> np.ndarray:
    X, Y, Z = dims
    return (rng.random((Z, Y, X, 12), dtype=np.float32) * np.float32(hi)).astype(np.float32)


def random_rulesets(cells: np.ndarray, rng: np.random.Generator, cofactor_frac: float = 0.25) -> None:
    n = cells.size
    rs = cells["ruleset"]
    rs["receptors"]["k_half"] = rng.random((n, 8), dtype=np.float32)
    rs["receptors"]["n_hill"] = np.float32(2.0)
    rs["receptors"]["gain"] = rng.random((n, 8), dtype=np.float32)
    tp = rs["transport"]
    tp["uptake_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["secrete_rate"] = rng.random((n, 8), dtype=np.float32)
    tp["ext_species"] = rng.integers(0, 12, (n, 8))
    tp["int_species"] = rng.integers(0, 16, (n, 8))
    rx = rs["reactions"]
    rx["substrate"] = rng.integers(0, 16, (n, 16))
    rx["product"] = rng.integers(0, 16, (n, 16))
    cat = rng.integers(0, 16, (n, 16))
    cat[rng.random((n, 16)) < 0.25] = 15  # light-catalysed
    rx["catalyst"] = cat
    cof = np.full((n, 16), 0xFF, np.int64)
    m = rng.random((n, 16)) < cofactor_frac
    cof[m] = rng.integers(0, 16, m.sum())
    rx["cofactor"] = cof
    rx["k_m"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    rx["v_max"] = rng.lognormal(0.0, 1.0, (n, 16)).astype(np.float32)
    rx["k_cat"] = (0.01 + 0.99 * rng.random((n, 16))).astype(np.float32)
    ef = rs["effectors"]
    ef["threshold"] = rng.random((n, 8), dtype=np.float32)
    ef["rate"] = rng.random((n, 8), dtype=np.float32)
    ef["int_species"] = rng.integers(0, 16, (n, 8))
    ef["ext_species"] = rng.integers(0, 12, (n, 8))
    rs["fate"]["division_energy"] = (0.5 + rng.random(n)).astype(np.float32)
    rs["fate"]["death_energy"] = (0.05 * rng.random(n)).astype(np.float32)
    rs["fate"]["quiescence_energy"] = (0.2 * rng.random(n)).astype(np.float32)
    rs["fate"]["division_prep_ticks"] = rng.integers(1, 25, n).astype(np.float32)
    rs["hgt_propensity"] = np.float32(0.1)
    rs["mutation_rate"] = np.float32(0.05)


def random_cells(dims, n: int, rng: np.random.Generator, positions: np.ndarray | None = None,
                 cofactor_frac: float = 0.25) -> np.ndarray:
    """n cells at unique random voxels (or the given [n,3] x,y,z positions)."""
    X, Y, Z = dims
    if positions is None:
        flat = rng.choice(X * Y * Z, size=n, replace=False)
        z, rem = np.divmod(flat, X * Y)
        y, x = np.divmod(rem, X)
        positions = np.stack([x, y, z], axis=1)
    cells = np.zeros(len(positions), CELL_DTYPE)
    cells["pos"] = positions.astype(np.uint16)
    cells["internal"] = rng.random((len(positions), 16), dtype=np.float32)
    cells["quiescent"] = (rng.random(len(positions)) < 0.2).astype(np.uint8)
    cells["starter_type"] = rng.integers(0, 3, len(positions))
    cells["prep_remaining"] = np.where(rng.random(len(positions)) < 0.2, rng.integers(1, 4, len(positions)), 0)
    cells["age"] = rng.integers(0, 100, len(positions))
    cells["lineage_id"] = rng.integers(0, 2**63, len(positions), dtype=np.int64).astype(np.uint64)
    random_rulesets(cells, rng, cofactor_frac)
    return cells


def clustered_positions(dims, frac: float, rng: np.random.Generator, rmin: int = 2, rmax: int = 4) -> np.ndarray:
    """Occupied voxels as random balls of radius U{rmin..rmax} until `frac` of the grid is covered."""
    X, Y, Z = dims
    occ = np.zeros((Z, Y, X), bool)
    target = int(frac * X * Y * Z)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    while occ.sum() < target:
        r = rng.integers(rmin, rmax + 1)
        cx, cy, cz = rng.integers(0, X), rng.integers(0, Y), rng.integers(0, Z)
        occ |= (xx - cx) ** 2 + (yy - cy) ** 2 + (zz - cz) ** 2 <= r * r
    z, y, x = np.nonzero(occ)
    pos = np.stack([x, y, z], axis=1)
    return pos[rng.permutation(len(pos))]
