"""TEST INFRASTRUCTURE ONLY — second, independent restatement of the reference
hot path in numpy float32, used to cross-check the C++ oracle (oracle.cpp).

* Diffusion follows the reference WGSL shader
  (crates/marl-gpu/src/shaders/field_diffuse.wgsl:55-95): `neighbor_or_center`
  returns the centre value for out-of-grid or occupied neighbours, occupied
  voxels are copied, `new = max(c + dt_sub*(d*lap - decay), 0)`.  It is
  vectorised over the whole grid, unlike the C++ oracle's per-voxel loops
  (crates/marl-field/src/field.rs:107-203).
* Boundary sources: crates/marl-field/src/field.rs:231-250.
* Light: crates/marl-field/src/light.rs:29-59, vectorised over columns.  exp is
  evaluated in float64 and rounded to float32 (glibc expf is within 0.502 ulp,
  so light agrees with the C++ oracle to a few ulp, not bit-for-bit).
* Cell tick and neighbour gather/scatter: crates/marl-cell/src/cell.rs:193-369,
  crates/marl-sim/src/spatial.rs:18-110, scalar np.float32 arithmetic.

Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
FACE = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))  # spatial.rs:8-15


def _fmax(a, b):
    return b if np.isnan(a) else (a if np.isnan(b) else (a if a > b else b))


def _fmin(a, b):
    return b if np.isnan(a) else (a if np.isnan(b) else (a if a < b else b))


def sources(field: np.ndarray, p) -> None:
    """field[z, y, x, s] in place (field.rs:231-250)."""
    cmax = f32(p.c_max)
    field[0, :, :, 1] = np.minimum(field[0, :, :, 1] + f32(p.source_rate_oxidant), cmax)
    field[0, :, :, 3] = np.minimum(field[0, :, :, 3] + f32(p.source_rate_carbon), cmax)
    field[-1, :, :, 2] = np.minimum(field[-1, :, :, 2] + f32(p.source_rate_reductant), cmax)


def diffusion_step(src: np.ndarray, occ: np.ndarray, p, dt_sub) -> np.ndarray:
    """One substep, WGSL formulation (field_diffuse.wgsl:72-95)."""
    Z, Y, X, S = src.shape
    occ = occ.astype(bool)
    c = src
    dt_sub = f32(dt_sub)
    structural = c[..., 7]
    niche = (f32(1.0) - f32(p.alpha_eps) * structural / (f32(p.k_eps) + structural))[..., None]

    def nb(axis: int, step: int) -> np.ndarray:
        # neighbor_or_center (field_diffuse.wgsl:40-53)
        shifted = np.roll(c, -step, axis=axis)
        occ_sh = np.roll(occ, -step, axis=axis)
        n = c.shape[axis]
        idx = np.arange(n)
        oob = (idx + step < 0) | (idx + step >= n)
        shape = [1, 1, 1]
        shape[axis] = n
        wall = oob.reshape(shape) | occ_sh
        return np.where(wall[..., None], c, shifted)

    xm, xp = nb(2, -1), nb(2, 1)
    ym, yp = nb(1, -1), nb(1, 1)
    zm, zp = nb(0, -1), nb(0, 1)
    lap = xm + xp + ym + yp + zm + zp - f32(6.0) * c
    d = np.array(list(p.d_voxel), np.float32) * niche
    decay = np.array(list(p.lambda_decay), np.float32) * c
    new = np.maximum(c + dt_sub * (d * lap - decay), f32(0.0))
    return np.where(occ[..., None], c, new).astype(np.float32)


def diffuse_tick(field: np.ndarray, occ: np.ndarray, p, substeps: int) -> np.ndarray:
    dt_sub = f32(p.dt) / f32(p.diffusion_substeps)
    f = field.astype(np.float32, copy=True)
    for _ in range(substeps):
        f = diffusion_step(f, occ, p, dt_sub)
    return f


def _exp32(v) -> np.ndarray:
    return np.exp(np.asarray(v, np.float64)).astype(np.float32)


def light(field: np.ndarray, occ: np.ndarray, p) -> np.ndarray:
    """LightField::update (light.rs:29-59), vectorised over (y, x) columns."""
    Z = field.shape[0]
    out = np.empty(field.shape[:3], np.float32)
    inten = np.full(field.shape[1:3], f32(p.surface_intensity), np.float32)
    cell_f = _exp32(-f32(p.cell_absorption))
    for z in range(Z):
        out[z] = inten
        inten = np.where(occ[z].astype(bool), inten * cell_f, inten).astype(np.float32)
        inten = (inten * _exp32(-f32(p.chemical_absorption) * field[z, :, :, 4])).astype(np.float32)
        inten = np.where(inten < f32(p.light_floor), f32(0.0), inten).astype(np.float32)
    return out


def cell_tick(cell, ext, light_value, p):
    """CellState::tick (cell.rs:193-369) on a CELL_DTYPE record; returns (cell, deltas, event)."""
    c = cell.copy()
    rs = c["ruleset"]
    x = [f32(v) for v in c["internal"]]
    ext = [f32(v) for v in ext]
    deltas = [f32(0.0)] * 12
    dt, cmax, thr = f32(p.dt), f32(p.c_max), f32(p.active_reaction_threshold)
    one = f32(1.0)
    for tp in rs["transport"]:  # cell.rs:223-238
        e, k = int(tp["ext_species"]), int(tp["int_species"])
        if e >= 12 or k >= 16:
            continue
        up = f32(tp["uptake_rate"]) * ext[e] / (one + ext[e])
        se = f32(tp["secrete_rate"]) * x[k] / (one + x[k])
        v = x[k] + (up - se) * dt
        if v < f32(0.0):
            v = f32(0.0)
        if v > cmax:
            v = cmax
        x[k] = v
        deltas[e] = deltas[e] + (se - up) * dt
    x[15] = f32(light_value)  # cell.rs:243
    eps = f32(np.finfo(np.float32).eps)
    for rx in rs["reactions"]:  # cell.rs:246-285
        vmax = f32(rx["v_max"])
        if abs(vmax) < thr or rx["substrate"] == rx["product"]:
            continue
        si, pi, ci, fi = int(rx["substrate"]), int(rx["product"]), int(rx["catalyst"]), int(rx["cofactor"])
        if si >= 16 or pi >= 16 or ci >= 16:
            continue
        s, cc = x[si], x[ci]
        st = s / (f32(rx["k_m"]) + s + eps)
        ct = f32(p.epsilon) + cc / (f32(rx["k_cat"]) + cc + eps)
        rate = vmax * st * ct
        if fi != 0xFF and fi < 16:
            cof = x[fi]
            rate = rate * (cof / (one + cof))
            x[fi] = x[fi] - _fmin(f32(0.5) * rate * dt, x[fi])
        flux = _fmin(rate * dt, x[si])
        x[si] = x[si] - flux
        x[pi] = _fmin(x[pi] + flux, cmax)
    if c["prep_remaining"] > 0:  # cell.rs:291-311
        evolved = _fmax(f32(rs["fate"]["division_prep_ticks"]), one)
        rush = _fmax(f32(p.base_division_prep) - evolved, f32(0.0))
        pm = f32(p.prep_maintenance_multiplier) + rush * f32(p.rush_penalty_rate)
    else:
        pm = one
    x[0] = x[0] * (one - f32(p.lambda_maintenance) * pm * dt)
    active = sum(1 for rx in rs["reactions"] if abs(f32(rx["v_max"])) > thr and rx["substrate"] != rx["product"])
    x[0] = _fmax(x[0] - f32(active) * f32(p.reaction_maintenance) * dt, f32(0.0))
    if not c["quiescent"]:  # cell.rs:314-329
        for ef in rs["effectors"]:
            k, e = int(ef["int_species"]), int(ef["ext_species"])
            if k >= 16 or e >= 12:
                continue
            if x[k] > f32(ef["threshold"]):
                amt = f32(ef["rate"]) * x[k] / (one + x[k]) * dt
                x[k] = _fmax(x[k] - amt, f32(0.0))
                deltas[e] = deltas[e] + amt
    energy = x[0]  # cell.rs:332-366
    c["age"] += 1
    eff_death = _fmax(f32(rs["fate"]["death_energy"]), f32(p.hard_death_floor))
    if energy < eff_death:
        c["prep_remaining"] = 0
        event = 2
    elif c["prep_remaining"] > 0:
        c["prep_remaining"] -= 1
        event = 1 if c["prep_remaining"] == 0 else 0
    elif energy > f32(rs["fate"]["division_energy"]):
        prep = _fmax(f32(rs["fate"]["division_prep_ticks"]), one)
        c["prep_remaining"] = 65535 if prep >= 65535 else int(prep)
        c["quiescent"] = 0
        event = 0
    elif energy < f32(rs["fate"]["quiescence_energy"]):
        c["quiescent"] = 1
        event = 3
    else:
        c["quiescent"] = 0
        event = 0
    c["internal"] = np.array(x, np.float32)
    return c, np.array(deltas, np.float32), event


def _empty_neighbors(pos, occupied: set, dims):
    X, Y, Z = dims
    out = []
    for dx, dy, dz in FACE:
        nx, ny, nz = int(pos[0]) + dx, int(pos[1]) + dy, int(pos[2]) + dz
        if 0 <= nx < X and 0 <= ny < Y and 0 <= nz < Z and (nx, ny, nz) not in occupied:
            out.append((nx, ny, nz))
    return out


def cell_phase(field: np.ndarray, light_arr: np.ndarray, cells: np.ndarray, dims, p):
    """Sequential cell loop (crates/marl-sim/src/lib.rs:206-217)."""
    f = field.astype(np.float32, copy=True)
    cells = cells.copy()
    occupied = {tuple(int(v) for v in c["pos"]) for c in cells}
    events = []
    for i in range(cells.size):
        pos = cells[i]["pos"]
        nb = _empty_neighbors(pos, occupied, dims)
        ext = np.zeros(12, np.float32)
        if nb:
            acc = [f32(0.0)] * 12
            for (x, y, z) in nb:
                for s in range(12):
                    acc[s] = acc[s] + f[z, y, x, s]
            n = f32(len(nb))
            ext = np.array([a / n for a in acc], np.float32)
        l = light_arr[int(pos[2]), int(pos[1]), int(pos[0])]
        c, deltas, ev = cell_tick(cells[i], ext, l, p)
        cells[i] = c
        events.append(ev)
        if nb:
            n = f32(len(nb))
            split = [d / n for d in deltas]
            for (x, y, z) in nb:
                for s in range(12):
                    f[z, y, x, s] = _fmax(f[z, y, x, s] + split[s], f32(0.0))
    return f, cells, np.array(events, np.int32)
