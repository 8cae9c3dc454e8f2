// TEST INFRASTRUCTURE ONLY.
//
// CPU oracle: a plain C++17 restatement of the MARL-OCHRE per-tick
// field-and-cell path, used ONLY as the checker by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
// library (libmarl_cuda.so) never links, loads or calls anything here.
//
// Every function cites the reference file:line it restates (paths inside the
// MARL-OCHRE workspace).  The reference is Rust and cannot be built here (no
// cargo/rustc, no crates.io cache), so it is restated, not compiled.
//
// Parity pin status:
//   * diffusion / boundary sources: pinned to the reference's own tests and
//     fixtures — crates/marl-field/src/field.rs:257-312 (deterministic fixture,
//     occupied-voxel-unchanged, finite and non-negative) and
//     crates/marl-gpu/tests/gpu_diffusion.rs:7-150 (wave fixture, 4 occupancy
//     patterns, substeps 1/2/10, max abs 1e-4) — and cross-checked bit-exactly
//     against an independent numpy restatement of the reference WGSL shader
//     (crates/marl-gpu/src/shaders/field_diffuse.wgsl:55-95), oracle/ref_numpy.py.
//   * light, cell tick, neighbour gather/scatter, fate/compaction, seeding:
//     parity unpinned — the reference has no tests and no golden vectors for
//     them and cannot be run here.  They are pinned only by the cited source,
//     by hand-checkable known-answer tests and by the numpy restatement.
//   * RNG-driven steps (seeding, division placement, mutation): the
//     reference's OS-seeded ChaCha12 stream cannot be reproduced; a documented
//     seeded generator stands in (oracle_rng.h).
//
// Float conventions: compiled with -O2 -ffp-contract=off and without
// fast-math, operations in the reference's source order, glibc expf for
// Rust's f32::exp.  Rust's f32::max/min are IEEE maxNum/minNum (std::fmax/
// std::fmin); f32::clamp keeps NaN (restated literally).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/marl_cuda.h"
#include "oracle_rng.h"

namespace oracle {

static int g_threads = 1;

struct Dims {
    int X, Y, Z;
    size_t V() const { return (size_t)X * Y * Z; }
    // crates/marl-field/src/field.rs:33-35 (Field::idx), voxel part
    size_t vox(int x, int y, int z) const { return ((size_t)z * Y + y) * X + x; }
};

template <typename T>
static inline T rclamp(T v, T lo, T hi) {  // Rust f32::clamp
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// crates/marl-config/src/lib.rs:108-168
void default_params(marl_sim_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->dx = 100.0e-6f;
    p->dt = 1.0f;
    p->diffusion_substeps = 10;
    const float d[12] = {0.0f, 1.5f, 1.0f, 1.2f, 0.8f, 0.5f, 0.5f, 0.1f, 0.3f, 0.3f, 0.3f, 0.3f};
    const float l[12] = {0.0f, 0.01f, 0.01f, 0.005f, 0.03f, 0.05f, 0.05f, 0.002f, 0.01f, 0.01f, 0.01f, 0.01f};
    for (int s = 0; s < 12; ++s) {
        p->d_voxel[s] = d[s];
        p->lambda_decay[s] = l[s];
    }
    p->source_rate_oxidant = 0.4f;
    p->source_rate_carbon = 0.15f;
    p->source_rate_reductant = 0.5f;
    p->epsilon = 0.001f;
    p->c_max = 10.0f;
    p->lambda_maintenance = 0.12f;
    p->hard_death_floor = 0.01f;
    p->reaction_maintenance = 0.003f;
    p->base_division_prep = 20.0f;
    p->prep_maintenance_multiplier = 2.0f;
    p->rush_penalty_rate = 0.05f;
    p->alpha_eps = 0.8f;
    p->k_eps = 2.0f;
    p->light_efficiency = 0.0f;
    p->surface_intensity = 1.0f;
    p->cell_absorption = 0.3f;
    p->chemical_absorption = 0.05f;
    p->light_floor = 1e-7f;
    p->mutation_stddev = 0.1f;
    p->structural_mutation_rate_mult = 0.1f;
    p->meta_mutation_rate = 0.01f;
    p->meta_mutation_clamp_low = 0.001f;
    p->meta_mutation_clamp_high = 0.5f;
    p->hill_exponent_clamp_low = 0.5f;
    p->hill_exponent_clamp_high = 8.0f;
    p->active_reaction_threshold = 1e-9f;
    p->seed_margin = 5;
    p->phototroph_z_lo = 0.0f;
    p->phototroph_z_hi = 3.0f;
    p->chemolithotroph_z_lo = 80.0f;
    p->chemolithotroph_z_hi = 130.0f;
    p->anaerobe_z_lo = 120.0f;
    p->anaerobe_z_hi = 180.0f;
    p->division_neighbor_distance = 2;
    p->boundary_prime_layers = 2;
    p->boundary_prime_oxidant = 0.5f;
    p->boundary_prime_carbon = 0.3f;
    p->boundary_prime_reductant = 0.5f;
    p->source_mode = MARL_SOURCES_ADDITIVE;
}

// ---------------------------------------------------------------- field ----

// crates/marl-field/src/field.rs:231-250 (Field::apply_boundary_sources).
// Dirichlet mode is an extension (pins the sourced planes to the
// boundary_prime_* values).
template <typename T>
void apply_boundary_sources(T* f, const Dims& g, const marl_sim_params& p) {
    const T cmax = (T)p.c_max;
    for (int y = 0; y < g.Y; ++y)
        for (int x = 0; x < g.X; ++x) {
            T* v = f + g.vox(x, y, 0) * 12;
            if (p.source_mode == MARL_SOURCES_DIRICHLET) {
                v[1] = (T)p.boundary_prime_oxidant;
                v[3] = (T)p.boundary_prime_carbon;
            } else {
                v[1] = std::fmin(v[1] + (T)p.source_rate_oxidant, cmax);
                v[3] = std::fmin(v[3] + (T)p.source_rate_carbon, cmax);
            }
        }
    for (int y = 0; y < g.Y; ++y)
        for (int x = 0; x < g.X; ++x) {
            T* v = f + g.vox(x, y, g.Z - 1) * 12;
            if (p.source_mode == MARL_SOURCES_DIRICHLET)
                v[2] = (T)p.boundary_prime_reductant;
            else
                v[2] = std::fmin(v[2] + (T)p.source_rate_reductant, cmax);
        }
}

// crates/marl-field/src/field.rs:107-198 (Field::diffusion_step_inner), one
// z-layer.  `occ` may be null (Field::diffuse_tick, field.rs:221-226).
template <typename T>
static void diffuse_layer(const T* src, T* dst, const uint8_t* occ, const Dims& g,
                          const marl_sim_params& p, T dt_sub, int z) {
    auto occ_at = [&](int x, int y, int zz) -> bool { return occ && occ[g.vox(x, y, zz)]; };
    for (int y = 0; y < g.Y; ++y)
        for (int x = 0; x < g.X; ++x) {
            const T* c0 = src + g.vox(x, y, z) * 12;
            T* out = dst + g.vox(x, y, z) * 12;
            if (occ_at(x, y, z)) {  // field.rs:130-136: copied unchanged
                for (int s = 0; s < 12; ++s) out[s] = c0[s];
                continue;
            }
            const T structural = c0[7];  // field.rs:141-143
            const T niche = (T)1.0 - (T)p.alpha_eps * structural / ((T)p.k_eps + structural);
            const bool wxm = x == 0 || occ_at(x - 1, y, z);
            const bool wxp = x >= g.X - 1 || occ_at(x + 1, y, z);
            const bool wym = y == 0 || occ_at(x, y - 1, z);
            const bool wyp = y >= g.Y - 1 || occ_at(x, y + 1, z);
            const bool wzm = z == 0 || occ_at(x, y, z - 1);
            const bool wzp = z >= g.Z - 1 || occ_at(x, y, z + 1);
            for (int s = 0; s < 12; ++s) {  // field.rs:152-195
                const T c = c0[s];
                const T d = (T)p.d_voxel[s] * niche;
                const T xm = wxm ? c : src[g.vox(x - 1, y, z) * 12 + s];
                const T xp = wxp ? c : src[g.vox(x + 1, y, z) * 12 + s];
                const T ym = wym ? c : src[g.vox(x, y - 1, z) * 12 + s];
                const T yp = wyp ? c : src[g.vox(x, y + 1, z) * 12 + s];
                const T zm = wzm ? c : src[g.vox(x, y, z - 1) * 12 + s];
                const T zp = wzp ? c : src[g.vox(x, y, z + 1) * 12 + s];
                const T lap = xm + xp + ym + yp + zm + zp - (T)6.0 * c;
                const T decay = (T)p.lambda_decay[s] * c;
                const T nc = c + dt_sub * (d * lap - decay);
                out[s] = std::fmax(nc, (T)0.0);
            }
        }
}

template <typename T>
void diffusion_step(const T* src, T* dst, const uint8_t* occ, const Dims& g, const marl_sim_params& p,
                    T dt_sub) {
#ifdef _OPENMP
    // Same split as the reference's rayon par_chunks_mut over z (field.rs:117-120);
    // layers are independent, so the result does not depend on the thread count.
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
#endif
    for (int z = 0; z < g.Z; ++z) diffuse_layer(src, dst, occ, g, p, dt_sub, z);
}

// crates/marl-field/src/field.rs:212-217 (Field::diffuse_tick_with_cells),
// in place with an internal scratch buffer (field.rs:200-202 swaps buffers).
template <typename T>
void diffuse_tick(T* f, const uint8_t* occ, const Dims& g, const marl_sim_params& p, uint32_t substeps) {
    // dt_sub is computed in f32 as the reference does (field.rs:213).
    const float dt_sub_f = p.dt / (float)p.diffusion_substeps;
    const T dt_sub = (T)dt_sub_f;
    std::vector<T> scratch(g.V() * 12);
    T* a = f;
    T* b = scratch.data();
    for (uint32_t i = 0; i < substeps; ++i) {
        diffusion_step(a, b, occ, g, p, dt_sub);
        std::swap(a, b);
    }
    if (a != f) std::memcpy(f, a, g.V() * 12 * sizeof(T));
}

// ---------------------------------------------------------------- light ----

template <typename T>
static inline T oexp(T v);
template <>
inline float oexp<float>(float v) {
    return expf(v);
}
template <>
inline double oexp<double>(double v) {
    return std::exp(v);
}

// crates/marl-field/src/light.rs:29-59 (LightField::update).  Occupancy
// stands for `cells.contains_key(&pos)`.
template <typename T>
void light_update(T* light, const T* field, const uint8_t* occ, const Dims& g, const marl_sim_params& p) {
    for (int y = 0; y < g.Y; ++y)
        for (int x = 0; x < g.X; ++x) {
            T intensity = (T)p.surface_intensity;
            for (int z = 0; z < g.Z; ++z) {
                const size_t v = g.vox(x, y, z);
                light[v] = intensity;
                if (occ[v]) intensity *= oexp<T>(-(T)p.cell_absorption);
                const T absorber = field[v * 12 + 4];
                intensity *= oexp<T>(-(T)p.chemical_absorption * absorber);
                if (intensity < (T)p.light_floor) intensity = (T)0.0;
            }
        }
}

// ----------------------------------------------------------------- cell ----

// crates/marl-cell/src/cell.rs:193-369 (CellState::tick), with internal state
// of type T.  Phase 1 (receptors, cell.rs:203-220) writes only `_activation`,
// which nothing reads, so it has no observable effect and is omitted.
// Returns the CellEvent; deltas receive the field deltas.
template <typename T>
int cell_tick(marl_cell& cell, T* internal, const T ext[12], T light, const marl_sim_params& sim,
              T deltas[12]) {
    const marl_ruleset& rs = cell.ruleset;
    for (int s = 0; s < 12; ++s) deltas[s] = (T)0.0;
    const T dt = (T)sim.dt;
    const T cmax = (T)sim.c_max;
    const T thr = (T)sim.active_reaction_threshold;

    // PHASE 2: transport (cell.rs:223-238)
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) {
        const marl_transport_params& tp = rs.transport[i];
        const int e = tp.ext_species, k = tp.int_species;
        if (e >= MARL_S_EXT || k >= MARL_M_INT) continue;
        const T uptake = (T)tp.uptake_rate * ext[e] / ((T)1.0 + ext[e]);
        const T secretion = (T)tp.secrete_rate * internal[k] / ((T)1.0 + internal[k]);
        internal[k] = rclamp(internal[k] + (uptake - secretion) * dt, (T)0.0, cmax);
        deltas[e] += (secretion - uptake) * dt;
    }
    // light slot (cell.rs:243)
    internal[MARL_M_INT - 1] = light;

    // PHASE 3: reactions (cell.rs:246-285)
    const T feps = (T)1.1920928955078125e-07f;  // f32::EPSILON
    for (int r = 0; r < MARL_R_MAX; ++r) {
        const marl_reaction& rx = rs.reactions[r];
        if (std::fabs((T)rx.v_max) < thr) continue;
        if (rx.substrate == rx.product) continue;
        const int si = rx.substrate, pi = rx.product, ci = rx.catalyst;
        if (si >= MARL_M_INT || pi >= MARL_M_INT || ci >= MARL_M_INT) continue;
        const T s = internal[si];
        const T c = internal[ci];
        const T substrate_term = s / ((T)rx.k_m + s + feps);
        const T catalyst_term = (T)sim.epsilon + c / ((T)rx.k_cat + c + feps);
        T rate = (T)rx.v_max * substrate_term * catalyst_term;
        if (rx.cofactor != MARL_NO_COFACTOR) {
            const int fi = rx.cofactor;
            if (fi < MARL_M_INT) {
                const T cof = internal[fi];
                rate *= cof / ((T)1.0 + cof);
                const T consumed = std::fmin((T)0.5 * rate * dt, internal[fi]);
                internal[fi] -= consumed;
            }
        }
        const T flux = std::fmin(rate * dt, internal[si]);
        internal[si] -= flux;
        internal[pi] = std::fmin(internal[pi] + flux, cmax);
    }

    // maintenance (cell.rs:291-311)
    T prep_mult;
    if (cell.prep_remaining > 0) {
        const T evolved = std::fmax((T)rs.fate.division_prep_ticks, (T)1.0);
        const T rush = std::fmax((T)sim.base_division_prep - evolved, (T)0.0);
        prep_mult = (T)sim.prep_maintenance_multiplier + rush * (T)sim.rush_penalty_rate;
    } else {
        prep_mult = (T)1.0;
    }
    internal[0] *= (T)1.0 - (T)sim.lambda_maintenance * prep_mult * dt;
    int active = 0;
    for (int r = 0; r < MARL_R_MAX; ++r) {
        const marl_reaction& rx = rs.reactions[r];
        if (std::fabs((T)rx.v_max) > thr && rx.substrate != rx.product) ++active;
    }
    internal[0] = std::fmax(internal[0] - (T)active * (T)sim.reaction_maintenance * dt, (T)0.0);

    // PHASE 4: effectors (cell.rs:314-329)
    if (!cell.quiescent) {
        for (int i = 0; i < MARL_S_EFFECTORS; ++i) {
            const marl_effector_params& ef = rs.effectors[i];
            const int k = ef.int_species, e = ef.ext_species;
            if (k >= MARL_M_INT || e >= MARL_S_EXT) continue;
            if (internal[k] > (T)ef.threshold) {
                const T amount = (T)ef.rate * internal[k] / ((T)1.0 + internal[k]) * dt;
                internal[k] = std::fmax(internal[k] - amount, (T)0.0);
                deltas[e] += amount;
            }
        }
    }

    // PHASE 5: fate (cell.rs:332-366)
    const T energy = internal[0];
    cell.age += 1;
    const T eff_death = std::fmax((T)rs.fate.death_energy, (T)sim.hard_death_floor);
    int event;
    if (energy < eff_death) {
        cell.prep_remaining = 0;
        event = MARL_EVENT_DEATH;
    } else if (cell.prep_remaining > 0) {
        cell.prep_remaining -= 1;
        event = cell.prep_remaining == 0 ? MARL_EVENT_DIVISION : MARL_EVENT_NONE;
    } else if (energy > (T)rs.fate.division_energy) {
        // `prep as u16`: Rust's saturating float->int cast.
        const float prep = std::fmax(rs.fate.division_prep_ticks, 1.0f);
        cell.prep_remaining = prep >= 65535.0f ? 65535 : (uint16_t)prep;
        cell.quiescent = 0;
        event = MARL_EVENT_NONE;
    } else if (energy < (T)rs.fate.quiescence_energy) {
        cell.quiescent = 1;
        event = MARL_EVENT_QUIESCENCE;
    } else {
        cell.quiescent = 0;
        event = MARL_EVENT_NONE;
    }
    return event;
}

// Phase 1 of CellState::tick (crates/marl-cell/src/cell.rs:206-220): the Hill
// activation of receptor i from the gathered species i.  The reference keeps
// the result in `_activation`, which nothing reads yet.
void receptor_activations(const marl_cell& cell, const float ext[12], const marl_sim_params& sim, float act[8]) {
    for (int i = 0; i < MARL_S_RECEPTORS; ++i) {
        act[i] = 0.0f;
        const marl_receptor_params& r = cell.ruleset.receptors[i];
        if (i < MARL_S_EXT && std::fabs(r.gain) > sim.active_reaction_threshold) {
            const float c = ext[i];
            const float k = std::fmax(r.k_half, 1e-6f);
            const float n = rclamp(r.n_hill, sim.hill_exponent_clamp_low, sim.hill_exponent_clamp_high);
            const float kn = powf(k, n);
            const float cn = powf(std::fmax(c, 0.0f), n);
            act[i] = r.gain * cn / (kn + cn + 1e-9f);
        }
    }
}

// crates/marl-cell/src/hgt.rs:7-27 (transfer_reaction): a random active
// reaction of the donor replaces the recipient's first inactive slot, or a
// random slot when every slot is active.
template <class R>
void transfer_reaction(const marl_ruleset& donor, marl_ruleset& recipient, R& rng) {
    int active[MARL_R_MAX];
    int na = 0;
    for (int i = 0; i < MARL_R_MAX; ++i)
        if (std::fabs(donor.reactions[i].v_max) > 1e-9f) active[na++] = i;
    if (na == 0) return;
    const int donor_idx = active[rng.range(0, (uint32_t)na)];
    const marl_reaction donated = donor.reactions[donor_idx];
    int target = -1;
    for (int i = 0; i < MARL_R_MAX && target < 0; ++i)
        if (std::fabs(recipient.reactions[i].v_max) < 1e-9f) target = i;
    if (target < 0) target = (int)rng.range(0, MARL_R_MAX);
    recipient.reactions[target] = donated;
}

// -------------------------------------------------------------- spatial ----

// crates/marl-sim/src/spatial.rs:8-15
static const int FACE[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// crates/marl-sim/src/spatial.rs:18-43 (empty_neighbors); `cmap` >= 0 marks
// an occupied voxel (cell_map.contains_key).
static int empty_neighbors(const uint16_t pos[3], const int32_t* cmap, const Dims& g, size_t out[6]) {
    int n = 0;
    for (int f = 0; f < 6; ++f) {
        const int nx = pos[0] + FACE[f][0], ny = pos[1] + FACE[f][1], nz = pos[2] + FACE[f][2];
        if (nx >= 0 && nx < g.X && ny >= 0 && ny < g.Y && nz >= 0 && nz < g.Z) {
            const size_t v = g.vox(nx, ny, nz);
            if (cmap[v] < 0) out[n++] = v;
        }
    }
    return n;
}

// crates/marl-sim/src/spatial.rs:56-77 (read_neighbor_environment)
template <typename T>
static void read_neighbor_environment(const uint16_t pos[3], const T* field, const int32_t* cmap,
                                      const Dims& g, T out[12]) {
    size_t nb[6];
    const int n = empty_neighbors(pos, cmap, g, nb);
    for (int s = 0; s < 12; ++s) out[s] = (T)0.0;
    if (n == 0) return;
    for (int k = 0; k < n; ++k)
        for (int s = 0; s < 12; ++s) out[s] += field[nb[k] * 12 + s];
    const T nf = (T)n;
    for (int s = 0; s < 12; ++s) out[s] /= nf;
}

// crates/marl-sim/src/spatial.rs:87-110 (apply_deltas_to_neighbors) with
// crates/marl-field/src/field.rs:57-62 (Field::apply_deltas)
template <typename T>
static void apply_deltas_to_neighbors(const uint16_t pos[3], T* field, const int32_t* cmap, const Dims& g,
                                      const T deltas[12]) {
    size_t nb[6];
    const int n = empty_neighbors(pos, cmap, g, nb);
    if (n == 0) return;
    const T nf = (T)n;
    T split[12];
    for (int s = 0; s < 12; ++s) split[s] = deltas[s] / nf;
    for (int k = 0; k < n; ++k)
        for (int s = 0; s < 12; ++s) {
            T& c = field[nb[k] * 12 + s];
            c = std::fmax(c + split[s], (T)0.0);
        }
}

// crates/marl-sim/src/spatial.rs:115-154 (find_empty_neighbor)
template <class R>
static bool find_empty_neighbor(const uint16_t pos[3], const int32_t* cmap, const Dims& g, R& rng,
                                const marl_sim_params& sim, uint16_t out[3]) {
    const int dist = (int)sim.division_neighbor_distance;
    uint16_t cand[6][3];
    int nc = 0;
    for (int f = 0; f < 6; ++f) {
        const int nx = pos[0] + FACE[f][0] * dist, ny = pos[1] + FACE[f][1] * dist,
                  nz = pos[2] + FACE[f][2] * dist;
        if (nx >= 0 && nx < g.X && ny >= 0 && ny < g.Y && nz >= 0 && nz < g.Z) {
            if (cmap[g.vox(nx, ny, nz)] < 0) {
                cand[nc][0] = (uint16_t)nx;
                cand[nc][1] = (uint16_t)ny;
                cand[nc][2] = (uint16_t)nz;
                ++nc;
            }
        }
    }
    if (nc > 0) {
        const uint32_t i = rng.range(0, (uint32_t)nc);
        std::memcpy(out, cand[i], sizeof(uint16_t) * 3);
        return true;
    }
    int na = 0;
    uint16_t adj[6][3];
    for (int f = 0; f < 6; ++f) {
        const int nx = pos[0] + FACE[f][0], ny = pos[1] + FACE[f][1], nz = pos[2] + FACE[f][2];
        if (nx >= 0 && nx < g.X && ny >= 0 && ny < g.Y && nz >= 0 && nz < g.Z && cmap[g.vox(nx, ny, nz)] < 0) {
            adj[na][0] = (uint16_t)nx;
            adj[na][1] = (uint16_t)ny;
            adj[na][2] = (uint16_t)nz;
            ++na;
        }
    }
    if (na == 0) return false;
    const uint32_t i = rng.range(0, (uint32_t)na);
    std::memcpy(out, adj[i], sizeof(uint16_t) * 3);
    return true;
}

// ------------------------------------------------------------- mutation ----

// crates/marl-cell/src/cell.rs:406-524 (Ruleset::mutate) over the stand-in RNG.
template <class R>
static void maybe_mutate(float& v, float rate, float stddev, R& rng) {
    if (rng.next_f32() < rate) {
        v += rng.normal(stddev);
        v = std::fmax(v, 0.0f);
    }
}

template <class R>
void mutate(marl_ruleset& rs, R& rng, const marl_sim_params& sim) {
    const float rate = rs.mutation_rate;
    const float sd = sim.mutation_stddev;
    const float smr = rate * sim.structural_mutation_rate_mult;
    for (auto& r : rs.receptors) {
        maybe_mutate(r.k_half, rate, sd, rng);
        maybe_mutate(r.n_hill, rate, sd, rng);
        r.n_hill = rclamp(r.n_hill, sim.hill_exponent_clamp_low, sim.hill_exponent_clamp_high);
        maybe_mutate(r.gain, rate, sd, rng);
    }
    for (auto& t : rs.transport) {
        maybe_mutate(t.uptake_rate, rate, sd, rng);
        maybe_mutate(t.secrete_rate, rate, sd, rng);
        if (rng.next_f32() < smr) t.ext_species = (uint8_t)rng.range(0, MARL_S_EXT);
        if (rng.next_f32() < smr) t.int_species = (uint8_t)rng.range(0, MARL_M_INT);
    }
    int active[MARL_R_MAX];
    int na = 0;
    for (int i = 0; i < MARL_R_MAX; ++i)
        if (std::fabs(rs.reactions[i].v_max) > sim.active_reaction_threshold) active[na++] = i;
    for (int i = 0; i < MARL_R_MAX; ++i) {
        marl_reaction& rx = rs.reactions[i];
        maybe_mutate(rx.k_m, rate, sd, rng);
        maybe_mutate(rx.v_max, rate, sd, rng);
        maybe_mutate(rx.k_cat, rate, sd, rng);
        for (int which = 0; which < 3; ++which) {
            if (rng.next_f32() < smr) {
                const uint32_t pick = rng.range(0, (uint32_t)std::max(na, 1));
                if ((int)pick < na) {
                    const int donor = active[pick];
                    if (donor != i) {
                        const marl_reaction& d = rs.reactions[donor];
                        if (which == 0) rx.substrate = d.substrate;
                        if (which == 1) rx.product = d.product;
                        if (which == 2) rx.catalyst = d.catalyst;
                    }
                } else {
                    const uint8_t v = (uint8_t)rng.range(0, MARL_M_INT);
                    if (which == 0) rx.substrate = v;
                    if (which == 1) rx.product = v;
                    if (which == 2) rx.catalyst = v;
                }
            }
        }
    }
    for (auto& e : rs.effectors) {
        maybe_mutate(e.threshold, rate, sd, rng);
        maybe_mutate(e.rate, rate, sd, rng);
    }
    maybe_mutate(rs.fate.division_energy, rate, sd, rng);
    maybe_mutate(rs.fate.death_energy, rate, sd, rng);
    maybe_mutate(rs.fate.quiescence_energy, rate, sd, rng);
    maybe_mutate(rs.fate.division_prep_ticks, rate, sd, rng);
    rs.fate.division_prep_ticks = std::fmax(rs.fate.division_prep_ticks, 1.0f);
    maybe_mutate(rs.hgt_propensity, rate, sd, rng);
    if (rng.next_f32() < sim.meta_mutation_rate) {
        rs.mutation_rate += rng.normal(sd) * sim.meta_mutation_rate;
        rs.mutation_rate = rclamp(rs.mutation_rate, sim.meta_mutation_clamp_low, sim.meta_mutation_clamp_high);
    }
}

// ------------------------------------------------------------- starters ----

// crates/marl-sim/src/starter_metabolisms.rs:6-42 (inactive defaults)
static void inactive_ruleset(marl_ruleset& rs) {
    std::memset(&rs, 0, sizeof(rs));
    for (auto& r : rs.receptors) r = {1.0f, 2.0f, 0.0f};
    for (auto& t : rs.transport) t = {0.0f, 0.0f, 0, 0, {0, 0}};
    for (auto& r : rs.reactions) r = {0, 0, 0, MARL_NO_COFACTOR, 1.0f, 0.0f, 0.5f};
    for (auto& e : rs.effectors) e = {10.0f, 0.0f, 0, 0, {0, 0}};
}

static marl_cell blank_cell(const uint16_t pos[3], uint64_t lineage, uint8_t starter) {
    marl_cell c;
    std::memset(&c, 0, sizeof(c));
    std::memcpy(c.pos, pos, sizeof(c.pos));
    c.lineage_id = lineage;
    c.starter_type = starter;
    inactive_ruleset(c.ruleset);
    c.ruleset.hgt_propensity = 0.1f;
    c.ruleset.mutation_rate = 0.05f;
    return c;
}

// crates/marl-sim/src/starter_metabolisms.rs:46-187
marl_cell make_phototroph(const uint16_t pos[3], uint64_t lineage) {
    marl_cell c = blank_cell(pos, lineage, 0);
    marl_ruleset& r = c.ruleset;
    r.receptors[2] = {0.3f, 2.0f, 1.0f};
    r.receptors[3] = {0.5f, 2.0f, 1.0f};
    r.transport[0] = {0.6f, 0.0f, 3, 3, {0, 0}};
    r.transport[1] = {0.0f, 0.6f, 1, 1, {0, 0}};
    r.transport[2] = {0.0f, 0.3f, 4, 4, {0, 0}};
    r.transport[3] = {0.1f, 0.0f, 2, 2, {0, 0}};
    r.reactions[0] = {3, 0, 15, MARL_NO_COFACTOR, 0.2f, 0.8f, 0.1f};
    r.reactions[1] = {3, 1, 15, MARL_NO_COFACTOR, 0.2f, 0.4f, 0.1f};
    r.reactions[2] = {3, 4, 0, MARL_NO_COFACTOR, 0.3f, 0.3f, 0.3f};
    r.reactions[3] = {3, 5, 6, MARL_NO_COFACTOR, 0.3f, 0.15f, 0.1f};
    r.reactions[4] = {3, 6, 5, MARL_NO_COFACTOR, 0.3f, 0.1f, 0.1f};
    r.effectors[0] = {0.5f, 0.8f, 1, 1, {0, 0}};
    r.effectors[1] = {1.0f, 0.2f, 4, 4, {0, 0}};
    r.fate = {1.2f, 0.05f, 0.15f, 20.0f};
    c.internal[0] = 0.3f;
    c.internal[3] = 0.3f;
    c.internal[5] = 0.05f;
    c.internal[6] = 0.05f;
    return c;
}

// crates/marl-sim/src/starter_metabolisms.rs:191-326
marl_cell make_chemolithotroph(const uint16_t pos[3], uint64_t lineage) {
    marl_cell c = blank_cell(pos, lineage, 1);
    marl_ruleset& r = c.ruleset;
    r.receptors[1] = {0.3f, 2.0f, 1.0f};
    r.receptors[2] = {0.3f, 2.0f, 1.0f};
    r.transport[0] = {0.7f, 0.0f, 1, 1, {0, 0}};
    r.transport[1] = {0.7f, 0.0f, 2, 2, {0, 0}};
    r.transport[2] = {0.2f, 0.0f, 3, 3, {0, 0}};
    r.transport[3] = {0.0f, 0.3f, 4, 4, {0, 0}};
    r.reactions[0] = {2, 0, 5, 1, 0.15f, 0.7f, 0.1f};
    r.reactions[1] = {1, 4, 0, MARL_NO_COFACTOR, 0.3f, 0.3f, 0.2f};
    r.reactions[2] = {7, 0, 5, MARL_NO_COFACTOR, 0.3f, 0.15f, 0.1f};
    r.reactions[3] = {3, 5, 6, MARL_NO_COFACTOR, 0.3f, 0.15f, 0.1f};
    r.reactions[4] = {3, 6, 5, MARL_NO_COFACTOR, 0.3f, 0.1f, 0.1f};
    r.effectors[0] = {0.5f, 0.3f, 4, 4, {0, 0}};
    r.fate = {1.0f, 0.05f, 0.12f, 20.0f};
    c.internal[0] = 1.5f;
    c.internal[1] = 0.5f;
    c.internal[2] = 0.5f;
    c.internal[5] = 0.05f;
    c.internal[6] = 0.05f;
    c.internal[7] = 5.0f;
    return c;
}

// crates/marl-sim/src/starter_metabolisms.rs:330-459
marl_cell make_anaerobe(const uint16_t pos[3], uint64_t lineage) {
    marl_cell c = blank_cell(pos, lineage, 2);
    marl_ruleset& r = c.ruleset;
    r.receptors[2] = {0.3f, 2.0f, 1.0f};
    r.transport[0] = {0.9f, 0.0f, 2, 2, {0, 0}};
    r.transport[1] = {0.3f, 0.0f, 3, 3, {0, 0}};
    r.transport[2] = {0.0f, 0.5f, 4, 4, {0, 0}};
    r.transport[3] = {0.1f, 0.0f, 1, 1, {0, 0}};
    r.reactions[0] = {2, 0, 5, MARL_NO_COFACTOR, 0.15f, 0.8f, 0.1f};
    r.reactions[1] = {3, 4, 0, MARL_NO_COFACTOR, 0.2f, 0.3f, 0.2f};
    r.reactions[2] = {0, 3, 1, MARL_NO_COFACTOR, 0.01f, 2.0f, 0.01f};
    r.reactions[3] = {3, 5, 6, MARL_NO_COFACTOR, 0.3f, 0.15f, 0.1f};
    r.reactions[4] = {3, 6, 5, MARL_NO_COFACTOR, 0.3f, 0.1f, 0.1f};
    r.effectors[0] = {0.5f, 0.5f, 4, 4, {0, 0}};
    r.fate = {0.8f, 0.05f, 0.1f, 20.0f};
    c.internal[0] = 0.5f;
    c.internal[2] = 0.7f;
    c.internal[5] = 0.05f;
    c.internal[6] = 0.05f;
    return c;
}

// ---------------------------------------------------------------- world ----

struct World {
    Dims g;
    marl_sim_params p;
    Rng rng;
    uint64_t seed;
    int fate_mode = 0;  // 0: one sequential stream (rng); 1: per-division streams keyed by (seed, tick, parent)
    std::vector<float> field, light;
    std::vector<int32_t> cmap;  // HashMap<[u16;3], usize> as a dense voxel map
    std::vector<marl_cell> cells;
    uint64_t total_div = 0, total_death = 0, tick_div = 0, tick_death = 0, tick = 0;

    World(int X, int Y, int Z, const marl_sim_params& sp, uint64_t seed)
        : g{X, Y, Z}, p(sp), rng(seed), seed(seed), field(g.V() * 12, 0.0f), light(g.V(), 0.0f), cmap(g.V(), -1) {}

    void rebuild_map() {
        std::fill(cmap.begin(), cmap.end(), -1);
        for (size_t i = 0; i < cells.size(); ++i)
            cmap[g.vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = (int32_t)i;
    }
    std::vector<uint8_t> occupancy() const {  // crates/marl-sim/src/lib.rs:174-179
        std::vector<uint8_t> occ(g.V(), 0);
        for (size_t v = 0; v < g.V(); ++v) occ[v] = cmap[v] >= 0;
        return occ;
    }

    // crates/marl-sim/src/seeding.rs:9-26
    void init_field_boundaries() {
        const int layers = (int)p.boundary_prime_layers;
        for (int y = 0; y < g.Y; ++y)
            for (int x = 0; x < g.X; ++x) {
                for (int z = 0; z < layers; ++z) {
                    field[g.vox(x, y, z) * 12 + 1] = p.boundary_prime_oxidant;
                    field[g.vox(x, y, z) * 12 + 3] = p.boundary_prime_carbon;
                }
                for (int z = g.Z - layers; z < g.Z; ++z) field[g.vox(x, y, z) * 12 + 2] = p.boundary_prime_reductant;
            }
    }

    // crates/marl-sim/src/seeding.rs:28-58
    void seed_cells(uint32_t count, uint16_t z_lo, uint16_t z_hi, marl_cell (*factory)(const uint16_t*, uint64_t)) {
        const uint32_t margin = p.seed_margin;
        uint32_t seeded = 0;
        for (uint32_t a = 0; a < count * 8; ++a) {
            if (seeded >= count) break;
            const uint16_t x = (uint16_t)rng.range(margin, (uint32_t)g.X - margin);
            const uint16_t y = (uint16_t)rng.range(margin, (uint32_t)g.Y - margin);
            const uint16_t z = (uint16_t)rng.range(z_lo, std::min<uint32_t>(z_hi, (uint32_t)g.Z));
            const uint16_t pos[3] = {x, y, z};
            const size_t v = g.vox(x, y, z);
            if (cmap[v] >= 0) continue;
            marl_cell c = factory(pos, rng.next_u64());
            cmap[v] = (int32_t)cells.size();
            cells.push_back(c);
            ++seeded;
        }
    }

    // crates/marl-sim/src/lib.rs:50-105 (Rust `as u16` truncates toward zero)
    void seed_default(uint32_t seed_count) {
        init_field_boundaries();
        const float z_scale = (float)g.Z / 200.0f;
        const uint16_t photo_lo = (uint16_t)(p.phototroph_z_lo * z_scale);
        const uint16_t photo_hi = (uint16_t)std::fmax(p.phototroph_z_hi * z_scale, (float)photo_lo + 1.0f);
        seed_cells(seed_count, photo_lo, photo_hi, make_phototroph);
        const uint16_t chemo_lo = (uint16_t)(p.chemolithotroph_z_lo * z_scale);
        const uint16_t chemo_hi = (uint16_t)std::fmax(p.chemolithotroph_z_hi * z_scale, (float)chemo_lo + 3.0f);
        seed_cells(seed_count, chemo_lo, chemo_hi, make_chemolithotroph);
        const uint16_t ana_lo = (uint16_t)(p.anaerobe_z_lo * z_scale);
        const uint16_t ana_hi = (uint16_t)std::fmax(p.anaerobe_z_hi * z_scale, (float)ana_lo + 3.0f);
        seed_cells(seed_count, ana_lo, ana_hi, make_anaerobe);
    }

    void sources() { apply_boundary_sources(field.data(), g, p); }
    void diffuse(uint32_t substeps) {
        const std::vector<uint8_t> occ = occupancy();
        diffuse_tick(field.data(), occ.data(), g, p, substeps);
    }
    void update_light() {
        const std::vector<uint8_t> occ = occupancy();
        light_update(light.data(), field.data(), occ.data(), g, p);
    }
    // crates/marl-sim/src/lib.rs:204-217 (sequential cell loop)
    void cell_phase(std::vector<int>& events) {
        events.resize(cells.size());
        for (size_t i = 0; i < cells.size(); ++i) {
            marl_cell& c = cells[i];
            float ext[12], deltas[12];
            read_neighbor_environment(c.pos, field.data(), cmap.data(), g, ext);
            const float l = light[g.vox(c.pos[0], c.pos[1], c.pos[2])];
            events[i] = cell_tick<float>(c, c.internal, ext, l, p, deltas);
            apply_deltas_to_neighbors(c.pos, field.data(), cmap.data(), g, deltas);
        }
    }
    // crates/marl-sim/src/lib.rs:219-277 (fate processing)
    void fate(const std::vector<int>& events) {
        tick_div = tick_death = 0;
        std::vector<marl_cell> births;
        std::vector<uint32_t> deaths;
        for (size_t i = 0; i < events.size(); ++i) {
            if (events[i] == MARL_EVENT_DIVISION) {
                uint16_t dpos[3];
                if (fate_mode == 1) {
                    FateRng r(seed, tick, (uint32_t)i);
                    if (find_empty_neighbor(cells[i].pos, cmap.data(), g, r, p, dpos)) {
                        marl_cell d = cells[i];
                        std::memcpy(d.pos, dpos, sizeof(dpos));
                        d.age = 0;
                        d.prep_remaining = 0;
                        d.lineage_id = r.next_u64();
                        for (int k = 0; k < MARL_M_INT; ++k) {
                            d.internal[k] *= 0.5f;
                            cells[i].internal[k] *= 0.5f;
                        }
                        mutate(d.ruleset, r, p);
                        births.push_back(d);
                        ++tick_div;
                    }
                } else if (find_empty_neighbor(cells[i].pos, cmap.data(), g, rng, p, dpos)) {
                    marl_cell d = cells[i];
                    std::memcpy(d.pos, dpos, sizeof(dpos));
                    d.age = 0;
                    d.prep_remaining = 0;
                    d.lineage_id = rng.next_u64();
                    for (int k = 0; k < MARL_M_INT; ++k) {
                        d.internal[k] *= 0.5f;
                        cells[i].internal[k] *= 0.5f;
                    }
                    mutate(d.ruleset, rng, p);
                    births.push_back(d);
                    ++tick_div;
                }
            } else if (events[i] == MARL_EVENT_DEATH) {
                deaths.push_back((uint32_t)i);
                ++tick_death;
            }
        }
        total_div += tick_div;
        total_death += tick_death;
        std::sort(deaths.begin(), deaths.end());
        deaths.erase(std::unique(deaths.begin(), deaths.end()), deaths.end());
        for (auto it = deaths.rbegin(); it != deaths.rend(); ++it) {
            const uint32_t i = *it;
            cmap[g.vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = -1;
            cells[i] = cells.back();
            cells.pop_back();
            if (i < cells.size()) cmap[g.vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = (int32_t)i;
        }
        for (auto& b : births) {
            const size_t v = g.vox(b.pos[0], b.pos[1], b.pos[2]);
            if (cmap[v] < 0) {
                cmap[v] = (int32_t)cells.size();
                cells.push_back(b);
            }
        }
    }
    // crates/marl-sim/src/lib.rs:160-277 (one iteration of the tick loop)
    void full_tick() {
        sources();
        diffuse(p.diffusion_substeps);
        update_light();
        std::vector<int> ev;
        cell_phase(ev);
        fate(ev);
        ++tick;
    }
};

}  // namespace oracle

// ================================================================ C API ====
using namespace oracle;

extern "C" {

void oracle_default_params(marl_sim_params* p) { default_params(p); }

// Layout of the shared ABI structs as the C compiler sees them:
// sizes of marl_sim_params, marl_ruleset, marl_cell, marl_change, then
// offsets of marl_cell.lineage_id, .internal, .ruleset and
// marl_ruleset.reactions, .effectors, .fate.
void oracle_struct_layout(uint64_t out[10]) {
    out[0] = sizeof(marl_sim_params);
    out[1] = sizeof(marl_ruleset);
    out[2] = sizeof(marl_cell);
    out[3] = sizeof(marl_change);
    out[4] = offsetof(marl_cell, lineage_id);
    out[5] = offsetof(marl_cell, internal);
    out[6] = offsetof(marl_cell, ruleset);
    out[7] = offsetof(marl_ruleset, reactions);
    out[8] = offsetof(marl_ruleset, effectors);
    out[9] = offsetof(marl_ruleset, fate);
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
    g_threads = n < 1 ? 1 : n;
#else
    (void)n;
    g_threads = 1;
#endif
}
int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_sources_f32(float* f, int X, int Y, int Z, const marl_sim_params* p) {
    apply_boundary_sources(f, Dims{X, Y, Z}, *p);
}
void oracle_diffuse_f32(float* f, const uint8_t* occ, int X, int Y, int Z, const marl_sim_params* p,
                        uint32_t substeps) {
    diffuse_tick(f, occ, Dims{X, Y, Z}, *p, substeps);
}
// FP64 instantiation: input in float, computed and returned in double.
void oracle_diffuse_f64(const float* in, double* out, const uint8_t* occ, int X, int Y, int Z,
                        const marl_sim_params* p, uint32_t substeps, int apply_sources) {
    const Dims g{X, Y, Z};
    for (size_t i = 0; i < g.V() * 12; ++i) out[i] = (double)in[i];
    if (apply_sources) apply_boundary_sources(out, g, *p);
    diffuse_tick(out, occ, g, *p, substeps);
}
void oracle_light_f32(float* light, const float* field, const uint8_t* occ, int X, int Y, int Z,
                      const marl_sim_params* p) {
    light_update(light, field, occ, Dims{X, Y, Z}, *p);
}
void oracle_light_f64(double* light, const float* field, const uint8_t* occ, int X, int Y, int Z,
                      const marl_sim_params* p) {
    const Dims g{X, Y, Z};
    std::vector<double> f(g.V() * 12);
    for (size_t i = 0; i < f.size(); ++i) f[i] = field[i];
    light_update(light, f.data(), occ, g, *p);
}
// One CellState::tick on a standalone cell; returns the event.
int oracle_cell_tick(marl_cell* cell, const float ext[12], float light, const marl_sim_params* p,
                     float deltas[12]) {
    return cell_tick<float>(*cell, cell->internal, ext, light, *p, deltas);
}

// The sequential cell loop on explicit state (field in/out, light, cells
// in/out), FP32; events_out gets one event per cell.
void oracle_cell_phase_f32(float* field, const float* light, marl_cell* cells, uint32_t n, int X, int Y, int Z,
                           const marl_sim_params* p, int32_t* events_out) {
    const Dims g{X, Y, Z};
    std::vector<int32_t> cmap(g.V(), -1);
    for (uint32_t i = 0; i < n; ++i) cmap[g.vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = (int32_t)i;
    for (uint32_t i = 0; i < n; ++i) {
        marl_cell& c = cells[i];
        float ext[12], deltas[12];
        read_neighbor_environment(c.pos, field, cmap.data(), g, ext);
        const float l = light[g.vox(c.pos[0], c.pos[1], c.pos[2])];
        const int ev = cell_tick<float>(c, c.internal, ext, l, *p, deltas);
        if (events_out) events_out[i] = ev;
        apply_deltas_to_neighbors(c.pos, field, cmap.data(), g, deltas);
    }
}
// The same loop, also returning each cell's receptor activations (phase 1,
// from the environment it gathered), act_out [n][8].
void oracle_cell_phase_act_f32(float* field, const float* light, marl_cell* cells, uint32_t n, int X, int Y, int Z,
                               const marl_sim_params* p, int32_t* events_out, float* act_out) {
    const Dims g{X, Y, Z};
    std::vector<int32_t> cmap(g.V(), -1);
    for (uint32_t i = 0; i < n; ++i) cmap[g.vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = (int32_t)i;
    for (uint32_t i = 0; i < n; ++i) {
        marl_cell& c = cells[i];
        float ext[12], deltas[12];
        read_neighbor_environment(c.pos, field, cmap.data(), g, ext);
        receptor_activations(c, ext, *p, act_out + (size_t)i * 8);
        const float l = light[g.vox(c.pos[0], c.pos[1], c.pos[2])];
        const int ev = cell_tick<float>(c, c.internal, ext, l, *p, deltas);
        if (events_out) events_out[i] = ev;
        apply_deltas_to_neighbors(c.pos, field, cmap.data(), g, deltas);
    }
}

// Horizontal gene transfer over pairs in order: pair k moves a reaction from
// cells[donor[k]] to cells[recipient[k]] with its own stream, FateRng keyed by
// (seed ^ kHgtSalt, tick, k).
void oracle_hgt(marl_cell* cells, uint32_t n, const uint32_t* donor, const uint32_t* recipient, uint32_t pairs,
                uint64_t seed, uint64_t tick) {
    for (uint32_t k = 0; k < pairs; ++k) {
        if (donor[k] >= n || recipient[k] >= n) continue;
        FateRng rng(seed ^ 0x4847545452414E53ull, tick, k);  // "HGTTRANS"
        transfer_reaction(cells[donor[k]].ruleset, cells[recipient[k]].ruleset, rng);
    }
}

// Same loop in FP64 (field, light and internals in double); internal_out is
// [n][16].  Cell fate flags are updated in `cells` as well.
void oracle_cell_phase_f64(double* field, const double* light, marl_cell* cells, uint32_t n, int X, int Y, int Z,
                           const marl_sim_params* p, double* internal_out) {
    const Dims g{X, Y, Z};
    std::vector<int32_t> cmap(g.V(), -1);
    for (uint32_t i = 0; i < n; ++i) cmap[g.vox(cells[i].pos[0], cells[i].pos[1], cells[i].pos[2])] = (int32_t)i;
    for (uint32_t i = 0; i < n; ++i) {
        marl_cell& c = cells[i];
        double in[16], ext[12], deltas[12];
        for (int k = 0; k < 16; ++k) in[k] = c.internal[k];
        read_neighbor_environment(c.pos, field, cmap.data(), g, ext);
        const double l = light[g.vox(c.pos[0], c.pos[1], c.pos[2])];
        cell_tick<double>(c, in, ext, l, *p, deltas);
        for (int k = 0; k < 16; ++k) internal_out[(size_t)i * 16 + k] = in[k];
        apply_deltas_to_neighbors(c.pos, field, cmap.data(), g, deltas);
    }
}

void oracle_mutate(marl_ruleset* rs, uint64_t rng_state[4], const marl_sim_params* p) {
    Rng r;
    std::memcpy(r.s, rng_state, sizeof(r.s));
    mutate(*rs, r, *p);
    std::memcpy(rng_state, r.s, sizeof(r.s));
}
void oracle_rng_seed(uint64_t seed, uint64_t state_out[4]) {
    Rng r(seed);
    std::memcpy(state_out, r.s, sizeof(r.s));
}
uint64_t oracle_rng_next_u64(uint64_t state[4]) {
    Rng r;
    std::memcpy(r.s, state, sizeof(r.s));
    const uint64_t v = r.next_u64();
    std::memcpy(state, r.s, sizeof(r.s));
    return v;
}
void oracle_make_starter(int kind, const uint16_t pos[3], uint64_t lineage, marl_cell* out) {
    *out = kind == 0 ? make_phototroph(pos, lineage) : kind == 1 ? make_chemolithotroph(pos, lineage)
                                                                 : make_anaerobe(pos, lineage);
}

// ---- world (stateful run-loop restatement) ----
void* oracle_world_create(int X, int Y, int Z, const marl_sim_params* p, uint64_t seed, uint32_t seed_count) {
    World* w = new World(X, Y, Z, *p, seed);
    w->seed_default(seed_count);
    return w;
}
void* oracle_world_create_empty(int X, int Y, int Z, const marl_sim_params* p, uint64_t seed) {
    return new World(X, Y, Z, *p, seed);
}
void oracle_world_destroy(void* w) { delete (World*)w; }
void oracle_world_set_field(void* w, const float* f) {
    World* W = (World*)w;
    std::memcpy(W->field.data(), f, W->field.size() * sizeof(float));
}
void oracle_world_get_field(void* w, float* f) {
    World* W = (World*)w;
    std::memcpy(f, W->field.data(), W->field.size() * sizeof(float));
}
void oracle_world_set_light(void* w, const float* l) {
    World* W = (World*)w;
    std::memcpy(W->light.data(), l, W->light.size() * sizeof(float));
}
void oracle_world_get_light(void* w, float* l) {
    World* W = (World*)w;
    std::memcpy(l, W->light.data(), W->light.size() * sizeof(float));
}
void oracle_world_set_cells(void* w, const marl_cell* c, uint32_t n) {
    World* W = (World*)w;
    W->cells.assign(c, c + n);
    W->rebuild_map();
}
uint32_t oracle_world_cell_count(void* w) { return (uint32_t)((World*)w)->cells.size(); }
uint32_t oracle_world_get_cells(void* w, marl_cell* out, uint32_t cap) {
    World* W = (World*)w;
    const uint32_t n = (uint32_t)std::min<size_t>(cap, W->cells.size());
    std::memcpy(out, W->cells.data(), n * sizeof(marl_cell));
    return (uint32_t)W->cells.size();
}
void oracle_world_get_occupancy(void* w, uint8_t* occ) {
    World* W = (World*)w;
    const std::vector<uint8_t> o = W->occupancy();
    std::memcpy(occ, o.data(), o.size());
}
void oracle_world_get_rng(void* w, uint64_t s[4]) { std::memcpy(s, ((World*)w)->rng.s, sizeof(uint64_t) * 4); }
void oracle_world_sources(void* w) { ((World*)w)->sources(); }
void oracle_world_diffuse(void* w, uint32_t substeps) { ((World*)w)->diffuse(substeps); }
void oracle_world_light(void* w) { ((World*)w)->update_light(); }
void oracle_world_cell_phase(void* w, int32_t* events_out) {
    World* W = (World*)w;
    std::vector<int> ev;
    W->cell_phase(ev);
    if (events_out)
        for (size_t i = 0; i < ev.size(); ++i) events_out[i] = ev[i];
}
void oracle_world_fate(void* w, const int32_t* events, uint32_t n) {
    std::vector<int> ev(events, events + n);
    ((World*)w)->fate(ev);
}
void oracle_world_tick(void* w, uint32_t ticks) {
    World* W = (World*)w;
    for (uint32_t t = 0; t < ticks; ++t) W->full_tick();
}
void oracle_world_set_fate_mode(void* w, int mode) { ((World*)w)->fate_mode = mode; }
void oracle_world_set_tick(void* w, uint64_t tick) { ((World*)w)->tick = tick; }
// Stream of device fate: `count` u64 draws, and `count` normals of a fresh
// stream with the same key.
void oracle_fate_stream(uint64_t seed, uint64_t tick, uint32_t parent, uint32_t count, float stddev, uint64_t* u64_out,
                        float* normal_out) {
    FateRng a(seed, tick, parent);
    for (uint32_t i = 0; i < count; ++i) u64_out[i] = a.next_u64();
    FateRng b(seed, tick, parent);
    for (uint32_t i = 0; i < count; ++i) normal_out[i] = b.normal(stddev);
}
void oracle_fate_log(const double* x, uint32_t n, double* out) {
    for (uint32_t i = 0; i < n; ++i) out[i] = fate_log(x[i]);
}
void oracle_world_stats(void* w, uint64_t out[6]) {
    World* W = (World*)w;
    out[0] = W->tick;
    out[1] = W->cells.size();
    out[2] = W->total_div;
    out[3] = W->total_death;
    out[4] = W->tick_div;
    out[5] = W->tick_death;
}

}  // extern "C"
