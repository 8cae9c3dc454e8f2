// Cell kernels: neighbour schedule, the cell update (gather -> tick -> scatter)
// in the reference's sequential order, ordered event compaction, and cell-table
// edits (halving, deaths, swap_remove moves, births).
//
// The reference updates cells one after another in Vec order and applies each
// cell's field deltas immediately (crates/marl-sim/src/lib.rs:206-217), so cell
// j reads the field as cells 0..j-1 left it.  Cell j reads and writes exactly
// the empty face-neighbour voxels N(j) (crates/marl-sim/src/spatial.rs:18-110);
// occupancy does not change during the loop.  Two cells therefore interact
// only through a shared empty voxel, and for every empty voxel v the cells
// touching it form a chain in index order.  The schedule kernel records, for
// every face f of cell j whose voxel v is empty, dep[f][j] = the largest cell
// index i < j that also touches v.  The update kernel hands out cells in
// ascending index order (warp tickets from an atomic counter) and a cell
// starts only after its <= 6 dependencies have published their `done` epoch.
// This reproduces the sequential result bit-for-bit while independent cells
// run in parallel.  Progress: a cell only waits for smaller indices, which
// were ticketed earlier by warps that are already resident; every wait is
// bounded and reports kErrTimeoutDeps on expiry.
//
// This file is compiled with -fmad=false; every expression keeps the
// reference's operation order (crates/marl-cell/src/cell.rs:193-369).
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include "common.cuh"
#include "internal.h"
#include "kernel_setup.h"
#include "mlp.h"
#include "table_ops.cuh"

namespace marl {

__constant__ int c_face[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

// ---------------------------------------------------------- schedule -----
// The empty-face bits of cell j at packed position P, and through each face
// f its dependency (the largest cell index below j touching that voxel, or
// -1), handed to put_dep(f, dep); returns the bits.
template <class PutDep>
__device__ __forceinline__ uint32_t schedule_of(const Grid g, const int32_t* __restrict__ cmap, const uint32_t P,
                                                const uint32_t j, PutDep put_dep) {
    const int x = pos_x(P), y = pos_y(P), z = pos_z(P);
    uint32_t nb = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int nx = x + c_face[f][0], ny = y + c_face[f][1], nz = z + c_face[f][2];
        int dep = -1;
        if (nx >= 0 && nx < g.X && ny >= 0 && ny < g.Y && nz >= 0 && nz < g.Z &&
            cmap[((size_t)nz * g.Y + ny) * g.X + nx] < 0) {
            nb |= 1u << f;
#pragma unroll
            for (int h = 0; h < 6; ++h) {
                const int ux = nx + c_face[h][0], uy = ny + c_face[h][1], uz = nz + c_face[h][2];
                if (ux >= 0 && ux < g.X && uy >= 0 && uy < g.Y && uz >= 0 && uz < g.Z) {
                    const int32_t i = cmap[((size_t)uz * g.Y + uy) * g.X + ux];
                    if (i >= 0 && (uint32_t)i < j && i > dep) dep = i;
                }
            }
        }
        put_dep(f, dep);
    }
    return nb;
}

__device__ __forceinline__ void schedule_cell(const CellTable& t, const Grid g, const int32_t* __restrict__ cmap,
                                              const uint32_t j) {
    t.nb[j] = schedule_of(g, cmap, t.pos[j], j, [&](int f, int32_t dep) { t.dep[(size_t)f * t.cap + j] = dep; });
}

// n_dev (nullable): device-resident cell count, which then replaces n.
__global__ void k_cell_schedule(CellTable t, uint32_t n, const uint32_t* __restrict__ n_dev, Grid g,
                                const int32_t* __restrict__ cmap) {
    if (n_dev) n = *n_dev;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        schedule_cell(t, g, cmap, j);
}

// Run of the batch that global cell index `gi` belongs to (runs are stored in
// ascending cell_base order).
__device__ __forceinline__ int find_run(const RunDesc* __restrict__ runs, int n_runs, uint32_t gi) {
    int lo = 0, hi = n_runs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (runs[mid].cell_base <= gi) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t batch_total(const RunDesc* __restrict__ runs, int n_runs) {
    return runs[n_runs - 1].cell_base + runs[n_runs - 1].n;
}

__global__ void k_cell_schedule_batch(const RunDesc* __restrict__ runs, int n_runs) {
    const uint32_t total = batch_total(runs, n_runs);
    for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < total; gi += gridDim.x * blockDim.x) {
        const int r = find_run(runs, n_runs, gi);
        const RunDesc& R = runs[r];
        schedule_cell(R.t, R.g, R.cmap, gi - R.cell_base);
    }
}

// ------------------------------------------------------------ update -----
constexpr int kTickThreads = 128;

// Per-thread staging, [item][thread] so that dynamic indices never cause bank
// conflicts: everything a cell's update reads from the cell table is copied in
// with cp.async (independent loads in flight together, no registers held).
struct CellScratch {
    uint4 rx[MARL_R_MAX][kTickThreads];
    float2 tp[MARL_S_TRANSPORTERS][kTickThreads];
    float2 ef[MARL_S_EFFECTORS][kTickThreads];
    uint4 idx[2][kTickThreads];  // transporter pairs, effector pairs
    float4 fate[kTickThreads];
    float x[MARL_M_INT][kTickThreads];
    float ext[MARL_S_EXT][kTickThreads];
    float del[MARL_S_EXT][kTickThreads];
    uint32_t hdr[10][kTickThreads];  // nb, pos, state, age, dep[0..5]
};
constexpr int kTickSmem = (int)sizeof(CellScratch);

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ float4 ld4(const float* p) { return __ldcg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void st4(float* p, float4 v) { __stcg(reinterpret_cast<float4*>(p), v); }

__device__ __forceinline__ float rclamp(float v, float lo, float hi) {  // Rust f32::clamp (keeps NaN)
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// The staged schedule and state words of a cell (no other cell of this tick
// writes them).
struct CellPre {
    uint32_t nb, pos, state, age;
};

__device__ __forceinline__ CellPre staged_pre(const CellScratch& S) {
    const int tid = threadIdx.x;
    return CellPre{S.hdr[0][tid], S.hdr[1][tid], S.hdr[2][tid], S.hdr[3][tid]};
}

__device__ __forceinline__ int32_t staged_dep(const CellScratch& S, int f) {
    return (int32_t)S.hdr[4 + f][threadIdx.x];
}

// What one lane needs to know about the run its cell belongs to.
struct CellRunView {
    const CellTable* t;
    Grid g;
    float* field;
    const float* light;
    uint32_t epoch;
    const SurrView* sv;  // surrogate modes only
    float* act;          // receptor activations [8][cap], or null
    const int32_t* cmap; // voxel -> cell map (for a schedule computed in the loop)
};

// Issues (and commits as one group) the asynchronous copies of cell j's table
// entries into the lane's staging slots; cp_async_wait_all() completes them.
// With schedule_here the empty-face bits and dependencies are computed from
// the cell map instead of read from the table (no schedule kernel ran).
__device__ __forceinline__ void stage_cell(const CellRunView& v, CellScratch& S, uint32_t j,
                                           bool schedule_here = false) {
    const int tid = threadIdx.x;
    const CellTable& t = *v.t;
    const size_t cap = t.cap;
#pragma unroll
    for (int r = 0; r < MARL_R_MAX; ++r) cp_async16(&S.rx[r][tid], &t.rx[r * cap + j]);
#pragma unroll
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) cp_async8(&S.tp[i][tid], &t.tp_rate[i * cap + j]);
#pragma unroll
    for (int i = 0; i < MARL_S_EFFECTORS; ++i) cp_async8(&S.ef[i][tid], &t.ef_par[i * cap + j]);
    cp_async16(&S.idx[0][tid], &t.tp_idx[j]);
    cp_async16(&S.idx[1][tid], &t.ef_idx[j]);
    cp_async16(&S.fate[tid], &t.fate[j]);
#pragma unroll
    for (int k = 0; k < MARL_M_INT; ++k) cp_async4(&S.x[k][tid], &t.internal[k * cap + j]);
    cp_async4(&S.hdr[1][tid], &t.pos[j]);
    cp_async4(&S.hdr[2][tid], &t.state[j]);
    cp_async4(&S.hdr[3][tid], &t.age[j]);
    if (schedule_here) {
        S.hdr[0][tid] = schedule_of(v.g, v.cmap, t.pos[j], j,
                                    [&](int f, int32_t dep) { S.hdr[4 + f][tid] = (uint32_t)dep; });
    } else {
        cp_async4(&S.hdr[0][tid], &t.nb[j]);
        // The schedule stores -1 for faces that are not empty in-grid voxels.
#pragma unroll
        for (int f = 0; f < 6; ++f) cp_async4(&S.hdr[4 + f][tid], &t.dep[(size_t)f * cap + j]);
    }
    cp_async_commit();
}

// Gather and transport of the staged cell (spatial.rs:56-77, cell.rs:223-243):
// the neighbour mean into S.ext, S.del zeroed then holding the transport
// deltas, S.x the internal state after transport with the light in slot 15.
// Returns the light at the cell's voxel.  Shared by the cell loop and the
// surrogate's pre-pass, so both produce the same bits from the same field.
__device__ __forceinline__ float gather_transport(const CellRunView& v, const CellConsts& c, CellScratch& S,
                                                  const CellPre& pre, float4 (&nv)[6][3]) {
    const int tid = threadIdx.x;
    const Grid g = v.g;
    const uint32_t nb = pre.nb;
    const uint32_t P = pre.pos;
    const int x = pos_x(P), y = pos_y(P), z = pos_z(P);
    const size_t vox = ((size_t)z * g.Y + y) * g.X + x;
    const long long off[6] = {1, -1, (long long)g.X, -(long long)g.X, (long long)g.X * g.Y,
                              -(long long)g.X * g.Y};
    const int n = __popc(nb);
    const float light = __ldg(v.light + vox);

    // Gather: mean of the empty face neighbours (spatial.rs:56-77), summed in
    // face order from 0.0.  Dividing by n = 1, 2 or 4 is done as an exact
    // multiplication (a power-of-two divisor gives the identical IEEE result).
    // All neighbour loads are issued before the first sum, so they are in
    // flight together.
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if ((nb >> f) & 1u) {
            const float* src = v.field + (size_t)((long long)vox + off[f]) * 12;
            nv[f][0] = ld4(src), nv[f][1] = ld4(src + 4), nv[f][2] = ld4(src + 8);
        }
    }
    float acc[12];
#pragma unroll
    for (int s = 0; s < 12; ++s) acc[s] = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!((nb >> f) & 1u)) continue;
        const float4 q0 = nv[f][0], q1 = nv[f][1], q2 = nv[f][2];
        const float vals[12] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w};
#pragma unroll
        for (int s = 0; s < 12; ++s) acc[s] = acc[s] + vals[s];
    }
    if (n == 2 || n == 4) {
        const float inv = n == 2 ? 0.5f : 0.25f;
#pragma unroll
        for (int s = 0; s < 12; ++s) acc[s] = acc[s] * inv;
    } else if (n > 1) {
        div12_small_n(acc, n);  // n = 3, 5 or 6
    }
#pragma unroll
    for (int s = 0; s < 12; ++s) S.ext[s][tid] = acc[s];

    // CellState::tick (cell.rs:193-369).  Phase 1 (receptors) only writes an
    // unused local and is omitted.
#pragma unroll
    for (int s = 0; s < 12; ++s) S.del[s][tid] = 0.0f;
    const float dt = c.dt;

    // Phase 2: transport (cell.rs:223-238).  Uptake depends only on the
    // gathered environment, so all eight are evaluated first; secretion
    // follows the internal state transporter by transporter.
    const uint4 tpi = S.idx[0][tid];
    const uint32_t tpw[4] = {tpi.x, tpi.y, tpi.z, tpi.w};
    float uptakes[MARL_S_TRANSPORTERS];
#pragma unroll
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) {
        const uint32_t e = (tpw[i >> 1] >> ((i & 1) * 16)) & 0xFFu;
        const float ev = e < MARL_S_EXT ? S.ext[e][tid] : 0.0f;
        uptakes[i] = div_rn(S.tp[i][tid].x * ev, 1.0f + ev);
    }
#pragma unroll
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) {
        const uint32_t pair = (tpw[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
        const uint32_t e = pair & 0xFF, k = pair >> 8;
        if (e >= MARL_S_EXT || k >= MARL_M_INT) continue;
        const float2 r = S.tp[i][tid];
        // Both operands of the transporter are read before either is written.
        const float xk = S.x[k][tid];
        const float de = S.del[e][tid];
        const float uptake = uptakes[i];
        const float secretion = div_rn(r.y * xk, 1.0f + xk);
        S.x[k][tid] = rclamp(xk + (uptake - secretion) * dt, 0.0f, c.c_max);
        S.del[e][tid] = de + (secretion - uptake) * dt;
    }
    S.x[MARL_M_INT - 1][tid] = light;  // cell.rs:243
    return light;
}

// Phase 1 of CellState::tick (cell.rs:206-220): receptor i's Hill activation
// from gathered species i, into act[i][j].  The reference computes it into an
// unused local; here it is an optional output.  Not inlined, so that the
// update's register allocation does not carry it when the output is off.
__device__ __noinline__ void receptor_activations(const CellConsts& c, const CellTable& t, uint32_t j,
                                                  const CellScratch& S, float* act) {
    const float* r = t.cold + (size_t)j * kColdFloats;  // receptors: k_half, n_hill, gain
#pragma unroll 1
    for (int i = 0; i < MARL_S_RECEPTORS; ++i) {
        float a = 0.0f;
        const float gain = r[3 * i + 2];
        if (fabsf(gain) > c.thr) {
            const float cc = S.ext[i][threadIdx.x];
            const float k = fmaxf(r[3 * i], 1e-6f);
            const float n = rclamp(r[3 * i + 1], c.hill_lo, c.hill_hi);
            const float kn = powf(k, n);
            const float cn = powf(fmaxf(cc, 0.0f), n);
            a = div_rn(gain * cn, kn + cn + 1e-9f);
        }
        act[(size_t)i * t.cap + j] = a;
    }
}

// Phase 3 of CellState::tick: the reactions, strictly in slot order
// (cell.rs:246-285), on S.x.  Returns the number of active reactions.
__device__ __forceinline__ int reactions(const CellConsts& c, CellScratch& S) {
    const int tid = threadIdx.x;
    const float dt = c.dt;
    const float feps = 1.1920928955078125e-07f;
    int active = 0;
    // The next reaction's record is loaded while the current one runs.
    uint4 qn = S.rx[0][tid];
#pragma unroll 4
    for (int r = 0; r < MARL_R_MAX; ++r) {
        const uint4 q = qn;
        if (r + 1 < MARL_R_MAX) qn = S.rx[r + 1][tid];
        const uint32_t si = q.x & 0xFF, pi = (q.x >> 8) & 0xFF, ci = (q.x >> 16) & 0xFF, fi = q.x >> 24;
        const float km = __uint_as_float(q.y), vmax = __uint_as_float(q.z), kcat = __uint_as_float(q.w);
        if (fabsf(vmax) > c.thr && si != pi) ++active;
        if (fabsf(vmax) < c.thr) continue;
        if (si == pi) continue;
        if (si >= MARL_M_INT || pi >= MARL_M_INT || ci >= MARL_M_INT) continue;
        const bool has_cof = fi != MARL_NO_COFACTOR && fi < MARL_M_INT;
        // The reaction's operands are read together before any is written;
        // its own writes are forwarded in registers (the cofactor's new value
        // is what a later read of the same species would see).
        const float s = S.x[si][tid];
        const float cc = S.x[ci][tid];
        const float p = S.x[pi][tid];
        const float cof = has_cof ? S.x[fi][tid] : 0.0f;
        const float substrate_term = div_rn(s, km + s + feps);
        const float catalyst_term = c.epsilon + div_rn(cc, kcat + cc + feps);
        float rate = vmax * substrate_term * catalyst_term;
        float s_now = s, p_now = p;
        if (has_cof) {
            rate *= div_rn(cof, 1.0f + cof);
            const float consumed = fminf(0.5f * rate * dt, cof);
            const float cof_left = cof - consumed;
            S.x[fi][tid] = cof_left;
            if (fi == si) s_now = cof_left;
            if (fi == pi) p_now = cof_left;
        }
        const float flux = fminf(rate * dt, s_now);
        S.x[si][tid] = s_now - flux;
        S.x[pi][tid] = fminf(p_now + flux, c.c_max);
    }
    return active;
}

// Active-reaction count alone (the maintenance term of cell.rs:291-311),
// for cells whose reaction phase the surrogate replaces.
__device__ __forceinline__ int active_reactions(const CellConsts& c, const CellScratch& S) {
    int active = 0;
#pragma unroll
    for (int r = 0; r < MARL_R_MAX; ++r) {
        const uint4 q = S.rx[r][threadIdx.x];
        const uint32_t si = q.x & 0xFF, pi = (q.x >> 8) & 0xFF;
        if (fabsf(__uint_as_float(q.z)) > c.thr && si != pi) ++active;
    }
    return active;
}

// One raw surrogate row from the staged cell after gather_transport:
// x_T[16], ext[12], light, then per reaction k_m, v_max, k_cat, cofactor flag.
template <class Put>
__device__ __forceinline__ void surrogate_features(const CellScratch& S, float light, Put put) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int k = 0; k < MARL_M_INT; ++k) put(k, S.x[k][tid]);
#pragma unroll
    for (int e = 0; e < MARL_S_EXT; ++e) put(16 + e, S.ext[e][tid]);
    put(28, light);
#pragma unroll
    for (int r = 0; r < MARL_R_MAX; ++r) {
        const uint4 q = S.rx[r][tid];
        put(29 + 4 * r, __uint_as_float(q.y));
        put(30 + 4 * r, __uint_as_float(q.z));
        put(31 + 4 * r, __uint_as_float(q.w));
        put(32 + 4 * r, (q.x >> 24) != MARL_NO_COFACTOR ? 1.0f : 0.0f);
    }
}

// Maintenance and effectors (phases 3b-4 of CellState::tick, cell.rs:291-329)
// on the reaction phase's output in S.x; effector secretions go to S.del.
__device__ __forceinline__ void maintenance_effectors(const CellConsts& c, CellScratch& S, const float4 fate,
                                                      uint32_t prep, uint32_t quiescent, int active) {
    const int tid = threadIdx.x;
    const float dt = c.dt;
    // Maintenance (cell.rs:291-311)
    float pm;
    if (prep > 0) {
        const float evolved = fmaxf(fate.w, 1.0f);
        const float rush = fmaxf(c.base_division_prep - evolved, 0.0f);
        pm = c.prep_maintenance_multiplier + rush * c.rush_penalty_rate;
    } else {
        pm = 1.0f;
    }
    float x0 = S.x[0][tid];
    x0 *= 1.0f - c.lambda_maintenance * pm * dt;
    x0 = fmaxf(x0 - (float)active * c.reaction_maintenance * dt, 0.0f);
    S.x[0][tid] = x0;

    // Effectors (cell.rs:314-329)
    if (!quiescent) {
        const uint4 efi = S.idx[1][tid];
        const uint32_t efw[4] = {efi.x, efi.y, efi.z, efi.w};
#pragma unroll
        for (int i = 0; i < MARL_S_EFFECTORS; ++i) {
            const uint32_t pair = (efw[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
            const uint32_t k = pair & 0xFF, e = pair >> 8;
            if (k >= MARL_M_INT || e >= MARL_S_EXT) continue;
            const float2 pr = S.ef[i][tid];
            const float xk = S.x[k][tid];
            const float de = S.del[e][tid];
            if (xk > pr.x) {
                const float amount = div_rn(pr.y * xk, 1.0f + xk) * dt;
                S.x[k][tid] = fmaxf(xk - amount, 0.0f);
                S.del[e][tid] = de + amount;
            }
        }
    }
}

// Gather -> tick -> scatter of cell j, after all its dependencies are done.
// MODE: kModePlain, kModeCapture (also writes the cell's surrogate training
// row), kModeGated / kModeTrusted (reaction phase from the surrogate where
// the pre-pass speculation holds; see SurrView).
template <int MODE>
__device__ void update_cell(const CellRunView& v, const CellConsts& c, CellScratch& S, uint32_t j) {
    const int tid = threadIdx.x;
    const CellTable& t = *v.t;
    const CellPre pre = staged_pre(S);
    const Grid g = v.g;
    const uint32_t nb = pre.nb;
    const uint32_t P = pre.pos;
    const int x = pos_x(P), y = pos_y(P), z = pos_z(P);
    const size_t vox = ((size_t)z * g.Y + y) * g.X + x;
    const long long off[6] = {1, -1, (long long)g.X, -(long long)g.X, (long long)g.X * g.Y,
                              -(long long)g.X * g.Y};
    const int n = __popc(nb);
    const uint32_t st = pre.state;
    uint32_t prep = st & 0xFFFFu;
    uint32_t quiescent = (st >> 16) & 1u;
    const float4 fate = S.fate[tid];

    // The gathered neighbour values are also the scatter's starting values:
    // no other cell touches N(j) while this cell holds it.
    float4 nv[6][3];
    const float light = gather_transport(v, c, S, pre, nv);
    if (v.act) receptor_activations(c, t, j, S, v.act);

    int active;
    bool finished = false;  // maintenance and effectors already applied
    if constexpr (MODE == kModePlain) {
        active = reactions(c, S);
    } else if constexpr (MODE == kModeCapture) {
        const SurrView& sv = *v.sv;
        const bool cap_row = j < sv.raw_rows;
        float* row = sv.raw + (size_t)j * MARL_SURR_RAW_STRIDE;
        if (cap_row) surrogate_features(S, light, [&](int f, float val) { row[f] = val; });
        active = reactions(c, S);
        if (cap_row) {
#pragma unroll
            for (int k = 0; k < MARL_M_INT; ++k) row[MARL_SURR_FEATURES + k] = S.x[k][tid] - row[k];
        }
    } else {
        const SurrView& sv = *v.sv;
        const size_t ld = sv.ld;
        const size_t row = sv.row0 + j;
        bool spec = true;
#pragma unroll
        for (int k = 0; k < MARL_M_INT; ++k)
            spec = spec && __float_as_uint(S.x[k][tid]) == __float_as_uint(sv.xt[k * ld + row]);
        uint8_t status = kSurrNotSpeculated;
        float err = 0.0f;
        if (MODE == kModeTrusted && spec) {
            active = active_reactions(c, S);
#pragma unroll
            for (int k = 0; k < MARL_M_INT; ++k)
                S.x[k][tid] = fminf(fmaxf(S.x[k][tid] + sv.pred[k * ld + row], 0.0f), c.c_max);
            status = kSurrAccepted;
        } else {
            active = reactions(c, S);
            if (MODE == kModeGated && spec) {
                // The plain kernel judges the state the cell keeps: maintenance
                // and effectors run on the plain reaction output and on the
                // predicted one, and the prediction is kept only when the two
                // final states agree within tol (normwise relative error over
                // the 16 species).  Its effector secretions go with it.
                float del_t[MARL_S_EXT], xp[MARL_M_INT], dp[MARL_S_EXT];
#pragma unroll
                for (int e = 0; e < MARL_S_EXT; ++e) del_t[e] = S.del[e][tid];
                maintenance_effectors(c, S, fate, prep, quiescent, active);
#pragma unroll
                for (int k = 0; k < MARL_M_INT; ++k) {
                    xp[k] = S.x[k][tid];
                    S.x[k][tid] = fminf(fmaxf(sv.xt[k * ld + row] + sv.pred[k * ld + row], 0.0f), c.c_max);
                }
#pragma unroll
                for (int e = 0; e < MARL_S_EXT; ++e) {
                    dp[e] = S.del[e][tid];
                    S.del[e][tid] = del_t[e];
                }
                maintenance_effectors(c, S, fate, prep, quiescent, active);
                float num = 0.0f, den = 0.0f;
#pragma unroll
                for (int k = 0; k < MARL_M_INT; ++k) {
                    num = fmaxf(num, fabsf(S.x[k][tid] - xp[k]));
                    den = fmaxf(den, fabsf(xp[k]));
                }
                err = num / fmaxf(den, 1e-6f);
                if (err <= sv.tol) {
                    status = kSurrAccepted;
                } else {
#pragma unroll
                    for (int k = 0; k < MARL_M_INT; ++k) S.x[k][tid] = xp[k];
#pragma unroll
                    for (int e = 0; e < MARL_S_EXT; ++e) S.del[e][tid] = dp[e];
                    status = kSurrRejected;
                }
                finished = true;
            }
        }
        sv.status[row] = status;
        sv.err[row] = err;
    }
    if (!finished) maintenance_effectors(c, S, fate, prep, quiescent, active);

    // Phase 5: fate (cell.rs:332-366)
    const float energy = S.x[0][tid];
    const float eff_death = fmaxf(fate.y, c.hard_death_floor);
    uint8_t event;
    if (energy < eff_death) {
        prep = 0;
        event = MARL_EVENT_DEATH;
    } else if (prep > 0) {
        prep -= 1;
        event = prep == 0 ? MARL_EVENT_DIVISION : MARL_EVENT_NONE;
    } else if (energy > fate.x) {
        const float pt = fmaxf(fate.w, 1.0f);  // `as u16` saturates
        prep = pt >= 65535.0f ? 65535u : (uint32_t)pt;
        quiescent = 0;
        event = MARL_EVENT_NONE;
    } else if (energy < fate.z) {
        quiescent = 1;
        event = MARL_EVENT_QUIESCENCE;
    } else {
        quiescent = 0;
        event = MARL_EVENT_NONE;
    }

    // Scatter: split deltas over the same neighbours, clamp after each add
    // (spatial.rs:87-110, field.rs:57-62).
    if (n > 0) {
        float split[12];
        if (n == 1 || n == 2 || n == 4) {
            const float inv = n == 1 ? 1.0f : (n == 2 ? 0.5f : 0.25f);
#pragma unroll
            for (int s = 0; s < 12; ++s) split[s] = S.del[s][tid] * inv;
        } else {
#pragma unroll
            for (int s = 0; s < 12; ++s) split[s] = S.del[s][tid];
            div12_small_n(split, n);  // n = 3, 5 or 6
        }
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (!((nb >> f) & 1u)) continue;
            float* dst = v.field + (size_t)((long long)vox + off[f]) * 12;
            float4 q0 = nv[f][0], q1 = nv[f][1], q2 = nv[f][2];
            q0 = make_float4(fmaxf(q0.x + split[0], 0.0f), fmaxf(q0.y + split[1], 0.0f), fmaxf(q0.z + split[2], 0.0f),
                             fmaxf(q0.w + split[3], 0.0f));
            q1 = make_float4(fmaxf(q1.x + split[4], 0.0f), fmaxf(q1.y + split[5], 0.0f), fmaxf(q1.z + split[6], 0.0f),
                             fmaxf(q1.w + split[7], 0.0f));
            q2 = make_float4(fmaxf(q2.x + split[8], 0.0f), fmaxf(q2.y + split[9], 0.0f),
                             fmaxf(q2.z + split[10], 0.0f), fmaxf(q2.w + split[11], 0.0f));
            st4(dst, q0);
            st4(dst + 4, q1);
            st4(dst + 8, q2);
        }
    }
    // Publish: the scatter's writes are visible before the done flag (release).
    // Only later kernels read the cell's own state, so it is stored after.
    st_release_u32(&t.done[j], v.epoch);
    t.age[j] = pre.age + 1;
    t.state[j] = (st & 0xFF000000u) | (quiescent << 16) | prep;
    t.events[j] = event;
#pragma unroll
    for (int k = 0; k < MARL_M_INT; ++k) t.internal[(size_t)k * t.cap + j] = S.x[k][tid];
}

// The ticket loops shared by the single-run and the batched kernel.  `resolve`
// maps a ticket (global cell index) to the lane's run view and local index.
//
// Warp tickets: each warp takes `lanes` consecutive cells, stages them, and
// updates each as soon as its dependencies are done; it takes the next ticket
// when all of them are finished.  Used when every cell gets a lane at once
// (the grid's lanes cover the cells), where it is the shortest path.
template <int MODE, class Resolve>
__device__ __forceinline__ void cell_tick_loop_tickets(CellScratch& S, const CellConsts& c, uint32_t total,
                                                       uint32_t* ticket, uint32_t* err, uint32_t lanes,
                                                       Resolve resolve) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(ticket, lanes);
        base = __shfl_sync(FULL, base, 0);
        if (base >= total) break;
        const uint32_t gi = base + lane;
        bool pending = (uint32_t)lane < lanes && gi < total;
        CellRunView v{};
        uint32_t j = 0;
        if (pending) {
            resolve(gi, v, j);
            stage_cell(v, S, j, c.schedule_here != 0);
        }
        cp_async_wait_all();
        // Dependencies not yet seen finished (bit f: face f).  A poll loads
        // them with relaxed loads, all in flight together; once every one has
        // been seen, one acquire fence orders the update after the writers.
        uint32_t remaining = 0;
#pragma unroll
        for (int f = 0; f < 6; ++f) remaining |= (pending && staged_dep(S, f) >= 0 ? 1u : 0u) << f;
        uint32_t spins = 0;
        while (__any_sync(FULL, pending)) {
            if (pending) {
                const CellTable& t = *v.t;
                uint32_t seen[6];
#pragma unroll
                for (int f = 0; f < 6; ++f)
                    seen[f] = ((remaining >> f) & 1u) ? ld_relaxed_u32(&t.done[staged_dep(S, f)]) : 0u;
#pragma unroll
                for (int f = 0; f < 6; ++f)
                    if (((remaining >> f) & 1u) && seen[f] == v.epoch) remaining &= ~(1u << f);
                if (remaining == 0) {
                    fence_acquire_gpu();
                    update_cell<MODE>(v, c, S, j);  // publishes done[j] itself
                    pending = false;
                }
            }
            if (__any_sync(FULL, pending)) {
                if (++spins > c.wait_limit) {
                    if (pending) {
                        const CellTable& t = *v.t;
                        atomicOr(err, kErrTimeoutDeps);
                        t.events[j] = MARL_EVENT_NONE;
                        st_release_u32(&t.done[j], v.epoch);
                        pending = false;
                    }
                } else {
                    __nanosleep(64);
                }
            }
        }
    }
}

// Lane refill: each warp keeps up to `lanes` cells in flight, one per lane,
// and works in rounds: poll the dependencies of its staged cells, update the
// ready ones together, then hand every lane that is free the next index from
// the ticket counter (in lane order, so indices still go out in ascending
// order) and stage its cell.  A cell whose dependency is still running holds only its
// own lane; the other lanes move on to new cells.  Staging writes only shared
// memory (cp.async), and its copies are awaited at the start of the next
// round, so an update never waits on another lane's loads.  The ticket request
// is sent before the updates and its reply is read after them.
template <int MODE, class Resolve>
__device__ __forceinline__ void cell_tick_loop_refill(CellScratch& S, const CellConsts& c, uint32_t total,
                                                      uint32_t* ticket, uint32_t* err, uint32_t lanes,
                                                      Resolve resolve) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const bool usable = (uint32_t)lane < lanes;
    constexpr uint32_t kUnscanned = 1u << 6;  // dependencies of a fresh cell not yet read
    bool pending = false, more = true;
    uint32_t gi = 0, remaining = 0, spins = 0;
    for (;;) {
        cp_async_wait_all();  // the previous round's staging
        bool ready = false;
        CellRunView v{};
        uint32_t j = 0;
        if (pending) {
            resolve(gi, v, j);
            if (remaining & kUnscanned) {
                remaining = 0;
#pragma unroll
                for (int f = 0; f < 6; ++f) remaining |= (staged_dep(S, f) >= 0 ? 1u : 0u) << f;
            }
            // The remaining flags, loaded relaxed and all in flight together;
            // once every one has been seen, one acquire fence orders the
            // update after the writers.
            const CellTable& t = *v.t;
            uint32_t seen[6];
#pragma unroll
            for (int f = 0; f < 6; ++f)
                seen[f] = ((remaining >> f) & 1u) ? ld_relaxed_u32(&t.done[staged_dep(S, f)]) : 0u;
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if (((remaining >> f) & 1u) && seen[f] == v.epoch) remaining &= ~(1u << f);
            ready = remaining == 0;
        }
        const unsigned freed = __ballot_sync(FULL, usable && (!pending || ready));
        uint32_t base = 0;
        if (more && freed && lane == 0) base = atomicAdd(ticket, (uint32_t)__popc(freed));
        if (ready) {
            fence_acquire_gpu();
            update_cell<MODE>(v, c, S, j);  // publishes done[j] itself
            pending = false;
        } else if (pending && ++spins > c.wait_limit) {
            const CellTable& t = *v.t;
            atomicOr(err, kErrTimeoutDeps);
            t.events[j] = MARL_EVENT_NONE;
            st_release_u32(&t.done[j], v.epoch);
            pending = false;
        }
        if (more && freed) {
            base = __shfl_sync(FULL, base, 0);
            if (base >= total) {
                more = false;
            } else if ((freed >> lane) & 1u) {
                const uint32_t next = base + (uint32_t)__popc(freed & ((1u << lane) - 1u));
                if (next < total) {
                    gi = next;
                    resolve(gi, v, j);
                    stage_cell(v, S, j, c.schedule_here != 0);
                    pending = true;
                    spins = 0;
                    remaining = kUnscanned;
                }
            }
        }
        if (!__any_sync(FULL, pending)) break;
        // Back off only when no lane of the warp made progress this round.
        if (!__any_sync(FULL, ready)) __nanosleep(64);
    }
}

// Warp tickets when the grid's lanes cover every cell, lane refill otherwise
// (the choice is uniform over the grid: it depends only on the cell count).
template <int MODE, class Resolve>
__device__ __forceinline__ void cell_tick_loop(CellScratch& S, const CellConsts& c, uint32_t total, uint32_t* ticket,
                                               uint32_t* err, uint32_t lanes, Resolve resolve) {
    const uint64_t grid_lanes = (uint64_t)gridDim.x * (kTickThreads / 32) * lanes;
    if (total <= grid_lanes)
        cell_tick_loop_tickets<MODE>(S, c, total, ticket, err, lanes, resolve);
    else
        cell_tick_loop_refill<MODE>(S, c, total, ticket, err, lanes, resolve);
}

template <int MODE>
__global__ void __launch_bounds__(kTickThreads) k_cell_tick(const __grid_constant__ CellLaunch a) {
    extern __shared__ __align__(16) unsigned char tick_smem[];
    CellScratch& S = *reinterpret_cast<CellScratch*>(tick_smem);
    const uint32_t total = a.n_dev ? *a.n_dev : a.n;
    cell_tick_loop<MODE>(S, a.k, total, a.ticket, a.err, a.lanes, [&](uint32_t gi, CellRunView& v, uint32_t& j) {
        v = CellRunView{&a.t, a.g, a.field, a.light, a.epoch, &a.sv, a.act, a.cmap};
        j = gi;
    });
}

// One cell of the surrogate pre-pass: gather and transport of cell j from the
// current field, its post-transport state into row `row` of xt [16][ld], and
// its standardised BF16 features into row `row` of X [.][128].
__device__ __forceinline__ void prepass_cell(const CellRunView& v, const CellConsts& c, CellScratch& S, uint32_t j,
                                             uint32_t row, size_t ld, const float* __restrict__ norm,
                                             float* __restrict__ xt, __nv_bfloat16* __restrict__ X) {
    stage_cell(v, S, j);
    cp_async_wait_all();
    const CellPre pre = staged_pre(S);
    float4 nv[6][3];
    const float light = gather_transport(v, c, S, pre, nv);
#pragma unroll
    for (int k = 0; k < MARL_M_INT; ++k) xt[k * ld + row] = S.x[k][threadIdx.x];
    float f[mlp::kInPad];
#pragma unroll
    for (int i = mlp::kIn; i < mlp::kInPad; ++i) f[i] = 0.0f;
    surrogate_features(S, light, [&](int i, float val) {
        f[i] = (mlp::feature_transform(i, val) - norm[i]) / norm[mlp::kIn + i];
    });
    uint4* dst = reinterpret_cast<uint4*>(X + (size_t)row * mlp::kInPad);
#pragma unroll
    for (int q = 0; q < mlp::kInPad / 8; ++q) {
        __nv_bfloat162 h0 = __floats2bfloat162_rn(f[8 * q], f[8 * q + 1]);
        __nv_bfloat162 h1 = __floats2bfloat162_rn(f[8 * q + 2], f[8 * q + 3]);
        __nv_bfloat162 h2 = __floats2bfloat162_rn(f[8 * q + 4], f[8 * q + 5]);
        __nv_bfloat162 h3 = __floats2bfloat162_rn(f[8 * q + 6], f[8 * q + 7]);
        dst[q] = make_uint4(*reinterpret_cast<uint32_t*>(&h0), *reinterpret_cast<uint32_t*>(&h1),
                            *reinterpret_cast<uint32_t*>(&h2), *reinterpret_cast<uint32_t*>(&h3));
    }
}

// Surrogate pre-pass: gather_transport of every cell on the tick's starting
// field, with no dependency waits.  A cell none of whose neighbour voxels is
// written by an earlier cell gets exactly the state the cell loop will see.
__global__ void __launch_bounds__(kTickThreads) k_surrogate_prepass(const __grid_constant__ CellLaunch a,
                                                                   const float* __restrict__ norm,
                                                                   float* __restrict__ xt,
                                                                   __nv_bfloat16* __restrict__ X) {
    extern __shared__ __align__(16) unsigned char tick_smem[];
    CellScratch& S = *reinterpret_cast<CellScratch*>(tick_smem);
    const CellRunView v{&a.t, a.g, a.field, a.light, a.epoch, nullptr, nullptr};
    for (uint32_t base = blockIdx.x * kTickThreads; base < a.n; base += gridDim.x * kTickThreads) {
        const uint32_t j = base + threadIdx.x;
        if (j < a.n) prepass_cell(v, a.k, S, j, j, a.t.cap, norm, xt, X);
    }
}

// Batched form: global row gi = cell_base(run) + j.
__global__ void __launch_bounds__(kTickThreads) k_surrogate_prepass_batch(const RunDesc* __restrict__ runs, int n_runs,
                                                                         uint32_t total, CellConsts c, int parity,
                                                                         const float* __restrict__ norm,
                                                                         float* __restrict__ xt, uint32_t ld,
                                                                         __nv_bfloat16* __restrict__ X) {
    extern __shared__ __align__(16) unsigned char tick_smem[];
    CellScratch& S = *reinterpret_cast<CellScratch*>(tick_smem);
    for (uint32_t base = blockIdx.x * kTickThreads; base < total; base += gridDim.x * kTickThreads) {
        const uint32_t gi = base + threadIdx.x;
        if (gi < total) {
            const RunDesc& R = runs[find_run(runs, n_runs, gi)];
            const CellRunView v{&R.t, R.g, R.field[parity], R.light, R.epoch, nullptr, nullptr};
            prepass_cell(v, c, S, gi - R.cell_base, gi, ld, norm, xt, X);
        }
    }
}

__global__ void k_surrogate_count(const uint8_t* __restrict__ status, const float* __restrict__ err, uint32_t n,
                                  unsigned long long* __restrict__ counters, uint32_t* __restrict__ max_bits) {
    __shared__ unsigned int s_cnt[3];
    __shared__ uint32_t s_max;
    if (threadIdx.x < 3) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_max = 0;
    __syncthreads();
    unsigned int spec = 0, acc = 0, rej = 0;
    uint32_t mx = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint8_t st = status[j];
        spec += st != kSurrNotSpeculated;
        acc += st == kSurrAccepted;
        rej += st == kSurrRejected;
        if (st == kSurrAccepted) mx = max(mx, __float_as_uint(err[j]));
    }
    atomicAdd(&s_cnt[0], spec);
    atomicAdd(&s_cnt[1], acc);
    atomicAdd(&s_cnt[2], rej);
    atomicMax(&s_max, mx);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (blockIdx.x == 0) atomicAdd(&counters[0], (unsigned long long)n);
        atomicAdd(&counters[1], (unsigned long long)s_cnt[0]);
        atomicAdd(&counters[2], (unsigned long long)s_cnt[1]);
        atomicAdd(&counters[3], (unsigned long long)s_cnt[2]);
        atomicMax(max_bits, s_max);
    }
}

// Batched form: tickets run over the cells of all runs, run-major (run r's
// cell j is ticket cell_base(r) + j), so every dependency of a cell, which lies
// in the same run at a smaller index, also has a smaller ticket.
template <int MODE>
__global__ void __launch_bounds__(kTickThreads) k_cell_tick_batch(const RunDesc* __restrict__ runs, int n_runs,
                                                                  BatchScalars* __restrict__ bs, CellConsts c,
                                                                  int parity) {
    extern __shared__ __align__(16) unsigned char tick_smem[];
    CellScratch& S = *reinterpret_cast<CellScratch*>(tick_smem);
    cell_tick_loop<MODE>(S, c, batch_total(runs, n_runs), &bs->ticket, &bs->err, 32u, [&](uint32_t gi, CellRunView& v, uint32_t& j) {
        const RunDesc& R = runs[find_run(runs, n_runs, gi)];
        v = CellRunView{&R.t, R.g, R.field[parity], R.light, R.epoch, &R.sv, nullptr, R.cmap};
        j = gi - R.cell_base;
    });
}

// -------------------------------------------------------- compaction -----
constexpr int kCompactThreads = 256;
constexpr int kCompactPerThread = 4;
constexpr int kCompactPerBlock = kCompactThreads * kCompactPerThread;

__device__ __forceinline__ bool is_change(uint8_t e) { return e == MARL_EVENT_DIVISION || e == MARL_EVENT_DEATH; }

// Change-list entries of the thread's flagged cells first + i (bit i of
// `flags`), written from slot `pos` on (slots >= cap are dropped).  All loads
// are issued before any store: the sources are scattered over the table, so
// this costs one memory latency per thread instead of one per loaded value.
__device__ __forceinline__ void write_changes(const CellTable& t, uint32_t first, uint32_t flags, uint32_t pos,
                                              marl_change* __restrict__ out, uint32_t cap) {
    float vals[kCompactPerThread][MARL_M_INT];
    uint32_t st[kCompactPerThread];
    uint8_t evs[kCompactPerThread];
#pragma unroll
    for (int i = 0; i < kCompactPerThread; ++i) {
        if (!((flags >> i) & 1u)) continue;
        const uint32_t j = first + i;
        evs[i] = t.events[j];
        st[i] = t.state[j];
#pragma unroll
        for (int k = 0; k < MARL_M_INT; ++k) vals[i][k] = __ldcg(&t.internal[(size_t)k * t.cap + j]);
    }
#pragma unroll
    for (int i = 0; i < kCompactPerThread; ++i) {
        if (!((flags >> i) & 1u)) continue;
        if (pos < cap) {
            marl_change& r = out[pos];
            r.cell = first + i;
            r.event = evs[i];
            r.quiescent = (uint8_t)((st[i] >> 16) & 1u);
            r._pad = 0;
            // entries are 72 bytes, so internal[] is 8-byte aligned only
#pragma unroll
            for (int k = 0; k < MARL_M_INT; k += 2)
                *reinterpret_cast<float2*>(&r.internal[k]) = make_float2(vals[i][k], vals[i][k + 1]);
        }
        ++pos;
    }
}

__global__ void __launch_bounds__(kCompactThreads) k_count_events(const uint8_t* __restrict__ ev, uint32_t n,
                                                                  uint32_t* __restrict__ block_counts) {
    __shared__ uint32_t warp_sums[kCompactThreads / 32];
    const uint32_t first = blockIdx.x * kCompactPerBlock + threadIdx.x * kCompactPerThread;
    uint32_t cnt = 0;
#pragma unroll
    for (int i = 0; i < kCompactPerThread; ++i) cnt += (first + i < n && is_change(ev[first + i])) ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kCompactThreads / 32; ++w) s += warp_sums[w];
        block_counts[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(kCompactThreads) k_scatter_events(CellTable t, uint32_t n,
                                                                    const uint32_t* __restrict__ block_counts,
                                                                    ChangeHeader* hdr, marl_change* __restrict__ out,
                                                                    uint32_t cap) {
    __shared__ uint32_t red[kCompactThreads];
    __shared__ uint32_t warp_tot[kCompactThreads / 32];
    // offset of this block = sum of the counts of earlier blocks
    uint32_t part = 0;
    for (uint32_t b = threadIdx.x; b < blockIdx.x; b += kCompactThreads) part += block_counts[b];
    red[threadIdx.x] = part;
    __syncthreads();
    for (int w = kCompactThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    const uint32_t block_off = red[0];
    const uint32_t first = blockIdx.x * kCompactPerBlock + threadIdx.x * kCompactPerThread;
    uint32_t flags = 0, cnt = 0;
#pragma unroll
    for (int i = 0; i < kCompactPerThread; ++i)
        if (first + i < n && is_change(t.events[first + i])) {
            flags |= 1u << i;
            ++cnt;
        }
    // exclusive scan of cnt over the block, in thread (= cell) order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    uint32_t warp_off = 0;
    for (int w = 0; w < warp; ++w) warp_off += warp_tot[w];
    uint32_t pos = block_off + warp_off + incl - cnt;
    write_changes(t, first, flags, pos, out, cap);
    pos += cnt;
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kCompactThreads - 1) {
        hdr->count = pos;
        hdr->n_cells = n;
    }
}

// Batched compaction: block r compacts run r's events chunk by chunk in cell
// order, carrying the running offset, into that run's change list.
__global__ void __launch_bounds__(kCompactThreads) k_compact_batch(const RunDesc* __restrict__ runs) {
    __shared__ uint32_t warp_tot[kCompactThreads / 32];
    __shared__ uint32_t s_off;
    const RunDesc& R = runs[blockIdx.x];
    const CellTable& t = R.t;
    const uint32_t n = R.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_off = 0;
    __syncthreads();
    for (uint32_t chunk = 0; chunk < n; chunk += kCompactPerBlock) {
        const uint32_t first = chunk + threadIdx.x * kCompactPerThread;
        uint32_t flags = 0, cnt = 0;
#pragma unroll
        for (int i = 0; i < kCompactPerThread; ++i)
            if (first + i < n && is_change(t.events[first + i])) {
                flags |= 1u << i;
                ++cnt;
            }
        uint32_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        uint32_t warp_off = 0, block_tot = 0;
        for (int w = 0; w < kCompactThreads / 32; ++w) {
            if (w < warp) warp_off += warp_tot[w];
            block_tot += warp_tot[w];
        }
        const uint32_t pos = s_off + warp_off + incl - cnt;
        write_changes(t, first, flags, pos, R.changes, R.change_cap);
        __syncthreads();
        if (threadIdx.x == 0) s_off += block_tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        R.hdr->count = s_off;
        R.hdr->n_cells = n;
    }
}

// Block r copies run r's change list behind those of runs < r.
__global__ void __launch_bounds__(256) k_pack_changes(const RunDesc* __restrict__ runs, int n_runs,
                                                      BatchScalars* __restrict__ bs, marl_change* __restrict__ packed) {
    __shared__ uint32_t red[256];
    uint32_t part = 0;
    for (int q = threadIdx.x; q < (int)blockIdx.x; q += 256) part += min(runs[q].hdr->count, runs[q].change_cap);
    red[threadIdx.x] = part;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    const uint32_t off = red[0];
    const RunDesc& R = runs[blockIdx.x];
    const uint32_t cnt = min(R.hdr->count, R.change_cap);
    const uint32_t words = cnt * (uint32_t)(sizeof(marl_change) / 4);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(R.changes);
    uint32_t* dst = reinterpret_cast<uint32_t*>(packed + off);
    for (uint32_t i = threadIdx.x; i < words; i += 256) dst[i] = src[i];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) bs->changes = off + cnt;
}

// ------------------------------------------------------------- edits -----
// One warp per birth.  The warp copies the 656-byte record into shared
// memory with 16-byte loads, then its lanes write the table's arrays in
// parallel (lane r: reaction r and internal species r; lanes < 8: transporter
// and effector rates; lanes < 26: cold floats; lanes 26-30: scalars).
constexpr int kBirthWarps = 4;

__device__ __forceinline__ void birth_warp(CellTable t, const Grid g, int32_t* cmap, uint8_t* mask, uint32_t slot,
                                           const marl_cell* __restrict__ rec, uint4* stage, uint32_t* err) {
    const int l = threadIdx.x & 31;
    const uint4* src = reinterpret_cast<const uint4*>(rec);
    for (int q = l; q < kRecordU4; q += 32) stage[q] = src[q];
    __syncwarp();
    const marl_cell& c = *reinterpret_cast<const marl_cell*>(stage);
    if (c.pos[0] >= g.X || c.pos[1] >= g.Y || c.pos[2] >= g.Z) {
        if (l == 0) atomicOr(err, kErrBadIndex);
        return;
    }
    write_record_warp(t, g, cmap, mask, slot, c);
}

__global__ void __launch_bounds__(32 * kBirthWarps) k_cells_from_records(const marl_cell* __restrict__ rec,
                                                                         uint32_t count, uint32_t base, CellTable t,
                                                                         Grid g, int32_t* __restrict__ cmap,
                                                                         uint8_t* __restrict__ mask, uint32_t* err) {
    __shared__ uint4 stage[kBirthWarps][kRecordU4];
    const uint32_t i = blockIdx.x * kBirthWarps + (threadIdx.x >> 5);
    if (i < count) birth_warp(t, g, cmap, mask, base + i, rec + i, stage[threadIdx.x >> 5], err);
}

__global__ void __launch_bounds__(32 * kBirthWarps) k_births_batch(const RunDesc* __restrict__ runs,
                                                                   const marl_cell* __restrict__ recs,
                                                                   const uint2* __restrict__ slots, uint32_t count,
                                                                   uint32_t* err) {
    __shared__ uint4 stage[kBirthWarps][kRecordU4];
    const uint32_t i = blockIdx.x * kBirthWarps + (threadIdx.x >> 5);
    if (i >= count) return;
    const RunDesc& R = runs[slots[i].x];
    birth_warp(R.t, R.g, R.cmap, R.mask, slots[i].y, recs + i, stage[threadIdx.x >> 5], err);
}

__global__ void k_cells_to_records(CellTable t, uint32_t n, marl_cell* __restrict__ rec) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const size_t cap = t.cap;
    marl_cell& c = rec[j];
    const uint32_t P = t.pos[j];
    c.pos[0] = (uint16_t)pos_x(P);
    c.pos[1] = (uint16_t)pos_y(P);
    c.pos[2] = (uint16_t)pos_z(P);
    const uint32_t st = t.state[j];
    c.quiescent = (uint8_t)((st >> 16) & 1u);
    c.starter_type = (uint8_t)(st >> 24);
    c.age = t.age[j];
    c.prep_remaining = (uint16_t)(st & 0xFFFFu);
    c._pad0 = 0;
    c.lineage_id = t.lineage[j];
    for (int k = 0; k < MARL_M_INT; ++k) c.internal[k] = t.internal[k * cap + j];
    marl_ruleset& r = c.ruleset;
    const uint4 tpi = t.tp_idx[j];
    const uint32_t w[4] = {tpi.x, tpi.y, tpi.z, tpi.w};
    for (int i = 0; i < MARL_S_TRANSPORTERS; ++i) {
        const float2 rr = t.tp_rate[i * cap + j];
        const uint32_t pair = (w[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
        r.transport[i].uptake_rate = rr.x;
        r.transport[i].secrete_rate = rr.y;
        r.transport[i].ext_species = (uint8_t)(pair & 0xFF);
        r.transport[i].int_species = (uint8_t)(pair >> 8);
        r.transport[i]._pad[0] = r.transport[i]._pad[1] = 0;
    }
    for (int i = 0; i < MARL_R_MAX; ++i) {
        const uint4 q = t.rx[i * cap + j];
        r.reactions[i].substrate = (uint8_t)(q.x & 0xFF);
        r.reactions[i].product = (uint8_t)((q.x >> 8) & 0xFF);
        r.reactions[i].catalyst = (uint8_t)((q.x >> 16) & 0xFF);
        r.reactions[i].cofactor = (uint8_t)(q.x >> 24);
        r.reactions[i].k_m = __uint_as_float(q.y);
        r.reactions[i].v_max = __uint_as_float(q.z);
        r.reactions[i].k_cat = __uint_as_float(q.w);
    }
    const uint4 efi = t.ef_idx[j];
    const uint32_t e[4] = {efi.x, efi.y, efi.z, efi.w};
    for (int i = 0; i < MARL_S_EFFECTORS; ++i) {
        const float2 pr = t.ef_par[i * cap + j];
        const uint32_t pair = (e[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
        r.effectors[i].threshold = pr.x;
        r.effectors[i].rate = pr.y;
        r.effectors[i].int_species = (uint8_t)(pair & 0xFF);
        r.effectors[i].ext_species = (uint8_t)(pair >> 8);
        r.effectors[i]._pad[0] = r.effectors[i]._pad[1] = 0;
    }
    const float4 f = t.fate[j];
    r.fate.division_energy = f.x;
    r.fate.death_energy = f.y;
    r.fate.quiescence_energy = f.z;
    r.fate.division_prep_ticks = f.w;
    const float* cold = t.cold + (size_t)j * kColdFloats;
    for (int i = 0; i < MARL_S_RECEPTORS; ++i) {
        r.receptors[i].k_half = cold[3 * i];
        r.receptors[i].n_hill = cold[3 * i + 1];
        r.receptors[i].gain = cold[3 * i + 2];
    }
    r.hgt_propensity = cold[24];
    r.mutation_rate = cold[25];
}

// Division halving (crates/marl-sim/src/lib.rs:237-240): parent internals *= 0.5.
__device__ __forceinline__ void halve_one(const CellTable& t, uint32_t p, uint32_t k) {
    float& v = t.internal[(size_t)k * t.cap + p];
    v = v * 0.5f;
}

__global__ void k_halve_batch(const RunDesc* __restrict__ runs, const uint2* __restrict__ items, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count * MARL_M_INT) return;
    const uint2 it = items[i / MARL_M_INT];
    halve_one(runs[it.x].t, it.y, i % MARL_M_INT);
}

// Dead cells leave the occupancy (cell_map.remove, lib.rs:261-262).
__device__ __forceinline__ void clear_dead_one(const CellTable& t, const Grid g, int32_t* cmap, uint8_t* mask,
                                               uint32_t idx) {
    const uint32_t P = t.pos[idx];
    const size_t row = (size_t)pos_z(P) * g.Y + pos_y(P);
    cmap[row * g.X + pos_x(P)] = -1;
    mask[row * mask_pitch(g.X) + pos_x(P)] = 0;
}

__global__ void k_clear_dead_batch(const RunDesc* __restrict__ runs, const uint2* __restrict__ items, uint32_t count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const RunDesc& R = runs[items[i].x];
    clear_dead_one(R.t, R.g, R.cmap, R.mask, items[i].y);
}

// Halving and dead-cell clearing of one edit list in one launch: threads
// [0, 16 n_halve) halve, the next n_dead clear.  A cell of the change list
// either divides or dies, so the two touch different cells; both must finish
// before the moves (a moved parent is copied halved, a dead slot's position
// is read before a move overwrites it).
__global__ void k_halve_clear(CellTable t, const uint32_t* __restrict__ halve_idx, uint32_t n_halve,
                              const uint32_t* __restrict__ dead_idx, uint32_t n_dead, Grid g,
                              int32_t* __restrict__ cmap, uint8_t* __restrict__ mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nh = n_halve * MARL_M_INT;
    if (i < nh)
        halve_one(t, halve_idx[i / MARL_M_INT], i % MARL_M_INT);
    else if (i - nh < n_dead)
        clear_dead_one(t, g, cmap, mask, dead_idx[i - nh]);
}

// swap_remove moves (lib.rs:258-267), one warp per move (move_one, table_ops.cuh).
__global__ void k_moves(CellTable t, const uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, uint32_t count,
                        Grid g, int32_t* __restrict__ cmap) {
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i < count) move_one(t, g, cmap, dst[i], src[i], threadIdx.x & 31);
}

__global__ void k_moves_batch(const RunDesc* __restrict__ runs, const uint4* __restrict__ items, uint32_t count) {
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= count) return;
    const uint4 it = items[i];
    const RunDesc& R = runs[it.x];
    move_one(R.t, R.g, R.cmap, it.y, it.z, threadIdx.x & 31);
}

__global__ void k_rebuild_maps(CellTable t, uint32_t n, Grid g, int32_t* __restrict__ cmap,
                               uint8_t* __restrict__ mask) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t P = t.pos[j];
    const size_t row = (size_t)pos_z(P) * g.Y + pos_y(P);
    cmap[row * g.X + pos_x(P)] = (int32_t)j;
    mask[row * mask_pitch(g.X) + pos_x(P)] = 1;
}

// ======================================================== launchers ======
static inline unsigned blocks_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

cudaError_t launch_cell_schedule(const CellLaunch& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    const unsigned blocks = blocks_for(a.n, 256);
    k_cell_schedule<<<blocks < 4096u ? blocks : 4096u, 256, 0, s>>>(a.t, a.n, a.n_dev, a.g, a.cmap);
    return cudaGetLastError();
}

__global__ void k_hold_dependency(CellTable t, uint32_t cell, int face, uint32_t slot, uint32_t* err) {
    if ((t.nb[cell] >> face) & 1u)
        t.dep[(size_t)face * t.cap + cell] = (int32_t)slot;
    else
        atomicOr(err, kErrBadIndex);
}

cudaError_t launch_hold_dependency(const CellTable& t, uint32_t cell, int face, uint32_t slot, uint32_t* err,
                                   cudaStream_t s) {
    k_hold_dependency<<<1, 1, 0, s>>>(t, cell, face, slot, err);
    return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_cell_tick_mode(const CellLaunch& a, int num_sms, cudaStream_t s) {
    static std::atomic<int> setup[kSetupDevices];
    int per_sm = 1;
    cudaError_t e = setup_once(setup, &per_sm, [](int* v) {
        cudaError_t r = cudaFuncSetAttribute(k_cell_tick<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTickSmem);
        if (r != cudaSuccess) return r;
        r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(v, k_cell_tick<MODE>, kTickThreads, kTickSmem);
        if (*v < 1) *v = 1;
        return r;
    });
    if (e != cudaSuccess) return e;
    const uint32_t warps_needed = (a.n + a.lanes - 1) / a.lanes;
    const uint32_t blocks_needed = (warps_needed + (kTickThreads / 32) - 1) / (kTickThreads / 32);
    // Persistent: never more blocks than can be resident at once, so every
    // ticket holder is running (the dependency waits rely on it).
    const uint32_t resident = (uint32_t)per_sm * (uint32_t)num_sms;
    const uint32_t blocks = blocks_needed < resident ? blocks_needed : resident;
    k_cell_tick<MODE><<<blocks, kTickThreads, kTickSmem, s>>>(a);
    return cudaGetLastError();
}

bool cell_tick_covers(uint32_t n, uint32_t lanes, int num_sms) {
    static std::atomic<int> setup[kSetupDevices];
    int per_sm = 1;
    if (setup_once(setup, &per_sm, [](int* v) {
            cudaError_t r = cudaFuncSetAttribute(k_cell_tick<kModePlain>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 kTickSmem);
            if (r != cudaSuccess) return r;
            r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(v, k_cell_tick<kModePlain>, kTickThreads, kTickSmem);
            if (*v < 1) *v = 1;
            return r;
        }) != cudaSuccess)
        return false;
    return (uint64_t)n <= (uint64_t)per_sm * (uint64_t)num_sms * (kTickThreads / 32) * lanes;
}

cudaError_t launch_cell_tick(const CellLaunch& a, int num_sms, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    switch (a.mode) {
        case kModePlain: return launch_cell_tick_mode<kModePlain>(a, num_sms, s);
        case kModeCapture: return launch_cell_tick_mode<kModeCapture>(a, num_sms, s);
        case kModeGated: return launch_cell_tick_mode<kModeGated>(a, num_sms, s);
        case kModeTrusted: return launch_cell_tick_mode<kModeTrusted>(a, num_sms, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_surrogate_prepass(const CellLaunch& a, const float* norm, float* xt, void* X, int num_sms,
                                     cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    static std::atomic<int> setup[kSetupDevices];
    cudaError_t e = set_smem_once(setup, k_surrogate_prepass, kTickSmem);
    if (e != cudaSuccess) return e;
    const uint32_t blocks_needed = (a.n + kTickThreads - 1) / kTickThreads;
    const uint32_t cap_blocks = (uint32_t)num_sms * 8u;
    k_surrogate_prepass<<<blocks_needed < cap_blocks ? blocks_needed : cap_blocks, kTickThreads, kTickSmem, s>>>(
        a, norm, xt, reinterpret_cast<__nv_bfloat16*>(X));
    return cudaGetLastError();
}

cudaError_t launch_surrogate_prepass_batch(const RunDesc* runs, int n_runs, uint32_t total, const CellConsts& k,
                                           int parity, const float* norm, float* xt, uint32_t ld, void* X,
                                           int num_sms, cudaStream_t s) {
    if (total == 0) return cudaSuccess;
    static std::atomic<int> setup[kSetupDevices];
    cudaError_t e = set_smem_once(setup, k_surrogate_prepass_batch, kTickSmem);
    if (e != cudaSuccess) return e;
    const uint32_t blocks_needed = (total + kTickThreads - 1) / kTickThreads;
    const uint32_t cap_blocks = (uint32_t)num_sms * 8u;
    k_surrogate_prepass_batch<<<blocks_needed < cap_blocks ? blocks_needed : cap_blocks, kTickThreads, kTickSmem, s>>>(
        runs, n_runs, total, k, parity, norm, xt, ld, reinterpret_cast<__nv_bfloat16*>(X));
    return cudaGetLastError();
}

cudaError_t launch_surrogate_count(const uint8_t* status, const float* err, uint32_t n,
                                   unsigned long long* counters, uint32_t* max_bits, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks = (n + 255) / 256 < 296 ? (n + 255) / 256 : 296;
    k_surrogate_count<<<blocks, 256, 0, s>>>(status, err, n, counters, max_bits);
    return cudaGetLastError();
}

uint32_t compaction_blocks(uint32_t n) { return n == 0 ? 1 : (n + kCompactPerBlock - 1) / kCompactPerBlock; }

cudaError_t launch_compact_events(const CellTable& t, uint32_t n, uint32_t* block_counts, ChangeHeader* hdr,
                                  marl_change* changes, uint32_t cap, cudaStream_t s) {
    const uint32_t nb = compaction_blocks(n);
    k_count_events<<<nb, kCompactThreads, 0, s>>>(t.events, n, block_counts);
    k_scatter_events<<<nb, kCompactThreads, 0, s>>>(t, n, block_counts, hdr, changes, cap);
    return cudaGetLastError();
}

cudaError_t launch_cells_from_records(const marl_cell* rec, uint32_t count, uint32_t base, CellTable t, const Grid& g,
                                      int32_t* cmap, uint8_t* mask, uint32_t* err, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_cells_from_records<<<blocks_for(count, kBirthWarps), 32 * kBirthWarps, 0, s>>>(rec, count, base, t, g, cmap,
                                                                                      mask, err);
    return cudaGetLastError();
}

cudaError_t launch_cells_to_records(const CellTable& t, uint32_t n, marl_cell* rec, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_cells_to_records<<<blocks_for(n, 128), 128, 0, s>>>(t, n, rec);
    return cudaGetLastError();
}

cudaError_t launch_halve_clear(const CellTable& t, const uint32_t* halve_idx, uint32_t n_halve,
                               const uint32_t* dead_idx, uint32_t n_dead, const Grid& g, int32_t* cmap, uint8_t* mask,
                               cudaStream_t s) {
    const size_t items = (size_t)n_halve * MARL_M_INT + n_dead;
    if (items == 0) return cudaSuccess;
    k_halve_clear<<<blocks_for(items, 256), 256, 0, s>>>(t, halve_idx, n_halve, dead_idx, n_dead, g, cmap, mask);
    return cudaGetLastError();
}

cudaError_t launch_moves(CellTable t, const uint32_t* dst, const uint32_t* src, uint32_t count, const Grid& g,
                         int32_t* cmap, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_moves<<<blocks_for((size_t)count * 32, 128), 128, 0, s>>>(t, dst, src, count, g, cmap);
    return cudaGetLastError();
}

cudaError_t launch_rebuild_maps(const CellTable& t, uint32_t n, const Grid& g, int32_t* cmap, uint8_t* mask,
                                cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_rebuild_maps<<<blocks_for(n, 256), 256, 0, s>>>(t, n, g, cmap, mask);
    return cudaGetLastError();
}

cudaError_t launch_cell_schedule_batch(const RunDesc* runs, int n_runs, int num_sms, cudaStream_t s) {
    k_cell_schedule_batch<<<num_sms * 4, 256, 0, s>>>(runs, n_runs);
    return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_cell_tick_batch_mode(const RunDesc* runs, int n_runs, BatchScalars* bs, const CellConsts& k,
                                               int parity, int num_sms, cudaStream_t s) {
    static std::atomic<int> setup[kSetupDevices];
    int per_sm = 1;
    cudaError_t e = setup_once(setup, &per_sm, [](int* v) {
        cudaError_t r =
            cudaFuncSetAttribute(k_cell_tick_batch<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTickSmem);
        if (r != cudaSuccess) return r;
        r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(v, k_cell_tick_batch<MODE>, kTickThreads, kTickSmem);
        if (*v < 1) *v = 1;
        return r;
    });
    if (e != cudaSuccess) return e;
    // Persistent over all resident slots; the cell count is read on the device.
    k_cell_tick_batch<MODE><<<per_sm * num_sms, kTickThreads, kTickSmem, s>>>(runs, n_runs, bs, k, parity);
    return cudaGetLastError();
}

cudaError_t launch_cell_tick_batch(const RunDesc* runs, int n_runs, BatchScalars* bs, const CellConsts& k, int parity,
                                   int num_sms, int mode, cudaStream_t s) {
    switch (mode) {
        case kModePlain: return launch_cell_tick_batch_mode<kModePlain>(runs, n_runs, bs, k, parity, num_sms, s);
        case kModeGated: return launch_cell_tick_batch_mode<kModeGated>(runs, n_runs, bs, k, parity, num_sms, s);
        case kModeTrusted: return launch_cell_tick_batch_mode<kModeTrusted>(runs, n_runs, bs, k, parity, num_sms, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_compact_batch(const RunDesc* runs, int n_runs, cudaStream_t s) {
    k_compact_batch<<<n_runs, kCompactThreads, 0, s>>>(runs);
    return cudaGetLastError();
}

cudaError_t launch_pack_changes(const RunDesc* runs, int n_runs, BatchScalars* bs, marl_change* packed,
                                cudaStream_t s) {
    k_pack_changes<<<n_runs, 256, 0, s>>>(runs, n_runs, bs, packed);
    return cudaGetLastError();
}

cudaError_t launch_halve_batch(const RunDesc* runs, const uint2* items, uint32_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_halve_batch<<<blocks_for((size_t)count * MARL_M_INT, 256), 256, 0, s>>>(runs, items, count);
    return cudaGetLastError();
}

cudaError_t launch_clear_dead_batch(const RunDesc* runs, const uint2* items, uint32_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_clear_dead_batch<<<blocks_for(count, 256), 256, 0, s>>>(runs, items, count);
    return cudaGetLastError();
}

cudaError_t launch_moves_batch(const RunDesc* runs, const uint4* items, uint32_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_moves_batch<<<blocks_for((size_t)count * 32, 128), 128, 0, s>>>(runs, items, count);
    return cudaGetLastError();
}

cudaError_t launch_births_batch(const RunDesc* runs, const marl_cell* recs, const uint2* slots, uint32_t count,
                                uint32_t* err, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_births_batch<<<blocks_for(count, kBirthWarps), 32 * kBirthWarps, 0, s>>>(runs, recs, slots, count, err);
    return cudaGetLastError();
}

// Every finite float x, for n = 3, 5 and 6: the value the gather and scatter
// use for x / n (div_small_n where div12_small_n takes it, the IEEE operator
// otherwise) against the IEEE operator, bit for bit.
__global__ void k_selftest_small_division(unsigned long long* __restrict__ mismatches) {
    unsigned long long bad = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < (1ull << 32); i += stride) {
        const float x = __uint_as_float((uint32_t)i);
        const float a = fabsf(x);
        if (!(a <= 3.40282346638528859812e38f)) continue;  // finite only
        const bool fast = x == 0.0f || a >= 0x1p-125f;
#pragma unroll
        for (int n = 3; n <= 6; ++n) {
            if (n == 4) continue;
            const float nf = (float)n;
            const float got = fast ? div_small_n(x, small_divisor_inverse(n), nf) : div_rn(x, nf);
            bad += __float_as_uint(got) != __float_as_uint(__fdiv_rn(x, nf));
        }
    }
    atomicAdd(mismatches, bad);
}

}  // namespace marl

#include "ctx_impl.h"

using marl::check_device;
using marl::cuda_fail;
using marl::fail;

extern "C" marl_status marl_selftest_small_division(uint64_t* mismatches) {
    if (!mismatches) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    int dev, sms;
    marl_status st = check_device(&dev, &sms);
    if (st) return st;
    unsigned long long* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        marl::k_selftest_small_division<<<sms * 16, 256>>>(d);
        e = cudaGetLastError();
    }
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "marl_selftest_small_division");
    *mismatches = h;
    return MARL_OK;
}
