// Device fate processing: the reference's per-tick fate step
// (crates/marl-sim/src/lib.rs:219-277) on the GPU, so that a tick needs no
// host round trip.  The step consumes the events the cell loop left in the
// table (one per cell) and performs, in the reference's semantics:
//   * division placement (find_empty_neighbor, crates/marl-sim/src/spatial.rs:115-154)
//     on the cell map as it stood before the step,
//   * halving of every placed parent's internal species (lib.rs:237-240),
//   * the daughters: clone, lineage draw, Ruleset::mutate (lib.rs:230-245),
//   * deaths by swap_remove from the back (lib.rs:256-267),
//   * births appended in division order unless an earlier daughter of the same
//     step took the voxel (lib.rs:269-277).
// Random draws come from one counter-based stream per dividing cell
// (fate_stream.h), so every division is placed and mutated independently.
//
// Kernels of one step (n = cells at its start, all counts device-resident):
//   k_fate_count / k_fate_scatter   ordered compaction of Division and Death
//                                   events into ascending lists (2048 cells per block)
//   k_fate_resolve (two blocks)     block 0: placement + voxel claims (atomicMin
//                                   of the division ordinal), birth slots in
//                                   division order, halving, new population;
//                                   block 1: the swap_remove permutation
//   k_fate_moves                    dead voxels cleared; one warp per swap_remove move
//   k_fate_births                   one warp per daughter: gather the parent's
//                                   row, draw + mutate on one lane, write the slot
//
// swap_remove in closed form.  Removing the ascending deaths d from the back
// leaves n1 = n - |deaths| cells.  Let D(x) be the number of deaths below x,
// b_0 = n1, and b_{k+1} = b_k + D(b_k) - D(b_{k-1}) (D(b_{-1}) = 0) until the
// increment is zero.  The deaths below b_0 are the holes that receive cells;
// a death q in [b_{k-1}, b_k) is first refilled from position
// b_k + D(q) - D(b_{k-1}).  Following that map from the i-th hole's first
// source (n1 + i) through dead positions ends at the cell that the sequential
// back-to-front swap_remove leaves in hole i.  Each level consumes at least one
// death, so a chain has at most as many steps as there are levels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "ctx_impl.h"
#include "fate_stream.h"
#include "internal.h"
#include "table_ops.cuh"

namespace marl {

constexpr int kFateThreads = 256;
constexpr int kFatePerThread = 8;
constexpr uint32_t kFateChunk = (uint32_t)kFateThreads * kFatePerThread;
constexpr int kResolveThreads = 512;
constexpr int kFateBirthWarps = 4;
constexpr uint32_t kPlacedBit = 1u << 31;
constexpr unsigned kFull = 0xFFFFFFFFu;

uint32_t fate_blocks(uint32_t cap) { return (cap + kFateChunk - 1) / kFateChunk; }

// crates/marl-sim/src/spatial.rs:8-15 (FACE order)
__constant__ int c_fate_face[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

__device__ __forceinline__ size_t vox_of(uint32_t P, const Grid& g) {
    return ((size_t)pos_z(P) * g.Y + pos_y(P)) * g.X + pos_x(P);
}

// Exclusive scan of v over the block (blockDim.x a multiple of 32); `total`
// receives the block sum.  wb: 33 words of shared memory.  Ends with a
// barrier, so wb may be reused at once.
__device__ __forceinline__ uint32_t block_scan_excl(uint32_t v, uint32_t* wb, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wb[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < nw ? wb[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < nw) wb[lane] = wi - w;
        if (lane == 31) wb[32] = wi;
    }
    __syncthreads();
    const uint32_t r = wb[warp] + incl - v;
    total = wb[32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* wb) {
    uint32_t total;
    block_scan_excl(v, wb, total);
    return total;
}

// Events of cells first .. first+7 (those below n).
__device__ __forceinline__ void load_events8(const uint8_t* __restrict__ ev, uint32_t first, uint32_t n, uint8_t e[8]) {
    if (first + 8 <= n) {
        const uint2 w = *reinterpret_cast<const uint2*>(ev + first);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            e[i] = (uint8_t)(w.x >> (8 * i));
            e[4 + i] = (uint8_t)(w.y >> (8 * i));
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) e[i] = first + i < n ? ev[first + i] : (uint8_t)MARL_EVENT_NONE;
    }
}

__device__ __forceinline__ uint32_t packed_counts(const uint8_t e[8]) {
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        c += (e[i] == MARL_EVENT_DIVISION ? 1u : 0u) + (e[i] == MARL_EVENT_DEATH ? (1u << 16) : 0u);
    return c;
}

// Grid (chunks, runs): block (x, r) counts the Division and Death events of
// run r's cells [2048 x, 2048 x + 2048).
__global__ void __launch_bounds__(kFateThreads) k_fate_count(const FateRun* __restrict__ runs) {
    __shared__ uint32_t wb[33];
    const FateRun& R = runs[blockIdx.y];
    const uint32_t n = R.f.fs->n;
    if (blockIdx.x * kFateChunk >= n) return;
    const uint32_t first = blockIdx.x * kFateChunk + threadIdx.x * kFatePerThread;
    uint8_t e[8];
    load_events8(R.t.events, first, n, e);
    const uint32_t tot = block_sum(packed_counts(e), wb);
    if (threadIdx.x == 0) R.f.blk[blockIdx.x] = tot;
}

// Same grid: the chunk's events into the run's ascending Division and Death lists.
__global__ void __launch_bounds__(kFateThreads) k_fate_scatter(const FateRun* __restrict__ runs) {
    __shared__ uint32_t wb[33];
    const FateRun& R = runs[blockIdx.y];
    const uint32_t n = R.f.fs->n;
    if (blockIdx.x == 0 && threadIdx.x == 0) R.f.fs->n_old = n;  // the population the step starts from
    if (blockIdx.x * kFateChunk >= n) return;
    uint32_t od = 0, ox = 0;  // Division and Death counts of the chunks before this one
    for (uint32_t b = threadIdx.x; b < blockIdx.x; b += kFateThreads) {
        const uint32_t v = R.f.blk[b];
        od += v & 0xFFFFu;
        ox += v >> 16;
    }
    od = block_sum(od, wb);
    ox = block_sum(ox, wb);
    const uint32_t first = blockIdx.x * kFateChunk + threadIdx.x * kFatePerThread;
    uint8_t e[8];
    load_events8(R.t.events, first, n, e);
    uint32_t tot;
    const uint32_t ex = block_scan_excl(packed_counts(e), wb, tot);
    uint32_t pd = od + (ex & 0xFFFFu), px = ox + (ex >> 16);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (e[i] == MARL_EVENT_DIVISION) R.f.div_list[pd++] = first + i;
        else if (e[i] == MARL_EVENT_DEATH) R.f.death_list[px++] = first + i;
    }
}

// find_empty_neighbor (crates/marl-sim/src/spatial.rs:115-154): the empty
// in-grid voxels at `division_neighbor_distance` along the six faces, else the
// empty face neighbours; one uniform pick among them.
__device__ __forceinline__ bool place_daughter(uint32_t P, const int32_t* __restrict__ cmap, const Grid& g,
                                               long long dist, fate::Stream& r, uint32_t& out) {
    const long long x = pos_x(P), y = pos_y(P), z = pos_z(P);
    uint32_t cand[6];
    uint32_t nc = 0;
    for (int pass = 0; pass < 2 && nc == 0; ++pass) {
        const long long d = pass == 0 ? dist : 1;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const long long nx = x + c_fate_face[f][0] * d, ny = y + c_fate_face[f][1] * d,
                            nz = z + c_fate_face[f][2] * d;
            if (nx >= 0 && nx < g.X && ny >= 0 && ny < g.Y && nz >= 0 && nz < g.Z &&
                cmap[((size_t)nz * g.Y + ny) * g.X + nx] < 0)
                cand[nc++] = pack_pos((uint32_t)nx, (uint32_t)ny, (uint32_t)nz);
        }
    }
    if (nc == 0) return false;
    out = cand[r.range(0, nc)];
    return true;
}

// Grid (2, runs).  Block 0 of run r places the daughters, picks the births
// and halves the placed parents; block 1 works out the swap_remove
// permutation.  Neither touches what the other reads, so they run side by
// side.
__global__ void __launch_bounds__(kResolveThreads) k_fate_resolve(const FateRun* __restrict__ runs,
                                                                  const __grid_constant__ marl_sim_params sim,
                                                                  uint32_t* err_out) {
    __shared__ uint32_t wb[33];
    __shared__ uint32_t s_win, s_placed, s_run, s_levels, s_err;
    const FateRun& R = runs[blockIdx.y];
    const FateBuffers& F = R.f;
    FateScalars* fs = F.fs;
    const CellTable& t = R.t;
    const Grid g = R.g;
    const uint32_t cap = t.cap;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t n = fs->n_old;

    // Totals of the compaction.
    uint32_t part = 0;
    const uint32_t chunks = (n + kFateChunk - 1) / kFateChunk;
    for (uint32_t b = tid; b < chunks; b += nthr) part += F.blk[b] & 0xFFFFu;
    const uint32_t ndiv = block_sum(part, wb);
    part = 0;
    for (uint32_t b = tid; b < chunks; b += nthr) part += F.blk[b] >> 16;
    const uint32_t ndeath = block_sum(part, wb);
    const uint32_t n1 = n - ndeath;
    if (tid == 0) s_win = s_placed = s_run = s_err = 0;
    __syncthreads();

    if (blockIdx.x == 0) {
        const unsigned long long seed = fs->seed, tick = fs->tick;
        // A. Placement on the cell map as it stood before the step, and claims.
        const long long dist = (long long)sim.division_neighbor_distance;
        for (uint32_t k = tid; k < ndiv; k += nthr) {
            const uint32_t p = F.div_list[k];
            fate::Stream r(fate::stream_key(seed, tick, p));
            uint32_t target = 0;
            const bool ok = place_daughter(t.pos[p], R.cmap, g, dist, r, target);
            F.div_info[k] = make_uint2(target, r.draws | (ok ? kPlacedBit : 0u));
            if (ok) atomicMin(&F.claim[vox_of(target, g)], k);
        }
        __syncthreads();

        // B. A daughter is born when its division holds the lowest ordinal
        // among the claims on its voxel; slots follow division order.  Every
        // placed parent is halved, whether or not its daughter survives the
        // collision.
        for (uint32_t base = 0; base < ndiv; base += nthr) {
            const uint32_t k = base + tid;
            uint32_t flags = 0;  // won | placed << 16
            if (k < ndiv) {
                const uint2 info = F.div_info[k];
                if (info.y & kPlacedBit) flags = (1u << 16) | (F.claim[vox_of(info.x, g)] == k ? 1u : 0u);
            }
            uint32_t tot;
            const uint32_t ex = block_scan_excl(flags, wb, tot);
            if (k < ndiv) {
                uint32_t slot = kFateNoSlot;
                if (flags & 1u) {
                    const uint64_t sl = (uint64_t)n1 + s_win + (ex & 0xFFFFu);
                    slot = sl < cap ? (uint32_t)sl : kFateDropped;
                }
                F.div_slot[k] = slot;
                if (flags >> 16) {
                    const uint32_t p = F.div_list[k];
#pragma unroll
                    for (int sp = 0; sp < MARL_M_INT; ++sp) {
                        float& v = t.internal[(size_t)sp * cap + p];
                        v = v * 0.5f;
                    }
                }
            }
            __syncthreads();
            if (tid == 0) {
                s_win += tot & 0xFFFFu;
                s_placed += tot >> 16;
            }
            __syncthreads();
        }

        // Population and counters.
        if (tid == 0) {
            const uint32_t room = cap - n1;
            const uint32_t births = s_win < room ? s_win : room;
            if (births < s_win) atomicOr(err_out, kErrCapacity);
            fs->n = n1 + births;
            fs->n1 = n1;
            fs->ndiv = ndiv;
            fs->ndeath = ndeath;
            fs->placed = s_placed;
            fs->births = births;
            fs->key_tick = tick;
            fs->tick = tick + 1;
            fs->total_div += s_placed;
            fs->total_death += ndeath;
        }
        return;
    }

    // C. Positions of the dying cells, for k_fate_moves to clear their voxels
    // (lib.rs:261-262) once block 0's placement has read the cell map.
    for (uint32_t i = tid; i < ndeath; i += nthr) F.dead_pos[i] = t.pos[F.death_list[i]];

    // D. cnt[o] = deaths in [n1, n1 + o) over the tail [n1, n).
    for (uint32_t base = 0; base < ndeath; base += nthr) {
        const uint32_t o = base + tid;
        const uint32_t dead = (o < ndeath && t.events[n1 + o] == MARL_EVENT_DEATH) ? 1u : 0u;
        uint32_t tot;
        const uint32_t ex = block_scan_excl(dead, wb, tot);
        if (o < ndeath) F.cnt[o] = s_run + ex;
        __syncthreads();
        if (tid == 0) s_run += tot;
        __syncthreads();
    }
    const uint32_t m0 = ndeath - s_run;  // holes below n1 = cells that move
    if (tid == 0) F.cnt[ndeath] = s_run;
    __syncthreads();

    // E. Level boundaries b_k and D(b_{k-1}).
    if (tid == 0) {
        uint32_t L = 0, b = n1, db = 0;
        for (;;) {
            F.lev_b[L] = b;
            F.lev_d[L] = db;
            ++L;
            const uint32_t Db = m0 + F.cnt[b - n1];
            const uint32_t m = Db - db;
            if (m == 0 || L > ndeath + 1) break;
            if (m > n - b) {  // b never passes n for events consistent with the death list
                atomicOr(&s_err, kErrFateChain);
                break;
            }
            db = Db;
            b += m;
        }
        s_levels = L;
    }
    __syncthreads();

    // F. The cell that ends in hole i, and the new slot of every tail survivor.
    const uint32_t L = s_levels;
    for (uint32_t i = tid; i < m0; i += nthr) {
        const uint32_t h = F.death_list[i];
        uint32_t q = n1 + i;
        uint32_t steps = 0;
        bool bad = false;
        while (t.events[q] == MARL_EVENT_DEATH) {
            // level k: lev_b[k-1] <= q < lev_b[k]
            uint32_t lo = 0, hi = L;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (F.lev_b[mid] <= q) lo = mid + 1; else hi = mid;
            }
            if (++steps > L || lo == 0 || lo >= L) {
                bad = true;
                break;
            }
            const uint32_t nq = F.lev_b[lo] + (m0 + F.cnt[q - n1]) - F.lev_d[lo];
            if (nq >= n || nq < n1) {
                bad = true;
                break;
            }
            q = nq;
        }
        if (bad) atomicOr(&s_err, kErrFateChain);
        F.move_dst[i] = h;
        F.move_src[i] = q;
        F.newidx[q - n1] = h;
    }
    __syncthreads();
    if (tid == 0) {
        if (s_err) atomicOr(err_out, s_err);
        fs->moves = m0;
        fs->levels = L;
    }
}

// Grid (x, runs): the dying cells' voxels are cleared, and warps of the
// blocks of run r take its moves in turn.  A cleared voxel belongs to a dead
// cell and a moved cell keeps its own voxel, so the two never meet.
__global__ void __launch_bounds__(256) k_fate_moves(const FateRun* __restrict__ runs) {
    const FateRun& R = runs[blockIdx.y];
    const Grid g = R.g;
    const uint32_t ndeath = R.f.fs->ndeath;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ndeath; i += gridDim.x * blockDim.x) {
        const uint32_t P = R.f.dead_pos[i];
        const size_t row = (size_t)pos_z(P) * g.Y + pos_y(P);
        R.cmap[row * g.X + pos_x(P)] = -1;
        R.mask[row * mask_pitch(g.X) + pos_x(P)] = 0;
    }
    const uint32_t moves = R.f.fs->moves;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < moves; i += warps)
        move_one(R.t, R.g, R.cmap, R.f.move_dst[i], R.f.move_src[i], threadIdx.x & 31);
}

// Grid (x, runs): one warp per division of run r.
__global__ void __launch_bounds__(32 * kFateBirthWarps) k_fate_births(const FateRun* __restrict__ runs,
                                                                      const __grid_constant__ marl_sim_params sim) {
    __shared__ __align__(16) marl_cell rec[kFateBirthWarps];
    const FateRun& R = runs[blockIdx.y];
    const FateScalars* fs = R.f.fs;
    const uint32_t ndiv = fs->ndiv, n1 = fs->n1;
    const unsigned long long seed = fs->seed, tick = fs->key_tick;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    for (uint32_t k = blockIdx.x * kFateBirthWarps + w; k < ndiv; k += gridDim.x * kFateBirthWarps) {
        const uint32_t slot = R.f.div_slot[k];
        if (slot == kFateNoSlot) continue;
        const uint2 info = R.f.div_info[k];
        if (l == 0) R.f.claim[vox_of(info.x, R.g)] = 0xFFFFFFFFu;  // the winner releases its voxel's claim
        if (slot == kFateDropped) continue;
        const uint32_t p = R.f.div_list[k];
        const uint32_t pn = p < n1 ? p : R.f.newidx[p - n1];
        marl_cell& c = rec[w];
        read_record_warp(R.t, pn, c);
        __syncwarp();
        if (l == 0) {
            fate::Stream r(fate::stream_key(seed, tick, p));
            r.skip(info.y & ~kPlacedBit);
            c.pos[0] = (uint16_t)pos_x(info.x);
            c.pos[1] = (uint16_t)pos_y(info.x);
            c.pos[2] = (uint16_t)pos_z(info.x);
            c.age = 0;
            c.prep_remaining = 0;
            c.lineage_id = r.u64();
            fate::mutate_ruleset(c.ruleset, r, sim);
        }
        __syncwarp();
        write_record_warp(R.t, R.g, R.cmap, R.mask, slot, c);
        __syncwarp();
    }
}

// Batch: every run's population and first global cell index from its fate
// scalars, and the next tick's completion epoch (one block).
__global__ void __launch_bounds__(1024) k_batch_population(RunDesc* __restrict__ runs, int n_runs,
                                                           const FateRun* __restrict__ fr) {
    __shared__ uint32_t wb[33];
    __shared__ uint32_t s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (int base = 0; base < n_runs; base += blockDim.x) {
        const int r = base + (int)threadIdx.x;
        const uint32_t n = r < n_runs ? fr[r].f.fs->n : 0u;
        uint32_t tot;
        const uint32_t ex = block_scan_excl(n, wb, tot);
        if (r < n_runs) {
            runs[r].n = n;
            runs[r].cell_base = s_base + ex;
            runs[r].epoch = runs[r].epoch + 1u;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_base += tot;
        __syncthreads();
    }
}

__global__ void k_set_population(FateScalars* fs, uint32_t n) { fs->n = n; }

__global__ void k_fate_init(FateScalars* fs, unsigned long long seed, unsigned long long tick,
                            unsigned long long total_div, unsigned long long total_death) {
    fs->seed = seed;
    fs->tick = tick;
    fs->total_div = total_div;
    fs->total_death = total_death;
}

// Diagnostics of the stream specification: `count` u64 outputs of one stream,
// `count` normals of a fresh stream with the same key, and stream_ln of x[].
__global__ void k_stream_probe(unsigned long long seed, unsigned long long tick, uint32_t parent, uint32_t count,
                               float stddev, unsigned long long* u64_out, float* normal_out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    fate::Stream a(fate::stream_key(seed, tick, parent));
    for (uint32_t i = 0; i < count; ++i) u64_out[i] = a.u64();
    fate::Stream b(fate::stream_key(seed, tick, parent));
    for (uint32_t i = 0; i < count; ++i) normal_out[i] = b.normal(stddev);
}

__global__ void k_stream_ln(const double* __restrict__ x, uint32_t n, double* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = fate::stream_ln(x[i]);
}

// ----------------------------------------------------------- host side ---

cudaError_t alloc_fate(FateBuffers& f, uint32_t cap, size_t voxels, FateScalars* fs_external) {
    f = FateBuffers{};
    cudaError_t e;
    if (fs_external) {
        f.fs = fs_external;
        f.own_fs = false;
    }
#define A(field, type, count)                                                               \
    if ((e = cudaMalloc((void**)&f.field, sizeof(type) * (size_t)(count))) != cudaSuccess) \
        return e;
    if (!fs_external) A(fs, FateScalars, 1);
    A(blk, uint32_t, fate_blocks(cap));
    A(div_list, uint32_t, cap);
    A(death_list, uint32_t, cap);
    A(div_info, uint2, cap);
    A(div_slot, uint32_t, cap);
    A(cnt, uint32_t, (size_t)cap + 1);
    A(lev_b, uint32_t, (size_t)cap + 2);
    A(lev_d, uint32_t, (size_t)cap + 2);
    A(move_dst, uint32_t, cap);
    A(move_src, uint32_t, cap);
    A(newidx, uint32_t, cap);
    A(dead_pos, uint32_t, cap);
    A(claim, uint32_t, voxels);
#undef A
    if ((e = cudaMemset(f.fs, 0, sizeof(FateScalars))) != cudaSuccess) return e;  // zeroed by the owner too
    return cudaMemset(f.claim, 0xFF, voxels * 4);
}

void free_fate(FateBuffers& f) {
    void* p[] = {f.own_fs ? f.fs : nullptr, f.blk, f.div_list, f.death_list, f.div_info, f.div_slot, f.cnt, f.lev_b, f.lev_d,
                 f.move_dst, f.move_src, f.newidx, f.dead_pos, f.claim};
    for (void* q : p)
        if (q) cudaFree(q);
    f = FateBuffers{};
}

cudaError_t launch_set_population(FateScalars* fs, uint32_t n, cudaStream_t s) {
    k_set_population<<<1, 1, 0, s>>>(fs, n);
    return cudaGetLastError();
}

cudaError_t launch_fate_init(FateScalars* fs, unsigned long long seed, unsigned long long tick,
                             unsigned long long total_div, unsigned long long total_death, cudaStream_t s) {
    k_fate_init<<<1, 1, 0, s>>>(fs, seed, tick, total_div, total_death);
    return cudaGetLastError();
}

cudaError_t launch_fate(const FateRun* d_runs, int n_runs, uint32_t max_cap, uint32_t* err, const marl_sim_params& sim,
                        int num_sms, cudaStream_t s) {
    if (n_runs <= 0) return cudaSuccess;
    const dim3 chunks(fate_blocks(max_cap), (unsigned)n_runs);
    k_fate_count<<<chunks, kFateThreads, 0, s>>>(d_runs);
    k_fate_scatter<<<chunks, kFateThreads, 0, s>>>(d_runs);
    k_fate_resolve<<<dim3(2, n_runs), kResolveThreads, 0, s>>>(d_runs, sim, err);
    const unsigned per_run = (unsigned)std::max(1, 2 * num_sms / n_runs);
    k_fate_moves<<<dim3(per_run, n_runs), 256, 0, s>>>(d_runs);
    k_fate_births<<<dim3(per_run, n_runs), 32 * kFateBirthWarps, 0, s>>>(d_runs, sim);
    return cudaGetLastError();
}

cudaError_t launch_batch_population(RunDesc* runs, int n_runs, const FateRun* fr, cudaStream_t s) {
    k_batch_population<<<1, 1024, 0, s>>>(runs, n_runs, fr);
    return cudaGetLastError();
}

}  // namespace marl

using namespace marl;

#define CK(expr)                                            \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

namespace marl {

marl_status begin_device_population(marl_ctx* c) {
    if (!c->fate_ready) {
        CK(alloc_fate(c->fate, c->t.cap, c->g.V()));
        FateRun fr;
        fr.f = c->fate;
        fr.t = c->t;
        fr.g = c->g;
        fr.cmap = c->cmap;
        fr.mask = c->mask;
        CK(cudaMalloc((void**)&c->d_fate_run, sizeof(FateRun)));
        CK(cudaMemcpy(c->d_fate_run, &fr, sizeof(FateRun), cudaMemcpyHostToDevice));
        c->fate_ready = true;
    }
    if (!c->n_on_device) {
        CK(launch_set_population(c->fate.fs, c->n, c->stream));
        c->n_on_device = true;
        c->schedule_dirty = true;
    }
    return MARL_OK;
}

marl_status sync_population(marl_ctx* c) {
    if (!c->n_on_device) return MARL_OK;
    uint32_t n = 0;
    CK(cudaMemcpyAsync(c->h_hdr, c->d_hdr, sizeof(ChangeHeader), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&n, &c->fate.fs->n, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->d2h_bytes += sizeof(ChangeHeader) + 4;
    c->n = n;
    c->n_on_device = false;
    c->schedule_dirty = true;
    return collect_device_errors(c, c->h_hdr->err);
}

marl_status enqueue_fate(marl_ctx* c) {
    marl_status st = begin_device_population(c);
    if (st) return st;
    c->c4_valid = false;
    CK(launch_fate(c->d_fate_run, 1, c->t.cap, &c->d_hdr->err, c->sim, c->num_sms, c->stream));
    c->launches += 5;
    c->schedule_dirty = true;
    return MARL_OK;
}

}  // namespace marl

extern "C" {

marl_status marl_ctx_fate_init(marl_ctx* c, uint64_t seed, uint64_t tick, uint64_t total_divisions,
                               uint64_t total_deaths) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    marl_status st = begin_device_population(c);
    if (st) return st;
    CK(launch_fate_init(c->fate.fs, seed, tick, total_divisions, total_deaths, c->stream));
    return MARL_OK;
}

marl_status marl_ctx_fate(marl_ctx* c) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    return enqueue_fate(c);
}

marl_status marl_ctx_fate_stats(marl_ctx* c, marl_fate_stats* out) {
    if (!c || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    marl_status st = begin_device_population(c);
    if (st) return st;
    FateScalars h;
    CK(cudaMemcpyAsync(&h, c->fate.fs, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    st = sync_and_check(c);
    c->d2h_bytes += sizeof(h);
    if (st) return st;
    out->tick = h.tick;
    out->population = h.n;
    out->total_divisions = h.total_div;
    out->total_deaths = h.total_death;
    out->tick_divisions = h.placed;
    out->tick_deaths = h.ndeath;
    out->tick_births = h.births;
    out->tick_moves = h.moves;
    return MARL_OK;
}

marl_status marl_ctx_set_events(marl_ctx* c, const uint8_t* events, uint32_t n) {
    if (!c || (n && !events)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    marl_status st = sync_population(c);
    if (st) return st;
    if (n != c->n) return fail(MARL_ERR_INVALID_INPUT, "%u events for %u cells", n, c->n);
    for (uint32_t i = 0; i < n; ++i)
        if (events[i] > MARL_EVENT_QUIESCENCE) return fail(MARL_ERR_INVALID_INPUT, "event %u of cell %u", events[i], i);
    if (n) {
        CK(cudaMemcpyAsync(c->t.events, events, n, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->h2d_bytes += n;
    }
    return MARL_OK;
}

marl_status marl_fate_stream_probe(uint64_t seed, uint64_t tick, uint32_t parent, uint32_t count, float stddev,
                                   uint64_t* u64_out, float* normal_out) {
    if (!u64_out || !normal_out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (count == 0) return MARL_OK;
    int dev, sms;
    marl_status st = check_device(&dev, &sms);
    if (st) return st;
    unsigned long long* du = nullptr;
    float* dn = nullptr;
    CK(cudaMalloc((void**)&du, (size_t)count * 8));
    cudaError_t e = cudaMalloc((void**)&dn, (size_t)count * 4);
    if (e == cudaSuccess) {
        k_stream_probe<<<1, 32>>>(seed, tick, parent, count, stddev, du, dn);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(u64_out, du, (size_t)count * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(normal_out, dn, (size_t)count * 4, cudaMemcpyDeviceToHost);
    cudaFree(du);
    if (dn) cudaFree(dn);
    if (e != cudaSuccess) return cuda_fail(e, "marl_fate_stream_probe");
    return MARL_OK;
}

marl_status marl_fate_stream_ln(const double* x, uint32_t n, double* out) {
    if (!x || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (n == 0) return MARL_OK;
    int dev, sms;
    marl_status st = check_device(&dev, &sms);
    if (st) return st;
    double* d = nullptr;
    CK(cudaMalloc((void**)&d, (size_t)n * 16));
    cudaError_t e = cudaMemcpy(d, x, (size_t)n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_stream_ln<<<(n + 255) / 256, 256>>>(d, n, d + n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + n, (size_t)n * 8, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "marl_fate_stream_ln");
    return MARL_OK;
}

}  // extern "C"
