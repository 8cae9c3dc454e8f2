// Field kernels: boundary sources, masked 7-point diffusion, Beer-Lambert
// light, FP64 mass reduction, occupancy repacking.
//
// Layout in HBM: the field is AoS [z][y][x][12] f32 (48 B per voxel, 16-B
// aligned), exactly the reference's Field::data order
// (crates/marl-field/src/field.rs:15-35), two ping-pong buffers; the occupancy
// mask is u8 [z][y][pitch] with pitch = X rounded up to 16; light is f32
// [z][y][x]; the last diffusion substep of a tick also writes species 4
// compactly, f32 [z][y][x], for the light scan.
//
// Arithmetic is restated in the reference's operation order and this file is
// compiled with -fmad=false, so diffusion and sources are bit-identical to the
// reference CPU path.
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "kernel_setup.h"

namespace marl {

// ---------------------------------------------------------- sources ------
// crates/marl-field/src/field.rs:231-250 (additive + clamp); Dirichlet pins
// the value (microbenchmark option).
__device__ __forceinline__ void source_voxel(float* v, int z, int Z, const FieldConsts& k) {
    if (z == 0) {
        if (k.source_mode == MARL_SOURCES_DIRICHLET) {
            v[1] = k.prime_ox;
            v[3] = k.prime_ca;
        } else {
            v[1] = fminf(v[1] + k.src_ox, k.c_max);
            v[3] = fminf(v[3] + k.src_ca, k.c_max);
        }
    }
    if (z == Z - 1) {
        if (k.source_mode == MARL_SOURCES_DIRICHLET)
            v[2] = k.prime_re;
        else
            v[2] = fminf(v[2] + k.src_re, k.c_max);
    }
}

__global__ void k_sources(float* __restrict__ f, Grid g, FieldConsts k) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int plane = g.X * g.Y;
    if (i >= plane) return;
    // Top plane (z = 0) then bottom plane (z = Z-1), as the reference orders them.
    float* top = f + (size_t)i * 12;
    if (g.Z == 1) {
        source_voxel(top, 0, 1, k);
        return;
    }
    source_voxel(top, 0, g.Z, k);
    float* bot = f + ((size_t)(g.Z - 1) * plane + i) * 12;
    source_voxel(bot, g.Z - 1, g.Z, k);
}

// -------------------------------------------------------- diffusion ------
// Stencil arithmetic: 1 (default) = packed FP32x2 adds with scalar
// multiplies, 0 = all scalar.  Both are bit-identical to the reference.  The
// multiplies stay scalar because ptxas may contract a packed multiply that
// feeds a packed add into one fused FFMA2 (observed: 45% of results off by an
// ulp), while a scalar __fmul_rn feeding a packed add is never fused.
#ifndef MARL_STENCIL_MODE
#define MARL_STENCIL_MODE 1
#endif
constexpr int kDiffTX = 16;

// DIRECT: results go from registers straight to global memory (coalesced
// 16-byte stores) instead of through a triple-buffered shared tile and a TMA
// store, and the xy neighbours are read one species pair at a time.  That
// drops OUT_BUFS * OUT_BYTES of shared memory and about 40 live registers per
// thread, so more CTAs fit on an SM; the autotuner decides per grid.
template <int TY, int STAGES, bool DIRECT = false>
struct DiffTile {
    static constexpr int TX = kDiffTX;
    static constexpr int PW = TX + 2, PH = TY + 2;
    static constexpr int ROWF = PW * 12;  // floats per staged row: 216
    static constexpr int PLANE_BYTES = PH * ROWF * 4;
    static constexpr int MW = TX + 32;  // mask box starts 16 columns left of the tile
    static constexpr int MASK_BYTES = MW * PH;
    static constexpr int MASK_REGION = (MASK_BYTES + 127) / 128 * 128;
    static constexpr int PLANE_REGION = (PLANE_BYTES + 127) / 128 * 128;
    static constexpr int STAGE_BYTES = MASK_REGION + PLANE_REGION;
    static constexpr int OUT_BYTES = TY * TX * 48;
    static constexpr int OUT_BUFS = DIRECT ? 0 : 3;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + OUT_BUFS * OUT_BYTES + STAGES * 8;
    static_assert(ROWF <= 256 && TX * 12 <= 256 && PH <= 256 && MW <= 256, "TMA box dims are limited to 256");
    static_assert(OUT_BYTES % 128 == 0, "output staging alignment");
    static_assert(STAGES == 3 || STAGES == 4, "3 or 4 plane stages");
};

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Twelve species as six float2 pairs (species 2q, 2q+1).
struct Vox {
    float2 v[6];
};
__device__ __forceinline__ void load_vox(Vox& d, const float* s) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const float4 a = reinterpret_cast<const float4*>(s)[q];
        d.v[2 * q] = make_float2(a.x, a.y);
        d.v[2 * q + 1] = make_float2(a.z, a.w);
    }
}

// Packed FP32x2 add: each lane is the IEEE round-to-nearest single-precision
// sum (checked lane by lane against add.rn.f32 on the device).
__device__ __forceinline__ uint64_t pk2(float2 v) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
    return r;
}
__device__ __forceinline__ float2 upk2(uint64_t r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
    return upk2(r);
}

// Per-voxel update: the reference expression
//   c + dt*(d*(xm+xp+ym+yp+zm+zp - 6c) - lambda*c), then max(., 0)
// evaluated in the same order (a - b is a + (-b) exactly).
__device__ __forceinline__ void stencil(float out[12], const Vox& c, const Vox& xm, const Vox& xp, const Vox& ym,
                                        const Vox& yp, const Vox& below, const Vox& above, bool wzm, bool wzp,
                                        const FieldConsts& k) {
    const float structural = c.v[3].y;  // species 7
    const float niche = 1.0f - div_rn(k.alpha_eps * structural, k.k_eps + structural);
#if MARL_STENCIL_MODE == 0
    // Scalar IEEE operations (no contraction possible).
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float2 cc = c.v[q];
        const float2 zm = wzm ? cc : below.v[q];
        const float2 zp = wzp ? cc : above.v[q];
        float r[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float cv = h ? cc.y : cc.x;
            const float d = __fmul_rn(k.d_voxel[2 * q + h], niche);
            float lap = __fadd_rn(h ? xm.v[q].y : xm.v[q].x, h ? xp.v[q].y : xp.v[q].x);
            lap = __fadd_rn(lap, h ? ym.v[q].y : ym.v[q].x);
            lap = __fadd_rn(lap, h ? yp.v[q].y : yp.v[q].x);
            lap = __fadd_rn(lap, h ? zm.y : zm.x);
            lap = __fadd_rn(lap, h ? zp.y : zp.x);
            lap = __fsub_rn(lap, __fmul_rn(6.0f, cv));
            const float t = __fsub_rn(__fmul_rn(d, lap), __fmul_rn(k.lambda_decay[2 * q + h], cv));
            r[h] = fmaxf(__fadd_rn(cv, __fmul_rn(k.dt_sub, t)), 0.0f);
        }
        out[2 * q] = r[0];
        out[2 * q + 1] = r[1];
    }
#else
    // Packed adds, scalar multiplies.
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float2 cc = c.v[q];
        const float2 zm = wzm ? cc : below.v[q];
        const float2 zp = wzp ? cc : above.v[q];
        const float2 d = make_float2(__fmul_rn(k.d_voxel[2 * q], niche), __fmul_rn(k.d_voxel[2 * q + 1], niche));
        float2 lap = add2_rn(xm.v[q], xp.v[q]);
        lap = add2_rn(lap, ym.v[q]);
        lap = add2_rn(lap, yp.v[q]);
        lap = add2_rn(lap, zm);
        lap = add2_rn(lap, zp);
        lap = add2_rn(lap, make_float2(__fmul_rn(-6.0f, cc.x), __fmul_rn(-6.0f, cc.y)));
        const float2 ndecay = make_float2(__fmul_rn(-k.lambda_decay[2 * q], cc.x),
                                          __fmul_rn(-k.lambda_decay[2 * q + 1], cc.y));
        const float2 t = add2_rn(make_float2(__fmul_rn(d.x, lap.x), __fmul_rn(d.y, lap.y)), ndecay);
        const float2 nc = add2_rn(cc, make_float2(__fmul_rn(k.dt_sub, t.x), __fmul_rn(k.dt_sub, t.y)));
        out[2 * q] = fmaxf(nc.x, 0.0f);
        out[2 * q + 1] = fmaxf(nc.y, 0.0f);
    }
#endif

}

// The same update with the four xy neighbours read from the staged plane one
// species pair at a time (8-byte shared loads) instead of as whole voxels:
// bit-identical, fewer live registers.  Packed adds, scalar multiplies, as
// stencil() does.
__device__ __forceinline__ void stencil_pairwise(float out[12], const Vox& c, const float* xm, const float* xp,
                                                 const float* ym, const float* yp, const Vox& below,
                                                 const Vox& above, bool wzm, bool wzp, const FieldConsts& k) {
    const float structural = c.v[3].y;  // species 7
    const float niche = 1.0f - div_rn(k.alpha_eps * structural, k.k_eps + structural);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const float2 cc = c.v[q];
        const float2 zm = wzm ? cc : below.v[q];
        const float2 zp = wzp ? cc : above.v[q];
        const float2 d = make_float2(__fmul_rn(k.d_voxel[2 * q], niche), __fmul_rn(k.d_voxel[2 * q + 1], niche));
        float2 lap = add2_rn(reinterpret_cast<const float2*>(xm)[q], reinterpret_cast<const float2*>(xp)[q]);
        lap = add2_rn(lap, reinterpret_cast<const float2*>(ym)[q]);
        lap = add2_rn(lap, reinterpret_cast<const float2*>(yp)[q]);
        lap = add2_rn(lap, zm);
        lap = add2_rn(lap, zp);
        lap = add2_rn(lap, make_float2(__fmul_rn(-6.0f, cc.x), __fmul_rn(-6.0f, cc.y)));
        const float2 ndecay = make_float2(__fmul_rn(-k.lambda_decay[2 * q], cc.x),
                                          __fmul_rn(-k.lambda_decay[2 * q + 1], cc.y));
        const float2 t = add2_rn(make_float2(__fmul_rn(d.x, lap.x), __fmul_rn(d.y, lap.y)), ndecay);
        const float2 nc = add2_rn(cc, make_float2(__fmul_rn(k.dt_sub, t.x), __fmul_rn(k.dt_sub, t.y)));
        out[2 * q] = fmaxf(nc.x, 0.0f);
        out[2 * q + 1] = fmaxf(nc.y, 0.0f);
    }
}

// crates/marl-field/src/field.rs:107-203 (Field::diffusion_step_inner).
//
// 2.5D z-marching stencil.  A CTA owns a 16 x TY column tile and a chunk of
// `zc` planes.  Each xy plane of the tile plus a one-voxel halo is one TMA
// load of a 3-D view of the field, {12*X floats, Y, Z}, whose box rows are
// whole tile rows (18 voxels = 864 B); the matching occupancy rows come with
// it on the same mbarrier.  Planes stream through a ring of STAGES stages,
// STAGES-1 planes ahead of the plane being computed.  A thread owns one
// (x, y) column: the below / centre / above values of its voxel rotate
// through three register sets (the loop is unrolled by three, no copies),
// the four xy neighbours come from the staged plane, and the wall flags of
// the next plane are read one plane early so the neighbour loads never wait
// on them.  Results go to a triple-buffered shared tile; one TMA bulk-tensor
// store per plane writes it back (with DIRECT, coalesced 16-byte stores from
// registers into dst_field).  One barrier per plane.
template <int TY, int STAGES, bool DIRECT>
__device__ __forceinline__ void diffuse_tile(const CUtensorMap* tm_src, const CUtensorMap* tm_dst,
                                             const CUtensorMap* tm_mask, const Grid g, const int bx, const int by,
                                             const int bz, const int zc, const FieldConsts& k, const int apply_sources,
                                             float* __restrict__ c4_out, uint32_t* __restrict__ err,
                                             float* __restrict__ dst_field) {
    using T = DiffTile<TY, STAGES, DIRECT>;
    constexpr int TX = T::TX;
    extern __shared__ __align__(128) unsigned char smem[];
    float* outbuf = reinterpret_cast<float*>(smem + STAGES * T::STAGE_BYTES);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * T::STAGE_BYTES + T::OUT_BUFS * T::OUT_BYTES);
    // Abort flags, one per step parity: a flag is only ever set (on a bounded
    // wait that expired) and is read by all threads after that step's barrier,
    // so the decision to stop is uniform across the CTA.
    __shared__ int s_abort[2];

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x0 = bx * TX, y0 = by * TY, z0 = bz * zc;
    const int z1 = min(z0 + zc, g.Z);
    const int nplanes = z1 - z0 + 2;  // planes z0-1 .. z1
    const int last = nplanes - 2;     // centre planes 1 .. last
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < g.X && y < g.Y;
    const bool edge_xm = x == 0, edge_xp = x >= g.X - 1, edge_ym = y == 0, edge_yp = y >= g.Y - 1;

    auto mask_of = [&](int p) -> const uint8_t* { return smem + (p % STAGES) * T::STAGE_BYTES; };
    auto plane_of = [&](int p) -> float* {
        return reinterpret_cast<float*>(smem + (p % STAGES) * T::STAGE_BYTES + T::MASK_REGION);
    };
    auto issue = [&](int p) {
        uint64_t* bar = &bars[p % STAGES];
        mbar_arrive_expect_tx(bar, T::PLANE_BYTES + T::MASK_BYTES);
        // Planes outside the grid are never read (walls use the centre
        // value), so they are loaded from a clamped in-grid z.
        const int zz = min(max(z0 - 1 + p, 0), g.Z - 1);
        tma_load_3d(plane_of(p), tm_src, (x0 - 1) * 12, y0 - 1, zz, bar);
        tma_load_3d((void*)mask_of(p), tm_mask, x0 - 16, y0 - 1, zz, bar);
    };
    auto is_source_plane = [&](int p) {
        const int z = z0 - 1 + p;
        return apply_sources && (z == 0 || z == g.Z - 1);
    };
    auto transform = [&](int p) {  // boundary sources applied to a staged plane
        const int z = z0 - 1 + p;
        float* P = plane_of(p);
        for (int i = tid; i < T::PW * T::PH; i += TX * TY) source_voxel(P + i * 12, z, g.Z, k);
    };

    const int ci = ((ty + 1) * T::PW + (tx + 1)) * 12;  // own voxel in a staged plane
    const int mi = (ty + 1) * T::MW + tx + 16;           // own column in a staged mask
    // Wall flags of a centre plane: bit 0..3 = -x, +x, -y, +y neighbour reads the centre.
    auto walls_of = [&](int p) -> uint32_t {
        const uint8_t* M = mask_of(p);
        return (uint32_t)(edge_xm || M[mi - 1]) | ((uint32_t)(edge_xp || M[mi + 1]) << 1) |
               ((uint32_t)(edge_ym || M[mi - T::MW]) << 2) | ((uint32_t)(edge_yp || M[mi + T::MW]) << 3);
    };

    int issued = 0, waited = 0;
    bool aborted = false;
    // The next substep's blocks may be scheduled as soon as all of this
    // launch's blocks are running; nothing of the previous launch's output is
    // read or overwritten before griddep_wait.
    griddep_launch_dependents();
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        s_abort[0] = s_abort[1] = 0;
    }
    griddep_wait();
    __syncthreads();
    if (tid == 0) {
        const int pre = min(STAGES, nplanes);
        for (int p = 0; p < pre; ++p) issue(p);
        issued = pre;
    }

    bool ok = mbar_wait_bounded(&bars[0], 0);
    ok = mbar_wait_bounded(&bars[1], 0) && ok;
    if (!ok) {
        atomicOr(err, kErrTimeoutMbar);
        s_abort[0] = 1;
    }
    waited = 2;
    __syncthreads();
    aborted = s_abort[0] != 0;
    if (!aborted && apply_sources) {
        if (is_source_plane(0)) transform(0);
        if (is_source_plane(1)) transform(1);
    }
    __syncthreads();

    Vox r0, r1, r2;
    bool m0 = false, m1 = false, m2 = false;
    uint32_t walls = 0;
    if (!aborted) {
        load_vox(r0, plane_of(0) + ci);
        load_vox(r1, plane_of(1) + ci);
        m0 = mask_of(0)[mi] != 0;
        m1 = mask_of(1)[mi] != 0;
        walls = walls_of(1);
    }

    // One centre plane p: B = below, C = centre, A receives the plane above.
    auto step = [&](Vox& B, Vox& C, Vox& A, bool& mB, bool& mC, bool& mA, int p) -> bool {
        if (tid == 0) {
            if (p + STAGES - 1 < nplanes) {
                fence_proxy_async_smem();
                issue(p + STAGES - 1);
                issued = p + STAGES;
            }
        }
        if (!mbar_wait_bounded(&bars[(p + 1) % STAGES], ((p + 1) / STAGES) & 1)) {
            atomicOr(err, kErrTimeoutMbar);
            s_abort[p & 1] = 1;
        }
        waited = p + 2;
        if (is_source_plane(p + 1)) {  // uniform across the CTA
            __syncthreads();
            if (!s_abort[p & 1]) transform(p + 1);
            __syncthreads();
        }
        // After an expired wait the staged data may be stale; the step still
        // runs to its barrier (all reads stay inside shared memory) and the
        // CTA stops after it.

        load_vox(A, plane_of(p + 1) + ci);
        mA = mask_of(p + 1)[mi] != 0;
        const uint32_t next_walls = walls_of(p + 1);

        const int z = z0 - 1 + p;
        float out[12];
        if (mC) {  // occupied: copied unchanged (field.rs:130-136)
#pragma unroll
            for (int q = 0; q < 6; ++q) out[2 * q] = C.v[q].x, out[2 * q + 1] = C.v[q].y;
        } else {
            const float* P = plane_of(p);
            // A wall or occupied neighbour reads as the centre value: point
            // its load at the centre voxel.
            if constexpr (DIRECT) {
                stencil_pairwise(out, C, P + ci - ((walls & 1u) ? 0 : 12), P + ci + ((walls & 2u) ? 0 : 12),
                                 P + ci - ((walls & 4u) ? 0 : T::ROWF), P + ci + ((walls & 8u) ? 0 : T::ROWF), B, A,
                                 z == 0 || mB, z >= g.Z - 1 || mA, k);
            } else {
                Vox xm, xp, ym, yp;
                load_vox(xm, P + ci - ((walls & 1u) ? 0 : 12));
                load_vox(xp, P + ci + ((walls & 2u) ? 0 : 12));
                load_vox(ym, P + ci - ((walls & 4u) ? 0 : T::ROWF));
                load_vox(yp, P + ci + ((walls & 8u) ? 0 : T::ROWF));
                stencil(out, C, xm, xp, ym, yp, B, A, z == 0 || mB, z >= g.Z - 1 || mA, k);
            }
        }
        if constexpr (DIRECT) {
            if (active) {
                float4* dst = reinterpret_cast<float4*>(dst_field + (((size_t)z * g.Y + y) * g.X + x) * 12);
                __stcg(dst, make_float4(out[0], out[1], out[2], out[3]));
                __stcg(dst + 1, make_float4(out[4], out[5], out[6], out[7]));
                __stcg(dst + 2, make_float4(out[8], out[9], out[10], out[11]));
            }
        } else {
            float* ob = outbuf + (p % 3) * (T::OUT_BYTES / 4) + (ty * TX + tx) * 12;
            reinterpret_cast<float4*>(ob)[0] = make_float4(out[0], out[1], out[2], out[3]);
            reinterpret_cast<float4*>(ob)[1] = make_float4(out[4], out[5], out[6], out[7]);
            reinterpret_cast<float4*>(ob)[2] = make_float4(out[8], out[9], out[10], out[11]);
        }
        if (c4_out && active) c4_out[((size_t)z * g.Y + y) * g.X + x] = out[4];
        walls = next_walls;
        if constexpr (!DIRECT) fence_proxy_async_smem();
        __syncthreads();
        if (s_abort[p & 1]) {
            aborted = true;
            return false;
        }
        if constexpr (!DIRECT) {
            if (tid == 0) {
                tma_store_3d(tm_dst, outbuf + (p % 3) * (T::OUT_BYTES / 4), x0 * 12, y0, z);
                bulk_commit();
                bulk_wait_read<1>();  // the store of plane p-1 has read its buffer
            }
        }
        return true;
    };

    if (!aborted) {
        int p = 1;
        bool go = true;
        for (; go && p + 2 <= last; p += 3) {
            go = step(r0, r1, r2, m0, m1, m2, p) && step(r1, r2, r0, m1, m2, m0, p + 1) &&
                 step(r2, r0, r1, m2, m0, m1, p + 2);
        }
        if (go && p <= last) go = step(r0, r1, r2, m0, m1, m2, p);
        if (go && p + 1 <= last) go = step(r1, r2, r0, m1, m2, m0, p + 1);
    }

    if (tid == 0) {
        if constexpr (!DIRECT) bulk_wait_all();
        // After an abort, wait (bounded) for loads still in flight so no copy
        // lands in shared memory after the CTA exits.
        if (aborted)
            for (int q = waited; q < issued; ++q) mbar_wait_bounded(&bars[q % STAGES], (q / STAGES) & 1);
    }
}

// Resident CTAs per SM each form is compiled for, which sets its register
// budget: 128 registers a thread for the staged-store tiles, 96-102 for the
// direct-store tiles of 4 and 8 rows.
template <int TY, bool DIRECT>
constexpr int diff_min_blocks() {
    return DIRECT ? (TY <= 4 ? 10 : (TY <= 8 ? 5 : (TY <= 16 ? 2 : 1)))
                  : (TY <= 4 ? 8 : (TY <= 8 ? 4 : (TY <= 16 ? 2 : 1)));
}

template <int TY, int STAGES, bool DIRECT>
__global__ void __launch_bounds__(kDiffTX* TY, (diff_min_blocks<TY, DIRECT>()))
    k_diffuse(const __grid_constant__ CUtensorMap tm_src, const __grid_constant__ CUtensorMap tm_dst,
              const __grid_constant__ CUtensorMap tm_mask, Grid g, int zc, FieldConsts k, int apply_sources,
              float* __restrict__ c4_out, uint32_t* __restrict__ err, float* __restrict__ dst_field) {
    diffuse_tile<TY, STAGES, DIRECT>(&tm_src, &tm_dst, &tm_mask, g, blockIdx.x, blockIdx.y, blockIdx.z, zc, k,
                                     apply_sources, c4_out, err, dst_field);
}

// Batched form: one launch advances one substep of every run.  CTA b owns
// work item items[b] = (run, tile x, tile y, z-chunk); the run's tensor maps
// (loads from buffer 0/1, stores into buffer 0/1, mask) are read from global
// memory.  All runs share the ping-pong parity of the substep.
template <int TY, int STAGES, bool DIRECT>
__global__ void __launch_bounds__(kDiffTX* TY, (diff_min_blocks<TY, DIRECT>()))
    k_diffuse_batch(const RunDesc* __restrict__ runs, const CUtensorMap* __restrict__ maps,
                    const int4* __restrict__ items, int zc, FieldConsts k, int parity, int apply_sources, int emit_c4,
                    uint32_t* __restrict__ err) {
    griddep_wait();
    const int4 it = items[blockIdx.x];
    const RunDesc& r = runs[it.x];
    const CUtensorMap* m = maps + (size_t)it.x * kMapsPerRun;
    diffuse_tile<TY, STAGES, DIRECT>(&m[parity], &m[2 + (parity ^ 1)], &m[4], r.g, it.y, it.z, it.w, zc, k,
                                     apply_sources, emit_c4 ? r.c4 : nullptr, err, r.field[parity ^ 1]);
}

// ------------------------------------------------------------ light ------
// crates/marl-field/src/light.rs:29-59.  The running intensity of a column is
// an exclusive product with a floor to zero; the floor makes it
// non-associative, so each column is multiplied strictly in z order.  A block
// covers 32 columns of one y row and walks z in 64-plane segments.  The
// attenuation factors of a segment (exp in double, rounded to float: the
// reference calls glibc expf, within 0.502 ulp) and its occupancy go to one of
// two shared buffers; while warp 0 runs the 32 sequential column products
// through segment s, warps 1-7 load and evaluate segment s+1 into the other
// buffer.  Each thread issues all its loads of a segment before it uses any.
constexpr int kLightCols = 32;
constexpr int kLightSeg = 64;
constexpr int kLightThreads = 256;

// Factors and occupancy of planes zs .. zs+nz-1 into buffer (fac, occ), by
// the NT threads t = 0 .. NT-1.
template <int NT>
__device__ __forceinline__ void light_fill(const float* __restrict__ c4, const float* __restrict__ field,
                                           const uint8_t* __restrict__ mask, const Grid& g, const FieldConsts& k,
                                           int x0, int y, int zs, int nz, int t, float (*fac)[kLightCols],
                                           uint8_t (*occ)[kLightCols]) {
    constexpr int kItems = (kLightSeg * kLightCols + NT - 1) / NT;
    const int pitch = mask_pitch(g.X);
    const float neg_chem = -k.chemical_absorption;
    float a[kItems];
    uint8_t o[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = t + j * NT, zz = i / kLightCols, xg = x0 + i % kLightCols;
        a[j] = 0.0f;
        o[j] = 0;
        if (zz < nz && xg < g.X) {
            const size_t v = ((size_t)(zs + zz) * g.Y + y) * g.X + xg;
            a[j] = c4 ? c4[v] : field[v * 12 + 4];
            o[j] = mask[((size_t)(zs + zz) * g.Y + y) * pitch + xg];
        }
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = t + j * NT, zz = i / kLightCols, xi = i % kLightCols;
        if (zz < nz && x0 + xi < g.X) {
            fac[zz][xi] = (float)exp((double)(neg_chem * a[j]));
            occ[zz][xi] = o[j];
        }
    }
}

__device__ __forceinline__ void light_columns(const float* __restrict__ c4, const float* __restrict__ field,
                                              const uint8_t* __restrict__ mask, float* __restrict__ light,
                                              const Grid g, const FieldConsts& k, const int x0, const int y) {
    __shared__ float fac[2][kLightSeg][kLightCols];
    __shared__ uint8_t occ[2][kLightSeg][kLightCols];
    const int tid = threadIdx.x, lane = tid & 31;
    const int nseg = (g.Z + kLightSeg - 1) / kLightSeg;
    float inten = k.surface_intensity;
    light_fill<kLightThreads>(c4, field, mask, g, k, x0, y, 0, min(kLightSeg, g.Z), tid, fac[0], occ[0]);
    __syncthreads();
    for (int s = 0; s < nseg; ++s) {
        const int zs = s * kLightSeg, nz = min(kLightSeg, g.Z - zs);
        const int buf = s & 1;
        if (tid < 32) {
            if (x0 + lane < g.X) {
                float* out = light + ((size_t)zs * g.Y + y) * g.X + x0 + lane;
                const size_t plane = (size_t)g.X * g.Y;
                for (int zz = 0; zz < nz; ++zz) {
                    out[zz * plane] = inten;
                    if (occ[buf][zz][lane]) inten *= k.cell_factor;
                    inten *= fac[buf][zz][lane];
                    if (inten < k.light_floor) inten = 0.0f;
                }
            }
        } else if (s + 1 < nseg) {
            const int zn = zs + kLightSeg;
            light_fill<kLightThreads - 32>(c4, field, mask, g, k, x0, y, zn, min(kLightSeg, g.Z - zn), tid - 32,
                                           fac[buf ^ 1], occ[buf ^ 1]);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_light(const float* __restrict__ c4, const float* __restrict__ field,
                                               const uint8_t* __restrict__ mask, float* __restrict__ light, Grid g,
                                               FieldConsts k) {
    griddep_launch_dependents();
    griddep_wait();  // the last substep's output
    light_columns(c4, field, mask, light, g, k, blockIdx.x * kLightCols, blockIdx.y);
}

// Batched form: block b handles item (run, column chunk, y) of any run.
// With use_c4 species 4 comes from the run's compact copy written by the
// last substep, otherwise from field[parity].
__global__ void __launch_bounds__(256) k_light_batch(const RunDesc* __restrict__ runs, const int4* __restrict__ items,
                                                     FieldConsts k, int parity, int use_c4) {
    griddep_launch_dependents();
    griddep_wait();  // the last substep's output
    const int4 it = items[blockIdx.x];
    const RunDesc& r = runs[it.x];
    light_columns(use_c4 ? r.c4 : nullptr, r.field[parity], r.mask, r.light, r.g, k, it.y * kLightCols, it.z);
}

// ------------------------------------------------------------- mass ------
// Per-species FP64 sums in a fixed order: kMassBlocks x 256 threads, each
// thread sums a strided voxel range sequentially, then fixed-shape tree
// reductions (block, then a single block over the partials).
constexpr int kMassBlocks = 592;  // 4 x 148 SMs
__global__ void __launch_bounds__(256) k_mass_partial(const float* __restrict__ f, size_t V,
                                                      double* __restrict__ partial) {
    __shared__ double red[12][256];
    double acc[12];
#pragma unroll
    for (int s = 0; s < 12; ++s) acc[s] = 0.0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += stride) {
        const float4* p = reinterpret_cast<const float4*>(f + v * 12);
        const float4 a = p[0], b = p[1], c = p[2];
        acc[0] += a.x, acc[1] += a.y, acc[2] += a.z, acc[3] += a.w;
        acc[4] += b.x, acc[5] += b.y, acc[6] += b.z, acc[7] += b.w;
        acc[8] += c.x, acc[9] += c.y, acc[10] += c.z, acc[11] += c.w;
    }
#pragma unroll
    for (int s = 0; s < 12; ++s) red[s][threadIdx.x] = acc[s];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int s = 0; s < 12; ++s) red[s][threadIdx.x] += red[s][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 12) partial[blockIdx.x * 12 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void __launch_bounds__(256) k_mass_final(const double* __restrict__ partial, int nblocks,
                                                    double* __restrict__ out) {
    __shared__ double red[12][256];
    double acc[12];
#pragma unroll
    for (int s = 0; s < 12; ++s) acc[s] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 256)
        for (int s = 0; s < 12; ++s) acc[s] += partial[b * 12 + s];
    for (int s = 0; s < 12; ++s) red[s][threadIdx.x] = acc[s];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int s = 0; s < 12; ++s) red[s][threadIdx.x] += red[s][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 12) out[threadIdx.x] = red[threadIdx.x][0];
}

// ------------------------------------------------------- occupancy -------
// Dense one-byte-per-voxel occupancy (the reference's `&[bool]`) -> pitched
// mask rows.
__global__ void k_repack_mask(const uint8_t* __restrict__ occ, uint8_t* __restrict__ mask, Grid g) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int pitch = mask_pitch(g.X);
    const size_t rows = (size_t)g.Y * g.Z;
    if (i >= rows * pitch) return;
    const size_t row = i / pitch;
    const int x = (int)(i % pitch);
    mask[i] = x < g.X ? (occ[row * g.X + x] != 0) : 0;
}

__global__ void k_unpack_mask(const uint8_t* __restrict__ mask, uint8_t* __restrict__ occ, Grid g) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.V()) return;
    const size_t row = i / g.X;
    const int x = (int)(i % g.X);
    occ[i] = mask[row * mask_pitch(g.X) + x];
}

// ======================================================== launchers ======

// Tile table: (rows per tile, plane stages, store form).  The autotuner picks
// one.  Tiles 0-3: 4 stages, 4-7: 3 stages, both through a shared output tile
// and a TMA store; 8-11: 3 stages, direct stores.
static const int kTileTY[] = {8, 16, 4, 32, 8, 16, 4, 32, 4, 8, 16, 32};

int diffusion_tile_count() { return 12; }

void diffusion_tile_shape(int tile, int* tx, int* ty) {
    *tx = kDiffTX;
    *ty = kTileTY[tile];
}

template <int TY, int STAGES, bool DIRECT = false>
static cudaError_t launch_diffuse_t(const DiffusionPlan& plan, int which_src, const Grid& g, const FieldConsts& k,
                                    int apply_sources, float* c4_out, uint32_t* err, cudaStream_t s) {
    using T = DiffTile<TY, STAGES, DIRECT>;
    static std::atomic<int> setup[kSetupDevices];
    cudaError_t e = set_smem_once(setup, k_diffuse<TY, STAGES, DIRECT>, T::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    dim3 grid((g.X + kDiffTX - 1) / kDiffTX, (g.Y + TY - 1) / TY, (g.Z + plan.zc - 1) / plan.zc);
    return launch_dependent(k_diffuse<TY, STAGES, DIRECT>, grid, dim3(kDiffTX * TY), T::SMEM_BYTES, s,
                            plan.tm_load[which_src], plan.tm_store[which_src ^ 1], plan.tm_mask, g, plan.zc, k,
                            apply_sources, c4_out, err, plan.buf[which_src ^ 1]);
}

cudaError_t launch_diffuse(const DiffusionPlan& plan, int which_src, const Grid& g, const FieldConsts& k,
                           int apply_sources, float* c4_out, uint32_t* err, cudaStream_t s) {
    switch (plan.tile) {
        case 0: return launch_diffuse_t<8, 4>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 1: return launch_diffuse_t<16, 4>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 2: return launch_diffuse_t<4, 4>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 3: return launch_diffuse_t<32, 4>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 4: return launch_diffuse_t<8, 3>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 5: return launch_diffuse_t<16, 3>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 6: return launch_diffuse_t<4, 3>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 7: return launch_diffuse_t<32, 3>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 8: return launch_diffuse_t<4, 3, true>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 9: return launch_diffuse_t<8, 3, true>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        case 10: return launch_diffuse_t<16, 3, true>(plan, which_src, g, k, apply_sources, c4_out, err, s);
        default: return launch_diffuse_t<32, 3, true>(plan, which_src, g, k, apply_sources, c4_out, err, s);
    }
}

template <int TY, int STAGES, bool DIRECT = false>
static cudaError_t launch_diffuse_batch_t(const RunDesc* runs, const CUtensorMap* maps, const int4* items, int n_items,
                                          int zc, const FieldConsts& k, int parity, int apply_sources, int emit_c4,
                                          uint32_t* err, cudaStream_t s) {
    using T = DiffTile<TY, STAGES, DIRECT>;
    if (n_items == 0) return cudaSuccess;
    static std::atomic<int> setup[kSetupDevices];
    cudaError_t e = set_smem_once(setup, k_diffuse_batch<TY, STAGES, DIRECT>, T::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    return launch_dependent(k_diffuse_batch<TY, STAGES, DIRECT>, dim3(n_items), dim3(kDiffTX * TY), T::SMEM_BYTES, s,
                            runs, maps, items, zc, k, parity, apply_sources, emit_c4, err);
}

cudaError_t launch_diffuse_batch(int tile, const RunDesc* runs, const CUtensorMap* maps, const int4* items,
                                 int n_items, int zc, const FieldConsts& k, int parity, int apply_sources, int emit_c4,
                                 uint32_t* err, cudaStream_t s) {
    switch (tile) {
        case 0: return launch_diffuse_batch_t<8, 4>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 1: return launch_diffuse_batch_t<16, 4>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 2: return launch_diffuse_batch_t<4, 4>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 3: return launch_diffuse_batch_t<32, 4>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 4: return launch_diffuse_batch_t<8, 3>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 5: return launch_diffuse_batch_t<16, 3>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 6: return launch_diffuse_batch_t<4, 3>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 7: return launch_diffuse_batch_t<32, 3>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 8: return launch_diffuse_batch_t<4, 3, true>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 9: return launch_diffuse_batch_t<8, 3, true>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        case 10: return launch_diffuse_batch_t<16, 3, true>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
        default: return launch_diffuse_batch_t<32, 3, true>(runs, maps, items, n_items, zc, k, parity, apply_sources, emit_c4, err, s);
    }
}

cudaError_t launch_light_batch(const RunDesc* runs, const int4* items, int n_items, const FieldConsts& k, int parity,
                               int use_c4, cudaStream_t s) {
    if (n_items == 0) return cudaSuccess;
    return launch_dependent(k_light_batch, dim3(n_items), dim3(256), 0, s, runs, items, k, parity, use_c4);
}

cudaError_t launch_sources(float* f, const Grid& g, const FieldConsts& k, cudaStream_t s) {
    const int n = g.X * g.Y;
    k_sources<<<(n + 255) / 256, 256, 0, s>>>(f, g, k);
    return cudaGetLastError();
}

cudaError_t launch_light(const float* c4, const float* f, const uint8_t* mask, float* light, const Grid& g,
                         const FieldConsts& k, cudaStream_t s) {
    dim3 grid((g.X + kLightCols - 1) / kLightCols, g.Y);
    return launch_dependent(k_light, grid, dim3(256), 0, s, c4, f, mask, light, g, k);
}

cudaError_t launch_mass(const float* f, const Grid& g, double* partial, double* out, cudaStream_t s) {
    k_mass_partial<<<kMassBlocks, 256, 0, s>>>(f, g.V(), partial);
    k_mass_final<<<1, 256, 0, s>>>(partial, kMassBlocks, out);
    return cudaGetLastError();
}
size_t mass_partial_doubles() { return (size_t)kMassBlocks * 12; }

cudaError_t launch_repack_mask(const uint8_t* occ, uint8_t* mask, const Grid& g, cudaStream_t s) {
    const size_t n = (size_t)g.Y * g.Z * mask_pitch(g.X);
    k_repack_mask<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(occ, mask, g);
    return cudaGetLastError();
}

cudaError_t launch_unpack_mask(const uint8_t* mask, uint8_t* occ, const Grid& g, cudaStream_t s) {
    const size_t n = g.V();
    k_unpack_mask<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mask, occ, g);
    return cudaGetLastError();
}

// ------------------------------------------------------- tensor maps -----
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D view {12*X floats, Y, Z} of a field buffer with a box of `box_voxels`
// voxels by `box_rows` rows by one plane.
bool encode_field_map(CUtensorMap* m, const float* base, const Grid& g, int box_voxels, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g.X * 12, (cuuint64_t)g.Y, (cuuint64_t)g.Z};
    const cuuint64_t strides[2] = {(cuuint64_t)g.X * 48, (cuuint64_t)g.X * g.Y * 48};
    const cuuint32_t box[3] = {(cuuint32_t)(box_voxels * 12), (cuuint32_t)box_rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool encode_mask_map(CUtensorMap* m, const uint8_t* base, const Grid& g, int tx, int ty) {
    auto fn = encode_fn();
    if (!fn) return false;
    const int pitch = mask_pitch(g.X);
    const cuuint64_t dims[3] = {(cuuint64_t)g.X, (cuuint64_t)g.Y, (cuuint64_t)g.Z};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch, (cuuint64_t)pitch * g.Y};
    const cuuint32_t box[3] = {(cuuint32_t)(tx + 32), (cuuint32_t)(ty + 2), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool plan_diffusion(DiffusionPlan* plan, const float* a, const float* b, const uint8_t* mask, const Grid& g,
                    int tile, int zc) {
    int tx, ty;
    diffusion_tile_shape(tile, &tx, &ty);
    plan->tile = tile;
    plan->zc = zc > 0 ? zc : 16;
    plan->buf[0] = const_cast<float*>(a);
    plan->buf[1] = const_cast<float*>(b);
    const float* bufs[2] = {a, b};
    for (int i = 0; i < 2; ++i) {
        if (!encode_field_map(&plan->tm_load[i], bufs[i], g, tx + 2, ty + 2)) return false;
        if (!encode_field_map(&plan->tm_store[i], bufs[i], g, tx, ty)) return false;
    }
    return encode_mask_map(&plan->tm_mask, mask, g, tx, ty);
}

}  // namespace marl
