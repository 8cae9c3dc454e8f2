// Field kernels: boundary sources, masked 7-point diffusion, Beer-Lambert
// light, FP64 mass reduction, occupancy repacking.
//
// Layout in HBM: the field is AoS [z][y][x][12] f32 (48 B per voxel, 16-B
// aligned), exactly the reference's Field::data order
// (crates/marl-field/src/field.rs:15-35), two ping-pong buffers; the occupancy
// mask is u8 [z][y][pitch] with pitch = X rounded up to 16; light is f32
// [z][y][x].
//
// Arithmetic is restated in the reference's operation order and this file is
// compiled with -fmad=false, so diffusion and sources are bit-identical to the
// reference CPU path.
#include <cuda.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

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
// crates/marl-field/src/field.rs:107-203 (Field::diffusion_step_inner).
//
// 2.5D z-marching stencil.  A CTA owns a TX x TY column tile and a chunk of
// `zc` planes.  Each xy plane of the tile plus a one-voxel halo (and the
// matching occupancy rows) is brought into shared memory by one TMA load into
// a 4-stage ring, three planes ahead of the plane being computed.  A thread
// owns one (x, y) column: the z-1 and z+1 values of its own voxel live in
// registers, the four xy neighbours come from the staged plane.
template <int TX, int TY>
struct DiffTile {
    static constexpr int PW = TX + 2, PH = TY + 2;
    static constexpr int PLANE_BYTES = PW * PH * 12 * 4;
    static constexpr int MW = TX + 32;  // mask box starts 16 columns left of the tile
    static constexpr int MASK_BYTES = MW * PH;
    static constexpr int MASK_REGION = (MASK_BYTES + 127) / 128 * 128;
    static constexpr int STAGE_BYTES = MASK_REGION + (PLANE_BYTES + 127) / 128 * 128;
    static constexpr int STAGES = 4;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + STAGES * 8;
    static_assert(TX % 16 == 0, "mask TMA box needs 16-byte aligned x start");
    static_assert(PW <= 256 && PH <= 256 && MW <= 256, "TMA box dims are limited to 256");
};

template <int TX, int TY>
__global__ void __launch_bounds__(TX* TY) k_diffuse(const __grid_constant__ CUtensorMap tm_field,
                                                    const __grid_constant__ CUtensorMap tm_mask,
                                                    float* __restrict__ dst, Grid g, int zc, FieldConsts k,
                                                    int apply_sources, uint32_t* __restrict__ err) {
    using T = DiffTile<TX, TY>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + T::STAGES * T::STAGE_BYTES);
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * zc;
    const int z1 = min(z0 + zc, g.Z);
    const int nplanes = z1 - z0 + 2;  // planes z0-1 .. z1
    const int x = x0 + tx, y = y0 + ty;
    const bool active = x < g.X && y < g.Y;

    auto mask_of = [&](int p) -> const uint8_t* { return smem + (p % T::STAGES) * T::STAGE_BYTES; };
    auto plane_of = [&](int p) -> float* {
        return reinterpret_cast<float*>(smem + (p % T::STAGES) * T::STAGE_BYTES + T::MASK_REGION);
    };
    auto issue = [&](int p) {
        uint64_t* bar = &bars[p % T::STAGES];
        mbar_arrive_expect_tx(bar, T::PLANE_BYTES + T::MASK_BYTES);
        // Planes outside the grid are never read (walls use the centre
        // value), so they are loaded from a clamped in-grid z.
        const int zz = min(max(z0 - 1 + p, 0), g.Z - 1);
        tma_load_4d(plane_of(p), &tm_field, 0, x0 - 1, y0 - 1, zz, bar);
        tma_load_3d((void*)mask_of(p), &tm_mask, x0 - 16, y0 - 1, zz, bar);
    };
    auto transform = [&](int p) {  // boundary sources applied to a staged plane
        const int z = z0 - 1 + p;
        if (z != 0 && z != g.Z - 1) return;
        float* P = plane_of(p);
        for (int i = tid; i < T::PW * T::PH; i += TX * TY) source_voxel(P + i * 12, z, g.Z, k);
    };

    int issued = 0;
    if (tid == 0) {
        for (int s = 0; s < T::STAGES; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        s_abort = 0;
    }
    __syncthreads();
    if (tid == 0) {
        const int pre = min(T::STAGES, nplanes);
        for (int p = 0; p < pre; ++p) issue(p);
        issued = pre;
    }

    bool ok = mbar_wait_bounded(&bars[0], 0);
    ok = mbar_wait_bounded(&bars[1], 0) && ok;
    if (!ok) {
        atomicOr(err, kErrTimeoutMbar);
        s_abort = 1;
    }
    __syncthreads();
    int waited = 2;
    if (!s_abort && apply_sources) {
        transform(0);
        transform(1);
    }
    __syncthreads();

    const int ci = ((ty + 1) * T::PW + (tx + 1)) * 12;  // own voxel in a staged plane
    const int mi = (ty + 1) * T::MW + tx + 16;           // own column in a staged mask
    float below[12], cur[12], above[12];
    bool mb = false, mc = false, ma = false;
    if (!s_abort) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float4 a = reinterpret_cast<const float4*>(plane_of(0) + ci)[q];
            const float4 b = reinterpret_cast<const float4*>(plane_of(1) + ci)[q];
            below[4 * q] = a.x, below[4 * q + 1] = a.y, below[4 * q + 2] = a.z, below[4 * q + 3] = a.w;
            cur[4 * q] = b.x, cur[4 * q + 1] = b.y, cur[4 * q + 2] = b.z, cur[4 * q + 3] = b.w;
        }
        mb = mask_of(0)[mi] != 0;
        mc = mask_of(1)[mi] != 0;
    }
    __syncthreads();

    for (int p = 1; p <= nplanes - 2 && !s_abort; ++p) {
        if (tid == 0 && p + 3 < nplanes) {
            fence_proxy_async_smem();
            issue(p + 3);
            issued = p + 4;
        }
        if (!mbar_wait_bounded(&bars[(p + 1) % T::STAGES], ((p + 1) / T::STAGES) & 1)) {
            atomicOr(err, kErrTimeoutMbar);
            s_abort = 1;
        }
        waited = p + 2;
        if (apply_sources) transform(p + 1);
        __syncthreads();
        if (s_abort) break;

        const float* Pn = plane_of(p + 1);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const float4 a = reinterpret_cast<const float4*>(Pn + ci)[q];
            above[4 * q] = a.x, above[4 * q + 1] = a.y, above[4 * q + 2] = a.z, above[4 * q + 3] = a.w;
        }
        ma = mask_of(p + 1)[mi] != 0;

        const int z = z0 - 1 + p;
        if (active) {
            float out[12];
            if (mc) {  // occupied: copied unchanged (field.rs:130-136)
#pragma unroll
                for (int s = 0; s < 12; ++s) out[s] = cur[s];
            } else {
                const float* P = plane_of(p);
                const uint8_t* M = mask_of(p);
                const float structural = cur[7];
                const float niche = 1.0f - k.alpha_eps * structural / (k.k_eps + structural);
                const bool wxm = x == 0 || M[mi - 1];
                const bool wxp = x >= g.X - 1 || M[mi + 1];
                const bool wym = y == 0 || M[mi - T::MW];
                const bool wyp = y >= g.Y - 1 || M[mi + T::MW];
                const bool wzm = z == 0 || mb;
                const bool wzp = z >= g.Z - 1 || ma;
                float nxm[12], nxp[12], nym[12], nyp[12];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float4 a = reinterpret_cast<const float4*>(P + ci - 12)[q];
                    const float4 b = reinterpret_cast<const float4*>(P + ci + 12)[q];
                    const float4 c = reinterpret_cast<const float4*>(P + ci - T::PW * 12)[q];
                    const float4 d = reinterpret_cast<const float4*>(P + ci + T::PW * 12)[q];
                    nxm[4 * q] = a.x, nxm[4 * q + 1] = a.y, nxm[4 * q + 2] = a.z, nxm[4 * q + 3] = a.w;
                    nxp[4 * q] = b.x, nxp[4 * q + 1] = b.y, nxp[4 * q + 2] = b.z, nxp[4 * q + 3] = b.w;
                    nym[4 * q] = c.x, nym[4 * q + 1] = c.y, nym[4 * q + 2] = c.z, nym[4 * q + 3] = c.w;
                    nyp[4 * q] = d.x, nyp[4 * q + 1] = d.y, nyp[4 * q + 2] = d.z, nyp[4 * q + 3] = d.w;
                }
#pragma unroll
                for (int s = 0; s < 12; ++s) {  // field.rs:152-195
                    const float c = cur[s];
                    const float d = k.d_voxel[s] * niche;
                    const float xm = wxm ? c : nxm[s];
                    const float xp = wxp ? c : nxp[s];
                    const float ym = wym ? c : nym[s];
                    const float yp = wyp ? c : nyp[s];
                    const float zm = wzm ? c : below[s];
                    const float zp = wzp ? c : above[s];
                    const float lap = xm + xp + ym + yp + zm + zp - 6.0f * c;
                    const float decay = k.lambda_decay[s] * c;
                    const float nc = c + k.dt_sub * (d * lap - decay);
                    out[s] = fmaxf(nc, 0.0f);
                }
            }
            float4* o = reinterpret_cast<float4*>(dst + (((size_t)z * g.Y + y) * g.X + x) * 12);
            o[0] = make_float4(out[0], out[1], out[2], out[3]);
            o[1] = make_float4(out[4], out[5], out[6], out[7]);
            o[2] = make_float4(out[8], out[9], out[10], out[11]);
        }
#pragma unroll
        for (int s = 0; s < 12; ++s) {
            below[s] = cur[s];
            cur[s] = above[s];
        }
        mb = mc;
        mc = ma;
        __syncthreads();
    }

    // Drain: after an abort, wait (bounded) for loads still in flight so no
    // copy lands in shared memory after the CTA exits.
    if (s_abort && tid == 0) {
        for (int q = waited; q < issued; ++q) mbar_wait_bounded(&bars[q % T::STAGES], (q / T::STAGES) & 1);
    }
}

// ------------------------------------------------------------ light ------
// crates/marl-field/src/light.rs:29-59.  One thread per (x, y) column, z in
// order: the running intensity is an exclusive product with a floor to zero,
// which is not associative, so it is kept sequential per column to stay
// identical to the reference.  exp is evaluated in double and rounded to
// float (the reference calls glibc expf, which is within 0.502 ulp).
__global__ void k_light(const float* __restrict__ field, const uint8_t* __restrict__ mask, float* __restrict__ light,
                        Grid g, FieldConsts k) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= g.X * g.Y) return;
    const int x = col % g.X, y = col / g.X;
    const int pitch = mask_pitch(g.X);
    const size_t plane = (size_t)g.X * g.Y;
    float inten = k.surface_intensity;
    const float neg_chem = -k.chemical_absorption;
    constexpr int U = 8;
    int z = 0;
    for (; z + U <= g.Z; z += U) {
        float a[U];
        uint8_t m[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const size_t v = (size_t)(z + u) * plane + col;
            a[u] = __ldg(field + v * 12 + 4);
            m[u] = __ldg(mask + ((size_t)(z + u) * g.Y + y) * pitch + x);
        }
        float e[U];
#pragma unroll
        for (int u = 0; u < U; ++u) e[u] = (float)exp((double)(neg_chem * a[u]));
#pragma unroll
        for (int u = 0; u < U; ++u) {
            light[(size_t)(z + u) * plane + col] = inten;
            if (m[u]) inten *= k.cell_factor;
            inten *= e[u];
            if (inten < k.light_floor) inten = 0.0f;
        }
    }
    for (; z < g.Z; ++z) {
        const size_t v = (size_t)z * plane + col;
        light[v] = inten;
        if (mask[((size_t)z * g.Y + y) * pitch + x]) inten *= k.cell_factor;
        inten *= (float)exp((double)(neg_chem * field[v * 12 + 4]));
        if (inten < k.light_floor) inten = 0.0f;
    }
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

template <int TX, int TY>
static cudaError_t launch_diffuse_t(const DiffusionPlan& plan, const CUtensorMap* tm_field, const float* src,
                                    float* dst, const Grid& g, const FieldConsts& k, int apply_sources,
                                    uint32_t* err, cudaStream_t s) {
    using T = DiffTile<TX, TY>;
    (void)src;
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(k_diffuse<TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             T::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    dim3 grid((g.X + TX - 1) / TX, (g.Y + TY - 1) / TY, (g.Z + plan.zc - 1) / plan.zc);
    k_diffuse<TX, TY><<<grid, TX * TY, T::SMEM_BYTES, s>>>(*tm_field, plan.tm_mask, dst, g, plan.zc, k,
                                                            apply_sources, err);
    return cudaGetLastError();
}

int diffusion_tile_count() { return 4; }

void diffusion_tile_shape(int tile, int* tx, int* ty) {
    static const int shapes[4][2] = {{32, 8}, {32, 4}, {64, 4}, {16, 16}};
    *tx = shapes[tile][0];
    *ty = shapes[tile][1];
}

cudaError_t launch_diffuse(const DiffusionPlan& plan, int which_src, const float* src, float* dst, const Grid& g,
                           const FieldConsts& k, int apply_sources, uint32_t* err, cudaStream_t s) {
    const CUtensorMap* tm = which_src == 0 ? &plan.tm_field[0] : &plan.tm_field[1];
    switch (plan.tile) {
        case 0: return launch_diffuse_t<32, 8>(plan, tm, src, dst, g, k, apply_sources, err, s);
        case 1: return launch_diffuse_t<32, 4>(plan, tm, src, dst, g, k, apply_sources, err, s);
        case 2: return launch_diffuse_t<64, 4>(plan, tm, src, dst, g, k, apply_sources, err, s);
        default: return launch_diffuse_t<16, 16>(plan, tm, src, dst, g, k, apply_sources, err, s);
    }
}

cudaError_t launch_sources(float* f, const Grid& g, const FieldConsts& k, cudaStream_t s) {
    const int n = g.X * g.Y;
    k_sources<<<(n + 255) / 256, 256, 0, s>>>(f, g, k);
    return cudaGetLastError();
}

cudaError_t launch_light(const float* f, const uint8_t* mask, float* light, const Grid& g, const FieldConsts& k,
                         cudaStream_t s) {
    const int n = g.X * g.Y;
    k_light<<<(n + 127) / 128, 128, 0, s>>>(f, mask, light, g, k);
    return cudaGetLastError();
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

bool encode_field_map(CUtensorMap* m, const float* base, const Grid& g, int tx, int ty) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[4] = {12, (cuuint64_t)g.X, (cuuint64_t)g.Y, (cuuint64_t)g.Z};
    const cuuint64_t strides[3] = {48, (cuuint64_t)g.X * 48, (cuuint64_t)g.X * g.Y * 48};
    const cuuint32_t box[4] = {12, (cuuint32_t)(tx + 2), (cuuint32_t)(ty + 2), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void*)base, dims, strides, box, estr,
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
    return encode_field_map(&plan->tm_field[0], a, g, tx, ty) && encode_field_map(&plan->tm_field[1], b, g, tx, ty) &&
           encode_mask_map(&plan->tm_mask, mask, g, tx, ty);
}

}  // namespace marl
