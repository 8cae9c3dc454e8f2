// Shared device-side definitions for libmarl_cuda: data layout of the
// device-resident state, kernel argument blocks, and the sm_100a PTX wrappers
// (mbarrier, TMA, acquire/release) used by the kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/marl_cuda.h"

namespace marl {

// Spin limits.  Every device-side wait is bounded; on expiry the kernel sets a
// bit in its error word and leaves the wait.
constexpr uint32_t kMbarSpinLimit = 1u << 22;  // try_wait rounds (each ~ up to a few us)
constexpr uint32_t kFlagSpinLimit = 1u << 22;  // default polls of a dependency flag (with nanosleep)

// Error bits written by kernels (read back with the change-list header).
constexpr uint32_t kErrTimeoutMbar = 1u << 0;
constexpr uint32_t kErrTimeoutDeps = 1u << 1;
constexpr uint32_t kErrBadIndex = 1u << 2;
constexpr uint32_t kErrCapacity = 1u << 3;   // births dropped: the cell table is full
constexpr uint32_t kErrFateChain = 1u << 4;  // swap_remove chain longer than its level count (inconsistent events)

// Packed cell position: x | y << 11 | z << 22 (x, y < 2048, z < 1024).
constexpr int kMaxXY = 2048;
constexpr int kMaxZ = 1024;
__host__ __device__ inline uint32_t pack_pos(uint32_t x, uint32_t y, uint32_t z) {
    return x | (y << 11) | (z << 22);
}
__host__ __device__ inline uint32_t pos_x(uint32_t p) { return p & 0x7FFu; }
__host__ __device__ inline uint32_t pos_y(uint32_t p) { return (p >> 11) & 0x7FFu; }
__host__ __device__ inline uint32_t pos_z(uint32_t p) { return p >> 22; }

// Occupancy mask rows are padded to a multiple of 16 bytes so the mask can be
// read by TMA (global strides must be multiples of 16 bytes).
__host__ __device__ inline int mask_pitch(int X) { return (X + 15) & ~15; }

// Per-cell state in HBM, structure of arrays over `cap` slots.  Hot arrays are
// read by the tick kernel; cold arrays only travel with cells (upload,
// compaction moves, births, download).
struct CellTable {
    uint32_t cap;
    float* internal;   // [16][cap]
    uint32_t* pos;     // [cap] packed position
    uint32_t* age;     // [cap]
    uint32_t* state;   // [cap] prep_remaining | quiescent << 16 | starter << 24
    float2* tp_rate;   // [8][cap]  (uptake_rate, secrete_rate)
    uint4* tp_idx;     // [cap]     8 x u16 (ext | int << 8)
    uint4* rx;         // [16][cap] (sub | prod<<8 | cat<<16 | cof<<24, k_m, v_max, k_cat)
    float2* ef_par;    // [8][cap]  (threshold, rate)
    uint4* ef_idx;     // [cap]     8 x u16 (int | ext << 8)
    float4* fate;      // [cap]     (division, death, quiescence, prep_ticks)
    uint64_t* lineage; // [cap]     cold
    float* cold;       // [cap][26] cold: receptors (24 floats), hgt_propensity, mutation_rate
    // per-tick schedule
    uint32_t* nb;      // [cap] bit f set: face f (spatial.rs FACE order) is an empty in-grid voxel
    int32_t* dep;      // [6][cap] dependency through face f: largest cell index < j touching that voxel, or -1
    uint32_t* done;    // [cap] epoch at which the cell finished this tick's update
    uint8_t* events;   // [cap]
};
constexpr int kColdFloats = 26;

// Simulation constants consumed by the field kernels.
struct FieldConsts {
    float dt_sub, alpha_eps, k_eps, c_max;
    float d_voxel[MARL_S_EXT];
    float lambda_decay[MARL_S_EXT];
    float src_ox, src_ca, src_re;      // additive source rates
    float prime_ox, prime_ca, prime_re; // Dirichlet values
    int source_mode;
    float surface_intensity, cell_factor, chemical_absorption, light_floor;
};

// Simulation constants consumed by the cell kernel.
struct CellConsts {
    float dt, c_max, epsilon, thr;
    float lambda_maintenance, reaction_maintenance, hard_death_floor;
    float base_division_prep, prep_maintenance_multiplier, rush_penalty_rate;
    uint32_t wait_limit;  // polls of a dependency flag before the wait gives up (kErrTimeoutDeps)
    float hill_lo, hill_hi;  // receptor Hill exponent clamp (receptor activations)
    uint32_t schedule_here;  // the cell loop computes the schedule itself (no schedule kernel ran)
};

struct Grid {
    int X, Y, Z;
    __host__ __device__ size_t V() const { return (size_t)X * Y * Z; }
};

// IEEE round-to-nearest division a / b.  The division itself never sees a
// zero numerator: it takes a slow path for one (measured ~250 cycles against
// ~45 on B200) and zeros are common in the field and in cell states.  For
// a == 0 the quotient is formed directly: a signed zero (sign of a XOR sign of
// b) when b is nonzero or infinite, a quiet NaN when b is zero or NaN.  The
// division always runs, on 1.5 in place of a zero numerator; the choice of
// numerator is made in inline PTX so the compiler cannot split the division
// into one per select arm (which would divide zero again).
__device__ __forceinline__ float div_rn(float a, float b) {
    const bool zero = a == 0.0f;
    float num;
    asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %3, 0;\n\tselp.f32 %0, %1, %2, p;\n\t}"
        : "=f"(num)
        : "f"(1.5f), "f"(a), "r"((unsigned)zero));
    const float q = num / b;
    const float zq = (b != b || b == 0.0f) ? __uint_as_float(0x7fc00000u)
                                           : __uint_as_float((__float_as_uint(a) ^ __float_as_uint(b)) & 0x80000000u);
    return zero ? zq : q;
}

// IEEE round-to-nearest division of the 12 values v[] by the same n = 3, 5
// or 6 (the empty-face count of a cell's gather and scatter).  With
// c = RN(1/n), q0 = RN(x c) is within one ulp of x/n, the remainder
// x - n q0 is exact in one FMA, and RN(q0 + r c) is the correctly rounded
// quotient (Markstein's theorem: P. Markstein, IBM J. Res. Dev. 34(1), 1990).
// Checked bitwise against the IEEE division over every finite float for each
// n (marl_selftest_small_division): it differs only for -0 (kept from q0,
// which has the right sign) and, for n = 6, below 2^-125.  So values that are
// zero use q0, and if any value is non-zero with a magnitude below 2^-125, or
// not finite, the 12 are divided by the IEEE operator instead.  Three
// branch-free FMAs per value instead of a division each, which the compiler
// would issue one after another.
__device__ __forceinline__ float small_divisor_inverse(int n) {
    return n == 3 ? 0x1.555556p-2f : (n == 5 ? 0x1.99999ap-3f : 0x1.555556p-3f);
}
__device__ __forceinline__ float div_small_n(float x, float c, float nf) {
    const float q0 = __fmul_rn(x, c);
    const float r = __fmaf_rn(-q0, nf, x);
    const float q1 = __fmaf_rn(r, c, q0);
    return x == 0.0f ? q0 : q1;
}
__device__ __forceinline__ void div12_small_n(float (&v)[12], int n) {
    const float nf = (float)n, c = small_divisor_inverse(n);
    bool exact = true;
#pragma unroll
    for (int s = 0; s < 12; ++s) {
        const float a = fabsf(v[s]);
        exact = exact && (v[s] == 0.0f || (a >= 0x1p-125f && a <= 3.40282346638528859812e38f));
    }
    if (exact) {
#pragma unroll
        for (int s = 0; s < 12; ++s) v[s] = div_small_n(v[s], c, nf);
    } else {
#pragma unroll
        for (int s = 0; s < 12; ++s) v[s] = div_rn(v[s], nf);
    }
}

// ---------------------------------------------------------------- PTX ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < kMbarSpinLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// 4-D tiled TMA load, global -> shared, completion on an mbarrier.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// 3-D tiled TMA load.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Acquire fence at GPU scope: with relaxed loads that observed release
// stores before it, it orders every later access after those stores' writers.
__device__ __forceinline__ void fence_acquire_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization may start while the previous kernel of its stream is still
// running, once every block of that kernel has called
// griddep_launch_dependents (or exited).  It must not touch global memory
// that the previous kernel reads or writes before griddep_wait() returns,
// which is when the previous kernel has completed and its writes are
// visible.  Without such a predecessor both are no-ops.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace marl
