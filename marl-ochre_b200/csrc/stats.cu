// Device-side statistics of a context: the quantities of print_stats and
// print_z_profile (crates/marl-sim/src/stats.rs:9-103), reduced on the GPU so
// that only a few hundred bytes cross to the host instead of the cell table
// and the field.
//
// Counts (population, per-z-third, per-z) and the centre-column samples are
// exact.  The averages of internal species 0, 5 and 6 and of the active
// reaction count are the ticks.csv columns of DataLogger::log_tick, which the
// reference accumulates in f64 (crates/marl-output/src/data.rs:207-232); they
// are summed in FP64 here too (per-thread partials, warp shuffles, one FP64
// atomic per block).  print_stats averages the same quantities with f32 sums
// (stats.rs:22-34); the FP64 result is the exact average up to FP64 rounding.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "ctx_impl.h"

using namespace marl;

namespace marl {

constexpr int kStatsThreads = 256;
constexpr int kStatsMaxZ = 1024;

struct StatsAccum {
    double energy_sum;
    double enzyme_sum;
    double enzyme_b_sum;
    double active_sum;
    unsigned long long thirds[3];
    unsigned long long per_z[kStatsMaxZ];
};

// thr: a reaction counts as active when |v_max| > thr (stats.rs:31 uses 1e-9).
__global__ void __launch_bounds__(kStatsThreads) k_cell_stats(CellTable t, uint32_t n, int Z, float thr,
                                                             StatsAccum* __restrict__ acc) {
    __shared__ unsigned int s_z[kStatsMaxZ];
    __shared__ unsigned int s_third[3];
    for (int i = threadIdx.x; i < Z; i += blockDim.x) s_z[i] = 0;
    if (threadIdx.x < 3) s_third[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t z_third = (uint32_t)(Z / 3);
    double e = 0.0, enz = 0.0, enzb = 0.0, act = 0.0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        e += (double)t.internal[j];                 // internal[0]
        enz += (double)t.internal[5 * (size_t)t.cap + j];
        enzb += (double)t.internal[6 * (size_t)t.cap + j];
        int a = 0;
#pragma unroll
        for (int r = 0; r < MARL_R_MAX; ++r) a += fabsf(__uint_as_float(t.rx[(size_t)r * t.cap + j].z)) > thr ? 1 : 0;
        act += (double)a;
        const uint32_t z = pos_z(t.pos[j]);
        atomicAdd(&s_z[z], 1u);
        atomicAdd(&s_third[z < z_third ? 0 : (z < 2 * z_third ? 1 : 2)], 1u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xFFFFFFFFu, e, o);
        enz += __shfl_xor_sync(0xFFFFFFFFu, enz, o);
        enzb += __shfl_xor_sync(0xFFFFFFFFu, enzb, o);
        act += __shfl_xor_sync(0xFFFFFFFFu, act, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc->energy_sum, e);
        atomicAdd(&acc->enzyme_sum, enz);
        atomicAdd(&acc->enzyme_b_sum, enzb);
        atomicAdd(&acc->active_sum, act);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < Z; i += blockDim.x)
        if (s_z[i]) atomicAdd(&acc->per_z[i], (unsigned long long)s_z[i]);
    if (threadIdx.x < 3 && s_third[threadIdx.x]) atomicAdd(&acc->thirds[threadIdx.x], (unsigned long long)s_third[threadIdx.x]);
}

// Centre column (X/2, Y/2) of the light and of species 1-4, [5][Z].
__global__ void k_centre_column(const float* __restrict__ field, const float* __restrict__ light, Grid g,
                                float* __restrict__ out) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= g.Z) return;
    const size_t v = ((size_t)z * g.Y + g.Y / 2) * g.X + g.X / 2;
    out[z] = light[v];
    for (int s = 1; s <= 4; ++s) out[(size_t)s * g.Z + z] = field[v * 12 + s];
}

}  // namespace marl

extern "C" {

marl_status marl_ctx_stats(marl_ctx* c, marl_stats* out, uint32_t* cells_per_z, float* centre_column) {
    if (!c || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->g.Z > kStatsMaxZ) return fail(MARL_ERR_INVALID_INPUT, "Z %d above %d", c->g.Z, kStatsMaxZ);
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    const Grid g = c->g;
    cudaStream_t s = c->stream;
    StatsAccum* d = nullptr;
    float* col = nullptr;
    const size_t col_bytes = (size_t)5 * g.Z * 4;
    if (cudaMallocAsync((void**)&d, sizeof(StatsAccum), s) != cudaSuccess ||
        cudaMallocAsync((void**)&col, col_bytes, s) != cudaSuccess) {
        if (d) cudaFreeAsync(d, s);
        return fail(MARL_ERR_OUT_OF_MEMORY, "stats buffers");
    }
    cudaError_t e = cudaMemsetAsync(d, 0, sizeof(StatsAccum), s);
    if (e == cudaSuccess && c->n) {
        const uint32_t blocks = (c->n + kStatsThreads - 1) / kStatsThreads;
        k_cell_stats<<<blocks < 592u ? blocks : 592u, kStatsThreads, 0, s>>>(c->t, c->n, g.Z, 1e-9f, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_centre_column<<<(g.Z + 127) / 128, 128, 0, s>>>(c->field[c->cur], c->light, g, col);
        e = cudaGetLastError();
    }
    StatsAccum h;
    std::vector<float> hc((size_t)5 * g.Z);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), col, col_bytes, cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d, s);
    cudaFreeAsync(col, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "marl_ctx_stats");
    c->d2h_bytes += sizeof(h) + col_bytes;
    std::memset(out, 0, sizeof(*out));
    out->population = c->n;
    out->top = h.thirds[0];
    out->middle = h.thirds[1];
    out->bottom = h.thirds[2];
    if (c->n) {
        out->avg_energy = h.energy_sum / c->n;
        out->avg_enzyme = h.enzyme_sum / c->n;
        out->avg_enzyme_b = h.enzyme_b_sum / c->n;
        out->avg_active_reactions = h.active_sum / c->n;
    }
    const int zm = g.Z / 2;
    out->oxidant_top = hc[(size_t)1 * g.Z + 0];
    out->oxidant_middle = hc[(size_t)1 * g.Z + zm];
    out->reductant_bottom = hc[(size_t)2 * g.Z + g.Z - 1];
    out->organic_middle = hc[(size_t)4 * g.Z + zm];
    if (cells_per_z)
        for (int z = 0; z < g.Z; ++z) cells_per_z[z] = (uint32_t)h.per_z[z];
    if (centre_column) std::memcpy(centre_column, hc.data(), col_bytes);
    return MARL_OK;
}

}  // extern "C"
