// Host-side interface of the surrogate's tensor-core kernels (mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/marl_cuda.h"

namespace marl {
namespace mlp {

constexpr int kIn = MARL_SURR_FEATURES;  // 93 features
constexpr int kInPad = 128;              // first-layer K, zero-padded
constexpr int kHid = 256;
constexpr int kOut = 16;
constexpr int kOutPad = 64;              // K of the output layer's input-gradient GEMM

// Flat parameter layout (FP32 master copy, gradients, Adam moments).
constexpr uint32_t kOffW1 = 0;
constexpr uint32_t kOffB1 = kOffW1 + kHid * kInPad;
constexpr uint32_t kOffW2 = kOffB1 + kHid;
constexpr uint32_t kOffB2 = kOffW2 + kHid * kHid;
constexpr uint32_t kOffW3 = kOffB2 + kHid;
constexpr uint32_t kOffB3 = kOffW3 + kOut * kHid;
constexpr uint32_t kParams = kOffB3 + kOut;
static_assert(kParams == MARL_SURR_PARAMS, "parameter layout");

#ifdef __CUDACC__
// Feature transform before standardisation: log(|v| + 1e-3) for k_m, v_max
// and k_cat (features 29 + 4r + {0, 1, 2}), identity otherwise.
__device__ __forceinline__ float feature_transform(int f, float v) {
    if (f >= 29 && ((f - 29) & 3) != 3) return logf(fabsf(v) + 1e-3f);
    return v;
}
#endif

enum Epi : int { EPI_BIAS_GELU = 0, EPI_BIAS_OUT = 1, EPI_GELU_BWD = 2, EPI_ATOMIC = 3, EPI_BIAS_GELU_FAST = 4 };

struct GemmArgs {
    const __nv_bfloat16* A = nullptr;  // [M][lda], K contiguous
    int lda = 0;
    const __nv_bfloat16* B = nullptr;  // [N][ldb], K contiguous
    int ldb = 0;
    int M = 0, N = 0, K = 0;
    int k_per_split = 0;               // 0: whole K in one CTA (split-K only with EPI_ATOMIC)
    const float* bias = nullptr;       // [N]
    const float* scale = nullptr;      // [N] optional (EPI_BIAS_OUT)
    const float* shift = nullptr;      // [N] with scale
    __nv_bfloat16* out_bf = nullptr;   // [M][ldo]
    int ldo = 0;
    __nv_bfloat16* out_t = nullptr;    // [N][ldt] transposed BF16 copy
    int ldt = 0;
    float* out_f = nullptr;            // FP32 output / pre-activation / atomic target
    int ldf = 0;
    int out_col_major = 0;             // out_f as [N][ldf] (EPI_BIAS_OUT, EPI_ATOMIC)
    const float* z_in = nullptr;       // [M][ldz] pre-activation (EPI_GELU_BWD)
    int ldz = 0;
    float* colsum = nullptr;           // [N] column sums of the output (EPI_GELU_BWD)
    uint32_t* err = nullptr;           // kErr* bits on a wait timeout
};

// Arguments of the fused inference kernel: standardised BF16 inputs x
// [M][128], BF16 weights, FP32 biases, de-standardisation, and the output
// y [16][ldy] (species-major).
struct FusedArgs {
    const __nv_bfloat16* x = nullptr;
    int M = 0;
    const __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    const float *b1 = nullptr, *b2 = nullptr, *b3 = nullptr;
    const float *scale = nullptr, *shift = nullptr;
    float* y = nullptr;
    uint32_t ldy = 0;
    uint32_t* err = nullptr;
};
cudaError_t launch_mlp_fused(const FusedArgs& a, int num_sms, cudaStream_t s);

// bn: 16, 128 or 256 (the instantiated tile widths for each epilogue).
cudaError_t launch_gemm(const GemmArgs& a, int bn, int epi, cudaStream_t s);
cudaError_t launch_loss(const float* y, const float* t, uint32_t B, __nv_bfloat16* dy, __nv_bfloat16* dyt,
                        float* db3, float* loss_sum, cudaStream_t s);
cudaError_t launch_gather_batch(const __nv_bfloat16* X, const float* T, uint32_t n_rows, uint64_t seed, uint64_t step,
                                uint32_t B, __nv_bfloat16* xb, __nv_bfloat16* xbt, float* tb, cudaStream_t s);
cudaError_t launch_transpose_batch(const __nv_bfloat16* xb, uint32_t B, __nv_bfloat16* xbt, cudaStream_t s);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                        uint64_t t, cudaStream_t s);
cudaError_t launch_weights_bf16(const float* p, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3,
                                __nv_bfloat16* w2t, __nv_bfloat16* w3t, cudaStream_t s);
cudaError_t launch_raw_stats(const float* raw, uint32_t n, double* acc, cudaStream_t s);
cudaError_t launch_standardise(const float* raw, uint32_t n, const float* norm, __nv_bfloat16* X, float* T,
                               cudaStream_t s);
cudaError_t launch_eval_rows(const float* raw, const float* pred, uint32_t ldp, uint32_t n, const float* norm,
                             float tol, float c_max, float* err_out, double* acc, uint32_t* max_bits,
                             cudaStream_t s);
cudaError_t launch_init_weights(float* p, uint64_t seed, cudaStream_t s);

}  // namespace mlp
}  // namespace marl
