// Definition of the opaque marl_surrogate and the calls the context's tick
// makes into it (surrogate.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/marl_cuda.h"
#include "mlp.h"

struct marl_surrogate {
    int device = 0;
    int num_sms = 0;
    bool fused = true;  // inference through the fused persistent kernel (else three GEMM launches)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    marl_surrogate_config cfg{};

    float* raw = nullptr;  // [max_pairs][MARL_SURR_RAW_STRIDE] raw pair store
    uint32_t rows = 0;     // rows captured or uploaded

    bool prepared = false;
    uint32_t n_prepared = 0;  // rows standardised into X / T
    uint32_t n_train = 0;
    __nv_bfloat16* X = nullptr;  // [n_prepared][128]
    float* T = nullptr;          // [n_prepared][16]
    float* norm = nullptr;       // device: in_mean, in_std, out_mean, out_std
    float h_norm[MARL_SURR_NORM] = {};

    float* p = nullptr;  // FP32 master parameters
    float* g = nullptr;  // gradients
    float* m = nullptr;  // Adam moments
    float* v = nullptr;
    __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *w2t = nullptr, *w3t = nullptr;
    uint64_t adam_t = 0;
    uint64_t batches = 0;  // batch counter (sampling stream)

    // Training work buffers for `work_b` rows.
    uint32_t work_b = 0;
    __nv_bfloat16 *xb = nullptr, *xbt = nullptr, *h1 = nullptr, *h1t = nullptr, *h2 = nullptr, *h2t = nullptr;
    __nv_bfloat16 *dy = nullptr, *dyt = nullptr, *dz2 = nullptr, *dz2t = nullptr, *dz1 = nullptr, *dz1t = nullptr;
    float *tb = nullptr, *z1 = nullptr, *z2 = nullptr, *y = nullptr;

    // Inference work buffers for `infer_rows` rows.
    uint32_t infer_rows = 0;
    __nv_bfloat16 *ih1 = nullptr, *ih2 = nullptr;

    float* d_scalars = nullptr;  // per-step loss sums (train) / scratch
    uint32_t scalars_cap = 0;
    double* d_acc = nullptr;     // statistics / evaluation accumulators (256 doubles)
    uint32_t* d_err = nullptr;   // kErr* bits of the GEMMs (index 0), max-error bits (index 1)
};

namespace marl {
// Forward pass of the prepared network on standardised BF16 rows x [n][128]
// into de-standardised deltas y [16][ldy], ordered on `stream`.
marl_status surrogate_infer(marl_surrogate* s, const __nv_bfloat16* x, uint32_t n, float* y, uint32_t ldy,
                            cudaStream_t stream);
}  // namespace marl
