// C ABI of the learned reaction surrogate: pair store, standardisation,
// training (forward, backward, Adam on the tcgen05 GEMM of mlp.cu),
// evaluation, inference, and the hooks of a context's cell loop.
//
// Training step on a batch of B rows (all GEMMs C = A * B^T, K-major):
//   h1 = gelu(x W1^T + b1)        A = x [B][128],     B = W1 [256][128]
//   h2 = gelu(h1 W2^T + b2)       A = h1 [B][256],    B = W2 [256][256]
//   y  = h2 W3^T + b3             A = h2 [B][256],    B = W3 [16][256]
//   dy = 2 (y - t) / (16 B)
//   dW3^T = h2^T dy               A = h2^T [256][B],  B = dy^T [16][B]
//   dz2 = (dy W3) * gelu'(z2)     A = dy [B][64],     B = W3^T [256][64]
//   dW2 = dz2^T h1                A = dz2^T [256][B], B = h1^T [256][B]
//   dz1 = (dz2 W2) * gelu'(z1)    A = dz2 [B][256],   B = W2^T [256][256]
//   dW1 = dz1^T x                 A = dz1^T [256][B], B = x^T [128][B]
// Weight gradients use split-K with FP32 atomic accumulation; bias gradients
// are column sums taken in the epilogues.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ctx_impl.h"
#include "surrogate.h"

using namespace marl;

namespace marl {

#define SCK(expr)                                             \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr);   \
    } while (0)

static constexpr int kSplitK = 512;

static void free_all(std::initializer_list<void*> ptrs) {
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

static marl_status ensure_work(marl_surrogate* s, uint32_t B) {
    if (B <= s->work_b) return MARL_OK;
    cudaStreamSynchronize(s->stream);
    free_all({s->xb, s->xbt, s->h1, s->h1t, s->h2, s->h2t, s->dy, s->dyt, s->dz2, s->dz2t, s->dz1, s->dz1t, s->tb,
              s->z1, s->z2, s->y});
    s->work_b = 0;
    const size_t b = B;
    SCK(cudaMalloc((void**)&s->xb, b * mlp::kInPad * 2));
    SCK(cudaMalloc((void**)&s->xbt, b * mlp::kInPad * 2));
    SCK(cudaMalloc((void**)&s->h1, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->h1t, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->h2, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->h2t, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->dy, b * mlp::kOutPad * 2));
    SCK(cudaMalloc((void**)&s->dyt, b * mlp::kOut * 2));
    SCK(cudaMalloc((void**)&s->dz2, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->dz2t, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->dz1, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->dz1t, b * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->tb, b * mlp::kOut * 4));
    SCK(cudaMalloc((void**)&s->z1, b * mlp::kHid * 4));
    SCK(cudaMalloc((void**)&s->z2, b * mlp::kHid * 4));
    SCK(cudaMalloc((void**)&s->y, b * mlp::kOut * 4));
    s->work_b = B;
    return MARL_OK;
}

static marl_status ensure_infer(marl_surrogate* s, uint32_t n) {
    if (n <= s->infer_rows) return MARL_OK;
    cudaStreamSynchronize(s->stream);
    free_all({s->ih1, s->ih2});
    s->ih1 = s->ih2 = nullptr;
    s->infer_rows = 0;
    const size_t rows = ((size_t)n + 127) / 128 * 128;
    SCK(cudaMalloc((void**)&s->ih1, rows * mlp::kHid * 2));
    SCK(cudaMalloc((void**)&s->ih2, rows * mlp::kHid * 2));
    s->infer_rows = (uint32_t)rows;
    return MARL_OK;
}

static marl_status ensure_scalars(marl_surrogate* s, uint32_t n) {
    if (n <= s->scalars_cap) return MARL_OK;
    cudaStreamSynchronize(s->stream);
    if (s->d_scalars) cudaFree(s->d_scalars);
    s->d_scalars = nullptr;
    s->scalars_cap = 0;
    SCK(cudaMalloc((void**)&s->d_scalars, (size_t)n * 4));
    s->scalars_cap = n;
    return MARL_OK;
}

static marl_status gemm(const mlp::GemmArgs& a, int bn, int epi, cudaStream_t st) {
    SCK(mlp::launch_gemm(a, bn, epi, st));
    return MARL_OK;
}

#define SST(expr)                                   \
    do {                                            \
        marl_status _s = (expr);                    \
        if (_s != MARL_OK) return _s;               \
    } while (0)

// Forward of the first two layers for training (keeps z, h and h^T).
static marl_status forward_train(marl_surrogate* s, uint32_t B) {
    cudaStream_t st = s->stream;
    mlp::GemmArgs a;
    a.err = s->d_err;
    a.A = s->xb, a.lda = mlp::kInPad, a.B = s->w1, a.ldb = mlp::kInPad;
    a.M = (int)B, a.N = mlp::kHid, a.K = mlp::kInPad;
    a.bias = s->p + mlp::kOffB1, a.out_bf = s->h1, a.ldo = mlp::kHid, a.out_t = s->h1t, a.ldt = (int)B;
    a.out_f = s->z1, a.ldf = mlp::kHid;
    SST(gemm(a, 256, mlp::EPI_BIAS_GELU, st));
    a.A = s->h1, a.lda = mlp::kHid, a.B = s->w2, a.ldb = mlp::kHid, a.K = mlp::kHid;
    a.bias = s->p + mlp::kOffB2, a.out_bf = s->h2, a.out_t = s->h2t, a.out_f = s->z2;
    SST(gemm(a, 256, mlp::EPI_BIAS_GELU, st));
    mlp::GemmArgs o;
    o.err = s->d_err;
    o.A = s->h2, o.lda = mlp::kHid, o.B = s->w3, o.ldb = mlp::kHid;
    o.M = (int)B, o.N = mlp::kOut, o.K = mlp::kHid;
    o.bias = s->p + mlp::kOffB3, o.out_f = s->y, o.ldf = mlp::kOut;
    SST(gemm(o, 16, mlp::EPI_BIAS_OUT, st));
    return MARL_OK;
}

// Gradients into s->g (zeroed here) from the batch in xb/xbt/tb; the loss
// sum is added to *loss_sum.
static marl_status backward(marl_surrogate* s, uint32_t B, float* loss_sum) {
    cudaStream_t st = s->stream;
    SCK(cudaMemsetAsync(s->g, 0, (size_t)mlp::kParams * 4, st));
    SCK(mlp::launch_loss(s->y, s->tb, B, s->dy, s->dyt, s->g + mlp::kOffB3, loss_sum, st));
    const int kps = (int)B < kSplitK ? (int)B : kSplitK;
    {  // dW3^T [256][16] = h2^T dy, stored as dW3 [16][256]
        mlp::GemmArgs a;
        a.err = s->d_err;
        a.A = s->h2t, a.lda = (int)B, a.B = s->dyt, a.ldb = (int)B;
        a.M = mlp::kHid, a.N = mlp::kOut, a.K = (int)B, a.k_per_split = kps;
        a.out_f = s->g + mlp::kOffW3, a.ldf = mlp::kHid, a.out_col_major = 1;
        SST(gemm(a, 16, mlp::EPI_ATOMIC, st));
    }
    {  // dz2 = (dy W3) * gelu'(z2)
        mlp::GemmArgs a;
        a.err = s->d_err;
        a.A = s->dy, a.lda = mlp::kOutPad, a.B = s->w3t, a.ldb = mlp::kOutPad;
        a.M = (int)B, a.N = mlp::kHid, a.K = mlp::kOutPad;
        a.z_in = s->z2, a.ldz = mlp::kHid, a.out_bf = s->dz2, a.ldo = mlp::kHid, a.out_t = s->dz2t, a.ldt = (int)B;
        a.colsum = s->g + mlp::kOffB2;
        SST(gemm(a, 256, mlp::EPI_GELU_BWD, st));
    }
    {  // dW2 [256][256] = dz2^T h1
        mlp::GemmArgs a;
        a.err = s->d_err;
        a.A = s->dz2t, a.lda = (int)B, a.B = s->h1t, a.ldb = (int)B;
        a.M = mlp::kHid, a.N = mlp::kHid, a.K = (int)B, a.k_per_split = kps;
        a.out_f = s->g + mlp::kOffW2, a.ldf = mlp::kHid;
        SST(gemm(a, 256, mlp::EPI_ATOMIC, st));
    }
    {  // dz1 = (dz2 W2) * gelu'(z1)
        mlp::GemmArgs a;
        a.err = s->d_err;
        a.A = s->dz2, a.lda = mlp::kHid, a.B = s->w2t, a.ldb = mlp::kHid;
        a.M = (int)B, a.N = mlp::kHid, a.K = mlp::kHid;
        a.z_in = s->z1, a.ldz = mlp::kHid, a.out_bf = s->dz1, a.ldo = mlp::kHid, a.out_t = s->dz1t, a.ldt = (int)B;
        a.colsum = s->g + mlp::kOffB1;
        SST(gemm(a, 256, mlp::EPI_GELU_BWD, st));
    }
    {  // dW1 [256][128] = dz1^T x
        mlp::GemmArgs a;
        a.err = s->d_err;
        a.A = s->dz1t, a.lda = (int)B, a.B = s->xbt, a.ldb = (int)B;
        a.M = mlp::kHid, a.N = mlp::kInPad, a.K = (int)B, a.k_per_split = kps;
        a.out_f = s->g + mlp::kOffW1, a.ldf = mlp::kInPad;
        SST(gemm(a, 128, mlp::EPI_ATOMIC, st));
    }
    return MARL_OK;
}

static marl_status check_err(marl_surrogate* s) {
    uint32_t err = 0;
    SCK(cudaMemcpyAsync(&err, s->d_err, 4, cudaMemcpyDeviceToHost, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    if (err) {
        cudaMemsetAsync(s->d_err, 0, 4, s->stream);
        return fail(MARL_ERR_TIMEOUT, "surrogate kernel wait gave up (error bits 0x%x)", err);
    }
    return MARL_OK;
}

marl_status surrogate_infer(marl_surrogate* s, const __nv_bfloat16* x, uint32_t n, float* y, uint32_t ldy,
                            cudaStream_t stream) {
    if (!s->prepared) return fail(MARL_ERR_STATE, "surrogate not prepared (marl_surrogate_prepare)");
    if (n == 0) return MARL_OK;
    if (s->fused) {
        mlp::FusedArgs f;
        f.x = x, f.M = (int)n, f.w1 = s->w1, f.w2 = s->w2, f.w3 = s->w3;
        f.b1 = s->p + mlp::kOffB1, f.b2 = s->p + mlp::kOffB2, f.b3 = s->p + mlp::kOffB3;
        f.scale = s->norm + 2 * mlp::kIn + mlp::kOut, f.shift = s->norm + 2 * mlp::kIn;
        f.y = y, f.ldy = ldy, f.err = s->d_err;
        SCK(mlp::launch_mlp_fused(f, s->num_sms, stream));
        return MARL_OK;
    }
    SST(ensure_infer(s, n));
    mlp::GemmArgs a;
    a.err = s->d_err;
    a.A = x, a.lda = mlp::kInPad, a.B = s->w1, a.ldb = mlp::kInPad;
    a.M = (int)n, a.N = mlp::kHid, a.K = mlp::kInPad;
    a.bias = s->p + mlp::kOffB1, a.out_bf = s->ih1, a.ldo = mlp::kHid;
    SST(gemm(a, 256, mlp::EPI_BIAS_GELU_FAST, stream));
    a.A = s->ih1, a.lda = mlp::kHid, a.B = s->w2, a.ldb = mlp::kHid, a.K = mlp::kHid;
    a.bias = s->p + mlp::kOffB2, a.out_bf = s->ih2;
    SST(gemm(a, 256, mlp::EPI_BIAS_GELU_FAST, stream));
    mlp::GemmArgs o;
    o.err = s->d_err;
    o.A = s->ih2, o.lda = mlp::kHid, o.B = s->w3, o.ldb = mlp::kHid;
    o.M = (int)n, o.N = mlp::kOut, o.K = mlp::kHid;
    o.bias = s->p + mlp::kOffB3, o.scale = s->norm + 2 * mlp::kIn + mlp::kOut, o.shift = s->norm + 2 * mlp::kIn;
    o.out_f = y, o.ldf = (int)ldy, o.out_col_major = 1;
    SST(gemm(o, 16, mlp::EPI_BIAS_OUT, stream));
    return MARL_OK;
}

}  // namespace marl

// ================================================================= ABI ====
extern "C" {

marl_status marl_surrogate_config_default(marl_surrogate_config* c) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null config");
    c->max_pairs = 1u << 22;
    c->batch = 8192;
    c->lr = 1e-3f;
    c->beta1 = 0.9f;
    c->beta2 = 0.999f;
    c->adam_eps = 1e-8f;
    c->seed = 1;
    return MARL_OK;
}

void marl_surrogate_destroy(marl_surrogate* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_all({s->raw, s->X, s->T, s->norm, s->p, s->g, s->m, s->v, s->w1, s->w2, s->w3, s->w2t, s->w3t, s->xb,
              s->xbt, s->h1, s->h1t, s->h2, s->h2t, s->dy, s->dyt, s->dz2, s->dz2t, s->dz1, s->dz1t, s->tb, s->z1,
              s->z2, s->y, s->ih1, s->ih2, s->d_scalars, s->d_acc, s->d_err});
    if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
}

marl_status marl_surrogate_create(const marl_surrogate_config* cfg, marl_surrogate** out) {
    if (!cfg || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *out = nullptr;
    if (cfg->max_pairs == 0 || cfg->batch == 0 || cfg->batch % 128)
        return fail(MARL_ERR_INVALID_INPUT, "max_pairs must be > 0 and batch a positive multiple of 128");
    int dev = 0, sms = 0;
    marl_status st = check_device(&dev, &sms);
    if (st) return st;
    marl_surrogate* s = new marl_surrogate();
    s->device = dev;
    s->num_sms = sms;
    s->cfg = *cfg;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    s->own_stream = e == cudaSuccess;
    auto bad = [&](cudaError_t err, const char* where) {
        marl_status r = cuda_fail(err, where);
        marl_surrogate_destroy(s);
        return r;
    };
    if (e != cudaSuccess) return bad(e, "cudaStreamCreate");
    const size_t P = mlp::kParams;
    if ((e = cudaMalloc((void**)&s->raw, (size_t)cfg->max_pairs * MARL_SURR_RAW_STRIDE * 4))) return bad(e, "pair store");
    for (float** p : {&s->p, &s->g, &s->m, &s->v})
        if ((e = cudaMalloc((void**)p, P * 4))) return bad(e, "parameters");
    if ((e = cudaMalloc((void**)&s->w1, (size_t)mlp::kHid * mlp::kInPad * 2)) ||
        (e = cudaMalloc((void**)&s->w2, (size_t)mlp::kHid * mlp::kHid * 2)) ||
        (e = cudaMalloc((void**)&s->w3, (size_t)mlp::kOut * mlp::kHid * 2)) ||
        (e = cudaMalloc((void**)&s->w2t, (size_t)mlp::kHid * mlp::kHid * 2)) ||
        (e = cudaMalloc((void**)&s->w3t, (size_t)mlp::kHid * mlp::kOutPad * 2)) ||
        (e = cudaMalloc((void**)&s->norm, MARL_SURR_NORM * 4)) || (e = cudaMalloc((void**)&s->d_acc, 256 * 8)) ||
        (e = cudaMalloc((void**)&s->d_err, 16)))
        return bad(e, "surrogate buffers");
    cudaMemsetAsync(s->m, 0, P * 4, s->stream);
    cudaMemsetAsync(s->v, 0, P * 4, s->stream);
    cudaMemsetAsync(s->d_err, 0, 16, s->stream);
    if ((e = mlp::launch_init_weights(s->p, cfg->seed, s->stream))) return bad(e, "init weights");
    if ((e = mlp::launch_weights_bf16(s->p, s->w1, s->w2, s->w3, s->w2t, s->w3t, s->stream))) return bad(e, "bf16 weights");
    if ((e = cudaStreamSynchronize(s->stream))) return bad(e, "surrogate create");
    *out = s;
    return MARL_OK;
}

marl_status marl_surrogate_set_stream(marl_surrogate* s, void* stream) {
    if (!s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    SCK(cudaStreamSynchronize(s->stream));
    if (s->own_stream) SCK(cudaStreamDestroy(s->stream));
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
    return MARL_OK;
}

marl_status marl_surrogate_pair_count(marl_surrogate* s, uint32_t* rows) {
    if (!s || !rows) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *rows = s->rows;
    return MARL_OK;
}

marl_status marl_surrogate_download_pairs(marl_surrogate* s, uint32_t row0, uint32_t n, float* out) {
    if (!s || (!out && n)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if ((uint64_t)row0 + n > s->rows) return fail(MARL_ERR_INVALID_INPUT, "rows %u+%u beyond %u", row0, n, s->rows);
    SCK(cudaStreamSynchronize(s->stream));
    SCK(cudaMemcpy(out, s->raw + (size_t)row0 * MARL_SURR_RAW_STRIDE, (size_t)n * MARL_SURR_RAW_STRIDE * 4,
                   cudaMemcpyDeviceToHost));
    return MARL_OK;
}

marl_status marl_surrogate_upload_pairs(marl_surrogate* s, const float* rows, uint32_t n) {
    if (!s || (!rows && n)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if ((uint64_t)s->rows + n > s->cfg.max_pairs)
        return fail(MARL_ERR_CAPACITY, "pair store holds %u rows", s->cfg.max_pairs);
    // Ordered on the surrogate's stream (the kernels that read the rows run there).
    SCK(cudaMemcpyAsync(s->raw + (size_t)s->rows * MARL_SURR_RAW_STRIDE, rows, (size_t)n * MARL_SURR_RAW_STRIDE * 4,
                        cudaMemcpyHostToDevice, s->stream));
    SCK(cudaStreamSynchronize(s->stream));
    s->rows += n;
    return MARL_OK;
}

marl_status marl_surrogate_prepare(marl_surrogate* s, uint32_t n_train) {
    if (!s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    if (n_train == 0 || n_train > s->rows)
        return fail(MARL_ERR_INVALID_INPUT, "n_train %u must be in [1, %u]", n_train, s->rows);
    cudaStream_t st = s->stream;
    constexpr int kCols = mlp::kIn + mlp::kOut;
    SCK(cudaMemsetAsync(s->d_acc, 0, 2 * kCols * 8, st));
    SCK(mlp::launch_raw_stats(s->raw, n_train, s->d_acc, st));
    double acc[2 * kCols];
    SCK(cudaMemcpyAsync(acc, s->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    for (int i = 0; i < kCols; ++i) {
        const double mean = acc[i] / n_train;
        double var = acc[kCols + i] / n_train - mean * mean;
        double sd = var > 0 ? std::sqrt(var) : 0.0;
        if (!(sd > 1e-6)) sd = 1.0;  // constant column: pass through centred
        if (i < mlp::kIn) {
            s->h_norm[i] = (float)mean;
            s->h_norm[mlp::kIn + i] = (float)sd;
        } else {
            s->h_norm[2 * mlp::kIn + (i - mlp::kIn)] = (float)mean;
            s->h_norm[2 * mlp::kIn + mlp::kOut + (i - mlp::kIn)] = (float)sd;
        }
    }
    SCK(cudaMemcpyAsync(s->norm, s->h_norm, sizeof(s->h_norm), cudaMemcpyHostToDevice, st));
    if (s->n_prepared < s->rows) {
        free_all({s->X, s->T});
        s->X = nullptr;
        s->T = nullptr;
        s->n_prepared = 0;
        SCK(cudaMalloc((void**)&s->X, (size_t)s->rows * mlp::kInPad * 2));
        SCK(cudaMalloc((void**)&s->T, (size_t)s->rows * mlp::kOut * 4));
    }
    SCK(mlp::launch_standardise(s->raw, s->rows, s->norm, s->X, s->T, st));
    SCK(cudaStreamSynchronize(st));
    s->n_prepared = s->rows;
    s->n_train = n_train;
    s->prepared = true;
    return MARL_OK;
}

marl_status marl_surrogate_train(marl_surrogate* s, uint32_t steps, float* loss_out) {
    if (!s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    if (!s->prepared) return fail(MARL_ERR_STATE, "surrogate not prepared (marl_surrogate_prepare)");
    if (steps == 0) return MARL_OK;
    const uint32_t B = s->cfg.batch;
    marl_status st = ensure_work(s, B);
    if (st) return st;
    if ((st = ensure_scalars(s, steps))) return st;
    cudaStream_t cs = s->stream;
    SCK(cudaMemsetAsync(s->d_scalars, 0, (size_t)steps * 4, cs));
    for (uint32_t i = 0; i < steps; ++i) {
        SCK(mlp::launch_gather_batch(s->X, s->T, s->n_train, s->cfg.seed, s->batches++, B, s->xb, s->xbt, s->tb, cs));
        SST(forward_train(s, B));
        SST(backward(s, B, s->d_scalars + i));
        ++s->adam_t;
        SCK(mlp::launch_adam(s->p, s->g, s->m, s->v, s->cfg.lr, s->cfg.beta1, s->cfg.beta2, s->cfg.adam_eps,
                             s->adam_t, cs));
        SCK(mlp::launch_weights_bf16(s->p, s->w1, s->w2, s->w3, s->w2t, s->w3t, cs));
    }
    if (loss_out) {
        SCK(cudaMemcpyAsync(loss_out, s->d_scalars, (size_t)steps * 4, cudaMemcpyDeviceToHost, cs));
    }
    SST(check_err(s));
    if (loss_out)
        for (uint32_t i = 0; i < steps; ++i) loss_out[i] /= (float)B * mlp::kOut;
    return MARL_OK;
}

marl_status marl_surrogate_set_inference(marl_surrogate* s, int32_t fused) {
    if (!s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    s->fused = fused != 0;
    return MARL_OK;
}

marl_status marl_surrogate_set_lr(marl_surrogate* s, float lr) {
    if (!s || !(lr > 0.0f)) return fail(MARL_ERR_INVALID_INPUT, "null surrogate or lr <= 0");
    s->cfg.lr = lr;
    return MARL_OK;
}

marl_status marl_surrogate_evaluate(marl_surrogate* s, uint32_t row0, uint32_t n, float tol, marl_surrogate_eval* out,
                                    float* row_err_out) {
    if (!s || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (!s->prepared) return fail(MARL_ERR_STATE, "surrogate not prepared (marl_surrogate_prepare)");
    if (n == 0 || (uint64_t)row0 + n > s->n_prepared)
        return fail(MARL_ERR_INVALID_INPUT, "rows %u+%u beyond the %u prepared rows", row0, n, s->n_prepared);
    cudaStream_t cs = s->stream;
    float* pred = nullptr;
    float* errs = nullptr;
    SCK(cudaMalloc((void**)&pred, (size_t)n * mlp::kOut * 4));
    if (row_err_out && cudaMalloc((void**)&errs, (size_t)n * 4) != cudaSuccess) {
        cudaFree(pred);
        return fail(MARL_ERR_OUT_OF_MEMORY, "evaluation buffers");
    }
    marl_status st = surrogate_infer(s, s->X + (size_t)row0 * mlp::kInPad, n, pred, n, cs);
    double acc[3] = {0, 0, 0};
    uint32_t maxb = 0;
    if (!st) {
        cudaMemsetAsync(s->d_acc, 0, 3 * 8, cs);
        cudaMemsetAsync(s->d_err + 1, 0, 4, cs);
        cudaError_t e = mlp::launch_eval_rows(s->raw + (size_t)row0 * MARL_SURR_RAW_STRIDE, pred, n, n, s->norm, tol,
                                              10.0f, errs, s->d_acc, s->d_err + 1, cs);
        if (e) st = cuda_fail(e, "evaluate");
        if (!st) {
            cudaMemcpyAsync(acc, s->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, cs);
            cudaMemcpyAsync(&maxb, s->d_err + 1, 4, cudaMemcpyDeviceToHost, cs);
            if (row_err_out) cudaMemcpyAsync(row_err_out, errs, (size_t)n * 4, cudaMemcpyDeviceToHost, cs);
            st = check_err(s);
        }
    }
    cudaStreamSynchronize(cs);
    cudaFree(pred);
    if (errs) cudaFree(errs);
    if (st) return st;
    out->rows = n;
    out->accepted = (uint32_t)acc[0];
    out->mean_err = (float)(acc[1] / n);
    std::memcpy(&out->max_err, &maxb, 4);
    out->mse_normalised = (float)(acc[2] / ((double)n * mlp::kOut));
    return MARL_OK;
}

marl_status marl_surrogate_get_weights(marl_surrogate* s, float* params, float* norm) {
    if (!s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    SCK(cudaStreamSynchronize(s->stream));
    if (params) SCK(cudaMemcpy(params, s->p, (size_t)mlp::kParams * 4, cudaMemcpyDeviceToHost));
    if (norm) std::memcpy(norm, s->h_norm, sizeof(s->h_norm));
    return MARL_OK;
}

marl_status marl_surrogate_set_weights(marl_surrogate* s, const float* params, const float* norm) {
    if (!s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    SCK(cudaStreamSynchronize(s->stream));
    // Ordered on the surrogate's stream, ahead of the kernels that read them.
    if (params) {
        SCK(cudaMemcpyAsync(s->p, params, (size_t)mlp::kParams * 4, cudaMemcpyHostToDevice, s->stream));
        SCK(mlp::launch_weights_bf16(s->p, s->w1, s->w2, s->w3, s->w2t, s->w3t, s->stream));
    }
    if (norm) {
        std::memcpy(s->h_norm, norm, sizeof(s->h_norm));
        SCK(cudaMemcpyAsync(s->norm, s->h_norm, sizeof(s->h_norm), cudaMemcpyHostToDevice, s->stream));
        s->prepared = true;  // explicit statistics make inference possible
    }
    SCK(cudaStreamSynchronize(s->stream));
    return MARL_OK;
}

marl_status marl_surrogate_gradients(marl_surrogate* s, const uint16_t* x, const float* t, uint32_t batch,
                                     float* grads_out, float* loss_out, float* y_out) {
    if (!s || !x || !t || !grads_out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (batch == 0 || batch % 128) return fail(MARL_ERR_INVALID_INPUT, "batch must be a positive multiple of 128");
    marl_status st = ensure_work(s, batch);
    if (st) return st;
    if ((st = ensure_scalars(s, 1))) return st;
    cudaStream_t cs = s->stream;
    SCK(cudaMemcpyAsync(s->xb, x, (size_t)batch * mlp::kInPad * 2, cudaMemcpyHostToDevice, cs));
    SCK(cudaMemcpyAsync(s->tb, t, (size_t)batch * mlp::kOut * 4, cudaMemcpyHostToDevice, cs));
    SCK(mlp::launch_transpose_batch(s->xb, batch, s->xbt, cs));
    SCK(cudaMemsetAsync(s->d_scalars, 0, 4, cs));
    SST(forward_train(s, batch));
    SST(backward(s, batch, s->d_scalars));
    SCK(cudaMemcpyAsync(grads_out, s->g, (size_t)mlp::kParams * 4, cudaMemcpyDeviceToHost, cs));
    float loss = 0.0f;
    SCK(cudaMemcpyAsync(&loss, s->d_scalars, 4, cudaMemcpyDeviceToHost, cs));
    if (y_out) SCK(cudaMemcpyAsync(y_out, s->y, (size_t)batch * mlp::kOut * 4, cudaMemcpyDeviceToHost, cs));
    SST(check_err(s));
    if (loss_out) *loss_out = loss / ((float)batch * mlp::kOut);
    return MARL_OK;
}

marl_status marl_surrogate_infer_device(marl_surrogate* s, const uint16_t* x_dev, uint32_t n, float* y_dev,
                                        uint32_t ldy) {
    if (!s || (n && (!x_dev || !y_dev))) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (ldy < n) return fail(MARL_ERR_INVALID_INPUT, "ldy %u < n %u", ldy, n);
    return surrogate_infer(s, reinterpret_cast<const __nv_bfloat16*>(x_dev), n, y_dev, ldy, s->stream);
}

marl_status marl_ctx_set_surrogate(marl_ctx* c, marl_surrogate* s, int32_t mode, float tol) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (mode < MARL_SURR_OFF || mode > MARL_SURR_TRUSTED) return fail(MARL_ERR_INVALID_INPUT, "unknown mode %d", mode);
    if (mode != MARL_SURR_OFF && !s) return fail(MARL_ERR_INVALID_INPUT, "null surrogate");
    if ((mode == MARL_SURR_GATED || mode == MARL_SURR_TRUSTED) && !s->prepared)
        return fail(MARL_ERR_STATE, "surrogate not prepared (marl_surrogate_prepare or set_weights with norm)");
    if (mode == MARL_SURR_GATED && !(tol >= 0.0f)) return fail(MARL_ERR_INVALID_INPUT, "tol must be >= 0");
    SCK(cudaStreamSynchronize(c->stream));
    if (s) SCK(cudaStreamSynchronize(s->stream));
    if ((mode == MARL_SURR_GATED || mode == MARL_SURR_TRUSTED) && !c->surr_xt) {
        const size_t cap = c->t.cap;
        SCK(cudaMalloc((void**)&c->surr_xt, cap * MARL_M_INT * 4));
        SCK(cudaMalloc((void**)&c->surr_pred, cap * MARL_M_INT * 4));
        SCK(cudaMalloc((void**)&c->surr_x, cap * mlp::kInPad * 2));
        SCK(cudaMalloc((void**)&c->surr_status, cap));
        SCK(cudaMalloc((void**)&c->surr_err, cap * 4));
        SCK(cudaMalloc((void**)&c->surr_counters, 64));
        SCK(cudaMemsetAsync(c->surr_counters, 0, 64, c->stream));
    }
    c->surr = mode == MARL_SURR_OFF ? nullptr : s;
    c->surr_mode = mode;
    c->surr_tol = tol;
    return MARL_OK;
}

marl_status marl_ctx_surrogate_counters(marl_ctx* c, marl_surrogate_counters* out) {
    if (!c || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    std::memset(out, 0, sizeof(*out));
    SCK(cudaStreamSynchronize(c->stream));
    if (!c->surr_counters) return MARL_OK;
    unsigned long long h[8];
    SCK(cudaMemcpy(h, c->surr_counters, 64, cudaMemcpyDeviceToHost));
    out->cells = h[0];
    out->speculated = h[1];
    out->accepted = h[2];
    out->rejected = h[3];
    const uint32_t bits = (uint32_t)h[4];
    std::memcpy(&out->max_err, &bits, 4);
    return MARL_OK;
}

}  // extern "C"
