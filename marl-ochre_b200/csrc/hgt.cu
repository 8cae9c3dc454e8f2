// Horizontal gene transfer: crates/marl-cell/src/hgt.rs:7-27
// (transfer_reaction) applied to the device cell table for a list of
// (donor, recipient) pairs, in list order.
//
// The reference defines the primitive but does not call it from the tick
// (crates/marl-sim/src/lib.rs has no HGT step).  Pair k draws from its own
// counter-based stream (the device fate streams of fate_stream.h, keyed by
// (seed ^ kHgtSalt, tick, k)), so the result does not depend on scheduling.
// Pairs run in waves: pair k goes into the first wave after every earlier pair
// that wrote one of its cells or read its recipient, so each wave's pairs are
// independent and the waves reproduce the sequential order exactly.  One
// thread per pair.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "ctx_impl.h"
#include "fate_stream.h"

using namespace marl;

namespace marl {

constexpr uint64_t kHgtSalt = 0x4847545452414E53ull;  // "HGTTRANS"

__global__ void k_hgt(CellTable t, const uint4* __restrict__ items, uint32_t count, uint64_t seed, uint64_t tick) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint4 it = items[i];  // donor, recipient, pair index
    const size_t cap = t.cap;
    uint32_t active_mask = 0;
    int na = 0;
#pragma unroll
    for (int r = 0; r < MARL_R_MAX; ++r)
        if (fabsf(__uint_as_float(t.rx[(size_t)r * cap + it.x].z)) > 1e-9f) active_mask |= 1u << r, ++na;
    if (na == 0) return;
    fate::Stream rng(fate::stream_key(seed ^ kHgtSalt, tick, it.z));
    uint32_t pick = rng.range(0, (uint32_t)na);  // the pick-th active slot, in slot order
    int donor_idx = 0;
    for (int r = 0; r < MARL_R_MAX; ++r)
        if ((active_mask >> r) & 1u) {
            if (pick == 0) {
                donor_idx = r;
                break;
            }
            --pick;
        }
    const uint4 donated = t.rx[(size_t)donor_idx * cap + it.x];
    int target = -1;
    for (int r = 0; r < MARL_R_MAX && target < 0; ++r)
        if (fabsf(__uint_as_float(t.rx[(size_t)r * cap + it.y].z)) < 1e-9f) target = r;
    if (target < 0) target = (int)rng.range(0, MARL_R_MAX);
    t.rx[(size_t)target * cap + it.y] = donated;
}

cudaError_t launch_hgt(const CellTable& t, const uint4* items, uint32_t count, uint64_t seed, uint64_t tick,
                       cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    k_hgt<<<(count + 127) / 128, 128, 0, s>>>(t, items, count, seed, tick);
    return cudaGetLastError();
}

}  // namespace marl

extern "C" marl_status marl_ctx_hgt(marl_ctx* c, const uint32_t* donors, const uint32_t* recipients, uint32_t n_pairs,
                                    uint64_t seed, uint64_t tick) {
    if (!c || (n_pairs && (!donors || !recipients))) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    if (n_pairs == 0) return MARL_OK;
    const uint32_t n = c->n;
    for (uint32_t k = 0; k < n_pairs; ++k)
        if (donors[k] >= n || recipients[k] >= n)
            return fail(MARL_ERR_INVALID_INPUT, "pair %u: (%u, %u) with %u cells", k, donors[k], recipients[k], n);
    // Waves: a pair reads its donor's reactions and writes one of its
    // recipient's, so it must follow every earlier pair that wrote either
    // cell, and every earlier pair that read its recipient.
    std::vector<uint32_t> last_write(n, 0), last_read(n, 0), wave(n_pairs);
    uint32_t waves = 0;
    for (uint32_t k = 0; k < n_pairs; ++k) {
        const uint32_t d = donors[k], r = recipients[k];
        const uint32_t w = std::max({last_write[d], last_write[r], last_read[r]}) + 1;
        wave[k] = w;
        last_write[r] = w;
        last_read[d] = std::max(last_read[d], w);
        waves = std::max(waves, w);
    }
    std::vector<uint32_t> order(n_pairs);
    for (uint32_t k = 0; k < n_pairs; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return wave[a] < wave[b]; });
    std::vector<uint4> items(n_pairs);
    for (uint32_t i = 0; i < n_pairs; ++i) {
        const uint32_t k = order[i];
        items[i] = make_uint4(donors[k], recipients[k], k, 0);
    }
    uint4* d_items = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&d_items, items.size() * sizeof(uint4), c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(uint4), cudaMemcpyHostToDevice, c->stream);
    uint32_t first = 0;
    for (uint32_t w = 1; e == cudaSuccess && w <= waves; ++w) {
        uint32_t last = first;
        while (last < n_pairs && wave[order[last]] == w) ++last;
        e = launch_hgt(c->t, d_items + first, last - first, seed, tick, c->stream);
        ++c->launches;
        first = last;
    }
    if (d_items) cudaFreeAsync(d_items, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);  // the host items outlive the copy
    if (e != cudaSuccess) return cuda_fail(e, "marl_ctx_hgt");
    c->h2d_bytes += items.size() * sizeof(uint4);
    return sync_and_check(c);
}
