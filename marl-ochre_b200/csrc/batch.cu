// marl_batch: many independent runs of marl_sim::run advanced together on one
// GPU.  Every device phase of a tick is one launch over all runs (work lists
// of (run, tile) items for diffusion and light, global tickets for the cell
// loop, one block per run for compaction), the device part of a tick is
// captured once as a CUDA graph and replayed, and fate processing
// (crates/marl-sim/src/lib.rs:219-277) runs on host worker threads, one run
// per task, each run with its own RNG stream.
//
// Device memory per run: the same buffers a marl_ctx holds (ping-pong field,
// padded occupancy mask, cell map, light, compact species 4, cell table,
// change list).  Shared: the RunDesc table, the tensor maps (five per run),
// the work lists, and one read-back block
//   [BatchScalars][ChangeHeader x runs][packed change lists]
// whose head (scalars, headers and the first kPrefetch packed changes) comes
// back to the host in one copy per tick.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/marl_cuda.h"
#include "common.cuh"
#include "ctx_impl.h"
#include "engine_host.h"
#include "internal.h"
#include "surrogate.h"

namespace marl {
namespace {

#define CK(expr)                                            \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr); \
    } while (0)

constexpr uint32_t kPrefetch = 2048;  // packed change entries read back with the headers

// Fixed set of worker threads running index-parallel jobs; the calling thread
// takes part.  run() returns when every index has been processed.
class WorkerPool {
   public:
    ~WorkerPool() { resize(0); }

    // Not concurrent with run().
    void resize(int n) {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
        threads_.clear();
        stop_ = false;
        const uint64_t g = gen_;
        for (int i = 0; i < n; ++i) threads_.emplace_back([this, g] { loop(g); });
    }

    void run(int count, const std::function<void(int)>& fn) {
        if (threads_.empty() || count <= 1) {
            for (int i = 0; i < count; ++i) fn(i);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(m_);
            job_ = &fn;
            count_ = count;
            next_.store(0);
            active_ = (int)threads_.size();
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [this] { return active_ == 0; });
        job_ = nullptr;
    }

   private:
    void work() {
        for (int i = next_.fetch_add(1); i < count_; i = next_.fetch_add(1)) (*job_)(i);
    }
    void loop(uint64_t seen) {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> lk(m_);
            if (--active_ == 0) done_cv_.notify_one();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* job_ = nullptr;
    int count_ = 0;
    std::atomic<int> next_{0};
    int active_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

struct BatchRun {
    Grid g{0, 0, 0};
    uint32_t cap = 0;
    float* field[2] = {nullptr, nullptr};
    uint8_t* mask = nullptr;
    int32_t* cmap = nullptr;
    float* light = nullptr;
    float* c4 = nullptr;
    CellTable t{};
    marl_change* changes = nullptr;
    uint32_t n = 0;
    HostRun host;
    EditData edits;
    marl_status st = MARL_OK;
};

}  // namespace
}  // namespace marl

using namespace marl;

struct marl_batch {
    int device = 0, num_sms = 0;
    marl_sim_params sim{};
    FieldConsts fk{};
    CellConsts ck{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t capture_stream = nullptr;

    std::vector<BatchRun> runs;
    int cur = 0;
    uint32_t epoch = 0;
    int tile = 0, zc = 16;

    RunDesc* d_runs = nullptr;
    RunDesc* h_runs = nullptr;  // pinned mirror, copied to d_runs at the start of each tick
    CUtensorMap* d_maps = nullptr;
    int4* d_diff_items = nullptr;
    int n_diff_items = 0, diff_items_cap = 0;
    int4* d_light_items = nullptr;
    int n_light_items = 0;

    uint8_t* d_rb = nullptr;  // [BatchScalars][ChangeHeader x runs][packed changes]
    uint8_t* h_rb = nullptr;  // pinned head of the same layout (kPrefetch packed entries)
    size_t rb_head_bytes = 0;
    uint32_t packed_cap = 0;
    std::vector<marl_change> overflow;

    void* d_edit = nullptr;
    void* h_edit = nullptr;
    size_t edit_bytes = 0;
    marl_cell* d_records = nullptr;
    marl_cell* h_records = nullptr;
    uint32_t records_cap = 0;

    // Reaction surrogate (marl_batch_set_surrogate); its arrays hold one row
    // per cell slot of the batch, run r's cells from the run's cell_base.
    marl_surrogate* surr = nullptr;
    int surr_mode = MARL_SURR_OFF;
    float surr_tol = 0.0f;
    uint32_t surr_rows = 0;  // sum of the runs' capacities
    float* surr_xt = nullptr;
    float* surr_pred = nullptr;
    void* surr_x = nullptr;
    uint8_t* surr_status = nullptr;
    float* surr_err = nullptr;
    unsigned long long* surr_counters = nullptr;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool use_graph = true;
    bool direct_since_change = false;  // a direct tick ran since the last graph invalidation

    // Device fate (marl_batch_set_device_fate): per-run fate buffers, their
    // FateRun table and scalars; while it is on, populations, tick counters and
    // completion epochs advance on the device and the host copies are stale
    // until sync_fate_state.
    bool device_fate = false;
    bool fate_stale = false;  // host per-run state behind the device
    std::vector<FateBuffers> fate;
    FateRun* d_fate_runs = nullptr;
    FateScalars* d_fate_scalars = nullptr;  // [runs]
    FateScalars* h_fate_scalars = nullptr;  // pinned [runs]
    uint32_t max_cap = 0;
    cudaGraphExec_t fate_graph[2] = {nullptr, nullptr};

    WorkerPool pool;

    uint64_t h2d = 0, d2h = 0, launches = 0, ticks = 0;
    uint64_t h2d_last = 0, d2h_last = 0;
    double device_us = 0.0;
    struct Span {
        cudaEvent_t a, b;
    };
    std::vector<Span> span_pool, spans_pending;

    BatchScalars* d_scalars() { return reinterpret_cast<BatchScalars*>(d_rb); }
    ChangeHeader* d_headers() { return reinterpret_cast<ChangeHeader*>(d_rb + sizeof(BatchScalars)); }
    marl_change* d_packed() {
        return reinterpret_cast<marl_change*>(d_rb + sizeof(BatchScalars) + runs.size() * sizeof(ChangeHeader));
    }
    const BatchScalars* h_scalars() const { return reinterpret_cast<const BatchScalars*>(h_rb); }
    const ChangeHeader* h_headers() const {
        return reinterpret_cast<const ChangeHeader*>(h_rb + sizeof(BatchScalars));
    }
    const marl_change* h_packed() const {
        return reinterpret_cast<const marl_change*>(h_rb + sizeof(BatchScalars) + runs.size() * sizeof(ChangeHeader));
    }
};

namespace {

void invalidate_graphs(marl_batch* b) {
    for (auto& g : b->fate_graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (auto& g : b->graph)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    b->direct_since_change = false;
}

void batch_free(marl_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    invalidate_graphs(b);
    for (auto& r : b->runs) {
        void* p[] = {r.field[0], r.field[1], r.mask, r.cmap, r.light, r.c4, r.changes};
        for (void* q : p)
            if (q) cudaFree(q);
        free_table(r.t);
    }
    for (auto& f : b->fate) free_fate(f);
    void* dev[] = {b->d_fate_runs, b->d_fate_scalars, b->d_runs, b->d_maps, b->d_diff_items, b->d_light_items, b->d_rb, b->d_edit, b->d_records,
                   b->surr_xt, b->surr_pred, b->surr_x, b->surr_status, b->surr_err, b->surr_counters};
    for (void* p : dev)
        if (p) cudaFree(p);
    void* host[] = {b->h_runs, b->h_rb, b->h_edit, b->h_records, b->h_fate_scalars};
    for (void* p : host)
        if (p) cudaFreeHost(p);
    for (auto* v : {&b->span_pool, &b->spans_pending})
        for (auto& s : *v) {
            cudaEventDestroy(s.a);
            cudaEventDestroy(s.b);
        }
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
}

int span_begin(marl_batch* b) {
    marl_batch::Span s;
    if (!b->span_pool.empty()) {
        s = b->span_pool.back();
        b->span_pool.pop_back();
    } else if (cudaEventCreate(&s.a) != cudaSuccess || cudaEventCreate(&s.b) != cudaSuccess) {
        return -1;
    }
    cudaEventRecord(s.a, b->stream);
    b->spans_pending.push_back(s);
    return (int)b->spans_pending.size() - 1;
}

void span_end(marl_batch* b, int idx) {
    if (idx >= 0) cudaEventRecord(b->spans_pending[idx].b, b->stream);
}

void resolve_spans(marl_batch* b) {
    for (auto& s : b->spans_pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, s.a, s.b) == cudaSuccess) b->device_us += 1000.0 * ms;
        b->span_pool.push_back(s);
    }
    b->spans_pending.clear();
}

marl_status ensure_edit(marl_batch* b, size_t bytes) {
    if (bytes <= b->edit_bytes) return MARL_OK;
    size_t nb = b->edit_bytes ? b->edit_bytes : (1 << 16);
    while (nb < bytes) nb *= 2;
    if (b->d_edit) CK(cudaFree(b->d_edit));
    if (b->h_edit) CK(cudaFreeHost(b->h_edit));
    b->d_edit = b->h_edit = nullptr;
    b->edit_bytes = 0;
    CK(cudaMalloc(&b->d_edit, nb));
    CK(cudaMallocHost(&b->h_edit, nb));
    b->edit_bytes = nb;
    return MARL_OK;
}

marl_status ensure_records(marl_batch* b, uint32_t n) {
    if (n <= b->records_cap) return MARL_OK;
    uint32_t cap = b->records_cap ? b->records_cap : 1024;
    while (cap < n) cap *= 2;
    if (b->d_records) CK(cudaFree(b->d_records));
    if (b->h_records) CK(cudaFreeHost(b->h_records));
    b->d_records = nullptr;
    b->h_records = nullptr;
    b->records_cap = 0;
    CK(cudaMalloc((void**)&b->d_records, (size_t)cap * sizeof(marl_cell)));
    CK(cudaMallocHost((void**)&b->h_records, (size_t)cap * sizeof(marl_cell)));
    b->records_cap = cap;
    return MARL_OK;
}

// Tensor maps and work lists for one tile choice.  Diffusion items are
// ordered run by run; every item covers zc planes of one (TX x TY) column.
marl_status plan_tiles(marl_batch* b, int tile, int zc, cudaStream_t s) {
    const int n_runs = (int)b->runs.size();
    std::vector<CUtensorMap> maps((size_t)n_runs * kMapsPerRun);
    std::vector<int4> items;
    int tx, ty;
    diffusion_tile_shape(tile, &tx, &ty);
    for (int r = 0; r < n_runs; ++r) {
        const BatchRun& R = b->runs[r];
        DiffusionPlan p;
        if (!plan_diffusion(&p, R.field[0], R.field[1], R.mask, R.g, tile, zc))
            return fail(MARL_ERR_CUDA, "cuTensorMapEncodeTiled failed for run %d", r);
        CUtensorMap* m = &maps[(size_t)r * kMapsPerRun];
        m[0] = p.tm_load[0];
        m[1] = p.tm_load[1];
        m[2] = p.tm_store[0];
        m[3] = p.tm_store[1];
        m[4] = p.tm_mask;
        const int nbx = (R.g.X + tx - 1) / tx, nby = (R.g.Y + ty - 1) / ty, nbz = (R.g.Z + zc - 1) / zc;
        for (int bz = 0; bz < nbz; ++bz)
            for (int by = 0; by < nby; ++by)
                for (int bx = 0; bx < nbx; ++bx) items.push_back(make_int4(r, bx, by, bz));
    }
    if ((int)items.size() > b->diff_items_cap) {
        if (b->d_diff_items) CK(cudaFree(b->d_diff_items));
        b->d_diff_items = nullptr;
        b->diff_items_cap = 0;
        CK(cudaMalloc((void**)&b->d_diff_items, items.size() * sizeof(int4)));
        b->diff_items_cap = (int)items.size();
    }
    // The copies are ordered on `s`, behind any work still reading the old
    // maps and ahead of every launch that reads the new ones.  A plain
    // cudaMemcpy would not do: it runs on the legacy default stream, which a
    // non-blocking `s` does not wait for, and from pageable memory it may
    // return before the data has landed.  The stream is synchronized before
    // the host vectors go out of scope.
    CK(cudaMemcpyAsync(b->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b->d_diff_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    b->n_diff_items = (int)items.size();
    b->tile = tile;
    b->zc = zc;
    return MARL_OK;
}

void fill_desc(marl_batch* b) {
    uint32_t base = 0;
    for (size_t r = 0; r < b->runs.size(); ++r) {
        BatchRun& R = b->runs[r];
        RunDesc& d = b->h_runs[r];
        d.n = R.n;
        d.epoch = b->epoch;
        d.cell_base = base;
        d.sv = SurrView{};
        if (b->surr) {
            d.sv.xt = b->surr_xt;
            d.sv.pred = b->surr_pred;
            d.sv.tol = b->surr_tol;
            d.sv.status = b->surr_status;
            d.sv.err = b->surr_err;
            d.sv.row0 = base;
            d.sv.ld = b->surr_rows;
        }
        base += R.n;
    }
}

uint32_t batch_cells(const marl_batch* b) {
    uint32_t n = 0;
    for (const auto& R : b->runs) n += R.n;
    return n;
}

int surrogate_cell_mode(const marl_batch* b) {
    if (!b->surr) return kModePlain;
    return b->surr_mode == MARL_SURR_TRUSTED ? kModeTrusted : kModeGated;
}

// The device part of one tick (crates/marl-sim/src/lib.rs:164-217 for every
// run): descriptor upload, schedule, sources + diffusion, light, the cell
// loop, compaction, packing, and the read-back of the block head.  Ends with
// b->cur flipped by the number of substeps.
marl_status enqueue_device_tick(marl_batch* b, cudaStream_t s, int cur) {
    const int n_runs = (int)b->runs.size();
    CK(cudaMemcpyAsync(b->d_runs, b->h_runs, (size_t)n_runs * sizeof(RunDesc), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(&b->d_scalars()->ticket, 0, 4, s));
    CK(launch_cell_schedule_batch(b->d_runs, n_runs, b->num_sms, s));
    const uint32_t S = b->sim.diffusion_substeps;
    uint32_t* err = &b->d_scalars()->err;
    if (S == 0) {
        for (auto& R : b->runs) CK(launch_sources(R.field[cur], R.g, b->fk, s));
    }
    for (uint32_t i = 0; i < S; ++i) {
        CK(launch_diffuse_batch(b->tile, b->d_runs, b->d_maps, b->d_diff_items, b->n_diff_items, b->zc, b->fk, cur,
                                i == 0 ? 1 : 0, i + 1 == S ? 1 : 0, err, s));
        cur ^= 1;
    }
    CK(launch_light_batch(b->d_runs, b->d_light_items, b->n_light_items, b->fk, cur, S > 0 ? 1 : 0, s));
    const int mode = surrogate_cell_mode(b);
    const uint32_t total = batch_cells(b);
    if (mode != kModePlain && total > 0) {
        // Launched directly, never captured: the row count changes every tick.
        CK(launch_surrogate_prepass_batch(b->d_runs, n_runs, total, b->ck, cur, b->surr->norm, b->surr_xt,
                                          b->surr_rows, b->surr_x, b->num_sms, s));
        marl_status st = surrogate_infer(b->surr, reinterpret_cast<const __nv_bfloat16*>(b->surr_x), total,
                                         b->surr_pred, b->surr_rows, s);
        if (st) return st;
    }
    CK(launch_cell_tick_batch(b->d_runs, n_runs, b->d_scalars(), b->ck, cur, b->num_sms, mode, s));
    if (mode != kModePlain && total > 0)
        CK(launch_surrogate_count(b->surr_status, b->surr_err, total, b->surr_counters,
                                  reinterpret_cast<uint32_t*>(b->surr_counters + 4), s));
    CK(launch_compact_batch(b->d_runs, n_runs, s));
    CK(launch_pack_changes(b->d_runs, n_runs, b->d_scalars(), b->d_packed(), s));
    CK(cudaMemcpyAsync(b->h_rb, b->d_rb, b->rb_head_bytes, cudaMemcpyDeviceToHost, s));
    return MARL_OK;
}

uint64_t device_tick_launches(const marl_batch* b) {
    const uint32_t S = b->sim.diffusion_substeps;
    return 1 + (S ? S : b->runs.size()) + 4 + (b->surr ? 5 : 0);
}

marl_status launch_tick(marl_batch* b) {
    const int cur = b->cur;
    if (b->use_graph && b->direct_since_change && !b->surr) {
        if (!b->graph[cur]) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
            marl_status st = enqueue_device_tick(b, b->capture_stream, cur);
            cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
            if (st) {
                if (g) cudaGraphDestroy(g);
                return st;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&b->graph[cur], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                b->graph[cur] = nullptr;
                return cuda_fail(e, "cudaGraphInstantiate");
            }
        }
        CK(cudaGraphLaunch(b->graph[cur], b->stream));
    } else {
        marl_status st = enqueue_device_tick(b, b->stream, cur);
        if (st) return st;
        b->direct_since_change = true;
    }
    if (b->sim.diffusion_substeps & 1u) b->cur ^= 1;
    b->launches += device_tick_launches(b);
    return MARL_OK;
}

marl_status collect_errors(marl_batch* b, uint32_t bits) {
    if (!bits) return MARL_OK;
    cudaMemsetAsync(&b->d_scalars()->err, 0, 4, b->stream);
    cudaStreamSynchronize(b->stream);
    if (bits & (kErrTimeoutMbar | kErrTimeoutDeps))
        return fail(MARL_ERR_TIMEOUT, "device wait gave up (error bits 0x%x)", bits);
    if (bits & kErrCapacity) return fail(MARL_ERR_CAPACITY, "a run's cell table is full: births dropped (0x%x)", bits);
    if (bits & kErrFateChain) return fail(MARL_ERR_STATE, "inconsistent death events in device fate (0x%x)", bits);
    return fail(MARL_ERR_INVALID_INPUT, "device rejected input (error bits 0x%x)", bits);
}

// Flattens the runs' edit lists into one staging buffer
//   [moves uint4][halve uint2][deaths uint2][birth slots uint2][pad][births]
// and launches the four batched edit kernels in the single-run order.
marl_status apply_edits(marl_batch* b) {
    uint32_t nh = 0, nd = 0, nm = 0, nb = 0;
    for (size_t r = 0; r < b->runs.size(); ++r) {
        const BatchRun& R = b->runs[r];
        const EditData& e = R.edits;
        if ((uint64_t)e.n_after_deaths + e.births.size() > R.cap)
            return fail(MARL_ERR_CAPACITY, "run %zu: %u + %zu births exceed capacity %u", r, e.n_after_deaths,
                        e.births.size(), R.cap);
        nh += (uint32_t)e.halve.size();
        nd += (uint32_t)e.deaths.size();
        nm += (uint32_t)e.move_dst.size();
        nb += (uint32_t)e.births.size();
    }
    const size_t o_moves = 0, o_halve = o_moves + (size_t)nm * 16, o_deaths = o_halve + (size_t)nh * 8,
                 o_slots = o_deaths + (size_t)nd * 8, o_births = (o_slots + (size_t)nb * 8 + 15) & ~(size_t)15,
                 total = o_births + (size_t)nb * sizeof(marl_cell);
    if (total == 0) {
        for (auto& R : b->runs) R.n = R.edits.n_after_deaths;
        return MARL_OK;
    }
    marl_status st = ensure_edit(b, total);
    if (st) return st;
    uint8_t* h = (uint8_t*)b->h_edit;
    uint4* moves = (uint4*)(h + o_moves);
    uint2* halve = (uint2*)(h + o_halve);
    uint2* deaths = (uint2*)(h + o_deaths);
    uint2* slots = (uint2*)(h + o_slots);
    marl_cell* births = (marl_cell*)(h + o_births);
    for (size_t r = 0; r < b->runs.size(); ++r) {
        BatchRun& R = b->runs[r];
        const EditData& e = R.edits;
        const uint32_t ru = (uint32_t)r;
        for (uint32_t i : e.halve) *halve++ = make_uint2(ru, i);
        for (uint32_t i : e.deaths) *deaths++ = make_uint2(ru, i);
        for (size_t i = 0; i < e.move_dst.size(); ++i) *moves++ = make_uint4(ru, e.move_dst[i], e.move_src[i], 0);
        for (size_t i = 0; i < e.births.size(); ++i) {
            *slots++ = make_uint2(ru, e.n_after_deaths + (uint32_t)i);
            *births++ = e.births[i];
        }
        R.n = e.n_after_deaths + (uint32_t)e.births.size();
    }
    const int span = span_begin(b);
    uint8_t* d = (uint8_t*)b->d_edit;
    CK(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, b->stream));
    b->h2d += total;
    b->h2d_last += total;
    CK(launch_halve_batch(b->d_runs, (const uint2*)(d + o_halve), nh, b->stream));
    CK(launch_clear_dead_batch(b->d_runs, (const uint2*)(d + o_deaths), nd, b->stream));
    CK(launch_moves_batch(b->d_runs, (const uint4*)(d + o_moves), nm, b->stream));
    CK(launch_births_batch(b->d_runs, (const marl_cell*)(d + o_births), (const uint2*)(d + o_slots), nb,
                           &b->d_scalars()->err, b->stream));
    span_end(b, span);
    b->launches += (nh > 0) + (nd > 0) + (nm > 0) + (nb > 0);
    return MARL_OK;
}

// ---- device fate ----

// One tick of every run with fate on the device (lib.rs:160-277): populations,
// first global cell indices and epochs from the previous fate step, schedule,
// sources + diffusion, light, the cell loop, fate.  Nothing crosses to the
// host; ends with b->cur flipped by the number of substeps.
marl_status enqueue_device_fate_tick(marl_batch* b, cudaStream_t s, int cur) {
    const int n_runs = (int)b->runs.size();
    CK(launch_batch_population(b->d_runs, n_runs, b->d_fate_runs, s));
    CK(cudaMemsetAsync(&b->d_scalars()->ticket, 0, 4, s));
    CK(launch_cell_schedule_batch(b->d_runs, n_runs, b->num_sms, s));
    const uint32_t S = b->sim.diffusion_substeps;
    uint32_t* err = &b->d_scalars()->err;
    if (S == 0) {
        for (auto& R : b->runs) CK(launch_sources(R.field[cur], R.g, b->fk, s));
    }
    for (uint32_t i = 0; i < S; ++i) {
        CK(launch_diffuse_batch(b->tile, b->d_runs, b->d_maps, b->d_diff_items, b->n_diff_items, b->zc, b->fk, cur,
                                i == 0 ? 1 : 0, i + 1 == S ? 1 : 0, err, s));
        cur ^= 1;
    }
    CK(launch_light_batch(b->d_runs, b->d_light_items, b->n_light_items, b->fk, cur, S > 0 ? 1 : 0, s));
    CK(launch_cell_tick_batch(b->d_runs, n_runs, b->d_scalars(), b->ck, cur, b->num_sms, kModePlain, s));
    CK(launch_fate(b->d_fate_runs, n_runs, b->max_cap, err, b->sim, b->num_sms, s));
    return MARL_OK;
}

uint64_t device_fate_tick_launches(const marl_batch* b) {
    const uint32_t S = b->sim.diffusion_substeps;
    return 1 + 1 + (S ? S : b->runs.size()) + 1 + 1 + 5;
}

marl_status launch_device_fate_tick(marl_batch* b) {
    const int cur = b->cur;
    if (b->use_graph) {
        if (!b->fate_graph[cur]) {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
            marl_status st = enqueue_device_fate_tick(b, b->capture_stream, cur);
            cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
            if (st) {
                if (g) cudaGraphDestroy(g);
                return st;
            }
            if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&b->fate_graph[cur], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                b->fate_graph[cur] = nullptr;
                return cuda_fail(e, "cudaGraphInstantiate");
            }
        }
        CK(cudaGraphLaunch(b->fate_graph[cur], b->stream));
    } else {
        marl_status st = enqueue_device_fate_tick(b, b->stream, cur);
        if (st) return st;
    }
    if (b->sim.diffusion_substeps & 1u) b->cur ^= 1;
    b->launches += device_fate_tick_launches(b);
    return MARL_OK;
}

// Synchronises and brings every run's population and counters back to the
// host (one copy of the scalar array).
marl_status sync_fate_state(marl_batch* b) {
    if (!b->fate_stale) return MARL_OK;
    const size_t bytes = b->runs.size() * sizeof(FateScalars);
    CK(cudaMemcpyAsync(b->h_fate_scalars, b->d_fate_scalars, bytes, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaMemcpyAsync(b->h_rb, b->d_rb, sizeof(BatchScalars), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    resolve_spans(b);
    b->d2h += bytes + sizeof(BatchScalars);
    b->d2h_last += bytes + sizeof(BatchScalars);
    for (size_t r = 0; r < b->runs.size(); ++r) {
        BatchRun& R = b->runs[r];
        const FateScalars& f = b->h_fate_scalars[r];
        R.n = f.n;
        R.host.tick = f.tick;
        R.host.total_div = f.total_div;
        R.host.total_death = f.total_death;
        R.host.tick_div = f.placed;
        R.host.tick_death = f.ndeath;
    }
    b->fate_stale = false;
    return collect_errors(b, b->h_scalars()->err);
}

marl_status device_fate_steps(marl_batch* b, uint32_t ticks) {
    b->h2d_last = b->d2h_last = 0;
    uint32_t done = 0;
    while (done < ticks) {
        if (b->epoch == 0xFFFFFFFFu) {  // the next epoch would wrap: clear stale completion epochs
            marl_status st = sync_fate_state(b);
            if (st) return st;
            for (auto& R : b->runs) CK(cudaMemsetAsync(R.t.done, 0, (size_t)R.t.cap * 4, b->stream));
            b->epoch = 0;
            fill_desc(b);
            CK(cudaMemcpyAsync(b->d_runs, b->h_runs, b->runs.size() * sizeof(RunDesc), cudaMemcpyHostToDevice,
                               b->stream));
            CK(cudaStreamSynchronize(b->stream));
        }
        const uint32_t chunk = std::min<uint32_t>(ticks - done, 0xFFFFFFFFu - b->epoch);
        const int span = span_begin(b);
        for (uint32_t t = 0; t < chunk; ++t) {
            b->epoch += 1;  // the device adds one to every run's epoch at the start of the tick
            marl_status st = launch_device_fate_tick(b);
            if (st) return st;
            b->fate_stale = true;
            ++b->ticks;
        }
        span_end(b, span);
        done += chunk;
    }
    return sync_fate_state(b);
}

marl_status enable_device_fate(marl_batch* b) {
    if (b->surr) return fail(MARL_ERR_STATE, "device fate runs with the batch surrogate off");
    const size_t n_runs = b->runs.size();
    if (b->fate.empty()) {
        b->fate.resize(n_runs);
        CK(cudaMalloc((void**)&b->d_fate_scalars, n_runs * sizeof(FateScalars)));
        CK(cudaMallocHost((void**)&b->h_fate_scalars, n_runs * sizeof(FateScalars)));
        CK(cudaMalloc((void**)&b->d_fate_runs, n_runs * sizeof(FateRun)));
        std::vector<FateRun> fr(n_runs);
        for (size_t r = 0; r < n_runs; ++r) {
            BatchRun& R = b->runs[r];
            CK(alloc_fate(b->fate[r], R.cap, R.g.V(), b->d_fate_scalars + r));
            fr[r].f = b->fate[r];
            fr[r].t = R.t;
            fr[r].g = R.g;
            fr[r].cmap = R.cmap;
            fr[r].mask = R.mask;
            b->max_cap = std::max(b->max_cap, R.cap);
        }
        CK(cudaMemcpy(b->d_fate_runs, fr.data(), n_runs * sizeof(FateRun), cudaMemcpyHostToDevice));
    }
    CK(cudaStreamSynchronize(b->stream));
    for (size_t r = 0; r < n_runs; ++r) {
        const BatchRun& R = b->runs[r];
        FateScalars& f = b->h_fate_scalars[r];
        std::memset(&f, 0, sizeof(f));
        f.seed = R.host.seed;
        f.tick = R.host.tick;
        f.total_div = R.host.total_div;
        f.total_death = R.host.total_death;
        f.n = R.n;
        f.placed = (uint32_t)R.host.tick_div;
        f.ndeath = (uint32_t)R.host.tick_death;
    }
    // The population kernel adds one to the epoch at the start of each tick.
    fill_desc(b);
    CK(cudaMemcpyAsync(b->d_fate_scalars, b->h_fate_scalars, n_runs * sizeof(FateScalars), cudaMemcpyHostToDevice,
                       b->stream));
    CK(cudaMemcpyAsync(b->d_runs, b->h_runs, n_runs * sizeof(RunDesc), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->h2d += n_runs * (sizeof(FateScalars) + sizeof(RunDesc));
    b->device_fate = true;
    b->fate_stale = false;
    return MARL_OK;
}

// Back to host fate: each run's host side adopts its device cell vector (its
// sequential stream continues where it stood).
marl_status disable_device_fate(marl_batch* b) {
    marl_status st = sync_fate_state(b);
    if (st) return st;
    std::vector<marl_cell> cells;
    for (size_t r = 0; r < b->runs.size(); ++r) {
        BatchRun& R = b->runs[r];
        cells.resize(std::max<uint32_t>(R.n, 1));
        if (R.n) {
            if ((st = ensure_records(b, R.n))) return st;
            CK(launch_cells_to_records(R.t, R.n, b->d_records, b->stream));
            CK(cudaMemcpyAsync(b->h_records, b->d_records, (size_t)R.n * sizeof(marl_cell), cudaMemcpyDeviceToHost,
                               b->stream));
            CK(cudaStreamSynchronize(b->stream));
            std::memcpy(cells.data(), b->h_records, (size_t)R.n * sizeof(marl_cell));
            b->d2h += (size_t)R.n * sizeof(marl_cell);
        }
        const uint64_t tick = R.host.tick, td = R.host.total_div, tx = R.host.total_death, d1 = R.host.tick_div,
                       x1 = R.host.tick_death;
        R.host.adopt(cells.data(), R.n);
        R.host.tick = tick, R.host.total_div = td, R.host.total_death = tx, R.host.tick_div = d1,
        R.host.tick_death = x1;
    }
    b->device_fate = false;
    return MARL_OK;
}

marl_status step_once(marl_batch* b) {
    b->h2d_last = b->d2h_last = 0;
    b->epoch += 1;
    if (b->epoch == 0) {  // wrapped: clear stale completion epochs
        for (auto& R : b->runs) CK(cudaMemsetAsync(R.t.done, 0, (size_t)R.t.cap * 4, b->stream));
        b->epoch = 1;
    }
    fill_desc(b);
    const int span = span_begin(b);
    marl_status st = launch_tick(b);
    if (st) return st;
    span_end(b, span);
    CK(cudaStreamSynchronize(b->stream));
    resolve_spans(b);
    const size_t desc_bytes = b->runs.size() * sizeof(RunDesc);
    b->h2d += desc_bytes;
    b->d2h += b->rb_head_bytes;
    b->h2d_last += desc_bytes;
    b->d2h_last += b->rb_head_bytes;
    ++b->ticks;
    if ((st = collect_errors(b, b->h_scalars()->err))) return st;

    // The change lists, run after run.
    const uint32_t total = b->h_scalars()->changes;
    const marl_change* all = b->h_packed();
    if (total > kPrefetch) {
        if (b->overflow.size() < total) b->overflow.resize(total);
        std::memcpy(b->overflow.data(), b->h_packed(), (size_t)kPrefetch * sizeof(marl_change));
        CK(cudaMemcpy(b->overflow.data() + kPrefetch, b->d_packed() + kPrefetch,
                      (size_t)(total - kPrefetch) * sizeof(marl_change), cudaMemcpyDeviceToHost));
        b->d2h += (size_t)(total - kPrefetch) * sizeof(marl_change);
        b->d2h_last += (size_t)(total - kPrefetch) * sizeof(marl_change);
        all = b->overflow.data();
    }
    std::vector<uint32_t> offset(b->runs.size());
    uint32_t off = 0;
    for (size_t r = 0; r < b->runs.size(); ++r) {
        offset[r] = off;
        off += b->h_headers()[r].count;
    }
    if (off != total) return fail(MARL_ERR_STATE, "change counts %u != packed total %u", off, total);
    b->pool.run((int)b->runs.size(), [&](int r) {
        BatchRun& R = b->runs[r];
        R.st = R.host.process(all + offset[r], b->h_headers()[r].count, R.edits);
    });
    for (size_t r = 0; r < b->runs.size(); ++r)
        if (b->runs[r].st) return fail(b->runs[r].st, "run %zu: fate processing failed (status %d)", r, b->runs[r].st);
    return apply_edits(b);
}

}  // namespace

// ================================================================= ABI ====
extern "C" {

marl_status marl_batch_create(const marl_run_spec* specs, uint32_t n_runs, const marl_sim_params* sim,
                              marl_batch** out) {
    if (!out || !sim || (n_runs && !specs)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *out = nullptr;
    if (n_runs == 0) return fail(MARL_ERR_INVALID_INPUT, "a batch needs at least one run");
    if (sim->source_mode > MARL_SOURCES_DIRICHLET) return fail(MARL_ERR_INVALID_INPUT, "unknown source_mode");
    marl_status st;
    for (uint32_t r = 0; r < n_runs; ++r)
        if ((st = validate_dims(specs[r].gx, specs[r].gy, specs[r].gz))) return st;
    int dev = 0, sms = 0;
    if ((st = check_device(&dev, &sms))) return st;

    marl_batch* b = new (std::nothrow) marl_batch();
    if (!b) return fail(MARL_ERR_OUT_OF_MEMORY, "host allocation");
    b->device = dev;
    b->num_sms = sms;
    b->sim = *sim;
    derive_consts(b->sim, &b->fk, &b->ck);
    b->runs.resize(n_runs);
    auto bail = [&](marl_status s) {
        batch_free(b);
        return s;
    };
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    step(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
    step(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking));
    if (e != cudaSuccess) return bail(cuda_fail(e, "stream creation"));

    // Host side of every run: seeding with the run's own RNG.
    std::vector<std::vector<float>> fields(n_runs);
    std::vector<std::vector<marl_cell>> cells(n_runs);
    uint64_t total_cap = 0;
    for (uint32_t r = 0; r < n_runs; ++r) {
        const marl_run_spec& sp = specs[r];
        BatchRun& R = b->runs[r];
        R.g = Grid{sp.gx, sp.gy, sp.gz};
        const uint64_t V = R.g.V();
        R.cap = sp.cell_capacity ? sp.cell_capacity : (uint32_t)std::max<uint64_t>(1024, V / 8);
        R.host.init(sp.gx, sp.gy, sp.gz, *sim, sp.rng_seed);
        if ((st = R.host.seed_default(sp.seed_count, fields[r], cells[r]))) return bail(st);
        if (cells[r].size() > R.cap)
            return bail(fail(MARL_ERR_CAPACITY, "run %u: %zu seeded cells exceed capacity %u", r, cells[r].size(),
                             R.cap));
        R.n = (uint32_t)cells[r].size();
        total_cap += R.cap;
    }
    if (total_cap > 0xFFFFFFFFull) return bail(fail(MARL_ERR_CAPACITY, "total cell capacity exceeds 2^32"));
    b->packed_cap = (uint32_t)total_cap;

    // Device buffers.
    for (uint32_t r = 0; r < n_runs && e == cudaSuccess; ++r) {
        BatchRun& R = b->runs[r];
        const size_t V = R.g.V(), mbytes = (size_t)R.g.Z * R.g.Y * mask_pitch(R.g.X);
        step(cudaMalloc((void**)&R.field[0], V * 48));
        step(cudaMalloc((void**)&R.field[1], V * 48));
        step(cudaMalloc((void**)&R.mask, mbytes));
        step(cudaMalloc((void**)&R.cmap, V * 4));
        step(cudaMalloc((void**)&R.light, V * 4));
        step(cudaMalloc((void**)&R.c4, V * 4));
        step(cudaMalloc((void**)&R.changes, (size_t)R.cap * sizeof(marl_change)));
        if (e == cudaSuccess) step(alloc_table(R.t, R.cap));
        if (e == cudaSuccess) {
            step(cudaMemcpy(R.field[0], fields[r].data(), V * 48, cudaMemcpyHostToDevice));
            step(cudaMemset(R.field[1], 0, V * 48));
            step(cudaMemset(R.mask, 0, mbytes));
            step(cudaMemset(R.cmap, 0xFF, V * 4));
            step(cudaMemset(R.light, 0, V * 4));
            step(cudaMemset(R.c4, 0, V * 4));
            b->h2d += V * 48;
        }
    }
    const size_t rb_bytes = sizeof(BatchScalars) + (size_t)n_runs * sizeof(ChangeHeader) +
                            (size_t)b->packed_cap * sizeof(marl_change);
    b->rb_head_bytes = sizeof(BatchScalars) + (size_t)n_runs * sizeof(ChangeHeader) +
                       (size_t)std::min<uint32_t>(kPrefetch, b->packed_cap) * sizeof(marl_change);
    step(cudaMalloc((void**)&b->d_runs, (size_t)n_runs * sizeof(RunDesc)));
    step(cudaMallocHost((void**)&b->h_runs, (size_t)n_runs * sizeof(RunDesc)));
    step(cudaMalloc((void**)&b->d_maps, (size_t)n_runs * kMapsPerRun * sizeof(CUtensorMap)));
    step(cudaMalloc((void**)&b->d_rb, rb_bytes));
    step(cudaMallocHost((void**)&b->h_rb, b->rb_head_bytes));
    if (e == cudaSuccess) step(cudaMemset(b->d_rb, 0, sizeof(BatchScalars) + (size_t)n_runs * sizeof(ChangeHeader)));
    if (e != cudaSuccess) return bail(cuda_fail(e, "marl_batch_create"));

    // Run descriptors (the per-tick fields n, epoch, cell_base are filled by fill_desc).
    ChangeHeader* hdrs = b->d_headers();
    for (uint32_t r = 0; r < n_runs; ++r) {
        BatchRun& R = b->runs[r];
        RunDesc& d = b->h_runs[r];
        std::memset(&d, 0, sizeof(d));
        d.g = R.g;
        d.field[0] = R.field[0];
        d.field[1] = R.field[1];
        d.mask = R.mask;
        d.cmap = R.cmap;
        d.light = R.light;
        d.c4 = R.c4;
        d.t = R.t;
        d.hdr = hdrs + r;
        d.changes = R.changes;
        d.change_cap = R.cap;
    }
    fill_desc(b);
    if (cudaMemcpy(b->d_runs, b->h_runs, (size_t)n_runs * sizeof(RunDesc), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(MARL_ERR_CUDA, "descriptor upload"));

    // Light work list: (run, 32-column chunk, y).
    std::vector<int4> light_items;
    for (uint32_t r = 0; r < n_runs; ++r) {
        const Grid& g = b->runs[r].g;
        for (int y = 0; y < g.Y; ++y)
            for (int cx = 0; cx < (g.X + 31) / 32; ++cx) light_items.push_back(make_int4((int)r, cx, y, 0));
    }
    step(cudaMalloc((void**)&b->d_light_items, light_items.size() * sizeof(int4)));
    if (e == cudaSuccess)
        step(cudaMemcpy(b->d_light_items, light_items.data(), light_items.size() * sizeof(int4),
                        cudaMemcpyHostToDevice));
    b->n_light_items = (int)light_items.size();
    if (e != cudaSuccess) return bail(cuda_fail(e, "light work list"));

    // Seeded cells into each run's table.
    for (uint32_t r = 0; r < n_runs; ++r) {
        BatchRun& R = b->runs[r];
        if (cells[r].empty()) continue;
        if ((st = ensure_records(b, (uint32_t)cells[r].size()))) return bail(st);
        e = cudaMemcpy(b->d_records, cells[r].data(), cells[r].size() * sizeof(marl_cell), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = launch_cells_from_records(b->d_records, (uint32_t)cells[r].size(), 0, R.t, R.g, R.cmap, R.mask,
                                          &b->d_scalars()->err, nullptr);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return bail(cuda_fail(e, "cell upload"));
        b->h2d += cells[r].size() * sizeof(marl_cell);
    }
    if ((st = plan_tiles(b, 0, 16, b->stream))) return bail(st);
    // Everything issued on the legacy default stream above (copies, memsets)
    // completes before any launch on the batch's non-blocking stream.
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(cuda_fail(e, "marl_batch_create sync"));
    const unsigned hw = std::thread::hardware_concurrency();
    b->pool.resize((int)std::min<unsigned>(std::min<unsigned>(hw ? hw : 1, 64), n_runs) - 1);
    *out = b;
    return MARL_OK;
}

void marl_batch_destroy(marl_batch* b) { batch_free(b); }

marl_status marl_batch_set_stream(marl_batch* b, void* stream) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    CK(cudaStreamSynchronize(b->stream));
    if (b->own_stream) CK(cudaStreamDestroy(b->stream));
    b->stream = (cudaStream_t)stream;
    b->own_stream = false;
    return MARL_OK;
}

marl_status marl_batch_set_host_threads(marl_batch* b, int32_t threads) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    if (threads < 0) return fail(MARL_ERR_INVALID_INPUT, "threads < 0");
    if (threads == 0) {
        const unsigned hw = std::thread::hardware_concurrency();
        threads = (int32_t)std::min<unsigned>(hw ? hw : 1, 64);
    }
    b->pool.resize(std::max(0, std::min<int>(threads, (int)b->runs.size()) - 1));
    return MARL_OK;
}

marl_status marl_batch_set_tile(marl_batch* b, int32_t tile, int32_t zc) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    if (tile < 0 || tile >= diffusion_tile_count() || zc < 1 || zc > kMaxZ)
        return fail(MARL_ERR_INVALID_INPUT, "tile %d / zc %d out of range", tile, zc);
    marl_status st = plan_tiles(b, tile, zc, b->stream);
    invalidate_graphs(b);
    return st;
}

marl_status marl_batch_get_tile(marl_batch* b, int32_t* tile, int32_t* zc) {
    if (!b || !tile || !zc) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *tile = b->tile;
    *zc = b->zc;
    return MARL_OK;
}

marl_status marl_batch_autotune(marl_batch* b, int32_t reps, float* best_us_out) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    if (reps < 1) reps = 3;
    int maxZ = 0;
    for (auto& R : b->runs) maxZ = std::max(maxZ, R.g.Z);
    const int zcs[] = {4, 8, 10, 12, 13, 16, 21, 32, 64};  // 10-21: chunk counts that fill the SMs on common Z
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_tile = b->tile, best_zc = b->zc;
    uint32_t* err = &b->d_scalars()->err;
    marl_status st = MARL_OK;
    for (int tile = 0; tile < diffusion_tile_count() && !st; ++tile) {
        for (int zc : zcs) {
            if (zc > maxZ * 2 && zc != 4) continue;
            if ((st = plan_tiles(b, tile, zc, b->stream))) break;
            auto sub = [&] {
                return launch_diffuse_batch(tile, b->d_runs, b->d_maps, b->d_diff_items, b->n_diff_items, zc, b->fk,
                                            b->cur, 0, 0, err, b->stream);
            };
            for (int i = 0; i < 2; ++i) CK(sub());
            CK(cudaEventRecord(e0, b->stream));
            for (int i = 0; i < reps; ++i) CK(sub());
            CK(cudaEventRecord(e1, b->stream));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            const float us = ms * 1000.0f / reps;
            if (us < best) best = us, best_tile = tile, best_zc = zc;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    // The substeps wrote only the buffer that is not live.
    if ((st = plan_tiles(b, best_tile, best_zc, b->stream))) return st;
    invalidate_graphs(b);
    if (best_us_out) *best_us_out = best;
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaMemcpy(b->h_rb, b->d_rb, sizeof(BatchScalars), cudaMemcpyDeviceToHost));
    return collect_errors(b, b->h_scalars()->err);
}

marl_status marl_batch_set_graph(marl_batch* b, int32_t use_graph) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    b->use_graph = use_graph != 0;
    return MARL_OK;
}

marl_status marl_batch_set_device_fate(marl_batch* b, int32_t enable) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    const bool on = enable != 0;
    if (on == b->device_fate) return MARL_OK;
    return on ? enable_device_fate(b) : disable_device_fate(b);
}

marl_status marl_batch_set_surrogate(marl_batch* b, marl_surrogate* s, int32_t mode, float tol) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    if (mode != MARL_SURR_OFF && b->device_fate)
        return fail(MARL_ERR_STATE, "the batch surrogate runs with host fate (device fate is on)");
    if (mode != MARL_SURR_OFF && mode != MARL_SURR_GATED && mode != MARL_SURR_TRUSTED)
        return fail(MARL_ERR_INVALID_INPUT, "batch surrogate mode must be OFF, GATED or TRUSTED");
    if (mode != MARL_SURR_OFF && (!s || !s->prepared))
        return fail(MARL_ERR_STATE, "surrogate missing or not prepared");
    if (mode == MARL_SURR_GATED && !(tol >= 0.0f)) return fail(MARL_ERR_INVALID_INPUT, "tol must be >= 0");
    CK(cudaStreamSynchronize(b->stream));
    if (mode != MARL_SURR_OFF && !b->surr_xt) {
        uint64_t rows = 0;
        for (const auto& R : b->runs) rows += R.cap;
        if (rows > 0xFFFFFFFFull) return fail(MARL_ERR_CAPACITY, "batch capacity exceeds 2^32 cells");
        b->surr_rows = (uint32_t)rows;
        CK(cudaMalloc((void**)&b->surr_xt, rows * MARL_M_INT * 4));
        CK(cudaMalloc((void**)&b->surr_pred, rows * MARL_M_INT * 4));
        CK(cudaMalloc((void**)&b->surr_x, rows * mlp::kInPad * 2));
        CK(cudaMalloc((void**)&b->surr_status, rows));
        CK(cudaMalloc((void**)&b->surr_err, rows * 4));
        CK(cudaMalloc((void**)&b->surr_counters, 64));
        CK(cudaMemsetAsync(b->surr_counters, 0, 64, b->stream));
    }
    b->surr = mode == MARL_SURR_OFF ? nullptr : s;
    b->surr_mode = mode;
    b->surr_tol = tol;
    invalidate_graphs(b);
    return MARL_OK;
}

marl_status marl_batch_surrogate_counters(marl_batch* b, marl_surrogate_counters* out) {
    if (!b || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    std::memset(out, 0, sizeof(*out));
    CK(cudaStreamSynchronize(b->stream));
    if (!b->surr_counters) return MARL_OK;
    unsigned long long h[8];
    CK(cudaMemcpy(h, b->surr_counters, 64, cudaMemcpyDeviceToHost));
    out->cells = h[0];
    out->speculated = h[1];
    out->accepted = h[2];
    out->rejected = h[3];
    const uint32_t bits = (uint32_t)h[4];
    std::memcpy(&out->max_err, &bits, 4);
    return MARL_OK;
}

marl_status marl_batch_step(marl_batch* b, uint32_t ticks) {
    if (!b) return fail(MARL_ERR_INVALID_INPUT, "null batch");
    if (b->device_fate) return device_fate_steps(b, ticks);
    for (uint32_t t = 0; t < ticks; ++t) {
        marl_status st = step_once(b);
        if (st) return st;
    }
    return MARL_OK;
}

marl_status marl_batch_run_count(marl_batch* b, uint32_t* n) {
    if (!b || !n) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *n = (uint32_t)b->runs.size();
    return MARL_OK;
}

marl_status marl_batch_stats_get(marl_batch* b, uint32_t run, marl_engine_stats* s) {
    if (!b || !s) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (run >= b->runs.size()) return fail(MARL_ERR_INVALID_INPUT, "run %u of %zu", run, b->runs.size());
    marl_status st = sync_fate_state(b);
    if (st) return st;
    const HostRun& h = b->runs[run].host;
    s->tick = h.tick;
    s->population = b->device_fate ? b->runs[run].n : h.cells.size();
    s->total_divisions = h.total_div;
    s->total_deaths = h.total_death;
    s->tick_divisions = h.tick_div;
    s->tick_deaths = h.tick_death;
    // Transfers are not split by run: these are the batch's.
    s->h2d_bytes_last_tick = b->h2d_last;
    s->d2h_bytes_last_tick = b->d2h_last;
    return MARL_OK;
}

marl_status marl_batch_get_cells(marl_batch* b, uint32_t run, marl_cell* out, uint32_t cap, uint32_t* n_out) {
    if (!b || !n_out || (cap && !out)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (run >= b->runs.size()) return fail(MARL_ERR_INVALID_INPUT, "run %u of %zu", run, b->runs.size());
    marl_status sf = sync_fate_state(b);
    if (sf) return sf;
    BatchRun& R = b->runs[run];
    *n_out = R.n;
    if (R.n > cap) return fail(MARL_ERR_CAPACITY, "%u cells, buffer holds %u", R.n, cap);
    if (R.n == 0) return MARL_OK;
    marl_status st = ensure_records(b, R.n);
    if (st) return st;
    CK(launch_cells_to_records(R.t, R.n, b->d_records, b->stream));
    CK(cudaMemcpyAsync(b->h_records, b->d_records, (size_t)R.n * sizeof(marl_cell), cudaMemcpyDeviceToHost,
                       b->stream));
    CK(cudaStreamSynchronize(b->stream));
    std::memcpy(out, b->h_records, (size_t)R.n * sizeof(marl_cell));
    b->d2h += (size_t)R.n * sizeof(marl_cell);
    return MARL_OK;
}

marl_status marl_batch_get_field(marl_batch* b, uint32_t run, float* field) {
    if (!b || !field) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (run >= b->runs.size()) return fail(MARL_ERR_INVALID_INPUT, "run %u of %zu", run, b->runs.size());
    const BatchRun& R = b->runs[run];
    CK(cudaMemcpyAsync(field, R.field[b->cur], R.g.V() * 48, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->d2h += R.g.V() * 48;
    return MARL_OK;
}

marl_status marl_batch_get_light(marl_batch* b, uint32_t run, float* light) {
    if (!b || !light) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (run >= b->runs.size()) return fail(MARL_ERR_INVALID_INPUT, "run %u of %zu", run, b->runs.size());
    const BatchRun& R = b->runs[run];
    CK(cudaMemcpyAsync(light, R.light, R.g.V() * 4, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->d2h += R.g.V() * 4;
    return MARL_OK;
}

marl_status marl_batch_counters(marl_batch* b, marl_counters* out) {
    if (!b || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    CK(cudaStreamSynchronize(b->stream));
    resolve_spans(b);
    out->h2d_bytes = b->h2d;
    out->d2h_bytes = b->d2h;
    out->kernel_launches = b->launches;
    out->ticks = b->ticks;
    out->device_us = b->device_us;
    return MARL_OK;
}

}  // extern "C"
