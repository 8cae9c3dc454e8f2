// C-ABI layer of libmarl_cuda.so: the device context (field, light,
// occupancy, cell table), per-phase entry points, the per-tick sequence and the
// change-list / edit-list transfers.  Every entry point returns a marl_status;
// nothing throws across the ABI.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/marl_cuda.h"
#include "common.cuh"
#include "ctx_impl.h"
#include "surrogate.h"
#include "internal.h"

using namespace marl;

namespace marl {

static thread_local std::string g_last_error;

marl_status fail(marl_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

marl_status cuda_fail(cudaError_t e, const char* where) {
    return fail(e == cudaErrorMemoryAllocation ? MARL_ERR_OUT_OF_MEMORY : MARL_ERR_CUDA, "%s: %s", where,
                cudaGetErrorString(e));
}

#define CK(expr)                                              \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return cuda_fail(_e, #expr);   \
    } while (0)

marl_status check_device(int* dev, int* sms) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return fail(MARL_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    CK(cudaGetDevice(dev));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, *dev));
    if (prop.major != 10) return fail(MARL_ERR_NO_DEVICE, "device %s is sm_%d%d; this library is built for sm_100a",
                                      prop.name, prop.major, prop.minor);
    *sms = prop.multiProcessorCount;
    return MARL_OK;
}

void derive_consts(const marl_sim_params& p, FieldConsts* fk, CellConsts* ck) {
    // dt_sub in f32 as the reference computes it (crates/marl-field/src/field.rs:213).
    fk->dt_sub = p.diffusion_substeps ? p.dt / (float)p.diffusion_substeps : 0.0f;
    fk->alpha_eps = p.alpha_eps;
    fk->k_eps = p.k_eps;
    fk->c_max = p.c_max;
    for (int s = 0; s < MARL_S_EXT; ++s) {
        fk->d_voxel[s] = p.d_voxel[s];
        fk->lambda_decay[s] = p.lambda_decay[s];
    }
    fk->src_ox = p.source_rate_oxidant;
    fk->src_ca = p.source_rate_carbon;
    fk->src_re = p.source_rate_reductant;
    fk->prime_ox = p.boundary_prime_oxidant;
    fk->prime_ca = p.boundary_prime_carbon;
    fk->prime_re = p.boundary_prime_reductant;
    fk->source_mode = (int)p.source_mode;
    fk->surface_intensity = p.surface_intensity;
    // (-cell_absorption).exp() is a per-run constant; it is evaluated once with
    // the same libm call the reference makes (crates/marl-field/src/light.rs:41).
    fk->cell_factor = expf(-p.cell_absorption);
    fk->chemical_absorption = p.chemical_absorption;
    fk->light_floor = p.light_floor;
    ck->dt = p.dt;
    ck->c_max = p.c_max;
    ck->epsilon = p.epsilon;
    ck->thr = p.active_reaction_threshold;
    ck->lambda_maintenance = p.lambda_maintenance;
    ck->reaction_maintenance = p.reaction_maintenance;
    ck->hard_death_floor = p.hard_death_floor;
    ck->base_division_prep = p.base_division_prep;
    ck->prep_maintenance_multiplier = p.prep_maintenance_multiplier;
    ck->rush_penalty_rate = p.rush_penalty_rate;
    ck->wait_limit = kFlagSpinLimit;
    ck->schedule_here = 0;
    ck->hill_lo = p.hill_exponent_clamp_low;
    ck->hill_hi = p.hill_exponent_clamp_high;
}

marl_status validate_dims(int32_t gx, int32_t gy, int32_t gz) {
    if (gx < 1 || gy < 1 || gz < 1 || gx > kMaxXY || gy > kMaxXY || gz > kMaxZ)
        return fail(MARL_ERR_INVALID_INPUT, "grid %dx%dx%d outside 1..%d x 1..%d x 1..%d", gx, gy, gz, kMaxXY,
                    kMaxXY, kMaxZ);
    return MARL_OK;
}

template <typename T>
static cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, count * sizeof(T) + 16);
}

void free_table(CellTable& t) {
    void* ptrs[] = {t.internal, t.pos, t.age, t.state, t.tp_rate, t.tp_idx, t.rx, t.ef_par, t.ef_idx, t.fate,
                    t.lineage, t.cold, t.nb, t.dep, t.done, t.events};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    std::memset(&t, 0, sizeof(t));
}

cudaError_t alloc_table(CellTable& t, uint32_t cap) {
    std::memset(&t, 0, sizeof(t));
    t.cap = cap;
    cudaError_t e;
#define A(field, type, count)                           \
    if ((e = dalloc<type>(&t.field, (size_t)(count))) != cudaSuccess) return e;
    A(internal, float, (size_t)MARL_M_INT * cap);
    A(pos, uint32_t, cap);
    A(age, uint32_t, cap);
    A(state, uint32_t, cap);
    A(tp_rate, float2, (size_t)MARL_S_TRANSPORTERS * cap);
    A(tp_idx, uint4, cap);
    A(rx, uint4, (size_t)MARL_R_MAX * cap);
    A(ef_par, float2, (size_t)MARL_S_EFFECTORS * cap);
    A(ef_idx, uint4, cap);
    A(fate, float4, cap);
    A(lineage, uint64_t, cap);
    A(cold, float, (size_t)kColdFloats * cap);
    A(nb, uint32_t, cap);
    A(dep, int32_t, (size_t)6 * cap);
    A(done, uint32_t, cap);
    A(events, uint8_t, cap);
#undef A
    if ((e = cudaMemset(t.done, 0, (size_t)cap * 4)) != cudaSuccess) return e;
    return cudaMemset(t.events, 0, cap);
}

void ctx_free(marl_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* dev[] = {c->field[0], c->field[1], c->mask, c->cmap, c->light, c->c4, c->d_hdr, c->d_changes, c->d_block_counts,
                   c->d_edit, c->d_mass_partial, c->d_mass_out, c->d_records, c->d_occ_stage, c->d_seam_mask,
                   c->d_events_stage, c->surr_xt, c->surr_pred, c->surr_x, c->surr_status, c->surr_err,
                   c->surr_counters, c->receptor_act};
    for (void* p : dev)
        if (p) cudaFree(p);
    void* host[] = {c->h_hdr, c->h_edit, c->h_records, c->h_mass};
    for (void* p : host)
        if (p) cudaFreeHost(p);
    free_table(c->t);
    free_fate(c->fate);
    if (c->d_fate_run) cudaFree(c->d_fate_run);
    for (auto* v : {&c->span_pool, &c->spans_pending})
        for (auto& s : *v) {
            cudaEventDestroy(s.a);
            cudaEventDestroy(s.b);
        }
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

marl_status ensure_edit_capacity(marl_ctx* c, size_t bytes) {
    if (bytes <= c->edit_bytes) return MARL_OK;
    size_t nb = c->edit_bytes ? c->edit_bytes : (1 << 16);
    while (nb < bytes) nb *= 2;
    if (c->d_edit) CK(cudaFree(c->d_edit));
    if (c->h_edit) CK(cudaFreeHost(c->h_edit));
    c->d_edit = nullptr;
    c->h_edit = nullptr;
    c->edit_bytes = 0;
    CK(cudaMalloc(&c->d_edit, nb));
    CK(cudaMallocHost(&c->h_edit, nb));
    c->edit_bytes = nb;
    return MARL_OK;
}

marl_status ensure_records(marl_ctx* c, uint32_t n) {
    if (n <= c->records_cap) return MARL_OK;
    uint32_t cap = c->records_cap ? c->records_cap : 1024;
    while (cap < n) cap *= 2;
    if (c->d_records) CK(cudaFree(c->d_records));
    if (c->h_records) CK(cudaFreeHost(c->h_records));
    c->d_records = nullptr;
    c->h_records = nullptr;
    c->records_cap = 0;
    CK(cudaMalloc((void**)&c->d_records, (size_t)cap * sizeof(marl_cell)));
    CK(cudaMallocHost((void**)&c->h_records, (size_t)cap * sizeof(marl_cell)));
    c->records_cap = cap;
    return MARL_OK;
}

CellLaunch cell_launch(marl_ctx* c) {
    CellLaunch a;
    a.t = c->t;
    a.n = c->n;
    if (c->n_on_device) {  // device fate: the kernels read the population
        a.n = c->t.cap;
        a.n_dev = &c->fate.fs->n;
    }
    a.g = c->g;
    a.mask = c->mask;
    a.cmap = c->cmap;
    a.field = c->field[c->cur];
    a.light = c->light;
    a.k = c->ck;
    a.k.wait_limit = c->wait_limit;
    a.epoch = c->epoch;
    a.ticket = &c->d_hdr->pad[0];
    a.lanes = c->cell_lanes;
    a.err = &c->d_hdr->err;
    a.act = c->receptor_act;
    return a;
}

// `substeps` substeps; with emit_c4 the last one also writes species 4
// compactly into c->c4 for the light scan (returns whether it did).
marl_status enqueue_diffuse(marl_ctx* c, uint32_t substeps, bool fuse_sources, bool emit_c4 = false,
                            bool* c4_written = nullptr) {
    if (c4_written) *c4_written = false;
    if (substeps > 0) c->c4_valid = false;
    if (substeps == 0) {
        if (fuse_sources) {
            CK(launch_sources(c->field[c->cur], c->g, c->fk, c->stream));
            ++c->launches;
        }
        return MARL_OK;
    }
    for (uint32_t i = 0; i < substeps; ++i) {
        float* c4 = (emit_c4 && i + 1 == substeps) ? c->c4 : nullptr;
        CK(launch_diffuse(c->plan, c->cur, c->g, c->fk, (fuse_sources && i == 0) ? 1 : 0, c4, &c->d_hdr->err,
                          c->stream));
        c->cur ^= 1;
        ++c->launches;
        if (c4) c->c4_valid = true;
        if (c4 && c4_written) *c4_written = true;
    }
    return MARL_OK;
}

marl_status enqueue_cell_phase(marl_ctx* c) {
    if (c->n == 0 && !c->n_on_device) return MARL_OK;
    c->c4_valid = false;  // the scatter writes every species
    CellLaunch a = cell_launch(c);
    // When every cell gets a lane at once and nothing else needs the table's
    // schedule this phase (no surrogate, no dependency hold, population on
    // the host), the cell kernel computes each cell's schedule while staging
    // it, and the schedule kernel is skipped.  The table's schedule is then
    // left stale (schedule_dirty stays set) for any later phase that reads it.
    const bool schedule_here = (!c->surr || c->surr_mode == MARL_SURR_OFF) && c->hold_cell < 0 &&
                               !c->n_on_device && cell_tick_covers(c->n, c->cell_lanes, c->num_sms);
    a.k.schedule_here = schedule_here ? 1u : 0u;
    if (c->schedule_dirty && !schedule_here) {
        CK(launch_cell_schedule(a, c->stream));
        c->schedule_dirty = false;
        ++c->launches;
    }
    if (c->hold_cell >= 0) {  // marl_ctx_test_hold_dependency: this phase only
        CK(launch_hold_dependency(c->t, (uint32_t)c->hold_cell, c->hold_face, c->hold_slot, &c->d_hdr->err,
                                  c->stream));
        ++c->launches;
        c->hold_cell = -1;
        c->schedule_dirty = true;  // the next phase recomputes the true dependencies
    }
    c->epoch += 1;
    if (c->epoch == 0) {  // wrapped: clear stale epochs
        CK(cudaMemsetAsync(c->t.done, 0, (size_t)c->t.cap * 4, c->stream));
        c->epoch = 1;
    }
    a.epoch = c->epoch;
    CK(cudaMemsetAsync(&c->d_hdr->pad[0], 0, 4, c->stream));
    uint32_t captured = 0;
    if (c->surr && c->surr_mode == MARL_SURR_CAPTURE) {
        marl_surrogate* s = c->surr;
        captured = s->rows < s->cfg.max_pairs ? std::min(c->n, s->cfg.max_pairs - s->rows) : 0;
        a.mode = captured ? kModeCapture : kModePlain;
        a.sv.raw = s->raw + (size_t)s->rows * MARL_SURR_RAW_STRIDE;
        a.sv.raw_rows = captured;
    } else if (c->surr && (c->surr_mode == MARL_SURR_GATED || c->surr_mode == MARL_SURR_TRUSTED)) {
        a.mode = c->surr_mode == MARL_SURR_GATED ? kModeGated : kModeTrusted;
        CK(launch_surrogate_prepass(a, c->surr->norm, c->surr_xt, c->surr_x, c->num_sms, c->stream));
        marl_status st = surrogate_infer(c->surr, reinterpret_cast<const __nv_bfloat16*>(c->surr_x), c->n,
                                         c->surr_pred, c->t.cap, c->stream);
        if (st) return st;
        c->launches += 4;
        a.sv.xt = c->surr_xt;
        a.sv.pred = c->surr_pred;
        a.sv.tol = c->surr_tol;
        a.sv.status = c->surr_status;
        a.sv.err = c->surr_err;
        a.sv.row0 = 0;
        a.sv.ld = c->t.cap;
    }
    CK(launch_cell_tick(a, c->num_sms, c->stream));
    ++c->launches;
    if (a.mode == kModeGated || a.mode == kModeTrusted) {
        CK(launch_surrogate_count(c->surr_status, c->surr_err, c->n, c->surr_counters,
                                  reinterpret_cast<uint32_t*>(c->surr_counters + 4), c->stream));
        ++c->launches;
    }
    if (captured) c->surr->rows += captured;
    return MARL_OK;
}

// Device-time spans (marl_counters::device_us).
static int span_begin(marl_ctx* c) {
    marl_ctx::Span s;
    if (!c->span_pool.empty()) {
        s = c->span_pool.back();
        c->span_pool.pop_back();
    } else if (cudaEventCreate(&s.a) != cudaSuccess || cudaEventCreate(&s.b) != cudaSuccess) {
        return -1;
    }
    cudaEventRecord(s.a, c->stream);
    c->spans_pending.push_back(s);
    return (int)c->spans_pending.size() - 1;
}

static void span_end(marl_ctx* c, int idx) {
    if (idx >= 0) cudaEventRecord(c->spans_pending[idx].b, c->stream);
}

// Call only after the stream has synchronized.
static void resolve_spans(marl_ctx* c) {
    for (auto& s : c->spans_pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, s.a, s.b) == cudaSuccess) c->device_us += 1000.0 * ms;
        c->span_pool.push_back(s);
    }
    c->spans_pending.clear();
}

// Reads and clears the device error word; maps it to a status.
marl_status collect_device_errors(marl_ctx* c, uint32_t err_bits) {
    if (!err_bits) return MARL_OK;
    cudaMemsetAsync(&c->d_hdr->err, 0, 4, c->stream);
    if (err_bits & (kErrTimeoutMbar | kErrTimeoutDeps))
        return fail(MARL_ERR_TIMEOUT, "device wait gave up (error bits 0x%x)", err_bits);
    if (err_bits & kErrCapacity)
        return fail(MARL_ERR_CAPACITY, "cell table full: births dropped (error bits 0x%x)", err_bits);
    if (err_bits & kErrFateChain)
        return fail(MARL_ERR_STATE, "inconsistent death events in device fate (error bits 0x%x)", err_bits);
    return fail(MARL_ERR_INVALID_INPUT, "device rejected input (error bits 0x%x)", err_bits);
}

marl_status sync_and_check(marl_ctx* c) {
    CK(cudaMemcpyAsync(c->h_hdr, c->d_hdr, sizeof(ChangeHeader), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    resolve_spans(c);
    return collect_device_errors(c, c->h_hdr->err);
}

}  // namespace marl

// ================================================================= ABI ====
extern "C" {

uint32_t marl_abi_version(void) { return 0x000100; }

uint64_t marl_internal_ctx_h2d(marl_ctx* c) { return c ? c->h2d_bytes : 0; }
uint64_t marl_internal_ctx_d2h(marl_ctx* c) { return c ? c->d2h_bytes : 0; }

const char* marl_last_error(void) { return g_last_error.c_str(); }

marl_status marl_sim_params_default(marl_sim_params* p) {
    if (!p) return fail(MARL_ERR_INVALID_INPUT, "null params");
    // crates/marl-config/src/lib.rs:108-168
    std::memset(p, 0, sizeof(*p));
    p->dx = 100.0e-6f;
    p->dt = 1.0f;
    p->diffusion_substeps = 10;
    static const float d[12] = {0.0f, 1.5f, 1.0f, 1.2f, 0.8f, 0.5f, 0.5f, 0.1f, 0.3f, 0.3f, 0.3f, 0.3f};
    static const float l[12] = {0.0f, 0.01f, 0.01f, 0.005f, 0.03f, 0.05f, 0.05f, 0.002f, 0.01f, 0.01f, 0.01f, 0.01f};
    std::memcpy(p->d_voxel, d, sizeof(d));
    std::memcpy(p->lambda_decay, l, sizeof(l));
    p->source_rate_oxidant = 0.4f;
    p->source_rate_carbon = 0.15f;
    p->source_rate_reductant = 0.5f;
    p->epsilon = 0.001f;
    p->c_max = 10.0f;
    p->lambda_maintenance = 0.12f;
    p->hard_death_floor = 0.01f;
    p->reaction_maintenance = 0.003f;
    p->base_division_prep = 20.0f;
    p->prep_maintenance_multiplier = 2.0f;
    p->rush_penalty_rate = 0.05f;
    p->alpha_eps = 0.8f;
    p->k_eps = 2.0f;
    p->light_efficiency = 0.0f;
    p->surface_intensity = 1.0f;
    p->cell_absorption = 0.3f;
    p->chemical_absorption = 0.05f;
    p->light_floor = 1e-7f;
    p->mutation_stddev = 0.1f;
    p->structural_mutation_rate_mult = 0.1f;
    p->meta_mutation_rate = 0.01f;
    p->meta_mutation_clamp_low = 0.001f;
    p->meta_mutation_clamp_high = 0.5f;
    p->hill_exponent_clamp_low = 0.5f;
    p->hill_exponent_clamp_high = 8.0f;
    p->active_reaction_threshold = 1e-9f;
    p->seed_margin = 5;
    p->phototroph_z_lo = 0.0f;
    p->phototroph_z_hi = 3.0f;
    p->chemolithotroph_z_lo = 80.0f;
    p->chemolithotroph_z_hi = 130.0f;
    p->anaerobe_z_lo = 120.0f;
    p->anaerobe_z_hi = 180.0f;
    p->division_neighbor_distance = 2;
    p->boundary_prime_layers = 2;
    p->boundary_prime_oxidant = 0.5f;
    p->boundary_prime_carbon = 0.3f;
    p->boundary_prime_reductant = 0.5f;
    p->source_mode = MARL_SOURCES_ADDITIVE;
    return MARL_OK;
}

marl_status marl_ctx_create(int32_t gx, int32_t gy, int32_t gz, const marl_sim_params* sim, uint32_t cell_capacity,
                            marl_ctx** out) {
    if (!out || !sim) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *out = nullptr;
    marl_status st = validate_dims(gx, gy, gz);
    if (st) return st;
    if (cell_capacity == 0) return fail(MARL_ERR_INVALID_INPUT, "cell_capacity must be >= 1");
    if (sim->source_mode > MARL_SOURCES_DIRICHLET) return fail(MARL_ERR_INVALID_INPUT, "unknown source_mode");
    int dev = 0, sms = 0;
    if ((st = check_device(&dev, &sms))) return st;

    marl_ctx* c = new (std::nothrow) marl_ctx();
    if (!c) return fail(MARL_ERR_OUT_OF_MEMORY, "host allocation");
    c->device = dev;
    c->num_sms = sms;
    c->g = Grid{gx, gy, gz};
    c->sim = *sim;
    derive_consts(c->sim, &c->fk, &c->ck);
    const size_t V = c->g.V();
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    step(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
    step(cudaMalloc((void**)&c->field[0], V * 48));
    step(cudaMalloc((void**)&c->field[1], V * 48));
    step(cudaMalloc((void**)&c->mask, (size_t)gz * gy * mask_pitch(gx)));
    step(cudaMalloc((void**)&c->cmap, V * 4));
    step(cudaMalloc((void**)&c->light, V * 4));
    step(cudaMalloc((void**)&c->c4, V * 4));
    step(cudaMalloc((void**)&c->d_hdr, sizeof(ChangeHeader)));
    step(cudaMallocHost((void**)&c->h_hdr, sizeof(ChangeHeader) + (size_t)kPrefetchChanges * sizeof(marl_change)));
    step(cudaMalloc((void**)&c->d_changes, (size_t)cell_capacity * sizeof(marl_change)));
    step(cudaMalloc((void**)&c->d_block_counts, (size_t)compaction_blocks(cell_capacity) * 4));
    step(cudaMalloc((void**)&c->d_mass_partial, mass_partial_doubles() * 8));
    step(cudaMalloc((void**)&c->d_mass_out, 12 * 8));
    step(cudaMallocHost((void**)&c->h_mass, 12 * 8));
    step(cudaMalloc((void**)&c->d_events_stage, cell_capacity));
    if (e == cudaSuccess) e = alloc_table(c->t, cell_capacity);
    if (e == cudaSuccess) {
        step(cudaMemset(c->field[0], 0, V * 48));
        step(cudaMemset(c->field[1], 0, V * 48));
        step(cudaMemset(c->mask, 0, (size_t)gz * gy * mask_pitch(gx)));
        step(cudaMemset(c->cmap, 0xFF, V * 4));
        step(cudaMemset(c->light, 0, V * 4));
        step(cudaMemset(c->d_hdr, 0, sizeof(ChangeHeader)));
    }
    if (e != cudaSuccess) {
        marl_status s2 = cuda_fail(e, "marl_ctx_create");
        ctx_free(c);
        return s2;
    }
    c->cur = 0;
    c->n = 0;
    c->epoch = 0;
    c->schedule_dirty = true;
    if (!plan_diffusion(&c->plan, c->field[0], c->field[1], c->mask, c->g, 0, 16)) {
        ctx_free(c);
        return fail(MARL_ERR_CUDA, "cuTensorMapEncodeTiled failed for the field/mask tensor maps");
    }
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        marl_status s2 = cuda_fail(e, "marl_ctx_create sync");
        ctx_free(c);
        return s2;
    }
    *out = c;
    return MARL_OK;
}

void marl_ctx_destroy(marl_ctx* c) { ctx_free(c); }

marl_status marl_ctx_set_stream(marl_ctx* c, void* stream) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    CK(cudaStreamSynchronize(c->stream));
    if (c->own_stream) CK(cudaStreamDestroy(c->stream));
    // NULL is the legacy default stream (what torch reports as stream 0).
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return MARL_OK;
}

marl_status marl_ctx_set_params(marl_ctx* c, const marl_sim_params* sim) {
    if (!c || !sim) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (sim->source_mode > MARL_SOURCES_DIRICHLET) return fail(MARL_ERR_INVALID_INPUT, "unknown source_mode");
    c->sim = *sim;
    derive_consts(c->sim, &c->fk, &c->ck);
    return MARL_OK;
}

marl_status marl_ctx_synchronize(marl_ctx* c) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    return sync_and_check(c);
}

marl_status marl_ctx_counters(marl_ctx* c, marl_counters* out) {
    if (!c || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    marl_status st = sync_and_check(c);
    out->h2d_bytes = c->h2d_bytes;
    out->d2h_bytes = c->d2h_bytes;
    out->kernel_launches = c->launches;
    out->ticks = c->ticks;
    out->device_us = c->device_us;
    return st;
}

marl_status marl_ctx_set_tile(marl_ctx* c, int32_t tile, int32_t zc) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (tile < 0 || tile >= diffusion_tile_count() || zc < 1 || zc > kMaxZ)
        return fail(MARL_ERR_INVALID_INPUT, "tile %d / zc %d out of range", tile, zc);
    DiffusionPlan p;
    if (!plan_diffusion(&p, c->field[0], c->field[1], c->mask, c->g, tile, zc))
        return fail(MARL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    c->plan = p;
    return MARL_OK;
}

marl_status marl_ctx_set_cell_lanes(marl_ctx* c, uint32_t lanes) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (lanes < 1 || lanes > 32) return fail(MARL_ERR_INVALID_INPUT, "lanes %u outside 1..32", lanes);
    c->cell_lanes = lanes;
    return MARL_OK;
}

marl_status marl_ctx_set_wait_limit(marl_ctx* c, uint32_t polls) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    c->wait_limit = polls ? polls : kFlagSpinLimit;
    return MARL_OK;
}

marl_status marl_ctx_test_hold_dependency(marl_ctx* c, uint32_t cell, uint32_t face, uint32_t slot) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    if (cell >= c->n || face >= 6 || slot < c->n || slot >= c->t.cap)
        return fail(MARL_ERR_INVALID_INPUT, "hold: cell %u (population %u), face %u, slot %u (capacity %u)", cell,
                    c->n, face, slot, c->t.cap);
    c->hold_cell = (int32_t)cell;
    c->hold_face = (int)face;
    c->hold_slot = slot;
    return MARL_OK;
}

marl_status marl_ctx_set_receptor_output(marl_ctx* c, int32_t enable) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (enable && !c->receptor_act) {
        CK(cudaMalloc((void**)&c->receptor_act, (size_t)MARL_S_RECEPTORS * c->t.cap * sizeof(float)));
        CK(cudaMemsetAsync(c->receptor_act, 0, (size_t)MARL_S_RECEPTORS * c->t.cap * sizeof(float), c->stream));
    } else if (!enable && c->receptor_act) {
        CK(cudaStreamSynchronize(c->stream));
        cudaFree(c->receptor_act);
        c->receptor_act = nullptr;
    }
    return MARL_OK;
}

marl_status marl_ctx_download_receptor_activations(marl_ctx* c, float* out, uint32_t cap, uint32_t* n_out) {
    if (!c || !n_out || (cap && !out)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (!c->receptor_act) return fail(MARL_ERR_STATE, "receptor output is off (marl_ctx_set_receptor_output)");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    const uint32_t n = c->n;
    *n_out = n;
    if (n > cap) return fail(MARL_ERR_CAPACITY, "%u cells, buffer holds %u", n, cap);
    std::vector<float> rows((size_t)MARL_S_RECEPTORS * n);
    for (int i = 0; i < MARL_S_RECEPTORS && n; ++i)
        CK(cudaMemcpyAsync(rows.data() + (size_t)i * n, c->receptor_act + (size_t)i * c->t.cap, (size_t)n * 4,
                           cudaMemcpyDeviceToHost, c->stream));
    marl_status st = sync_and_check(c);
    if (st) return st;
    for (uint32_t j = 0; j < n; ++j)
        for (int i = 0; i < MARL_S_RECEPTORS; ++i) out[(size_t)j * MARL_S_RECEPTORS + i] = rows[(size_t)i * n + j];
    c->d2h_bytes += rows.size() * 4;
    return MARL_OK;
}

marl_status marl_ctx_get_tile(marl_ctx* c, int32_t* tile, int32_t* zc) {
    if (!c || !tile || !zc) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    *tile = c->plan.tile;
    *zc = c->plan.zc;
    return MARL_OK;
}

// Tile autotuner: times `reps` substeps for every (tile shape, z-chunk)
// candidate on this context's own grid with CUDA events and keeps the fastest.
// All candidates compute bit-identical results; the field is restored.
marl_status marl_ctx_autotune(marl_ctx* c, int32_t reps, float* best_us_out) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (reps < 1) reps = 3;
    const int zcs[] = {4, 8, 10, 12, 13, 16, 21, 32, 64};  // 10-21: chunk counts that fill the SMs on common Z
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    DiffusionPlan best_plan = c->plan;
    const int saved_cur = c->cur;
    for (int tile = 0; tile < diffusion_tile_count(); ++tile) {
        for (int zc : zcs) {
            if (zc > c->g.Z * 2 && zc != 4) continue;
            DiffusionPlan p;
            if (!plan_diffusion(&p, c->field[0], c->field[1], c->mask, c->g, tile, zc)) continue;
            std::swap(p, c->plan);
            // warm-up, then timed
            for (int i = 0; i < 2; ++i)
                CK(launch_diffuse(c->plan, c->cur, c->g, c->fk, 0, nullptr, &c->d_hdr->err, c->stream));
            CK(cudaEventRecord(e0, c->stream));
            for (int i = 0; i < reps; ++i)
                CK(launch_diffuse(c->plan, c->cur, c->g, c->fk, 0, nullptr, &c->d_hdr->err, c->stream));
            CK(cudaEventRecord(e1, c->stream));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            const float us = ms * 1000.0f / reps;
            if (us < best) {
                best = us;
                best_plan = c->plan;
            }
            std::swap(p, c->plan);
        }
    }
    c->plan = best_plan;
    c->cur = saved_cur;  // substeps wrote only the other buffer
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_us_out) *best_us_out = best;
    return sync_and_check(c);
}

marl_status marl_upload_field(marl_ctx* c, const float* f) {
    if (!c || !f) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    c->c4_valid = false;
    CK(cudaMemcpyAsync(c->field[c->cur], f, c->g.V() * 48, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return MARL_OK;
}

marl_status marl_download_field(marl_ctx* c, float* f) {
    if (!c || !f) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    CK(cudaMemcpyAsync(f, c->field[c->cur], c->g.V() * 48, cudaMemcpyDeviceToHost, c->stream));
    return sync_and_check(c);
}

marl_status marl_upload_light(marl_ctx* c, const float* l) {
    if (!c || !l) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    CK(cudaMemcpyAsync(c->light, l, c->g.V() * 4, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return MARL_OK;
}

marl_status marl_download_light(marl_ctx* c, float* l) {
    if (!c || !l) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    CK(cudaMemcpyAsync(l, c->light, c->g.V() * 4, cudaMemcpyDeviceToHost, c->stream));
    return sync_and_check(c);
}

marl_status marl_upload_cells(marl_ctx* c, const marl_cell* cells, uint32_t n) {
    if (!c || (n && !cells)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    if (n > c->t.cap) return fail(MARL_ERR_CAPACITY, "%u cells exceed capacity %u", n, c->t.cap);
    // Positions must be in the grid and unique (cell_map is a map).
    std::vector<uint8_t> seen(c->g.V(), 0);
    for (uint32_t i = 0; i < n; ++i) {
        const uint16_t* p = cells[i].pos;
        if (p[0] >= c->g.X || p[1] >= c->g.Y || p[2] >= c->g.Z)
            return fail(MARL_ERR_INVALID_INPUT, "cell %u at (%u,%u,%u) is outside the grid", i, p[0], p[1], p[2]);
        const size_t v = ((size_t)p[2] * c->g.Y + p[1]) * c->g.X + p[0];
        if (seen[v]) return fail(MARL_ERR_INVALID_INPUT, "cell %u duplicates position (%u,%u,%u)", i, p[0], p[1], p[2]);
        seen[v] = 1;
    }
    marl_status st = ensure_records(c, n ? n : 1);
    if (st) return st;
    if (n) std::memcpy(c->h_records, cells, (size_t)n * sizeof(marl_cell));
    CK(cudaMemsetAsync(c->cmap, 0xFF, c->g.V() * 4, c->stream));
    CK(cudaMemsetAsync(c->mask, 0, (size_t)c->g.Z * c->g.Y * mask_pitch(c->g.X), c->stream));
    if (n) {
        CK(cudaMemcpyAsync(c->d_records, c->h_records, (size_t)n * sizeof(marl_cell), cudaMemcpyHostToDevice,
                           c->stream));
        CK(launch_cells_from_records(c->d_records, n, 0, c->t, c->g, c->cmap, c->mask, &c->d_hdr->err, c->stream));
    }
    c->n = n;
    c->schedule_dirty = true;
    return sync_and_check(c);
}

marl_status marl_download_cells(marl_ctx* c, marl_cell* out, uint32_t cap, uint32_t* n_out) {
    if (!c || (!out && cap)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    if (n_out) *n_out = c->n;
    const uint32_t n = c->n < cap ? c->n : cap;
    if (n == 0) return MARL_OK;
    marl_status st = ensure_records(c, n);
    if (st) return st;
    CK(launch_cells_to_records(c->t, n, c->d_records, c->stream));
    CK(cudaMemcpyAsync(c->h_records, c->d_records, (size_t)n * sizeof(marl_cell), cudaMemcpyDeviceToHost, c->stream));
    st = sync_and_check(c);
    if (st) return st;
    std::memcpy(out, c->h_records, (size_t)n * sizeof(marl_cell));
    if (c->n > cap) return fail(MARL_ERR_CAPACITY, "%u cells, buffer holds %u", c->n, cap);
    return MARL_OK;
}

marl_status marl_cell_count(marl_ctx* c, uint32_t* n) {
    if (!c || !n) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    *n = c->n;
    return MARL_OK;
}

marl_status marl_download_occupancy(marl_ctx* c, uint8_t* occ) {
    if (!c || !occ) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (!c->d_occ_stage) CK(cudaMalloc((void**)&c->d_occ_stage, c->g.V()));
    CK(launch_unpack_mask(c->mask, c->d_occ_stage, c->g, c->stream));
    CK(cudaMemcpyAsync(occ, c->d_occ_stage, c->g.V(), cudaMemcpyDeviceToHost, c->stream));
    return sync_and_check(c);
}

marl_status marl_apply_boundary_sources(marl_ctx* c) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    CK(launch_sources(c->field[c->cur], c->g, c->fk, c->stream));
    return MARL_OK;
}

marl_status marl_diffuse(marl_ctx* c, uint32_t substeps, int32_t fuse_sources) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (substeps > 0 && c->sim.diffusion_substeps == 0)
        return fail(MARL_ERR_INVALID_INPUT, "sim.diffusion_substeps == 0 gives no dt_sub");
    // The last substep also writes species 4 compactly for a following light scan.
    return enqueue_diffuse(c, substeps, fuse_sources != 0, true);
}

marl_status marl_light_update(marl_ctx* c) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    CK(launch_light(c->c4_valid ? c->c4 : nullptr, c->field[c->cur], c->mask, c->light, c->g, c->fk, c->stream));
    ++c->launches;
    return MARL_OK;
}

marl_status marl_cell_phase(marl_ctx* c, uint8_t* events_out) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    marl_status st = enqueue_cell_phase(c);
    if (st) return st;
    if (events_out && c->n) {
        CK(cudaMemcpyAsync(events_out, c->t.events, c->n, cudaMemcpyDeviceToHost, c->stream));
        return sync_and_check(c);
    }
    return MARL_OK;
}

marl_status marl_tick(marl_ctx* c, marl_change* changes, uint32_t cap, uint32_t* n_changes) {
    if (!c || !n_changes || (cap && !changes)) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    *n_changes = 0;
    // crates/marl-sim/src/lib.rs:164-217: sources (fused into the first
    // substep), diffusion, light, the cell loop; then the ordered change list.
    const int span = span_begin(c);
    bool c4_ready = false;
    marl_status st = enqueue_diffuse(c, c->sim.diffusion_substeps, true, true, &c4_ready);
    if (st) return st;
    CK(launch_light(c4_ready ? c->c4 : nullptr, c->field[c->cur], c->mask, c->light, c->g, c->fk, c->stream));
    ++c->launches;
    if ((st = enqueue_cell_phase(c))) return st;
    CK(launch_compact_events(c->t, c->n, c->d_block_counts, c->d_hdr, c->d_changes, c->t.cap, c->stream));
    c->launches += 2;
    // The header and the first kPrefetchChanges entries come back together.
    const size_t pre = (size_t)kPrefetchChanges * sizeof(marl_change);
    CK(cudaMemcpyAsync(c->h_hdr, c->d_hdr, sizeof(ChangeHeader), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->h_changes_prefix(), c->d_changes, pre, cudaMemcpyDeviceToHost, c->stream));
    span_end(c, span);
    CK(cudaStreamSynchronize(c->stream));
    resolve_spans(c);
    ++c->ticks;
    c->d2h_bytes += sizeof(ChangeHeader) + pre;
    const uint32_t err = c->h_hdr->err;
    const uint32_t count = c->n ? c->h_hdr->count : 0;
    if (err) return collect_device_errors(c, err);
    const uint32_t first = count < kPrefetchChanges ? count : kPrefetchChanges;
    const uint32_t w1 = first < cap ? first : cap;
    if (w1) std::memcpy(changes, c->h_changes_prefix(), (size_t)w1 * sizeof(marl_change));
    if (count > kPrefetchChanges && cap > kPrefetchChanges) {
        const uint32_t rest = (count < cap ? count : cap) - kPrefetchChanges;
        CK(cudaMemcpy(changes + kPrefetchChanges, c->d_changes + kPrefetchChanges, (size_t)rest * sizeof(marl_change),
                      cudaMemcpyDeviceToHost));
        c->d2h_bytes += (size_t)rest * sizeof(marl_change);
    }
    *n_changes = count;
    if (count > cap) return fail(MARL_ERR_CAPACITY, "%u changes, buffer holds %u", count, cap);
    return MARL_OK;
}

marl_status marl_ctx_run_ticks(marl_ctx* c, uint32_t ticks) {
    if (!c) return fail(MARL_ERR_INVALID_INPUT, "null ctx");
    if (c->surr && c->surr_mode != MARL_SURR_OFF)
        return fail(MARL_ERR_STATE, "device fate runs with the surrogate off (mode %d attached)", c->surr_mode);
    marl_status st = begin_device_population(c);
    if (st) return st;
    // crates/marl-sim/src/lib.rs:160-277 per tick, all on the stream: sources
    // (fused into the first substep), diffusion, light, the cell loop, fate.
    const int span = span_begin(c);
    for (uint32_t k = 0; k < ticks; ++k) {
        bool c4_ready = false;
        if ((st = enqueue_diffuse(c, c->sim.diffusion_substeps, true, true, &c4_ready))) return st;
        CK(launch_light(c4_ready ? c->c4 : nullptr, c->field[c->cur], c->mask, c->light, c->g, c->fk, c->stream));
        ++c->launches;
        c->schedule_dirty = true;  // the previous fate step may have moved cells
        if ((st = enqueue_cell_phase(c))) return st;
        if ((st = enqueue_fate(c))) return st;
        ++c->ticks;
    }
    span_end(c, span);
    return MARL_OK;
}

marl_status marl_apply_edits(marl_ctx* c, const marl_edit_list* e) {
    if (!c || !e) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->n_on_device) {
        marl_status sp = sync_population(c);
        if (sp) return sp;
    }
    const uint32_t n = c->n;
    if (e->n_deaths > n || e->n_after_deaths != n - e->n_deaths)
        return fail(MARL_ERR_INVALID_INPUT, "n_after_deaths %u != %u cells - %u deaths", e->n_after_deaths, n,
                    e->n_deaths);
    if ((uint64_t)e->n_after_deaths + e->n_births > c->t.cap)
        return fail(MARL_ERR_CAPACITY, "%u + %u births exceed capacity %u", e->n_after_deaths, e->n_births, c->t.cap);
    for (uint32_t i = 0; i < e->n_halve; ++i)
        if (e->halve[i] >= n) return fail(MARL_ERR_INVALID_INPUT, "halve index %u >= %u", e->halve[i], n);
    for (uint32_t i = 0; i < e->n_deaths; ++i) {
        if (e->deaths[i] >= n) return fail(MARL_ERR_INVALID_INPUT, "death index %u >= %u", e->deaths[i], n);
        if (i && e->deaths[i] <= e->deaths[i - 1]) return fail(MARL_ERR_INVALID_INPUT, "deaths not ascending/unique");
    }
    for (uint32_t i = 0; i < e->n_moves; ++i)
        if (e->move_dst[i] >= e->n_after_deaths || e->move_src[i] < e->n_after_deaths || e->move_src[i] >= n)
            return fail(MARL_ERR_INVALID_INPUT, "move %u: %u <- %u outside the swap_remove ranges", i, e->move_dst[i],
                        e->move_src[i]);
    for (uint32_t i = 0; i < e->n_births; ++i) {
        const uint16_t* p = e->births[i].pos;
        if (p[0] >= c->g.X || p[1] >= c->g.Y || p[2] >= c->g.Z)
            return fail(MARL_ERR_INVALID_INPUT, "birth %u outside the grid", i);
    }
    // One staging buffer, one H2D copy: [halve][deaths][dst][src][pad16][births].
    const size_t b_halve = (size_t)e->n_halve * 4, b_deaths = (size_t)e->n_deaths * 4, b_mv = (size_t)e->n_moves * 4;
    size_t off_births = b_halve + b_deaths + 2 * b_mv;
    off_births = (off_births + 15) & ~(size_t)15;
    const size_t total = off_births + (size_t)e->n_births * sizeof(marl_cell);
    if (total == 0) return MARL_OK;
    marl_status st = ensure_edit_capacity(c, total);
    if (st) return st;
    uint8_t* h = (uint8_t*)c->h_edit;
    uint8_t* d = (uint8_t*)c->d_edit;
    size_t o = 0;
    std::memcpy(h + o, e->halve, b_halve), o += b_halve;
    std::memcpy(h + o, e->deaths, b_deaths), o += b_deaths;
    std::memcpy(h + o, e->move_dst, b_mv), o += b_mv;
    std::memcpy(h + o, e->move_src, b_mv), o += b_mv;
    if (e->n_births) std::memcpy(h + off_births, e->births, (size_t)e->n_births * sizeof(marl_cell));
    const int span = span_begin(c);
    CK(cudaMemcpyAsync(d, h, total, cudaMemcpyHostToDevice, c->stream));
    c->h2d_bytes += total;
    const uint32_t* dh = (const uint32_t*)d;
    const uint32_t* dd = (const uint32_t*)(d + b_halve);
    const uint32_t* dmd = (const uint32_t*)(d + b_halve + b_deaths);
    const uint32_t* dms = (const uint32_t*)(d + b_halve + b_deaths + b_mv);
    CK(launch_halve_clear(c->t, dh, e->n_halve, dd, e->n_deaths, c->g, c->cmap, c->mask, c->stream));
    CK(launch_moves(c->t, dmd, dms, e->n_moves, c->g, c->cmap, c->stream));
    CK(launch_cells_from_records((const marl_cell*)(d + off_births), e->n_births, e->n_after_deaths, c->t, c->g,
                                 c->cmap, c->mask, &c->d_hdr->err, c->stream));
    span_end(c, span);
    c->launches += (e->n_halve > 0 || e->n_deaths > 0) + (e->n_moves > 0) + (e->n_births > 0);
    c->n = e->n_after_deaths + e->n_births;
    if (e->n_deaths || e->n_births || e->n_moves) c->schedule_dirty = true;
    return MARL_OK;
}

marl_status marl_mass_f64(marl_ctx* c, double out[MARL_S_EXT]) {
    if (!c || !out) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    CK(launch_mass(c->field[c->cur], c->g, c->d_mass_partial, c->d_mass_out, c->stream));
    CK(cudaMemcpyAsync(c->h_mass, c->d_mass_out, 12 * 8, cudaMemcpyDeviceToHost, c->stream));
    marl_status st = sync_and_check(c);
    if (st) return st;
    std::memcpy(out, c->h_mass, 12 * 8);
    return MARL_OK;
}

marl_status marl_diffuse_tick_with_cells(marl_ctx* c, float* field, const uint8_t* occupancy) {
    if (c) c->c4_valid = false;
    if (!c || !field || !occupancy) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    if (c->sim.diffusion_substeps == 0) return MARL_OK;  // field_diffusion.rs:176-178
    const size_t V = c->g.V();
    if (!c->d_seam_mask) {
        CK(cudaMalloc((void**)&c->d_seam_mask, (size_t)c->g.Z * c->g.Y * mask_pitch(c->g.X)));
        if (!c->d_occ_stage) CK(cudaMalloc((void**)&c->d_occ_stage, V));
        if (!plan_diffusion(&c->seam_plan, c->field[0], c->field[1], c->d_seam_mask, c->g, c->plan.tile, c->plan.zc))
            return fail(MARL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    }
    CK(cudaMemcpyAsync(c->field[c->cur], field, V * 48, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_occ_stage, occupancy, V, cudaMemcpyHostToDevice, c->stream));
    CK(launch_repack_mask(c->d_occ_stage, c->d_seam_mask, c->g, c->stream));
    for (uint32_t i = 0; i < c->sim.diffusion_substeps; ++i) {
        CK(launch_diffuse(c->seam_plan, c->cur, c->g, c->fk, 0, nullptr, &c->d_hdr->err, c->stream));
        c->cur ^= 1;
    }
    CK(cudaMemcpyAsync(field, c->field[c->cur], V * 48, cudaMemcpyDeviceToHost, c->stream));
    return sync_and_check(c);
}

marl_status marl_diffuse_device(float* field_dev, float* scratch_dev, const uint8_t* occ_dev, int32_t gx, int32_t gy,
                                int32_t gz, const marl_sim_params* sim, uint32_t substeps, void* stream) {
    if (!field_dev || !scratch_dev || !occ_dev || !sim) return fail(MARL_ERR_INVALID_INPUT, "null argument");
    marl_status st = validate_dims(gx, gy, gz);
    if (st) return st;
    if (substeps == 0) return MARL_OK;
    if (sim->diffusion_substeps == 0) return fail(MARL_ERR_INVALID_INPUT, "sim.diffusion_substeps == 0");
    if (((uintptr_t)field_dev | (uintptr_t)scratch_dev) & 15)
        return fail(MARL_ERR_INVALID_INPUT, "field and scratch must be 16-byte aligned");
    int dev, sms;
    if ((st = check_device(&dev, &sms))) return st;
    const Grid g{gx, gy, gz};
    cudaStream_t s = (cudaStream_t)stream;
    FieldConsts fk;
    CellConsts ck;
    derive_consts(*sim, &fk, &ck);
    uint8_t* mask = nullptr;
    uint32_t* err = nullptr;
    CK(cudaMallocAsync((void**)&mask, (size_t)gz * gy * mask_pitch(gx), s));
    CK(cudaMallocAsync((void**)&err, 4, s));
    CK(cudaMemsetAsync(err, 0, 4, s));
    CK(launch_repack_mask(occ_dev, mask, g, s));
    DiffusionPlan plan;
    if (!plan_diffusion(&plan, field_dev, scratch_dev, mask, g, 0, 16)) {
        cudaFreeAsync(mask, s);
        cudaFreeAsync(err, s);
        return fail(MARL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    }
    int cur = 0;  // 0: field_dev holds the live state, 1: scratch_dev does
    for (uint32_t i = 0; i < substeps; ++i) {
        CK(launch_diffuse(plan, cur, g, fk, 0, nullptr, err, s));
        cur ^= 1;
    }
    if (cur != 0) CK(cudaMemcpyAsync(field_dev, scratch_dev, g.V() * 48, cudaMemcpyDeviceToDevice, s));
    uint32_t h_err = 0;
    CK(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(mask, s));
    CK(cudaFreeAsync(err, s));
    CK(cudaStreamSynchronize(s));
    if (h_err) return fail(MARL_ERR_TIMEOUT, "device wait gave up (error bits 0x%x)", h_err);
    return MARL_OK;
}

}  // extern "C"
