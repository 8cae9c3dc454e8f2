// Definition of the opaque marl_ctx (device-resident state of one grid) and
// helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/marl_cuda.h"
#include "common.cuh"
#include "internal.h"

namespace marl {

constexpr uint32_t kPrefetchChanges = 256;  // change-list entries fetched with the header

}  // namespace marl

struct marl_ctx {
    int device = 0;
    int num_sms = 0;
    marl::Grid g{0, 0, 0};
    marl_sim_params sim{};
    marl::FieldConsts fk{};
    marl::CellConsts ck{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    float* field[2] = {nullptr, nullptr};  // ping-pong; field[cur] is live
    int cur = 0;
    uint8_t* mask = nullptr;   // [z][y][pitch] occupancy of the cell table
    int32_t* cmap = nullptr;   // [z][y][x] cell index or -1
    float* light = nullptr;    // [z][y][x]
    float* c4 = nullptr;       // [z][y][x] species 4 after the last substep of a tick
    bool c4_valid = false;     // c4 equals species 4 of field[cur]
    marl::CellTable t{};
    uint32_t cell_lanes = 32;  // cells per warp ticket of the cell loop
    uint32_t wait_limit = marl::kFlagSpinLimit;  // polls of a dependency flag (marl_ctx_set_wait_limit)
    int32_t hold_cell = -1;    // marl_ctx_test_hold_dependency: cell, face and slot for the next phase
    int hold_face = 0;
    uint32_t hold_slot = 0;
    float* receptor_act = nullptr;  // [8][cap] receptor activations of the last cell phase (optional output)
    uint32_t n = 0;
    uint32_t epoch = 0;
    bool schedule_dirty = true;
    marl::DiffusionPlan plan{};

    marl::ChangeHeader* d_hdr = nullptr;  // device header (count, err, ticket)
    marl::ChangeHeader* h_hdr = nullptr;  // pinned: header followed by kPrefetchChanges entries
    marl_change* d_changes = nullptr;
    uint32_t* d_block_counts = nullptr;

    void* d_edit = nullptr;  // edit-list staging
    void* h_edit = nullptr;
    size_t edit_bytes = 0;
    marl_cell* d_records = nullptr;  // AoS cell records staging
    marl_cell* h_records = nullptr;
    uint32_t records_cap = 0;

    double* d_mass_partial = nullptr;
    double* d_mass_out = nullptr;
    double* h_mass = nullptr;
    uint8_t* d_events_stage = nullptr;

    // GpuFieldDiffuser seam: occupancy supplied by the caller
    uint8_t* d_occ_stage = nullptr;  // dense one byte per voxel
    uint8_t* d_seam_mask = nullptr;
    marl::DiffusionPlan seam_plan{};

    // Device fate (fate.cu).  While n_on_device is set the population lives in
    // fate.fs->n and `n` above is stale; sync_population brings it back.
    marl::FateBuffers fate{};
    marl::FateRun* d_fate_run = nullptr;  // device copy of this context's FateRun
    bool fate_ready = false;
    bool n_on_device = false;

    // Reaction surrogate (marl_ctx_set_surrogate)
    marl_surrogate* surr = nullptr;
    int surr_mode = 0;  // MARL_SURR_*
    float surr_tol = 0.0f;
    float* surr_xt = nullptr;      // [16][cap] pre-pass post-transport state
    float* surr_pred = nullptr;    // [16][cap] predicted deltas
    void* surr_x = nullptr;        // [cap][128] BF16 standardised features
    uint8_t* surr_status = nullptr;
    float* surr_err = nullptr;
    unsigned long long* surr_counters = nullptr;  // cells, speculated, accepted, rejected, max-error bits

    uint64_t h2d_bytes = 0;  // transfer counters (engine statistics)
    uint64_t d2h_bytes = 0;
    uint64_t launches = 0;   // kernels enqueued by this context
    uint64_t ticks = 0;

    // Device-time spans: event pairs recorded around the device work of
    // marl_tick / marl_apply_edits, resolved after the stream has synchronized.
    struct Span {
        cudaEvent_t a, b;
    };
    std::vector<Span> span_pool, spans_pending;
    double device_us = 0.0;

    marl_change* h_changes_prefix() {
        return reinterpret_cast<marl_change*>(reinterpret_cast<uint8_t*>(h_hdr) + sizeof(marl::ChangeHeader));
    }
};

namespace marl {
marl_status fail(marl_status st, const char* fmt, ...);
marl_status cuda_fail(cudaError_t e, const char* where);
// Current device and its SM count; MARL_ERR_NO_DEVICE unless it is sm_100.
marl_status check_device(int* dev, int* sms);
marl_status validate_dims(int32_t gx, int32_t gy, int32_t gz);
void derive_consts(const marl_sim_params& p, FieldConsts* fk, CellConsts* ck);
// Device cell table of `cap` slots (done[] and events[] zeroed).
cudaError_t alloc_table(CellTable& t, uint32_t cap);
void free_table(CellTable& t);
marl_status sync_and_check(marl_ctx* c);
marl_status collect_device_errors(marl_ctx* c, uint32_t err_bits);
// Device fate: allocates its buffers on first use and moves the population to
// the device; sync_population moves it back (synchronising the stream).
marl_status begin_device_population(marl_ctx* c);
marl_status sync_population(marl_ctx* c);
marl_status enqueue_fate(marl_ctx* c);
}  // namespace marl
