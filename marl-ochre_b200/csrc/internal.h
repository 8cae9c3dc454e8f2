// Internal host-side interface between the C-ABI layer (ctx.cu, engine.cpp)
// and the kernel translation units (field.cu, cells.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "common.cuh"

namespace marl {

// Tensor maps and tile choice for the diffusion kernel over one pair of
// ping-pong buffers and one occupancy mask.
struct DiffusionPlan {
    CUtensorMap tm_load[2];   // halo'd plane loads from buffer 0 / buffer 1
    CUtensorMap tm_store[2];  // tile stores into buffer 0 / buffer 1
    CUtensorMap tm_mask;
    float* buf[2] = {nullptr, nullptr};  // the two buffers (direct-store tiles write into them)
    int tile = 0;  // index into the tile-shape table
    int zc = 16;   // z-chunk per CTA
};

int diffusion_tile_count();
void diffusion_tile_shape(int tile, int* tx, int* ty);
bool encode_field_map(CUtensorMap* m, const float* base, const Grid& g, int box_voxels, int box_rows);
bool encode_mask_map(CUtensorMap* m, const uint8_t* base, const Grid& g, int tx, int ty);
bool plan_diffusion(DiffusionPlan* plan, const float* a, const float* b, const uint8_t* mask, const Grid& g,
                    int tile, int zc);

cudaError_t launch_sources(float* f, const Grid& g, const FieldConsts& k, cudaStream_t s);
// One substep from buffer `which_src` into the other buffer of the plan.
// c4_out (nullable) receives species 4 of the result, [z][y][x].
cudaError_t launch_diffuse(const DiffusionPlan& plan, int which_src, const Grid& g, const FieldConsts& k,
                           int apply_sources, float* c4_out, uint32_t* err, cudaStream_t s);
// c4 (nullable): compact species 4 of `f`; when null species 4 is read from f.
cudaError_t launch_light(const float* c4, const float* f, const uint8_t* mask, float* light, const Grid& g,
                         const FieldConsts& k, cudaStream_t s);
cudaError_t launch_mass(const float* f, const Grid& g, double* partial, double* out, cudaStream_t s);
size_t mass_partial_doubles();
cudaError_t launch_repack_mask(const uint8_t* occ, uint8_t* mask, const Grid& g, cudaStream_t s);
cudaError_t launch_unpack_mask(const uint8_t* mask, uint8_t* occ, const Grid& g, cudaStream_t s);

// ---- cells ----
struct ChangeHeader {  // device-written, read back with the change list
    uint32_t count;     // Division + Death events this tick
    uint32_t err;       // kErr* bits accumulated by kernels
    uint32_t n_cells;
    uint32_t pad[13];
};
static_assert(sizeof(ChangeHeader) == 64, "change header is 64 bytes");

// Surrogate hooks of the cell loop (modes of k_cell_tick).
constexpr int kModePlain = 0;
constexpr int kModeCapture = 1;   // plain, and each cell writes its raw training row
constexpr int kModeGated = 2;     // prediction checked against the plain reaction phase
constexpr int kModeTrusted = 3;   // prediction taken unchecked where speculation holds
constexpr uint8_t kSurrNotSpeculated = 0;
constexpr uint8_t kSurrAccepted = 1;
constexpr uint8_t kSurrRejected = 2;

// Cell j of a run is row row0 + j of the surrogate arrays; species k of a
// row is at k * ld + row.
struct SurrView {
    float* raw = nullptr;        // capture: row j (MARL_SURR_RAW_STRIDE floats) for cell j
    uint32_t raw_rows = 0;       // capture: cells j < raw_rows write a row
    const float* xt = nullptr;   // [16][ld] post-transport state from the pre-pass
    const float* pred = nullptr; // [16][ld] predicted reaction deltas
    float tol = 0.0f;
    uint8_t* status = nullptr;   // [ld] kSurr*
    float* err = nullptr;        // [ld] normwise error of the prediction (gated mode)
    uint32_t row0 = 0;
    uint32_t ld = 0;
};

// One run of a batch, as the batched kernels see it (device memory).
struct RunDesc {
    Grid g;
    uint32_t n;          // cells
    uint32_t epoch;      // this tick's completion epoch
    uint32_t cell_base;  // global ticket of this run's cell 0
    uint32_t pad;
    float* field[2];
    uint8_t* mask;
    int32_t* cmap;
    float* light;
    float* c4;
    CellTable t;
    ChangeHeader* hdr;
    marl_change* changes;
    uint32_t change_cap;
    uint32_t pad2;
    SurrView sv;  // surrogate arrays of the batch, rows from cell_base
};
// Tensor maps per run in the batch's map array: load from buffer 0 / 1,
// store into buffer 0 / 1, occupancy mask.
constexpr int kMapsPerRun = 5;

// Batch-wide scalars in device memory.  The cell total of the batch is not
// stored: it is cell_base + n of the last run.
struct BatchScalars {
    uint32_t ticket;   // cell-tick ticket counter (zeroed before each tick)
    uint32_t err;      // kErr* bits of every batched kernel
    uint32_t changes;  // Division/Death events over all runs (set by the pack kernel)
    uint32_t pad[13];
};
static_assert(sizeof(BatchScalars) == 64, "batch scalars are 64 bytes");

// Batched launchers (one launch covers every run).
cudaError_t launch_diffuse_batch(int tile, const RunDesc* runs, const CUtensorMap* maps, const int4* items,
                                 int n_items, int zc, const FieldConsts& k, int parity, int apply_sources, int emit_c4,
                                 uint32_t* err, cudaStream_t s);
cudaError_t launch_light_batch(const RunDesc* runs, const int4* items, int n_items, const FieldConsts& k, int parity,
                               int use_c4, cudaStream_t s);
cudaError_t launch_cell_schedule_batch(const RunDesc* runs, int n_runs, int num_sms, cudaStream_t s);
// mode: kModePlain, kModeGated or kModeTrusted (the runs' sv hold the arrays).
cudaError_t launch_cell_tick_batch(const RunDesc* runs, int n_runs, BatchScalars* bs, const CellConsts& k, int parity,
                                   int num_sms, int mode, cudaStream_t s);
// Surrogate pre-pass over the first `total` cells of the batch (global rows):
// xt [16][ld] and standardised BF16 features X [rows][128].
cudaError_t launch_surrogate_prepass_batch(const RunDesc* runs, int n_runs, uint32_t total, const CellConsts& k,
                                           int parity, const float* norm, float* xt, uint32_t ld, void* X,
                                           int num_sms, cudaStream_t s);
cudaError_t launch_compact_batch(const RunDesc* runs, int n_runs, cudaStream_t s);
// Concatenates the runs' change lists in run order into `packed` (run r's
// entries start at the sum of the counts of runs < r) and stores the total
// in bs->changes.
cudaError_t launch_pack_changes(const RunDesc* runs, int n_runs, BatchScalars* bs, marl_change* packed,
                                cudaStream_t s);
// Edit items: (run, index) pairs, (run, dst, src) moves, (run, slot) births.
cudaError_t launch_halve_batch(const RunDesc* runs, const uint2* items, uint32_t count, cudaStream_t s);
cudaError_t launch_clear_dead_batch(const RunDesc* runs, const uint2* items, uint32_t count, cudaStream_t s);
cudaError_t launch_moves_batch(const RunDesc* runs, const uint4* items, uint32_t count, cudaStream_t s);
cudaError_t launch_births_batch(const RunDesc* runs, const marl_cell* recs, const uint2* slots, uint32_t count,
                                uint32_t* err, cudaStream_t s);

struct CellLaunch {
    int mode = kModePlain;
    SurrView sv;
    CellTable t;
    uint32_t n;                     // cells (an upper bound when n_dev is set)
    const uint32_t* n_dev = nullptr;  // device-resident cell count (device fate), read by the kernels
    uint32_t lanes = 32;              // cells per warp ticket (1..32)
    Grid g;
    const uint8_t* mask;
    const int32_t* cmap;
    float* field;
    const float* light;
    CellConsts k;
    uint32_t epoch;
    uint32_t* ticket;
    uint32_t* err;
    float* act = nullptr;  // receptor activations [8][cap] of the cells updated (nullable)
};

cudaError_t launch_cell_schedule(const CellLaunch& a, cudaStream_t s);
// Test hook: cell `cell` waits through face `face` for slot `slot` (a slot no
// cell of the tick publishes); kErrBadIndex if that face is not an empty
// in-grid voxel of the cell (its dependency would not be read).
cudaError_t launch_hold_dependency(const CellTable& t, uint32_t cell, int face, uint32_t slot, uint32_t* err,
                                   cudaStream_t s);
cudaError_t launch_cell_tick(const CellLaunch& a, int num_sms, cudaStream_t s);
// Whether the plain cell kernel's grid gives each of n cells its own lane at
// once (warp tickets); then the kernel can compute the schedule itself.
bool cell_tick_covers(uint32_t n, uint32_t lanes, int num_sms);
// Surrogate pre-pass: every cell's gather and transport on the current field
// (as the cell loop would compute them if no earlier cell had written its
// neighbourhood): xt [16][cap] and the standardised BF16 features X [cap][128].
cudaError_t launch_surrogate_prepass(const CellLaunch& a, const float* norm, float* xt, void* X, int num_sms,
                                     cudaStream_t s);
// Adds the tick's per-cell statuses to counters[0..3] = cells, speculated,
// accepted, rejected and the largest accepted error's bits to *max_bits.
cudaError_t launch_surrogate_count(const uint8_t* status, const float* err, uint32_t n,
                                   unsigned long long* counters, uint32_t* max_bits, cudaStream_t s);
// Ordered compaction of Division/Death events into `changes` (after a
// 64-byte ChangeHeader); block_counts needs compaction_blocks(n) words.
uint32_t compaction_blocks(uint32_t n);
cudaError_t launch_compact_events(const CellTable& t, uint32_t n, uint32_t* block_counts, ChangeHeader* hdr,
                                  marl_change* changes, uint32_t cap, cudaStream_t s);

cudaError_t launch_cells_from_records(const marl_cell* rec, uint32_t count, uint32_t base, CellTable t, const Grid& g,
                                      int32_t* cmap, uint8_t* mask, uint32_t* err, cudaStream_t s);
cudaError_t launch_cells_to_records(const CellTable& t, uint32_t n, marl_cell* rec, cudaStream_t s);
// Halving of the parents and clearing of the dead cells of one edit list, in
// one launch.
cudaError_t launch_halve_clear(const CellTable& t, const uint32_t* halve_idx, uint32_t n_halve,
                               const uint32_t* dead_idx, uint32_t n_dead, const Grid& g, int32_t* cmap, uint8_t* mask,
                               cudaStream_t s);
cudaError_t launch_moves(CellTable t, const uint32_t* dst, const uint32_t* src, uint32_t count, const Grid& g,
                         int32_t* cmap, cudaStream_t s);
cudaError_t launch_rebuild_maps(const CellTable& t, uint32_t n, const Grid& g, int32_t* cmap, uint8_t* mask,
                                cudaStream_t s);

// ---- horizontal gene transfer (hgt.cu) ----
// items: (donor, recipient, pair index, 0), one conflict-free wave.
cudaError_t launch_hgt(const CellTable& t, const uint4* items, uint32_t count, uint64_t seed, uint64_t tick,
                       cudaStream_t s);

// ---- device fate (fate.cu) ----
// Scalars of a context's device fate processing.  While the context runs
// device fate the population lives here (n) and the host copy is stale.
struct FateScalars {
    unsigned long long seed;         // run seed of the per-division streams
    unsigned long long tick;         // tick of the next fate step
    unsigned long long key_tick;     // tick the last step's streams were keyed by
    unsigned long long total_div;    // divisions that found a voxel, all steps
    unsigned long long total_death;
    uint32_t n;       // population
    uint32_t n_old;   // population at the start of the last step
    uint32_t n1;      // after its deaths
    uint32_t ndiv;    // Division events of the last step
    uint32_t ndeath;  // Death events of the last step
    uint32_t placed;  // divisions of the last step that found a voxel
    uint32_t births;  // daughters appended by the last step
    uint32_t moves;   // swap_remove moves of the last step
    uint32_t levels;  // swap_remove levels of the last step
    uint32_t pad[5];
};

// Scratch of device fate over a table of `cap` slots and a grid of V voxels.
struct FateBuffers {
    FateScalars* fs = nullptr;
    uint32_t* blk = nullptr;         // [fate_blocks(cap)] packed Division | Death << 16 counts per chunk
    uint32_t* div_list = nullptr;    // [cap] dividing cells, ascending
    uint32_t* death_list = nullptr;  // [cap] dying cells, ascending
    uint2* div_info = nullptr;       // [cap] (packed target voxel, stream draws | placed << 31)
    uint32_t* div_slot = nullptr;    // [cap] birth slot of division k, or kFateNoSlot / kFateDropped
    uint32_t* cnt = nullptr;         // [cap + 1] deaths in [n1, n1 + o) for tail offset o
    uint32_t* lev_b = nullptr;       // [cap + 2] swap_remove level boundaries
    uint32_t* lev_d = nullptr;       // [cap + 2] deaths below the previous boundary
    uint32_t* move_dst = nullptr;    // [cap]
    uint32_t* move_src = nullptr;    // [cap]
    uint32_t* newidx = nullptr;      // [cap] new slot of the tail survivor at offset o
    uint32_t* dead_pos = nullptr;    // [cap] packed positions of the dying cells
    uint32_t* claim = nullptr;       // [V] lowest division ordinal claiming the voxel, else 0xFFFFFFFF
    bool own_fs = true;              // fs allocated with the buffers (else part of a caller's array)
};
constexpr uint32_t kFateNoSlot = 0xFFFFFFFFu;
constexpr uint32_t kFateDropped = 0xFFFFFFFEu;
uint32_t fate_blocks(uint32_t cap);
// fs_external (nullable): the run's scalars inside a caller-owned array.
cudaError_t alloc_fate(FateBuffers& f, uint32_t cap, size_t voxels, FateScalars* fs_external = nullptr);
void free_fate(FateBuffers& f);
cudaError_t launch_set_population(FateScalars* fs, uint32_t n, cudaStream_t s);
cudaError_t launch_fate_init(FateScalars* fs, unsigned long long seed, unsigned long long tick,
                             unsigned long long total_div, unsigned long long total_death, cudaStream_t s);
// One run as the fate kernels see it (a device array, pointers fixed).
struct FateRun {
    FateBuffers f;
    CellTable t;
    Grid g;
    int32_t* cmap;
    uint8_t* mask;
};
// The fate step of every run in d_runs over the events of its first fs->n
// cells; max_cap: the largest table capacity among them.
cudaError_t launch_fate(const FateRun* d_runs, int n_runs, uint32_t max_cap, uint32_t* err, const marl_sim_params& sim,
                        int num_sms, cudaStream_t s);
// Batch: runs[r].n and .cell_base from the runs' fate scalars, runs[r].epoch += 1.
cudaError_t launch_batch_population(RunDesc* runs, int n_runs, const FateRun* fr, cudaStream_t s);

}  // namespace marl
