/*
 * marl_cuda.h — C ABI of libmarl_cuda.so, the sm_100a backend for MARL's
 * per-tick field-and-cell hot path.
 *
 * Plain C: fixed-width integers, plain pointers and sizes, an int32 status on
 * every call, no exceptions and no torch/CUDA types in any signature (a CUDA
 * stream travels as `void*`).  Host buffers are caller-allocated.
 *
 * Reference interface each group replaces (paths are inside the MARL-OCHRE
 * workspace):
 *   - marl_sim_params           crates/marl-config/src/lib.rs:41-106 (SimulationConfig)
 *   - marl_sim_params_default   crates/marl-config/src/lib.rs:108-168 (Default impl)
 *   - marl_status               crates/marl-gpu/src/context.rs:5-10 (GpuError)
 *   - marl_cell / marl_ruleset  crates/marl-cell/src/cell.rs:50-183 (CellState, Ruleset)
 *   - marl_ctx_create           crates/marl-gpu/src/field_diffusion.rs:32 (GpuFieldDiffuser::new)
 *   - marl_diffuse_tick_with_cells
 *                               crates/marl-gpu/src/field_diffusion.rs:158-268
 *                               (GpuFieldDiffuser::diffuse_tick_with_cells) and
 *                               crates/marl-field/src/field.rs:212-217
 *   - marl_apply_boundary_sources  crates/marl-field/src/field.rs:231-250
 *   - marl_diffuse              crates/marl-field/src/field.rs:107-217
 *   - marl_light_update         crates/marl-field/src/light.rs:29-59
 *   - marl_cell_phase           crates/marl-sim/src/lib.rs:206-217 (cell loop:
 *                               spatial.rs:56-110 gather/scatter + cell.rs:193-369 tick)
 *   - marl_tick                 crates/marl-sim/src/lib.rs:164-217 (steps 1-4 of a tick)
 *   - marl_apply_edits          crates/marl-sim/src/lib.rs:220-277 (fate results:
 *                               halving, swap_remove deaths, appended births)
 *   - marl_engine_*             crates/marl-sim/src/lib.rs:34-277 (run(): seeding
 *                               and the tick loop, without file output)
 *
 * Threading: one stream per context; a context is not thread-safe, distinct
 * contexts may be used from distinct host threads.
 */
#ifndef MARL_CUDA_H
#define MARL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Compile-time species/ruleset counts (crates/marl-config/src/lib.rs:22-29).
 * The grid size is a runtime parameter here (the reference fixes it at
 * compile time, lib.rs:17-19). */
#define MARL_S_EXT 12
#define MARL_M_INT 16
#define MARL_R_MAX 16
#define MARL_S_RECEPTORS 8
#define MARL_S_TRANSPORTERS 8
#define MARL_S_EFFECTORS 8
#define MARL_NO_COFACTOR 0xFF

/* Status codes.  GpuError::{NoAdapter, DeviceRequest, BufferMap, InvalidInput}
 * map to NO_DEVICE, CUDA, CUDA, INVALID_INPUT. */
typedef enum marl_status {
    MARL_OK = 0,
    MARL_ERR_INVALID_INPUT = 1,
    MARL_ERR_NO_DEVICE = 2,
    MARL_ERR_CUDA = 3,
    MARL_ERR_OUT_OF_MEMORY = 4,
    MARL_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
    MARL_ERR_CAPACITY = 6,  /* cell table or change list capacity exceeded */
    MARL_ERR_STATE = 7      /* call not valid in the context's current state */
} marl_status;

/* Cell events returned by the tick (crates/marl-cell/src/cell.rs:155-160). */
enum {
    MARL_EVENT_NONE = 0,
    MARL_EVENT_DIVISION = 1,
    MARL_EVENT_DEATH = 2,
    MARL_EVENT_QUIESCENCE = 3
};

/* Boundary source modes.  ADDITIVE is the reference (field.rs:231-250:
 * c = min(c + rate, c_max)).  DIRICHLET is a microbenchmark option that pins
 * the sourced planes to the boundary_prime_* values. */
enum {
    MARL_SOURCES_ADDITIVE = 0,
    MARL_SOURCES_DIRICHLET = 1
};

/* SimulationConfig, field for field and in declaration order
 * (crates/marl-config/src/lib.rs:41-106).  usize/u16/u8 fields are widened
 * to uint32_t.  `source_mode` is an extension (see above). */
typedef struct marl_sim_params {
    float dx;
    float dt;
    uint32_t diffusion_substeps;
    float d_voxel[MARL_S_EXT];
    float lambda_decay[MARL_S_EXT];
    float source_rate_oxidant;
    float source_rate_carbon;
    float source_rate_reductant;
    float epsilon;
    float c_max;
    float lambda_maintenance;
    float hard_death_floor;
    float reaction_maintenance;
    float base_division_prep;
    float prep_maintenance_multiplier;
    float rush_penalty_rate;
    float alpha_eps;
    float k_eps;
    float light_efficiency;
    float surface_intensity;
    float cell_absorption;
    float chemical_absorption;
    float light_floor;
    float mutation_stddev;
    float structural_mutation_rate_mult;
    float meta_mutation_rate;
    float meta_mutation_clamp_low;
    float meta_mutation_clamp_high;
    float hill_exponent_clamp_low;
    float hill_exponent_clamp_high;
    float active_reaction_threshold;
    uint32_t seed_margin;
    float phototroph_z_lo;
    float phototroph_z_hi;
    float chemolithotroph_z_lo;
    float chemolithotroph_z_hi;
    float anaerobe_z_lo;
    float anaerobe_z_hi;
    uint32_t division_neighbor_distance;
    uint32_t boundary_prime_layers;
    float boundary_prime_oxidant;
    float boundary_prime_carbon;
    float boundary_prime_reductant;
    uint32_t source_mode;
} marl_sim_params;

/* Ruleset pieces (crates/marl-cell/src/cell.rs:50-151), naturally aligned.
 * The canonical packed 536-byte on-disk form (crates/marl-format/src/lib.rs:70-89)
 * is produced by marl_ruleset_pack_canonical. */
typedef struct marl_receptor_params {
    float k_half, n_hill, gain;
} marl_receptor_params;

typedef struct marl_transport_params {
    float uptake_rate, secrete_rate;
    uint8_t ext_species, int_species, _pad[2];
} marl_transport_params;

typedef struct marl_reaction {
    uint8_t substrate, product, catalyst, cofactor;
    float k_m, v_max, k_cat;
} marl_reaction;

typedef struct marl_effector_params {
    float threshold, rate;
    uint8_t int_species, ext_species, _pad[2];
} marl_effector_params;

typedef struct marl_fate_params {
    float division_energy, death_energy, quiescence_energy, division_prep_ticks;
} marl_fate_params;

typedef struct marl_ruleset {
    marl_receptor_params receptors[MARL_S_RECEPTORS];
    marl_transport_params transport[MARL_S_TRANSPORTERS];
    marl_reaction reactions[MARL_R_MAX];
    marl_effector_params effectors[MARL_S_EFFECTORS];
    marl_fate_params fate;
    float hgt_propensity;
    float mutation_rate;
} marl_ruleset; /* 568 bytes */

/* CellState (crates/marl-cell/src/cell.rs:169-183). 656 bytes. */
typedef struct marl_cell {
    uint16_t pos[3];
    uint8_t quiescent;
    uint8_t starter_type;
    uint32_t age;
    uint16_t prep_remaining;
    uint16_t _pad0;
    uint64_t lineage_id;
    float internal[MARL_M_INT];
    marl_ruleset ruleset;
} marl_cell;

/* One entry of the compacted per-tick change list: a Division or Death event
 * of cell `cell` (its index in the cell vector at the start of the tick), in
 * ascending cell order.  For divisions `internal`/`quiescent` hold the
 * parent's post-tick state, which the host clones into the daughter
 * (crates/marl-sim/src/lib.rs:223-245). 72 bytes. */
typedef struct marl_change {
    uint32_t cell;
    uint8_t event;
    uint8_t quiescent;
    uint16_t _pad;
    float internal[MARL_M_INT];
} marl_change;

/* Result of the host fate step (crates/marl-sim/src/lib.rs:220-277), applied
 * to the device cell table in this order:
 *   1. halve[]      parents whose 16 internal species are multiplied by 0.5
 *                   (indices at the start of the tick)
 *   2. deaths[]     ascending, unique; their voxels become empty
 *   3. moves        swap_remove result: slot move_dst[k] (< n_after_deaths)
 *                   receives the cell from slot move_src[k] (>= n_after_deaths)
 *   4. births[]     appended at n_after_deaths, n_after_deaths+1, ...
 */
typedef struct marl_edit_list {
    uint32_t n_halve;
    const uint32_t* halve;
    uint32_t n_deaths;
    const uint32_t* deaths;
    uint32_t n_moves;
    const uint32_t* move_dst;
    const uint32_t* move_src;
    uint32_t n_after_deaths;
    uint32_t n_births;
    const marl_cell* births;
} marl_edit_list;

typedef struct marl_ctx marl_ctx;

/* ---- parameters, errors ------------------------------------------------ */
marl_status marl_sim_params_default(marl_sim_params* out);
/* Message of the last failed call on this host thread ("" if none). */
const char* marl_last_error(void);
/* Library/ABI version: 0xMMmmpp. */
uint32_t marl_abi_version(void);

/* ---- context (device-resident field, light, occupancy, cell table) ------ */
marl_status marl_ctx_create(int32_t gx, int32_t gy, int32_t gz, const marl_sim_params* sim,
                            uint32_t cell_capacity, marl_ctx** out);
void marl_ctx_destroy(marl_ctx* ctx);
/* All later work of the context is ordered on `cuda_stream` (a cudaStream_t;
 * NULL = the legacy default stream).  A context starts on a stream of its own. */
marl_status marl_ctx_set_stream(marl_ctx* ctx, void* cuda_stream);
marl_status marl_ctx_set_params(marl_ctx* ctx, const marl_sim_params* sim);
/* Waits for the context's stream and reports device-side errors. */
marl_status marl_ctx_synchronize(marl_ctx* ctx);
/* Diffusion tile shape (index into the kernel's tile table) and z-chunk.
 * Every choice gives bit-identical results; only speed differs. */
marl_status marl_ctx_set_tile(marl_ctx* ctx, int32_t tile, int32_t zc);
marl_status marl_ctx_get_tile(marl_ctx* ctx, int32_t* tile, int32_t* zc);
/* Cells per warp of the cell loop (1..32, default 32): a warp holds at most
 * that many cells at once and leaves its other lanes idle.  While the grid's
 * lanes cover every cell, a warp takes that many consecutive cells per
 * ticket; with more cells than lanes, a lane whose cell is finished takes the
 * next one (lane refill).  Fewer cells per warp serialise less work inside a
 * warp along the dependency chains, at the cost of more warps.  Results do
 * not depend on it. */
marl_status marl_ctx_set_cell_lanes(marl_ctx* ctx, uint32_t lanes);
/* Bound of the cell loop's dependency waits (no reference counterpart; the
 * reference loop is sequential and never waits).  A cell that has polled an
 * unfinished dependency `polls` times gives up: it is left un-updated with
 * event None, the phase finishes, and the call that reads the device status
 * returns MARL_ERR_TIMEOUT.  0 restores the default (4,194,304 polls of at
 * least 64 ns each). */
marl_status marl_ctx_set_wait_limit(marl_ctx* ctx, uint32_t polls);
/* Failure-injection hook for tests (no reference counterpart): during the
 * next cell phase only, cell `cell` (< population) also waits, through its
 * face `face` (0..5 in FACE_OFFSETS order, which must be an empty in-grid
 * voxel), for the completion flag of slot `slot`, with population <= slot <
 * capacity: a slot that no cell completes in that phase.  The wait runs out
 * after the limit set by marl_ctx_set_wait_limit and the phase reports
 * MARL_ERR_TIMEOUT; the phase after it recomputes the true dependencies.  A
 * face that is occupied or outside the grid gives MARL_ERR_INVALID_INPUT. */
marl_status marl_ctx_test_hold_dependency(marl_ctx* ctx, uint32_t cell, uint32_t face, uint32_t slot);
/* Receptor pass (phase 1 of CellState::tick, crates/marl-cell/src/cell.rs:
 * 206-220) as an optional output.  The reference computes each receptor's
 * Hill activation gain * c^n / (k^n + c^n + 1e-9) from the environment the
 * cell gathered and keeps it in an unused local (receptor-gated transport is
 * not wired upstream, cell.rs:203-205).  With the output on, every cell phase
 * writes each updated cell's 8 activations; they change nothing else.
 * marl_ctx_download_receptor_activations copies the last phase's [n][8]
 * activations (MARL_ERR_STATE when the output is off; powf as CUDA computes
 * it, within 1e-5 relative of the reference's). */
marl_status marl_ctx_set_receptor_output(marl_ctx* ctx, int32_t enable);
marl_status marl_ctx_download_receptor_activations(marl_ctx* ctx, float* out, uint32_t cap_cells, uint32_t* n_out);
/* Horizontal gene transfer (crates/marl-cell/src/hgt.rs:7-27,
 * transfer_reaction; defined upstream, not called by its tick loop) for the
 * pairs (donors[k], recipients[k]), k = 0..n_pairs-1, in that order: a
 * random active reaction (|v_max| > 1e-9) of the donor overwrites the
 * recipient's first inactive slot, or a random slot when all are active.
 * Pair k draws from its own counter-based stream keyed by (seed, tick, k)
 * (the device fate stream specification), so results do not depend on
 * scheduling; independent pairs run in parallel.  Indices are cell indices
 * (< population). */
marl_status marl_ctx_hgt(marl_ctx* ctx, const uint32_t* donors, const uint32_t* recipients, uint32_t n_pairs,
                         uint64_t seed, uint64_t tick);
/* Tile autotuner (no reference counterpart): times `reps` substeps of every
 * tile shape / z-chunk candidate on this context's grid with CUDA events and
 * keeps the fastest.  The live field is not modified. */
marl_status marl_ctx_autotune(marl_ctx* ctx, int32_t reps, float* best_us_per_substep);

/* Cumulative counters of a context (no reference counterpart; used for
 * measurement).  device_us sums the CUDA-event spans, on the context's
 * stream, of the device work of every marl_tick (kernels and the change-list
 * copy) and marl_apply_edits (edit copy and kernels).  Synchronizes first. */
typedef struct marl_counters {
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
    uint64_t kernel_launches;
    uint64_t ticks;
    double device_us;
} marl_counters;
marl_status marl_ctx_counters(marl_ctx* ctx, marl_counters* out);

marl_status marl_upload_field(marl_ctx* ctx, const float* field /* [z][y][x][12] */);
marl_status marl_download_field(marl_ctx* ctx, float* field);
marl_status marl_upload_light(marl_ctx* ctx, const float* light /* [z][y][x] */);
marl_status marl_download_light(marl_ctx* ctx, float* light);
/* Replaces the cell table; occupancy follows the cells' positions. Duplicate
 * or out-of-grid positions are rejected. */
marl_status marl_upload_cells(marl_ctx* ctx, const marl_cell* cells, uint32_t n);
marl_status marl_download_cells(marl_ctx* ctx, marl_cell* out, uint32_t cap, uint32_t* n_out);
marl_status marl_cell_count(marl_ctx* ctx, uint32_t* n_out);
marl_status marl_download_occupancy(marl_ctx* ctx, uint8_t* occ /* [z][y][x] 0/1 */);

/* ---- per-phase entry points --------------------------------------------- */
marl_status marl_apply_boundary_sources(marl_ctx* ctx);
/* `substeps` diffusion substeps with dt_sub = dt / sim.diffusion_substeps.
 * With fuse_sources != 0 the boundary sources are applied inside the first
 * substep (same result as marl_apply_boundary_sources followed by
 * marl_diffuse with fuse_sources = 0). */
marl_status marl_diffuse(marl_ctx* ctx, uint32_t substeps, int32_t fuse_sources);
marl_status marl_light_update(marl_ctx* ctx);
/* The sequential cell loop of one tick on the current field and light.
 * events_out (nullable) receives one MARL_EVENT_* per cell. */
marl_status marl_cell_phase(marl_ctx* ctx, uint8_t* events_out);
/* Steps 1-4 of a tick (sources, diffusion, light, cell loop) and the
 * compacted change list of Division/Death events copied to `changes`.
 * *n_changes gets the total count; MARL_ERR_CAPACITY if it exceeds cap (the
 * first cap entries are still written). */
marl_status marl_tick(marl_ctx* ctx, marl_change* changes, uint32_t cap, uint32_t* n_changes);
marl_status marl_apply_edits(marl_ctx* ctx, const marl_edit_list* edits);
/* Per-species sum of the field in FP64, fixed reduction order. */
marl_status marl_mass_f64(marl_ctx* ctx, double out[MARL_S_EXT]);

/* GpuFieldDiffuser::diffuse_tick_with_cells: uploads `field` and `occupancy`
 * (one byte per voxel, nonzero = occupied), runs sim.diffusion_substeps
 * substeps, and downloads the result into `field`.  substeps == 0 returns
 * MARL_OK with no work, as the reference does. */
marl_status marl_diffuse_tick_with_cells(marl_ctx* ctx, float* field, const uint8_t* occupancy);

/* Device-pointer form of the diffusion tick, for callers that own their
 * device memory.  field_dev holds the input and receives the output;
 * scratch_dev is a second buffer of the same size (the reference's
 * Field::scratch, crates/marl-field/src/field.rs:18-20); occupancy_dev is
 * one byte per voxel.  The work is ordered on `cuda_stream` (NULL = legacy
 * default stream); the call synchronizes that stream before returning so that
 * device-side errors are reported. */
marl_status marl_diffuse_device(float* field_dev, float* scratch_dev, const uint8_t* occupancy_dev,
                                int32_t gx, int32_t gy, int32_t gz, const marl_sim_params* sim,
                                uint32_t substeps, void* cuda_stream);

/* Allocation-free form of marl_diffuse_device (no counterpart in the
 * reference).  For callers that must not allocate device memory while they
 * run — their device memory belongs to another allocator or a fixed pool, or
 * an allocation (and the synchronisation it can bring) is not acceptable in
 * their loop.  It calls no cudaMalloc/cudaFree and no allocating library
 * routine.  The ping-pong field copy, the padded occupancy mask and the error
 * word live in one static device array that every GPU loading the library holds
 * until exit (about 13 MiB).  Limits: at most 262,144 voxels, and
 * Y * Z * (X rounded up to 16) <= 1,048,576 bytes of mask; larger grids get
 * MARL_ERR_INVALID_INPUT.  Every call looks up the array's device address
 * on the current device (cudaGetSymbolAddress, no allocation), so a device
 * reset by the application does not leave a stale address behind.  The first
 * call on a device also loads the library's device code, which reserves the
 * array; it should come before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race and must not be issued.
 * Otherwise identical to marl_diffuse_device (same arguments minus
 * scratch_dev, same results and status codes, MARL_ERR_NO_DEVICE without an
 * sm_100 device, synchronizes `cuda_stream`). */
marl_status marl_diffuse_device_noalloc(float* field_dev, const uint8_t* occupancy_dev, int32_t gx, int32_t gy,
                                        int32_t gz, const marl_sim_params* sim, uint32_t substeps,
                                        void* cuda_stream);

/* ---- device fate ---------------------------------------------------------
 * The fate step of a tick (crates/marl-sim/src/lib.rs:219-277: division
 * placement, halving, cloning with a lineage draw and Ruleset::mutate,
 * swap_remove deaths, appended births) performed on the device from the
 * events the cell loop left in the table, so that ticks need no host round
 * trip.  No counterpart call in the reference, whose fate step is host code.
 * Random draws: one counter-based stream per dividing cell, keyed by
 * (seed, tick, index of the parent at the start of the step) -- xoshiro256**
 * seeded from a splitmix64 mix of the key; normals by Marsaglia's polar
 * method with a series logarithm, so that host and device draw the same
 * bits.  The results therefore differ from those of the host fate step
 * (marl_engine default mode), which draws from one sequential stream.
 * While a context runs device fate its population lives on the device; calls
 * that need it on the host (download, count, statistics, marl_tick,
 * marl_apply_edits, ...) synchronise the stream and fetch it. */
typedef struct marl_fate_stats {
    uint64_t tick;            /* tick of the next fate step */
    uint64_t population;
    uint64_t total_divisions; /* divisions that found a voxel, all steps */
    uint64_t total_deaths;
    uint64_t tick_divisions;  /* last step */
    uint64_t tick_deaths;
    uint64_t tick_births;     /* daughters appended (divisions minus voxel collisions) */
    uint64_t tick_moves;      /* swap_remove moves */
} marl_fate_stats;

/* Seed of the streams, tick of the next step and the running totals. */
marl_status marl_ctx_fate_init(marl_ctx* ctx, uint64_t seed, uint64_t tick, uint64_t total_divisions,
                               uint64_t total_deaths);
/* Enqueues one fate step over the current events (asynchronous). */
marl_status marl_ctx_fate(marl_ctx* ctx);
/* Synchronises; counters of the device fate state. */
marl_status marl_ctx_fate_stats(marl_ctx* ctx, marl_fate_stats* out);
/* Replaces the per-cell events (one MARL_EVENT_* per current cell), e.g. to
 * drive marl_ctx_fate from an external cell loop. */
marl_status marl_ctx_set_events(marl_ctx* ctx, const uint8_t* events, uint32_t n);
/* `ticks` whole ticks (lib.rs:160-277) with device fate, enqueued on the
 * context's stream without synchronising; device errors surface at the next
 * synchronising call.  The surrogate must be off. */
marl_status marl_ctx_run_ticks(marl_ctx* ctx, uint32_t ticks);
/* Diagnostics of the stream specification (run on the current device):
 * `count` u64 outputs of the stream keyed by (seed, tick, parent) and `count`
 * normals(stddev) of a fresh stream with the same key; and the stream's
 * logarithm of x[i] in (0, 1). */
marl_status marl_fate_stream_probe(uint64_t seed, uint64_t tick, uint32_t parent, uint32_t count, float stddev,
                                   uint64_t* u64_out, float* normal_out);
marl_status marl_fate_stream_ln(const double* x, uint32_t n, double* out);
/* Self-test of the cell loop's division by an empty-face count of 3, 5 or 6
 * (a reciprocal and one exact-remainder correction instead of an IEEE
 * division): compares it bit for bit with the IEEE division for every finite
 * float and each of the three divisors, and stores the number of differences
 * (0 expected) in *mismatches.  Runs on the current device (about a second). */
marl_status marl_selftest_small_division(uint64_t* mismatches);

/* ---- statistics ----------------------------------------------------------
 * print_stats / print_z_profile (crates/marl-sim/src/stats.rs:9-103) reduced
 * on the device.  Counts and the centre-column samples are exact; the three
 * averages are FP64 (the reference sums in f32, sequentially). */
typedef struct marl_stats {
    uint64_t population;
    uint64_t top, middle, bottom;   /* cells with z < Z/3, < 2(Z/3), the rest */
    double avg_energy;              /* mean internal[0] */
    double avg_enzyme;              /* mean internal[5] (ticks.csv avg_enzyme_a) */
    double avg_enzyme_b;            /* mean internal[6] (ticks.csv avg_enzyme_b, data.rs:214-217) */
    double avg_active_reactions;    /* mean count of reactions with |v_max| > 1e-9 */
    float oxidant_top;              /* field at (X/2, Y/2, 0), species 1 */
    float oxidant_middle;           /* (X/2, Y/2, Z/2), species 1 */
    float reductant_bottom;         /* (X/2, Y/2, Z-1), species 2 */
    float organic_middle;           /* (X/2, Y/2, Z/2), species 4 */
} marl_stats;
/* cells_per_z (nullable) gets Z counts; centre_column (nullable) gets the
 * column (X/2, Y/2) as [5][Z]: light, then species 1 to 4 (print_z_profile's
 * light, oxidant, reductant, carbon, organic).  Z <= 1024. */
marl_status marl_ctx_stats(marl_ctx* ctx, marl_stats* out, uint32_t* cells_per_z, float* centre_column);

/* ---- binary snapshots ----------------------------------------------------
 * The reference's field and cell dumps (crates/marl-output/src/binary_dump.rs:
 * 109-120) and run_meta.json (crates/marl-format/src/lib.rs:130-218),
 * uncompressed.  marl_ctx_viewer_cells packs one 25-byte ViewerCellRecord
 * per cell on the device (marl-format lib.rs:351-364: pos 3 x f32,
 * lineage_id u64, starter_type u8, energy f32, little endian, in
 * cell-vector order) and copies n * 25 bytes to `out`; MARL_ERR_CAPACITY when
 * cap_bytes is too small (*n_out still gets the count). */
marl_status marl_ctx_viewer_cells(marl_ctx* ctx, uint8_t* out, uint64_t cap_bytes, uint32_t* n_out);
/* Host-side writer: <dir>/run_meta.json, <dir>/tick_<tick>.field.bin (field:
 * [z][y][x][12] f32, nullable) and <dir>/tick_<tick>.cells.bin
 * (viewer_cells: n_cells packed records, nullable).  Each file is written to
 * a temporary name and renamed, as the reference does. */
marl_status marl_write_dump(const char* dir, uint64_t tick, int32_t gx, int32_t gy, int32_t gz, const float* field,
                            const uint8_t* viewer_cells, uint32_t n_cells);

/* Ruleset sidecar dumps (crates/marl-output/src/binary_dump.rs:121-350,
 * formats crates/marl-format/src/lib.rs:51-98), uncompressed:
 *   MARL_RULESETS_LAYERS: <dir>/tick_<tick>.ruleset_layers.bin, one 448-byte
 *     record per z layer (z u16, 0 u16, cell count u32, then the averages of
 *     the 110 float fields of the rulesets of the layer's cells: receptors,
 *     transporter rates, reaction k_m/v_max/k_cat, effector threshold/rate,
 *     fate, hgt_propensity, mutation_rate), summed in f64 in cell-vector
 *     order and rounded to f32, as the reference does;
 *   MARL_RULESETS_FULL: <dir>/tick_<tick>.rulesets.bin, the "MRSF" version-1
 *     deduplicated dump: a 24-byte header, the distinct canonical 536-byte
 *     rulesets in order of first occurrence, then per cell (x, y, z) u16 and
 *     its dictionary id u32.
 * Each call also rewrites <dir>/run_meta.json with ruleset_output_mode and
 * the sidecar layout keys (the keys marl_write_dump writes plus the ruleset
 * ones), so call it after marl_write_dump for the same directory.
 * marl_ctx_write_ruleset_dumps reduces the layer averages on the device
 * (Z x 448 bytes cross to the host) and packs the canonical rulesets on the
 * device (deduplicated on the host); marl_write_ruleset_dumps does the same
 * from host cells.  The two give identical files. */
enum { MARL_RULESETS_LAYERS = 1, MARL_RULESETS_FULL = 2, MARL_RULESETS_BOTH = 3 };
marl_status marl_ctx_write_ruleset_dumps(marl_ctx* ctx, const char* dir, uint64_t tick, int32_t mode);
marl_status marl_write_ruleset_dumps(const char* dir, uint64_t tick, int32_t gx, int32_t gy, int32_t gz,
                                     const marl_cell* cells, uint32_t n, int32_t mode);

/* ---- formats ------------------------------------------------------------ */
/* Canonical 536-byte ruleset payload (crates/marl-format/src/lib.rs:70-89). */
marl_status marl_ruleset_pack_canonical(const marl_ruleset* rs, uint8_t out[536]);
marl_status marl_ruleset_unpack_canonical(const uint8_t in[536], marl_ruleset* rs);

/* ---- engine: the tick loop of marl_sim::run over a context -------------- */
typedef struct marl_engine marl_engine;

typedef struct marl_engine_stats {
    uint64_t tick;
    uint64_t population;
    uint64_t total_divisions;
    uint64_t total_deaths;
    uint64_t tick_divisions;
    uint64_t tick_deaths;
    uint64_t h2d_bytes_last_tick;
    uint64_t d2h_bytes_last_tick;
} marl_engine_stats;

/* init_field_boundaries + seed_cells x3 (crates/marl-sim/src/seeding.rs:9-58,
 * lib.rs:59-105) with a seeded host RNG (xoshiro256** seeded by splitmix64). */
marl_status marl_engine_create(int32_t gx, int32_t gy, int32_t gz, const marl_sim_params* sim,
                               uint64_t rng_seed, uint32_t seed_count, uint32_t cell_capacity,
                               marl_engine** out);
/* Engine over a caller-provided state (field + cells). */
marl_status marl_engine_create_from_state(int32_t gx, int32_t gy, int32_t gz,
                                          const marl_sim_params* sim, uint64_t rng_seed,
                                          const float* field, const marl_cell* cells, uint32_t n,
                                          uint32_t cell_capacity, marl_engine** out);
void marl_engine_destroy(marl_engine* e);
marl_status marl_engine_set_stream(marl_engine* e, void* cuda_stream);
/* `ticks` iterations of lib.rs:160-277: device tick, change list to host,
 * fate processing with the host RNG, edit list to device. */
marl_status marl_engine_step(marl_engine* e, uint32_t ticks);
marl_status marl_engine_stats_get(marl_engine* e, marl_engine_stats* out);
/* Full cell vector in the reference's Vec order. */
marl_status marl_engine_get_cells(marl_engine* e, marl_cell* out, uint32_t cap, uint32_t* n_out);
marl_status marl_engine_get_field(marl_engine* e, float* field);
marl_status marl_engine_get_light(marl_engine* e, float* light);
marl_ctx* marl_engine_ctx(marl_engine* e);
/* Switches the engine's fate step between the host (default: one sequential
 * seeded stream, the reference's draw order) and the device (per-division
 * streams keyed by the engine's rng_seed; see marl_ctx_run_ticks).  With
 * device fate marl_engine_step enqueues all its ticks and synchronises once. */
marl_status marl_engine_set_device_fate(marl_engine* e, int32_t enable);

/* ---- batch: many independent runs advanced together --------------------
 * No counterpart in the reference, which advances one run per process
 * (crates/marl-sim/src/lib.rs:34-277).  Each run of a batch behaves exactly
 * like a marl_engine created with the same grid, parameters, rng_seed and
 * seed_count: same field, cells and change lists, bit for bit.  The runs may
 * have different grid sizes.  Every device phase of a tick (diffusion
 * substeps, light, the cell loop, compaction) is one kernel launch covering
 * all runs, and the device part of a tick is replayed from a CUDA graph; fate
 * processing runs on the host, one run per worker thread.  All runs share
 * `sim`.  Not thread-safe; one stream. */
typedef struct marl_batch marl_batch;

typedef struct marl_run_spec {
    int32_t gx, gy, gz;
    uint32_t seed_count;     /* cells per starter metabolism */
    uint64_t rng_seed;
    uint32_t cell_capacity;  /* 0: X*Y*Z/4, at least 1024 */
    uint32_t _pad;
} marl_run_spec;

marl_status marl_batch_create(const marl_run_spec* runs, uint32_t n_runs, const marl_sim_params* sim,
                              marl_batch** out);
void marl_batch_destroy(marl_batch* b);
/* NULL = legacy default stream.  The tick graphs are rebuilt lazily. */
marl_status marl_batch_set_stream(marl_batch* b, void* cuda_stream);
/* Host threads for fate processing (0: hardware concurrency, capped at 64). */
marl_status marl_batch_set_host_threads(marl_batch* b, int32_t threads);
/* Diffusion tile choice shared by all runs (indices as marl_ctx_set_tile). */
marl_status marl_batch_set_tile(marl_batch* b, int32_t tile, int32_t zc);
marl_status marl_batch_get_tile(marl_batch* b, int32_t* tile, int32_t* zc);
/* Times `reps` batched substeps for every tile candidate and keeps the
 * fastest; the runs' fields are not modified. */
marl_status marl_batch_autotune(marl_batch* b, int32_t reps, float* best_us_per_substep);
/* use_graph = 0 launches the device tick kernel by kernel instead of
 * replaying the captured graph (same results). */
marl_status marl_batch_set_graph(marl_batch* b, int32_t use_graph);
marl_status marl_batch_step(marl_batch* b, uint32_t ticks);
marl_status marl_batch_run_count(marl_batch* b, uint32_t* n_runs);
marl_status marl_batch_stats_get(marl_batch* b, uint32_t run, marl_engine_stats* out);
marl_status marl_batch_get_cells(marl_batch* b, uint32_t run, marl_cell* out, uint32_t cap, uint32_t* n_out);
marl_status marl_batch_get_field(marl_batch* b, uint32_t run, float* field);
marl_status marl_batch_get_light(marl_batch* b, uint32_t run, float* light);
/* As marl_ctx_counters, over the whole batch (ticks counts batch ticks). */
marl_status marl_batch_counters(marl_batch* b, marl_counters* out);
/* Fate on the device for every run (per-division streams keyed by each run's
 * rng_seed, as marl_engine_set_device_fate), or back on the host.  With device
 * fate a batch tick is one CUDA graph with no host work, and marl_batch_step
 * synchronises once per call.  Needs the batch surrogate off. */
marl_status marl_batch_set_device_fate(marl_batch* b, int32_t enable);

/* ---- learned reaction surrogate ----------------------------------------
 * No counterpart in the reference.  A 93 -> 256 -> 256 -> 16 MLP (tanh-form
 * GELU, BF16 weights and activations, FP32 accumulation on the tcgen05 tensor
 * cores) that stands in for the reaction phase of CellState::tick
 * (crates/marl-cell/src/cell.rs:246-285).  Input features, per cell:
 *   [0,16)   internal species after transport, light in slot 15 (cell.rs:243)
 *   [16,28)  gathered neighbour environment (spatial.rs:56-77)
 *   [28]     light at the cell's voxel
 *   [29,93)  per reaction r: k_m, v_max, k_cat, cofactor flag (1 = has one)
 * Output: the 16 internal-species deltas of the reaction phase.  k_m, |v_max|
 * and k_cat enter as log(v + 1e-3); every feature and target is standardised
 * with statistics of the training set.
 *
 * Training pairs come from the plain cell kernel itself: a context in capture
 * mode appends one raw row per updated cell and tick (features, then the
 * plain kernel's deltas).  Training runs forward, backward and Adam on the
 * GPU.  In a tick, the gated mode predicts every cell's deltas from a
 * pre-pass over the tick's starting field; a cell whose post-transport state
 * equals the pre-pass state takes the prediction when it agrees with the
 * plain reaction phase within `tol` (normwise: max |x_mlp - x_plain| /
 * max |x_plain| over the 16 species); every other cell keeps the plain
 * result.  The trusted mode skips the plain reaction phase for such cells and
 * takes the prediction unchecked. */
#define MARL_SURR_FEATURES 93
#define MARL_SURR_RAW_STRIDE 112 /* floats per raw row: 93 features, 16 deltas, pad */

typedef struct marl_surrogate marl_surrogate;

typedef struct marl_surrogate_config {
    uint32_t max_pairs;   /* capacity of the pair store (rows) */
    uint32_t batch;       /* training rows per step (multiple of 128) */
    float lr;             /* Adam step size */
    float beta1, beta2, adam_eps;
    uint64_t seed;        /* weight init and batch sampling */
} marl_surrogate_config;

typedef struct marl_surrogate_eval {
    uint32_t rows;
    uint32_t accepted;    /* rows with normwise relative error <= tol */
    float max_err;
    float mean_err;
    float mse_normalised; /* loss on standardised targets */
} marl_surrogate_eval;

typedef struct marl_surrogate_counters {
    uint64_t cells;       /* cells updated in surrogate mode */
    uint64_t speculated;  /* post-transport state equal to the pre-pass state */
    uint64_t accepted;    /* took the network's prediction */
    uint64_t rejected;    /* speculated but over tolerance: plain result kept */
    float max_err;        /* largest normwise error among accepted cells (gated mode) */
} marl_surrogate_counters;

enum { MARL_SURR_OFF = 0, MARL_SURR_CAPTURE = 1, MARL_SURR_GATED = 2, MARL_SURR_TRUSTED = 3 };

marl_status marl_surrogate_config_default(marl_surrogate_config* out);
marl_status marl_surrogate_create(const marl_surrogate_config* cfg, marl_surrogate** out);
void marl_surrogate_destroy(marl_surrogate* s);
marl_status marl_surrogate_set_stream(marl_surrogate* s, void* cuda_stream);
/* Rows captured so far. */
marl_status marl_surrogate_pair_count(marl_surrogate* s, uint32_t* rows);
/* Raw rows [row0, row0 + n) to the host, MARL_SURR_RAW_STRIDE floats each. */
marl_status marl_surrogate_download_pairs(marl_surrogate* s, uint32_t row0, uint32_t n, float* out);
/* Appends raw rows from the host (same layout). */
marl_status marl_surrogate_upload_pairs(marl_surrogate* s, const float* rows, uint32_t n);
/* Standardisation statistics over rows [0, n_train) and the standardised
 * BF16 training matrix of all rows.  Call before training or inference. */
marl_status marl_surrogate_prepare(marl_surrogate* s, uint32_t n_train);
/* Adam step size for later training steps. */
marl_status marl_surrogate_set_lr(marl_surrogate* s, float lr);
/* `steps` Adam steps on random batches of rows [0, n_train); loss_out
 * (nullable) receives the mean loss of each step. */
marl_status marl_surrogate_train(marl_surrogate* s, uint32_t steps, float* loss_out);
/* Prediction error on rows [row0, row0 + n) against the stored plain deltas. */
marl_status marl_surrogate_evaluate(marl_surrogate* s, uint32_t row0, uint32_t n, float tol,
                                    marl_surrogate_eval* out, float* row_err_out /* nullable, n */);
/* Master weights, FP32, flat: W1[256][128] (inputs 93..127 are zero), b1[256],
 * W2[256][256], b2[256], W3[16][256], b3[16]; then the standardisation:
 * in_mean[93], in_std[93], out_mean[16], out_std[16]. */
#define MARL_SURR_PARAMS (256 * 128 + 256 + 256 * 256 + 256 + 16 * 256 + 16)
#define MARL_SURR_NORM (93 + 93 + 16 + 16)
marl_status marl_surrogate_get_weights(marl_surrogate* s, float* params, float* norm);
marl_status marl_surrogate_set_weights(marl_surrogate* s, const float* params, const float* norm);
/* One forward + backward pass without an update, for gradient checks: x is
 * standardised input as BF16 bits [batch][128], t standardised targets
 * [batch][16]; grads_out gets MARL_SURR_PARAMS floats (same layout as the
 * weights) of d(loss)/d(param), loss = mean over batch and outputs of
 * (y - t)^2; y_out (nullable) gets the network output [batch][16]. */
marl_status marl_surrogate_gradients(marl_surrogate* s, const uint16_t* x, const float* t, uint32_t batch,
                                     float* grads_out, float* loss_out, float* y_out);
/* Inference path: fused = 1 (default) runs the whole forward pass in one
 * persistent kernel with the weights in shared memory; fused = 0 runs one
 * GEMM launch per layer with the hidden activations in device memory.  Both
 * compute the same function; results may differ in the last bits of the
 * FP32 accumulation order. */
marl_status marl_surrogate_set_inference(marl_surrogate* s, int32_t fused);
/* Inference on device memory: x_dev standardised BF16 [n][128]; y_dev gets
 * the de-standardised deltas as [16][ldy] (species-major).  Asynchronous on
 * the surrogate's stream. */
marl_status marl_surrogate_infer_device(marl_surrogate* s, const uint16_t* x_dev, uint32_t n, float* y_dev,
                                        uint32_t ldy);
/* Surrogate mode of a context's cell loop (MARL_SURR_*); tol is used by the
 * gated mode.  The surrogate must outlive its use by the context. */
marl_status marl_ctx_set_surrogate(marl_ctx* ctx, marl_surrogate* s, int32_t mode, float tol);
marl_status marl_ctx_surrogate_counters(marl_ctx* ctx, marl_surrogate_counters* out);
/* The same for every run of a batch (modes OFF, GATED, TRUSTED): one
 * pre-pass over all runs' cells and one inference over all of them per tick.
 * While a surrogate is attached the device tick is launched directly rather
 * than replayed from the captured graph (the inference's row count changes
 * every tick). */
marl_status marl_batch_set_surrogate(marl_batch* b, marl_surrogate* s, int32_t mode, float tol);
marl_status marl_batch_surrogate_counters(marl_batch* b, marl_surrogate_counters* out);

#ifdef __cplusplus
}
#endif

#endif /* MARL_CUDA_H */
