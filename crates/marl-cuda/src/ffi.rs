//! Raw `extern "C"` declarations of libmarl_cuda.so: one `#[repr(C)]` struct
//! per C struct and one function per entry point of include/marl_cuda.h, with
//! the same names, field order and types (checked against the header by the
//! repository's CPU test suite).  Status codes are `Status` (an `i32`, 0 =
//! success); `marl_last_error` gives the message of the last failure on the
//! calling thread.

#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_void};

pub type Status = i32;

pub const MARL_S_EXT: usize = 12;
pub const MARL_M_INT: usize = 16;
pub const MARL_R_MAX: usize = 16;
pub const MARL_S_RECEPTORS: usize = 8;
pub const MARL_S_TRANSPORTERS: usize = 8;
pub const MARL_S_EFFECTORS: usize = 8;
pub const MARL_NO_COFACTOR: u8 = 0xFF;

pub const MARL_OK: Status = 0;
pub const MARL_ERR_INVALID_INPUT: Status = 1;
pub const MARL_ERR_NO_DEVICE: Status = 2;
pub const MARL_ERR_CUDA: Status = 3;
pub const MARL_ERR_OUT_OF_MEMORY: Status = 4;
pub const MARL_ERR_TIMEOUT: Status = 5;
pub const MARL_ERR_CAPACITY: Status = 6;
pub const MARL_ERR_STATE: Status = 7;

pub const MARL_EVENT_NONE: u8 = 0;
pub const MARL_EVENT_DIVISION: u8 = 1;
pub const MARL_EVENT_DEATH: u8 = 2;
pub const MARL_EVENT_QUIESCENCE: u8 = 3;

pub const MARL_SOURCES_ADDITIVE: u32 = 0;
pub const MARL_SOURCES_DIRICHLET: u32 = 1;

pub const MARL_RULESETS_LAYERS: i32 = 1;
pub const MARL_RULESETS_FULL: i32 = 2;
pub const MARL_RULESETS_BOTH: i32 = 3;

pub const MARL_SURR_FEATURES: usize = 93;
pub const MARL_SURR_RAW_STRIDE: usize = 112;
pub const MARL_SURR_PARAMS: usize = 256 * 128 + 256 + 256 * 256 + 256 + 16 * 256 + 16;
pub const MARL_SURR_NORM: usize = 93 + 93 + 16 + 16;
pub const MARL_SURR_OFF: i32 = 0;
pub const MARL_SURR_CAPTURE: i32 = 1;
pub const MARL_SURR_GATED: i32 = 2;
pub const MARL_SURR_TRUSTED: i32 = 3;

/// marl_sim_params: SimulationConfig field for field
/// (crates/marl-config/src/lib.rs:41-106), usize/u16/u8 widened to u32.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SimParams {
    pub dx: f32,
    pub dt: f32,
    pub diffusion_substeps: u32,
    pub d_voxel: [f32; MARL_S_EXT],
    pub lambda_decay: [f32; MARL_S_EXT],
    pub source_rate_oxidant: f32,
    pub source_rate_carbon: f32,
    pub source_rate_reductant: f32,
    pub epsilon: f32,
    pub c_max: f32,
    pub lambda_maintenance: f32,
    pub hard_death_floor: f32,
    pub reaction_maintenance: f32,
    pub base_division_prep: f32,
    pub prep_maintenance_multiplier: f32,
    pub rush_penalty_rate: f32,
    pub alpha_eps: f32,
    pub k_eps: f32,
    pub light_efficiency: f32,
    pub surface_intensity: f32,
    pub cell_absorption: f32,
    pub chemical_absorption: f32,
    pub light_floor: f32,
    pub mutation_stddev: f32,
    pub structural_mutation_rate_mult: f32,
    pub meta_mutation_rate: f32,
    pub meta_mutation_clamp_low: f32,
    pub meta_mutation_clamp_high: f32,
    pub hill_exponent_clamp_low: f32,
    pub hill_exponent_clamp_high: f32,
    pub active_reaction_threshold: f32,
    pub seed_margin: u32,
    pub phototroph_z_lo: f32,
    pub phototroph_z_hi: f32,
    pub chemolithotroph_z_lo: f32,
    pub chemolithotroph_z_hi: f32,
    pub anaerobe_z_lo: f32,
    pub anaerobe_z_hi: f32,
    pub division_neighbor_distance: u32,
    pub boundary_prime_layers: u32,
    pub boundary_prime_oxidant: f32,
    pub boundary_prime_carbon: f32,
    pub boundary_prime_reductant: f32,
    pub source_mode: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct ReceptorParams {
    pub k_half: f32,
    pub n_hill: f32,
    pub gain: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TransportParams {
    pub uptake_rate: f32,
    pub secrete_rate: f32,
    pub ext_species: u8,
    pub int_species: u8,
    pub _pad: [u8; 2],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Reaction {
    pub substrate: u8,
    pub product: u8,
    pub catalyst: u8,
    pub cofactor: u8,
    pub k_m: f32,
    pub v_max: f32,
    pub k_cat: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct EffectorParams {
    pub threshold: f32,
    pub rate: f32,
    pub int_species: u8,
    pub ext_species: u8,
    pub _pad: [u8; 2],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct FateParams {
    pub division_energy: f32,
    pub death_energy: f32,
    pub quiescence_energy: f32,
    pub division_prep_ticks: f32,
}

/// marl_ruleset (568 bytes): Ruleset (crates/marl-cell/src/cell.rs:139-151).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Ruleset {
    pub receptors: [ReceptorParams; MARL_S_RECEPTORS],
    pub transport: [TransportParams; MARL_S_TRANSPORTERS],
    pub reactions: [Reaction; MARL_R_MAX],
    pub effectors: [EffectorParams; MARL_S_EFFECTORS],
    pub fate: FateParams,
    pub hgt_propensity: f32,
    pub mutation_rate: f32,
}

/// marl_cell (656 bytes): CellState (crates/marl-cell/src/cell.rs:169-183).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Cell {
    pub pos: [u16; 3],
    pub quiescent: u8,
    pub starter_type: u8,
    pub age: u32,
    pub prep_remaining: u16,
    pub _pad0: u16,
    pub lineage_id: u64,
    pub internal: [f32; MARL_M_INT],
    pub ruleset: Ruleset,
}

/// marl_change (72 bytes): one Division or Death event of the tick, in
/// ascending cell order, with the cell's post-tick internal state.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Change {
    pub cell: u32,
    pub event: u8,
    pub quiescent: u8,
    pub _pad: u16,
    pub internal: [f32; MARL_M_INT],
}

/// marl_edit_list: the host fate step's result (crates/marl-sim/src/lib.rs:220-277).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct EditList {
    pub n_halve: u32,
    pub halve: *const u32,
    pub n_deaths: u32,
    pub deaths: *const u32,
    pub n_moves: u32,
    pub move_dst: *const u32,
    pub move_src: *const u32,
    pub n_after_deaths: u32,
    pub n_births: u32,
    pub births: *const Cell,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Counters {
    pub h2d_bytes: u64,
    pub d2h_bytes: u64,
    pub kernel_launches: u64,
    pub ticks: u64,
    pub device_us: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct FateStats {
    pub tick: u64,
    pub population: u64,
    pub total_divisions: u64,
    pub total_deaths: u64,
    pub tick_divisions: u64,
    pub tick_deaths: u64,
    pub tick_births: u64,
    pub tick_moves: u64,
}

/// marl_stats: print_stats quantities (crates/marl-sim/src/stats.rs:9-82).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct Stats {
    pub population: u64,
    pub top: u64,
    pub middle: u64,
    pub bottom: u64,
    pub avg_energy: f64,
    pub avg_enzyme: f64,
    pub avg_enzyme_b: f64,
    pub avg_active_reactions: f64,
    pub oxidant_top: f32,
    pub oxidant_middle: f32,
    pub reductant_bottom: f32,
    pub organic_middle: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct EngineStats {
    pub tick: u64,
    pub population: u64,
    pub total_divisions: u64,
    pub total_deaths: u64,
    pub tick_divisions: u64,
    pub tick_deaths: u64,
    pub h2d_bytes_last_tick: u64,
    pub d2h_bytes_last_tick: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct RunSpec {
    pub gx: i32,
    pub gy: i32,
    pub gz: i32,
    pub seed_count: u32,
    pub rng_seed: u64,
    pub cell_capacity: u32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SurrogateConfig {
    pub max_pairs: u32,
    pub batch: u32,
    pub lr: f32,
    pub beta1: f32,
    pub beta2: f32,
    pub adam_eps: f32,
    pub seed: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SurrogateEval {
    pub rows: u32,
    pub accepted: u32,
    pub max_err: f32,
    pub mean_err: f32,
    pub mse_normalised: f32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct SurrogateCounters {
    pub cells: u64,
    pub speculated: u64,
    pub accepted: u64,
    pub rejected: u64,
    pub max_err: f32,
}

/// Opaque handles.
pub enum Ctx {}
pub enum Engine {}
pub enum Batch {}
pub enum Surrogate {}

// Sizes the C side states (a layout check at compile time).
const _: () = assert!(std::mem::size_of::<Ruleset>() == 568);
const _: () = assert!(std::mem::size_of::<Cell>() == 656);
const _: () = assert!(std::mem::size_of::<Change>() == 72);

unsafe extern "C" {
    // parameters, errors
    pub fn marl_sim_params_default(out: *mut SimParams) -> Status;
    pub fn marl_last_error() -> *const c_char;
    pub fn marl_abi_version() -> u32;

    // context
    pub fn marl_ctx_create(gx: i32, gy: i32, gz: i32, sim: *const SimParams, cell_capacity: u32,
                           out: *mut *mut Ctx) -> Status;
    pub fn marl_ctx_destroy(ctx: *mut Ctx);
    pub fn marl_ctx_set_stream(ctx: *mut Ctx, cuda_stream: *mut c_void) -> Status;
    pub fn marl_ctx_set_params(ctx: *mut Ctx, sim: *const SimParams) -> Status;
    pub fn marl_ctx_synchronize(ctx: *mut Ctx) -> Status;
    pub fn marl_ctx_set_tile(ctx: *mut Ctx, tile: i32, zc: i32) -> Status;
    pub fn marl_ctx_get_tile(ctx: *mut Ctx, tile: *mut i32, zc: *mut i32) -> Status;
    pub fn marl_ctx_set_cell_lanes(ctx: *mut Ctx, lanes: u32) -> Status;
    pub fn marl_ctx_set_wait_limit(ctx: *mut Ctx, polls: u32) -> Status;
    pub fn marl_ctx_test_hold_dependency(ctx: *mut Ctx, cell: u32, face: u32, slot: u32) -> Status;
    pub fn marl_ctx_set_receptor_output(ctx: *mut Ctx, enable: i32) -> Status;
    pub fn marl_ctx_download_receptor_activations(ctx: *mut Ctx, out: *mut f32, cap_cells: u32, n_out: *mut u32)
        -> Status;
    pub fn marl_ctx_hgt(ctx: *mut Ctx, donors: *const u32, recipients: *const u32, n_pairs: u32, seed: u64,
                        tick: u64) -> Status;
    pub fn marl_ctx_autotune(ctx: *mut Ctx, reps: i32, best_us_per_substep: *mut f32) -> Status;
    pub fn marl_ctx_counters(ctx: *mut Ctx, out: *mut Counters) -> Status;
    pub fn marl_upload_field(ctx: *mut Ctx, field: *const f32) -> Status;
    pub fn marl_download_field(ctx: *mut Ctx, field: *mut f32) -> Status;
    pub fn marl_upload_light(ctx: *mut Ctx, light: *const f32) -> Status;
    pub fn marl_download_light(ctx: *mut Ctx, light: *mut f32) -> Status;
    pub fn marl_upload_cells(ctx: *mut Ctx, cells: *const Cell, n: u32) -> Status;
    pub fn marl_download_cells(ctx: *mut Ctx, out: *mut Cell, cap: u32, n_out: *mut u32) -> Status;
    pub fn marl_cell_count(ctx: *mut Ctx, n_out: *mut u32) -> Status;
    pub fn marl_download_occupancy(ctx: *mut Ctx, occ: *mut u8) -> Status;

    // per-phase entry points and the tick
    pub fn marl_apply_boundary_sources(ctx: *mut Ctx) -> Status;
    pub fn marl_diffuse(ctx: *mut Ctx, substeps: u32, fuse_sources: i32) -> Status;
    pub fn marl_light_update(ctx: *mut Ctx) -> Status;
    pub fn marl_cell_phase(ctx: *mut Ctx, events_out: *mut u8) -> Status;
    pub fn marl_tick(ctx: *mut Ctx, changes: *mut Change, cap: u32, n_changes: *mut u32) -> Status;
    pub fn marl_apply_edits(ctx: *mut Ctx, edits: *const EditList) -> Status;
    pub fn marl_mass_f64(ctx: *mut Ctx, out: *mut f64) -> Status;

    // the GpuFieldDiffuser seam and its device-pointer forms
    pub fn marl_diffuse_tick_with_cells(ctx: *mut Ctx, field: *mut f32, occupancy: *const u8) -> Status;
    pub fn marl_diffuse_device(field_dev: *mut f32, scratch_dev: *mut f32, occupancy_dev: *const u8, gx: i32,
                               gy: i32, gz: i32, sim: *const SimParams, substeps: u32,
                               cuda_stream: *mut c_void) -> Status;
    pub fn marl_diffuse_device_noalloc(field_dev: *mut f32, occupancy_dev: *const u8, gx: i32, gy: i32, gz: i32,
                                       sim: *const SimParams, substeps: u32, cuda_stream: *mut c_void) -> Status;

    // device fate
    pub fn marl_ctx_fate_init(ctx: *mut Ctx, seed: u64, tick: u64, total_divisions: u64,
                              total_deaths: u64) -> Status;
    pub fn marl_ctx_fate(ctx: *mut Ctx) -> Status;
    pub fn marl_ctx_fate_stats(ctx: *mut Ctx, out: *mut FateStats) -> Status;
    pub fn marl_ctx_set_events(ctx: *mut Ctx, events: *const u8, n: u32) -> Status;
    pub fn marl_ctx_run_ticks(ctx: *mut Ctx, ticks: u32) -> Status;
    pub fn marl_fate_stream_probe(seed: u64, tick: u64, parent: u32, count: u32, stddev: f32, u64_out: *mut u64,
                                  normal_out: *mut f32) -> Status;
    pub fn marl_fate_stream_ln(x: *const f64, n: u32, out: *mut f64) -> Status;
    pub fn marl_selftest_small_division(mismatches: *mut u64) -> Status;

    // statistics and snapshots
    pub fn marl_ctx_stats(ctx: *mut Ctx, out: *mut Stats, cells_per_z: *mut u32, centre_column: *mut f32)
        -> Status;
    pub fn marl_ctx_viewer_cells(ctx: *mut Ctx, out: *mut u8, cap_bytes: u64, n_out: *mut u32) -> Status;
    pub fn marl_write_dump(dir: *const c_char, tick: u64, gx: i32, gy: i32, gz: i32, field: *const f32,
                           viewer_cells: *const u8, n_cells: u32) -> Status;
    pub fn marl_ctx_write_ruleset_dumps(ctx: *mut Ctx, dir: *const c_char, tick: u64, mode: i32) -> Status;
    pub fn marl_write_ruleset_dumps(dir: *const c_char, tick: u64, gx: i32, gy: i32, gz: i32, cells: *const Cell,
                                    n: u32, mode: i32) -> Status;
    pub fn marl_ruleset_pack_canonical(rs: *const Ruleset, out: *mut u8) -> Status;
    pub fn marl_ruleset_unpack_canonical(input: *const u8, rs: *mut Ruleset) -> Status;

    // engine (run(): seeding and the tick loop with host fate)
    pub fn marl_engine_create(gx: i32, gy: i32, gz: i32, sim: *const SimParams, rng_seed: u64, seed_count: u32,
                              cell_capacity: u32, out: *mut *mut Engine) -> Status;
    pub fn marl_engine_create_from_state(gx: i32, gy: i32, gz: i32, sim: *const SimParams, rng_seed: u64,
                                         field: *const f32, cells: *const Cell, n: u32, cell_capacity: u32,
                                         out: *mut *mut Engine) -> Status;
    pub fn marl_engine_destroy(e: *mut Engine);
    pub fn marl_engine_set_stream(e: *mut Engine, cuda_stream: *mut c_void) -> Status;
    pub fn marl_engine_step(e: *mut Engine, ticks: u32) -> Status;
    pub fn marl_engine_stats_get(e: *mut Engine, out: *mut EngineStats) -> Status;
    pub fn marl_engine_get_cells(e: *mut Engine, out: *mut Cell, cap: u32, n_out: *mut u32) -> Status;
    pub fn marl_engine_get_field(e: *mut Engine, field: *mut f32) -> Status;
    pub fn marl_engine_get_light(e: *mut Engine, light: *mut f32) -> Status;
    pub fn marl_engine_ctx(e: *mut Engine) -> *mut Ctx;
    pub fn marl_engine_set_device_fate(e: *mut Engine, enable: i32) -> Status;

    // batched ensemble
    pub fn marl_batch_create(runs: *const RunSpec, n_runs: u32, sim: *const SimParams, out: *mut *mut Batch)
        -> Status;
    pub fn marl_batch_destroy(b: *mut Batch);
    pub fn marl_batch_set_stream(b: *mut Batch, cuda_stream: *mut c_void) -> Status;
    pub fn marl_batch_set_host_threads(b: *mut Batch, threads: i32) -> Status;
    pub fn marl_batch_set_tile(b: *mut Batch, tile: i32, zc: i32) -> Status;
    pub fn marl_batch_get_tile(b: *mut Batch, tile: *mut i32, zc: *mut i32) -> Status;
    pub fn marl_batch_autotune(b: *mut Batch, reps: i32, best_us_per_substep: *mut f32) -> Status;
    pub fn marl_batch_set_graph(b: *mut Batch, use_graph: i32) -> Status;
    pub fn marl_batch_step(b: *mut Batch, ticks: u32) -> Status;
    pub fn marl_batch_run_count(b: *mut Batch, n_runs: *mut u32) -> Status;
    pub fn marl_batch_stats_get(b: *mut Batch, run: u32, out: *mut EngineStats) -> Status;
    pub fn marl_batch_get_cells(b: *mut Batch, run: u32, out: *mut Cell, cap: u32, n_out: *mut u32) -> Status;
    pub fn marl_batch_get_field(b: *mut Batch, run: u32, field: *mut f32) -> Status;
    pub fn marl_batch_get_light(b: *mut Batch, run: u32, light: *mut f32) -> Status;
    pub fn marl_batch_counters(b: *mut Batch, out: *mut Counters) -> Status;
    pub fn marl_batch_set_device_fate(b: *mut Batch, enable: i32) -> Status;

    // learned reaction surrogate
    pub fn marl_surrogate_config_default(out: *mut SurrogateConfig) -> Status;
    pub fn marl_surrogate_create(cfg: *const SurrogateConfig, out: *mut *mut Surrogate) -> Status;
    pub fn marl_surrogate_destroy(s: *mut Surrogate);
    pub fn marl_surrogate_set_stream(s: *mut Surrogate, cuda_stream: *mut c_void) -> Status;
    pub fn marl_surrogate_pair_count(s: *mut Surrogate, rows: *mut u32) -> Status;
    pub fn marl_surrogate_download_pairs(s: *mut Surrogate, row0: u32, n: u32, out: *mut f32) -> Status;
    pub fn marl_surrogate_upload_pairs(s: *mut Surrogate, rows: *const f32, n: u32) -> Status;
    pub fn marl_surrogate_prepare(s: *mut Surrogate, n_train: u32) -> Status;
    pub fn marl_surrogate_set_lr(s: *mut Surrogate, lr: f32) -> Status;
    pub fn marl_surrogate_train(s: *mut Surrogate, steps: u32, loss_out: *mut f32) -> Status;
    pub fn marl_surrogate_evaluate(s: *mut Surrogate, row0: u32, n: u32, tol: f32, out: *mut SurrogateEval,
                                   row_err_out: *mut f32) -> Status;
    pub fn marl_surrogate_get_weights(s: *mut Surrogate, params: *mut f32, norm: *mut f32) -> Status;
    pub fn marl_surrogate_set_weights(s: *mut Surrogate, params: *const f32, norm: *const f32) -> Status;
    pub fn marl_surrogate_gradients(s: *mut Surrogate, x: *const u16, t: *const f32, batch: u32,
                                    grads_out: *mut f32, loss_out: *mut f32, y_out: *mut f32) -> Status;
    pub fn marl_surrogate_set_inference(s: *mut Surrogate, fused: i32) -> Status;
    pub fn marl_surrogate_infer_device(s: *mut Surrogate, x_dev: *const u16, n: u32, y_dev: *mut f32, ldy: u32)
        -> Status;
    pub fn marl_ctx_set_surrogate(ctx: *mut Ctx, s: *mut Surrogate, mode: i32, tol: f32) -> Status;
    pub fn marl_ctx_surrogate_counters(ctx: *mut Ctx, out: *mut SurrogateCounters) -> Status;
    pub fn marl_batch_set_surrogate(b: *mut Batch, s: *mut Surrogate, mode: i32, tol: f32) -> Status;
    pub fn marl_batch_surrogate_counters(b: *mut Batch, out: *mut SurrogateCounters) -> Status;
}
