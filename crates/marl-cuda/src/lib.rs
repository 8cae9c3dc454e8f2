//! marl-cuda: MARL's per-tick field-and-cell path on a B200 (sm_100a), as a
//! drop-in beside marl-gpu's wgpu prototype.
//!
//! Two safe types sit over the C ABI of libmarl_cuda.so (`ffi`):
//!
//! - [`CudaFieldDiffuser`] has the shape of `marl_gpu::GpuFieldDiffuser`
//!   (crates/marl-gpu/src/field_diffusion.rs:32,158-268): `new()` and
//!   `diffuse_tick_with_cells(&mut Field, &[bool], &SimulationConfig)`, the
//!   field updated in place, `diffusion_substeps == 0` doing nothing, and
//!   errors as [`GpuError`] with the reference's variants.  marl-sim calls it
//!   where the `gpu` feature calls the wgpu diffuser today
//!   (crates/marl-sim/src/lib.rs:133-146,180-193).
//! - [`CudaTickEngine`] keeps the field, light, occupancy and the cell table in
//!   device memory across ticks and runs steps 1-5 of a tick
//!   (crates/marl-sim/src/lib.rs:164-217: sources, diffusion, light and the
//!   sequential cell loop, reproduced exactly).  Each [`CudaTickEngine::tick`]
//!   returns the ordered Division/Death change list; the unchanged host fate
//!   code (lib.rs:219-277) runs on it and its record ([`Edits`]) goes back with
//!   [`CudaTickEngine::apply_edits`].
//!
//! There is no CPU fallback: every failure is returned, never masked.

pub mod ffi;

use std::ffi::CStr;
use std::fmt;

use marl_cell::cell::{
    CellEvent, CellState, EffectorParams, FateParams, Reaction, ReceptorParams, Ruleset, TransportParams,
};
use marl_config::{GRID_X, GRID_Y, GRID_Z, M_INT, R_MAX, S_EFFECTORS, S_EXT, S_RECEPTORS, S_TRANSPORTERS,
                  SimulationConfig};
use marl_field::field::Field;
use marl_field::light::LightField;

const VOXELS: usize = GRID_X * GRID_Y * GRID_Z;

/// Errors of the CUDA backend.  The first four variants are those of
/// `marl_gpu::GpuError` (crates/marl-gpu/src/context.rs:5-10), so callers that
/// report a GPU failure handle both alike.
#[derive(Debug, Clone)]
pub enum GpuError {
    NoAdapter,
    DeviceRequest(String),
    BufferMap(String),
    InvalidInput(String),
    /// A bounded device-side wait gave up (MARL_ERR_TIMEOUT).
    Timeout(String),
    /// Cell table or change list full (MARL_ERR_CAPACITY).
    Capacity(String),
    /// Call not valid in the backend's current state (MARL_ERR_STATE).
    State(String),
}

impl fmt::Display for GpuError {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        match self {
            Self::NoAdapter => write!(f, "no sm_100 CUDA device found"),
            Self::DeviceRequest(e) => write!(f, "CUDA device error: {e}"),
            Self::BufferMap(e) => write!(f, "device transfer failed: {e}"),
            Self::InvalidInput(e) => write!(f, "invalid CUDA backend input: {e}"),
            Self::Timeout(e) => write!(f, "device wait timed out: {e}"),
            Self::Capacity(e) => write!(f, "capacity exceeded: {e}"),
            Self::State(e) => write!(f, "invalid backend state: {e}"),
        }
    }
}

impl std::error::Error for GpuError {}

fn last_error() -> String {
    // SAFETY: marl_last_error returns a NUL-terminated thread-local string.
    unsafe { CStr::from_ptr(ffi::marl_last_error()) }.to_string_lossy().into_owned()
}

/// Maps a status code of the C ABI to a Result.
pub fn check(st: ffi::Status) -> Result<(), GpuError> {
    match st {
        ffi::MARL_OK => Ok(()),
        ffi::MARL_ERR_INVALID_INPUT => Err(GpuError::InvalidInput(last_error())),
        ffi::MARL_ERR_NO_DEVICE => Err(GpuError::NoAdapter),
        ffi::MARL_ERR_TIMEOUT => Err(GpuError::Timeout(last_error())),
        ffi::MARL_ERR_CAPACITY => Err(GpuError::Capacity(last_error())),
        ffi::MARL_ERR_STATE => Err(GpuError::State(last_error())),
        _ => Err(GpuError::DeviceRequest(last_error())),
    }
}

/// SimulationConfig (crates/marl-config/src/lib.rs:41-106) as the C ABI's
/// marl_sim_params: the same fields in the same order, usize/u16/u8 widened to
/// u32, boundary sources in the reference's additive form.
pub fn params_from(sim: &SimulationConfig) -> ffi::SimParams {
    ffi::SimParams {
        dx: sim.dx,
        dt: sim.dt,
        diffusion_substeps: sim.diffusion_substeps as u32,
        d_voxel: sim.d_voxel,
        lambda_decay: sim.lambda_decay,
        source_rate_oxidant: sim.source_rate_oxidant,
        source_rate_carbon: sim.source_rate_carbon,
        source_rate_reductant: sim.source_rate_reductant,
        epsilon: sim.epsilon,
        c_max: sim.c_max,
        lambda_maintenance: sim.lambda_maintenance,
        hard_death_floor: sim.hard_death_floor,
        reaction_maintenance: sim.reaction_maintenance,
        base_division_prep: sim.base_division_prep,
        prep_maintenance_multiplier: sim.prep_maintenance_multiplier,
        rush_penalty_rate: sim.rush_penalty_rate,
        alpha_eps: sim.alpha_eps,
        k_eps: sim.k_eps,
        light_efficiency: sim.light_efficiency,
        surface_intensity: sim.surface_intensity,
        cell_absorption: sim.cell_absorption,
        chemical_absorption: sim.chemical_absorption,
        light_floor: sim.light_floor,
        mutation_stddev: sim.mutation_stddev,
        structural_mutation_rate_mult: sim.structural_mutation_rate_mult,
        meta_mutation_rate: sim.meta_mutation_rate,
        meta_mutation_clamp_low: sim.meta_mutation_clamp_low,
        meta_mutation_clamp_high: sim.meta_mutation_clamp_high,
        hill_exponent_clamp_low: sim.hill_exponent_clamp_low,
        hill_exponent_clamp_high: sim.hill_exponent_clamp_high,
        active_reaction_threshold: sim.active_reaction_threshold,
        seed_margin: sim.seed_margin as u32,
        phototroph_z_lo: sim.phototroph_z_lo,
        phototroph_z_hi: sim.phototroph_z_hi,
        chemolithotroph_z_lo: sim.chemolithotroph_z_lo,
        chemolithotroph_z_hi: sim.chemolithotroph_z_hi,
        anaerobe_z_lo: sim.anaerobe_z_lo,
        anaerobe_z_hi: sim.anaerobe_z_hi,
        division_neighbor_distance: sim.division_neighbor_distance as u32,
        boundary_prime_layers: sim.boundary_prime_layers as u32,
        boundary_prime_oxidant: sim.boundary_prime_oxidant,
        boundary_prime_carbon: sim.boundary_prime_carbon,
        boundary_prime_reductant: sim.boundary_prime_reductant,
        source_mode: ffi::MARL_SOURCES_ADDITIVE,
    }
}

/// A CellState as the C ABI's 656-byte record.
pub fn cell_to_ffi(c: &CellState) -> ffi::Cell {
    let r = &c.ruleset;
    let mut out = ffi::Cell {
        pos: c.pos,
        quiescent: c.quiescent as u8,
        starter_type: c.starter_type,
        age: c.age,
        prep_remaining: c.prep_remaining,
        _pad0: 0,
        lineage_id: c.lineage_id,
        internal: c.internal,
        ruleset: ffi::Ruleset::default(),
    };
    let o = &mut out.ruleset;
    for i in 0..S_RECEPTORS {
        let p = &r.receptors[i];
        o.receptors[i] = ffi::ReceptorParams { k_half: p.k_half, n_hill: p.n_hill, gain: p.gain };
    }
    for i in 0..S_TRANSPORTERS {
        let p = &r.transport[i];
        o.transport[i] = ffi::TransportParams {
            uptake_rate: p.uptake_rate,
            secrete_rate: p.secrete_rate,
            ext_species: p.ext_species,
            int_species: p.int_species,
            _pad: [0; 2],
        };
    }
    for i in 0..R_MAX {
        let p = &r.reactions[i];
        o.reactions[i] = ffi::Reaction {
            substrate: p.substrate,
            product: p.product,
            catalyst: p.catalyst,
            cofactor: p.cofactor,
            k_m: p.k_m,
            v_max: p.v_max,
            k_cat: p.k_cat,
        };
    }
    for i in 0..S_EFFECTORS {
        let p = &r.effectors[i];
        o.effectors[i] = ffi::EffectorParams {
            threshold: p.threshold,
            rate: p.rate,
            int_species: p.int_species,
            ext_species: p.ext_species,
            _pad: [0; 2],
        };
    }
    o.fate = ffi::FateParams {
        division_energy: r.fate.division_energy,
        death_energy: r.fate.death_energy,
        quiescence_energy: r.fate.quiescence_energy,
        division_prep_ticks: r.fate.division_prep_ticks,
    };
    o.hgt_propensity = r.hgt_propensity;
    o.mutation_rate = r.mutation_rate;
    out
}

/// The inverse of [`cell_to_ffi`].
pub fn cell_from_ffi(c: &ffi::Cell) -> CellState {
    let o = &c.ruleset;
    let ruleset = Ruleset {
        receptors: std::array::from_fn(|i| {
            let p = &o.receptors[i];
            ReceptorParams { k_half: p.k_half, n_hill: p.n_hill, gain: p.gain }
        }),
        transport: std::array::from_fn(|i| {
            let p = &o.transport[i];
            TransportParams {
                uptake_rate: p.uptake_rate,
                secrete_rate: p.secrete_rate,
                ext_species: p.ext_species,
                int_species: p.int_species,
            }
        }),
        reactions: std::array::from_fn(|i| {
            let p = &o.reactions[i];
            Reaction {
                substrate: p.substrate,
                product: p.product,
                catalyst: p.catalyst,
                cofactor: p.cofactor,
                k_m: p.k_m,
                v_max: p.v_max,
                k_cat: p.k_cat,
            }
        }),
        effectors: std::array::from_fn(|i| {
            let p = &o.effectors[i];
            EffectorParams {
                threshold: p.threshold,
                rate: p.rate,
                int_species: p.int_species,
                ext_species: p.ext_species,
            }
        }),
        fate: FateParams {
            division_energy: o.fate.division_energy,
            death_energy: o.fate.death_energy,
            quiescence_energy: o.fate.quiescence_energy,
            division_prep_ticks: o.fate.division_prep_ticks,
        },
        hgt_propensity: o.hgt_propensity,
        mutation_rate: o.mutation_rate,
    };
    CellState {
        pos: c.pos,
        lineage_id: c.lineage_id,
        age: c.age,
        internal: c.internal,
        ruleset,
        quiescent: c.quiescent != 0,
        starter_type: c.starter_type,
        prep_remaining: c.prep_remaining,
    }
}

fn check_field_sizes(field: &Field, occupancy: &[bool]) -> Result<(), GpuError> {
    if field.data.len() != VOXELS * S_EXT {
        return Err(GpuError::InvalidInput(format!(
            "field has {} floats, expected {}",
            field.data.len(),
            VOXELS * S_EXT
        )));
    }
    if occupancy.len() != VOXELS {
        return Err(GpuError::InvalidInput(format!(
            "occupancy has {} entries, expected {VOXELS}",
            occupancy.len()
        )));
    }
    Ok(())
}

/// Drop-in for `marl_gpu::GpuFieldDiffuser` on the CUDA backend.
pub struct CudaFieldDiffuser {
    ctx: *mut ffi::Ctx,
}

impl CudaFieldDiffuser {
    /// Opens the device context for the compile-time grid.  Like the
    /// reference constructor, it takes no configuration: the parameters come
    /// with every diffusion call.
    pub fn new() -> Result<Self, GpuError> {
        let mut p = ffi::SimParams::default();
        check(unsafe { ffi::marl_sim_params_default(&mut p) })?;
        let mut ctx = std::ptr::null_mut();
        check(unsafe { ffi::marl_ctx_create(GRID_X as i32, GRID_Y as i32, GRID_Z as i32, &p, 1, &mut ctx) })?;
        Ok(Self { ctx })
    }

    /// `sim.diffusion_substeps` masked diffusion substeps of the host field in
    /// place (Field::diffuse_tick_with_cells, crates/marl-field/src/field.rs:
    /// 212-217); occupied voxels are copied unchanged.  Synchronous.
    pub fn diffuse_tick_with_cells(&mut self, field: &mut Field, occupancy: &[bool], sim: &SimulationConfig)
        -> Result<(), GpuError> {
        check_field_sizes(field, occupancy)?;
        if sim.diffusion_substeps == 0 {
            return Ok(());
        }
        let p = params_from(sim);
        check(unsafe { ffi::marl_ctx_set_params(self.ctx, &p) })?;
        // A Rust bool is one byte holding 0 or 1: the ABI's occupancy format.
        check(unsafe {
            ffi::marl_diffuse_tick_with_cells(self.ctx, field.data.as_mut_ptr(), occupancy.as_ptr() as *const u8)
        })
    }
}

impl Drop for CudaFieldDiffuser {
    fn drop(&mut self) {
        unsafe { ffi::marl_ctx_destroy(self.ctx) }
    }
}

/// One entry of a tick's change list (a Division or Death event).
#[derive(Clone, Debug)]
pub struct Change {
    /// Index of the cell in the cell vector at the start of the tick.
    pub cell: usize,
    pub event: CellEvent,
    /// The cell's state after its tick (what the host fate step clones).
    pub internal: [f32; M_INT],
    pub quiescent: bool,
}

/// What the host fate step did to the cell vector, in application order
/// (crates/marl-sim/src/lib.rs:220-277).
#[derive(Clone, Debug, Default)]
pub struct Edits {
    /// Parents whose internal state was halved (indices at the tick's start).
    pub halve: Vec<u32>,
    /// Dead cells, ascending and unique.
    pub deaths: Vec<u32>,
    /// swap_remove moves: slot `move_dst[k]` received the cell of `move_src[k]`.
    pub move_dst: Vec<u32>,
    pub move_src: Vec<u32>,
    /// Population after the deaths, before the births.
    pub n_after_deaths: u32,
    /// Daughters appended at `n_after_deaths`, `n_after_deaths + 1`, ...
    pub births: Vec<CellState>,
}

/// The device-resident tick loop: field, light, occupancy and the cell table
/// stay in HBM; the host keeps fate, division, mutation and lineage.
pub struct CudaTickEngine {
    ctx: *mut ffi::Ctx,
    capacity: u32,
    changes: Vec<ffi::Change>,
}

impl CudaTickEngine {
    /// Uploads the run's state: the field (with its boundary priming) and the
    /// cell vector.  `capacity` bounds the population the table can hold.
    pub fn new(sim: &SimulationConfig, field: &Field, cells: &[CellState], capacity: u32)
        -> Result<Self, GpuError> {
        if field.data.len() != VOXELS * S_EXT {
            return Err(GpuError::InvalidInput("field size".into()));
        }
        let p = params_from(sim);
        let mut ctx = std::ptr::null_mut();
        check(unsafe { ffi::marl_ctx_create(GRID_X as i32, GRID_Y as i32, GRID_Z as i32, &p, capacity, &mut ctx) })?;
        let mut e = Self { ctx, capacity, changes: Vec::new() };
        check(unsafe { ffi::marl_upload_field(e.ctx, field.data.as_ptr()) })?;
        e.upload_cells(cells)?;
        Ok(e)
    }

    /// Replaces the device cell table (and the occupancy built from it).
    pub fn upload_cells(&mut self, cells: &[CellState]) -> Result<(), GpuError> {
        let recs: Vec<ffi::Cell> = cells.iter().map(cell_to_ffi).collect();
        check(unsafe { ffi::marl_upload_cells(self.ctx, recs.as_ptr(), recs.len() as u32) })
    }

    /// Steps 1-5 of one tick on the device (crates/marl-sim/src/lib.rs:164-217);
    /// returns the Division and Death events in ascending cell order.
    pub fn tick(&mut self) -> Result<Vec<Change>, GpuError> {
        self.changes.resize(self.capacity as usize + 1, ffi::Change::default());
        let mut n = 0u32;
        check(unsafe {
            ffi::marl_tick(self.ctx, self.changes.as_mut_ptr(), self.changes.len() as u32, &mut n)
        })?;
        Ok(self.changes[..n as usize]
            .iter()
            .map(|c| Change {
                cell: c.cell as usize,
                event: if c.event == ffi::MARL_EVENT_DIVISION { CellEvent::Division } else { CellEvent::Death },
                internal: c.internal,
                quiescent: c.quiescent != 0,
            })
            .collect())
    }

    /// Applies the host fate step's record to the device cell table.
    pub fn apply_edits(&mut self, edits: &Edits) -> Result<(), GpuError> {
        if edits.move_dst.len() != edits.move_src.len() {
            return Err(GpuError::InvalidInput("move_dst and move_src differ in length".into()));
        }
        let births: Vec<ffi::Cell> = edits.births.iter().map(cell_to_ffi).collect();
        let list = ffi::EditList {
            n_halve: edits.halve.len() as u32,
            halve: edits.halve.as_ptr(),
            n_deaths: edits.deaths.len() as u32,
            deaths: edits.deaths.as_ptr(),
            n_moves: edits.move_dst.len() as u32,
            move_dst: edits.move_dst.as_ptr(),
            move_src: edits.move_src.as_ptr(),
            n_after_deaths: edits.n_after_deaths,
            n_births: births.len() as u32,
            births: births.as_ptr(),
        };
        check(unsafe { ffi::marl_apply_edits(self.ctx, &list) })
    }

    /// Copies the device state back for output at the stats/snapshot cadence.
    pub fn sync_to_host(&mut self, field: &mut Field, light: &mut LightField, cells: &mut Vec<CellState>)
        -> Result<(), GpuError> {
        if field.data.len() != VOXELS * S_EXT || light.data.len() != VOXELS {
            return Err(GpuError::InvalidInput("field or light size".into()));
        }
        check(unsafe { ffi::marl_download_field(self.ctx, field.data.as_mut_ptr()) })?;
        check(unsafe { ffi::marl_download_light(self.ctx, light.data.as_mut_ptr()) })?;
        let mut n = 0u32;
        check(unsafe { ffi::marl_cell_count(self.ctx, &mut n) })?;
        let mut recs = vec![ffi::Cell::default(); n as usize];
        let mut got = 0u32;
        check(unsafe { ffi::marl_download_cells(self.ctx, recs.as_mut_ptr(), n, &mut got) })?;
        cells.clear();
        cells.extend(recs[..got as usize].iter().map(cell_from_ffi));
        Ok(())
    }

    /// Per-species mass of the field, summed in f64 on the device.
    pub fn mass(&mut self) -> Result<[f64; S_EXT], GpuError> {
        let mut out = [0.0f64; S_EXT];
        check(unsafe { ffi::marl_mass_f64(self.ctx, out.as_mut_ptr()) })?;
        Ok(out)
    }
}

impl Drop for CudaTickEngine {
    fn drop(&mut self) {
        unsafe { ffi::marl_ctx_destroy(self.ctx) }
    }
}
