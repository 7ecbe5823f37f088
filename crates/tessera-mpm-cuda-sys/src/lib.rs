//! Raw bindings to `libtmpm.so`, the B200 (sm_100a) MLS-MPM substep library.
//!
//! Every item mirrors one declaration of `include/tmpm.h`, field for field and
//! argument for argument; the header documents the semantics and cites the
//! method of tessera-mpm's `GpuMpmResidentSession` (crates/tessera-mpm/src/
//! gpu.rs:206-662) or `MpmWorld` GPU convenience (gpu.rs:2168-2293) each entry
//! point replaces.  A `GpuMpmResidentSession` rebuilt on this crate keeps its
//! public API and error enum; [`status_error`] maps the integer status codes
//! onto the variants of `GpuMpmError` (gpu.rs:135-154) and `MpmError`
//! (world.rs:164-181) one to one.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_void};

/// Integer status of every fallible call (`TmpmStatus` in the header).
pub type TmpmStatus = i32;
pub const TMPM_OK: TmpmStatus = 0;
pub const TMPM_ERR_INVALID_INPUT: TmpmStatus = 1;
pub const TMPM_ERR_CAPACITY: TmpmStatus = 2;
pub const TMPM_ERR_PENDING_STEPS: TmpmStatus = 3;
pub const TMPM_ERR_READBACK: TmpmStatus = 4;
pub const TMPM_ERR_RESIDENT_UNAVAILABLE: TmpmStatus = 5;
pub const TMPM_ERR_MPM_INVALID_INPUT: TmpmStatus = 6;
pub const TMPM_ERR_EXCESSIVE_SUBSTEPS: TmpmStatus = 7;
pub const TMPM_ERR_NON_FINITE_STATE: TmpmStatus = 8;
pub const TMPM_ERR_UNKNOWN_CHUNK: TmpmStatus = 9;
pub const TMPM_ERR_PARTICLE_CAPACITY: TmpmStatus = 10;
pub const TMPM_ERR_DEVICE: TmpmStatus = 11;

/// Constitutive models, in the order of `MaterialModel` (material.rs:28-91).
pub type TmpmMaterialKind = i32;
pub const TMPM_MAT_ELASTIC: TmpmMaterialKind = 0;
pub const TMPM_MAT_NEO_HOOKEAN: TmpmMaterialKind = 1;
pub const TMPM_MAT_SAND: TmpmMaterialKind = 2;
pub const TMPM_MAT_FLUID: TmpmMaterialKind = 3;
pub const TMPM_MAT_SNOW: TmpmMaterialKind = 4;
pub const TMPM_MAT_SAND_NEO_HOOKEAN: TmpmMaterialKind = 5;

/// Obstacle shapes (obstacle.rs:10-61).
pub type TmpmObstacleShape = i32;
pub const TMPM_SHAPE_SPHERE: TmpmObstacleShape = 0;
pub const TMPM_SHAPE_BOX: TmpmObstacleShape = 1;
pub const TMPM_SHAPE_CAPSULE: TmpmObstacleShape = 2;
pub const TMPM_SHAPE_CYLINDER: TmpmObstacleShape = 3;
pub const TMPM_SHAPE_CONE: TmpmObstacleShape = 4;
pub const TMPM_SHAPE_GROUND: TmpmObstacleShape = 5;
pub const TMPM_SHAPE_TRIANGLE_PRISM: TmpmObstacleShape = 6;
pub const TMPM_SHAPE_CONVEX: TmpmObstacleShape = 7;

/// Boundary responses (obstacle.rs:63-77).
pub type TmpmBoundary = i32;
pub const TMPM_BOUNDARY_SLIP: TmpmBoundary = 0;
pub const TMPM_BOUNDARY_STICK: TmpmBoundary = 1;
pub const TMPM_BOUNDARY_SEPARATE: TmpmBoundary = 2;
pub const TMPM_BOUNDARY_NON_REFLECTING: TmpmBoundary = 3;
pub const TMPM_BOUNDARY_FREE_SLIP: TmpmBoundary = 4;

/// `MpmParams` (world.rs:27-49).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TmpmParams {
    pub cell_width: f64,
    pub gravity: [f64; 3],
    pub max_substep: f64,
    pub has_bounds: i32,
    pub wall_mode: i32,
    pub bounds_min: [f64; 3],
    pub bounds_max: [f64; 3],
}

/// Caller-owned structure-of-arrays view of `MpmParticle`s (world.rs:67-102);
/// matrices column-major, 9 doubles per particle.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct TmpmParticleArrays {
    pub count: usize,
    pub position: *mut f64,
    pub velocity: *mut f64,
    pub deformation: *mut f64,
    pub affine: *mut f64,
    pub force: *mut f64,
    pub mass: *mut f64,
    pub rest_volume: *mut f64,
    pub radius: *mut f64,
    pub damping: *mut f64,
    pub plastic: *mut f64,
    pub material: *mut i32,
    pub material_params: *mut f64,
    pub enabled: *mut u8,
    pub fixed: *mut u8,
    pub transfer_color: *mut u16,
    pub group_id: *mut u32,
    pub chunk_id: *mut u64,
}

/// One prescribed rigid obstacle (`RigidObstacle`, obstacle.rs:79-98).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct TmpmObstacle {
    pub shape: i32,
    pub boundary: i32,
    pub cpic_group: i32,
    pub plane_count: u32,
    pub center: [f64; 3],
    pub orientation: [f64; 4],
    pub linear_velocity: [f64; 3],
    pub angular_velocity: [f64; 3],
    pub friction: f64,
    pub dims: [f64; 3],
    pub vertices: [f64; 9],
    pub bound_radius: f64,
    pub planes: *const f64,
}

/// Optional session knobs; all-zero means defaults.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TmpmSessionOptions {
    pub device: i32,
    pub max_blocks: u32,
    pub resort_interval: u32,
    pub launch_shape: u32,
    pub next_chunk_id: u64,
    pub substeps: u64,
}

/// A rigid body of the MPM-owned two-way coupling (gpu_rigid_sync.rs:62-500).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TmpmRigidBody {
    pub position: [f64; 3],
    pub inverse_mass: f64,
    pub orientation: [f64; 4],
    pub linear_velocity: [f64; 3],
    pub angular_velocity: [f64; 3],
    pub inverse_inertia: [f64; 3],
}

/// Obstacle -> body mapping of the coupling.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TmpmRigidMapping {
    pub body: i32,
    pub reserved: i32,
    pub local_center: [f64; 3],
    pub local_orientation: [f64; 4],
}

/// Options of a multi-scene batch.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct TmpmBatchOptions {
    pub device: i32,
    pub max_blocks: u32,
    pub use_graphs: u32,
    pub launch_shape: u32,
    pub particle_capacity: u64,
}

/// Opaque handles.
#[repr(C)]
pub struct TmpmSession {
    _private: [u8; 0],
}
#[repr(C)]
pub struct TmpmBatch {
    _private: [u8; 0],
}
#[repr(C)]
pub struct TmpmPreparedScene {
    _private: [u8; 0],
}
#[repr(C)]
pub struct TmpmAdjoint {
    _private: [u8; 0],
}

extern "C" {
    // session lifecycle (GpuMpmResidentSession)
    pub fn tmpm_session_create(params: *const TmpmParams, particles: *const TmpmParticleArrays,
                               obstacles: *const TmpmObstacle, obstacle_count: usize, use_cpic: i32,
                               substep_dt: f64, options: *const TmpmSessionOptions,
                               out: *mut *mut TmpmSession) -> TmpmStatus;
    pub fn tmpm_session_destroy(session: *mut TmpmSession);
    pub fn tmpm_submit_steps(session: *mut TmpmSession, steps: u32) -> TmpmStatus;
    pub fn tmpm_step(session: *mut TmpmSession, steps: u32) -> TmpmStatus;
    pub fn tmpm_synchronize(session: *mut TmpmSession) -> TmpmStatus;
    pub fn tmpm_pending_substeps(session: *const TmpmSession) -> u64;
    pub fn tmpm_has_pending_steps(session: *const TmpmSession) -> i32;
    pub fn tmpm_substeps(session: *const TmpmSession) -> u64;
    pub fn tmpm_particle_count(session: *const TmpmSession) -> usize;
    pub fn tmpm_read_particles(session: *const TmpmSession, out: *mut TmpmParticleArrays) -> TmpmStatus;
    pub fn tmpm_stable_timestep(session: *const TmpmSession) -> f64;
    pub fn tmpm_set_particle_force(session: *mut TmpmSession, index: usize, force: *const f64) -> TmpmStatus;
    pub fn tmpm_set_obstacles(session: *mut TmpmSession, obstacles: *const TmpmObstacle,
                              count: usize) -> TmpmStatus;
    pub fn tmpm_add_particles(session: *mut TmpmSession, particles: *const TmpmParticleArrays,
                              chunk_out: *mut u64) -> TmpmStatus;
    pub fn tmpm_remove_chunk(session: *mut TmpmSession, chunk: u64, removed_out: *mut usize) -> TmpmStatus;
    pub fn tmpm_write_particles(session: *mut TmpmSession, particles: *const TmpmParticleArrays) -> TmpmStatus;
    pub fn tmpm_encode_particle_snapshot(session: *mut TmpmSession, device_out: *mut c_void,
                                         capacity_bytes: usize, written: *mut u32) -> TmpmStatus;
    pub fn tmpm_substep_dt(session: *const TmpmSession) -> f64;
    pub fn tmpm_set_substep_dt(session: *mut TmpmSession, substep_dt: f64) -> TmpmStatus;

    // MpmWorld GPU conveniences
    pub fn tmpm_step_cfl(session: *mut TmpmSession, dt: f64) -> TmpmStatus;
    pub fn tmpm_step_cfl_with_reactions(session: *mut TmpmSession, dt: f64, reactions_out: *mut f64,
                                        obstacle_count: usize) -> TmpmStatus;

    // two-way rigid coupling, MPM-owned
    pub fn tmpm_rigid_attach(session: *mut TmpmSession, bodies: *const TmpmRigidBody, body_count: usize,
                             mappings: *const TmpmRigidMapping, mapping_count: usize) -> TmpmStatus;
    pub fn tmpm_rigid_step(session: *mut TmpmSession, substeps: u32, gravity: *const f64,
                           max_linear_speed: f64, integrate_pose: i32) -> TmpmStatus;
    pub fn tmpm_rigid_read(session: *mut TmpmSession, bodies: *mut TmpmRigidBody, body_count: usize) -> TmpmStatus;
    pub fn tmpm_rigid_detach(session: *mut TmpmSession);

    // allocation-free binning step
    pub fn tmpm_sort_by_block_noalloc(positions: *const f32, count: usize, stride: usize, cell_width: f64,
                                      order_out: *mut u32, keys_out: *mut u32, stream: *mut c_void) -> TmpmStatus;

    // multi-scene batches and serving
    pub fn tmpm_batch_create(options: *const TmpmBatchOptions, out: *mut *mut TmpmBatch) -> TmpmStatus;
    pub fn tmpm_batch_destroy(batch: *mut TmpmBatch);
    pub fn tmpm_scene_prepare(params: *const TmpmParams, particles: *const TmpmParticleArrays, substep_dt: f64,
                              out: *mut *mut TmpmPreparedScene) -> TmpmStatus;
    pub fn tmpm_scene_prepared_destroy(prepared: *mut TmpmPreparedScene);
    pub fn tmpm_scene_prepared_particle_count(prepared: *const TmpmPreparedScene) -> usize;
    pub fn tmpm_scene_prepared_bytes(prepared: *const TmpmPreparedScene) -> usize;
    pub fn tmpm_batch_admit(batch: *mut TmpmBatch, prepared: *mut TmpmPreparedScene,
                            scene_out: *mut u32) -> TmpmStatus;
    pub fn tmpm_batch_add_scene(batch: *mut TmpmBatch, params: *const TmpmParams,
                                particles: *const TmpmParticleArrays, substep_dt: f64,
                                scene_out: *mut u32) -> TmpmStatus;
    pub fn tmpm_batch_remove_scene(batch: *mut TmpmBatch, scene: u32) -> TmpmStatus;
    pub fn tmpm_batch_submit(batch: *mut TmpmBatch, ids: *const u32, steps: *const u32, count: usize) -> TmpmStatus;
    pub fn tmpm_batch_synchronize(batch: *mut TmpmBatch) -> TmpmStatus;
    pub fn tmpm_batch_pending(batch: *const TmpmBatch) -> i32;
    pub fn tmpm_batch_scene_status(batch: *const TmpmBatch, scene: u32) -> TmpmStatus;
    pub fn tmpm_batch_scene_substeps(batch: *const TmpmBatch, scene: u32) -> u64;
    pub fn tmpm_batch_scene_particle_count(batch: *const TmpmBatch, scene: u32) -> usize;
    pub fn tmpm_batch_read_scene(batch: *mut TmpmBatch, scene: u32, out: *mut TmpmParticleArrays) -> TmpmStatus;
    pub fn tmpm_batch_take_scene(batch: *mut TmpmBatch, scene: u32, out: *mut TmpmParticleArrays) -> TmpmStatus;
    pub fn tmpm_batch_last_ms(batch: *const TmpmBatch) -> f64;
    pub fn tmpm_batch_device_bytes(batch: *const TmpmBatch) -> usize;
    pub fn tmpm_batch_scene_bytes(particles: usize, home_blocks: usize) -> usize;
    pub fn tmpm_batch_last_error_message(batch: *const TmpmBatch) -> *const c_char;

    // differentiable rollout
    pub fn tmpm_adjoint_create(params: *const TmpmParams, particles: *const TmpmParticleArrays, substep_dt: f64,
                               substeps: u32, checkpoint_every: u32, device: i32,
                               out: *mut *mut TmpmAdjoint) -> TmpmStatus;
    pub fn tmpm_adjoint_destroy(adjoint: *mut TmpmAdjoint);
    pub fn tmpm_adjoint_particle_count(adjoint: *const TmpmAdjoint) -> usize;
    pub fn tmpm_adjoint_forward(adjoint: *mut TmpmAdjoint, velocity0: *const f64, young: *const f64,
                                position_out: *mut f64, velocity_out: *mut f64) -> TmpmStatus;
    pub fn tmpm_adjoint_backward(adjoint: *mut TmpmAdjoint, position_grad: *const f64, velocity_grad: *const f64,
                                 velocity0_grad: *mut f64, young_grad: *mut f64) -> TmpmStatus;
    pub fn tmpm_adjoint_last_error_message(adjoint: *const TmpmAdjoint) -> *const c_char;

    // errors, version, diagnostics
    pub fn tmpm_last_error_message(session: *const TmpmSession) -> *const c_char;
    pub fn tmpm_last_error() -> *const c_char;
    pub fn tmpm_version() -> *const c_char;
    pub fn tmpm_device_count(session: *const TmpmSession) -> usize;
    pub fn tmpm_debug_binning(session: *mut TmpmSession, world_index_out: *mut u32, base_cell_out: *mut i32,
                              key_out: *mut u32) -> TmpmStatus;
    pub fn tmpm_debug_p2g(session: *mut TmpmSession, cells_out: *mut i32, mass_momentum_out: *mut f32,
                          capacity: usize, count: *mut usize) -> TmpmStatus;
    pub fn tmpm_bench_substeps(session: *mut TmpmSession, steps: u32, ms: *mut f64, kernel_ms: *mut f64,
                               kernel_count: usize) -> TmpmStatus;

    // launch shapes of the transfer kernels
    pub fn tmpm_launch_shape_count() -> u32;
    pub fn tmpm_launch_shape_info(shape: u32, threads_per_cta: *mut u32, ctas_per_sm: *mut u32,
                                  block_edge: *mut u32) -> TmpmStatus;
    pub fn tmpm_session_launch_shape(session: *mut TmpmSession, ms_per_unit: *mut f64, count: usize) -> i32;
    pub fn tmpm_batch_launch_shape(batch: *mut TmpmBatch, ms_per_unit: *mut f64, count: usize) -> i32;
}

/// The error variants of the reference's `GpuMpmError` (gpu.rs:135-154) with
/// `GpuMpmError::Reference(MpmError)` (world.rs:164-181) flattened, plus the
/// device loss the CUDA runtime can report.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum TmpmError {
    InvalidInput,
    Capacity,
    PendingSteps,
    Readback,
    ResidentUnavailable,
    MpmInvalidInput,
    ExcessiveSubsteps,
    NonFiniteState,
    UnknownChunk,
    ParticleCapacity,
    Device,
    Unknown(i32),
}

/// `Ok(())` for `TMPM_OK`, else the matching error variant.
pub fn status_error(status: TmpmStatus) -> Result<(), TmpmError> {
    match status {
        TMPM_OK => Ok(()),
        TMPM_ERR_INVALID_INPUT => Err(TmpmError::InvalidInput),
        TMPM_ERR_CAPACITY => Err(TmpmError::Capacity),
        TMPM_ERR_PENDING_STEPS => Err(TmpmError::PendingSteps),
        TMPM_ERR_READBACK => Err(TmpmError::Readback),
        TMPM_ERR_RESIDENT_UNAVAILABLE => Err(TmpmError::ResidentUnavailable),
        TMPM_ERR_MPM_INVALID_INPUT => Err(TmpmError::MpmInvalidInput),
        TMPM_ERR_EXCESSIVE_SUBSTEPS => Err(TmpmError::ExcessiveSubsteps),
        TMPM_ERR_NON_FINITE_STATE => Err(TmpmError::NonFiniteState),
        TMPM_ERR_UNKNOWN_CHUNK => Err(TmpmError::UnknownChunk),
        TMPM_ERR_PARTICLE_CAPACITY => Err(TmpmError::ParticleCapacity),
        TMPM_ERR_DEVICE => Err(TmpmError::Device),
        other => Err(TmpmError::Unknown(other)),
    }
}
