/*
 * tmpm.h -- C ABI of the B200 (sm_100a) MLS-MPM substep library `libtmpm.so`.
 *
 * The library is a drop-in device backend for tessera-mpm's resident GPU path.
 * Every entry point below replaces one method of the reference's Rust type
 * `GpuMpmResidentSession` (crates/tessera-mpm/src/gpu.rs:206-662) or one of the
 * `MpmWorld` GPU conveniences (gpu.rs:2168-2293); the citation sits beside each
 * declaration.  Types are plain C: host pointers, sizes and integer status codes,
 * so a Rust `extern "C"` block, cgo or Python ctypes can bind them directly.
 *
 * Threading: a session is single-owner, like the reference's session (one wgpu
 * queue, `&mut self` methods).  Distinct sessions may be used from distinct
 * threads.  All calls are synchronous with respect to host memory: host arrays
 * passed in are not retained after the call returns.
 */
#ifndef TMPM_H
#define TMPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, one per variant of GpuMpmError (gpu.rs:135-154) and MpmError
 * (world.rs:164-181).  The Python binding maps every non-zero status onto
 * TesseraError.Failed(reason) exactly like tessera-python3d (lib.rs:82-95). */
typedef enum TmpmStatus {
    TMPM_OK = 0,
    TMPM_ERR_INVALID_INPUT = 1,        /* GpuMpmError::InvalidInput */
    TMPM_ERR_CAPACITY = 2,             /* GpuMpmError::Capacity */
    TMPM_ERR_PENDING_STEPS = 3,        /* GpuMpmError::PendingSteps */
    TMPM_ERR_READBACK = 4,             /* GpuMpmError::Readback(String) */
    TMPM_ERR_RESIDENT_UNAVAILABLE = 5, /* GpuMpmError::ResidentUnavailable */
    TMPM_ERR_MPM_INVALID_INPUT = 6,    /* GpuMpmError::Reference(MpmError::InvalidInput) */
    TMPM_ERR_EXCESSIVE_SUBSTEPS = 7,   /* MpmError::ExcessiveSubsteps */
    TMPM_ERR_NON_FINITE_STATE = 8,     /* MpmError::NonFiniteState */
    TMPM_ERR_UNKNOWN_CHUNK = 9,        /* MpmError::UnknownChunk */
    TMPM_ERR_PARTICLE_CAPACITY = 10,   /* MpmError::ParticleCapacity */
    TMPM_ERR_DEVICE = 11               /* CUDA runtime failure (wgpu device loss in the reference) */
} TmpmStatus;

/* Constitutive models, in the order of MaterialModel (material.rs:28-91). */
typedef enum TmpmMaterialKind {
    TMPM_MAT_ELASTIC = 0,          /* params: young, poisson (corotated, material.rs:440-455) */
    TMPM_MAT_NEO_HOOKEAN = 1,      /* params: young, poisson (material.rs:457-467) */
    TMPM_MAT_SAND = 2,             /* params: young, poisson, friction_angle, cohesion */
    TMPM_MAT_FLUID = 3,            /* params: bulk, gamma, viscosity, tensile_stiffness (material.rs:469-486) */
    TMPM_MAT_SNOW = 4,             /* params: young, poisson, critical_compression, critical_stretch, hardening */
    TMPM_MAT_SAND_NEO_HOOKEAN = 5  /* params: young, poisson, friction_angle, cohesion */
} TmpmMaterialKind;

/* Obstacle shapes (obstacle.rs:10-61). */
typedef enum TmpmObstacleShape {
    TMPM_SHAPE_SPHERE = 0,         /* dims[0] = radius */
    TMPM_SHAPE_BOX = 1,            /* dims = half extents */
    TMPM_SHAPE_CAPSULE = 2,        /* dims[0] = half_height, dims[1] = radius */
    TMPM_SHAPE_CYLINDER = 3,       /* dims[0] = half_height, dims[1] = radius */
    TMPM_SHAPE_CONE = 4,           /* dims[0] = half_height, dims[1] = radius */
    TMPM_SHAPE_GROUND = 5,         /* dims[0..2] = half extents x, y */
    TMPM_SHAPE_TRIANGLE_PRISM = 6, /* dims[0] = half_thickness, vertices = a, b, c */
    TMPM_SHAPE_CONVEX = 7          /* planes, plane_count, bound_radius */
} TmpmObstacleShape;

/* Boundary responses (obstacle.rs:63-77). */
typedef enum TmpmBoundary {
    TMPM_BOUNDARY_SLIP = 0,
    TMPM_BOUNDARY_STICK = 1,
    TMPM_BOUNDARY_SEPARATE = 2,
    TMPM_BOUNDARY_NON_REFLECTING = 3,
    TMPM_BOUNDARY_FREE_SLIP = 4
} TmpmBoundary;

/* Integration parameters, MpmParams (world.rs:27-49).  `wall_mode` 0 is the
 * reference's separating frictionless walls (world.rs:561-575); 1 selects
 * sticky walls (grid velocity zeroed within one cell of a wall), an extension
 * the reference does not have. */
typedef struct TmpmParams {
    double cell_width;
    double gravity[3];
    double max_substep;
    int32_t has_bounds;
    int32_t wall_mode;
    double bounds_min[3];
    double bounds_max[3];
} TmpmParams;

/* Caller-owned structure-of-arrays view of particles (MpmParticle,
 * world.rs:67-102).  Matrices are 9 doubles per particle in column-major order,
 * as MpmParticleState exposes them (tessera-python3d/src/mpm.rs:253-256).
 * On input, NULL optional arrays mean: force = 0, damping = 0, plastic state =
 * (1, 0, 0) (or hardening 1 for sand materials, world.rs:132-142), enabled = 1,
 * fixed = 0, transfer_color = 0, group_id = 0, chunk_id = 0.  On output (read)
 * every non-NULL array is filled. */
typedef struct TmpmParticleArrays {
    size_t count;
    double *position;        /* count x 3 */
    double *velocity;        /* count x 3 */
    double *deformation;     /* count x 9 */
    double *affine;          /* count x 9 */
    double *force;           /* count x 3, optional */
    double *mass;            /* count */
    double *rest_volume;     /* count */
    double *radius;          /* count */
    double *damping;         /* count, optional */
    double *plastic;         /* count x 3: plastic_det, hardening, log_volume_gain; optional */
    int32_t *material;       /* count, TmpmMaterialKind */
    double *material_params; /* count x 5 */
    uint8_t *enabled;        /* count, optional */
    uint8_t *fixed;          /* count, optional */
    uint16_t *transfer_color;/* count, optional */
    uint32_t *group_id;      /* count, optional */
    uint64_t *chunk_id;      /* count, optional (read only) */
} TmpmParticleArrays;

/* One prescribed rigid obstacle (RigidObstacle, obstacle.rs:79-98). */
typedef struct TmpmObstacle {
    int32_t shape;           /* TmpmObstacleShape */
    int32_t boundary;        /* TmpmBoundary */
    int32_t cpic_group;      /* -1 = none, else 0..31 (triangle prisms only) */
    uint32_t plane_count;    /* convex only */
    double center[3];
    double orientation[4];   /* unit quaternion x, y, z, w (local to world) */
    double linear_velocity[3];
    double angular_velocity[3];
    double friction;
    double dims[3];
    double vertices[9];      /* triangle prism local vertices a, b, c */
    double bound_radius;     /* convex only */
    const double *planes;    /* convex only: plane_count x (nx, ny, nz, offset), local frame */
} TmpmObstacle;

/* Optional session knobs.  Zero-initialised means defaults. */
typedef struct TmpmSessionOptions {
    int32_t device;          /* CUDA device ordinal; default 0 */
    uint32_t max_blocks;     /* block pool capacity per grid; 0 = sized from the scene */
    uint32_t resort_interval;/* substeps between particle re-sorts; 0 = once per submit */
    uint32_t launch_shape;   /* transfer-kernel launch shape: 0 = tuned on the first submits,
                                k > 0 = shape k - 1 of tmpm_launch_shape_info */
    uint64_t next_chunk_id;  /* MpmWorld's next chunk id (world.rs:220); 0 = max(chunk_id) + 1 */
    uint64_t substeps;       /* MpmWorld::substeps of the uploaded world (world.rs:215) */
} TmpmSessionOptions;

typedef struct TmpmSession TmpmSession;

/* ---------------- session lifecycle (GpuMpmResidentSession) ---------------- */

/* GpuMpmResidentSession::new (gpu.rs:253-280): validate (gpu.rs:664-677),
 * pack f64 -> f32, upload and keep device buffers.  `use_cpic` mirrors
 * MpmWorld::use_cpic (world.rs:216-219).  On failure *out is NULL and
 * tmpm_last_error() describes the reason. */
TmpmStatus tmpm_session_create(const TmpmParams *params,
                               const TmpmParticleArrays *particles,
                               const TmpmObstacle *obstacles, size_t obstacle_count,
                               int32_t use_cpic, double substep_dt,
                               const TmpmSessionOptions *options,
                               TmpmSession **out);

/* Drop (gpu.rs:205-216 owns buffers; dropping releases them). */
void tmpm_session_destroy(TmpmSession *session);

/* GpuMpmResidentSession::submit_steps (gpu.rs:303-322): 1..64 substeps queued
 * on the session's stream without waiting. */
TmpmStatus tmpm_submit_steps(TmpmSession *session, uint32_t steps);

/* GpuMpmResidentSession::step (gpu.rs:286-292): submit + synchronize. */
TmpmStatus tmpm_step(TmpmSession *session, uint32_t steps);

/* GpuMpmResidentSession::synchronize (gpu.rs:382-411): wait (5 s limit ->
 * TMPM_ERR_READBACK), check device failure flags, replace the host world only
 * on success.  Any error invalidates the session. */
TmpmStatus tmpm_synchronize(TmpmSession *session);

/* GpuMpmResidentSession::pending_substeps / has_pending_steps (gpu.rs:367-375). */
uint64_t tmpm_pending_substeps(const TmpmSession *session);
int32_t tmpm_has_pending_steps(const TmpmSession *session);

/* MpmWorld::substeps of the last synchronized world (world.rs:215). */
uint64_t tmpm_substeps(const TmpmSession *session);

/* world().particles.len() (gpu.rs:654-656). */
size_t tmpm_particle_count(const TmpmSession *session);

/* world() (gpu.rs:654-656): copy the last synchronized particles into caller
 * arrays.  out->count must equal tmpm_particle_count(). */
TmpmStatus tmpm_read_particles(const TmpmSession *session, TmpmParticleArrays *out);

/* MpmWorld::stable_timestep of the last synchronized world (world.rs:288-303). */
double tmpm_stable_timestep(const TmpmSession *session);

/* GpuMpmResidentSession::set_particle_force (gpu.rs:457-485). */
TmpmStatus tmpm_set_particle_force(TmpmSession *session, size_t index, const double force[3]);

/* GpuMpmResidentSession::set_obstacles (gpu.rs:491-529). */
TmpmStatus tmpm_set_obstacles(TmpmSession *session, const TmpmObstacle *obstacles, size_t count);

/* GpuMpmResidentSession::add_particles (gpu.rs:535-549). */
TmpmStatus tmpm_add_particles(TmpmSession *session, const TmpmParticleArrays *particles,
                              uint64_t *chunk_out);

/* GpuMpmResidentSession::remove_chunk (gpu.rs:553-564). */
TmpmStatus tmpm_remove_chunk(TmpmSession *session, uint64_t chunk, size_t *removed_out);

/* Replace the synchronized world's particles by `particles` (same semantics
 * as the private replace_particle_world, gpu.rs:566-579: validate, re-pack,
 * re-upload; device buffers are reused when they are large enough).  Chunk ids
 * are taken from particles->chunk_id when given. */
TmpmStatus tmpm_write_particles(TmpmSession *session, const TmpmParticleArrays *particles);

/* GpuMpmResidentSession::encode_particle_snapshot (gpu.rs:595-651): write one
 * 32-byte record (position xyz, mass; velocity xyz, rest volume) per particle,
 * in world order, into caller-owned DEVICE memory on the session's stream.
 * Disabled particles get zero mass.  *written = records written. */
TmpmStatus tmpm_encode_particle_snapshot(TmpmSession *session, void *device_out,
                                         size_t capacity_bytes, uint32_t *written);

/* The substep size this session was created with (gpu.rs:359-361). */
double tmpm_substep_dt(const TmpmSession *session);

/* Change the fixed substep of an idle session (the Python binding rebuilds the
 * session when dt changes, mpm.rs:813-832; here buffers are kept and only the
 * CFL validation of gpu.rs:664-677 is repeated). */
TmpmStatus tmpm_set_substep_dt(TmpmSession *session, double substep_dt);

/* ------------- MpmWorld GPU conveniences (gpu.rs:2168-2293) ------------- */

/* MpmWorld::step_with_gpu_transfers (gpu.rs:2208-2240): CFL-limited substeps
 * of total duration dt; each substep validated and synchronized. */
TmpmStatus tmpm_step_cfl(TmpmSession *session, double dt);

/* ---------------- two-way rigid coupling, MPM-owned ----------------
 * GpuRigidMpmCoupler (crates/tessera-mpm/src/gpu_rigid_sync.rs:62-500) in its
 * MPM-owned form (submit_mpm_owned_step / step_mpm_owned, gpu_rigid_sync.rs:
 * 187-214): rigid bodies live on the device beside the session; each coupled
 * substep sets every mapped obstacle's pose and velocity from its body
 * (gpu_rigid_sync.wgsl:46-61), runs one MPM substep accumulating the
 * per-obstacle impulses, and applies them to the bodies: velocity and
 * angular velocity, then gravity, an optional speed limit and the pose
 * integration (gpu_rigid_reaction.wgsl:71-150).  The rigid solver itself
 * (contacts, joints, sleep) belongs to tessera-physics and is not here.  The
 * session's host obstacle list keeps the poses it was given. */
typedef struct TmpmRigidBody {
    double position[3];
    double inverse_mass;       /* <= 0: not moved by impulses */
    double orientation[4];     /* unit quaternion x, y, z, w */
    double linear_velocity[3];
    double angular_velocity[3];
    double inverse_inertia[3]; /* body-frame principal inverse inertia */
} TmpmRigidBody;

typedef struct TmpmRigidMapping {
    int32_t body;              /* body index, or -1: the obstacle keeps its pose */
    int32_t reserved;
    double local_center[3];    /* obstacle centre in the body frame */
    double local_orientation[4];
} TmpmRigidMapping;

/* GpuRigidMpmCoupler::new (gpu_rigid_sync.rs:230-343): bodies and one mapping
 * per session obstacle, in obstacle order.  Replaces an earlier attachment. */
TmpmStatus tmpm_rigid_attach(TmpmSession *session, const TmpmRigidBody *bodies, size_t body_count,
                             const TmpmRigidMapping *mappings, size_t mapping_count);
/* `substeps` (1..64) coupled substeps of the session's substep, then a
 * synchronize.  integrate_pose != 0: step_mpm_owned (gpu_rigid_sync.rs:
 * 202-214), the impulses, gravity and the speed limit change the velocities
 * and the poses advance; 0: step_two_way (gpu_rigid_sync.rs:216-228), only
 * the impulses (and the speed limit) change the velocities, for a rigid
 * solver that integrates the bodies itself.  gravity: the rigid bodies'
 * gravity; max_linear_speed <= 0: no limit.  Needs no pending steps; not
 * with CPIC obstacles (their side masks would use the pose of the substep
 * before). */
TmpmStatus tmpm_rigid_step(TmpmSession *session, uint32_t substeps, const double gravity[3],
                           double max_linear_speed, int32_t integrate_pose);
/* The bodies' current state. */
TmpmStatus tmpm_rigid_read(TmpmSession *session, TmpmRigidBody *bodies, size_t body_count);
void tmpm_rigid_detach(TmpmSession *session);

/* MpmWorld::step_with_gpu_obstacle_reactions (gpu.rs:2247-2293): as
 * tmpm_step_cfl, also returning per-obstacle impulses, 6 doubles each
 * (linear xyz, angular xyz about the obstacle centre), in obstacle order. */
TmpmStatus tmpm_step_cfl_with_reactions(TmpmSession *session, double dt,
                                        double *reactions_out, size_t obstacle_count);

/* ---------------------- allocation-free binning step ---------------------- */

/* No counterpart in the reference.  For callers that must not allocate device
 * memory during a call: a loop with a frame-time budget (an allocation can
 * synchronize the device), a host application that owns every device buffer
 * through its own pool, or code that records work into a CUDA graph.  It runs
 * the binning step of the substep on `count` f32 positions stored
 * component-major on the device (x[0..count), then y and z, `stride` floats
 * apart) and writes, to caller-owned device buffers, the stable order of the
 * particles by their sort key (order_out) and, when
 * keys_out is not NULL, the sorted keys.  The key is the 21-bit Morton code
 * of the particle's 4^3 grid block (block coordinates taken modulo 128)
 * followed by the 6-bit Morton code of its cell inside the block, the key a
 * session's re-sort uses.  `stream` is a cudaStream_t (NULL =
 * the default stream); the call is asynchronous on it.
 * It allocates nothing: its scratch is a fixed array inside the library
 * (4,260,864 bytes, held on every device that loads the library until exit),
 * so `count` is limited to 262,144; larger counts return TMPM_ERR_CAPACITY
 * with the reason in tmpm_last_error().  Set-up: a call made outside a stream
 * capture looks up the scratch address in the current context; a call made
 * during a capture reuses the address of the last call outside one in the
 * same context, so make the first call on a device (and the first after a
 * cudaDeviceReset) before any stream capture.  On entry the call clears any
 * error an earlier CUDA call left unreported (cudaGetLastError), so that
 * only its own launches decide its status.  All calls share the scratch:
 * calls that overlap on the GPU (different streams, or different host
 * threads) race and must be ordered by the caller. */
TmpmStatus tmpm_sort_by_block_noalloc(const float *positions, size_t count, size_t stride,
                                      double cell_width, uint32_t *order_out, uint32_t *keys_out,
                                      void *stream);

/* --------------------------- multi-scene batches --------------------------- */

/* No single counterpart in the reference, which runs one MpmWorld per
 * GpuMpmResidentSession (gpu.rs:206-662).  A batch keeps many independent
 * scenes resident on one device and advances them together: every kernel of a
 * substep is one launch over the particles of all scenes, each scene with its
 * own MpmParams (cell width, gravity, bounds), substep dt and substep count.
 * Per scene the result is the same as a TmpmSession over that scene alone
 * (tmpm_session_create + tmpm_step), within f32 round-off: the transfer
 * arithmetic is the same, only the partition of particles into thread blocks
 * differs.  Limits: 256 live scenes, transfer colours below 256, no obstacles
 * and no per-particle forces.  Each scene is validated like
 * validate_resident_world (gpu.rs:664-677) when it is added. */
typedef struct TmpmBatch TmpmBatch;

typedef struct TmpmBatchOptions {
    int32_t device;            /* CUDA device ordinal */
    uint32_t max_blocks;       /* 0 = size the block pool from the scenes' occupied blocks */
    uint32_t use_graphs;       /* 1 = replay each batch as a CUDA graph (captured once per shape) */
    uint32_t launch_shape;     /* as TmpmSessionOptions::launch_shape */
    uint64_t particle_capacity; /* initial device rows (0 = grow on demand) */
} TmpmBatchOptions;

TmpmStatus tmpm_batch_create(const TmpmBatchOptions *options, TmpmBatch **out);
void tmpm_batch_destroy(TmpmBatch *batch);

/* A scene validated like validate_resident_world (gpu.rs:664-677) and packed
 * into host memory, not yet attached to a batch.  Preparing does no
 * device work and touches no batch, so scenes may be prepared on any thread,
 * also while a batch is in flight. */
typedef struct TmpmPreparedScene TmpmPreparedScene;
TmpmStatus tmpm_scene_prepare(const TmpmParams *params, const TmpmParticleArrays *particles,
                              double substep_dt, TmpmPreparedScene **out);
void tmpm_scene_prepared_destroy(TmpmPreparedScene *prepared);
size_t tmpm_scene_prepared_particle_count(const TmpmPreparedScene *prepared);
/* Device bytes the scene will hold in a batch (admission by footprint). */
size_t tmpm_scene_prepared_bytes(const TmpmPreparedScene *prepared);

/* Attach a prepared scene (the batch takes ownership, also on failure);
 * *scene_out receives its id (0..255).  Allowed while a batch is in flight.
 * When the allocated device rows have room, the rows are copied at once on the
 * batch's upload stream (overlapping the batch in flight; the call returns
 * once the host rows are staged); otherwise at the next submit, which grows
 * the rows first.  The scene joins the next submitted batch either way. */
TmpmStatus tmpm_batch_admit(TmpmBatch *batch, TmpmPreparedScene *prepared, uint32_t *scene_out);

/* tmpm_scene_prepare + tmpm_batch_admit (GpuMpmResidentSession::new for one
 * scene, gpu.rs:253-280). */
TmpmStatus tmpm_batch_add_scene(TmpmBatch *batch, const TmpmParams *params,
                                const TmpmParticleArrays *particles, double substep_dt,
                                uint32_t *scene_out);

/* Retire a scene (allowed while a batch is in flight).  Its device rows are
 * dropped by the next batch's re-sort and its id becomes free then. */
TmpmStatus tmpm_batch_remove_scene(TmpmBatch *batch, uint32_t scene);

/* Queue one batch: scene ids[k] advances steps[k] substeps (1..4096); scenes
 * not listed stay put.  Asynchronous, like submit_steps (gpu.rs:303-322); one
 * batch may be in flight. */
TmpmStatus tmpm_batch_submit(TmpmBatch *batch, const uint32_t *ids, const uint32_t *steps, size_t count);

/* Wait for the batch in flight (bounded, as gpu.rs:1853-1862) and record each
 * scene's outcome.  A scene whose resident checks failed (CFL, escape,
 * ill-conditioned F, unprojectable plastic state) is marked failed with
 * TMPM_ERR_RESIDENT_UNAVAILABLE and keeps its last read state; the other
 * scenes are unaffected.  Block-pool or hash-table overflow fails the batch. */
TmpmStatus tmpm_batch_synchronize(TmpmBatch *batch);
int32_t tmpm_batch_pending(const TmpmBatch *batch);

/* Per-scene state: outcome (TMPM_OK or the failure), completed substeps,
 * particle count, and the particles themselves (like world() after
 * synchronize, gpu.rs:654-661).  Reading a scene that the batch in flight does
 * not advance runs concurrently with that batch; a scene in the batch in
 * flight returns TMPM_ERR_PENDING_STEPS. */
TmpmStatus tmpm_batch_scene_status(const TmpmBatch *batch, uint32_t scene);
uint64_t tmpm_batch_scene_substeps(const TmpmBatch *batch, uint32_t scene);
size_t tmpm_batch_scene_particle_count(const TmpmBatch *batch, uint32_t scene);
TmpmStatus tmpm_batch_read_scene(TmpmBatch *batch, uint32_t scene, TmpmParticleArrays *out);

/* Read + remove in one call, for retiring a finished scene: the non-null
 * fields of `out` receive the scene's state (as tmpm_batch_read_scene would
 * return it) and the scene leaves the batch.  Only the requested per-particle
 * fields are copied from the device, and the scene's host world is not
 * brought up to date first, since the scene goes; the non-finite check of
 * collect_prepared (gpu.rs:1940-1989) still covers every transferred field.
 * A non-finite state fails the scene and keeps it, as a read does. */
TmpmStatus tmpm_batch_take_scene(TmpmBatch *batch, uint32_t scene, TmpmParticleArrays *out);

/* Device milliseconds of the last synchronized batch (CUDA events on the
 * batch stream around its kernels). */
double tmpm_batch_last_ms(const TmpmBatch *batch);

/* Device bytes held by the batch, and the bytes a scene of `particles`
 * particles over `home_blocks` occupied 4^3 blocks adds (admission control). */
size_t tmpm_batch_device_bytes(const TmpmBatch *batch);
size_t tmpm_batch_scene_bytes(size_t particles, size_t home_blocks);

const char *tmpm_batch_last_error_message(const TmpmBatch *batch);

/* ------------------------- differentiable rollout ------------------------- */

/* No counterpart in the reference (tessera-mpm has no adjoint).  A rollout of
 * `substeps` fixed substeps of MpmWorld::substep (world.rs:361-467) for
 * corotated elastic particles (material.rs:440-455) in a bounded domain, and
 * its hand-written adjoint: gradients of a loss on the final positions and
 * velocities with respect to the initial velocities and the per-particle
 * Young's moduli.  The forward stores the state every `checkpoint_every`
 * substeps; the backward replays each segment from its checkpoint.  All
 * arrays are host f64: 3 per particle for vectors, 1 for Young's modulus, in
 * the particle order given at creation. */
typedef struct TmpmAdjoint TmpmAdjoint;

TmpmStatus tmpm_adjoint_create(const TmpmParams *params, const TmpmParticleArrays *particles,
                               double substep_dt, uint32_t substeps, uint32_t checkpoint_every,
                               int32_t device, TmpmAdjoint **out);
void tmpm_adjoint_destroy(TmpmAdjoint *adjoint);
size_t tmpm_adjoint_particle_count(const TmpmAdjoint *adjoint);

/* Run the rollout from the creation state with the given initial velocities
 * and Young's moduli (NULL keeps the creation values); writes the final
 * positions and velocities (either may be NULL). */
TmpmStatus tmpm_adjoint_forward(TmpmAdjoint *adjoint, const double *velocity0, const double *young,
                                double *position_out, double *velocity_out);

/* Adjoint of the last forward: given dL/dx_T and dL/dv_T (NULL = zero),
 * writes dL/dv_0 and dL/dE (either may be NULL). */
TmpmStatus tmpm_adjoint_backward(TmpmAdjoint *adjoint, const double *position_grad,
                                 const double *velocity_grad, double *velocity0_grad,
                                 double *young_grad);

const char *tmpm_adjoint_last_error_message(const TmpmAdjoint *adjoint);

/* ------------------------------ diagnostics ------------------------------ */

/* Human-readable reason for the last failed call on this session. */
const char *tmpm_last_error_message(const TmpmSession *session);

/* Reason for the last failed session-less call on this thread. */
const char *tmpm_last_error(void);

/* Library version string. */
const char *tmpm_version(void);

/* Binning view of the device state (no reference counterpart; test hook).
 * Re-bins the current device particles exactly as a substep does and returns,
 * in DEVICE STORAGE order: the world index of each stored particle, its f32
 * base cell (3 ints) and its sort key.  Arrays hold tmpm_device_count() items. */
size_t tmpm_device_count(const TmpmSession *session);
TmpmStatus tmpm_debug_binning(TmpmSession *session, uint32_t *world_index_out,
                              int32_t *base_cell_out, uint32_t *key_out);

/* Grid view (test hook): run only P2G on the current device state with the
 * session's substep and return every node with non-zero mass: cell (3 ints per
 * node), mass and momentum (4 floats per node), plus the node count.  Arrays
 * must hold `capacity` nodes; *count receives the total. */
TmpmStatus tmpm_debug_p2g(TmpmSession *session, int32_t *cells_out, float *mass_momentum_out,
                          size_t capacity, size_t *count);

/* Kernel timing (bench hook): time `steps` substeps of the resident path on the
 * session stream with CUDA events; returns milliseconds via *ms (host waits
 * between submissions included).  The substeps go in submissions of at most 64,
 * each waited for before the next, as a caller stepping frame by frame runs
 * them.  Per-kernel averages (ms per launch) go to kernel_ms[0..n) in the order
 * p2g, grid, g2p2g, g2p, resort when kernel_ms is non-NULL. */
TmpmStatus tmpm_bench_substeps(TmpmSession *session, uint32_t steps, double *ms,
                               double *kernel_ms, size_t kernel_count);

/* ---------------- launch-shape tuning (no reference counterpart) ----------------
 * The transfer kernels (G2P, P2G and the fused G2P2G) and the grid update are
 * built for several launch shapes: particles per CTA, CTAs resident per SM,
 * and the edge of the sparse grid's blocks (4 or 8 cells).  Unless the options
 * fix one, a session or batch runs its first submitted segments under each
 * shape in turn (two rounds, real work; results differ between shapes only by
 * f32 summation order) and keeps the one with the least device time per
 * particle-substep, as CUDA events on its stream measured it.  8-cell blocks
 * are tried when the block pool holds the scene in them at most twice the
 * 4-cell pool's size (dense scenes).  Plastic materials and CPIC run shape 0
 * only.  A session keeps timing its full segments after the choice, because a
 * scene's best shape can change as it evolves: every sixth such segment runs
 * the best other shape by its latest time, which takes over when it beat the
 * chosen shape's recent mean by more than 1 %.  The times are read when later
 * segments are submitted, so a caller that submits one frame at a time (and
 * waits for it) gets the switch within a segment or two; a batch keeps its
 * first choice. */

/* Shape `shape` (0 ..< count): particles per CTA, CTAs per SM, block edge in cells. */
uint32_t tmpm_launch_shape_count(void);
TmpmStatus tmpm_launch_shape_info(uint32_t shape, uint32_t *threads_per_cta, uint32_t *ctas_per_sm,
                                  uint32_t *block_edge);

/* The shape in use: -1 while trials are outstanding, else its index.  When
 * `ms_per_unit` is non-NULL, it receives (up to `count` entries) the latest
 * measured milliseconds per particle-substep of each shape (infinity where no
 * trial has been read). */
int32_t tmpm_session_launch_shape(TmpmSession *session, double *ms_per_unit, size_t count);
int32_t tmpm_batch_launch_shape(TmpmBatch *batch, double *ms_per_unit, size_t count);

#ifdef __cplusplus
}
#endif

#endif /* TMPM_H */
