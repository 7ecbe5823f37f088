// tmpm_internal.h -- device data layout shared by the kernels and the host session.
//
// HBM layout (one session, one GPU):
//   * particles: structure of arrays in f32, component-major (x[c * cap + i]),
//     kept in "storage order" = sorted by the Morton key of each particle's 4^3
//     grid block, re-sorted at the start of every submitted batch;
//   * particle classes: one 48-byte record per distinct (material, mass, volume,
//     radius, damping, transfer colour) tuple, indexed by a u32 per particle;
//   * two sparse grids (ping-pong, step n and n+1), each an open-addressing hash
//     table of 4^3 blocks (64-bit key -> u32 block id) plus a block pool of
//     64 float4 nodes (mass, momentum xyz -> velocity xyz after the grid update).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

namespace tmpm {

constexpr int kBlockShift = 2;  // 4^3 cells per grid block (the default block edge)
constexpr int kNodesPerBlock = 64;
constexpr int kBigBlockShift = 3;  // 8^3 cells per grid block (a tuner candidate)
constexpr int kBigNodesPerBlock = 512;
constexpr unsigned long long kEmptyKey = ~0ull;
constexpr uint32_t kPendingId = 0xFFFFFFFFu;
constexpr uint32_t kInvalidId = 0xFFFFFFFEu;
constexpr int kBlockBias = 32768;      // block coordinate bias inside the 64-bit key
constexpr int kBlockCoordMin = -32767; // representable block coordinates
constexpr int kBlockCoordMax = 32766;
constexpr int kMaxProbe = 4096;        // hash probe limit before reporting Capacity
constexpr int kSpinLimit = 1 << 20;    // bounded wait for a block id to be published

// Device status word bits (or-ed by kernels, read by synchronize).
constexpr uint32_t kStatusResident = 1u;  // CFL, escape, irregular F, non-finite -> ResidentUnavailable
constexpr uint32_t kStatusCapacity = 2u;  // hash table or block pool exhausted -> Capacity
constexpr uint32_t kStatusTimeout = 4u;   // a bounded device wait gave up -> Readback

// GPU material codes (the reference shader's codes, gpu.rs:1171-1276).
constexpr int kMatNeoHookean = 1;
constexpr int kMatFluid = 2;
constexpr int kMatCorotated = 3;
constexpr int kMatSnow = 4;
constexpr int kMatSand = 5;
constexpr int kMatSandNeoHookean = 6;

#ifndef TMPM_TRANSFER_MIN_BLOCKS
#define TMPM_TRANSFER_MIN_BLOCKS 4  // CTAs per SM of the default transfer launch shape (measured best of 2-6)
#endif
// Launch shapes of the transfer kernels the tuner chooses among (particles per
// CTA, CTAs per SM the kernel is compiled for); shape 0 is the default and the
// only one for plastic and CPIC variants.
struct LaunchShape {
    int threads, min_blocks;
};
constexpr LaunchShape kLaunchShapes[] = {{256, TMPM_TRANSFER_MIN_BLOCKS}, {128, 8}, {256, 3}};
constexpr int kNumLaunchShapes = 3;
// Launch configurations: a shape and a grid block edge.  Configuration c runs
// shape c % kNumLaunchShapes on 4^3 blocks for c < kNumLaunchShapes, on 8^3
// blocks above.
constexpr int kNumLaunchConfigs = 2 * kNumLaunchShapes;
constexpr int config_shape(int c) { return c % kNumLaunchShapes; }
constexpr int config_block_shift(int c) { return c < kNumLaunchShapes ? kBlockShift : kBigBlockShift; }
constexpr int kMinTransferThreads = 128;  // per-CTA records are sized for the smallest shape
constexpr int kCacheStride = 144;      // per-CTA record: 16-int box header + up to 128 block ids

constexpr uint32_t kFixedBit = 0x80000000u;
constexpr uint32_t kClassMask = 0x7FFFFFFFu;

struct DevClass {
    float mass, volume, radius, damping;
    // corotated / NH: lambda, mu; fluid: bulk, gamma, viscosity, tensile;
    // sand / NH sand: lambda, mu, friction angle, cohesion;
    // snow: lambda, mu, hardening, critical compression, critical stretch (p4)
    float p0, p1, p2, p3;
    int32_t kind;          // kMat*
    float wave;            // CFL wave speed sqrt((lambda + 2 mu) / rho) or sqrt(K gamma / rho)
    uint32_t color;        // grid namespace: the transfer colour; in a multi-scene batch (scene << 8) | colour
    float p4;
};
static_assert(sizeof(DevClass) == 48, "DevClass layout");

// Per-scene integration parameters (MpmParams + the fixed substep), one entry
// per scene of a batch; a single-scene session has one entry.
struct SceneParams {
    float h, inv_h, inv_d, dt;
    float gx, gy, gz;
    int has_bounds;
    float bmin[3];
    int wall_mode;
    float bmax[3];
    int steps;                        // substeps this scene advances in the current batch
    int first_base[3];                // escape window of base cells (bounded worlds)
    int live;                         // 0 = removed: dropped by the next re-sort
    int last_base[3], pad;
    // Wall nodes (bounded worlds): node index i lies within one cell of the
    // lower wall of axis a when i <= wall_lo[a], of the upper wall when
    // i >= wall_hi[a].  The host derives both from the f64 comparisons of
    // apply_grid_boundary (world.rs:561-575), so a node exactly one cell from
    // a wall is classified as the f64 reference classifies it.
    int wall_lo[3], wall_hi[3];
};
static_assert(sizeof(SceneParams) == 120, "SceneParams layout");

struct DevObstacle {
    int32_t shape, boundary, cpic_group, plane_offset;
    int32_t plane_count, pad0, pad1, pad2;
    float center[4];    // xyz, bound (triangle prism / convex bounding radius)
    float q[4];         // x, y, z, w
    float lin[4];       // xyz, friction
    float ang[4];
    float dims[4];
    float verts[12];    // a, b, c (xyz + pad)
    // Local-frame box that holds the whole surface: |x| <= reach[0],
    // |y| <= reach[1], |z| <= reach[2]; reach[3] = 1 drops the lower z bound
    // (the ground, a half-space below its plane).  A point whose local
    // coordinates lie farther than a particle radius outside it cannot touch
    // the obstacle (obstacle_near).
    float reach[4];
};

// Rigid body of the two-way coupling (the reference's RigidState layout,
// gpu_rigid_reaction.wgsl:1-7): position | inverse mass, orientation (x, y, z,
// w), linear and angular velocity, body-frame inverse inertia | awake flag.
struct DevRigid {
    float4 pos_inv_mass;
    float4 q;
    float4 lin;
    float4 ang;
    float4 inv_inertia;
};
static_assert(sizeof(DevRigid) == 80, "DevRigid layout");

// Obstacle -> body mapping (gpu_rigid_sync.wgsl:21-25): body index (< 0: the
// obstacle keeps its pose), the obstacle's centre and orientation in the body frame.
struct DevRigidMap {
    int body;
    int pad[3];
    float4 local_center;
    float4 local_q;
};

struct RigidParams {
    float dt;
    float gravity[3];
    float max_speed;  // <= 0: no limit
    int integrate_pose;
};

struct GridTable {
    unsigned long long *keys;  // [capacity]
    uint32_t *vals;            // [capacity]
    uint32_t *count;           // allocated blocks
    float4 *pool;              // [max_blocks * 64]
    int4 *coords;              // [max_blocks]: bx, by, bz, colour
    uint32_t mask;             // capacity - 1
    uint32_t max_blocks;
};

// Grid namespace of a particle class in a multi-scene batch: scene << kSceneShift | colour.
constexpr int kSceneShift = 8;
constexpr int kMaxScenes = 256;   // scenes per batch (16-bit namespace field of the block key)
constexpr int kMaxBatchColors = 256;
constexpr int kSortBitsScene = 27;            // single scene: 21-bit block Morton key << 6 | cell in block
#ifndef TMPM_RESORT_SUBSTEPS
#define TMPM_RESORT_SUBSTEPS 64
#endif
constexpr uint32_t kResortSubsteps = TMPM_RESORT_SUBSTEPS;  // default substeps between re-sorts of a session
constexpr int kSortBitsBatch = 30;            // batch: scene << 21 | Morton, plus the removed-scene bit
constexpr uint32_t kDeadKey = 0x3FFFFFFFu;

struct SimParams {
    SceneParams s0;             // the scene of a single-scene session (kernel parameter, constant bank)
    const SceneParams *scenes;  // multi-scene batch: device scene table, indexed by namespace >> kSceneShift
    uint32_t *scene_status;     // multi-scene batch: per-scene resident failure flags
    // One scene: the fused transfer's deferred-chunk lists (layout at
    // DeferLists); null: every transfer takes the general kernel.
    uint32_t *defer;
    int multi;                  // 1 = multi-scene batch (per-particle scene lookup and step gating)
    int step_index;             // substep completed by this launch's G2P (-1 for the opening P2G)
    int num_obstacles;
    int reactions;
    int apply_force;
    int resident_checks;  // CFL / escape / conditioning flags (resident path only, gpu.rs:1429)
    int has_plastic;      // some particle class is snow, sand or NH sand
    int cpic;             // CPIC on: grid namespace = colour << 8 | side mask of the CPIC groups (< 8)
    int shape;            // transfer launch shape (index into kLaunchShapes)
    int block_shift;      // log2 of the grid block edge: kBlockShift (4^3) or kBigBlockShift (8^3)
    int defer_cap;        // entries per deferred-chunk list (transfer chunks of the smallest CTA)
    int pad_;
};
// The session's graph cache keys segments by the bytes of a SimParams: neither
// it nor SceneParams may hold padding, whose contents would be indeterminate.
static_assert(sizeof(SimParams) == sizeof(SceneParams) + 3 * sizeof(void *) + 12 * sizeof(int),
              "SimParams must have no padding bytes");

// Deferred-chunk lists of the fast fused transfer, in one device buffer of
// kDeferHeader + 4 * cap words: counts [0] P2G-only, [1] whole chunk,
// [2 + p] no record for a launch of step parity p; then the lists in that
// order (cap entries each).
constexpr int kDeferHeader = 8;
inline size_t defer_words(size_t cap) { return kDeferHeader + 4 * cap; }
static_assert(sizeof(SceneParams) == 30 * sizeof(float), "SceneParams must have no padding bytes");
constexpr int kMaxCpicGroups = 8;

struct ParticleSoA {
    float *x;       // 3 * cap
    float *v;       // 3 * cap
    float *C;       // 9 * cap, column-major components (col * 3 + row)
    float *F;       // 9 * cap
    float *pl;      // 3 * cap: plastic_det, hardening, log_volume_gain (plastic materials only)
    float *force;   // 3 * force_stride, indexed by WORLD index (one-shot forces)
    uint32_t *cls;  // class index | kFixedBit
    uint32_t *widx; // world index of each stored particle
    size_t cap;
    size_t force_stride;
};

struct SortBuffers {
    uint32_t *keys[2];
    uint32_t *vals[2];
    uint32_t *hist;    // 256 * tiles
    uint32_t *totals;  // 256
    size_t cap;
};

enum TransferMode { kModeP2G = 0, kModeG2P2G = 1, kModeG2P = 2 };

// A second stream and two events, for launches that fork work off `stream`
// and join it back (the fused transfer's deferred chunks).
struct ForkJoin {
    cudaStream_t side;
    cudaEvent_t fork, join;
};

// Launchers (tmpm_kernels.cu).  All run on `stream`.
// `cur` and `next` share one hash table (block ids are stable within a batch)
// and differ in their node pools; `cache` holds kCacheStride ints per CTA.
// With `fj`, sp.defer set and no CPIC (and, in a multi-scene batch, no
// plastic state), the fused transfer
// (kModeG2P2G) runs as the fast kernel beside the chunks without a record
// (on fj->side) and then the chunks the fast kernel deferred; the grid update
// before it must carry the same step_index.
void launch_transfer(int mode, const ParticleSoA &P, int n, const DevClass *classes, const GridTable &cur,
                     const GridTable &next, const SimParams &sp, const DevObstacle *obstacles,
                     const float *planes, double *reactions, uint32_t *status, int *cache, cudaStream_t stream,
                     const ForkJoin *fj = nullptr);
// Grid update of `g`'s pool; also zeroes the same blocks in `next`'s pool.
void launch_grid_update(const GridTable &g, const GridTable &next, const SimParams &sp,
                        const DevObstacle *obstacles, const float *planes, double *reactions,
                        uint32_t *status, cudaStream_t stream);
// Two-way rigid coupling: obstacle poses from their bodies; obstacle impulses
// (6 doubles per obstacle) applied to the bodies.
void launch_rigid_sync(const DevRigid *bodies, const DevRigidMap *maps, int obstacle_count, DevObstacle *obstacles,
                       cudaStream_t stream);
void launch_rigid_apply(DevRigid *bodies, int body_count, const DevRigidMap *maps, int obstacle_count,
                        const DevObstacle *obstacles, const double *reactions, const RigidParams &p,
                        cudaStream_t stream);

// Load the kernels of every tuner candidate (transfer modes x launch shapes x
// block edges, grid update) for the multi-scene variant or the single-scene one
// with or without obstacles, so that no trial pays a kernel's lazy module load.
void preload_launch_shapes(bool multi, bool obstacles);

// Empty the hash table of `g` and zero both node pools (g's and other's) over
// g.max_blocks blocks of edge 2^block_shift.
void launch_clear_table(const GridTable &g, const GridTable &other, int block_shift, cudaStream_t stream);
// Re-sort by block key into `dst`; particles of removed scenes sort last and the
// first `keep` particles are gathered.
void launch_resort(ParticleSoA &src, ParticleSoA &dst, int n, int keep, const DevClass *classes, const SimParams &sp,
                   SortBuffers &sb, cudaStream_t stream);
void launch_bin_keys(const ParticleSoA &P, int n, const DevClass *classes, const SimParams &sp, int32_t *cells,
                     uint32_t *keys, cudaStream_t stream);
// Morton block keys (and identity values) of `n` positions stored component-major with `stride`.
void launch_bin_keys_values(const float *x, size_t stride, int n, float inv_h, uint32_t *keys, uint32_t *vals,
                            cudaStream_t stream);
void launch_dump_grid(const GridTable &g, int32_t *cells, float4 *values, uint32_t *count, uint32_t capacity,
                      int block_shift, cudaStream_t stream);
void launch_snapshot(const ParticleSoA &P, int n, const DevClass *classes, float4 *out, cudaStream_t stream);
// 27 f32 rows (x, v, C, F, plastic) of the stored particles into world order, `stride` floats per row.
// Rows in world order: out[c * stride + widx[j]] = component c of stored row j
// (27 f32 components: x, v, C, F, plastic); `nonfinite`, when given, gets bit 0
// set if any of them is not finite.
void launch_unsort(const ParticleSoA &P, int n, float *out, size_t stride, cudaStream_t stream,
                   uint32_t *nonfinite = nullptr);
int device_sm_count();

// Thread-local reason reported by tmpm_last_error() (tmpm_session.cu).
void set_last_error(const std::string &msg);

// Radix sort (tmpm_sort.cu): stable sort of (key, value) pairs by `bits` low key
// bits, 8 bits per pass.  Returns r: the result is in sb.keys[r] / sb.vals[r].
int radix_sort_pairs(SortBuffers &sb, int n, int bits, cudaStream_t stream);

}  // namespace tmpm
