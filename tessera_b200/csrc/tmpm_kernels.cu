// tmpm_kernels.cu -- the MLS-MPM substep on sm_100a.
//
// One substep n of the resident path is two kernels:
//   k_grid(n):      v = p / m + g dt, walls, obstacles, reactions
//                   (world.rs:401-417, gpu.wgsl:772-819 / 1056-1108)
//   k_transfer(n):  G2P of step n fused with P2G of step n+1
//                   (world.rs:419-464 then 378-399; gpu.wgsl:821-1019, 711-770)
// A batch opens with a P2G-only transfer and closes with a G2P-only transfer,
// which alone writes velocity and the affine matrix back to HBM.
//
// Each CTA owns a chunk of consecutive particles in storage order (sorted by
// block and cell; 256 or 128 per chunk, the launch shape's CTA size, see
// kLaunchShapes; grid blocks of 4^3 or 8^3 cells, the template parameter BS).
// It stages the grid nodes its particles touch in a shared-memory
// box ("tile"): the gather tile holds step-n velocities, the scatter tile
// accumulates step-(n+1) mass and momentum with shared atomics and is flushed
// to the block pool with one float4 atomic per touched node.  Chunks whose box
// is too large (scattered particles) fall back to per-node global access.
//
// In a session the fused transfer of one scene runs as k_transfer_fast (the
// common path only) with k_transfer_deferred beside and after it for the
// chunks the common path does not cover (see transfer_chunk).

#include <climits>

#include "tmpm_device.cuh"


namespace tmpm {

namespace {

// Box edge in cells: only bounds the arithmetic (a padded entry count far
// inside int range); the entry and block counts decide whether a box fits.
// An elongated box (a chunk that wraps from one row of blocks to the next
// in storage order) fits when its volume does.
constexpr int kTileMaxDim = 64;
// Box nodes a CTA of `threads` particles stages: 9 per particle (2304 nodes,
// one 36 KB shared buffer, for 256; the most that keeps the static shared
// memory of the variants with the obstacle contact under 48 KB), used as the
// gather tile and then as the scatter tile.  Every transfer kernel stages the
// same box size, since a record one kernel writes is read by another.  On the
// evolved dam break 1.5 % of the chunks have boxes above 2048 entries and
// 1.0 % above 2304; those take the direct path (fused launch 0.428 -> 0.421 ms
// with the larger tile).
constexpr int tile_nodes(int threads) { return threads * 9; }
constexpr int kMaxTileBlocks = kCacheStride - 16;
constexpr int kCacheHeader = 16;
constexpr uint32_t kFatal = kStatusCapacity | kStatusTimeout | kStatusResident;

struct Box {
    int lo[3];
    int dim[3];
    int blo[3];
    int nb[3];
    int nodes;  // tile entries: dim[0] * s1
    int nbt;
    int ok;
    uint32_t color;
    int s1, s2;  // tile strides of x and y (z: 1)
};

// Tile strides padded against shared-memory bank conflicts.  The 32 lanes of
// a warp hold particles of 32 neighbouring cells (with 8 per cell, a 2 x 4 x 4
// group in the chunk's cell Morton order, see lane_cell); with a y stride of
// 4 mod 8 and an x stride of 16 mod 32 their tile entries x * 16 + y * 4 + z
// are distinct mod 32, so a scatter atomic of the warp touches 32 banks and a
// gather load of a quarter-warp (a 1 x 2 x 4 slab) 8 distinct bank groups.
// Measured on the dam break: 2.24 -> 1.35 wavefronts per shared atomic.
__device__ __forceinline__ void tile_strides(int d1, int d2, int &s1, int &s2) {
    s2 = d2 + ((4 - d2) & 7);
    s1 = d1 * s2;
    s1 += (16 - s1) & 31;
}

// Split a padded tile index t (strides s1, s2; t < 2^20) into (tx, ty, tz)
// without integer division (the float reciprocal is exact here, see Split3).
struct SplitP {
    int s1, s2;
    float inv_s1, inv_s2;
    __device__ __forceinline__ SplitP(int s1_, int s2_)
        : s1(s1_), s2(s2_), inv_s1(1.0f / static_cast<float>(s1_)), inv_s2(1.0f / static_cast<float>(s2_)) {}
    __device__ __forceinline__ void operator()(int t, int &tx, int &ty, int &tz) const {
        tx = static_cast<int>((static_cast<float>(t) + 0.5f) * inv_s1);
        const int r = t - tx * s1;
        ty = static_cast<int>((static_cast<float>(r) + 0.5f) * inv_s2);
        tz = r - ty * s2;
    }
};

// Node index inside its block of edge 2^BS cells (x-major).
template <int BS>
__device__ __forceinline__ int node_local(int cx, int cy, int cz) {
    constexpr int m = (1 << BS) - 1;
    return ((cx & m) << (2 * BS)) | ((cy & m) << BS) | (cz & m);
}

// Split a row-major tile index t (dims d0 x d1 x d2, t < 2^20) into (tx, ty, tz)
// without integer division: (t + 0.5) / d lies at least 1 / (2 d) from an
// integer, far above the f32 error of (t + 0.5) * (1 / d), so truncation is exact.
struct Split3 {
    int d1, d2;
    float inv_d1, inv_d2;
    __device__ __forceinline__ Split3(int d1_, int d2_)
        : d1(d1_), d2(d2_), inv_d1(1.0f / static_cast<float>(d1_)), inv_d2(1.0f / static_cast<float>(d2_)) {}
    __device__ __forceinline__ void operator()(int t, int &tx, int &ty, int &tz) const {
        const int q = static_cast<int>((static_cast<float>(t) + 0.5f) * inv_d2);
        tz = t - q * d2;
        tx = static_cast<int>((static_cast<float>(q) + 0.5f) * inv_d1);
        ty = q - tx * d1;
    }
};

// Block-wide min/max of base cells and colours; thread 0 fills `box`.
template <int THREADS, int BS>
__device__ __forceinline__ void reduce_box(bool valid, const int b[3], uint32_t color, int (*red)[8], Box &box) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int vals[8];
    for (int a = 0; a < 3; ++a) {
        vals[a] = valid ? b[a] : INT_MAX;
        vals[3 + a] = valid ? b[a] : INT_MIN;
    }
    vals[6] = valid ? static_cast<int>(color) : INT_MAX;
    vals[7] = valid ? static_cast<int>(color) : INT_MIN;
    int r[8];
    for (int a = 0; a < 3; ++a) r[a] = __reduce_min_sync(0xffffffffu, vals[a]);
    for (int a = 3; a < 6; ++a) r[a] = __reduce_max_sync(0xffffffffu, vals[a]);
    r[6] = __reduce_min_sync(0xffffffffu, vals[6]);
    r[7] = __reduce_max_sync(0xffffffffu, vals[7]);
    if (lane == 0)
        for (int a = 0; a < 8; ++a) red[warp][a] = r[a];
    __syncthreads();
    if (threadIdx.x == 0) {
        int m[8];
        for (int a = 0; a < 8; ++a) m[a] = red[0][a];
        for (int w = 1; w < THREADS / 32; ++w) {
            for (int a = 0; a < 3; ++a) m[a] = min(m[a], red[w][a]);
            for (int a = 3; a < 6; ++a) m[a] = max(m[a], red[w][a]);
            m[6] = min(m[6], red[w][6]);
            m[7] = max(m[7], red[w][7]);
        }
        bool any = m[0] <= m[3];
        int nodes = 1, nbt = 1;
        bool ok = any && m[6] == m[7];
        for (int a = 0; a < 3 && ok; ++a) {
            long long d = static_cast<long long>(m[3 + a]) - m[a] + 3;
            if (d > kTileMaxDim) ok = false;
        }
        if (ok) {
            for (int a = 0; a < 3; ++a) {
                box.lo[a] = m[a];
                box.dim[a] = m[3 + a] - m[a] + 3;
                box.blo[a] = m[a] >> BS;
                box.nb[a] = ((m[3 + a] + 2) >> BS) - box.blo[a] + 1;
                nodes *= box.dim[a];
                nbt *= box.nb[a];
            }
            int s1 = 0, s2 = 0;
            tile_strides(box.dim[1], box.dim[2], s1, s2);
            box.s1 = s1;
            box.s2 = s2;
            nodes = box.dim[0] * s1;
            ok = nodes <= tile_nodes(THREADS) && nbt <= kMaxTileBlocks;
        }
        box.nodes = nodes;
        box.nbt = nbt;
        box.ok = ok ? 1 : 0;
        box.color = static_cast<uint32_t>(m[6]);
    }
    __syncthreads();
}

// Box of base cells and colours plus the sums and maxima of two non-negative
// floats over the CTA, with one barrier: each warp reduces its lanes and
// publishes a partial, then every warp combines the partials itself (no second
// barrier, no shared result).  The maxima are taken on the float bits, whose
// integer order is the value order for non-negative floats.
template <int THREADS, int BS>
__device__ __forceinline__ void reduce_box_sums(bool valid, const int b[3], uint32_t color, float &sum_a, float &sum_b,
                                                float &max_a, float &max_b, int (*red)[8], float (*redf)[4],
                                                Box &box) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int r[8];
    for (int a = 0; a < 3; ++a) {
        r[a] = __reduce_min_sync(0xffffffffu, valid ? b[a] : INT_MAX);
        r[3 + a] = __reduce_max_sync(0xffffffffu, valid ? b[a] : INT_MIN);
    }
    r[6] = __reduce_min_sync(0xffffffffu, valid ? static_cast<int>(color) : INT_MAX);
    r[7] = __reduce_max_sync(0xffffffffu, valid ? static_cast<int>(color) : INT_MIN);
    float fa = sum_a, fb = sum_b;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        fa += __shfl_xor_sync(0xffffffffu, fa, off);
        fb += __shfl_xor_sync(0xffffffffu, fb, off);
    }
    const unsigned ma = __reduce_max_sync(0xffffffffu, __float_as_uint(max_a));
    const unsigned mb = __reduce_max_sync(0xffffffffu, __float_as_uint(max_b));
    if (lane == 0) {
        for (int a = 0; a < 8; ++a) red[warp][a] = r[a];
        redf[warp][0] = fa;
        redf[warp][1] = fb;
        redf[warp][2] = __uint_as_float(ma);
        redf[warp][3] = __uint_as_float(mb);
    }
    __syncthreads();
    constexpr int kWarps = THREADS / 32;
    const bool mine = lane < kWarps;
    int m[8];
    for (int a = 0; a < 3; ++a) {
        m[a] = __reduce_min_sync(0xffffffffu, mine ? red[lane][a] : INT_MAX);
        m[3 + a] = __reduce_max_sync(0xffffffffu, mine ? red[lane][3 + a] : INT_MIN);
    }
    m[6] = __reduce_min_sync(0xffffffffu, mine ? red[lane][6] : INT_MAX);
    m[7] = __reduce_max_sync(0xffffffffu, mine ? red[lane][7] : INT_MIN);
    fa = mine ? redf[lane][0] : 0.0f;
    fb = mine ? redf[lane][1] : 0.0f;
    max_a = __uint_as_float(__reduce_max_sync(0xffffffffu, mine ? __float_as_uint(redf[lane][2]) : 0u));
    max_b = __uint_as_float(__reduce_max_sync(0xffffffffu, mine ? __float_as_uint(redf[lane][3]) : 0u));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        fa += __shfl_xor_sync(0xffffffffu, fa, off);
        fb += __shfl_xor_sync(0xffffffffu, fb, off);
    }
    sum_a = fa;
    sum_b = fb;
    bool ok = m[0] <= m[3] && m[6] == m[7];
    int nodes = m[0] <= m[3] ? 1 : 0, nbt = 1;  // nodes 0: no valid particle
    for (int a = 0; a < 3 && ok; ++a)
        if (static_cast<long long>(m[3 + a]) - m[a] + 3 > kTileMaxDim) ok = false;
    if (ok) {
        for (int a = 0; a < 3; ++a) {
            box.lo[a] = m[a];
            box.dim[a] = m[3 + a] - m[a] + 3;
            box.blo[a] = m[a] >> BS;
            box.nb[a] = ((m[3 + a] + 2) >> BS) - box.blo[a] + 1;
            nodes *= box.dim[a];
            nbt *= box.nb[a];
        }
        tile_strides(box.dim[1], box.dim[2], box.s1, box.s2);
        nodes = box.dim[0] * box.s1;
        ok = nodes <= tile_nodes(THREADS) && nbt <= kMaxTileBlocks;
    }
    box.nodes = nodes;
    box.nbt = nbt;
    box.ok = ok ? 1 : 0;
    box.color = static_cast<uint32_t>(m[6]);
}

// A CTA in which one particle's mass or momentum bound exceeds this share of
// the CTA's total scatters through the direct path (f32 global atomics per
// node, each node accurate relative to its own magnitude): its fixed-point
// scale would be set by that particle alone and would coarsen the quantum of
// every node its neighbours reach.
constexpr float kFloatModeShare = 1.0f / 8.0f;

__device__ __forceinline__ void quad_weights(float f, float w[3]) {
    w[0] = 0.5f * (1.5f - f) * (1.5f - f);
    w[1] = 0.75f - (f - 1.0f) * (f - 1.0f);
    w[2] = 0.5f * (f - 0.5f) * (f - 0.5f);
}

template <int BS>
__device__ __forceinline__ int tile_block_index(const Box &bx, int cx, int cy, int cz) {
    return (((cx >> BS) - bx.blo[0]) * bx.nb[1] + ((cy >> BS) - bx.blo[1])) * bx.nb[2] + ((cz >> BS) - bx.blo[2]);
}

__device__ __forceinline__ M3f load_m3(const float *base, size_t cap, int i) {
    M3f m;
    m.c0 = mk(base[0 * cap + i], base[1 * cap + i], base[2 * cap + i]);
    m.c1 = mk(base[3 * cap + i], base[4 * cap + i], base[5 * cap + i]);
    m.c2 = mk(base[6 * cap + i], base[7 * cap + i], base[8 * cap + i]);
    return m;
}
__device__ __forceinline__ void store_m3(float *base, size_t cap, int i, const M3f &m) {
    base[0 * cap + i] = m.c0.x;
    base[1 * cap + i] = m.c0.y;
    base[2 * cap + i] = m.c0.z;
    base[3 * cap + i] = m.c1.x;
    base[4 * cap + i] = m.c1.y;
    base[5 * cap + i] = m.c1.z;
    base[6 * cap + i] = m.c2.x;
    base[7 * cap + i] = m.c2.y;
    base[8 * cap + i] = m.c2.z;
}

__device__ __forceinline__ void add_reaction(double *reactions, int oi, V3f center, V3f point, V3f impulse) {
    V3f ang = cross(point - center, impulse);
    double *r = reactions + 6 * oi;
    atomicAdd(r + 0, static_cast<double>(impulse.x));
    atomicAdd(r + 1, static_cast<double>(impulse.y));
    atomicAdd(r + 2, static_cast<double>(impulse.z));
    atomicAdd(r + 3, static_cast<double>(ang.x));
    atomicAdd(r + 4, static_cast<double>(ang.y));
    atomicAdd(r + 5, static_cast<double>(ang.z));
}

// Largest power of two s with total * s <= 2^30 (exponent clamped to the normal range).
__device__ __forceinline__ float pow2_scale(float total) {
    float e = floorf(30.0f - log2f(fmaxf(total, 1e-30f)));
    e = fminf(fmaxf(e, -120.0f), 120.0f);
    return exp2f(e);
}

// The blocks a particle's 3 x 3 x 3 stencil reaches from base cell b: at most
// two per axis, slot (qx << 2) | (qy << 1) | qz for block (b >> BS) + q.  Each
// thread looks up (or, INSERT, finds or inserts) the distinct ones and stores
// the ids at ids[slot * THREADS], the unreached slots -1.
template <int THREADS, int BS, bool INSERT>
__device__ __forceinline__ void stencil_blocks(const GridTable &g, const int b[3], uint32_t ns, int *ids,
                                               uint32_t *status) {
    const int g0 = b[0] >> BS, g1 = b[1] >> BS, g2 = b[2] >> BS;
    const int e0 = ((b[0] + 2) >> BS) - g0, e1 = ((b[1] + 2) >> BS) - g1, e2 = ((b[2] + 2) >> BS) - g2;
    for (int q = 0; q < 8; ++q) {
        const int qx = q >> 2, qy = (q >> 1) & 1, qz = q & 1;
        int id = -1;
        if (qx <= e0 && qy <= e1 && qz <= e2) {
            const unsigned long long key = block_key(g0 + qx, g1 + qy, g2 + qz, ns);
            if constexpr (INSERT)
                id = find_or_insert_block(g, key, make_int4(g0 + qx, g1 + qy, g2 + qz, static_cast<int>(ns)), status);
            else
                id = lookup_block(g, key);
        }
        ids[q * THREADS] = id;
    }
}
// The slot (stencil_blocks) of the block holding cell (cx, cy, cz) of the
// stencil based at b.
template <int BS>
__device__ __forceinline__ int stencil_block_slot(const int b[3], int cx, int cy, int cz) {
    return (((cx >> BS) - (b[0] >> BS)) << 2) | (((cy >> BS) - (b[1] >> BS)) << 1) | ((cz >> BS) - (b[2] >> BS));
}

// PLASTIC selects the variant that carries plastic state (snow, sand, NH sand);
// scenes without plastic materials run the leaner variant.  VARIANT selects
// kPlain (one scene without obstacles, parameters from the kernel parameters),
// kPlainObst (the same with rigid obstacles), kMulti (a multi-scene batch,
// which has no obstacles: each particle reads its scene's parameters from the
// scene table, scene = class namespace >> kSceneShift, and takes part only in
// the substeps its scene advances in this batch) or kCpic (one scene with
// obstacles whose grid namespace includes CPIC side masks).  Each costs
// registers only where used: the obstacle contact calls an out-of-line
// surface function, and with that call in the kernel the register allocator
// kept ~500 more bytes per thread in local memory on every particle's path
// (80 registers: 172 bytes of spill stores against 28 without it), which cost
// the obstacle-free dam break ~10 % of its fused transfer time.
enum Variant { kPlain = 0, kMulti = 1, kCpic = 2, kPlainObst = 3 };
constexpr bool has_obstacles(int variant) { return variant == kCpic || variant == kPlainObst; }

// Shared memory of a transfer CTA, as pointers to its arrays.  One buffer
// holds the G2P gather tile (float4 per node) and then the P2G scatter tile
// (4 fixed-point ints per node, component-major).
template <int THREADS, bool OBST>
struct TransferSmem {
    float4 *tile;
    float (*fred)[4];
    int *blk;
    int *blk2;
    int *used;
    int (*red)[8];
    Box *box;
    Box *gbox;  // the G2P box, whose block ids the P2G reuses (shared: not held in registers)
    int *abort;
    float (*park)[THREADS];  // the affine matrix across the obstacle contact
};
// The arrays, one set per kernel for each (THREADS, OBST): the deferred
// kernel's P2G-only and whole-chunk passes share them.
template <int THREADS, bool OBST>
__device__ __forceinline__ TransferSmem<THREADS, OBST> transfer_smem() {
    __shared__ float4 tile[tile_nodes(THREADS)];
    __shared__ float fred[THREADS / 32][4];
    __shared__ int blk[kMaxTileBlocks];
    __shared__ int blk2[kMaxTileBlocks];
    __shared__ int used[kMaxTileBlocks];
    __shared__ int red[THREADS / 32][8];
    __shared__ Box box;
    __shared__ Box gbox;
    __shared__ int abort_flag;
    __shared__ float park[OBST ? 9 : 1][THREADS];
    return TransferSmem<THREADS, OBST>{tile, fred, blk, blk2, used, red, &box, &gbox, &abort_flag, park};
}

// Deferred-chunk lists (layout at DeferLists): 0 = P2G only, 1 = whole
// chunk, 2 + p = no record for a launch of step parity p.
__device__ __forceinline__ void defer_push(const SimParams &sp, int list, int chunk) {
    const uint32_t slot = atomicAdd(sp.defer + list, 1u);
    if (slot < static_cast<uint32_t>(sp.defer_cap))
        sp.defer[kDeferHeader + static_cast<size_t>(list) * sp.defer_cap + slot] = static_cast<uint32_t>(chunk);
}
// The tag of the per-CTA records that the P2G of a launch with this step
// index writes (1 or 2); a G2P accepts the tag of its own step index.  The
// general chunks of a fused transfer run beside the fast kernel and write
// their records meanwhile: the tag keeps the fast kernel from reading them
// as records of its own step.
__device__ __forceinline__ int record_tag(int step_index) { return 1 + (step_index & 1); }

#define TMPM_TRANSFER_PARAMS                                                                                 \
    ParticleSoA P, int n, const DevClass *__restrict__ classes, GridTable cur, GridTable next, SimParams sp, \
        const DevObstacle *__restrict__ obstacles, const float *__restrict__ planes, double *reactions,      \
        uint32_t *status, int *__restrict__ cache
#define TMPM_TRANSFER_ARGS P, n, classes, cur, next, sp, obstacles, planes, reactions, status, cache

// One chunk of THREADS consecutive particles in storage order, by one CTA.
//
// FAST (the fused G2P2G of one scene without CPIC) compiles only the common
// path: the G2P box and block ids from the chunk's record, the gather from
// the tile and the fixed-point scatter tile.  A chunk without a record of
// this step is skipped (it is on the no-record list, which
// k_transfer_deferred runs beside the fast kernel); a chunk whose particles
// left the recorded box is deferred whole before any write; a chunk whose
// P2G box does not fit or has a dominant particle stores its particles'
// velocity and affine matrix and defers its P2G.  Without the fallback code
// (box reduction and hash lookups for the G2P, per-node global gathers and
// scatters) the fast kernel keeps the common path's values in registers: at
// 64 registers 24 / 28 bytes of spill stores / loads against 52 / 84 with the
// fallbacks compiled in.
template <int MODE, bool PLASTIC, int VARIANT, int THREADS, int BS, bool FAST>
__device__ __forceinline__ void transfer_chunk(TMPM_TRANSFER_PARAMS, const int chunk) {
    constexpr bool MULTI = VARIANT == kMulti;
    constexpr bool CPIC = VARIANT == kCpic;
    constexpr bool OBST = has_obstacles(VARIANT);
    // The obstacle contact is compiled into the general path only: the fast
    // path tests each particle against the obstacles' reach (inline, no call)
    // and defers a chunk that may touch one.
    constexpr bool CONTACT = OBST && !FAST;
    static_assert(!FAST || (MODE == kModeG2P2G && !CPIC), "the fast path is the fused transfer without CPIC");
    constexpr int kTileNodes = tile_nodes(THREADS);
    const TransferSmem<THREADS, CONTACT> S = transfer_smem<THREADS, CONTACT>();
    float4 *const s_gv = S.tile;
    int (*const s_sc)[kTileNodes] = reinterpret_cast<int (*)[kTileNodes]>(S.tile);
    float (*const s_fred)[4] = S.fred;
    int *const s_blk = S.blk;
    int *const s_blk2 = S.blk2;
    int *const s_used = S.used;
    int (*const s_red)[8] = S.red;
    Box &s_box = *S.box;
    Box &s_gbox = *S.gbox;
    int &s_abort = *S.abort;
    float (*const s_park)[THREADS] = S.park;

    const size_t cap = P.cap;
    const int i = chunk * THREADS + static_cast<int>(threadIdx.x);
    const bool valid = i < n;
    int *const cc = cache + static_cast<size_t>(chunk) * kCacheStride;

    if (threadIdx.x == 0) s_abort = (*reinterpret_cast<volatile uint32_t *>(status) & kFatal) != 0;
    if (MODE != kModeG2P) {
        // The first barrier of the kernel orders these.
        for (int t = threadIdx.x; t < kMaxTileBlocks; t += THREADS) s_used[t] = 0;
    }

    V3f x = mk(0, 0, 0);
    M3f F = m3_identity();
    uint32_t cw = 0;
    DevClass k;
    k.mass = 0.f;
    k.color = 0;
    if (valid) {
        x = mk(P.x[i], P.x[cap + i], P.x[2 * cap + i]);
        cw = P.cls[i];
        // the namespace and kind now; the whole record after the gather (below)
        k.color = classes[cw & kClassMask].color;
        k.kind = classes[cw & kClassMask].kind;
    }
    const int scene = MULTI ? static_cast<int>(k.color >> kSceneShift) : 0;
    const SceneParams *const scn = sp.scenes + scene;
#define SCN(f) (MULTI ? scn->f : sp.s0.f)
    const float h = SCN(h), inv_h = SCN(inv_h), inv_d = SCN(inv_d), dt = SCN(dt);
    // g2p_on: the particle completes substep step_index here; p2g_on: it scatters for step_index + 1.
    bool g2p_on = valid, p2g_on = valid;
    if (MULTI && valid) {
        const int steps = scn->steps;
        const bool dead = (__ldcg(sp.scene_status + scene) & kStatusResident) != 0;
        g2p_on = !dead && sp.step_index < steps;
        p2g_on = !dead && sp.step_index + 1 < steps;
    }
    uint32_t *const resident_flag = MULTI ? sp.scene_status + scene : status;
    // grid namespace at the current positions (colour, and CPIC side masks when on)
    uint32_t ns = CPIC ? particle_namespace(k.color, 1, sp.num_obstacles, obstacles, x) : k.color;
    const bool fixed = (cw & kFixedBit) != 0;
    const bool plastic = PLASTIC && g2p_on && k.kind >= kMatSnow;
    float pl[3] = {1.0f, 0.0f, 0.0f};
    if (plastic) {
        pl[0] = P.pl[i];
        pl[1] = P.pl[cap + i];
        pl[2] = P.pl[2 * cap + i];
    }
    V3f v = mk(0, 0, 0);
    M3f Cm = m3_zero();
    if (threadIdx.x == 0) s_gbox.ok = 0;

    if (MODE == kModeP2G) {
        if (valid) {
            F = load_m3(P.F, cap, i);
            k = classes[cw & kClassMask];
        }
        if (p2g_on) {
            v = mk(P.v[i], P.v[cap + i], P.v[2 * cap + i]);
            Cm = load_m3(P.C, cap, i);
        }
    } else {
        // ------------------------------------------------------------- G2P
        const int b[3] = {base_cell(x.x, inv_h), base_cell(x.y, inv_h), base_cell(x.z, inv_h)};
        // The previous P2G of this CTA recorded the box and block ids for these
        // very positions (ids are stable within a batch), so normally no box
        // reduction and no hash lookup is needed.  A record that does not
        // cover every particle sends the CTA through the general path.
        bool use_cache = cc[0] == record_tag(sp.step_index);
        if constexpr (FAST) {
            if (!use_cache) return;  // on the no-record list (CTA-uniform)
        }
        Box bx;
        for (int attempt = 0; attempt < (FAST ? 1 : 2); ++attempt) {
            if (use_cache) {
                bx.lo[0] = cc[8];
                bx.lo[1] = cc[9];
                bx.lo[2] = cc[10];
                bx.dim[0] = cc[11];
                bx.dim[1] = cc[12];
                bx.dim[2] = cc[13];
                bx.blo[0] = cc[1];
                bx.blo[1] = cc[2];
                bx.blo[2] = cc[3];
                bx.nb[0] = cc[4];
                bx.nb[1] = cc[5];
                bx.nb[2] = cc[6];
                bx.color = static_cast<uint32_t>(cc[7]);
                bx.nodes = cc[14];
                bx.nbt = cc[15];
                bx.ok = 1;
                tile_strides(bx.dim[1], bx.dim[2], bx.s1, bx.s2);
            } else if constexpr (!FAST) {
                reduce_box<THREADS, BS>(g2p_on, b, ns, s_red, s_box);
                bx = s_box;
                if (bx.ok) {
                    const Split3 split(bx.nb[1], bx.nb[2]);
                    for (int t = threadIdx.x; t < bx.nbt; t += THREADS) {
                        int tx, ty, tz;
                        split(t, tx, ty, tz);
                        s_blk[t] = lookup_block(cur, block_key(bx.blo[0] + tx, bx.blo[1] + ty, bx.blo[2] + tz, bx.color));
                    }
                    __syncthreads();
                }
            }
            bool bad = use_cache && g2p_on &&
                       (b[0] < bx.lo[0] || b[1] < bx.lo[1] || b[2] < bx.lo[2] || b[0] + 2 >= bx.lo[0] + bx.dim[0] ||
                        b[1] + 2 >= bx.lo[1] + bx.dim[1] || b[2] + 2 >= bx.lo[2] + bx.dim[2] || ns != bx.color);
            if (bx.ok && !bad) {
                const SplitP split(bx.s1, bx.s2);
                for (int t = threadIdx.x; t < bx.nodes; t += THREADS) {
                    int tx, ty, tz;
                    split(t, tx, ty, tz);
                    if (ty >= bx.dim[1] || tz >= bx.dim[2]) continue;  // padding
                    int cx = bx.lo[0] + tx, cy = bx.lo[1] + ty, cz = bx.lo[2] + tz;
                    int tb = tile_block_index<BS>(bx, cx, cy, cz);
                    int id = use_cache ? cc[kCacheHeader + tb] : s_blk[tb];
                    if (use_cache) s_blk[tb] = id;
                    if (id >= 0) {
                        // asynchronous 16-byte copy global -> shared (L2 only), no register staging
                        const float4 *src = cur.pool + static_cast<size_t>(id) * (1 << (3 * BS)) + node_local<BS>(cx, cy, cz);
                        const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(s_gv + t));
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
                    } else {
                        s_gv[t] = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
                asm volatile("cp.async.wait_all;" ::: "memory");
            }
            bad = __syncthreads_or(bad) != 0;
            if (!bad) break;
            if constexpr (FAST) {  // a particle left the recorded box: the whole chunk, nothing written yet
                if (threadIdx.x == 0) defer_push(sp, 1, chunk);
                return;
            }
            use_cache = false;
        }
        if (s_abort) return;
        const V3f gp = mk(x.x * inv_h, x.y * inv_h, x.z * inv_h);
        const V3f fx = mk(gp.x - static_cast<float>(b[0]), gp.y - static_cast<float>(b[1]), gp.z - static_cast<float>(b[2]));
        float wx[3], wy[3], wz[3];
        quad_weights(fx.x, wx);
        quad_weights(fx.y, wy);
        quad_weights(fx.z, wz);
        V3f vel = mk(0, 0, 0);
        M3f aff = m3_zero();
        if (g2p_on && !fixed) {
            float dxs[3], dys[3], dzs[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                dxs[a] = (a - fx.x) * h * inv_d;
                dys[a] = (a - fx.y) * h * inv_d;
                dzs[a] = (a - fx.z) * h * inv_d;
            }
            if (FAST || bx.ok) {
                const int ox = b[0] - bx.lo[0], oy = b[1] - bx.lo[1], oz = b[2] - bx.lo[2];
                // Paired f32 arithmetic (Blackwell FFMA2): accumulators
                // p0..p2 = (vel, C column 0) and q0..q2 = (C column 1, C column 2)
                // for the x, y, z components; per node (w, w dx) and (w dy, w dz).
                float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0, q0 = p0, q1 = p0, q2 = p0;
                float2 z1[3], z2[3];
#pragma unroll
                for (int e = 0; e < 3; ++e) {
                    z1[e] = make_float2(wz[e], wz[e]);
                    z2[e] = make_float2(wz[e], wz[e] * dzs[e]);
                }
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float wac = wx[a] * wy[c];
                        const float2 pa = make_float2(wac, wac * dxs[a]);
                        const float2 pb = make_float2(wac * dys[c], wac);
                        const int row = (ox + a) * bx.s1 + (oy + c) * bx.s2 + oz;
#pragma unroll
                        for (int e = 0; e < 3; ++e) {
                            const float4 g4 = s_gv[row + e];
                            const float2 s1 = __fmul2_rn(pa, z1[e]);  // (w, w dx)
                            const float2 s2 = __fmul2_rn(pb, z2[e]);  // (w dy, w dz)
                            const float2 nx = make_float2(g4.x, g4.x), ny = make_float2(g4.y, g4.y),
                                         nz = make_float2(g4.z, g4.z);
                            p0 = __ffma2_rn(nx, s1, p0);
                            p1 = __ffma2_rn(ny, s1, p1);
                            p2 = __ffma2_rn(nz, s1, p2);
                            q0 = __ffma2_rn(nx, s2, q0);
                            q1 = __ffma2_rn(ny, s2, q1);
                            q2 = __ffma2_rn(nz, s2, q2);
                        }
                    }
                vel = mk(p0.x, p1.x, p2.x);
                aff.c0 = mk(p0.y, p1.y, p2.y);
                aff.c1 = mk(q0.x, q1.x, q2.x);
                aff.c2 = mk(q0.y, q1.y, q2.y);
            } else {
                // Per-node global gather.  The stencil's blocks are looked up
                // first (the tile is unused on this path and holds each
                // thread's ids), so no node load waits on a lookup.
                int *const ids = reinterpret_cast<int *>(s_gv) + threadIdx.x;
                stencil_blocks<THREADS, BS, false>(cur, b, ns, ids, status);
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                        for (int e = 0; e < 3; ++e) {
                            const int cx = b[0] + a, cy = b[1] + c, cz = b[2] + e;
                            const int id = ids[stencil_block_slot<BS>(b, cx, cy, cz) * THREADS];
                            float4 val = make_float4(0.f, 0.f, 0.f, 0.f);
                            if (id >= 0)
                                val = __ldcg(cur.pool + static_cast<size_t>(id) * (1 << (3 * BS)) + node_local<BS>(cx, cy, cz));
                            const float w = wx[a] * wy[c] * wz[e];
                            const V3f nv = mk(val.x, val.y, val.z);
                            vel = vel + nv * w;
                            aff.c0 = aff.c0 + nv * (dxs[a] * w);
                            aff.c1 = aff.c1 + nv * (dys[c] * w);
                            aff.c2 = aff.c2 + nv * (dzs[e] * w);
                        }
            }
        }

        // the P2G below reuses the block ids of this box (read after its
        // barriers); published now, the box is dead through the update
        if (MODE != kModeG2P && threadIdx.x == 0) s_gbox = bx;
        // F is read only now: it is not needed during the gather, whose
        // accumulators and weights are the kernel's peak register demand.  With
        // the obstacle contact (an out-of-line call, around which everything
        // live is saved) an updating particle reads F after the contact.
        const bool updates = g2p_on && !fixed;
        if (valid) {
            if (!CONTACT || !updates) F = load_m3(P.F, cap, i);
            k = classes[cw & kClassMask];
        }
        V3f pos = x;
        if (updates) {
            // Particle update (gpu.wgsl:885-1003; world.rs:443-463).
            if (sp.apply_force) {
                const size_t w = P.widx[i], fs = P.force_stride;
                V3f f = mk(P.force[w], P.force[fs + w], P.force[2 * fs + w]);
                vel = vel + mk(f.x / k.mass, f.y / k.mass, f.z / k.mass) * dt;  // force / mass * dt (gpu.wgsl:885)
            }
            vel = vel * expf(-k.damping * dt);
            pos = x + vel * dt;
            const float radius = k.radius;
            if (SCN(has_bounds)) {
                for (int a = 0; a < 3; ++a) {
                    float lower = SCN(bmin[a]) + radius, upper = SCN(bmax[a]) - radius;
                    float pa = comp(pos, a), va = comp(vel, a);
                    if (pa < lower) {
                        set_comp(pos, a, lower);
                        set_comp(vel, a, fmaxf(va, 0.0f));
                    } else if (pa > upper) {
                        set_comp(pos, a, upper);
                        set_comp(vel, a, fminf(va, 0.0f));
                    }
                }
            }
            if constexpr (CONTACT) {
                // The surface function is an out-of-line call, around which
                // every live value is saved: the affine matrix waits in shared
                // memory and the class record is dropped (reloaded below), so
                // that only the position, velocity, radius and mass live across.
                const float pmass = k.mass;
                s_park[0][threadIdx.x] = aff.c0.x;
                s_park[1][threadIdx.x] = aff.c0.y;
                s_park[2][threadIdx.x] = aff.c0.z;
                s_park[3][threadIdx.x] = aff.c1.x;
                s_park[4][threadIdx.x] = aff.c1.y;
                s_park[5][threadIdx.x] = aff.c1.z;
                s_park[6][threadIdx.x] = aff.c2.x;
                s_park[7][threadIdx.x] = aff.c2.y;
                s_park[8][threadIdx.x] = aff.c2.z;
                for (int oi = 0; oi < sp.num_obstacles; ++oi) {
                    const DevObstacle &o = obstacles[oi];
                    if (!obstacle_may_contact(o, pos, radius)) continue;
                    V3f nrm;
                    float d = obstacle_surface(o, planes, pos, nrm);
                    if (d < radius) {
                        pos = pos + nrm * (radius - d);
                        V3f before = vel;
                        vel = contact_velocity(o, pos, vel, nrm);
                        if (sp.reactions)
                            add_reaction(reactions, oi, mk(o.center[0], o.center[1], o.center[2]), pos - nrm * radius,
                                         (before - vel) * pmass);
                    }
                }
                aff.c0 = mk(s_park[0][threadIdx.x], s_park[1][threadIdx.x], s_park[2][threadIdx.x]);
                aff.c1 = mk(s_park[3][threadIdx.x], s_park[4][threadIdx.x], s_park[5][threadIdx.x]);
                aff.c2 = mk(s_park[6][threadIdx.x], s_park[7][threadIdx.x], s_park[8][threadIdx.x]);
                k = classes[cw & kClassMask];
            }
        }
        if constexpr (OBST && FAST) {
            // A chunk in which some particle may touch an obstacle runs whole
            // through the general path, which has the contact: deferred here,
            // before this kernel writes anything or flags a failure for it.
            // The reach test is conservative (f32 rounding margins in the
            // reach and 5 % of a cell here), so a chunk that stays has no
            // contact, exactly as the general path would find.
            bool near = false;
            if (updates) {
                const float r = k.radius * 1.0001f + 0.05f * h;
                for (int oi = 0; oi < sp.num_obstacles; ++oi) near = near || obstacle_near(obstacles[oi], pos, r);
            }
            if (__syncthreads_or(near)) {
                if (threadIdx.x == 0) defer_push(sp, 1, chunk);
                return;
            }
        }
        if (updates) {
            if (CONTACT) F = load_m3(P.F, cap, i);
            M3f Fn = mul(add(m3_identity(), scale(aff, dt)), F);
            bool plastic_ok = true;
            if (k.kind == kMatFluid) {
                float sc = cbrtf(fmaxf(det(Fn), 1e-9f));
                Fn = scale(m3_identity(), sc);
            } else if (PLASTIC && k.kind >= kMatSnow) {
                plastic_ok = project_plastic(k, Fn, pl);
            }
            // Resident failure detection (gpu.wgsl:946-994).
            float ncx = floorf(__fsub_rn(__fmul_rn(pos.x, inv_h), 0.5f));
            float ncy = floorf(__fsub_rn(__fmul_rn(pos.y, inv_h), 0.5f));
            float ncz = floorf(__fsub_rn(__fmul_rn(pos.z, inv_h), 0.5f));
            bool failed = !finite3(pos) || !finite3(vel) || !finite_m(aff) || !finite_m(Fn);
            bool representable = ncx >= -131000.0f && ncx <= 131000.0f && ncy >= -131000.0f && ncy <= 131000.0f &&
                                 ncz >= -131000.0f && ncz <= 131000.0f;
            failed = failed || !representable;
            if (!failed && SCN(has_bounds)) {
                int nb3[3] = {static_cast<int>(ncx), static_cast<int>(ncy), static_cast<int>(ncz)};
                for (int a = 0; a < 3; ++a)
                    failed = failed || nb3[a] < SCN(first_base[a]) || nb3[a] > SCN(last_base[a]);
            }
            if (sp.resident_checks) {
                if (k.kind == kMatCorotated || k.kind == kMatSnow || k.kind == kMatSand)
                    failed = failed || !regular_corotated(Fn);
                if (k.kind == kMatSandNeoHookean) {  // CFL with the elastic volume (gpu.wgsl:983-987)
                    float wave = k.wave * sqrtf(fmaxf(det(Fn), 1e-6f));
                    failed = failed || dt * fmaxf(wave, len(vel)) > 0.5f * h * (1.0f + 1e-4f);
                } else {
                    failed = failed || dt * (k.wave + len(vel)) > 0.4f * h * (1.0f + 1e-4f);
                }
                failed = failed || !plastic_ok;
                if (failed) atomicOr(resident_flag, kStatusResident);
            } else {
                if (finite3(pos) && !representable) atomicOr(status, kStatusCapacity);  // beyond the key range
                // no CPU fallback on this path: an unprojectable plastic state is unavailable here
                if (!plastic_ok) atomicOr(resident_flag, kStatusResident);
            }
            x = pos;
            v = vel;
            Cm = aff;
            F = Fn;
        }
        if (g2p_on) {
            P.x[i] = x.x;
            P.x[cap + i] = x.y;
            P.x[2 * cap + i] = x.z;
            if (!fixed) store_m3(P.F, cap, i, F);
            if (plastic && !fixed) {
                P.pl[i] = pl[0];
                P.pl[cap + i] = pl[1];
                P.pl[2 * cap + i] = pl[2];
            }
            // the last substep of the batch (per scene in a multi-scene batch) writes v and C back
            if (MODE == kModeG2P || (MULTI && !p2g_on)) {
                P.v[i] = v.x;
                P.v[cap + i] = v.y;
                P.v[2 * cap + i] = v.z;
                store_m3(P.C, cap, i, Cm);
            }
        }
        if (MODE == kModeG2P) return;
    }

    // ----------------------------------------------------------------- P2G
    const int b[3] = {base_cell(x.x, inv_h), base_cell(x.y, inv_h), base_cell(x.z, inv_h)};
    const bool in_range =
        block_representable(b[0] >> BS, b[1] >> BS, b[2] >> BS) &&
        block_representable((b[0] + 2) >> BS, (b[1] + 2) >> BS, (b[2] + 2) >> BS);
    const bool active = p2g_on && in_range;
    if (p2g_on && !in_range) {
        if (sp.resident_checks) atomicOr(resident_flag, kStatusResident);
        else atomicOr(status, kStatusCapacity);
    }
    const V3f gp = mk(x.x * inv_h, x.y * inv_h, x.z * inv_h);
    const V3f fx = mk(gp.x - static_cast<float>(b[0]), gp.y - static_cast<float>(b[1]), gp.z - static_cast<float>(b[2]));
    float wx[3], wy[3], wz[3];
    quad_weights(fx.x, wx);
    quad_weights(fx.y, wy);
    quad_weights(fx.z, wz);
    M3f A = m3_zero();
    V3f mv = mk(0, 0, 0);
    float bound_m = 0.f, bound_p = 0.f;
    if (active) {
        M3f S = scaled_stress<!CONTACT && !PLASTIC>(k, F, Cm, -dt * inv_d, pl[0]);
        A = add(S, scale(Cm, k.mass));
        mv = v * k.mass;
        // |(m v + A dpos)_i| <= |m v_i| + 1.5 h sum_j |A_ij| and a particle's 27 weights sum to one,
        // so the chunk's sums bound every node value it produces.
        float r0 = fabsf(A.c0.x) + fabsf(A.c1.x) + fabsf(A.c2.x);
        float r1 = fabsf(A.c0.y) + fabsf(A.c1.y) + fabsf(A.c2.y);
        float r2 = fabsf(A.c0.z) + fabsf(A.c1.z) + fabsf(A.c2.z);
        bound_m = k.mass;
        bound_p = fmaxf(fmaxf(fabsf(mv.x) + 1.5f * h * r0, fabsf(mv.y) + 1.5f * h * r1), fabsf(mv.z) + 1.5f * h * r2);
        if (!(bound_p < 1e30f)) bound_p = 1e30f;  // non-finite state is flagged by the G2P checks
    }
    // the CTA's box and the sums of the bounds, with one barrier
    if (MODE != kModeP2G && CPIC) ns = particle_namespace(k.color, 1, sp.num_obstacles, obstacles, x);
    float tot_m = bound_m, tot_p = bound_p, max_m = bound_m, max_p = bound_p;
    Box bx;
    reduce_box_sums<THREADS, BS>(active, b, ns, tot_m, tot_p, max_m, max_p, s_red, s_fred, bx);
    if (MODE == kModeP2G && s_abort) return;
    // one dominant particle: the whole CTA takes the f32 direct path (CTA-uniform)
    if (max_m > tot_m * kFloatModeShare || max_p > tot_p * kFloatModeShare) bx.ok = 0;
    if constexpr (FAST) {
        if (!bx.ok) {
            // A chunk with nothing to scatter (every particle's scene is past
            // its last substep of the batch) needs no P2G and no record.
            if (bx.nodes == 0) {
                if (threadIdx.x == 0) cc[0] = 0;
                return;
            }
            // the P2G-only pass reads velocity and affine matrix from the
            // particle arrays (position, F and plastic state are stored)
            if (p2g_on) {
                P.v[i] = v.x;
                P.v[cap + i] = v.y;
                P.v[2 * cap + i] = v.z;
                store_m3(P.C, cap, i, Cm);
            }
            if (threadIdx.x == 0) defer_push(sp, 0, chunk);
            return;
        }
    }
    if (bx.ok) {
        // every warp has finished its gather (barrier above): the buffer becomes the scatter tile
        for (int t = threadIdx.x; t < bx.nodes; t += THREADS) {
            s_sc[0][t] = 0;
            s_sc[1][t] = 0;
            s_sc[2][t] = 0;
            s_sc[3][t] = 0;
        }
        __syncthreads();
        // Shared accumulation in 32-bit fixed point: integer shared atomics are
        // native, float ones are not.  Power-of-two scales from the chunk bounds
        // keep every node sum below 2^30 (no overflow) with unbiased rounding.
        const float sm = pow2_scale(tot_m), spv = pow2_scale(tot_p);
        if (active) {
            const int ox = b[0] - bx.lo[0], oy = b[1] - bx.lo[1], oz = b[2] - bx.lo[2];
            const float msc = k.mass * sm;
            float dxs[3], dys[3], dzs[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                dxs[a] = (a - fx.x) * h;
                dys[a] = (a - fx.y) * h;
                dzs[a] = (a - fx.z) * h;
            }
            // Paired f32 arithmetic: per node (m w s_m, w s_p) from (w_ac, w_ac) x (w_z m s_m, w_z s_p),
            // and the momentum's (x, y) pair.
            float2 zs[3];
#pragma unroll
            for (int e = 0; e < 3; ++e) zs[e] = make_float2(wz[e] * msc, wz[e] * spv);
            const float2 c2xy = make_float2(A.c2.x, A.c2.y);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const V3f qa = mv + A.c0 * dxs[a];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const V3f qac = qa + A.c1 * dys[c];
                    const float wac = wx[a] * wy[c];
                    const float2 wac2 = make_float2(wac, wac);
                    const float2 qacxy = make_float2(qac.x, qac.y);
                    const int row = (ox + a) * bx.s1 + (oy + c) * bx.s2 + oz;
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        const float2 qxy = __ffma2_rn(c2xy, make_float2(dzs[e], dzs[e]), qacxy);
                        const float qz = qac.z + A.c2.z * dzs[e];
                        const float2 mw = __fmul2_rn(wac2, zs[e]);  // (w m s_m, w s_p)
                        const float2 pxy = __fmul2_rn(qxy, make_float2(mw.y, mw.y));
                        const int t = row + e;
                        atomicAdd(reinterpret_cast<unsigned *>(&s_sc[0][t]), static_cast<unsigned>(__float2int_rn(mw.x)));
                        atomicAdd(reinterpret_cast<unsigned *>(&s_sc[1][t]), static_cast<unsigned>(__float2int_rn(pxy.x)));
                        atomicAdd(reinterpret_cast<unsigned *>(&s_sc[2][t]), static_cast<unsigned>(__float2int_rn(pxy.y)));
                        atomicAdd(reinterpret_cast<unsigned *>(&s_sc[3][t]), static_cast<unsigned>(__float2int_rn(qz * mw.y)));
                    }
                }
            }
            // mark the (at most 8) blocks this particle's stencil touches
            const int bx0 = (b[0] >> BS) - bx.blo[0], bx1 = ((b[0] + 2) >> BS) - bx.blo[0];
            const int by0 = (b[1] >> BS) - bx.blo[1], by1 = ((b[1] + 2) >> BS) - bx.blo[1];
            const int bz0 = (b[2] >> BS) - bx.blo[2], bz1 = ((b[2] + 2) >> BS) - bx.blo[2];
            s_used[(bx0 * bx.nb[1] + by0) * bx.nb[2] + bz0] = 1;
            s_used[(bx0 * bx.nb[1] + by0) * bx.nb[2] + bz1] = 1;
            s_used[(bx0 * bx.nb[1] + by1) * bx.nb[2] + bz0] = 1;
            s_used[(bx0 * bx.nb[1] + by1) * bx.nb[2] + bz1] = 1;
            s_used[(bx1 * bx.nb[1] + by0) * bx.nb[2] + bz0] = 1;
            s_used[(bx1 * bx.nb[1] + by0) * bx.nb[2] + bz1] = 1;
            s_used[(bx1 * bx.nb[1] + by1) * bx.nb[2] + bz0] = 1;
            s_used[(bx1 * bx.nb[1] + by1) * bx.nb[2] + bz1] = 1;
        }
        __syncthreads();
        const Split3 split_b(bx.nb[1], bx.nb[2]);
        for (int t = threadIdx.x; t < bx.nbt; t += THREADS) {
            int id = -1;
            if (s_used[t]) {
                int tx, ty, tz;
                split_b(t, tx, ty, tz);
                int gx = bx.blo[0] + tx, gy = bx.blo[1] + ty, gz = bx.blo[2] + tz;
                // reuse the id the G2P box already holds for this block (same table)
                if (s_gbox.ok && s_gbox.color == bx.color) {
                    int rx = gx - s_gbox.blo[0], ry = gy - s_gbox.blo[1], rz = gz - s_gbox.blo[2];
                    if (rx >= 0 && ry >= 0 && rz >= 0 && rx < s_gbox.nb[0] && ry < s_gbox.nb[1] && rz < s_gbox.nb[2])
                        id = s_blk[(rx * s_gbox.nb[1] + ry) * s_gbox.nb[2] + rz];
                }
                if (id < 0)
                    id = find_or_insert_block(next, block_key(gx, gy, gz, bx.color),
                                              make_int4(gx, gy, gz, static_cast<int>(bx.color)), status);
            }
            s_blk2[t] = id;
            cc[kCacheHeader + t] = id;
        }
        if (threadIdx.x == 0) {
            cc[0] = record_tag(sp.step_index + 1);
            cc[1] = bx.blo[0];
            cc[2] = bx.blo[1];
            cc[3] = bx.blo[2];
            cc[4] = bx.nb[0];
            cc[5] = bx.nb[1];
            cc[6] = bx.nb[2];
            cc[7] = static_cast<int>(bx.color);
            cc[8] = bx.lo[0];
            cc[9] = bx.lo[1];
            cc[10] = bx.lo[2];
            cc[11] = bx.dim[0];
            cc[12] = bx.dim[1];
            cc[13] = bx.dim[2];
            cc[14] = bx.nodes;
            cc[15] = bx.nbt;
        }
        __syncthreads();
        const float inv_sm = 1.0f / sm, inv_sp = 1.0f / spv;
        const SplitP split_n(bx.s1, bx.s2);
        for (int t = threadIdx.x; t < bx.nodes; t += THREADS) {
            const int m = s_sc[0][t], px = s_sc[1][t], py = s_sc[2][t], pz = s_sc[3][t];
            if ((m | px | py | pz) == 0) continue;  // also every padding entry
            int tx, ty, tz;
            split_n(t, tx, ty, tz);
            if (ty >= bx.dim[1] || tz >= bx.dim[2]) continue;  // padding (zero by construction; never flushed)
            int cx = bx.lo[0] + tx, cy = bx.lo[1] + ty, cz = bx.lo[2] + tz;
            int id = s_blk2[tile_block_index<BS>(bx, cx, cy, cz)];
            if (id < 0) continue;
            atomicAdd(next.pool + static_cast<size_t>(id) * (1 << (3 * BS)) + node_local<BS>(cx, cy, cz),
                      make_float4(static_cast<float>(m) * inv_sm, static_cast<float>(px) * inv_sp,
                                  static_cast<float>(py) * inv_sp, static_cast<float>(pz) * inv_sp));
        }
    } else {
        if (threadIdx.x == 0) {
            cc[0] = 0;
            if (sp.defer) defer_push(sp, 2 + ((sp.step_index + 1) & 1), chunk);
        }
        if (active) {
            // Per-node global scatter, the stencil's blocks found or inserted
            // first (the tile is unused on this path: every warp is past its
            // gather, the barrier of the box reduction orders it).
            int *const ids = reinterpret_cast<int *>(s_gv) + threadIdx.x;
            stencil_blocks<THREADS, BS, true>(next, b, ns, ids, status);
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int e = 0; e < 3; ++e) {
                        const int cx = b[0] + a, cy = b[1] + c, cz = b[2] + e;
                        const int id = ids[stencil_block_slot<BS>(b, cx, cy, cz) * THREADS];
                        if (id < 0) continue;
                        float w = wx[a] * wy[c] * wz[e];
                        V3f dpos = mk((a - fx.x) * h, (c - fx.y) * h, (e - fx.z) * h);
                        V3f mom = (mv + mul(A, dpos)) * w;
                        atomicAdd(next.pool + static_cast<size_t>(id) * (1 << (3 * BS)) + node_local<BS>(cx, cy, cz),
                                  make_float4(w * k.mass, mom.x, mom.y, mom.z));
                    }
        }
    }
#undef SCN
}

// The general transfer: every chunk, one CTA each.
template <int MODE, bool PLASTIC, int VARIANT, int THREADS, int MINB, int BS>
__global__ void __launch_bounds__(THREADS, MINB) k_transfer(TMPM_TRANSFER_PARAMS) {
    transfer_chunk<MODE, PLASTIC, VARIANT, THREADS, BS, false>(TMPM_TRANSFER_ARGS, blockIdx.x);
}

// The fast fused transfer: every chunk with a record of this step.
template <bool PLASTIC, int VARIANT, int THREADS, int MINB, int BS>
__global__ void __launch_bounds__(THREADS, MINB) k_transfer_fast(TMPM_TRANSFER_PARAMS) {
    transfer_chunk<kModeG2P2G, PLASTIC, VARIANT, THREADS, BS, true>(TMPM_TRANSFER_ARGS, blockIdx.x);
}

// The deferred chunks of a fast fused transfer through the general path, a
// grid-stride loop of CTAs over a list.  PRE: the chunks without a record of
// this step (written by the previous launch's general P2Gs), run beside the
// fast kernel; otherwise the chunks the fast kernel deferred: P2G only, then
// whole chunks.  The register bound is the general kernel's: a CTA of this
// kernel running beside the fast kernel then takes one CTA slot of an SM, not
// the whole register file.
template <bool PRE, bool PLASTIC, int VARIANT, int THREADS, int BS>
__global__ void __launch_bounds__(THREADS, THREADS == 256 ? TMPM_TRANSFER_MIN_BLOCKS : 8)
    k_transfer_deferred(TMPM_TRANSFER_PARAMS) {
    const uint32_t cap = static_cast<uint32_t>(sp.defer_cap);
    const uint32_t *const lists = sp.defer + kDeferHeader;
    if (PRE) {
        const int list = 2 + (sp.step_index & 1);
        const uint32_t count = min(sp.defer[list], cap);
        for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
            __syncthreads();  // the previous chunk's last reads of shared memory
            transfer_chunk<kModeG2P2G, PLASTIC, VARIANT, THREADS, BS, false>(
                TMPM_TRANSFER_ARGS, static_cast<int>(lists[list * cap + e]));
        }
    } else {
        const uint32_t np = min(sp.defer[0], cap), nw = min(sp.defer[1], cap);
        for (uint32_t e = blockIdx.x; e < np + nw; e += gridDim.x) {
            __syncthreads();
            if (e < np)
                transfer_chunk<kModeP2G, PLASTIC, VARIANT, THREADS, BS, false>(TMPM_TRANSFER_ARGS,
                                                                               static_cast<int>(lists[e]));
            else
                transfer_chunk<kModeG2P2G, PLASTIC, VARIANT, THREADS, BS, false>(
                    TMPM_TRANSFER_ARGS, static_cast<int>(lists[cap + (e - np)]));
        }
    }
}
#undef TMPM_TRANSFER_ARGS
#undef TMPM_TRANSFER_PARAMS

// Grid update over all allocated blocks; also zeroes those blocks in the other pool.
// MULTI: each block takes its scene's parameters from the scene table
// (scene = block namespace >> kSceneShift).  Blocks have edge 2^BS cells.
// OBST: the scene has rigid obstacles (a batch never has).
template <bool MULTI, int BS, bool OBST>
__global__ void __launch_bounds__(256) k_grid(GridTable g, GridTable nxt, SimParams sp,
                                               const DevObstacle *__restrict__ obstacles,
                                               const float *__restrict__ planes, double *reactions, uint32_t *status) {
    __shared__ int s_abort;
    // empty the deferred-chunk lists that the next transfer (step_index) fills
    if (sp.defer && blockIdx.x == 0 && threadIdx.x == 0) {
        sp.defer[0] = 0;
        sp.defer[1] = 0;
        sp.defer[2 + ((sp.step_index + 1) & 1)] = 0;
    }
    if (threadIdx.x == 0) s_abort = (*reinterpret_cast<volatile uint32_t *>(status) & kFatal) != 0;
    __syncthreads();
    if (s_abort) return;
    const size_t gtid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    uint32_t nblocks = min(*g.count, g.max_blocks);
    constexpr int kM = (1 << BS) - 1;
    const size_t nodes = static_cast<size_t>(nblocks) << (3 * BS);
    float4 *next_pool = nxt.pool;
    for (size_t node = gtid; node < nodes; node += stride) {
        float4 mp = g.pool[node];
        // the other pool receives the next P2G: zero every allocated block of it
        if (next_pool) next_pool[node] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (mp.x <= 0.0f) {
            g.pool[node] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        int4 c = g.coords[node >> (3 * BS)];
        int l = static_cast<int>(node) & ((1 << (3 * BS)) - 1);
        int cx = (c.x << BS) + (l >> (2 * BS)), cy = (c.y << BS) + ((l >> BS) & kM), cz = (c.z << BS) + (l & kM);
        const SceneParams *const scn = sp.scenes + (MULTI ? (static_cast<uint32_t>(c.w) >> kSceneShift) : 0u);
#define SCN(f) (MULTI ? scn->f : sp.s0.f)
        const float h = SCN(h), dt = SCN(dt);
        V3f vel = mk(mp.y / mp.x + SCN(gx) * dt, mp.z / mp.x + SCN(gy) * dt, mp.w / mp.x + SCN(gz) * dt);
        V3f pos = mk(static_cast<float>(cx) * h, static_cast<float>(cy) * h, static_cast<float>(cz) * h);
        if (SCN(has_bounds)) {
            // walls by node index (thresholds from the f64 comparisons, see SceneParams)
            const int ci[3] = {cx, cy, cz};
            if (SCN(wall_mode) == 1) {
                bool near = false;
                for (int a = 0; a < 3; ++a) near = near || ci[a] <= SCN(wall_lo[a]) || ci[a] >= SCN(wall_hi[a]);
                if (near) vel = mk(0, 0, 0);
            } else {
                for (int a = 0; a < 3; ++a) {
                    const float va = comp(vel, a);
                    if ((ci[a] <= SCN(wall_lo[a]) && va < 0.0f) || (ci[a] >= SCN(wall_hi[a]) && va > 0.0f))
                        set_comp(vel, a, 0.0f);
                }
            }
        }
#undef SCN
        for (int oi = 0; OBST && oi < sp.num_obstacles; ++oi) {
            const DevObstacle &o = obstacles[oi];
            if (!obstacle_may_contact(o, pos, h)) continue;
            V3f nrm;
            float d = obstacle_surface(o, planes, pos, nrm);
            if (d <= h * (1.0f + 1e-5f)) {
                V3f before = vel;
                vel = contact_velocity(o, pos, vel, nrm);
                if (sp.reactions)
                    add_reaction(reactions, oi, mk(o.center[0], o.center[1], o.center[2]), pos - nrm * d,
                                 (before - vel) * mp.x);
            }
        }
        g.pool[node] = make_float4(vel.x, vel.y, vel.z, mp.x);
    }
}

__global__ void k_clear_table(GridTable g) {
    const size_t gtid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t s = gtid; s <= g.mask; s += stride) {
        g.keys[s] = kEmptyKey;
        g.vals[s] = kPendingId;
    }
    if (gtid == 0) *g.count = 0;
}

// Sort key of each particle.  Single scene: the block's 21-bit Morton code
// followed by the cell's 6-bit Morton code inside the block, so particles of
// one cell are contiguous after the sort.  With a scene table (multi-scene
// batch): scene << 21 | block Morton, the scene from the particle's class and
// its cell width from the table.
__global__ void k_bin_keys(const float *x, size_t cap, int n, float inv_h, const uint32_t *__restrict__ cls,
                           const DevClass *__restrict__ classes, const SceneParams *__restrict__ scenes,
                           int32_t *cells, uint32_t *keys, uint32_t *vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t scene = 0;
    if (scenes) {
        scene = classes[cls[i] & kClassMask].color >> kSceneShift;
        if (!scenes[scene].live) {  // removed scene: sorts after every live particle
            keys[i] = kDeadKey;
            if (vals) vals[i] = static_cast<uint32_t>(i);
            return;
        }
        inv_h = scenes[scene].inv_h;
    }
    int b0 = base_cell(x[i], inv_h), b1 = base_cell(x[cap + i], inv_h), b2 = base_cell(x[2 * cap + i], inv_h);
    if (cells) {
        cells[3 * i] = b0;
        cells[3 * i + 1] = b1;
        cells[3 * i + 2] = b2;
    }
    const uint32_t block = morton_block(b0 >> kBlockShift, b1 >> kBlockShift, b2 >> kBlockShift, scene);
    keys[i] = scenes ? block : (block << 6) | cell_in_block(b0, b1, b2);
    if (vals) vals[i] = static_cast<uint32_t>(i);
}

// dst[j] = src[perm[s(j)]] for every particle field.  With `interleave` = T,
// each full chunk of T sorted particles (one transfer CTA) is stored
// transposed: thread kk of the chunk (warp w = kk / 32, lane l = kk % 32) holds
// sorted particle l * G + w with G = T / 32, so the 32 lanes of
// a warp take one particle from each of 32 consecutive groups of G
// (cell-sorted: one or two cells each) and their stencils do not collide on
// the same shared-memory node.  The last, partial chunk is stored in sorted
// order.
// Lane l of a transfer warp takes the particles of the chunk's cell group
// lane_cell(l).  With 8 particles per cell the 32 groups of a chunk are 32
// cells in Morton order, a 2 x 4 x 4 block (x, y, z); the permutation hands
// each quarter-warp (the 8 lanes of one 128-bit shared-memory phase) a 1 x 2 x 4
// slab of it.  With the tile strides of tile_strides (y stride 4 mod 8, x
// stride 16 mod 32) the quarter-warp's gather loads then fall into distinct
// bank groups, and the warp's 32 scatter atomics into distinct banks.
__device__ __forceinline__ int lane_cell(int l) {
    const int p = l >> 3, q = l & 7;
    return (p & 1) * 16 + ((q >> 1) & 1) * 8 + (p >> 1) * 4 + (q >> 2) * 2 + (q & 1);
}

__global__ void k_gather(ParticleSoA src, ParticleSoA dst, const uint32_t *__restrict__ perm, int n, int interleave) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int sj = j;
    if (interleave) {  // interleave = particles per transfer CTA (0: stored in sorted order)
        const int chunk = j / interleave;
        if ((chunk + 1) * interleave <= n) {
            const int kk = j - chunk * interleave;
            sj = chunk * interleave + lane_cell(kk % 32) * (interleave / 32) + kk / 32;
        }
    }
    int s = static_cast<int>(perm[sj]);
    const size_t cs = src.cap, cd = dst.cap;
    for (int c = 0; c < 3; ++c) {
        dst.x[c * cd + j] = src.x[c * cs + s];
        dst.v[c * cd + j] = src.v[c * cs + s];
        dst.pl[c * cd + j] = src.pl[c * cs + s];
    }
    for (int c = 0; c < 9; ++c) {
        dst.C[c * cd + j] = src.C[c * cs + s];
        dst.F[c * cd + j] = src.F[c * cs + s];
    }
    dst.cls[j] = src.cls[s];
    dst.widx[j] = src.widx[s];
}

// Device rows back in world order: out[c * stride + widx[j]] = row c of stored
// particle j, for the 27 f32 components (x, v, C, F, plastic), so the host
// applies a readback sequentially instead of scattering through the sort
// permutation.
__global__ void k_unsort(ParticleSoA P, int n, float *__restrict__ out, size_t stride, uint32_t *nonfinite) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const size_t cap = P.cap, w = P.widx[j];
    bool finite = true;
    for (int c = 0; c < 3; ++c) {
        const float x = P.x[c * cap + j], v = P.v[c * cap + j], p = P.pl[c * cap + j];
        finite = finite && isfinite(x) && isfinite(v) && isfinite(p);
        out[c * stride + w] = x;
        out[(3 + c) * stride + w] = v;
        out[(24 + c) * stride + w] = p;
    }
    for (int c = 0; c < 9; ++c) {
        const float a = P.C[c * cap + j], f = P.F[c * cap + j];
        finite = finite && isfinite(a) && isfinite(f);
        out[(6 + c) * stride + w] = a;
        out[(15 + c) * stride + w] = f;
    }
    if (nonfinite && !finite) atomicOr(nonfinite, 1u);
}

template <int BS>
__global__ void k_dump_grid(GridTable g, int32_t *cells, float4 *values, uint32_t *count, uint32_t capacity) {
    uint32_t nblocks = min(*g.count, g.max_blocks);
    constexpr int kM = (1 << BS) - 1;
    size_t nodes = static_cast<size_t>(nblocks) << (3 * BS);
    for (size_t node = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; node < nodes;
         node += static_cast<size_t>(gridDim.x) * blockDim.x) {
        float4 mp = g.pool[node];
        if (mp.x == 0.0f) continue;
        uint32_t slot = atomicAdd(count, 1u);
        if (slot >= capacity) continue;
        int4 c = g.coords[node >> (3 * BS)];
        int l = static_cast<int>(node) & ((1 << (3 * BS)) - 1);
        cells[3 * slot] = (c.x << BS) + (l >> (2 * BS));
        cells[3 * slot + 1] = (c.y << BS) + ((l >> BS) & kM);
        cells[3 * slot + 2] = (c.z << BS) + (l & kM);
        values[slot] = mp;
    }
}

__global__ void k_snapshot(ParticleSoA P, int n, const DevClass *__restrict__ classes, float4 *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t cap = P.cap;
    const DevClass &k = classes[P.cls[i] & kClassMask];
    uint32_t w = P.widx[i];
    out[2 * w] = make_float4(P.x[i], P.x[cap + i], P.x[2 * cap + i], k.mass);
    out[2 * w + 1] = make_float4(P.v[i], P.v[cap + i], P.v[2 * cap + i], k.volume);
}

}  // namespace

int device_sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

namespace {
// The fused transfer of one scene as three kernels: the no-record chunks on
// fj.side beside the fast kernel on `stream`, then (after both) the chunks
// the fast kernel deferred.  The deferred kernels run one CTA per SM over
// their lists; an empty list costs one short launch.
void launch_fused(const ParticleSoA &P, int n, const DevClass *classes, const GridTable &cur, const GridTable &next,
                  const SimParams &sp, const DevObstacle *obstacles, const float *planes, double *reactions,
                  uint32_t *status, int *cache, cudaStream_t stream, const ForkJoin &fj) {
    const bool pl = sp.has_plastic != 0;
    const bool obst = sp.num_obstacles > 0;
    const int shape = pl ? 0 : sp.shape;
    const bool big = !pl && sp.block_shift == kBigBlockShift;
    const int sms = device_sm_count();
#define TMPM_FUSED(PL, V, T, B, BS)                                                                                \
    do {                                                                                                           \
        cudaEventRecord(fj.fork, stream);                                                                          \
        cudaStreamWaitEvent(fj.side, fj.fork, 0);                                                                  \
        k_transfer_deferred<true, PL, V, T, BS><<<sms, T, 0, fj.side>>>(P, n, classes, cur, next, sp, obstacles,   \
                                                                        planes, reactions, status, cache);         \
        cudaEventRecord(fj.join, fj.side);                                                                         \
        k_transfer_fast<PL, V, T, B, BS><<<dim3((n + (T) - 1) / (T)), T, 0, stream>>>(                             \
            P, n, classes, cur, next, sp, obstacles, planes, reactions, status, cache);                            \
        cudaStreamWaitEvent(stream, fj.join, 0);                                                                   \
        k_transfer_deferred<false, PL, V, T, BS><<<sms, T, 0, stream>>>(P, n, classes, cur, next, sp, obstacles,   \
                                                                        planes, reactions, status, cache);         \
    } while (0)
#define TMPM_FUSED_SHAPES_BS(V, BS)                                    \
    do {                                                               \
        if (shape == 1) TMPM_FUSED(false, V, 128, 8, BS);              \
        else if (shape == 2) TMPM_FUSED(false, V, 256, 3, BS);         \
        else TMPM_FUSED(false, V, 256, TMPM_TRANSFER_MIN_BLOCKS, BS);  \
    } while (0)
#define TMPM_FUSED_SHAPES(V)                                   \
    do {                                                       \
        if (big) TMPM_FUSED_SHAPES_BS(V, kBigBlockShift);      \
        else TMPM_FUSED_SHAPES_BS(V, kBlockShift);             \
    } while (0)
    if (sp.multi) TMPM_FUSED_SHAPES(kMulti);
    else if (pl) TMPM_FUSED(true, kPlainObst, 256, TMPM_TRANSFER_MIN_BLOCKS, kBlockShift);
    else if (obst) TMPM_FUSED_SHAPES(kPlainObst);
    else TMPM_FUSED_SHAPES(kPlain);
#undef TMPM_FUSED_SHAPES
#undef TMPM_FUSED_SHAPES_BS
#undef TMPM_FUSED
}
}  // namespace

void launch_transfer(int mode, const ParticleSoA &P, int n, const DevClass *classes, const GridTable &cur,
                     const GridTable &next, const SimParams &sp, const DevObstacle *obstacles, const float *planes,
                     double *reactions, uint32_t *status, int *cache, cudaStream_t stream, const ForkJoin *fj) {
    if (n <= 0) return;
    if (mode == kModeG2P2G && fj && sp.defer && !sp.cpic && !(sp.multi && sp.has_plastic)) {
        launch_fused(P, n, classes, cur, next, sp, obstacles, planes, reactions, status, cache, stream, *fj);
        return;
    }
    // Launch shapes other than the default exist for the variants the tuner
    // picks among (no plastic state; one scene or a batch).  Plastic state and
    // CPIC run with the obstacle contact compiled in, with or without obstacles.
    const bool pl = sp.has_plastic != 0;
    const bool obst = sp.num_obstacles > 0;
    // plastic and CPIC variants: default shape and 4^3 blocks only
    const int shape = (pl || sp.cpic) ? 0 : sp.shape;
    const bool big = !(pl || sp.cpic) && sp.block_shift == kBigBlockShift;
#define TMPM_LAUNCH(M, PL, V, T, B, BS) \
    k_transfer<M, PL, V, T, B, BS><<<dim3((n + (T) - 1) / (T)), T, 0, stream>>>(P, n, classes, cur, next, sp, \
                                                                               obstacles, planes, reactions, status, cache)
#define TMPM_LAUNCH_SHAPES_BS(M, V, BS)                                   \
    do {                                                                  \
        if (shape == 1) TMPM_LAUNCH(M, false, V, 128, 8, BS);             \
        else if (shape == 2) TMPM_LAUNCH(M, false, V, 256, 3, BS);        \
        else TMPM_LAUNCH(M, false, V, 256, TMPM_TRANSFER_MIN_BLOCKS, BS); \
    } while (0)
#define TMPM_LAUNCH_SHAPES(M, V)                                \
    do {                                                        \
        if (big) TMPM_LAUNCH_SHAPES_BS(M, V, kBigBlockShift);   \
        else TMPM_LAUNCH_SHAPES_BS(M, V, kBlockShift);          \
    } while (0)
#define TMPM_LAUNCH_MODE(M)                                                                   \
    do {                                                                                      \
        if (sp.multi) {                                                                       \
            if (pl) TMPM_LAUNCH(M, true, kMulti, 256, TMPM_TRANSFER_MIN_BLOCKS, kBlockShift); \
            else TMPM_LAUNCH_SHAPES(M, kMulti);                                               \
        } else if (sp.cpic) {                                                                 \
            if (pl) TMPM_LAUNCH(M, true, kCpic, 256, TMPM_TRANSFER_MIN_BLOCKS, kBlockShift);  \
            else TMPM_LAUNCH(M, false, kCpic, 256, TMPM_TRANSFER_MIN_BLOCKS, kBlockShift);    \
        } else {                                                                              \
            if (pl) TMPM_LAUNCH(M, true, kPlainObst, 256, TMPM_TRANSFER_MIN_BLOCKS, kBlockShift); \
            else if (obst) TMPM_LAUNCH_SHAPES(M, kPlainObst);                                 \
            else TMPM_LAUNCH_SHAPES(M, kPlain);                                               \
        }                                                                                     \
    } while (0)
    switch (mode) {
    case kModeP2G: TMPM_LAUNCH_MODE(kModeP2G); break;
    case kModeG2P2G: TMPM_LAUNCH_MODE(kModeG2P2G); break;
    default: TMPM_LAUNCH_MODE(kModeG2P); break;
    }
#undef TMPM_LAUNCH_MODE
#undef TMPM_LAUNCH_SHAPES
#undef TMPM_LAUNCH_SHAPES_BS
#undef TMPM_LAUNCH
}

void launch_grid_update(const GridTable &g, const GridTable &next, const SimParams &sp, const DevObstacle *obstacles,
                        const float *planes, double *reactions, uint32_t *status, cudaStream_t stream) {
    int blocks = device_sm_count() * 8;
    const bool obst = !sp.multi && sp.num_obstacles > 0;
#define TMPM_GRID(MU, BS, OB) k_grid<MU, BS, OB><<<blocks, 256, 0, stream>>>(g, next, sp, obstacles, planes, reactions, status)
    if (sp.block_shift == kBigBlockShift) {
        if (sp.multi) TMPM_GRID(true, kBigBlockShift, false);
        else if (obst) TMPM_GRID(false, kBigBlockShift, true);
        else TMPM_GRID(false, kBigBlockShift, false);
    } else {
        if (sp.multi) TMPM_GRID(true, kBlockShift, false);
        else if (obst) TMPM_GRID(false, kBlockShift, true);
        else TMPM_GRID(false, kBlockShift, false);
    }
#undef TMPM_GRID
}

namespace {
template <int M, int V, int T, int B, int BS>
void touch_transfer() {
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_transfer<M, false, V, T, B, BS>);
}
template <int V, int T, int B, int BS>
void touch_fused() {
    if constexpr (V == kPlain || V == kPlainObst || V == kMulti) {
        cudaFuncAttributes a;
        cudaFuncGetAttributes(&a, k_transfer_fast<false, V, T, B, BS>);
        cudaFuncGetAttributes(&a, k_transfer_deferred<true, false, V, T, BS>);
        cudaFuncGetAttributes(&a, k_transfer_deferred<false, false, V, T, BS>);
    }
}
template <int V, int BS>
void touch_shapes() {
    touch_fused<V, 256, TMPM_TRANSFER_MIN_BLOCKS, BS>();
    touch_fused<V, 128, 8, BS>();
    touch_fused<V, 256, 3, BS>();
    touch_transfer<kModeP2G, V, 256, TMPM_TRANSFER_MIN_BLOCKS, BS>();
    touch_transfer<kModeG2P2G, V, 256, TMPM_TRANSFER_MIN_BLOCKS, BS>();
    touch_transfer<kModeG2P, V, 256, TMPM_TRANSFER_MIN_BLOCKS, BS>();
    touch_transfer<kModeP2G, V, 128, 8, BS>();
    touch_transfer<kModeG2P2G, V, 128, 8, BS>();
    touch_transfer<kModeG2P, V, 128, 8, BS>();
    touch_transfer<kModeP2G, V, 256, 3, BS>();
    touch_transfer<kModeG2P2G, V, 256, 3, BS>();
    touch_transfer<kModeG2P, V, 256, 3, BS>();
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_grid<V == kMulti, BS, V == kPlainObst>);
}
}  // namespace

void preload_launch_shapes(bool multi, bool obstacles) {
    if (multi) {
        touch_shapes<kMulti, kBlockShift>();
        touch_shapes<kMulti, kBigBlockShift>();
    } else if (obstacles) {
        touch_shapes<kPlainObst, kBlockShift>();
        touch_shapes<kPlainObst, kBigBlockShift>();
    } else {
        touch_shapes<kPlain, kBlockShift>();
        touch_shapes<kPlain, kBigBlockShift>();
    }
    cudaGetLastError();
}

void launch_clear_table(const GridTable &g, const GridTable &other, int block_shift, cudaStream_t stream) {
    int blocks = device_sm_count() * 4;
    k_clear_table<<<blocks, 256, 0, stream>>>(g);
    // new block ids start from zero again: both pools start zero-filled
    const size_t bytes = (static_cast<size_t>(g.max_blocks) << (3 * block_shift)) * sizeof(float4);
    cudaMemsetAsync(g.pool, 0, bytes, stream);
    if (other.pool != g.pool) cudaMemsetAsync(other.pool, 0, bytes, stream);
}

void launch_bin_keys(const ParticleSoA &P, int n, const DevClass *classes, const SimParams &sp, int32_t *cells,
                     uint32_t *keys, cudaStream_t stream) {
    if (n <= 0) return;
    k_bin_keys<<<(n + 255) / 256, 256, 0, stream>>>(P.x, P.cap, n, sp.s0.inv_h, P.cls, classes,
                                                    sp.multi ? sp.scenes : nullptr, cells, keys, nullptr);
}

void launch_bin_keys_values(const float *x, size_t stride, int n, float inv_h, uint32_t *keys, uint32_t *vals,
                            cudaStream_t stream) {
    if (n <= 0) return;
    k_bin_keys<<<(n + 255) / 256, 256, 0, stream>>>(x, stride, n, inv_h, nullptr, nullptr, nullptr, nullptr, keys,
                                                    vals);
}

void launch_resort(ParticleSoA &src, ParticleSoA &dst, int n, int keep, const DevClass *classes, const SimParams &sp,
                   SortBuffers &sb, cudaStream_t stream) {
    if (n <= 0) return;
    k_bin_keys<<<(n + 255) / 256, 256, 0, stream>>>(src.x, src.cap, n, sp.s0.inv_h, src.cls, classes,
                                                    sp.multi ? sp.scenes : nullptr, nullptr, sb.keys[0], sb.vals[0]);
    const int r = radix_sort_pairs(sb, n, sp.multi ? kSortBitsBatch : kSortBitsScene, stream);
    const int interleave = sp.multi ? 0 : kLaunchShapes[sp.shape].threads;
    if (keep > 0) k_gather<<<(keep + 255) / 256, 256, 0, stream>>>(src, dst, sb.vals[r], keep, interleave);
}

void launch_dump_grid(const GridTable &g, int32_t *cells, float4 *values, uint32_t *count, uint32_t capacity,
                      int block_shift, cudaStream_t stream) {
    if (block_shift == kBigBlockShift)
        k_dump_grid<kBigBlockShift><<<device_sm_count() * 4, 256, 0, stream>>>(g, cells, values, count, capacity);
    else
        k_dump_grid<kBlockShift><<<device_sm_count() * 4, 256, 0, stream>>>(g, cells, values, count, capacity);
}

void launch_unsort(const ParticleSoA &P, int n, float *out, size_t stride, cudaStream_t stream, uint32_t *nonfinite) {
    if (n <= 0) return;
    k_unsort<<<(n + 255) / 256, 256, 0, stream>>>(P, n, out, stride, nonfinite);
}

void launch_snapshot(const ParticleSoA &P, int n, const DevClass *classes, float4 *out, cudaStream_t stream) {
    if (n <= 0) return;
    k_snapshot<<<(n + 255) / 256, 256, 0, stream>>>(P, n, classes, out);
}

}  // namespace tmpm
