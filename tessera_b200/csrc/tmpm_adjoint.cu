// tmpm_adjoint.cu -- differentiable rollout of the MLS-MPM substep: forward on
// the device with checkpoints, and a hand-written reverse-mode adjoint of
// G2P, the grid update and P2G (include/tmpm.h, "differentiable rollout").
//
// The forward is the reference substep (world.rs:361-467) for the corotated
// elastic material (material.rs:440-455) in a bounded domain with the
// reference's separating or sticky walls (world.rs:561-575, 632-644), on a
// dense node array covering the domain (the differentiable scenes are small
// and bounded, so no hashing is needed).  The state (x, v, C, F) is stored
// every `checkpoint_every` substeps; the backward pass replays each segment
// from its checkpoint and runs, per substep from last to first,
//   recompute P2G + grid of the substep (node mass, momentum, velocity),
//   G2P adjoint   -> adjoint of the node velocities, partial x and F adjoints,
//   grid adjoint  -> adjoint of node mass and momentum,
//   P2G adjoint   -> adjoint of the substep's input state, and dL/dE.
// The derivative of the polar factor uses, for F = R S and a skew variation
// dR = R [w]x, the identity [w]x S + S [w]x = [(tr(S) I - S) w]x, so the
// adjoint of R is F_bar += 2 R [w]x with (tr(S) I - S) w = axial(skew(R^T R_bar)).
//
// The quadratic B-spline has sum_i grad w_i = 0 and sum_i w_i dpos_i = 0, so
// the adjoint sums sum_i grad w_i s_i and sum_i w_i u_i dpos_i^T see only the
// variation of s and u over the stencil.  A loss gradient that is almost the
// same on every node would make them small differences of large f32 terms;
// they are evaluated as sum_i grad w_i (s_i - s_c) and sum_i w_i (u_i - u_c)
// dpos_i^T with s_c, u_c the values at the stencil's centre node, which is the
// same sum in exact arithmetic.

#include <climits>
#include <memory>

#include "tmpm_device.cuh"
#include "tmpm_host.h"

using namespace tmpm;

namespace {

constexpr int kRows = 24;  // x 0-2, v 3-5, C 6-14, F 15-23 (matrices column-major: col * 3 + row)
constexpr uint32_t kErrGrid = 1u;  // a stencil left the node array


struct AdjParams {
    float h, inv_h, inv_d, dt;
    float gx, gy, gz;
    int wall_mode;
    float bmin[3], bmax[3];
    int wall_lo[3], wall_hi[3];  // wall nodes by index, as SceneParams (f64 thresholds)
    int lo[3], dim[3];  // node array: cells lo .. lo + dim - 1 per axis
    int n;
    size_t stride;      // row stride of state arrays
};

struct Consts {
    const float *mass, *vol, *radius, *damping, *nu;
    const uint8_t *fixed;
};

__device__ __forceinline__ M3f load_m(const float *S, size_t st, int row0, int i) {
    M3f m;
    m.c0 = mk(S[(row0 + 0) * st + i], S[(row0 + 1) * st + i], S[(row0 + 2) * st + i]);
    m.c1 = mk(S[(row0 + 3) * st + i], S[(row0 + 4) * st + i], S[(row0 + 5) * st + i]);
    m.c2 = mk(S[(row0 + 6) * st + i], S[(row0 + 7) * st + i], S[(row0 + 8) * st + i]);
    return m;
}
__device__ __forceinline__ void store_m(float *S, size_t st, int row0, int i, const M3f &m) {
    S[(row0 + 0) * st + i] = m.c0.x;
    S[(row0 + 1) * st + i] = m.c0.y;
    S[(row0 + 2) * st + i] = m.c0.z;
    S[(row0 + 3) * st + i] = m.c1.x;
    S[(row0 + 4) * st + i] = m.c1.y;
    S[(row0 + 5) * st + i] = m.c1.z;
    S[(row0 + 6) * st + i] = m.c2.x;
    S[(row0 + 7) * st + i] = m.c2.y;
    S[(row0 + 8) * st + i] = m.c2.z;
}
__device__ __forceinline__ V3f load_v(const float *S, size_t st, int row0, int i) {
    return mk(S[row0 * st + i], S[(row0 + 1) * st + i], S[(row0 + 2) * st + i]);
}
__device__ __forceinline__ void store_v(float *S, size_t st, int row0, int i, V3f v) {
    S[row0 * st + i] = v.x;
    S[(row0 + 1) * st + i] = v.y;
    S[(row0 + 2) * st + i] = v.z;
}
__device__ __forceinline__ M3f outer(V3f a, V3f b) { return M3f{a * b.x, a * b.y, a * b.z}; }
__device__ __forceinline__ float ddot(const M3f &a, const M3f &b) {
    return dot(a.c0, b.c0) + dot(a.c1, b.c1) + dot(a.c2, b.c2);
}
__device__ __forceinline__ float trace(const M3f &m) { return m.c0.x + m.c1.y + m.c2.z; }
__device__ __forceinline__ M3f skew_of(V3f w) {  // [w]x
    return M3f{mk(0.f, w.z, -w.y), mk(-w.z, 0.f, w.x), mk(w.y, -w.x, 0.f)};
}
// inverse transpose of m (cofactor matrix / det)
__device__ __forceinline__ M3f inv_transpose(const M3f &m, float d) {
    float inv = 1.0f / d;
    return M3f{cross(m.c1, m.c2) * inv, cross(m.c2, m.c0) * inv, cross(m.c0, m.c1) * inv};
}

struct Stencil {
    int b[3];
    float fx[3];
    float w[3][3], dw[3][3];  // [axis][offset]; dw = d w / d fx
};

__device__ __forceinline__ void stencil(V3f x, float inv_h, Stencil &s) {
    const float xs[3] = {x.x, x.y, x.z};
    for (int a = 0; a < 3; ++a) {
        s.b[a] = base_cell(xs[a], inv_h);
        float f = xs[a] * inv_h - static_cast<float>(s.b[a]);
        s.fx[a] = f;
        s.w[a][0] = 0.5f * (1.5f - f) * (1.5f - f);
        s.w[a][1] = 0.75f - (f - 1.0f) * (f - 1.0f);
        s.w[a][2] = 0.5f * (f - 0.5f) * (f - 0.5f);
        s.dw[a][0] = -(1.5f - f);
        s.dw[a][1] = -2.0f * (f - 1.0f);
        s.dw[a][2] = f - 0.5f;
    }
}

// Node index of base + offset, or -1 outside the node array.
__device__ __forceinline__ int node_at(const AdjParams &P, const Stencil &s, int a, int b, int c) {
    int lx = s.b[0] + a - P.lo[0], ly = s.b[1] + b - P.lo[1], lz = s.b[2] + c - P.lo[2];
    if (lx < 0 || ly < 0 || lz < 0 || lx >= P.dim[0] || ly >= P.dim[1] || lz >= P.dim[2]) return -1;
    return (lx * P.dim[1] + ly) * P.dim[2] + lz;
}

// ---- box tiles.  A CTA stages the nodes its particles reach (the box of
// their base cells, 2 cells wider) in shared memory: gathers read the tile
// instead of 27 global loads per particle, scatters accumulate in it in 32-bit
// fixed point (one power-of-two scale per quantity from the CTA's bounds, as in
// the transfer kernels) and flush one float4 atomic per touched node.  A CTA
// whose box does not fit, leaves the node array, or has one particle that
// dominates a bound (above 1/8 of the CTA's total) takes the direct path.
constexpr int kTileThreads = 256;
constexpr int kAdjTile = 2048;  // nodes (32 KB of float4)

struct TileBox {
    int lo[3], dim[3], nodes, ok;
};

// Box of the valid particles' base cells, with the sums and maxima of two
// non-negative bounds over the CTA; one barrier (every warp combines the
// per-warp partials itself).
template <int T>
__device__ void tile_box(const AdjParams &P, bool valid, const int b[3], float &sa, float &sb, float &ma, float &mb,
                         int (*red)[6], float (*redf)[4], TileBox &box) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int r[6];
    for (int a = 0; a < 3; ++a) {
        r[a] = __reduce_min_sync(0xffffffffu, valid ? b[a] : INT_MAX);
        r[3 + a] = __reduce_max_sync(0xffffffffu, valid ? b[a] : INT_MIN);
    }
    float fa = sa, fb = sb;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        fa += __shfl_xor_sync(0xffffffffu, fa, off);
        fb += __shfl_xor_sync(0xffffffffu, fb, off);
    }
    const unsigned xa = __reduce_max_sync(0xffffffffu, __float_as_uint(ma));
    const unsigned xb = __reduce_max_sync(0xffffffffu, __float_as_uint(mb));
    if (lane == 0) {
        for (int a = 0; a < 6; ++a) red[warp][a] = r[a];
        redf[warp][0] = fa;
        redf[warp][1] = fb;
        redf[warp][2] = __uint_as_float(xa);
        redf[warp][3] = __uint_as_float(xb);
    }
    __syncthreads();
    const bool mine = lane < T / 32;
    int m[6];
    for (int a = 0; a < 3; ++a) {
        m[a] = __reduce_min_sync(0xffffffffu, mine ? red[lane][a] : INT_MAX);
        m[3 + a] = __reduce_max_sync(0xffffffffu, mine ? red[lane][3 + a] : INT_MIN);
    }
    fa = mine ? redf[lane][0] : 0.0f;
    fb = mine ? redf[lane][1] : 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        fa += __shfl_xor_sync(0xffffffffu, fa, off);
        fb += __shfl_xor_sync(0xffffffffu, fb, off);
    }
    sa = fa;
    sb = fb;
    ma = __uint_as_float(__reduce_max_sync(0xffffffffu, mine ? __float_as_uint(redf[lane][2]) : 0u));
    mb = __uint_as_float(__reduce_max_sync(0xffffffffu, mine ? __float_as_uint(redf[lane][3]) : 0u));
    bool ok = m[0] <= m[3];
    int nodes = 1;
    for (int a = 0; a < 3 && ok; ++a) {
        box.lo[a] = m[a];
        box.dim[a] = m[3 + a] - m[a] + 3;
        ok = box.dim[a] <= 64 && box.lo[a] >= P.lo[a] && box.lo[a] + box.dim[a] <= P.lo[a] + P.dim[a];
        nodes *= box.dim[a];
    }
    box.nodes = nodes;
    box.ok = ok && nodes <= kAdjTile;
}

// The box's nodes of the dense array `src` into the tile (16-byte cp.async copies), then a barrier.
template <int T>
__device__ void fill_tile(const AdjParams &P, const TileBox &box, const float4 *src, float4 *tile) {
    for (int t = threadIdx.x; t < box.nodes; t += T) {
        const int tz = t % box.dim[2], q = t / box.dim[2];
        const int ty = q % box.dim[1], tx = q / box.dim[1];
        const int id = ((box.lo[0] + tx - P.lo[0]) * P.dim[1] + (box.lo[1] + ty - P.lo[1])) * P.dim[2] +
                       (box.lo[2] + tz - P.lo[2]);
        const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(tile + t));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src + id) : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
}

// Where a particle's 27 nodes are read: the CTA's tile (t0 = the particle's
// base node in it) or, without one, the dense array.
struct TileRef {
    const float4 *tile;
    int t0, d1, d2;
};
__device__ __forceinline__ TileRef tile_ref(const TileBox &box, const Stencil &s, const float4 *tile) {
    TileRef r;
    r.tile = box.ok ? tile : nullptr;
    r.d1 = box.dim[1];
    r.d2 = box.dim[2];
    r.t0 = ((s.b[0] - box.lo[0]) * box.dim[1] + (s.b[1] - box.lo[1])) * box.dim[2] + (s.b[2] - box.lo[2]);
    return r;
}
// TILE: read the CTA's tile (every node of a valid particle is in it);
// otherwise the dense array, where a node outside it reads as absent.
template <bool TILE>
__device__ __forceinline__ bool node_value(const AdjParams &P, const Stencil &s, const float4 *glob, const TileRef &tr,
                                           int a, int b, int c, float4 &g) {
    if (TILE) {
        g = tr.tile[tr.t0 + (a * tr.d1 + b) * tr.d2 + c];
        return true;
    }
    const int id = node_at(P, s, a, b, c);
    if (id < 0) return false;
    g = glob[id];
    return true;
}

// Largest power of two s with total * s <= 2^30 (exponent clamped to the normal range).
__device__ __forceinline__ float pow2_scale30(float total) {
    float e = floorf(30.0f - log2f(fmaxf(total, 1e-30f)));
    e = fminf(fmaxf(e, -120.0f), 120.0f);
    return exp2f(e);
}

// The tile's fixed-point sums (component-major, `comps` of 4) added to the
// dense array: one float4 atomic per node with a non-zero sum.
template <int T>
__device__ void flush_tile(const AdjParams &P, const TileBox &box, int (*sc)[kAdjTile], int comps, float inv0,
                           float inv1, float4 *dst) {
    for (int t = threadIdx.x; t < box.nodes; t += T) {
        const int v0 = sc[0][t], v1 = sc[1][t], v2 = sc[2][t], v3 = comps > 3 ? sc[3][t] : 0;
        if ((v0 | v1 | v2 | v3) == 0) continue;
        const int tz = t % box.dim[2], q = t / box.dim[2];
        const int ty = q % box.dim[1], tx = q / box.dim[1];
        const int id = ((box.lo[0] + tx - P.lo[0]) * P.dim[1] + (box.lo[1] + ty - P.lo[1])) * P.dim[2] +
                       (box.lo[2] + tz - P.lo[2]);
        const float4 val = comps > 3 ? make_float4(v0 * inv0, v1 * inv1, v2 * inv1, v3 * inv1)
                                     : make_float4(v0 * inv0, v1 * inv0, v2 * inv0, 0.0f);
        red_add_v4(dst + id, val);
    }
}

__device__ __forceinline__ unsigned fx_round(float v) { return static_cast<unsigned>(__float2int_rn(v)); }

__device__ __forceinline__ void lame(float E, float nu, float &lambda, float &mu) {
    lambda = E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
    mu = E / (2.0f * (1.0f + nu));
}

// ---------------------------------------------------------------- forward

// Rout (optional): the polar factor R of each particle's F, 9 rows, for the
// P2G adjoint of the same substep.
__global__ void __launch_bounds__(kTileThreads) k_p2g(AdjParams P, Consts K, const float *__restrict__ S,
                                                      const float *__restrict__ E, float4 *grid, uint32_t *err,
                                                      float *__restrict__ Rout) {
    __shared__ float4 s_tile[kAdjTile];
    __shared__ int s_red[kTileThreads / 32][6];
    __shared__ float s_redf[kTileThreads / 32][4];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    const int ic = valid ? i : 0;
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, ic), v = load_v(S, st, 3, ic);
    M3f C = load_m(S, st, 6, ic), F = load_m(S, st, 15, ic);
    float lambda, mu;
    lame(E[ic], K.nu[ic], lambda, mu);
    M3f R = polar_rotation(F);
    if (Rout && valid) {
        const M3f &Rs = R;
        Rout[0 * st + i] = Rs.c0.x;
        Rout[1 * st + i] = Rs.c0.y;
        Rout[2 * st + i] = Rs.c0.z;
        Rout[3 * st + i] = Rs.c1.x;
        Rout[4 * st + i] = Rs.c1.y;
        Rout[5 * st + i] = Rs.c1.z;
        Rout[6 * st + i] = Rs.c2.x;
        Rout[7 * st + i] = Rs.c2.y;
        Rout[8 * st + i] = Rs.c2.z;
    }
    float J = det(F);
    M3f tau = scale(mul_bt(sub(F, R), F), 2.0f * mu);
    float iso = lambda * (J - 1.0f) * J;
    tau.c0.x += iso;
    tau.c1.y += iso;
    tau.c2.z += iso;
    const float m = K.mass[ic];
    M3f A = add(scale(tau, -P.dt * K.vol[ic] * P.inv_d), scale(C, m));
    Stencil s;
    stencil(x, P.inv_h, s);
    // node sums are bounded by the CTA's sums of m and |m v| + 1.5 h sum |A| (weights sum to one)
    float bm = 0.0f, bp = 0.0f;
    if (valid) {
        const V3f mv = v * m;
        bm = m;
        bp = fmaxf(fmaxf(fabsf(mv.x) + 1.5f * P.h * (fabsf(A.c0.x) + fabsf(A.c1.x) + fabsf(A.c2.x)),
                         fabsf(mv.y) + 1.5f * P.h * (fabsf(A.c0.y) + fabsf(A.c1.y) + fabsf(A.c2.y))),
                   fabsf(mv.z) + 1.5f * P.h * (fabsf(A.c0.z) + fabsf(A.c1.z) + fabsf(A.c2.z)));
        if (!(bp < 1e30f)) bp = 1e30f;
    }
    float sum_m = bm, sum_p = bp, max_m = bm, max_p = bp;
    TileBox box;
    tile_box<kTileThreads>(P, valid, s.b, sum_m, sum_p, max_m, max_p, s_red, s_redf, box);
    if (!box.ok || max_m > 0.125f * sum_m || max_p > 0.125f * sum_p) {  // direct path (CTA-uniform)
        if (!valid) return;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) {
                    int id = node_at(P, s, a, b, c);
                    if (id < 0) {
                        atomicOr(err, kErrGrid);
                        continue;
                    }
                    float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                    V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                    V3f mom = v * m + mul(A, dpos);
                    red_add_v4(grid + id, make_float4(w * m, w * mom.x, w * mom.y, w * mom.z));
                }
        return;
    }
    int (*sc)[kAdjTile] = reinterpret_cast<int (*)[kAdjTile]>(s_tile);
    for (int t = threadIdx.x; t < box.nodes; t += kTileThreads) sc[0][t] = sc[1][t] = sc[2][t] = sc[3][t] = 0;
    __syncthreads();
    const float sm = pow2_scale30(sum_m), sp = pow2_scale30(sum_p);
    if (valid) {
        const TileRef tr = tile_ref(box, s, s_tile);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int t = tr.t0 + (a * tr.d1 + b) * tr.d2 + c;
                    float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                    V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                    V3f mom = (v * m + mul(A, dpos)) * (w * sp);
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[0][t]), fx_round(w * m * sm));
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[1][t]), fx_round(mom.x));
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[2][t]), fx_round(mom.y));
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[3][t]), fx_round(mom.z));
                }
    }
    __syncthreads();
    flush_tile<kTileThreads>(P, box, sc, 4, 1.0f / sm, 1.0f / sp, grid);
}

// Node velocity with the wall rule; w = bitmask of the components the walls zeroed.
__device__ __forceinline__ float4 node_velocity(const AdjParams &P, int node, float4 mp) {
    int lz = node % P.dim[2], ly = (node / P.dim[2]) % P.dim[1], lx = node / (P.dim[2] * P.dim[1]);
    const int id[3] = {lx + P.lo[0], ly + P.lo[1], lz + P.lo[2]};
    float v[3] = {mp.y / mp.x + P.gx * P.dt, mp.z / mp.x + P.gy * P.dt, mp.w / mp.x + P.gz * P.dt};
    int mask = 0;
    for (int a = 0; a < 3; ++a) {
        const bool lower = id[a] <= P.wall_lo[a], upper = id[a] >= P.wall_hi[a];
        if (P.wall_mode == 1) {
            if (lower || upper) mask = 7;
        } else if ((lower && v[a] < 0.0f) || (upper && v[a] > 0.0f)) {
            mask |= 1 << a;
        }
    }
    for (int a = 0; a < 3; ++a)
        if (mask & (1 << a)) v[a] = 0.0f;
    return make_float4(v[0], v[1], v[2], static_cast<float>(mask));
}

__global__ void k_grid(AdjParams P, const float4 *__restrict__ grid, float4 *gv, int nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    float4 mp = grid[i];
    gv[i] = mp.x > 0.0f ? node_velocity(P, i, mp) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// Gather of one particle: velocity, affine matrix (4/h^2 sum w v dpos^T).
// The 27 nodes' loads are independent: unrolled, they are issued together.
template <bool TILE>
__device__ __forceinline__ void gather_nodes(const AdjParams &P, const Stencil &s, const float4 *gv, const TileRef &tr,
                                             V3f &vel, M3f &aff) {
    vel = mk(0, 0, 0);
    aff = m3_zero();
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float4 g;
                if (!node_value<TILE>(P, s, gv, tr, a, b, c, g)) continue;
                float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                V3f nv = mk(g.x, g.y, g.z);
                V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                vel = vel + nv * w;
                aff = add(aff, scale(outer(nv, dpos), w * P.inv_d));
            }
}
__device__ __forceinline__ void gather(const AdjParams &P, const Stencil &s, const float4 *gv, const TileRef &tr,
                                       V3f &vel, M3f &aff) {
    if (tr.tile) gather_nodes<true>(P, s, gv, tr, vel, aff);
    else gather_nodes<false>(P, s, gv, tr, vel, aff);
}

__global__ void __launch_bounds__(kTileThreads) k_g2p(AdjParams P, Consts K, const float *__restrict__ S,
                                                      float *__restrict__ Sn, const float4 *__restrict__ gv) {
    __shared__ float4 s_tile[kAdjTile];
    __shared__ int s_red[kTileThreads / 32][6];
    __shared__ float s_redf[kTileThreads / 32][4];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, valid ? i : 0);
    Stencil s;
    stencil(x, P.inv_h, s);
    float z0 = 0.f, z1 = 0.f, z2 = 0.f, z3 = 0.f;
    TileBox box;
    tile_box<kTileThreads>(P, valid, s.b, z0, z1, z2, z3, s_red, s_redf, box);
    if (box.ok) fill_tile<kTileThreads>(P, box, gv, s_tile);
    if (!valid) return;
    M3f F = load_m(S, st, 15, i);
    if (K.fixed[i]) {
        store_v(Sn, st, 0, i, x);
        store_v(Sn, st, 3, i, mk(0, 0, 0));
        store_m(Sn, st, 6, i, m3_zero());
        store_m(Sn, st, 15, i, F);
        return;
    }
    V3f vel;
    M3f aff;
    gather(P, s, gv, tile_ref(box, s, s_tile), vel, aff);
    vel = vel * expf(-K.damping[i] * P.dt);
    V3f pos = x + vel * P.dt;
    M3f Fn = mul(add(m3_identity(), scale(aff, P.dt)), F);
    const float r = K.radius[i];
    for (int a = 0; a < 3; ++a) {
        float lower = P.bmin[a] + r, upper = P.bmax[a] - r;
        float pa = comp(pos, a), va = comp(vel, a);
        if (pa < lower) {
            set_comp(pos, a, lower);
            set_comp(vel, a, fmaxf(va, 0.0f));
        } else if (pa > upper) {
            set_comp(pos, a, upper);
            set_comp(vel, a, fminf(va, 0.0f));
        }
    }
    store_v(Sn, st, 0, i, pos);
    store_v(Sn, st, 3, i, vel);
    store_m(Sn, st, 6, i, aff);
    store_m(Sn, st, 15, i, Fn);
}

// ---------------------------------------------------------------- adjoint

// G2P adjoint.  In: the substep's input state S, node velocities gv, the
// adjoint Ab of the substep's output state.  Out: partial adjoints of x and F
// (rows 0-2 and 15-23 of Q) and the node-velocity adjoint gvb (atomics).
// The position adjoint's node sum of the G2P adjoint (unrolled: the 27 node
// loads are independent).
template <bool TILE>
__device__ __forceinline__ void xbar_nodes(const AdjParams &P, const Stencil &s, const float4 *gv, const TileRef &tr,
                                           V3f velb, const M3f &Cb, V3f &xbar) {
    const M3f CbT = transpose(Cb);
    V3f nv_c = mk(0, 0, 0);
    {
        float4 g;
        if (node_value<TILE>(P, s, gv, tr, 1, 1, 1, g)) nv_c = mk(g.x, g.y, g.z);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float4 g;
                if (!node_value<TILE>(P, s, gv, tr, a, b, c, g)) continue;
                float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                V3f dw = mk(s.dw[0][a] * s.w[1][b] * s.w[2][c], s.w[0][a] * s.dw[1][b] * s.w[2][c],
                            s.w[0][a] * s.w[1][b] * s.dw[2][c]) * P.inv_h;
                V3f nv = mk(g.x, g.y, g.z);
                V3f dnv = nv - nv_c;
                V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                V3f Cd = mul(Cb, dpos);
                // grad w (v_i . velb + v_i . C_b dpos_i) - w C_b^T v_i with v_i -> v_i - v_c (file header)
                float gs = dot(dnv, velb) + P.inv_d * dot(dnv, Cd);
                xbar = xbar + dw * gs - mul(CbT, dnv) * (P.inv_d * w);
            }
}

// The P2G adjoint's node sums: velocity and affine adjoints, position adjoint.
template <bool TILE>
__device__ __forceinline__ void p2g_back_nodes(const AdjParams &P, const Stencil &s, const float4 *gmb,
                                               const TileRef &tr, float m, V3f v, const M3f &A, V3f &vbar,
                                               M3f &Abar, V3f &xbar) {
    const M3f AT = transpose(A);
    float4 gc = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!node_value<TILE>(P, s, gmb, tr, 1, 1, 1, gc)) gc = make_float4(0.f, 0.f, 0.f, 0.f);
    const V3f pb_c = mk(gc.y, gc.z, gc.w);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float4 g;
                if (!node_value<TILE>(P, s, gmb, tr, a, b, c, g)) continue;
                float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                V3f dw = mk(s.dw[0][a] * s.w[1][b] * s.w[2][c], s.w[0][a] * s.dw[1][b] * s.w[2][c],
                            s.w[0][a] * s.w[1][b] * s.dw[2][c]) * P.inv_h;
                V3f pb = mk(g.y, g.z, g.w);
                V3f dpb = pb - pb_c;
                V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                // grad w (m m_b + p_b . (m v + A dpos)) - w A^T p_b with m_b, p_b -> minus their centre values
                vbar = vbar + pb * (w * m);
                Abar = add(Abar, scale(outer(dpb, dpos), w));
                xbar = xbar + dw * (m * (g.x - gc.x) + m * dot(v, dpb) + dot(dpb, mul(A, dpos))) - mul(AT, dpb) * w;
            }
}

__global__ void __launch_bounds__(kTileThreads) k_g2p_back(AdjParams P, Consts K, const float *__restrict__ S,
                                                           const float4 *__restrict__ gv, const float *__restrict__ Ab,
                                                           float *__restrict__ Q, float4 *gvb) {
    __shared__ float4 s_tile[kAdjTile];
    __shared__ int s_red[kTileThreads / 32][6];
    __shared__ float s_redf[kTileThreads / 32][4];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    const int ic = valid ? i : 0;
    const bool active = valid && !K.fixed[ic];
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, ic);
    Stencil s;
    stencil(x, P.inv_h, s);
    float z0 = 0.f, z1 = 0.f, z2 = 0.f, z3 = 0.f;
    TileBox box;
    tile_box<kTileThreads>(P, valid, s.b, z0, z1, z2, z3, s_red, s_redf, box);
    if (box.ok) fill_tile<kTileThreads>(P, box, gv, s_tile);
    const TileRef tr = tile_ref(box, s, s_tile);
    V3f velb = mk(0, 0, 0);
    M3f Cb = m3_zero();
    float bg = 0.0f;  // bound of the particle's velocity-adjoint contributions
    if (valid) {
        M3f F = load_m(S, st, 15, i);
        V3f xb_o = load_v(Ab, st, 0, i), vb_o = load_v(Ab, st, 3, i);
        M3f Cb_o = load_m(Ab, st, 6, i), Fb_o = load_m(Ab, st, 15, i);
        if (!active) {  // x and F pass through; v and C are reset
            store_v(Q, st, 0, i, xb_o);
            store_m(Q, st, 15, i, Fb_o);
        } else {
            V3f vel;
            M3f aff;
            gather(P, s, gv, tr, vel, aff);
            const float ed = expf(-K.damping[i] * P.dt);
            V3f veld = vel * ed;
            V3f pos = x + veld * P.dt;
            const float r = K.radius[i];
            V3f xb = xb_o;
            velb = vb_o;
            for (int a = 0; a < 3; ++a) {
                float lower = P.bmin[a] + r, upper = P.bmax[a] - r;
                float pa = comp(pos, a), va = comp(veld, a);
                if (pa < lower) {
                    set_comp(xb, a, 0.0f);
                    if (!(va > 0.0f)) set_comp(velb, a, 0.0f);
                } else if (pa > upper) {
                    set_comp(xb, a, 0.0f);
                    if (!(va < 0.0f)) set_comp(velb, a, 0.0f);
                }
            }
            velb = (velb + xb * P.dt) * ed;                       // pos = x + dt v_damped
            Cb = add(Cb_o, scale(mul_bt(Fb_o, F), P.dt));         // Fn = (I + dt C) F
            M3f Fb = mul(transpose(add(m3_identity(), scale(aff, P.dt))), Fb_o);
            V3f xbar = xb;
            if (tr.tile) xbar_nodes<true>(P, s, gv, tr, velb, Cb, xbar);
            else xbar_nodes<false>(P, s, gv, tr, velb, Cb, xbar);
            store_v(Q, st, 0, i, xbar);
            store_m(Q, st, 15, i, Fb);
            // |gb_k| <= w (|velb_k| + 4/h^2 * 1.5 h sum_j |Cb_kj|), and the weights sum to one
            const float q = P.inv_d * 1.5f * P.h;
            bg = fmaxf(fmaxf(fabsf(velb.x) + q * (fabsf(Cb.c0.x) + fabsf(Cb.c1.x) + fabsf(Cb.c2.x)),
                             fabsf(velb.y) + q * (fabsf(Cb.c0.y) + fabsf(Cb.c1.y) + fabsf(Cb.c2.y))),
                       fabsf(velb.z) + q * (fabsf(Cb.c0.z) + fabsf(Cb.c1.z) + fabsf(Cb.c2.z)));
            if (!(bg < 1e30f)) bg = 1e30f;
        }
    }
    // the velocity-adjoint scatter; the reduction's barrier also ends every read of the gv tile
    float sum_g = bg, sum_0 = 0.0f, max_g = bg, max_0 = 0.0f;
    TileBox box2;
    tile_box<kTileThreads>(P, active, s.b, sum_g, sum_0, max_g, max_0, s_red, s_redf, box2);
    const bool tiled = box.ok && !(max_g > 0.125f * sum_g);
    if (!tiled) {
        if (!active) return;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) {
                    int id = node_at(P, s, a, b, c);
                    if (id < 0) continue;
                    float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                    V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                    V3f gb = velb * w + mul(Cb, dpos) * (P.inv_d * w);
                    red_add_v4(gvb + id, make_float4(gb.x, gb.y, gb.z, 0.0f));
                }
        return;
    }
    int (*sc)[kAdjTile] = reinterpret_cast<int (*)[kAdjTile]>(s_tile);
    for (int t = threadIdx.x; t < box.nodes; t += kTileThreads) sc[0][t] = sc[1][t] = sc[2][t] = 0;
    __syncthreads();
    const float sg = pow2_scale30(sum_g);
    if (active) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int t = tr.t0 + (a * tr.d1 + b) * tr.d2 + c;
                    float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                    V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                    V3f gb = (velb + mul(Cb, dpos) * P.inv_d) * (w * sg);
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[0][t]), fx_round(gb.x));
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[1][t]), fx_round(gb.y));
                    atomicAdd(reinterpret_cast<unsigned *>(&sc[2][t]), fx_round(gb.z));
                }
    }
    __syncthreads();
    flush_tile<kTileThreads>(P, box, sc, 3, 1.0f / sg, 1.0f / sg, gvb);
}

// Grid adjoint: node velocity v = p / m + g dt (walls zero some components).
// In place: gvb (velocity adjoint) becomes (m_bar, p_bar).
__global__ void k_grid_back(AdjParams P, const float4 *__restrict__ grid, const float4 *__restrict__ gv, float4 *gvb,
                            int nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    float4 mp = grid[i];
    if (!(mp.x > 0.0f)) {
        gvb[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    float4 b = gvb[i];
    int mask = static_cast<int>(gv[i].w);
    if (mask & 1) b.x = 0.0f;
    if (mask & 2) b.y = 0.0f;
    if (mask & 4) b.z = 0.0f;
    float inv_m = 1.0f / mp.x;
    float mbar = -(b.x * mp.y + b.y * mp.z + b.z * mp.w) * inv_m * inv_m;
    gvb[i] = make_float4(mbar, b.x * inv_m, b.y * inv_m, b.z * inv_m);
}

// P2G adjoint.  In: the substep's input state S, node (m_bar, p_bar), partial
// adjoints Q from the G2P adjoint.  Out: the adjoint of the substep's input
// state (Ain) and dL/dE accumulated into Eb.
__global__ void __launch_bounds__(kTileThreads) k_p2g_back(AdjParams P, Consts K, const float *__restrict__ S,
                                                           const float *__restrict__ E, const float4 *__restrict__ gmb,
                                                           const float *__restrict__ Q, float *__restrict__ Ain,
                                                           float *__restrict__ Eb, const float *__restrict__ Rin) {
    __shared__ float4 s_tile[kAdjTile];
    __shared__ int s_red[kTileThreads / 32][6];
    __shared__ float s_redf[kTileThreads / 32][4];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    const size_t st = P.stride;
    const V3f x = load_v(S, st, 0, valid ? i : 0);
    Stencil s;
    stencil(x, P.inv_h, s);
    float z0 = 0.f, z1 = 0.f, z2 = 0.f, z3 = 0.f;
    TileBox box;
    tile_box<kTileThreads>(P, valid, s.b, z0, z1, z2, z3, s_red, s_redf, box);
    if (box.ok) fill_tile<kTileThreads>(P, box, gmb, s_tile);
    if (!valid) return;
    const TileRef tr = tile_ref(box, s, s_tile);
    V3f v = load_v(S, st, 3, i);
    M3f C = load_m(S, st, 6, i), F = load_m(S, st, 15, i);
    const float m = K.mass[i];
    float lambda, mu;
    const float nu = K.nu[i];
    lame(E[i], nu, lambda, mu);
    const M3f R = load_m(Rin, st, 0, i);  // the polar factor the replayed P2G computed
    float J = det(F);
    M3f FmR_FT = mul_bt(sub(F, R), F);
    M3f tau = scale(FmR_FT, 2.0f * mu);
    float iso = lambda * (J - 1.0f) * J;
    tau.c0.x += iso;
    tau.c1.y += iso;
    tau.c2.z += iso;
    const float sc = -P.dt * K.vol[i] * P.inv_d;
    M3f A = add(scale(tau, sc), scale(C, m));
    V3f xbar = load_v(Q, st, 0, i);
    M3f Fbar = load_m(Q, st, 15, i);
    V3f vbar = mk(0, 0, 0);
    M3f Abar = m3_zero();
    if (tr.tile) p2g_back_nodes<true>(P, s, gmb, tr, m, v, A, vbar, Abar, xbar);
    else p2g_back_nodes<false>(P, s, gmb, tr, m, v, A, vbar, Abar, xbar);
    M3f Cbar = scale(Abar, m);
    M3f taub = scale(Abar, sc);
    float trt = trace(taub);
    float mub = 2.0f * ddot(taub, FmR_FT);
    float lamb = (J - 1.0f) * J * trt;
    // d tau / d F: 2 mu (F F^T - R F^T) + lambda (J^2 - J) I
    M3f tauT = transpose(taub);
    Fbar = add(Fbar, scale(mul(add(taub, tauT), F), 2.0f * mu));
    Fbar = sub(Fbar, scale(mul(tauT, R), 2.0f * mu));
    M3f Rb = scale(mul(taub, F), -2.0f * mu);
    M3f Sm = mul(transpose(R), F);
    M3f Ssym = scale(add(Sm, transpose(Sm)), 0.5f);
    M3f G = mul(transpose(R), Rb);
    // axial vector of skew(G) = (G - G^T) / 2
    V3f kx = mk(0.5f * (G.c1.z - G.c2.y), 0.5f * (G.c2.x - G.c0.z), 0.5f * (G.c0.y - G.c1.x));
    M3f Mx = scale(Ssym, -1.0f);
    float tS = trace(Ssym);
    Mx.c0.x += tS;
    Mx.c1.y += tS;
    Mx.c2.z += tS;
    float dM = det(Mx);
    V3f om = mul(transpose(inv_transpose(Mx, dM)), kx);  // Mx^-1 k
    Fbar = add(Fbar, scale(mul(R, skew_of(om)), 2.0f));
    Fbar = add(Fbar, scale(inv_transpose(F, J), lambda * (2.0f * J - 1.0f) * trt * J));
    store_v(Ain, st, 0, i, xbar);
    store_v(Ain, st, 3, i, vbar);
    store_m(Ain, st, 6, i, Cbar);
    store_m(Ain, st, 15, i, Fbar);
    Eb[i] += lamb * nu / ((1.0f + nu) * (1.0f - 2.0f * nu)) + mub / (2.0f * (1.0f + nu));
}

}  // namespace

struct TmpmAdjoint {
    int device = 0;
    cudaStream_t stream = nullptr;
    TmpmParams params{};
    double dt = 0.0;
    uint32_t substeps = 0, every = 16;
    HostWorld world;     // initial state (velocity and E replaced per forward)
    size_t n = 0;
    AdjParams P{};
    int nodes = 0;
    DevBuf<float> mass, vol, radius, damping, nu, E, Ebar;
    DevBuf<uint8_t> fixed;
    DevBuf<float> ckpt, adj[2], part;
    DevBuf<float4> grid, gv, gvb;
    // Two buffer sets for replayed segments (segment sg uses set sg & 1): per
    // substep of the segment, its state, the grid after P2G (mass and
    // momentum), the node velocities and the particles' polar factors, so the
    // adjoint sweep reuses them instead of recomputing P2G and the grid
    // update.  The forward ping-pongs between the first two states of set 0.
    DevBuf<float> seg[2];
    DevBuf<float4> seg_grid[2], seg_gv[2];
    DevBuf<float> seg_R[2];
    DevBuf<uint32_t> err;
    bool have_forward = false;
    std::string last_error;
    // The forward and adjoint sweeps (fixed launches over fixed buffers) are
    // captured as CUDA graphs on first use and replayed afterwards.
    cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;
    // The adjoint sweep replays segment sg - 1 on `side` while `stream` runs the
    // adjoint of segment sg: at the sizes this rollout is built for, each
    // kernel fills less than one wave of the GPU, so the two overlap.
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_replayed = nullptr, ev_swept = nullptr;

    ~TmpmAdjoint() {
        if (stream) cudaStreamSynchronize(stream);
        if (side) cudaStreamSynchronize(side);
        if (fwd_exec) cudaGraphExecDestroy(fwd_exec);
        if (bwd_exec) cudaGraphExecDestroy(bwd_exec);
        for (cudaEvent_t ev : {ev_fork, ev_replayed, ev_swept})
            if (ev) cudaEventDestroy(ev);
        if (side) cudaStreamDestroy(side);
        if (stream) cudaStreamDestroy(stream);
    }

    // Capture `launch` (stream work only) into *exec once, then launch it.
    template <typename Fn>
    cudaError_t replay(cudaGraphExec_t *exec, Fn launch) {
        cudaError_t e;
        if (!*exec) {
            cudaGraph_t g = nullptr;
            if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal))) return e;
            launch();
            if ((e = cudaStreamEndCapture(stream, &g))) return e;
            e = cudaGraphInstantiate(exec, g, 0);
            cudaGraphDestroy(g);
            if (e) {
                *exec = nullptr;
                return e;
            }
        }
        return cudaGraphLaunch(*exec, stream);
    }

    // The forward sweep: `substeps` substeps from seg[0] (its first state)
    // ping-ponging with its second state, a checkpoint every `every`.
    void forward_sweep() {
        float *cur = seg[0].ptr, *nxt = seg[0].ptr + state_floats();
        for (uint32_t s = 0; s < substeps; ++s) {
            if (s % every == 0)
                cudaMemcpyAsync(ckpt.ptr + (s / every) * state_floats(), cur, sizeof(float) * state_floats(),
                                cudaMemcpyDeviceToDevice, stream);
            substep(cur, nxt);
            std::swap(cur, nxt);
        }
    }

    // Replay segment sg from its checkpoint into buffer set sg & 1 on stream st:
    // per substep j its state, grid, node velocities and polar factors.
    void replay_segment(int sg, cudaStream_t st) {
        const int set = sg & 1;
        const uint32_t s0 = sg * every, s1 = std::min(substeps, s0 + every);
        float *S = seg[set].ptr;
        cudaMemcpyAsync(S, ckpt.ptr + sg * state_floats(), sizeof(float) * state_floats(), cudaMemcpyDeviceToDevice,
                        st);
        for (uint32_t s = s0; s < s1; ++s) {
            const uint32_t j = s - s0;
            float4 *g = seg_grid[set].ptr + static_cast<size_t>(j) * nodes;
            float4 *v = seg_gv[set].ptr + static_cast<size_t>(j) * nodes;
            p2g_grid(S + j * state_floats(), g, v, seg_R[set].ptr + static_cast<size_t>(j) * 9 * n, st);
            if (s + 1 < s1)
                k_g2p<<<blocks_n(), kTileThreads, 0, st>>>(P, consts(), S + j * state_floats(),
                                                           S + (j + 1) * state_floats(), v);
        }
    }

    // The adjoint of segment sg (replayed into set sg & 1), substep by substep
    // from its last; `a` is the adj buffer holding the adjoint of its final state.
    void sweep_segment(int sg, int &a) {
        const int set = sg & 1;
        const uint32_t s0 = sg * every, s1 = std::min(substeps, s0 + every);
        for (int s = static_cast<int>(s1) - 1; s >= static_cast<int>(s0); --s) {
            const uint32_t j = s - s0;
            const float *S = seg[set].ptr + j * state_floats();
            const float4 *g = seg_grid[set].ptr + static_cast<size_t>(j) * nodes;
            const float4 *v = seg_gv[set].ptr + static_cast<size_t>(j) * nodes;
            cudaMemsetAsync(gvb.ptr, 0, sizeof(float4) * nodes, stream);
            k_g2p_back<<<blocks_n(), kTileThreads, 0, stream>>>(P, consts(), S, v, adj[a].ptr, part.ptr, gvb.ptr);
            k_grid_back<<<blocks_nodes(), 256, 0, stream>>>(P, g, v, gvb.ptr, nodes);
            k_p2g_back<<<blocks_n(), kTileThreads, 0, stream>>>(P, consts(), S, E.ptr, gvb.ptr, part.ptr, adj[a ^ 1].ptr,
                                                                Ebar.ptr, seg_R[set].ptr + static_cast<size_t>(j) * 9 * n);
            a ^= 1;
        }
    }

    // The adjoint sweep from adj[0] (the loss gradient of the final state),
    // segment by segment from the last checkpoint back; the initial-state
    // adjoint ends in adj[substeps & 1].  Segment sg - 1 is replayed on `side`
    // while `stream` sweeps segment sg; the replay into a set waits for the
    // sweep that last read it (segment sg + 1), and each sweep for its replay.
    void backward_sweep() {
        int a = 0;
        const int segments = static_cast<int>((substeps + every - 1) / every);
        cudaEventRecord(ev_fork, stream);
        cudaStreamWaitEvent(side, ev_fork, 0);
        replay_segment(segments - 1, side);
        cudaEventRecord(ev_replayed, side);
        for (int sg = segments - 1; sg >= 0; --sg) {
            cudaStreamWaitEvent(stream, ev_replayed, 0);
            if (sg >= 1) {
                if (sg + 1 < segments) cudaStreamWaitEvent(side, ev_swept, 0);
                replay_segment(sg - 1, side);
                cudaEventRecord(ev_replayed, side);
            }
            sweep_segment(sg, a);
            cudaEventRecord(ev_swept, stream);
        }
        // every replay on `side` ends before a sweep that `stream` waits for
    }
    TmpmStatus fail(TmpmStatus st, const std::string &msg) {
        last_error = msg;
        g_last_error = msg;
        return st;
    }
    TmpmStatus cuda_fail(cudaError_t e, const char *what) {
        return fail(TMPM_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
    }
    Consts consts() const { return Consts{mass.ptr, vol.ptr, radius.ptr, damping.ptr, nu.ptr, fixed.ptr}; }
    size_t state_floats() const { return kRows * n; }
    int blocks_n() const { return static_cast<int>((n + kTileThreads - 1) / kTileThreads); }
    int blocks_nodes() const { return (nodes + 255) / 256; }

    // P2G + grid of state S into g / v (and the polar factors into R when given).
    void p2g_grid(const float *S, float4 *g, float4 *v, float *R, cudaStream_t st) {
        cudaMemsetAsync(g, 0, sizeof(float4) * nodes, st);
        k_p2g<<<blocks_n(), kTileThreads, 0, st>>>(P, consts(), S, E.ptr, g, err.ptr, R);
        k_grid<<<blocks_nodes(), 256, 0, st>>>(P, g, v, nodes);
    }
    void substep(const float *S, float *Sn) {
        p2g_grid(S, grid.ptr, gv.ptr, nullptr, stream);
        k_g2p<<<blocks_n(), kTileThreads, 0, stream>>>(P, consts(), S, Sn, gv.ptr);
    }

    TmpmStatus check_err() {
        uint32_t e = 0;
        cudaError_t ce = cudaMemcpy(&e, err.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (ce) return cuda_fail(ce, "adjoint status");
        if (e & kErrGrid) return fail(TMPM_ERR_CAPACITY, "a particle stencil left the domain's node array");
        return TMPM_OK;
    }

    TmpmStatus forward(const double *v0, const double *young, double *x_out, double *v_out) {
        // inputs -> the host world (for the CFL check) and the device initial state
        std::vector<float> Ef(n);
        ++world.version;
        for (size_t i = 0; i < n; ++i) {
            double e = young ? young[i] : world.mparams[5 * i];
            if (!std::isfinite(e) || !(e > 0.0)) return fail(TMPM_ERR_MPM_INVALID_INPUT, "young's modulus must be positive");
            world.mparams[5 * i] = e;
            Ef[i] = static_cast<float>(e);
            if (v0)
                for (int k = 0; k < 3; ++k) world.vel[3 * i + k] = v0[3 * i + k];
        }
        for (size_t i = 0; i < n; ++i)
            if (!valid_particle(world, i)) return fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM input");
        if (dt > stable_timestep(world, params))
            return fail(TMPM_ERR_INVALID_INPUT, "substep dt is above the CFL bound for these inputs");
        std::vector<float> S0(state_floats());
        for (size_t i = 0; i < n; ++i) {
            for (int k = 0; k < 3; ++k) {
                S0[k * n + i] = static_cast<float>(world.pos[3 * i + k]);
                S0[(3 + k) * n + i] = static_cast<float>(world.vel[3 * i + k]);
            }
            for (int k = 0; k < 9; ++k) {
                S0[(6 + k) * n + i] = static_cast<float>(world.C[9 * i + k]);
                S0[(15 + k) * n + i] = static_cast<float>(world.F[9 * i + k]);
            }
        }
        cudaError_t e;
        if ((e = cudaMemcpyAsync(E.ptr, Ef.data(), sizeof(float) * n, cudaMemcpyHostToDevice, stream)) ||
            (e = cudaMemcpyAsync(seg[0].ptr, S0.data(), sizeof(float) * state_floats(), cudaMemcpyHostToDevice, stream)) ||
            (e = cudaMemsetAsync(err.ptr, 0, sizeof(uint32_t), stream)))
            return cuda_fail(e, "adjoint upload");
        // seg[0] holds two ping-pong states during the forward; the final state
        // is in the first of them after an even number of substeps
        if ((e = replay(&fwd_exec, [&]() { forward_sweep(); }))) return cuda_fail(e, "adjoint forward");
        const float *cur = (substeps % 2 == 0) ? seg[0].ptr : seg[0].ptr + state_floats();
        std::vector<float> out(6 * n);
        if ((e = cudaMemcpyAsync(out.data(), cur, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost, stream)) ||
            (e = cudaStreamSynchronize(stream)))
            return cuda_fail(e, "adjoint forward");
        TmpmStatus st = check_err();
        if (st != TMPM_OK) return st;
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                float xv = out[k * n + i], vv = out[(3 + k) * n + i];
                if (!std::isfinite(xv) || !std::isfinite(vv))
                    return fail(TMPM_ERR_NON_FINITE_STATE, "MPM integration produced a non-finite state");
                if (x_out) x_out[3 * i + k] = xv;
                if (v_out) v_out[3 * i + k] = vv;
            }
        have_forward = true;
        return TMPM_OK;
    }

    TmpmStatus backward(const double *x_grad, const double *v_grad, double *v0_grad, double *young_grad) {
        if (!have_forward) return fail(TMPM_ERR_INVALID_INPUT, "backward needs a forward run first");
        std::vector<float> A0(state_floats(), 0.0f);
        for (size_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
                A0[k * n + i] = x_grad ? static_cast<float>(x_grad[3 * i + k]) : 0.0f;
                A0[(3 + k) * n + i] = v_grad ? static_cast<float>(v_grad[3 * i + k]) : 0.0f;
            }
        cudaError_t e;
        if ((e = cudaMemcpyAsync(adj[0].ptr, A0.data(), sizeof(float) * state_floats(), cudaMemcpyHostToDevice, stream)) ||
            (e = cudaMemsetAsync(Ebar.ptr, 0, sizeof(float) * n, stream)) ||
            (e = cudaMemsetAsync(err.ptr, 0, sizeof(uint32_t), stream)))
            return cuda_fail(e, "adjoint upload");
        // the parity of the final adj buffer: one flip per substep
        const int a = static_cast<int>(substeps & 1u);
        if ((e = replay(&bwd_exec, [&]() { backward_sweep(); }))) return cuda_fail(e, "adjoint backward");
        std::vector<float> vb(3 * n), eb(n);
        if ((e = cudaMemcpyAsync(vb.data(), adj[a].ptr + 3 * n, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, stream)) ||
            (e = cudaMemcpyAsync(eb.data(), Ebar.ptr, sizeof(float) * n, cudaMemcpyDeviceToHost, stream)) ||
            (e = cudaStreamSynchronize(stream)))
            return cuda_fail(e, "adjoint backward");
        TmpmStatus st = check_err();
        if (st != TMPM_OK) return st;
        for (size_t i = 0; i < n; ++i) {
            for (int k = 0; k < 3; ++k) {
                if (!std::isfinite(vb[k * n + i])) return fail(TMPM_ERR_NON_FINITE_STATE, "non-finite adjoint");
                if (v0_grad) v0_grad[3 * i + k] = vb[k * n + i];
            }
            if (!std::isfinite(eb[i])) return fail(TMPM_ERR_NON_FINITE_STATE, "non-finite adjoint");
            if (young_grad) young_grad[i] = eb[i];
        }
        return TMPM_OK;
    }
};

extern "C" {

TmpmStatus tmpm_adjoint_create(const TmpmParams *params, const TmpmParticleArrays *particles, double substep_dt,
                               uint32_t substeps, uint32_t checkpoint_every, int32_t device, TmpmAdjoint **out) {
    if (!out || !params) {
        g_last_error = "null argument";
        return TMPM_ERR_INVALID_INPUT;
    }
    *out = nullptr;
    if (!params_valid(*params)) {
        g_last_error = "invalid MPM input";
        return TMPM_ERR_MPM_INVALID_INPUT;
    }
    if (!params->has_bounds) {
        g_last_error = "the differentiable rollout needs a bounded domain";
        return TMPM_ERR_INVALID_INPUT;
    }
    if (substeps == 0 || checkpoint_every == 0) {
        g_last_error = "substeps and checkpoint interval must be positive";
        return TMPM_ERR_INVALID_INPUT;
    }
    auto a = std::make_unique<TmpmAdjoint>();
    std::string err;
    TmpmStatus st = load_checked(particles, a->world, err);
    if (st != TMPM_OK) {
        g_last_error = err;
        return st;
    }
    HostWorld &w = a->world;
    if (w.n == 0 || w.n > (1u << 26)) {
        g_last_error = "particle count must be 1 .. 2^26";
        return TMPM_ERR_INVALID_INPUT;
    }
    for (size_t i = 0; i < w.n; ++i) {
        if (w.material[i] != TMPM_MAT_ELASTIC || !w.enabled[i]) {
            g_last_error = "the differentiable rollout takes enabled corotated elastic particles";
            return TMPM_ERR_INVALID_INPUT;
        }
        for (int k = 0; k < 3; ++k)
            if (!(w.pos[3 * i + k] >= params->bounds_min[k] && w.pos[3 * i + k] <= params->bounds_max[k])) {
                g_last_error = "particles must start inside the domain bounds";
                return TMPM_ERR_INVALID_INPUT;
            }
    }
    if (!std::isfinite(substep_dt) || substep_dt <= 0.0 || substep_dt > stable_timestep(w, *params)) {
        g_last_error = "substep dt is not finite, not positive or above the CFL bound";
        return TMPM_ERR_INVALID_INPUT;
    }
    a->params = *params;
    a->dt = substep_dt;
    a->substeps = substeps;
    a->every = std::min(checkpoint_every, substeps);
    a->device = device;
    a->n = w.n;
    AdjParams &P = a->P;
    const double h = params->cell_width;
    P.h = static_cast<float>(h);
    P.inv_h = 1.0f / P.h;
    P.inv_d = static_cast<float>(4.0 / (h * h));
    P.dt = static_cast<float>(substep_dt);
    P.gx = static_cast<float>(params->gravity[0]);
    P.gy = static_cast<float>(params->gravity[1]);
    P.gz = static_cast<float>(params->gravity[2]);
    P.wall_mode = params->wall_mode;
    size_t nodes = 1;
    for (int k = 0; k < 3; ++k) {
        P.bmin[k] = static_cast<float>(params->bounds_min[k]);
        P.bmax[k] = static_cast<float>(params->bounds_max[k]);
        P.wall_lo[k] = wall_index_le(params->bounds_min[k] + h, h);
        P.wall_hi[k] = wall_index_ge(params->bounds_max[k] - h, h);
        int lo = static_cast<int>(std::floor(P.bmin[k] * P.inv_h - 0.5f)) - 1;
        int hi = static_cast<int>(std::floor(P.bmax[k] * P.inv_h - 0.5f)) + 3;
        P.lo[k] = lo;
        P.dim[k] = hi - lo + 1;
        nodes *= static_cast<size_t>(P.dim[k]);
    }
    if (nodes > (size_t(1) << 28)) {
        g_last_error = "domain too large for the dense node array";
        return TMPM_ERR_CAPACITY;
    }
    a->nodes = static_cast<int>(nodes);
    P.n = static_cast<int>(w.n);
    P.stride = w.n;
    const size_t n = w.n;
    std::vector<float> m(n), v(n), r(n), d(n), nu(n);
    std::vector<uint8_t> fx(n);
    for (size_t i = 0; i < n; ++i) {
        m[i] = static_cast<float>(w.mass[i]);
        v[i] = static_cast<float>(w.vol[i]);
        r[i] = static_cast<float>(w.radius[i]);
        d[i] = static_cast<float>(w.damping[i]);
        nu[i] = static_cast<float>(w.mparams[5 * i + 1]);
        fx[i] = w.fixed[i];
    }
    cudaError_t e;
    const uint32_t segments = (substeps + a->every - 1) / a->every;
    const size_t sf = kRows * n;
    if ((e = cudaSetDevice(device)) || (e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithFlags(&a->side, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&a->ev_fork, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&a->ev_replayed, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&a->ev_swept, cudaEventDisableTiming)) ||
        (e = a->mass.alloc(n)) || (e = a->vol.alloc(n)) || (e = a->radius.alloc(n)) || (e = a->damping.alloc(n)) ||
        (e = a->nu.alloc(n)) || (e = a->E.alloc(n)) || (e = a->Ebar.alloc(n)) || (e = a->fixed.alloc(n)) ||
        (e = a->ckpt.alloc(segments * sf)) || (e = a->adj[0].alloc(sf)) || (e = a->adj[1].alloc(sf)) ||
        (e = a->part.alloc(sf)) || (e = a->grid.alloc(nodes)) || (e = a->gv.alloc(nodes)) ||
        (e = a->gvb.alloc(nodes)) || (e = a->err.alloc(1))) {
        g_last_error = std::string("adjoint setup: ") + cudaGetErrorString(e);
        return TMPM_ERR_DEVICE;
    }
    for (int set = 0; set < 2; ++set)
        if ((e = a->seg[set].alloc(std::max<size_t>(a->every, 2) * sf)) ||
            (e = a->seg_grid[set].alloc(static_cast<size_t>(a->every) * nodes)) ||
            (e = a->seg_gv[set].alloc(static_cast<size_t>(a->every) * nodes)) ||
            (e = a->seg_R[set].alloc(a->every * 9 * n))) {
            g_last_error = std::string("adjoint setup: ") + cudaGetErrorString(e);
            return TMPM_ERR_DEVICE;
        }
    cudaMemcpyAsync(a->mass.ptr, m.data(), sizeof(float) * n, cudaMemcpyHostToDevice, a->stream);
    cudaMemcpyAsync(a->vol.ptr, v.data(), sizeof(float) * n, cudaMemcpyHostToDevice, a->stream);
    cudaMemcpyAsync(a->radius.ptr, r.data(), sizeof(float) * n, cudaMemcpyHostToDevice, a->stream);
    cudaMemcpyAsync(a->damping.ptr, d.data(), sizeof(float) * n, cudaMemcpyHostToDevice, a->stream);
    cudaMemcpyAsync(a->nu.ptr, nu.data(), sizeof(float) * n, cudaMemcpyHostToDevice, a->stream);
    cudaMemcpyAsync(a->fixed.ptr, fx.data(), n, cudaMemcpyHostToDevice, a->stream);
    if ((e = cudaStreamSynchronize(a->stream))) {
        g_last_error = std::string("adjoint setup: ") + cudaGetErrorString(e);
        return TMPM_ERR_DEVICE;
    }
    *out = a.release();
    return TMPM_OK;
}

void tmpm_adjoint_destroy(TmpmAdjoint *a) { delete a; }

size_t tmpm_adjoint_particle_count(const TmpmAdjoint *a) { return a ? a->n : 0; }

TmpmStatus tmpm_adjoint_forward(TmpmAdjoint *a, const double *velocity0, const double *young, double *position_out,
                                double *velocity_out) {
    if (!a) return TMPM_ERR_INVALID_INPUT;
    cudaSetDevice(a->device);
    a->have_forward = false;
    return a->forward(velocity0, young, position_out, velocity_out);
}

TmpmStatus tmpm_adjoint_backward(TmpmAdjoint *a, const double *position_grad, const double *velocity_grad,
                                 double *velocity0_grad, double *young_grad) {
    if (!a) return TMPM_ERR_INVALID_INPUT;
    cudaSetDevice(a->device);
    return a->backward(position_grad, velocity_grad, velocity0_grad, young_grad);
}

const char *tmpm_adjoint_last_error_message(const TmpmAdjoint *a) {
    return a ? a->last_error.c_str() : g_last_error.c_str();
}

}  // extern "C"
