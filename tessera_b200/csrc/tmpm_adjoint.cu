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

#include <memory>

#include "tmpm_device.cuh"
#include "tmpm_host.h"

using namespace tmpm;

namespace {

constexpr int kRows = 24;  // x 0-2, v 3-5, C 6-14, F 15-23 (matrices column-major: col * 3 + row)
constexpr uint32_t kErrGrid = 1u;  // a stencil left the node array
// Threads per CTA of the particle kernels.  A 64k-particle rollout is ~1.7
// waves of 256-thread CTAs on 148 SMs (some SMs with two CTAs, some with
// one); 64-thread CTAs spread the latency-bound particle work evenly.
constexpr int kParticleThreads = 64;

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

__device__ __forceinline__ void lame(float E, float nu, float &lambda, float &mu) {
    lambda = E * nu / ((1.0f + nu) * (1.0f - 2.0f * nu));
    mu = E / (2.0f * (1.0f + nu));
}

// ---------------------------------------------------------------- forward

// Rout (optional): the polar factor R of each particle's F, 9 rows, for the
// P2G adjoint of the same substep.
__global__ void k_p2g(AdjParams P, Consts K, const float *__restrict__ S, const float *__restrict__ E,
                      float4 *grid, uint32_t *err, float *__restrict__ Rout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, i), v = load_v(S, st, 3, i);
    M3f C = load_m(S, st, 6, i), F = load_m(S, st, 15, i);
    float lambda, mu;
    lame(E[i], K.nu[i], lambda, mu);
    M3f R = polar_rotation(F);
    if (Rout) {
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
    const float m = K.mass[i];
    M3f A = add(scale(tau, -P.dt * K.vol[i] * P.inv_d), scale(C, m));
    Stencil s;
    stencil(x, P.inv_h, s);
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
__device__ __forceinline__ void gather(const AdjParams &P, const Stencil &s, const float4 *gv, V3f &vel, M3f &aff) {
    vel = mk(0, 0, 0);
    aff = m3_zero();
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
                int id = node_at(P, s, a, b, c);
                if (id < 0) continue;
                float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                float4 g = gv[id];
                V3f nv = mk(g.x, g.y, g.z);
                V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                vel = vel + nv * w;
                aff = add(aff, scale(outer(nv, dpos), w * P.inv_d));
            }
}

__global__ void k_g2p(AdjParams P, Consts K, const float *__restrict__ S, float *__restrict__ Sn,
                      const float4 *__restrict__ gv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, i);
    M3f F = load_m(S, st, 15, i);
    if (K.fixed[i]) {
        store_v(Sn, st, 0, i, x);
        store_v(Sn, st, 3, i, mk(0, 0, 0));
        store_m(Sn, st, 6, i, m3_zero());
        store_m(Sn, st, 15, i, F);
        return;
    }
    Stencil s;
    stencil(x, P.inv_h, s);
    V3f vel;
    M3f aff;
    gather(P, s, gv, vel, aff);
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
__global__ void k_g2p_back(AdjParams P, Consts K, const float *__restrict__ S, const float4 *__restrict__ gv,
                           const float *__restrict__ Ab, float *__restrict__ Q, float4 *gvb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, i);
    M3f F = load_m(S, st, 15, i);
    V3f xb_o = load_v(Ab, st, 0, i), vb_o = load_v(Ab, st, 3, i);
    M3f Cb_o = load_m(Ab, st, 6, i), Fb_o = load_m(Ab, st, 15, i);
    if (K.fixed[i]) {  // x and F pass through; v and C are reset
        store_v(Q, st, 0, i, xb_o);
        store_m(Q, st, 15, i, Fb_o);
        return;
    }
    Stencil s;
    stencil(x, P.inv_h, s);
    V3f vel;
    M3f aff;
    gather(P, s, gv, vel, aff);
    const float ed = expf(-K.damping[i] * P.dt);
    V3f veld = vel * ed;
    V3f pos = x + veld * P.dt;
    const float r = K.radius[i];
    V3f xb = xb_o, velb = vb_o;
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
    M3f Cb = add(Cb_o, scale(mul_bt(Fb_o, F), P.dt));     // Fn = (I + dt C) F
    M3f Fb = mul(transpose(add(m3_identity(), scale(aff, P.dt))), Fb_o);
    V3f xbar = xb;
    const M3f CbT = transpose(Cb);
    V3f nv_c = mk(0, 0, 0);
    {
        int idc = node_at(P, s, 1, 1, 1);
        if (idc >= 0) nv_c = mk(gv[idc].x, gv[idc].y, gv[idc].z);
    }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
                int id = node_at(P, s, a, b, c);
                if (id < 0) continue;
                float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                V3f dw = mk(s.dw[0][a] * s.w[1][b] * s.w[2][c], s.w[0][a] * s.dw[1][b] * s.w[2][c],
                            s.w[0][a] * s.w[1][b] * s.dw[2][c]) * P.inv_h;
                float4 g = gv[id];
                V3f nv = mk(g.x, g.y, g.z);
                V3f dnv = nv - nv_c;
                V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                V3f Cd = mul(Cb, dpos);
                // grad w (v_i . velb + v_i . C_b dpos_i) - w C_b^T v_i with v_i -> v_i - v_c (file header)
                float gs = dot(dnv, velb) + P.inv_d * dot(dnv, Cd);
                xbar = xbar + dw * gs - mul(CbT, dnv) * (P.inv_d * w);
                V3f gb = velb * w + Cd * (P.inv_d * w);
                red_add_v4(gvb + id, make_float4(gb.x, gb.y, gb.z, 0.0f));
            }
    store_v(Q, st, 0, i, xbar);
    store_m(Q, st, 15, i, Fb);
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
__global__ void k_p2g_back(AdjParams P, Consts K, const float *__restrict__ S, const float *__restrict__ E,
                           const float4 *__restrict__ gmb, const float *__restrict__ Q, float *__restrict__ Ain,
                           float *__restrict__ Eb, const float *__restrict__ Rin) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const size_t st = P.stride;
    V3f x = load_v(S, st, 0, i), v = load_v(S, st, 3, i);
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
    const M3f AT = transpose(A);
    Stencil s;
    stencil(x, P.inv_h, s);
    V3f xbar = load_v(Q, st, 0, i);
    M3f Fbar = load_m(Q, st, 15, i);
    V3f vbar = mk(0, 0, 0);
    M3f Abar = m3_zero();
    float4 gc = make_float4(0.f, 0.f, 0.f, 0.f);
    {
        int idc = node_at(P, s, 1, 1, 1);
        if (idc >= 0) gc = gmb[idc];
    }
    const V3f pb_c = mk(gc.y, gc.z, gc.w);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 3; ++c) {
                int id = node_at(P, s, a, b, c);
                if (id < 0) continue;
                float w = s.w[0][a] * s.w[1][b] * s.w[2][c];
                V3f dw = mk(s.dw[0][a] * s.w[1][b] * s.w[2][c], s.w[0][a] * s.dw[1][b] * s.w[2][c],
                            s.w[0][a] * s.w[1][b] * s.dw[2][c]) * P.inv_h;
                float4 g = gmb[id];
                V3f pb = mk(g.y, g.z, g.w);
                V3f dpb = pb - pb_c;
                V3f dpos = mk((a - s.fx[0]) * P.h, (b - s.fx[1]) * P.h, (c - s.fx[2]) * P.h);
                // grad w (m m_b + p_b . (m v + A dpos)) - w A^T p_b with m_b, p_b -> minus their centre values
                vbar = vbar + pb * (w * m);
                Abar = add(Abar, scale(outer(dpb, dpos), w));
                xbar = xbar + dw * (m * (g.x - gc.x) + m * dot(v, dpb) + dot(dpb, mul(A, dpos))) - mul(AT, dpb) * w;
            }
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
    DevBuf<float> ckpt, seg, adj[2], part;
    DevBuf<float4> grid, gv, gvb;
    // per substep of the segment being replayed: the grid after P2G (mass and
    // momentum), the node velocities and the particles' polar factors, so the
    // adjoint sweep reuses them instead of recomputing P2G and the grid update
    DevBuf<float4> seg_grid, seg_gv;
    DevBuf<float> seg_R;
    DevBuf<uint32_t> err;
    bool have_forward = false;
    std::string last_error;
    // The forward and adjoint sweeps (fixed launches over fixed buffers) are
    // captured as CUDA graphs on first use and replayed afterwards.
    cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;

    ~TmpmAdjoint() {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        if (fwd_exec) cudaGraphExecDestroy(fwd_exec);
        if (bwd_exec) cudaGraphExecDestroy(bwd_exec);
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

    // The forward sweep: `substeps` substeps from seg[0] ping-ponging with
    // seg[1], a checkpoint every `every`.
    void forward_sweep() {
        float *cur = seg.ptr, *nxt = seg.ptr + state_floats();
        for (uint32_t s = 0; s < substeps; ++s) {
            if (s % every == 0)
                cudaMemcpyAsync(ckpt.ptr + (s / every) * state_floats(), cur, sizeof(float) * state_floats(),
                                cudaMemcpyDeviceToDevice, stream);
            substep(cur, nxt);
            std::swap(cur, nxt);
        }
    }

    // The adjoint sweep from adj[0] (the loss gradient of the final state),
    // segment by segment from the last checkpoint back; the initial-state
    // adjoint ends in adj[substeps & 1].
    void backward_sweep() {
        int a = 0;
        const uint32_t segments = (substeps + every - 1) / every;
        for (int sg = static_cast<int>(segments) - 1; sg >= 0; --sg) {
            const uint32_t s0 = sg * every, s1 = std::min(substeps, s0 + every);
            // replay the segment: seg[j] = state at substep s0 + j, with the
            // grid, node velocities and polar factors of each substep kept
            cudaMemcpyAsync(seg.ptr, ckpt.ptr + sg * state_floats(), sizeof(float) * state_floats(),
                            cudaMemcpyDeviceToDevice, stream);
            for (uint32_t s = s0; s < s1; ++s) {
                const uint32_t j = s - s0;
                float4 *g = seg_grid.ptr + static_cast<size_t>(j) * nodes, *v = seg_gv.ptr + static_cast<size_t>(j) * nodes;
                p2g_grid(seg.ptr + j * state_floats(), g, v, seg_R.ptr + static_cast<size_t>(j) * 9 * n);
                if (s + 1 < s1)
                    k_g2p<<<blocks_n(), kParticleThreads, 0, stream>>>(P, consts(), seg.ptr + j * state_floats(),
                                                                       seg.ptr + (j + 1) * state_floats(), v);
            }
            for (int s = static_cast<int>(s1) - 1; s >= static_cast<int>(s0); --s) {
                const uint32_t j = s - s0;
                const float *S = seg.ptr + j * state_floats();
                const float4 *g = seg_grid.ptr + static_cast<size_t>(j) * nodes, *v = seg_gv.ptr + static_cast<size_t>(j) * nodes;
                cudaMemsetAsync(gvb.ptr, 0, sizeof(float4) * nodes, stream);
                k_g2p_back<<<blocks_n(), kParticleThreads, 0, stream>>>(P, consts(), S, v, adj[a].ptr, part.ptr,
                                                                        gvb.ptr);
                k_grid_back<<<blocks_nodes(), 256, 0, stream>>>(P, g, v, gvb.ptr, nodes);
                k_p2g_back<<<blocks_n(), kParticleThreads, 0, stream>>>(P, consts(), S, E.ptr, gvb.ptr, part.ptr,
                                                                        adj[a ^ 1].ptr, Ebar.ptr,
                                                                        seg_R.ptr + static_cast<size_t>(j) * 9 * n);
                a ^= 1;
            }
        }
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
    int blocks_n() const { return static_cast<int>((n + kParticleThreads - 1) / kParticleThreads); }
    int blocks_nodes() const { return (nodes + 255) / 256; }

    // P2G + grid of state S into g / v (and the polar factors into R when given).
    void p2g_grid(const float *S, float4 *g, float4 *v, float *R) {
        cudaMemsetAsync(g, 0, sizeof(float4) * nodes, stream);
        k_p2g<<<blocks_n(), kParticleThreads, 0, stream>>>(P, consts(), S, E.ptr, g, err.ptr, R);
        k_grid<<<blocks_nodes(), 256, 0, stream>>>(P, g, v, nodes);
    }
    void substep(const float *S, float *Sn) {
        p2g_grid(S, grid.ptr, gv.ptr, nullptr);
        k_g2p<<<blocks_n(), kParticleThreads, 0, stream>>>(P, consts(), S, Sn, gv.ptr);
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
            (e = cudaMemcpyAsync(seg.ptr, S0.data(), sizeof(float) * state_floats(), cudaMemcpyHostToDevice, stream)) ||
            (e = cudaMemsetAsync(err.ptr, 0, sizeof(uint32_t), stream)))
            return cuda_fail(e, "adjoint upload");
        // seg holds two ping-pong states during the forward; the final state is
        // in the first of them after an even number of substeps
        if ((e = replay(&fwd_exec, [&]() { forward_sweep(); }))) return cuda_fail(e, "adjoint forward");
        const float *cur = (substeps % 2 == 0) ? seg.ptr : seg.ptr + state_floats();
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
        (e = a->mass.alloc(n)) || (e = a->vol.alloc(n)) || (e = a->radius.alloc(n)) || (e = a->damping.alloc(n)) ||
        (e = a->nu.alloc(n)) || (e = a->E.alloc(n)) || (e = a->Ebar.alloc(n)) || (e = a->fixed.alloc(n)) ||
        (e = a->ckpt.alloc(segments * sf)) || (e = a->seg.alloc(std::max<size_t>(a->every, 2) * sf)) ||
        (e = a->adj[0].alloc(sf)) || (e = a->adj[1].alloc(sf)) || (e = a->part.alloc(sf)) ||
        (e = a->grid.alloc(nodes)) || (e = a->gv.alloc(nodes)) || (e = a->gvb.alloc(nodes)) || (e = a->err.alloc(1)) ||
        (e = a->seg_grid.alloc(static_cast<size_t>(a->every) * nodes)) ||
        (e = a->seg_gv.alloc(static_cast<size_t>(a->every) * nodes)) || (e = a->seg_R.alloc(a->every * 9 * n))) {
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
