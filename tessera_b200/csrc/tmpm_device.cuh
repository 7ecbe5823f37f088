// tmpm_device.cuh -- f32 device math for the MLS-MPM substep.
//
// Matrices are column-major (three float3 columns), the layout of the
// reference's WGSL mat3x3 and of nalgebra's Matrix3 storage.
#pragma once

#include <cuda/atomic>

#include "tmpm_internal.h"

namespace tmpm {

// ------------------------------------------------------------------ vectors
struct V3f {
    float x, y, z;
};
__device__ __forceinline__ V3f mk(float a, float b, float c) { return V3f{a, b, c}; }
__device__ __forceinline__ V3f operator+(V3f a, V3f b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3f operator-(V3f a, V3f b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3f operator*(V3f a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3f operator*(float s, V3f a) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3f operator-(V3f a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(V3f a, V3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3f cross(V3f a, V3f b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len(V3f a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float comp(V3f a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ void set_comp(V3f &a, int i, float v) {
    if (i == 0) a.x = v;
    else if (i == 1) a.y = v;
    else a.z = v;
}
__device__ __forceinline__ bool finite3(V3f a) {
    return fabsf(a.x) < 1e30f && fabsf(a.y) < 1e30f && fabsf(a.z) < 1e30f;
}

// ------------------------------------------------------------------ matrices
struct M3f {
    V3f c0, c1, c2;  // columns
};
__device__ __forceinline__ M3f m3_identity() { return M3f{mk(1, 0, 0), mk(0, 1, 0), mk(0, 0, 1)}; }
__device__ __forceinline__ M3f m3_zero() { return M3f{mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)}; }
__device__ __forceinline__ V3f mul(const M3f &m, V3f v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }
__device__ __forceinline__ M3f mul(const M3f &a, const M3f &b) {
    return M3f{mul(a, b.c0), mul(a, b.c1), mul(a, b.c2)};
}
__device__ __forceinline__ M3f transpose(const M3f &m) {
    return M3f{mk(m.c0.x, m.c1.x, m.c2.x), mk(m.c0.y, m.c1.y, m.c2.y), mk(m.c0.z, m.c1.z, m.c2.z)};
}
__device__ __forceinline__ M3f add(const M3f &a, const M3f &b) { return M3f{a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2}; }
__device__ __forceinline__ M3f sub(const M3f &a, const M3f &b) { return M3f{a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2}; }
__device__ __forceinline__ M3f scale(const M3f &a, float s) { return M3f{a.c0 * s, a.c1 * s, a.c2 * s}; }
__device__ __forceinline__ float det(const M3f &m) { return dot(m.c0, cross(m.c1, m.c2)); }
__device__ __forceinline__ float fro2(const M3f &m) { return dot(m.c0, m.c0) + dot(m.c1, m.c1) + dot(m.c2, m.c2); }
__device__ __forceinline__ bool finite_m(const M3f &m) { return finite3(m.c0) && finite3(m.c1) && finite3(m.c2); }
// A B^T
__device__ __forceinline__ M3f mul_bt(const M3f &a, const M3f &b) {
    M3f bt = transpose(b);
    return mul(a, bt);
}

// Polar factor R of F by Newton's iteration R <- (R + R^-T) / 2, the iteration
// the reference shader uses (gpu.wgsl:467-482, ten steps); it stops early once
// the squared update falls below 1e-11: the iteration converges quadratically,
// so the iterate it returns is then accurate to ~1e-11, below f32 resolution.
// R^-T = cofactor(R) / det(R).
__device__ __forceinline__ M3f polar_rotation(const M3f &F) {
    M3f R = F;
#pragma unroll 1
    for (int it = 0; it < 10; ++it) {
        V3f a = R.c0, b = R.c1, c = R.c2;
        V3f bc = cross(b, c), ca = cross(c, a), ab = cross(a, b);
        float d = dot(a, bc);
        float inv = 1.0f / d;
        M3f next = M3f{(a + bc * inv) * 0.5f, (b + ca * inv) * 0.5f, (c + ab * inv) * 0.5f};
        M3f diff = sub(next, R);
        R = next;
        if (fro2(diff) < 1e-11f) break;
    }
    return R;
}

// regular_corotated (gpu.wgsl:451-465): conditioning guard of the resident path.
__device__ __forceinline__ bool regular_corotated(const M3f &F) {
    V3f a = F.c0, b = F.c1, c = F.c2;
    float d = dot(a, cross(b, c));
    float nrm = sqrtf(fro2(F));
    if (fabsf(d) < 1e-5f || nrm < 1e-5f || nrm > 20.0f) return false;
    V3f i0 = cross(b, c) * (1.0f / d), i1 = cross(c, a) * (1.0f / d), i2 = cross(a, b) * (1.0f / d);
    float inorm = sqrtf(dot(i0, i0) + dot(i1, i1) + dot(i2, i2));
    return nrm * inorm <= 100.0f;
}

// Corotated Kirchhoff stress 2 mu (F - R) F^T + lambda (J - 1) J I, scaled by
// snow's hardening factor (material.rs:272-283, 440-455).
__device__ __forceinline__ M3f corotated_stress_body(const DevClass &k, const M3f &F, float J, float plastic_det) {
    float factor = 1.0f;
    if (k.kind == kMatSnow) factor = fminf(fmaxf(expf(k.p2 * (1.0f - plastic_det)), 0.01f), 100.0f);
    float lambda = k.p0 * factor, mu = k.p1 * factor;
    M3f R = polar_rotation(F);
    float iso = lambda * (J - 1.0f) * J;
    M3f s = scale(mul_bt(sub(F, R), F), 2.0f * mu);
    s.c0.x += iso;
    s.c1.y += iso;
    s.c2.z += iso;
    return s;
}

// The same out of line.  Which placement holds fewer registers depends on the
// kernel variant: an out-of-line call takes the class record and F by
// reference, so they stay in local memory around it; inline, the polar
// iteration adds to the register peak.  With the obstacle contact (itself an
// out-of-line call) or plastic state in the kernel, the call spills less; in
// the lean variants inlining took the fused transfer from 0.499 to 0.451 ms
// on the dam break.
static __device__ __noinline__ M3f corotated_stress(const DevClass &k, const M3f &F, float J, float plastic_det) {
    return corotated_stress_body(k, F, J, plastic_det);
}

// Kirchhoff stress times -dt V0 4/h^2 (material.rs:233-284; the scaling is
// world.rs:391 / gpu.wgsl:700).  `plastic_det` feeds snow's hardening factor.
template <bool INLINE_COROTATED>
__device__ __forceinline__ M3f scaled_stress(const DevClass &k, const M3f &F, const M3f &Cm, float neg_dt_inv_d,
                                             float plastic_det) {
    float J = det(F);
    M3f s;
    if (k.kind == kMatNeoHookean || k.kind == kMatSandNeoHookean) {
        float lambda = k.p0, mu = k.p1;
        float sj = fmaxf(J, 1e-10f);
        float iso = lambda * logf(sj) - mu;
        s = scale(mul_bt(F, F), mu);
        s.c0.x += iso;
        s.c1.y += iso;
        s.c2.z += iso;
    } else if (k.kind == kMatFluid) {
        float bulk = k.p0, gamma = k.p1, visc = k.p2, tensile = k.p3;
        float sj = fmaxf(J, 1e-6f);
        float pressure = sj <= 1.0f ? bulk * (powf(sj, -gamma) - 1.0f) : -bulk * tensile * (sj - 1.0f);
        M3f sr = scale(add(Cm, transpose(Cm)), 0.5f);
        float tr3 = (sr.c0.x + sr.c1.y + sr.c2.z) * (1.0f / 3.0f);
        float diag = -2.0f * visc * sj * tr3 - pressure * sj;
        s = scale(sr, 2.0f * visc * sj);
        s.c0.x += diag;
        s.c1.y += diag;
        s.c2.z += diag;
    } else {  // corotated: elastic, sand, snow (with its hardening factor)
        s = INLINE_COROTATED ? corotated_stress_body(k, F, J, plastic_det) : corotated_stress(k, F, J, plastic_det);
    }
    return scale(s, neg_dt_inv_d * k.volume);
}

// ------------------------------------------------------ plastic return maps

// Eigen-decomposition of the symmetric S = F^T F by cyclic Jacobi rotations
// (Golub & Van Loan, Matrix Computations, sec. 8.5): S = V diag(w) V^T.
__device__ inline void sym_eigen3(const M3f &F, V3f &w, M3f &V) {
    float a00 = dot(F.c0, F.c0), a11 = dot(F.c1, F.c1), a22 = dot(F.c2, F.c2);
    float a01 = dot(F.c0, F.c1), a02 = dot(F.c0, F.c2), a12 = dot(F.c1, F.c2);
    V = m3_identity();
#pragma unroll 1
    for (int sweep = 0; sweep < 8; ++sweep) {
        float off = a01 * a01 + a02 * a02 + a12 * a12;
        if (off <= 1e-24f * (a00 * a00 + a11 * a11 + a22 * a22)) break;
#pragma unroll
        for (int pair = 0; pair < 3; ++pair) {
            // (p, q) = (0, 1), (0, 2), (1, 2)
            float app = pair == 2 ? a11 : a00;
            float aqq = pair == 0 ? a11 : a22;
            float apq = pair == 0 ? a01 : (pair == 1 ? a02 : a12);
            if (fabsf(apq) < 1e-30f) continue;
            float theta = (aqq - app) / (2.0f * apq);
            float t = copysignf(1.0f, theta) / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
            float c = rsqrtf(t * t + 1.0f), sn = t * c;
            float napp = app - t * apq, naqq = aqq + t * apq;
            if (pair == 0) {  // rotate rows/cols 0 and 1; r = 2
                float a2p = a02, a2q = a12;
                a02 = c * a2p - sn * a2q;
                a12 = sn * a2p + c * a2q;
                a00 = napp;
                a11 = naqq;
                a01 = 0.f;
                V3f vp = V.c0, vq = V.c1;
                V.c0 = vp * c - vq * sn;
                V.c1 = vp * sn + vq * c;
            } else if (pair == 1) {  // 0 and 2; r = 1
                float a1p = a01, a1q = a12;
                a01 = c * a1p - sn * a1q;
                a12 = sn * a1p + c * a1q;
                a00 = napp;
                a22 = naqq;
                a02 = 0.f;
                V3f vp = V.c0, vq = V.c2;
                V.c0 = vp * c - vq * sn;
                V.c2 = vp * sn + vq * c;
            } else {  // 1 and 2; r = 0
                float a0p = a01, a0q = a02;
                a01 = c * a0p - sn * a0q;
                a02 = sn * a0p + c * a0q;
                a11 = napp;
                a22 = naqq;
                a12 = 0.f;
                V3f vp = V.c1, vq = V.c2;
                V.c1 = vp * c - vq * sn;
                V.c2 = vp * sn + vq * c;
            }
        }
    }
    w = mk(a00, a11, a22);
}

// F V diag(target / sigma) V^T = U diag(target) V^T without forming U.
__device__ __forceinline__ M3f replace_stretches(const M3f &F, const M3f &V, V3f sigma, V3f target) {
    M3f FV = mul(F, V);
    FV.c0 = FV.c0 * (target.x / sigma.x);
    FV.c1 = FV.c1 * (target.y / sigma.y);
    FV.c2 = FV.c2 * (target.z / sigma.z);
    return mul_bt(FV, V);
}

// Return mapping of the plastic materials (material.rs:297-368, 488-532) in
// f32; `pl` = (plastic_det, hardening, log_volume_gain).  Returns false when
// F is too ill-conditioned to project on the device (the reference's GPU
// marks those particles for its CPU path, gpu.wgsl:569-573).
static __device__ __noinline__ bool project_plastic(const DevClass &k, M3f &F, float pl[3]) {
    if ((k.kind == kMatSand || k.kind == kMatSandNeoHookean) && k.p0 == 0.0f) return true;  // lambda == 0
    V3f w;
    M3f V;
    sym_eigen3(F, w, V);
    V3f sg = mk(sqrtf(fmaxf(w.x, 0.f)), sqrtf(fmaxf(w.y, 0.f)), sqrtf(fmaxf(w.z, 0.f)));
    float smin = fminf(fminf(sg.x, sg.y), sg.z), smax = fmaxf(fmaxf(sg.x, sg.y), sg.z);
    if (!(smin >= 1e-6f) || smax / smin > 100.0f) return false;
    if (k.kind == kMatSnow) {
        float lo = 1.0f - k.p3, hi = 1.0f + k.p4;
        V3f cl = mk(fminf(fmaxf(sg.x, lo), hi), fminf(fmaxf(sg.y, lo), hi), fminf(fmaxf(sg.z, lo), hi));
        float old_det = sg.x * sg.y * sg.z;
        float new_det = fmaxf(cl.x * cl.y * cl.z, 1e-12f);
        pl[0] = fminf(fmaxf(pl[0] * old_det / new_det, 0.1f), 4.0f);
        F = replace_stretches(F, V, sg, cl);
        return true;
    }
    const float lambda = k.p0, mu = k.p1, friction = k.p2, cohesion = k.p3;
    const float g3 = pl[2] * (1.0f / 3.0f);
    V3f strain = mk(logf(fmaxf(sg.x, 1e-12f)) + g3, logf(fmaxf(sg.y, 1e-12f)) + g3, logf(fmaxf(sg.z, 1e-12f)) + g3);
    float tr = strain.x + strain.y + strain.z;
    V3f dev = strain - mk(tr, tr, tr) * (1.0f / 3.0f);
    float nrm = len(dev);
    float shifted = tr - cohesion;
    float q = pl[1];
    float angle = friction + (0.15707963267948966f * q - 0.17453292519943295f) * expf(-0.2f * q);
    float sine = sinf(angle);
    float alpha = 0.81649658092772603f * (2.0f * sine) / (3.0f - sine);
    V3f plog;
    float inc;
    if (shifted > 0.0f || nrm <= 4.76837158203125e-7f) {  // apex (4 f32::EPSILON)
        plog = mk(cohesion, cohesion, cohesion) * (1.0f / 3.0f);
        inc = len(strain);
    } else {
        float gamma = nrm + (3.0f * lambda + 2.0f * mu) / (2.0f * mu) * shifted * alpha;
        if (gamma <= 0.0f) return true;  // elastic region: unchanged
        plog = strain - dev * (gamma / nrm);
        inc = gamma;
    }
    V3f pr = mk(expf(plog.x), expf(plog.y), expf(plog.z));
    float old_det = sg.x * sg.y * sg.z, new_det = pr.x * pr.y * pr.z;
    if (k.kind == kMatSand) {
        old_det = fmaxf(old_det, 1e-12f);
        new_det = fmaxf(new_det, 1e-12f);
    }
    float pd = pl[0] * old_det / new_det;
    if (k.kind == kMatSand) pd = fminf(fmaxf(pd, 0.01f), 100.0f);
    pl[0] = pd;
    pl[1] = q + inc;
    pl[2] = pl[2] + (logf(old_det) - logf(new_det));
    F = replace_stretches(F, V, sg, pr);
    return true;
}

// ---------------------------------------------------------------- obstacles
__device__ __forceinline__ V3f qrot(const float q[4], V3f v) {
    V3f qv = mk(q[0], q[1], q[2]);
    V3f t = cross(qv, v) * 2.0f;
    return v + t * q[3] + cross(qv, t);
}
__device__ __forceinline__ V3f qrot_inv(const float q[4], V3f v) {
    V3f qv = mk(-q[0], -q[1], -q[2]);
    V3f t = cross(qv, v) * 2.0f;
    return v + t * q[3] + cross(qv, t);
}

__device__ inline V3f closest_point_triangle(V3f p, V3f a, V3f b, V3f c) {
    V3f ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) return a;
    V3f bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) return b;
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return a + ab * (d1 / (d1 - d3));
    V3f cp = p - c;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) return c;
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return a + ac * (d2 / (d2 - d6));
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f) return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    float r = 1.0f / (va + vb + vc);
    return a + ab * (vb * r) + ac * (vc * r);
}

__device__ __forceinline__ V3f normalize(V3f v) { return v * (1.0f / len(v)); }

// Signed distance and outward world normal (obstacle.rs:372-472).
static __device__ __noinline__ float obstacle_surface(const DevObstacle &o, const float *planes, V3f point, V3f &normal) {
    V3f rel = point - mk(o.center[0], o.center[1], o.center[2]);
    if (o.shape == 0) {  // sphere
        float n = len(rel);
        normal = n > 1e-12f ? rel * (1.0f / n) : mk(0, 0, 1);
        return n - o.dims[0];
    }
    V3f local = qrot_inv(o.q, rel);
    if (o.shape == 1) {  // box
        V3f he = mk(o.dims[0], o.dims[1], o.dims[2]);
        V3f cl = mk(fminf(fmaxf(local.x, -he.x), he.x), fminf(fmaxf(local.y, -he.y), he.y),
                    fminf(fmaxf(local.z, -he.z), he.z));
        V3f out = local - cl;
        float n = len(out);
        if (n > 1e-12f) {
            normal = qrot(o.q, out * (1.0f / n));
            return n;
        }
        V3f d = mk(he.x - fabsf(local.x), he.y - fabsf(local.y), he.z - fabsf(local.z));
        int axis = (d.x <= d.y && d.x <= d.z) ? 0 : (d.y <= d.z ? 1 : 2);
        V3f nn = mk(0, 0, 0);
        set_comp(nn, axis, comp(local, axis) < 0.0f ? -1.0f : 1.0f);
        normal = qrot(o.q, nn);
        return -comp(d, axis);
    }
    if (o.shape == 2) {  // capsule
        float hh = o.dims[0], r = o.dims[1];
        V3f delta = local - mk(0, 0, fminf(fmaxf(local.z, -hh), hh));
        float n = len(delta);
        float eps = fmaxf(hh, r) * 1e-6f;
        normal = qrot(o.q, n > eps ? delta * (1.0f / n) : mk(1, 0, 0));
        return n - r;
    }
    if (o.shape == 3) {  // cylinder (obstacle.rs:542-587)
        float hh = o.dims[0], radius = o.dims[1];
        float radial = sqrtf(local.x * local.x + local.y * local.y);
        V3f rn = radial > 1e-12f ? mk(local.x / radial, local.y / radial, 0.0f) : mk(1, 0, 0);
        float rd = radial - radius, cd = fabsf(local.z) - hh;
        float eps = fmaxf(hh, radius) * 1e-6f;
        V3f capn = mk(0, 0, local.z < 0.0f ? -1.0f : 1.0f);
        if (fabsf(rd) <= eps && fabsf(cd) <= eps) {
            normal = qrot(o.q, normalize(rn + capn));
            return fmaxf(rd, cd);
        }
        V3f outside = rn * fmaxf(rd, 0.0f) + capn * fmaxf(cd, 0.0f);
        float ol = len(outside);
        if (ol > 1e-12f) {
            normal = qrot(o.q, outside * (1.0f / ol));
            return ol;
        }
        if (rd >= cd) {
            normal = qrot(o.q, rn);
            return rd;
        }
        normal = qrot(o.q, capn);
        return cd;
    }
    if (o.shape == 4) {  // cone (obstacle.rs:589-631)
        float hh = o.dims[0], radius = o.dims[1];
        float radial = sqrtf(local.x * local.x + local.y * local.y);
        V3f rn = radial > 1e-12f ? mk(local.x / radial, local.y / radial, 0.0f) : mk(1, 0, 0);
        float px = radial, py = local.z;
        float bx = fminf(fmaxf(radial, 0.0f), radius), by = -hh;
        float sx = radius, sy = -hh, dx = -radius, dy = 2.0f * hh;
        float t = fminf(fmaxf(((px - sx) * dx + (py - sy) * dy) / (dx * dx + dy * dy), 0.0f), 1.0f);
        float sidex = sx + dx * t, sidey = sy + dy * t;
        float eps = fmaxf(hh, radius) * 1e-6f;
        float bd2 = (px - bx) * (px - bx) + (py - by) * (py - by);
        float sd2 = (px - sidex) * (px - sidex) + (py - sidey) * (py - sidey);
        bool use_base = bd2 <= sd2;
        float cx = use_base ? bx : sidex, cy = use_base ? by : sidey;
        float ddx = px - cx, ddy = py - cy;
        float nrm = sqrtf(ddx * ddx + ddy * ddy);
        bool inside = local.z >= -hh - eps && local.z <= hh + eps && radial <= radius * (hh - local.z) / (2.0f * hh) + eps;
        float snl = sqrtf(4.0f * hh * hh + radius * radius);
        float snx = 2.0f * hh / snl, sny = radius / snl;
        bool corner = bd2 <= eps * eps && sd2 <= eps * eps;
        float fnx, fny;
        if (corner) {
            float ax = snx, ay = -1.0f + sny, al = sqrtf(ax * ax + ay * ay);
            fnx = ax / al;
            fny = ay / al;
        } else if (use_base) {
            fnx = 0.0f;
            fny = -1.0f;
        } else {
            fnx = snx;
            fny = sny;
        }
        float n2x = fnx, n2y = fny;
        if (!(inside || nrm <= eps)) {
            n2x = ddx / nrm;
            n2y = ddy / nrm;
        }
        normal = qrot(o.q, rn * n2x + mk(0, 0, n2y));
        return inside ? -nrm : nrm;
    }
    if (o.shape == 5) {  // ground (obstacle.rs:439-454)
        float ox = local.x - fminf(fmaxf(local.x, -o.dims[0]), o.dims[0]);
        float oy = local.y - fminf(fmaxf(local.y, -o.dims[1]), o.dims[1]);
        float hd = sqrtf(ox * ox + oy * oy);
        if (hd <= 1e-12f) {
            normal = qrot(o.q, mk(0, 0, 1));
            return local.z;
        }
        V3f out = mk(ox, oy, local.z);
        float d = len(out);
        normal = qrot(o.q, out * (1.0f / d));
        return d;
    }
    if (o.shape == 6) {  // triangle prism (obstacle.rs:633-694)
        V3f a = mk(o.verts[0], o.verts[1], o.verts[2]);
        V3f b = mk(o.verts[4], o.verts[5], o.verts[6]);
        V3f c = mk(o.verts[8], o.verts[9], o.verts[10]);
        float ht = o.dims[0];
        V3f n = normalize(cross(b - a, c - a));
        V3f off = n * ht;
        V3f pr[6] = {a + off, b + off, c + off, a - off, b - off, c - off};
        const int faces[8][3] = {{0, 1, 2}, {3, 5, 4}, {3, 4, 1}, {3, 1, 0}, {4, 5, 2}, {4, 2, 1}, {5, 3, 0}, {5, 0, 2}};
        float edge = fmaxf(fmaxf(len(b - a), len(c - b)), fmaxf(len(a - c), ht));
        float eps = edge * 1e-6f;
        bool inside = true;
        V3f closest = mk(0, 0, 0), best_n = n, tied = mk(0, 0, 0);
        float best = 1e30f;
        for (int f = 0; f < 8; ++f) {
            V3f fa = pr[faces[f][0]], fb = pr[faces[f][1]], fc = pr[faces[f][2]];
            V3f fn = normalize(cross(fb - fa, fc - fa));
            inside = inside && dot(local - fa, fn) <= eps;
            V3f cand = closest_point_triangle(local, fa, fb, fc);
            V3f dd = local - cand;
            float d2 = dot(dd, dd);
            if (d2 + eps * eps < best) {
                best = d2;
                closest = cand;
                best_n = fn;
                tied = fn;
            } else if (fabsf(d2 - best) <= eps * eps) {
                tied = tied + fn;
            }
        }
        float dist = sqrtf(best);
        float tl = len(tied);
        V3f feature = tl > 1e-12f ? tied * (1.0f / tl) : best_n;
        V3f outward = (inside || dist <= eps) ? feature : (local - closest) * (1.0f / dist);
        normal = qrot(o.q, outward);
        return inside ? -dist : dist;
    }
    // convex (obstacle.rs:696-745): planes in the local frame
    {
        const float *pl = planes + 4 * o.plane_offset;
        int count = o.plane_count;
        float maximum = -1e30f;
        V3f nearest = mk(0, 0, 1);
        for (int i = 0; i < count; ++i) {
            V3f pn = mk(pl[4 * i], pl[4 * i + 1], pl[4 * i + 2]);
            float d = dot(pn, local) - pl[4 * i + 3];
            if (d > maximum) {
                maximum = d;
                nearest = pn;
            }
        }
        if (maximum <= 0.0f) {
            normal = qrot(o.q, nearest);
            return maximum;
        }
        // Dykstra's alternating projection with per-plane corrections (at most 32 planes on device).
        V3f projected = local;
        V3f corr[32];
        int m = count < 32 ? count : 32;
        for (int i = 0; i < m; ++i) corr[i] = mk(0, 0, 0);
        float tol = fmaxf(o.center[3], 1.0f) * 1e-5f;
        for (int it = 0; it < 64; ++it) {
            V3f prev = projected;
            for (int i = 0; i < m; ++i) {
                V3f pn = mk(pl[4 * i], pl[4 * i + 1], pl[4 * i + 2]);
                V3f shifted = projected + corr[i];
                float viol = fmaxf(dot(pn, shifted) - pl[4 * i + 3], 0.0f);
                projected = shifted - pn * viol;
                corr[i] = shifted - projected;
            }
            if (len(projected - prev) <= tol) break;
        }
        V3f offset = local - projected;
        float d = len(offset);
        if (d > tol) {
            normal = qrot(o.q, offset * (1.0f / d));
            return d;
        }
        normal = qrot(o.q, nearest);
        return maximum;
    }
}

// RigidObstacle::may_contact (obstacle.rs:474-499); center[3] carries the bound radius.
__device__ __forceinline__ bool obstacle_may_contact(const DevObstacle &o, V3f p, float margin) {
    V3f d = p - mk(o.center[0], o.center[1], o.center[2]);
    if (o.shape == 2) {
        float b = o.dims[0] + o.dims[1] + margin;
        return dot(d, d) <= b * b;
    }
    if (o.shape == 6 || o.shape == 7) {
        float b = o.center[3] + margin;
        return dot(d, d) <= b * b;
    }
    return true;
}

// Whether a point may lie within `r` of an obstacle's surface: its local
// coordinates within r of the box that holds the surface (DevObstacle::reach).
// Inline and call-free; false guarantees obstacle_surface(o, p) >= r, so the
// particle has no contact with this obstacle.
__device__ __forceinline__ bool obstacle_near(const DevObstacle &o, V3f p, float r) {
    const V3f l = qrot_inv(o.q, p - mk(o.center[0], o.center[1], o.center[2]));
    return fabsf(l.x) <= o.reach[0] + r && fabsf(l.y) <= o.reach[1] + r && l.z <= o.reach[2] + r &&
           (o.reach[3] != 0.0f || l.z >= -o.reach[2] - r);
}

// RigidObstacle::contact_velocity (obstacle.rs:501-540).
__device__ __forceinline__ V3f contact_velocity(const DevObstacle &o, V3f point, V3f vel, V3f n) {
    V3f surface = mk(o.lin[0], o.lin[1], o.lin[2]) +
                  cross(mk(o.ang[0], o.ang[1], o.ang[2]), point - mk(o.center[0], o.center[1], o.center[2]));
    if (o.boundary == 3) return vel;
    if (o.boundary == 1) return surface;
    V3f rel = vel - surface;
    float ns = dot(rel, n);
    if (o.boundary == 4) return vel - n * ns;
    if (ns >= 0.0f) return vel;
    V3f tangent = rel - n * ns;
    if (o.boundary == 2) return surface + tangent;
    float ts = len(tangent);
    float sc = ts > 1e-12f ? fmaxf(1.0f - o.lin[3] * -ns / ts, 0.0f) : 0.0f;
    return surface + tangent * sc;
}

// RigidObstacle::cpic_side for a triangle prism (obstacle.rs:343-370; the
// reference shader's f32 form with its 1e-5 barycentric margin, gpu.wgsl:82-102):
// distance to the triangle's plane and the side, when the point projects into
// the triangle.
__device__ __forceinline__ bool cpic_side(const DevObstacle &o, V3f point, float &dist, bool &positive) {
    const V3f local = qrot_inv(o.q, point - mk(o.center[0], o.center[1], o.center[2]));
    const V3f a = mk(o.verts[0], o.verts[1], o.verts[2]);
    const V3f eb = mk(o.verts[4], o.verts[5], o.verts[6]) - a, ec = mk(o.verts[8], o.verts[9], o.verts[10]) - a;
    const V3f n = normalize(cross(eb, ec));
    const float sd = dot(local - a, n);
    const V3f proj = local - n * sd - a;
    const float d00 = dot(eb, eb), d01 = dot(eb, ec), d11 = dot(ec, ec), d20 = dot(proj, eb), d21 = dot(proj, ec);
    const float den = d00 * d11 - d01 * d01;
    const float v = (d11 * d20 - d01 * d21) / den, w = (d00 * d21 - d01 * d20) / den;
    if (v >= -1e-5f && w >= -1e-5f && v + w <= 1.0f + 1e-5f) {
        dist = fabsf(sd);
        positive = sd >= 0.0f;
        return true;
    }
    return false;
}

// Grid namespace of a particle (transfer_key, world.rs:470-490): the transfer
// colour, and with CPIC the side mask of each CPIC group's closest triangle
// prism (colour << 8 | mask; groups below kMaxCpicGroups, colours below 256).
__device__ __forceinline__ uint32_t particle_namespace(uint32_t color, int cpic, int num_obstacles,
                                                       const DevObstacle *obstacles, V3f x) {
    if (!cpic) return color;
    float best[kMaxCpicGroups];
    uint32_t mask = 0;
#pragma unroll
    for (int g = 0; g < kMaxCpicGroups; ++g) best[g] = 3.0e38f;
    for (int oi = 0; oi < num_obstacles; ++oi) {
        const int g = obstacles[oi].cpic_group;
        if (g < 0 || g >= kMaxCpicGroups) continue;
        float d;
        bool pos;
        if (!cpic_side(obstacles[oi], x, d, pos)) continue;
#pragma unroll
        for (int q = 0; q < kMaxCpicGroups; ++q)
            if (q == g && d < best[q]) {
                best[q] = d;
                mask = pos ? (mask | (1u << q)) : (mask & ~(1u << q));
            }
    }
    return (color << 8) | mask;
}

// ---------------------------------------------------------------- binning

// floor(x * inv_h - 0.5) with IEEE round-to-nearest and no contraction
// (gpu.rs:1145, gpu.wgsl:947), so the host restatement reproduces it bit for bit.
__device__ __forceinline__ int base_cell(float x, float inv_h) {
    return __float2int_rd(__fsub_rn(__fmul_rn(x, inv_h), 0.5f));
}

__device__ __forceinline__ bool block_representable(int bx, int by, int bz) {
    return bx >= kBlockCoordMin && bx <= kBlockCoordMax && by >= kBlockCoordMin && by <= kBlockCoordMax &&
           bz >= kBlockCoordMin && bz <= kBlockCoordMax;
}

__device__ __forceinline__ unsigned long long block_key(int bx, int by, int bz, uint32_t color) {
    return (static_cast<unsigned long long>(color & 0xFFFFu) << 48) |
           (static_cast<unsigned long long>(static_cast<uint32_t>(bx + kBlockBias) & 0xFFFFu) << 32) |
           (static_cast<unsigned long long>(static_cast<uint32_t>(by + kBlockBias) & 0xFFFFu) << 16) |
           static_cast<unsigned long long>(static_cast<uint32_t>(bz + kBlockBias) & 0xFFFFu);
}

// Slot of a block key: a full 64-bit avalanche (the fmix64 finalizer of
// MurmurHash3, public domain), so the namespace bits (scene, colour) in the top
// 16 bits of the key spread over every slot bit.  A multiply alone would leave
// the low slot bits independent of the high key bits, and scenes or colours
// with the same block coordinates would pile onto the same probe chain.
__device__ __forceinline__ uint32_t hash_slot(unsigned long long key, uint32_t mask) {
    unsigned long long h = key;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return static_cast<uint32_t>(h) & mask;
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// 6-bit Morton code of a cell's position inside its 4^3 block.
__device__ __forceinline__ uint32_t cell_in_block(int cx, int cy, int cz) {
    const uint32_t x = static_cast<uint32_t>(cx) & 3u, y = static_cast<uint32_t>(cy) & 3u,
                   z = static_cast<uint32_t>(cz) & 3u;
    return ((x & 2u) << 4) | ((y & 2u) << 3) | ((z & 2u) << 2) | ((x & 1u) << 2) | ((y & 1u) << 1) | (z & 1u);
}

// Sort key of a block: scene index (8 bits) above the 21-bit Morton code of the
// block coordinates taken modulo 128 (512 cells per axis); bit 29 marks
// particles of removed scenes (kDeadKey).
__device__ __forceinline__ uint32_t morton_block(int bx, int by, int bz, uint32_t scene) {
    return ((scene & 0xFFu) << 21) | (spread10(static_cast<uint32_t>(bx) & 0x7Fu) << 2) |
           (spread10(static_cast<uint32_t>(by) & 0x7Fu) << 1) | spread10(static_cast<uint32_t>(bz) & 0x7Fu);
}

// Find the block id of `key`, allocating the block if absent.  Ids grow from
// zero after each table clear and both node pools are zeroed with it, so a
// new block's nodes are zero already (the grid update zeroes the blocks in use
// for their next accumulation).  The allocating thread records the block's
// coordinates before publishing the id with a release store; other threads
// that find the key wait (bounded) for the id with acquire loads.  Returns -1
// and sets a status bit on exhaustion or timeout.
__device__ inline int find_or_insert_block(const GridTable &g, unsigned long long key, int4 coord, uint32_t *status) {
    uint32_t slot = hash_slot(key, g.mask);
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> kref(g.keys[slot]);
        unsigned long long k = kref.load(cuda::memory_order_relaxed);
        if (k == kEmptyKey) {
            unsigned long long expected = kEmptyKey;
            if (kref.compare_exchange_strong(expected, key, cuda::memory_order_relaxed)) {
                uint32_t id = atomicAdd(g.count, 1u);
                cuda::atomic_ref<uint32_t, cuda::thread_scope_device> vref(g.vals[slot]);
                if (id >= g.max_blocks) {
                    atomicOr(status, kStatusCapacity);
                    vref.store(kInvalidId, cuda::memory_order_release);
                    return -1;
                }
                g.coords[id] = coord;
                vref.store(id, cuda::memory_order_release);
                return static_cast<int>(id);
            }
            k = expected;
        }
        if (k == key) {
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device> vref(g.vals[slot]);
            for (int it = 0; it < kSpinLimit; ++it) {
                uint32_t v = vref.load(cuda::memory_order_acquire);
                if (v != kPendingId) return v == kInvalidId ? -1 : static_cast<int>(v);
                __nanosleep(64);
            }
            atomicOr(status, kStatusTimeout);
            return -1;
        }
        slot = (slot + 1) & g.mask;
    }
    atomicOr(status, kStatusCapacity);
    return -1;
}

// Read-only lookup in a table whose inserts completed in an earlier kernel.
__device__ __forceinline__ int lookup_block(const GridTable &g, unsigned long long key) {
    uint32_t slot = hash_slot(key, g.mask);
    for (int probe = 0; probe < kMaxProbe; ++probe) {
        unsigned long long k = __ldcg(g.keys + slot);
        if (k == key) {
            uint32_t v = __ldcg(g.vals + slot);
            return v >= kInvalidId ? -1 : static_cast<int>(v);
        }
        if (k == kEmptyKey) return -1;
        slot = (slot + 1) & g.mask;
    }
    return -1;
}

__device__ __forceinline__ void red_add_v4(float4 *addr, float4 v) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}

}  // namespace tmpm
