// mpm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A CPU restatement, in f64 and on one thread, of tessera-mpm's deterministic
// MLS-MPM reference pipeline:
//   * crates/tessera-mpm/src/world.rs    (world, substep, grid, walls, obstacles)
//   * crates/tessera-mpm/src/material.rs (stress, return maps, CFL bound)
//   * crates/tessera-mpm/src/obstacle.rs (shapes, signed distance, contact velocity)
// Each function cites the reference lines it follows.  The sparse grid is an
// ordered map keyed by (cell, transfer key) compared lexicographically, the same
// ordering as the reference's BTreeMap<([i32; 3], u64), GridNode>.
//
// Third-party arithmetic: the reference calls nalgebra 0.30.1 (Cargo.lock, not
// vendored) for Matrix3::svd (material.rs:534-537), determinant and products.
// The polar factor R = U V^T of a non-singular F is unique, so any correct f64
// polar decomposition reproduces it; here it is Newton's iteration
// X <- (X + X^-T) / 2 run to convergence.  Singular values for the plastic
// return maps come from a cyclic Jacobi eigen-decomposition of F^T F run to
// convergence; the projections U diag(f(sigma)) V^T are invariant to the SVD's
// ordering and sign conventions.

#include "mpm_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <thread>
#include <tuple>
#include <vector>

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kF32Eps = 1.1920928955078125e-7;  // f32::EPSILON

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    double &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
V3 operator*(double s, V3 a) { return {a.x * s, a.y * s, a.z * s}; }
V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
V3 &operator+=(V3 &a, V3 b) { a = a + b; return a; }
V3 &operator-=(V3 &a, V3 b) { a = a - b; return a; }
V3 &operator*=(V3 &a, double s) { a = a * s; return a; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double norm(V3 a) { return std::sqrt(dot(a, a)); }
double norm_sq(V3 a) { return dot(a, a); }
V3 normalize(V3 a) { return a / norm(a); }
bool finite3(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

struct M3 {
    double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // m[row][col]
    static M3 zeros() { return M3(); }
    static M3 identity() {
        M3 r;
        r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0;
        return r;
    }
    static M3 diag(V3 d) {
        M3 r;
        r.m[0][0] = d.x;
        r.m[1][1] = d.y;
        r.m[2][2] = d.z;
        return r;
    }
    V3 col(int c) const { return {m[0][c], m[1][c], m[2][c]}; }
};
M3 operator+(const M3 &a, const M3 &b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] + b.m[i][j];
    return r;
}
M3 operator-(const M3 &a, const M3 &b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] - b.m[i][j];
    return r;
}
M3 operator*(const M3 &a, double s) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j] * s;
    return r;
}
M3 operator*(const M3 &a, const M3 &b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += a.m[i][k] * b.m[k][j];
            r.m[i][j] = s;
        }
    return r;
}
V3 operator*(const M3 &a, V3 v) {
    return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z,
            a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
M3 &operator+=(M3 &a, const M3 &b) { a = a + b; return a; }
M3 transpose(const M3 &a) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[j][i];
    return r;
}
double det(const M3 &a) {
    return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
           a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
           a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
}
double trace(const M3 &a) { return a.m[0][0] + a.m[1][1] + a.m[2][2]; }
double fro(const M3 &a) {
    double s = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s += a.m[i][j] * a.m[i][j];
    return std::sqrt(s);
}
M3 outer(V3 a, V3 b) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a[i] * b[j];
    return r;
}
bool finite_m(const M3 &a) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (!std::isfinite(a.m[i][j])) return false;
    return true;
}
M3 from_cm(const double *cm) {
    M3 r;
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr) r.m[rr][c] = cm[c * 3 + rr];
    return r;
}
void to_cm(const M3 &a, double *cm) {
    for (int c = 0; c < 3; ++c)
        for (int rr = 0; rr < 3; ++rr) cm[c * 3 + rr] = a.m[rr][c];
}
bool inverse(const M3 &a, M3 &out) {
    double d = det(a);
    if (d == 0.0 || !std::isfinite(d)) return false;
    V3 c0 = a.col(0), c1 = a.col(1), c2 = a.col(2);
    // rows of the inverse are the cross products of the columns divided by det
    V3 r0 = cross(c1, c2) / d, r1 = cross(c2, c0) / d, r2 = cross(c0, c1) / d;
    for (int j = 0; j < 3; ++j) {
        out.m[0][j] = r0[j];
        out.m[1][j] = r1[j];
        out.m[2][j] = r2[j];
    }
    return true;
}

// Polar factor R of F = R S (unique for det F != 0): Newton X <- (X + X^-T)/2.
bool polar_rotation(const M3 &F, M3 &R) {
    M3 X = F;
    for (int it = 0; it < 100; ++it) {
        M3 inv;
        if (!inverse(X, inv)) return false;
        M3 next = (X + transpose(inv)) * 0.5;
        double change = fro(next - X);
        X = next;
        if (change <= 1e-15 * std::max(1.0, fro(X))) break;
    }
    R = X;
    return finite_m(R);
}

// Symmetric eigen-decomposition by cyclic Jacobi: A = V diag(w) V^T.
void sym_eigen(M3 A, V3 &w, M3 &V) {
    V = M3::identity();
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = A.m[0][1] * A.m[0][1] + A.m[0][2] * A.m[0][2] + A.m[1][2] * A.m[1][2];
        double scale = A.m[0][0] * A.m[0][0] + A.m[1][1] * A.m[1][1] + A.m[2][2] * A.m[2][2];
        if (off <= 1e-32 * scale || off == 0.0) break;
        const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
        for (auto &pq : pairs) {
            int p = pq[0], q = pq[1];
            double apq = A.m[p][q];
            if (apq == 0.0) continue;
            double theta = (A.m[q][q] - A.m[p][p]) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
            double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
            M3 J = M3::identity();
            J.m[p][p] = c;
            J.m[q][q] = c;
            J.m[p][q] = s;
            J.m[q][p] = -s;
            A = transpose(J) * A * J;
            A.m[p][q] = A.m[q][p] = 0.0;
            V = V * J;
        }
    }
    w = {A.m[0][0], A.m[1][1], A.m[2][2]};
}

// F = U diag(sigma) V^T with sigma >= 0 (material.rs:534-537 via nalgebra).
bool svd3(const M3 &F, M3 &U, V3 &sigma, M3 &V) {
    V3 w;
    sym_eigen(transpose(F) * F, w, V);
    for (int i = 0; i < 3; ++i) sigma[i] = std::sqrt(std::max(w[i], 0.0));
    V3 u[3];
    int good[3] = {0, 0, 0};
    double smax = std::max(sigma.x, std::max(sigma.y, sigma.z));
    for (int i = 0; i < 3; ++i) {
        if (sigma[i] > 1e-300 && sigma[i] > 1e-14 * smax) {
            u[i] = (F * V.col(i)) / sigma[i];
            good[i] = 1;
        }
    }
    int ngood = good[0] + good[1] + good[2];
    if (ngood == 0) {
        U = M3::identity();
    } else {
        // Gram-Schmidt the computed columns, then complete an orthonormal basis.
        for (int i = 0; i < 3; ++i) {
            if (!good[i]) continue;
            for (int j = 0; j < i; ++j)
                if (good[j]) u[i] -= u[j] * dot(u[i], u[j]);
            u[i] = normalize(u[i]);
        }
        for (int i = 0; i < 3; ++i) {
            if (good[i]) continue;
            V3 a = good[(i + 1) % 3] ? u[(i + 1) % 3] : V3(1, 0, 0);
            V3 b = good[(i + 2) % 3] ? u[(i + 2) % 3] : V3(0, 1, 0);
            V3 c = cross(a, b);
            if (norm(c) < 1e-12) c = cross(a, V3(0, 0, 1));
            u[i] = normalize(c);
            good[i] = 1;
        }
        for (int i = 0; i < 3; ++i)
            for (int r = 0; r < 3; ++r) U.m[r][i] = u[i][r];
    }
    return finite_m(U) && finite_m(V) && finite3(sigma);
}

// ---------------------------------------------------------------- materials

struct Material {
    int kind = TMPM_MAT_ELASTIC;
    double p[5] = {0, 0, 0, 0, 0};
};

struct Plastic {
    double det = 1.0;       // plastic_det
    double hardening = 0.0;
    double lvg = 0.0;       // log_volume_gain
};

// lame (material.rs:433-438)
void lame(double young, double poisson, double &lambda, double &mu) {
    lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    mu = young / (2.0 * (1.0 + poisson));
}

// valid_elasticity (material.rs:429-431)
bool valid_elasticity(double young, double poisson) {
    return std::isfinite(young) && young > 0.0 && std::isfinite(poisson) && poisson >= -1.0 && poisson < 0.5;
}

// MaterialModel::is_valid (material.rs:171-231)
bool material_valid(const Material &m) {
    const double *p = m.p;
    switch (m.kind) {
    case TMPM_MAT_ELASTIC:
    case TMPM_MAT_NEO_HOOKEAN:
        return valid_elasticity(p[0], p[1]);
    case TMPM_MAT_SAND:
    case TMPM_MAT_SAND_NEO_HOOKEAN:
        return valid_elasticity(p[0], p[1]) && std::isfinite(p[2]) && p[2] >= 0.0 &&
               p[2] < M_PI / 2.0 && std::isfinite(p[3]) && p[3] >= 0.0;
    case TMPM_MAT_FLUID:
        return std::isfinite(p[0]) && p[0] > 0.0 && std::isfinite(p[1]) && p[1] > 0.0 &&
               std::isfinite(p[2]) && p[2] >= 0.0 && std::isfinite(p[3]) && p[3] >= 0.0;
    case TMPM_MAT_SNOW:
        return valid_elasticity(p[0], p[1]) && std::isfinite(p[2]) && p[2] >= 0.0 && p[2] < 1.0 &&
               std::isfinite(p[3]) && p[3] >= 0.0 && std::isfinite(p[4]) && p[4] >= 0.0;
    default:
        return false;
    }
}

// corotated_stress (material.rs:440-455)
M3 corotated_stress(const M3 &F, double young, double poisson, double factor) {
    double lambda, mu;
    lame(young, poisson, lambda, mu);
    M3 R;
    if (!polar_rotation(F, R)) return M3::zeros();
    double j = det(F);
    M3 stress = (F - R) * transpose(F) * (2.0 * mu * factor);
    stress += M3::identity() * (lambda * factor * (j - 1.0) * j);
    return stress;
}

// neo_hookean_stress (material.rs:457-467)
M3 neo_hookean_stress(const M3 &F, double young, double poisson, double factor) {
    double lambda, mu;
    lame(young, poisson, lambda, mu);
    double j = std::max(det(F), 1e-10);
    return F * transpose(F) * (mu * factor) + M3::identity() * (factor * (lambda * std::log(j) - mu));
}

// fluid_stress (material.rs:469-486)
M3 fluid_stress(const M3 &F, const M3 &C, double bulk, double gamma, double viscosity, double tensile) {
    double j = std::max(det(F), 1e-6);
    double pressure = j <= 1.0 ? bulk * (std::pow(j, -gamma) - 1.0) : -bulk * tensile * (j - 1.0);
    M3 strain_rate = (C + transpose(C)) * 0.5;
    M3 deviatoric = strain_rate - M3::identity() * (trace(strain_rate) / 3.0);
    return deviatoric * (2.0 * viscosity * j) - M3::identity() * (pressure * j);
}

// MaterialModel::kirchhoff_stress (material.rs:233-284)
M3 kirchhoff_stress(const Material &m, const M3 &F, const M3 &C, const Plastic &pl) {
    const double *p = m.p;
    switch (m.kind) {
    case TMPM_MAT_ELASTIC:
        return corotated_stress(F, p[0], p[1], 1.0);
    case TMPM_MAT_NEO_HOOKEAN:
    case TMPM_MAT_SAND_NEO_HOOKEAN:
        return neo_hookean_stress(F, p[0], p[1], 1.0);
    case TMPM_MAT_SAND:
        return corotated_stress(F, p[0], p[1], 1.0);
    case TMPM_MAT_FLUID:
        return fluid_stress(F, C, p[0], p[1], p[2], p[3]);
    case TMPM_MAT_SNOW: {
        double factor = std::min(std::max(std::exp(p[4] * (1.0 - pl.det)), 0.01), 100.0);
        return corotated_stress(F, p[0], p[1], factor);
    }
    }
    return M3::zeros();
}

// project_sand (material.rs:488-532)
void project_sand(M3 &F, Plastic &pl, double young, double poisson, double friction, double cohesion) {
    double lambda, mu;
    lame(young, poisson, lambda, mu);
    if (lambda == 0.0) return;
    M3 U, Vm;
    V3 s;
    if (!svd3(F, U, s, Vm)) return;
    V3 strain;
    for (int i = 0; i < 3; ++i) strain[i] = std::log(std::max(s[i], 1e-12)) + pl.lvg / 3.0;
    double tr = strain.x + strain.y + strain.z;
    V3 dev = strain - V3(tr / 3.0, tr / 3.0, tr / 3.0);
    double nrm = norm(dev);
    double shifted = tr - cohesion;
    double q = pl.hardening;
    double angle = friction + (9.0 * M_PI / 180.0 * q - 10.0 * M_PI / 180.0) * std::exp(-0.2 * q);
    double sine = std::sin(angle);
    double alpha = std::sqrt(2.0 / 3.0) * (2.0 * sine) / (3.0 - sine);
    V3 plog;
    double inc;
    if (shifted > 0.0 || nrm <= 4.0 * kF32Eps) {
        plog = V3(cohesion / 3.0, cohesion / 3.0, cohesion / 3.0);
        inc = norm(strain);
    } else {
        double gamma = nrm + (3.0 * lambda + 2.0 * mu) / (2.0 * mu) * shifted * alpha;
        if (gamma <= 0.0) return;
        plog = strain - dev * (gamma / nrm);
        inc = gamma;
    }
    V3 proj(std::exp(plog.x), std::exp(plog.y), std::exp(plog.z));
    double old_det = std::max(s.x * s.y * s.z, 1e-12);
    double new_det = std::max(proj.x * proj.y * proj.z, 1e-12);
    pl.det = std::min(std::max(pl.det * old_det / new_det, 0.01), 100.0);
    pl.lvg += std::log(old_det) - std::log(new_det);
    pl.hardening += inc;
    F = U * M3::diag(proj) * transpose(Vm);
}

// MaterialModel::project_deformation (material.rs:286-371)
void project_deformation(const Material &m, M3 &F, Plastic &pl) {
    const double *p = m.p;
    switch (m.kind) {
    case TMPM_MAT_FLUID: {
        double j = std::max(det(F), 1e-9);
        F = M3::identity() * std::cbrt(j);
        return;
    }
    case TMPM_MAT_SNOW: {
        M3 U, Vm;
        V3 s;
        if (!svd3(F, U, s, Vm)) return;
        V3 cl;
        for (int i = 0; i < 3; ++i) cl[i] = std::min(std::max(s[i], 1.0 - p[2]), 1.0 + p[3]);
        double old_det = s.x * s.y * s.z;
        double new_det = std::max(cl.x * cl.y * cl.z, 1e-12);
        pl.det = std::min(std::max(pl.det * old_det / new_det, 0.1), 4.0);
        F = U * M3::diag(cl) * transpose(Vm);
        return;
    }
    case TMPM_MAT_SAND:
        project_sand(F, pl, p[0], p[1], p[2], p[3]);
        return;
    case TMPM_MAT_SAND_NEO_HOOKEAN: {
        double lambda, mu;
        lame(p[0], p[1], lambda, mu);
        if (lambda == 0.0) return;
        M3 U, Vm;
        V3 s;
        if (!svd3(F, U, s, Vm)) return;
        V3 strain;
        for (int i = 0; i < 3; ++i) strain[i] = std::log(s[i]) + pl.lvg / 3.0;
        double tr = strain.x + strain.y + strain.z;
        V3 dev = strain - V3(tr / 3.0, tr / 3.0, tr / 3.0);
        double nrm = norm(dev);
        double shifted = tr - p[3];
        double q = pl.hardening;
        double angle = p[2] + (9.0 * M_PI / 180.0 * q - 10.0 * M_PI / 180.0) * std::exp(-0.2 * q);
        double sine = std::sin(angle);
        double alpha = std::sqrt(2.0 / 3.0) * (2.0 * sine) / (3.0 - sine);
        bool isotropic = nrm <= 4.0 * kF32Eps;
        V3 plog;
        double inc;
        if (shifted > 0.0 || isotropic) {
            plog = V3(p[3] / 3.0, p[3] / 3.0, p[3] / 3.0);
            inc = norm(strain);
        } else {
            double gamma = nrm + (3.0 * lambda + 2.0 * mu) / (2.0 * mu) * shifted * alpha;
            if (gamma <= 0.0) return;
            plog = strain - dev * (gamma / nrm);
            inc = gamma;
        }
        V3 proj(std::exp(plog.x), std::exp(plog.y), std::exp(plog.z));
        double old_det = s.x * s.y * s.z;
        double new_det = proj.x * proj.y * proj.z;
        pl.det *= old_det / new_det;
        pl.lvg += std::log(old_det) - std::log(new_det);
        pl.hardening += inc;
        F = U * M3::diag(proj) * transpose(Vm);
        return;
    }
    default:
        return;  // LinearElastic, NeoHookean: unchanged (material.rs:369)
    }
}

// MaterialModel::timestep_bound_with_deformation (material.rs:378-426)
double timestep_bound(const Material &m, double density, V3 velocity, double h, double det_f) {
    const double *p = m.p;
    double wave;
    if (m.kind == TMPM_MAT_SAND_NEO_HOOKEAN) {
        double lambda, mu;
        lame(p[0], p[1], lambda, mu);
        double rho = density / std::max(det_f, 1e-6);
        double ws = std::sqrt((lambda + 2.0 * mu) / rho);
        return 0.5 * h / std::max(ws, norm(velocity));
    } else if (m.kind == TMPM_MAT_FLUID) {
        wave = std::sqrt(p[0] * p[1] / std::max(density, 1e-12));
    } else {
        double lambda, mu;
        lame(p[0], p[1], lambda, mu);
        wave = std::sqrt((lambda + 2.0 * mu) / std::max(density, 1e-12));
    }
    return 0.4 * h / std::max(wave + norm(velocity), 1e-12);
}

// ---------------------------------------------------------------- obstacles

struct Quat {
    double x = 0, y = 0, z = 0, w = 1;
};

// UnitQuaternion * v (nalgebra): t = 2 q_v x v; v + w t + q_v x t
V3 rotate(const Quat &q, V3 v) {
    V3 qv(q.x, q.y, q.z);
    V3 t = cross(qv, v) * 2.0;
    return v + t * q.w + cross(qv, t);
}
V3 inv_rotate(const Quat &q, V3 v) {
    Quat c{-q.x, -q.y, -q.z, q.w};
    return rotate(c, v);
}

struct Obstacle {
    int shape = TMPM_SHAPE_SPHERE;
    int boundary = TMPM_BOUNDARY_SLIP;
    int cpic_group = -1;
    V3 center;
    Quat q;
    V3 lin, ang;
    double friction = 0.0;
    double dims[3] = {0, 0, 0};
    V3 verts[3];
    double bound_radius = 0.0;
    std::vector<double> planes;  // 4 per plane
};

Obstacle obstacle_from(const TmpmObstacle &o) {
    Obstacle r;
    r.shape = o.shape;
    r.boundary = o.boundary;
    r.cpic_group = o.cpic_group;
    r.center = V3(o.center[0], o.center[1], o.center[2]);
    r.q = Quat{o.orientation[0], o.orientation[1], o.orientation[2], o.orientation[3]};
    r.lin = V3(o.linear_velocity[0], o.linear_velocity[1], o.linear_velocity[2]);
    r.ang = V3(o.angular_velocity[0], o.angular_velocity[1], o.angular_velocity[2]);
    r.friction = o.friction;
    for (int i = 0; i < 3; ++i) r.dims[i] = o.dims[i];
    for (int i = 0; i < 3; ++i) r.verts[i] = V3(o.vertices[3 * i], o.vertices[3 * i + 1], o.vertices[3 * i + 2]);
    r.bound_radius = o.bound_radius;
    if (o.shape == TMPM_SHAPE_CONVEX && o.planes && o.plane_count)
        r.planes.assign(o.planes, o.planes + 4 * static_cast<size_t>(o.plane_count));
    return r;
}

// RigidObstacle::is_valid (obstacle.rs:264-341)
bool obstacle_valid(const Obstacle &o) {
    bool shape_ok = false;
    const double *d = o.dims;
    switch (o.shape) {
    case TMPM_SHAPE_SPHERE:
        shape_ok = std::isfinite(d[0]) && d[0] > 0.0;
        break;
    case TMPM_SHAPE_BOX:
        shape_ok = std::isfinite(d[0]) && d[0] > 0 && std::isfinite(d[1]) && d[1] > 0 && std::isfinite(d[2]) && d[2] > 0;
        break;
    case TMPM_SHAPE_CAPSULE:
        shape_ok = std::isfinite(d[0]) && d[0] >= 0.0 && std::isfinite(d[1]) && d[1] >= 0.0 && (d[0] > 0.0 || d[1] > 0.0);
        break;
    case TMPM_SHAPE_CYLINDER:
    case TMPM_SHAPE_CONE:
        shape_ok = std::isfinite(d[0]) && d[0] > 0.0 && std::isfinite(d[1]) && d[1] > 0.0;
        break;
    case TMPM_SHAPE_GROUND:
        shape_ok = std::isfinite(d[0]) && d[0] > 0.0 && std::isfinite(d[1]) && d[1] > 0.0;
        break;
    case TMPM_SHAPE_TRIANGLE_PRISM: {
        double area_sq = norm_sq(cross(o.verts[1] - o.verts[0], o.verts[2] - o.verts[0]));
        shape_ok = std::isfinite(d[0]) && d[0] > 0.0 && finite3(o.verts[0]) && finite3(o.verts[1]) &&
                   finite3(o.verts[2]) && std::isfinite(area_sq) && area_sq > 1e-24;
        break;
    }
    case TMPM_SHAPE_CONVEX: {
        size_t n = o.planes.size() / 4;
        shape_ok = n >= 4 && std::isfinite(o.bound_radius) && o.bound_radius > 0.0;
        for (size_t i = 0; shape_ok && i < n; ++i) {
            const double *pl = &o.planes[4 * i];
            bool fin = std::isfinite(pl[0]) && std::isfinite(pl[1]) && std::isfinite(pl[2]) && std::isfinite(pl[3]);
            double n2 = std::fma(pl[0], pl[0], std::fma(pl[1], pl[1], pl[2] * pl[2]));
            shape_ok = fin && std::fabs(n2 - 1.0) <= 1e-4;
        }
        break;
    }
    default:
        shape_ok = false;
    }
    bool cpic_ok = o.cpic_group < 0 || (o.cpic_group < 32 && o.shape == TMPM_SHAPE_TRIANGLE_PRISM);
    bool boundary_ok = o.boundary >= 0 && o.boundary <= 4;
    return shape_ok && cpic_ok && boundary_ok && finite3(o.center) && std::isfinite(o.q.x) &&
           std::isfinite(o.q.y) && std::isfinite(o.q.z) && std::isfinite(o.q.w) && finite3(o.lin) &&
           finite3(o.ang) && std::isfinite(o.friction) && o.friction >= 0.0;
}

// cylinder_surface (obstacle.rs:542-587)
void cylinder_surface(V3 local, double hh, double radius, double &dist, V3 &normal) {
    double radial = std::hypot(local.x, local.y);
    V3 rn = radial > 1e-12 ? V3(local.x / radial, local.y / radial, 0.0) : V3(1, 0, 0);
    double rd = radial - radius;
    double cd = std::fabs(local.z) - hh;
    double eps = std::max(hh, radius) * 1e-6;
    if (std::fabs(rd) <= eps && std::fabs(cd) <= eps) {
        V3 cap = local.z < 0.0 ? V3(0, 0, -1) : V3(0, 0, 1);
        dist = std::max(rd, cd);
        normal = normalize(rn + cap);
        return;
    }
    double ro = std::max(rd, 0.0), co = std::max(cd, 0.0);
    V3 outside = rn * ro + V3(0, 0, 1) * (local.z < 0.0 ? -co : co);
    double ol = norm(outside);
    if (ol > 1e-12) {
        dist = ol;
        normal = outside / ol;
    } else if (rd >= cd) {
        dist = rd;
        normal = rn;
    } else {
        dist = cd;
        normal = local.z < 0.0 ? V3(0, 0, -1) : V3(0, 0, 1);
    }
}

// cone_surface (obstacle.rs:589-631)
void cone_surface(V3 local, double hh, double radius, double &dist, V3 &normal) {
    double radial = std::hypot(local.x, local.y);
    V3 rn = radial > 1e-12 ? V3(local.x / radial, local.y / radial, 0.0) : V3(1, 0, 0);
    double px = radial, py = local.z;
    double bx = std::min(std::max(radial, 0.0), radius), by = -hh;
    double sx = radius, sy = -hh;
    double dx = -radius, dy = 2.0 * hh;
    double t = ((px - sx) * dx + (py - sy) * dy) / (dx * dx + dy * dy);
    t = std::min(std::max(t, 0.0), 1.0);
    double sidex = sx + dx * t, sidey = sy + dy * t;
    double eps = std::max(hh, radius) * 1e-6;
    double bd2 = (px - bx) * (px - bx) + (py - by) * (py - by);
    double sd2 = (px - sidex) * (px - sidex) + (py - sidey) * (py - sidey);
    bool use_base = bd2 <= sd2;
    double cx = use_base ? bx : sidex, cy = use_base ? by : sidey;
    double ddx = px - cx, ddy = py - cy;
    double nrm = std::sqrt(ddx * ddx + ddy * ddy);
    bool inside = local.z >= -hh - eps && local.z <= hh + eps && radial <= radius * (hh - local.z) / (2.0 * hh) + eps;
    double bnx = 0.0, bny = -1.0;
    double snl = std::sqrt(4.0 * hh * hh + radius * radius);
    double snx = 2.0 * hh / snl, sny = radius / snl;
    bool near_corner = bd2 <= eps * eps && sd2 <= eps * eps;
    double fnx, fny;
    if (near_corner) {
        double ax = bnx + snx, ay = bny + sny;
        double al = std::sqrt(ax * ax + ay * ay);
        fnx = ax / al;
        fny = ay / al;
    } else if (use_base) {
        fnx = bnx;
        fny = bny;
    } else {
        fnx = snx;
        fny = sny;
    }
    double n2x, n2y;
    if (inside || nrm <= eps) {
        n2x = fnx;
        n2y = fny;
    } else {
        n2x = ddx / nrm;
        n2y = ddy / nrm;
    }
    normal = rn * n2x + V3(0, 0, 1) * n2y;
    dist = inside ? -nrm : nrm;
}

// closest_point_triangle (obstacle.rs:747-787)
V3 closest_point_triangle(V3 p, V3 a, V3 b, V3 c) {
    V3 ab = b - a, ac = c - a, ap = p - a;
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return a;
    V3 bp = p - b;
    double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return b;
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return a + ab * (d1 / (d1 - d3));
    V3 cp = p - c;
    double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return c;
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return a + ac * (d2 / (d2 - d6));
    double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && d4 - d3 >= 0.0 && d5 - d6 >= 0.0) return b + (c - b) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)));
    double rec = 1.0 / (va + vb + vc);
    return a + ab * (vb * rec) + ac * (vc * rec);
}

// triangle_prism_surface (obstacle.rs:633-694)
void triangle_prism_surface(V3 p, const V3 *v, double ht, double &dist, V3 &normal) {
    V3 a = v[0], b = v[1], c = v[2];
    V3 n = normalize(cross(b - a, c - a));
    V3 off = n * ht;
    V3 prism[6] = {a + off, b + off, c + off, a - off, b - off, c - off};
    const int faces[8][3] = {{0, 1, 2}, {3, 5, 4}, {3, 4, 1}, {3, 1, 0}, {4, 5, 2}, {4, 2, 1}, {5, 3, 0}, {5, 0, 2}};
    double edge = std::max(std::max(norm(b - a), norm(c - b)), std::max(norm(a - c), ht));
    double eps = edge * 1e-6;
    bool inside = true;
    V3 closest;
    double best = kInf;
    V3 best_n = n, tied;
    for (auto &f : faces) {
        V3 fa = prism[f[0]], fb = prism[f[1]], fc = prism[f[2]];
        V3 fn = normalize(cross(fb - fa, fc - fa));
        inside = inside && dot(p - fa, fn) <= eps;
        V3 cand = closest_point_triangle(p, fa, fb, fc);
        double d2 = norm_sq(p - cand);
        if (d2 + eps * eps < best) {
            best = d2;
            closest = cand;
            best_n = fn;
            tied = fn;
        } else if (std::fabs(d2 - best) <= eps * eps) {
            tied += fn;
        }
    }
    double distance = std::sqrt(best);
    double tn = norm(tied);
    V3 feature = tn > 1e-12 ? tied / tn : best_n;
    V3 outward = (inside || distance <= eps) ? feature : (p - closest) / distance;
    dist = inside ? -distance : distance;
    normal = outward;
}

// convex_surface (obstacle.rs:696-745)
void convex_surface(V3 p, const std::vector<double> &planes, double bound_radius, double &dist, V3 &normal) {
    size_t n = planes.size() / 4;
    double maximum = -kInf;
    V3 nearest(0, 0, 1);
    for (size_t i = 0; i < n; ++i) {
        V3 pn(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2]);
        double d = dot(pn, p) - planes[4 * i + 3];
        if (d > maximum) {
            maximum = d;
            nearest = pn;
        }
    }
    if (maximum <= 0.0) {
        dist = maximum;
        normal = nearest;
        return;
    }
    V3 projected = p;
    std::vector<V3> corr(n);
    double tol = std::max(bound_radius, 1.0) * 1e-10;
    for (int it = 0; it < 128; ++it) {
        V3 prev = projected;
        for (size_t i = 0; i < n; ++i) {
            V3 pn(planes[4 * i], planes[4 * i + 1], planes[4 * i + 2]);
            V3 shifted = projected + corr[i];
            double viol = std::max(dot(pn, shifted) - planes[4 * i + 3], 0.0);
            projected = shifted - pn * viol;
            corr[i] = shifted - projected;
        }
        if (norm(projected - prev) <= tol) break;
    }
    V3 offset = p - projected;
    double d = norm(offset);
    if (d > tol) {
        dist = d;
        normal = offset / d;
    } else {
        dist = maximum;
        normal = nearest;
    }
}

// RigidObstacle::surface (obstacle.rs:372-472)
void obstacle_surface(const Obstacle &o, V3 point, double &dist, V3 &normal) {
    V3 rel = point - o.center;
    switch (o.shape) {
    case TMPM_SHAPE_SPHERE: {
        double n = norm(rel);
        normal = n > 1e-12 ? rel / n : V3(0, 0, 1);
        dist = n - o.dims[0];
        return;
    }
    case TMPM_SHAPE_BOX: {
        V3 local = inv_rotate(o.q, rel);
        V3 he(o.dims[0], o.dims[1], o.dims[2]);
        V3 closest;
        for (int i = 0; i < 3; ++i) closest[i] = std::min(std::max(local[i], -he[i]), he[i]);
        V3 outside = local - closest;
        double n = norm(outside);
        if (n > 1e-12) {
            dist = n;
            normal = rotate(o.q, outside / n);
        } else {
            V3 d = he - V3(std::fabs(local.x), std::fabs(local.y), std::fabs(local.z));
            int axis = (d.x <= d.y && d.x <= d.z) ? 0 : (d.y <= d.z ? 1 : 2);
            V3 nn;
            nn[axis] = local[axis] < 0.0 ? -1.0 : 1.0;
            dist = -d[axis];
            normal = rotate(o.q, nn);
        }
        return;
    }
    case TMPM_SHAPE_CAPSULE: {
        double hh = o.dims[0], r = o.dims[1];
        V3 local = inv_rotate(o.q, rel);
        double cz = std::min(std::max(local.z, -hh), hh);
        V3 delta = local - V3(0, 0, cz);
        double n = norm(delta);
        double eps = std::max(hh, r) * 1e-6;
        V3 nn = n > eps ? delta / n : V3(1, 0, 0);
        dist = n - r;
        normal = rotate(o.q, nn);
        return;
    }
    case TMPM_SHAPE_CYLINDER: {
        V3 local = inv_rotate(o.q, rel);
        V3 nn;
        cylinder_surface(local, o.dims[0], o.dims[1], dist, nn);
        normal = rotate(o.q, nn);
        return;
    }
    case TMPM_SHAPE_CONE: {
        V3 local = inv_rotate(o.q, rel);
        V3 nn;
        cone_surface(local, o.dims[0], o.dims[1], dist, nn);
        normal = rotate(o.q, nn);
        return;
    }
    case TMPM_SHAPE_GROUND: {
        V3 local = inv_rotate(o.q, rel);
        double ox = local.x - std::min(std::max(local.x, -o.dims[0]), o.dims[0]);
        double oy = local.y - std::min(std::max(local.y, -o.dims[1]), o.dims[1]);
        V3 outside(ox, oy, local.z);
        double hd = std::hypot(ox, oy);
        if (hd <= 1e-12) {
            dist = local.z;
            normal = rotate(o.q, V3(0, 0, 1));
        } else {
            double d = norm(outside);
            dist = d;
            normal = rotate(o.q, outside / d);
        }
        return;
    }
    case TMPM_SHAPE_TRIANGLE_PRISM: {
        V3 local = inv_rotate(o.q, rel);
        V3 nn;
        triangle_prism_surface(local, o.verts, o.dims[0], dist, nn);
        normal = rotate(o.q, nn);
        return;
    }
    case TMPM_SHAPE_CONVEX: {
        V3 local = inv_rotate(o.q, rel);
        V3 nn;
        convex_surface(local, o.planes, o.bound_radius, dist, nn);
        normal = rotate(o.q, nn);
        return;
    }
    }
    dist = kInf;
    normal = V3(0, 0, 1);
}

// RigidObstacle::may_contact (obstacle.rs:474-499)
bool may_contact(const Obstacle &o, V3 point, double margin) {
    switch (o.shape) {
    case TMPM_SHAPE_CAPSULE: {
        double b = o.dims[0] + o.dims[1] + margin;
        return norm_sq(point - o.center) <= b * b;
    }
    case TMPM_SHAPE_TRIANGLE_PRISM: {
        double r = std::max(std::max(std::max(0.0, norm(o.verts[0])), norm(o.verts[1])), norm(o.verts[2])) + o.dims[0] + margin;
        return norm_sq(point - o.center) <= r * r;
    }
    case TMPM_SHAPE_CONVEX: {
        double b = o.bound_radius + margin;
        return norm_sq(point - o.center) <= b * b;
    }
    default:
        return true;
    }
}

// RigidObstacle::contact_velocity (obstacle.rs:501-540)
V3 contact_velocity(const Obstacle &o, V3 point, V3 velocity, V3 normal) {
    V3 surface = o.lin + cross(o.ang, point - o.center);
    if (o.boundary == TMPM_BOUNDARY_NON_REFLECTING) return velocity;
    if (o.boundary == TMPM_BOUNDARY_STICK) return surface;
    V3 rel = velocity - surface;
    double ns = dot(rel, normal);
    if (o.boundary == TMPM_BOUNDARY_FREE_SLIP) return velocity - normal * ns;
    if (ns >= 0.0) return velocity;
    V3 tangent = rel - normal * ns;
    if (o.boundary == TMPM_BOUNDARY_SEPARATE) return surface + tangent;
    double ts = norm(tangent);
    double scale = ts > 1e-12 ? std::max(1.0 - o.friction * -ns / ts, 0.0) : 0.0;
    return surface + tangent * scale;
}

// RigidObstacle::cpic_side (obstacle.rs:343-370)
bool cpic_side(const Obstacle &o, V3 point, double &abs_signed, bool &positive) {
    if (o.shape != TMPM_SHAPE_TRIANGLE_PRISM) return false;
    V3 local = inv_rotate(o.q, point - o.center);
    V3 a = o.verts[0], eb = o.verts[1] - a, ec = o.verts[2] - a;
    V3 n = normalize(cross(eb, ec));
    double s = dot(local - a, n);
    V3 proj = local - n * s - a;
    double d00 = dot(eb, eb), d01 = dot(eb, ec), d11 = dot(ec, ec), d20 = dot(proj, eb), d21 = dot(proj, ec);
    double den = d00 * d11 - d01 * d01;
    double v = (d11 * d20 - d01 * d21) / den, w = (d00 * d21 - d01 * d20) / den;
    if (v >= -1e-8 && w >= -1e-8 && v + w <= 1.0 + 1e-8) {
        abs_signed = std::fabs(s);
        positive = s >= 0.0;
        return true;
    }
    return false;
}

// ---------------------------------------------------------------- world

struct Particle {
    V3 pos, vel;
    M3 F = M3::identity(), C;
    V3 force;
    double mass = 0, vol = 0, radius = 0, damping = 0;
    Material mat;
    Plastic pl;
    uint32_t group = 0;
    uint16_t color = 0;
    bool enabled = true, fixed = false;
    uint64_t chunk = 0;
};

struct Reaction {
    V3 lin, ang;
    void record(V3 center, V3 point, V3 impulse) {
        lin += impulse;
        ang += cross(point - center, impulse);
    }
};

struct Params {
    double h = 0.1;
    V3 g{0, 0, -9.81};
    double max_substep = 1e-3;
    bool has_bounds = false;
    int wall_mode = 0;
    V3 bmin, bmax;
};

// MpmParams::validate (world.rs:51-65)
bool params_valid(const Params &p) {
    if (!std::isfinite(p.h) || p.h <= 0.0 || !finite3(p.g) || !std::isfinite(p.max_substep) || p.max_substep <= 0.0)
        return false;
    if (p.has_bounds) {
        if (!finite3(p.bmin) || !finite3(p.bmax)) return false;
        for (int i = 0; i < 3; ++i)
            if (!(p.bmax[i] - p.bmin[i] > 0.0)) return false;
    }
    return p.wall_mode == 0 || p.wall_mode == 1;
}

Params params_from(const TmpmParams &p) {
    Params r;
    r.h = p.cell_width;
    r.g = V3(p.gravity[0], p.gravity[1], p.gravity[2]);
    r.max_substep = p.max_substep;
    r.has_bounds = p.has_bounds != 0;
    r.wall_mode = p.wall_mode;
    r.bmin = V3(p.bounds_min[0], p.bounds_min[1], p.bounds_min[2]);
    r.bmax = V3(p.bounds_max[0], p.bounds_max[1], p.bounds_max[2]);
    return r;
}

// finite_particle_state (world.rs:505-515)
bool finite_particle(const Particle &p) {
    return finite3(p.pos) && finite3(p.vel) && finite_m(p.F) && finite_m(p.C) && finite3(p.force) &&
           std::isfinite(p.mass) && std::isfinite(p.vol) && std::isfinite(p.radius) && std::isfinite(p.damping);
}

// valid_particle (world.rs:492-503)
bool valid_particle(const Particle &p) {
    return finite_particle(p) && p.mass > 0.0 && p.vol > 0.0 && p.radius > 0.0 && material_valid(p.mat) &&
           p.damping >= 0.0 && std::isfinite(p.pl.det) && p.pl.det > 0.0 && std::isfinite(p.pl.hardening) &&
           std::isfinite(p.pl.lvg);
}

std::vector<Particle> particles_from(const TmpmParticleArrays &a) {
    std::vector<Particle> out(a.count);
    for (size_t i = 0; i < a.count; ++i) {
        Particle &p = out[i];
        p.pos = V3(a.position[3 * i], a.position[3 * i + 1], a.position[3 * i + 2]);
        p.vel = V3(a.velocity[3 * i], a.velocity[3 * i + 1], a.velocity[3 * i + 2]);
        p.F = a.deformation ? from_cm(a.deformation + 9 * i) : M3::identity();
        p.C = a.affine ? from_cm(a.affine + 9 * i) : M3::zeros();
        if (a.force) p.force = V3(a.force[3 * i], a.force[3 * i + 1], a.force[3 * i + 2]);
        p.mass = a.mass[i];
        p.vol = a.rest_volume[i];
        p.radius = a.radius[i];
        p.damping = a.damping ? a.damping[i] : 0.0;
        p.mat.kind = a.material[i];
        for (int k = 0; k < 5; ++k) p.mat.p[k] = a.material_params[5 * i + k];
        if (a.plastic) {
            p.pl.det = a.plastic[3 * i];
            p.pl.hardening = a.plastic[3 * i + 1];
            p.pl.lvg = a.plastic[3 * i + 2];
        } else {
            p.pl.hardening = (p.mat.kind == TMPM_MAT_SAND || p.mat.kind == TMPM_MAT_SAND_NEO_HOOKEAN) ? 1.0 : 0.0;
        }
        p.enabled = a.enabled ? a.enabled[i] != 0 : true;
        p.fixed = a.fixed ? a.fixed[i] != 0 : false;
        p.color = a.transfer_color ? a.transfer_color[i] : 0;
        p.group = a.group_id ? a.group_id[i] : 0;
        p.chunk = a.chunk_id ? a.chunk_id[i] : 0;
    }
    return out;
}

void particles_to(const std::vector<Particle> &ps, TmpmParticleArrays &a) {
    for (size_t i = 0; i < ps.size(); ++i) {
        const Particle &p = ps[i];
        for (int k = 0; k < 3; ++k) {
            if (a.position) a.position[3 * i + k] = p.pos[k];
            if (a.velocity) a.velocity[3 * i + k] = p.vel[k];
            if (a.force) a.force[3 * i + k] = p.force[k];
        }
        if (a.deformation) to_cm(p.F, a.deformation + 9 * i);
        if (a.affine) to_cm(p.C, a.affine + 9 * i);
        if (a.mass) a.mass[i] = p.mass;
        if (a.rest_volume) a.rest_volume[i] = p.vol;
        if (a.radius) a.radius[i] = p.radius;
        if (a.damping) a.damping[i] = p.damping;
        if (a.plastic) {
            a.plastic[3 * i] = p.pl.det;
            a.plastic[3 * i + 1] = p.pl.hardening;
            a.plastic[3 * i + 2] = p.pl.lvg;
        }
        if (a.material) a.material[i] = p.mat.kind;
        if (a.material_params)
            for (int k = 0; k < 5; ++k) a.material_params[5 * i + k] = p.mat.p[k];
        if (a.enabled) a.enabled[i] = p.enabled;
        if (a.fixed) a.fixed[i] = p.fixed;
        if (a.transfer_color) a.transfer_color[i] = p.color;
        if (a.group_id) a.group_id[i] = p.group;
        if (a.chunk_id) a.chunk_id[i] = p.chunk;
    }
}

using GridKey = std::tuple<int32_t, int32_t, int32_t, uint64_t>;
struct GridNode {
    double mass = 0;
    V3 momentum, velocity;
};

// base_cell (world.rs:517-523)
void base_cell(V3 gp, int32_t b[3]) {
    for (int i = 0; i < 3; ++i) b[i] = static_cast<int32_t>(std::floor(gp[i] - 0.5));
}

// quadratic_weights (world.rs:529-538)
void quadratic_weights(V3 fx, double w[3][3]) {
    for (int a = 0; a < 3; ++a) {
        double v = fx[a];
        w[a][0] = 0.5 * (1.5 - v) * (1.5 - v);
        w[a][1] = 0.75 - (v - 1.0) * (v - 1.0);
        w[a][2] = 0.5 * (v - 0.5) * (v - 0.5);
    }
}

// apply_grid_boundary (world.rs:561-575); wall_mode 1 = sticky extension
void apply_grid_boundary(const int32_t id[3], double h, const Params &p, V3 &vel) {
    for (int a = 0; a < 3; ++a) {
        double pos = id[a] * h;
        bool lower = pos <= p.bmin[a] + h, upper = pos >= p.bmax[a] - h;
        if (p.wall_mode == 1) {
            if (lower || upper) vel = V3(0, 0, 0);
            continue;
        }
        if ((lower && vel[a] < 0.0) || (upper && vel[a] > 0.0)) vel[a] = 0.0;
    }
}

// apply_particle_boundary (world.rs:632-644)
void apply_particle_boundary(const Params &p, Particle &q) {
    for (int a = 0; a < 3; ++a) {
        double lower = p.bmin[a] + q.radius, upper = p.bmax[a] - q.radius;
        if (q.pos[a] < lower) {
            q.pos[a] = lower;
            q.vel[a] = std::max(q.vel[a], 0.0);
        } else if (q.pos[a] > upper) {
            q.pos[a] = upper;
            q.vel[a] = std::min(q.vel[a], 0.0);
        }
    }
}

}  // namespace

struct OrcWorld {
    std::vector<Particle> particles;
    Params params;
    std::vector<Obstacle> obstacles;
    uint64_t substeps = 0;
    bool use_cpic = true;
    uint64_t next_chunk = 1;

    // transfer_key (world.rs:470-490)
    uint64_t transfer_key(const Particle &p, bool with_cpic) const {
        double best[32];
        bool has[32] = {false}, side[32] = {false};
        if (with_cpic) {
            for (const Obstacle &o : obstacles) {
                if (o.cpic_group < 0) continue;
                double d;
                bool pos;
                if (cpic_side(o, p.pos, d, pos)) {
                    int g = o.cpic_group;
                    if (!has[g] || d < best[g]) {
                        has[g] = true;
                        best[g] = d;
                        side[g] = pos;
                    }
                }
            }
        }
        uint32_t mask = 0;
        for (int g = 0; g < 32; ++g)
            if (has[g] && side[g]) mask |= (1u << g);
        return (static_cast<uint64_t>(p.color) << 32) | mask;
    }

    // MpmWorld::stable_timestep (world.rs:288-303)
    double stable_timestep() const {
        double dt = params.max_substep;
        for (const Particle &p : particles) {
            if (!p.enabled || p.fixed) continue;
            dt = std::min(dt, timestep_bound(p.mat, p.mass / p.vol, p.vel, params.h, det(p.F)));
        }
        return std::min(dt, params.max_substep);
    }

    // P2G half of MpmWorld::substep (world.rs:366-399)
    void p2g(double dt, std::map<GridKey, GridNode> &grid, std::vector<uint64_t> &keys) const {
        double h = params.h, inv_h = 1.0 / h, inv_d = 4.0 * inv_h * inv_h;
        keys.resize(particles.size());
        for (size_t i = 0; i < particles.size(); ++i) keys[i] = transfer_key(particles[i], use_cpic);
        for (size_t i = 0; i < particles.size(); ++i) {
            const Particle &p = particles[i];
            if (!p.enabled) continue;
            V3 gp = p.pos * inv_h;
            int32_t b[3];
            base_cell(gp, b);
            V3 fx = gp - V3(b[0], b[1], b[2]);
            double w[3][3];
            quadratic_weights(fx, w);
            M3 stress = kirchhoff_stress(p.mat, p.F, p.C, p.pl);
            M3 force_affine = stress * (-dt * p.vol * inv_d);
            M3 mom_affine = force_affine + p.C * p.mass;
            for (int a = 0; a < 3; ++a)
                for (int bb = 0; bb < 3; ++bb)
                    for (int c = 0; c < 3; ++c) {
                        double weight = w[0][a] * w[1][bb] * w[2][c];
                        V3 dpos = (V3(a, bb, c) - fx) * h;
                        GridNode &node = grid[GridKey(b[0] + a, b[1] + bb, b[2] + c, keys[i])];
                        node.mass += weight * p.mass;
                        node.momentum += weight * (p.vel * p.mass + mom_affine * dpos);
                    }
        }
    }

    // MpmWorld::substep (world.rs:361-467)
    int32_t substep(double dt, Reaction *reactions) {
        double h = params.h, inv_h = 1.0 / h, inv_d = 4.0 * inv_h * inv_h;
        std::map<GridKey, GridNode> grid;
        std::vector<uint64_t> keys;
        p2g(dt, grid, keys);

        for (auto &kv : grid) {
            GridNode &node = kv.second;
            if (node.mass <= 0.0) continue;
            node.velocity = node.momentum / node.mass + params.g * dt;
            int32_t id[3] = {std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first)};
            if (params.has_bounds) apply_grid_boundary(id, h, params, node.velocity);
            // apply_grid_obstacles (world.rs:577-603)
            V3 point = V3(id[0], id[1], id[2]) * h;
            for (size_t oi = 0; oi < obstacles.size(); ++oi) {
                const Obstacle &o = obstacles[oi];
                if (!may_contact(o, point, h)) continue;
                double d;
                V3 n;
                obstacle_surface(o, point, d, n);
                if (d <= h * (1.0 + 1e-5)) {
                    V3 before = node.velocity;
                    node.velocity = contact_velocity(o, point, node.velocity, n);
                    if (reactions) reactions[oi].record(o.center, point - n * d, (before - node.velocity) * node.mass);
                }
            }
        }

        for (size_t i = 0; i < particles.size(); ++i) {
            Particle &p = particles[i];
            if (!p.enabled) {
                p.force = V3();
                continue;
            }
            if (p.fixed) {
                p.vel = V3();
                p.C = M3::zeros();
                p.force = V3();
                continue;
            }
            V3 gp = p.pos * inv_h;
            int32_t b[3];
            base_cell(gp, b);
            V3 fx = gp - V3(b[0], b[1], b[2]);
            double w[3][3];
            quadratic_weights(fx, w);
            V3 vel;
            M3 aff;
            for (int a = 0; a < 3; ++a)
                for (int bb = 0; bb < 3; ++bb)
                    for (int c = 0; c < 3; ++c) {
                        double weight = w[0][a] * w[1][bb] * w[2][c];
                        V3 dpos = (V3(a, bb, c) - fx) * h;
                        auto it = grid.find(GridKey(b[0] + a, b[1] + bb, b[2] + c, keys[i]));
                        V3 nv = it == grid.end() ? V3() : it->second.velocity;
                        vel += nv * weight;
                        aff += outer(nv, dpos) * (weight * inv_d);
                    }
            vel += p.force / p.mass * dt;
            vel *= std::exp(-p.damping * dt);
            p.vel = vel;
            p.C = aff;
            p.pos += vel * dt;
            p.F = (M3::identity() + aff * dt) * p.F;
            project_deformation(p.mat, p.F, p.pl);
            p.force = V3();
            if (params.has_bounds) apply_particle_boundary(params, p);
            // apply_particle_obstacles_with_reactions (world.rs:605-630)
            for (size_t oi = 0; oi < obstacles.size(); ++oi) {
                const Obstacle &o = obstacles[oi];
                if (!may_contact(o, p.pos, p.radius)) continue;
                double d;
                V3 n;
                obstacle_surface(o, p.pos, d, n);
                if (d < p.radius) {
                    p.pos += n * (p.radius - d);
                    V3 before = p.vel;
                    p.vel = contact_velocity(o, p.pos, p.vel, n);
                    if (reactions) reactions[oi].record(o.center, p.pos - n * p.radius, (before - p.vel) * p.mass);
                }
            }
            if (!finite_particle(p)) return TMPM_ERR_NON_FINITE_STATE;
        }
        substeps += 1;
        return TMPM_OK;
    }

    // MpmWorld::advance (world.rs:332-359)
    int32_t advance(double dt, Reaction *reactions) {
        if (!std::isfinite(dt) || dt <= 0.0) return TMPM_ERR_MPM_INVALID_INPUT;
        for (const Obstacle &o : obstacles)
            if (!obstacle_valid(o)) return TMPM_ERR_MPM_INVALID_INPUT;
        double remaining = dt;
        size_t count = 0;
        while (remaining > 0.0) {
            double stable = stable_timestep();
            if (!std::isfinite(stable) || stable <= 1e-12) return TMPM_ERR_EXCESSIVE_SUBSTEPS;
            double sub = std::min(remaining, stable);
            int32_t st = substep(sub, reactions);
            if (st != TMPM_OK) return st;
            remaining = std::max(remaining - sub, 0.0);
            count += 1;
            if (count > 100000) return TMPM_ERR_EXCESSIVE_SUBSTEPS;
        }
        return TMPM_OK;
    }
};

namespace {
Material material_from(int32_t kind, const double *params) {
    Material m;
    m.kind = kind;
    for (int k = 0; k < 5; ++k) m.p[k] = params[k];
    return m;
}
}  // namespace

extern "C" {

OrcWorld *orc_world_create(const TmpmParams *params, const TmpmParticleArrays *particles, int32_t *status) {
    Params p = params_from(*params);
    if (!params_valid(p)) {
        if (status) *status = TMPM_ERR_MPM_INVALID_INPUT;
        return nullptr;
    }
    std::vector<Particle> ps;
    if (particles && particles->count) ps = particles_from(*particles);
    for (Particle &q : ps) {
        if (!valid_particle(q)) {
            if (status) *status = TMPM_ERR_MPM_INVALID_INPUT;
            return nullptr;
        }
        q.chunk = 0;
    }
    OrcWorld *w = new OrcWorld();
    w->params = p;
    w->particles = std::move(ps);
    if (status) *status = TMPM_OK;
    return w;
}

void orc_world_destroy(OrcWorld *world) { delete world; }

OrcWorld *orc_world_clone(const OrcWorld *world) { return new OrcWorld(*world); }

int32_t orc_world_add_particles(OrcWorld *w, const TmpmParticleArrays *particles, uint64_t *chunk) {
    if (!particles || particles->count == 0) return TMPM_ERR_MPM_INVALID_INPUT;
    std::vector<Particle> ps = particles_from(*particles);
    for (const Particle &q : ps)
        if (!valid_particle(q)) return TMPM_ERR_MPM_INVALID_INPUT;
    if (w->next_chunk == std::numeric_limits<uint64_t>::max()) return TMPM_ERR_PARTICLE_CAPACITY;
    uint64_t c = w->next_chunk;
    for (Particle &q : ps) q.chunk = c;
    w->particles.insert(w->particles.end(), ps.begin(), ps.end());
    w->next_chunk += 1;
    if (chunk) *chunk = c;
    return TMPM_OK;
}

int32_t orc_world_remove_chunk(OrcWorld *w, uint64_t chunk, size_t *removed) {
    size_t before = w->particles.size();
    w->particles.erase(std::remove_if(w->particles.begin(), w->particles.end(),
                                      [&](const Particle &p) { return p.chunk == chunk; }),
                       w->particles.end());
    size_t r = before - w->particles.size();
    if (removed) *removed = r;
    return r == 0 ? TMPM_ERR_UNKNOWN_CHUNK : TMPM_OK;
}

int32_t orc_world_set_obstacles(OrcWorld *w, const TmpmObstacle *obstacles, size_t count) {
    std::vector<Obstacle> os;
    for (size_t i = 0; i < count; ++i) {
        os.push_back(obstacle_from(obstacles[i]));
        if (!obstacle_valid(os.back())) return TMPM_ERR_MPM_INVALID_INPUT;
    }
    w->obstacles = std::move(os);
    return TMPM_OK;
}

void orc_world_set_use_cpic(OrcWorld *w, int32_t enabled) { w->use_cpic = enabled != 0; }

int32_t orc_world_set_params(OrcWorld *w, const TmpmParams *params) {
    Params p = params_from(*params);
    if (!params_valid(p)) return TMPM_ERR_MPM_INVALID_INPUT;
    w->params = p;
    return TMPM_OK;
}

double orc_world_stable_timestep(const OrcWorld *w) { return w->stable_timestep(); }

int32_t orc_world_step(OrcWorld *w, double dt) { return w->advance(dt, nullptr); }

int32_t orc_world_step_reactions(OrcWorld *w, double dt, double *out) {
    std::vector<Reaction> r(w->obstacles.size());
    int32_t st = w->advance(dt, r.data());
    for (size_t i = 0; i < r.size(); ++i) {
        for (int k = 0; k < 3; ++k) {
            out[6 * i + k] = r[i].lin[k];
            out[6 * i + 3 + k] = r[i].ang[k];
        }
    }
    if (st != TMPM_OK) return st;
    for (const Reaction &x : r)
        if (!finite3(x.lin) || !finite3(x.ang)) return TMPM_ERR_NON_FINITE_STATE;
    return TMPM_OK;
}

int32_t orc_world_substep_fixed(OrcWorld *w, double dt, double *out) {
    if (!std::isfinite(dt) || dt <= 0.0) return TMPM_ERR_MPM_INVALID_INPUT;
    std::vector<Reaction> r(w->obstacles.size());
    int32_t st = w->substep(dt, out ? r.data() : nullptr);
    if (out)
        for (size_t i = 0; i < r.size(); ++i)
            for (int k = 0; k < 3; ++k) {
                out[6 * i + k] = r[i].lin[k];
                out[6 * i + 3 + k] = r[i].ang[k];
            }
    return st;
}

size_t orc_world_count(const OrcWorld *w) { return w->particles.size(); }
uint64_t orc_world_substeps(const OrcWorld *w) { return w->substeps; }

int32_t orc_world_read(const OrcWorld *w, TmpmParticleArrays *out) {
    if (out->count != w->particles.size()) return TMPM_ERR_INVALID_INPUT;
    particles_to(w->particles, *out);
    return TMPM_OK;
}

int32_t orc_world_write(OrcWorld *w, const TmpmParticleArrays *in) {
    if (in->count != w->particles.size()) return TMPM_ERR_INVALID_INPUT;
    std::vector<Particle> ps = particles_from(*in);
    for (size_t i = 0; i < ps.size(); ++i) {
        if (!in->chunk_id) ps[i].chunk = w->particles[i].chunk;
    }
    w->particles = std::move(ps);
    return TMPM_OK;
}

int32_t orc_world_set_force(OrcWorld *w, size_t index, const double f[3]) {
    if (index >= w->particles.size()) return TMPM_ERR_INVALID_INPUT;
    w->particles[index].force = V3(f[0], f[1], f[2]);
    return TMPM_OK;
}

size_t orc_world_p2g(const OrcWorld *w, double dt, int64_t *keys_out, double *values_out, size_t capacity) {
    std::map<GridKey, GridNode> grid;
    std::vector<uint64_t> keys;
    w->p2g(dt, grid, keys);
    size_t i = 0;
    for (auto &kv : grid) {
        if (i < capacity) {
            keys_out[4 * i] = std::get<0>(kv.first);
            keys_out[4 * i + 1] = std::get<1>(kv.first);
            keys_out[4 * i + 2] = std::get<2>(kv.first);
            keys_out[4 * i + 3] = static_cast<int64_t>(std::get<3>(kv.first));
            values_out[4 * i] = kv.second.mass;
            values_out[4 * i + 1] = kv.second.momentum.x;
            values_out[4 * i + 2] = kv.second.momentum.y;
            values_out[4 * i + 3] = kv.second.momentum.z;
        }
        ++i;
    }
    return grid.size();
}

void orc_kirchhoff_stress(int32_t material, const double params[5], const double F_cm[9], const double C_cm[9],
                          const double plastic[3], double out_cm[9]) {
    Plastic pl;
    pl.det = plastic[0];
    pl.hardening = plastic[1];
    pl.lvg = plastic[2];
    M3 s = kirchhoff_stress(material_from(material, params), from_cm(F_cm), from_cm(C_cm), pl);
    to_cm(s, out_cm);
}

void orc_project_deformation(int32_t material, const double params[5], const double F_cm[9],
                             const double plastic_in[3], double F_out_cm[9], double plastic_out[3]) {
    Plastic pl;
    pl.det = plastic_in[0];
    pl.hardening = plastic_in[1];
    pl.lvg = plastic_in[2];
    M3 F = from_cm(F_cm);
    project_deformation(material_from(material, params), F, pl);
    to_cm(F, F_out_cm);
    plastic_out[0] = pl.det;
    plastic_out[1] = pl.hardening;
    plastic_out[2] = pl.lvg;
}

double orc_timestep_bound(int32_t material, const double params[5], double density, const double v[3],
                          double cell_width, double det_f) {
    return timestep_bound(material_from(material, params), density, V3(v[0], v[1], v[2]), cell_width, det_f);
}

int32_t orc_material_valid(int32_t material, const double params[5]) {
    return material_valid(material_from(material, params)) ? 1 : 0;
}

int32_t orc_obstacle_valid(const TmpmObstacle *o) { return obstacle_valid(obstacle_from(*o)) ? 1 : 0; }

void orc_obstacle_surface(const TmpmObstacle *o, const double point[3], double *distance, double normal[3]) {
    V3 n;
    obstacle_surface(obstacle_from(*o), V3(point[0], point[1], point[2]), *distance, n);
    for (int k = 0; k < 3; ++k) normal[k] = n[k];
}

void orc_obstacle_contact_velocity(const TmpmObstacle *o, const double point[3], const double velocity[3],
                                   const double normal[3], double out[3]) {
    V3 r = contact_velocity(obstacle_from(*o), V3(point[0], point[1], point[2]),
                            V3(velocity[0], velocity[1], velocity[2]), V3(normal[0], normal[1], normal[2]));
    for (int k = 0; k < 3; ++k) out[k] = r[k];
}

int32_t orc_obstacle_may_contact(const TmpmObstacle *o, const double point[3], double margin) {
    return may_contact(obstacle_from(*o), V3(point[0], point[1], point[2]), margin) ? 1 : 0;
}

double orc_bench_threads(const OrcWorld *world, int32_t threads, int32_t substeps, double dt) {
    if (threads < 1) threads = 1;
    std::vector<OrcWorld> copies(static_cast<size_t>(threads), *world);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t]() {
            for (int s = 0; s < substeps; ++s) copies[static_cast<size_t>(t)].substep(dt, nullptr);
        });
    for (auto &th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
