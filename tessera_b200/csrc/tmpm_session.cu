// tmpm_session.cu -- host side of the C ABI (include/tmpm.h).
//
// A TmpmSession is the B200 counterpart of the reference's
// GpuMpmResidentSession (crates/tessera-mpm/src/gpu.rs:206-662): it keeps the
// last synchronized world in f64 on the host, the packed f32 state and two
// sparse grids on the device, and one CUDA stream on which every substep is
// queued.  The world changes only after a synchronize has validated the device
// result; any device error invalidates the session (gpu.rs:382-411).

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tmpm.h"
#include "tmpm_internal.h"

using namespace tmpm;

namespace {

thread_local std::string g_last_error;

constexpr double kSyncTimeoutSeconds = 5.0;  // gpu.rs:1853-1862

unsigned host_threads() { return std::max(1u, std::min(32u, std::thread::hardware_concurrency())); }

// Run fn(chunk, begin, end) over [0, n) split into contiguous chunks, one per host thread.
template <typename Fn>
void parallel_chunks(size_t n, Fn fn, size_t min_per_chunk = 32768) {
    size_t chunks = std::min<size_t>(host_threads(), std::max<size_t>(1, n / min_per_chunk));
    if (chunks <= 1) {
        fn(size_t(0), size_t(0), n);
        return;
    }
    size_t per = (n + chunks - 1) / chunks;
    std::vector<std::thread> pool;
    for (size_t c = 0; c < chunks; ++c) {
        size_t a = c * per, b = std::min(n, a + per);
        if (a >= b) break;
        pool.emplace_back([=]() { fn(c, a, b); });
    }
    for (auto &t : pool) t.join();
}

template <typename Fn>
void parallel_for(size_t n, Fn fn) {
    parallel_chunks(n, [&](size_t, size_t a, size_t b) { fn(a, b); });
}

// --------------------------------------------------------------- host world

struct HostWorld {
    size_t n = 0;
    std::vector<double> pos, vel, F, C, force, mass, vol, radius, damping, plastic, mparams;
    std::vector<int32_t> material;
    std::vector<uint8_t> enabled, fixed;
    std::vector<uint16_t> color;
    std::vector<uint32_t> group;
    std::vector<uint64_t> chunk;

    // Sizes every field for `count` particles; existing storage is reused and
    // not cleared (load() writes every element).
    void resize(size_t count) {
        n = count;
        pos.resize(3 * n);
        vel.resize(3 * n);
        F.resize(9 * n);
        C.resize(9 * n);
        force.resize(3 * n);
        mass.resize(n);
        vol.resize(n);
        radius.resize(n);
        damping.resize(n);
        plastic.resize(3 * n);
        mparams.resize(5 * n);
        material.resize(n);
        enabled.resize(n);
        fixed.resize(n);
        color.resize(n);
        group.resize(n);
        chunk.resize(n);
    }

    void load(const TmpmParticleArrays &a) {
        resize(a.count);
        parallel_for(n, [&](size_t lo, size_t hi) { load_range(a, lo, hi); });
    }

    void load_range(const TmpmParticleArrays &a, size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
            for (int k = 0; k < 3; ++k) {
                pos[3 * i + k] = a.position[3 * i + k];
                vel[3 * i + k] = a.velocity[3 * i + k];
                force[3 * i + k] = a.force ? a.force[3 * i + k] : 0.0;
            }
            for (int k = 0; k < 9; ++k) {
                F[9 * i + k] = a.deformation ? a.deformation[9 * i + k] : ((k % 4 == 0) ? 1.0 : 0.0);
                C[9 * i + k] = a.affine ? a.affine[9 * i + k] : 0.0;
            }
            mass[i] = a.mass[i];
            vol[i] = a.rest_volume[i];
            radius[i] = a.radius[i];
            damping[i] = a.damping ? a.damping[i] : 0.0;
            material[i] = a.material[i];
            for (int k = 0; k < 5; ++k) mparams[5 * i + k] = a.material_params[5 * i + k];
            if (a.plastic) {
                for (int k = 0; k < 3; ++k) plastic[3 * i + k] = a.plastic[3 * i + k];
            } else {
                plastic[3 * i] = 1.0;
                plastic[3 * i + 1] = (material[i] == TMPM_MAT_SAND || material[i] == TMPM_MAT_SAND_NEO_HOOKEAN) ? 1.0 : 0.0;
                plastic[3 * i + 2] = 0.0;
            }
            enabled[i] = a.enabled ? (a.enabled[i] != 0) : 1;
            fixed[i] = a.fixed ? (a.fixed[i] != 0) : 0;
            color[i] = a.transfer_color ? a.transfer_color[i] : 0;
            group[i] = a.group_id ? a.group_id[i] : 0;
            chunk[i] = a.chunk_id ? a.chunk_id[i] : 0;
        }
    }

    void store(TmpmParticleArrays &a) const {
        parallel_for(n, [&](size_t lo, size_t hi) { store_range(a, lo, hi); });
    }

    void store_range(TmpmParticleArrays &a, size_t lo, size_t hi) const {
        for (size_t i = lo; i < hi; ++i) {
            for (int k = 0; k < 3; ++k) {
                if (a.position) a.position[3 * i + k] = pos[3 * i + k];
                if (a.velocity) a.velocity[3 * i + k] = vel[3 * i + k];
                if (a.force) a.force[3 * i + k] = force[3 * i + k];
                if (a.plastic) a.plastic[3 * i + k] = plastic[3 * i + k];
            }
            for (int k = 0; k < 9; ++k) {
                if (a.deformation) a.deformation[9 * i + k] = F[9 * i + k];
                if (a.affine) a.affine[9 * i + k] = C[9 * i + k];
            }
            if (a.mass) a.mass[i] = mass[i];
            if (a.rest_volume) a.rest_volume[i] = vol[i];
            if (a.radius) a.radius[i] = radius[i];
            if (a.damping) a.damping[i] = damping[i];
            if (a.material) a.material[i] = material[i];
            if (a.material_params)
                for (int k = 0; k < 5; ++k) a.material_params[5 * i + k] = mparams[5 * i + k];
            if (a.enabled) a.enabled[i] = enabled[i];
            if (a.fixed) a.fixed[i] = fixed[i];
            if (a.transfer_color) a.transfer_color[i] = color[i];
            if (a.group_id) a.group_id[i] = group[i];
            if (a.chunk_id) a.chunk_id[i] = chunk[i];
        }
    }

    void append(const HostWorld &o) {
        auto cat = [](auto &dst, const auto &src) { dst.insert(dst.end(), src.begin(), src.end()); };
        cat(pos, o.pos);
        cat(vel, o.vel);
        cat(F, o.F);
        cat(C, o.C);
        cat(force, o.force);
        cat(mass, o.mass);
        cat(vol, o.vol);
        cat(radius, o.radius);
        cat(damping, o.damping);
        cat(plastic, o.plastic);
        cat(mparams, o.mparams);
        cat(material, o.material);
        cat(enabled, o.enabled);
        cat(fixed, o.fixed);
        cat(color, o.color);
        cat(group, o.group);
        cat(chunk, o.chunk);
        n += o.n;
    }

    // Keep particles whose chunk differs (world.rs:267-277).
    size_t remove_chunk(uint64_t c) {
        size_t w = 0;
        for (size_t i = 0; i < n; ++i) {
            if (chunk[i] == c) continue;
            if (w != i) {
                for (int k = 0; k < 3; ++k) {
                    pos[3 * w + k] = pos[3 * i + k];
                    vel[3 * w + k] = vel[3 * i + k];
                    force[3 * w + k] = force[3 * i + k];
                    plastic[3 * w + k] = plastic[3 * i + k];
                }
                for (int k = 0; k < 9; ++k) {
                    F[9 * w + k] = F[9 * i + k];
                    C[9 * w + k] = C[9 * i + k];
                }
                for (int k = 0; k < 5; ++k) mparams[5 * w + k] = mparams[5 * i + k];
                mass[w] = mass[i];
                vol[w] = vol[i];
                radius[w] = radius[i];
                damping[w] = damping[i];
                material[w] = material[i];
                enabled[w] = enabled[i];
                fixed[w] = fixed[i];
                color[w] = color[i];
                group[w] = group[i];
                chunk[w] = chunk[i];
            }
            ++w;
        }
        size_t removed = n - w;
        n = w;
        pos.resize(3 * n);
        vel.resize(3 * n);
        force.resize(3 * n);
        plastic.resize(3 * n);
        F.resize(9 * n);
        C.resize(9 * n);
        mparams.resize(5 * n);
        mass.resize(n);
        vol.resize(n);
        radius.resize(n);
        damping.resize(n);
        material.resize(n);
        enabled.resize(n);
        fixed.resize(n);
        color.resize(n);
        group.resize(n);
        chunk.resize(n);
        return removed;
    }
};

// ------------------------------------------------------------- host math

double det9(const double *m) {  // column-major
    return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) + m[6] * (m[1] * m[5] - m[4] * m[2]);
}
double fro9(const double *m) {
    double s = 0;
    for (int k = 0; k < 9; ++k) s += m[k] * m[k];
    return std::sqrt(s);
}
bool inverse_norm9(const double *m, double &out) {
    double d = det9(m);
    if (d == 0.0 || !std::isfinite(d)) return false;
    // cofactors: the inverse's Frobenius norm equals that of the cofactor matrix / |det|
    const double *a = m, *b = m + 3, *c = m + 6;
    double bc[3] = {b[1] * c[2] - b[2] * c[1], b[2] * c[0] - b[0] * c[2], b[0] * c[1] - b[1] * c[0]};
    double ca[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
    double ab[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    double s = 0;
    for (int k = 0; k < 3; ++k) s += bc[k] * bc[k] + ca[k] * ca[k] + ab[k] * ab[k];
    out = std::sqrt(s) / std::fabs(d);
    return std::isfinite(out);
}

void lame(double young, double poisson, double &lambda, double &mu) {  // material.rs:433-438
    lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    mu = young / (2.0 * (1.0 + poisson));
}

bool valid_elasticity(double young, double poisson) {  // material.rs:429-431
    return std::isfinite(young) && young > 0.0 && std::isfinite(poisson) && poisson >= -1.0 && poisson < 0.5;
}

bool material_valid(int kind, const double *p) {  // material.rs:171-231
    switch (kind) {
    case TMPM_MAT_ELASTIC:
    case TMPM_MAT_NEO_HOOKEAN:
        return valid_elasticity(p[0], p[1]);
    case TMPM_MAT_SAND:
    case TMPM_MAT_SAND_NEO_HOOKEAN:
        return valid_elasticity(p[0], p[1]) && std::isfinite(p[2]) && p[2] >= 0.0 && p[2] < M_PI / 2.0 &&
               std::isfinite(p[3]) && p[3] >= 0.0;
    case TMPM_MAT_FLUID:
        return std::isfinite(p[0]) && p[0] > 0.0 && std::isfinite(p[1]) && p[1] > 0.0 && std::isfinite(p[2]) &&
               p[2] >= 0.0 && std::isfinite(p[3]) && p[3] >= 0.0;
    case TMPM_MAT_SNOW:
        return valid_elasticity(p[0], p[1]) && std::isfinite(p[2]) && p[2] >= 0.0 && p[2] < 1.0 &&
               std::isfinite(p[3]) && p[3] >= 0.0 && std::isfinite(p[4]) && p[4] >= 0.0;
    default:
        return false;
    }
}

// MaterialModel::timestep_bound_with_deformation (material.rs:378-426)
double timestep_bound(int kind, const double *p, double density, const double *v, double h, double det_f) {
    double speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double lambda, mu, wave;
    if (kind == TMPM_MAT_SAND_NEO_HOOKEAN) {
        lame(p[0], p[1], lambda, mu);
        double rho = density / std::max(det_f, 1e-6);
        double ws = std::sqrt((lambda + 2.0 * mu) / rho);
        return 0.5 * h / std::max(ws, speed);
    }
    if (kind == TMPM_MAT_FLUID) {
        wave = std::sqrt(p[0] * p[1] / std::max(density, 1e-12));
    } else {
        lame(p[0], p[1], lambda, mu);
        wave = std::sqrt((lambda + 2.0 * mu) / std::max(density, 1e-12));
    }
    return 0.4 * h / std::max(wave + speed, 1e-12);
}

bool finite_particle(const HostWorld &w, size_t i) {  // world.rs:505-515
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(w.pos[3 * i + k]) || !std::isfinite(w.vel[3 * i + k]) || !std::isfinite(w.force[3 * i + k]))
            return false;
    for (int k = 0; k < 9; ++k)
        if (!std::isfinite(w.F[9 * i + k]) || !std::isfinite(w.C[9 * i + k])) return false;
    return std::isfinite(w.mass[i]) && std::isfinite(w.vol[i]) && std::isfinite(w.radius[i]) &&
           std::isfinite(w.damping[i]);
}

bool valid_particle(const HostWorld &w, size_t i) {  // world.rs:492-503
    const double *pl = &w.plastic[3 * i];
    return finite_particle(w, i) && w.mass[i] > 0.0 && w.vol[i] > 0.0 && w.radius[i] > 0.0 &&
           material_valid(w.material[i], &w.mparams[5 * i]) && w.damping[i] >= 0.0 && std::isfinite(pl[0]) &&
           pl[0] > 0.0 && std::isfinite(pl[1]) && std::isfinite(pl[2]);
}

bool params_valid(const TmpmParams &p) {  // world.rs:51-65
    if (!std::isfinite(p.cell_width) || p.cell_width <= 0.0 || !std::isfinite(p.max_substep) || p.max_substep <= 0.0)
        return false;
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(p.gravity[k])) return false;
    if (p.has_bounds) {
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(p.bounds_min[k]) || !std::isfinite(p.bounds_max[k]) || !(p.bounds_max[k] - p.bounds_min[k] > 0.0))
                return false;
    }
    return p.wall_mode == 0 || p.wall_mode == 1;
}

double stable_timestep(const HostWorld &w, const TmpmParams &p) {  // world.rs:288-303
    std::vector<double> part(host_threads() + 1, p.max_substep);
    parallel_chunks(w.n, [&](size_t c, size_t lo, size_t hi) {
        double dt = p.max_substep;
        for (size_t i = lo; i < hi; ++i) {
            if (!w.enabled[i] || w.fixed[i]) continue;
            dt = std::min(dt, timestep_bound(w.material[i], &w.mparams[5 * i], w.mass[i] / w.vol[i], &w.vel[3 * i],
                                             p.cell_width, det9(&w.F[9 * i])));
        }
        part[c] = dt;
    });
    double dt = p.max_substep;
    for (double d : part) dt = std::min(dt, d);
    return std::min(dt, p.max_substep);
}

// RigidObstacle::is_valid (obstacle.rs:264-341)
bool obstacle_valid(const TmpmObstacle &o) {
    auto fin = [](double v) { return std::isfinite(v); };
    const double *d = o.dims;
    bool shape_ok = false;
    switch (o.shape) {
    case TMPM_SHAPE_SPHERE:
        shape_ok = fin(d[0]) && d[0] > 0.0;
        break;
    case TMPM_SHAPE_BOX:
        shape_ok = fin(d[0]) && d[0] > 0 && fin(d[1]) && d[1] > 0 && fin(d[2]) && d[2] > 0;
        break;
    case TMPM_SHAPE_CAPSULE:
        shape_ok = fin(d[0]) && d[0] >= 0.0 && fin(d[1]) && d[1] >= 0.0 && (d[0] > 0.0 || d[1] > 0.0);
        break;
    case TMPM_SHAPE_CYLINDER:
    case TMPM_SHAPE_CONE:
    case TMPM_SHAPE_GROUND:
        shape_ok = fin(d[0]) && d[0] > 0.0 && fin(d[1]) && d[1] > 0.0;
        break;
    case TMPM_SHAPE_TRIANGLE_PRISM: {
        const double *v = o.vertices;
        double e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]}, e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
        double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        double area_sq = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
        bool verts_ok = true;
        for (int k = 0; k < 9; ++k) verts_ok = verts_ok && fin(v[k]);
        shape_ok = fin(d[0]) && d[0] > 0.0 && verts_ok && fin(area_sq) && area_sq > 1e-24;
        break;
    }
    case TMPM_SHAPE_CONVEX: {
        shape_ok = o.plane_count >= 4 && o.planes != nullptr && fin(o.bound_radius) && o.bound_radius > 0.0;
        for (uint32_t i = 0; shape_ok && i < o.plane_count; ++i) {
            const double *pl = o.planes + 4 * i;
            bool f = fin(pl[0]) && fin(pl[1]) && fin(pl[2]) && fin(pl[3]);
            double n2 = std::fma(pl[0], pl[0], std::fma(pl[1], pl[1], pl[2] * pl[2]));
            shape_ok = f && std::fabs(n2 - 1.0) <= 1e-4;
        }
        break;
    }
    default:
        shape_ok = false;
    }
    bool cpic_ok = o.cpic_group < 0 || (o.cpic_group < 32 && o.shape == TMPM_SHAPE_TRIANGLE_PRISM);
    bool rest = o.boundary >= 0 && o.boundary <= 4 && fin(o.friction) && o.friction >= 0.0;
    for (int k = 0; k < 3; ++k)
        rest = rest && fin(o.center[k]) && fin(o.linear_velocity[k]) && fin(o.angular_velocity[k]);
    for (int k = 0; k < 4; ++k) rest = rest && fin(o.orientation[k]);
    return shape_ok && cpic_ok && rest;
}

bool f32_ok(double v, float &out) {  // finite_f32 (gpu.rs:1992-1999)
    out = static_cast<float>(v);
    return std::isfinite(out);
}

// ------------------------------------------------------------ device memory

template <typename T>
struct DevBuf {
    T *ptr = nullptr;
    size_t count = 0;
    cudaError_t alloc(size_t n) {
        release();
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&ptr), n * sizeof(T));
        if (e == cudaSuccess) count = n;
        else ptr = nullptr;
        return e;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

struct PinnedBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    bool ensure(size_t b) {
        if (b <= bytes) return true;
        release();
        if (cudaMallocHost(&ptr, b) != cudaSuccess) {
            ptr = nullptr;
            return false;
        }
        bytes = b;
        return true;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    ~PinnedBuf() { release(); }
};

struct ParticleBuffers {
    DevBuf<float> x, v, C, F, pl;
    DevBuf<uint32_t> cls, widx;
    size_t cap = 0;
    cudaError_t alloc(size_t c) {
        cudaError_t e;
        if ((e = x.alloc(3 * c)) || (e = v.alloc(3 * c)) || (e = C.alloc(9 * c)) || (e = F.alloc(9 * c)) ||
            (e = pl.alloc(3 * c)) || (e = cls.alloc(c)) || (e = widx.alloc(c)))
            return e;
        cap = c;
        return cudaSuccess;
    }
    ParticleSoA view(float *force, size_t force_stride) const {
        ParticleSoA p;
        p.x = x.ptr;
        p.v = v.ptr;
        p.C = C.ptr;
        p.F = F.ptr;
        p.pl = pl.ptr;
        p.force = force;
        p.cls = cls.ptr;
        p.widx = widx.ptr;
        p.cap = cap;
        p.force_stride = force_stride;
        return p;
    }
};

struct GridBuffers {
    DevBuf<unsigned long long> keys;
    DevBuf<uint32_t> vals, count;
    DevBuf<float4> pool;
    DevBuf<int4> coords;
    uint32_t capacity = 0, max_blocks = 0;
    cudaError_t alloc(uint32_t blocks) {
        uint32_t cap = 1024;
        while (cap < 2u * blocks) cap <<= 1;
        cudaError_t e;
        if ((e = keys.alloc(cap)) || (e = vals.alloc(cap)) || (e = count.alloc(1)) ||
            (e = pool.alloc(static_cast<size_t>(blocks) * kNodesPerBlock)) || (e = coords.alloc(blocks)))
            return e;
        capacity = cap;
        max_blocks = blocks;
        return cudaSuccess;
    }
    GridTable view() const {
        GridTable g;
        g.keys = keys.ptr;
        g.vals = vals.ptr;
        g.count = count.ptr;
        g.pool = pool.ptr;
        g.coords = coords.ptr;
        g.mask = capacity - 1;
        g.max_blocks = max_blocks;
        return g;
    }
};

// Device material codes, as the reference packs them (gpu.rs:1171-1276).
int class_kind(int material) {
    switch (material) {
    case TMPM_MAT_NEO_HOOKEAN:
        return kMatNeoHookean;
    case TMPM_MAT_FLUID:
        return kMatFluid;
    case TMPM_MAT_ELASTIC:
        return kMatCorotated;
    case TMPM_MAT_SNOW:
        return kMatSnow;
    case TMPM_MAT_SAND:
        return kMatSand;
    case TMPM_MAT_SAND_NEO_HOOKEAN:
        return kMatSandNeoHookean;
    default:
        return 0;
    }
}

}  // namespace

void tmpm::set_last_error(const std::string &msg) { g_last_error = msg; }

struct TmpmSession {
    // host world (last synchronized state)
    TmpmParams params{};
    HostWorld world;
    HostWorld spare;  // reused storage for tmpm_write_particles
    std::vector<TmpmObstacle> obstacles;
    std::vector<std::vector<double>> obstacle_planes;
    bool use_cpic = true;
    double substep_dt = 0.0;
    uint64_t substeps = 0;
    uint64_t next_chunk = 1;
    uint64_t pending = 0;
    bool valid = true;
    std::string last_error;
    TmpmSessionOptions options{};

    // device state
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    ParticleBuffers pbuf[2];
    int cur = 0;
    int n_dev = 0;  // enabled particles on the device
    DevBuf<float> force;  // 3 x world count, world-indexed
    DevBuf<DevClass> classes;
    GridBuffers grids[2];
    DevBuf<DevObstacle> dev_obstacles;
    DevBuf<float> dev_planes;
    DevBuf<uint32_t> status;
    DevBuf<double> reactions;
    DevBuf<int> cta_cache;  // kCacheStride ints per transfer CTA
    DevBuf<uint32_t> sort_keys[2], sort_vals[2], sort_hist, sort_totals;
    PinnedBuf staging;         // readback
    PinnedBuf upload_staging;  // packed f32 state for uploads
    bool force_dirty = false;
    bool has_plastic = false;  // class table holds a snow, sand or NH sand class
    uint64_t since_resort = 0;

    ~TmpmSession() {
        if (stream) {
            cudaStreamSynchronize(stream);
        }
        if (done) cudaEventDestroy(done);
        if (stream) cudaStreamDestroy(stream);
    }

    TmpmStatus fail(TmpmStatus st, const std::string &msg) {
        last_error = msg;
        g_last_error = msg;
        return st;
    }

    TmpmStatus cuda_fail(cudaError_t e, const char *what) {
        valid = false;
        return fail(TMPM_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
    }

    SimParams sim_params(double dt, bool resident) const {
        SimParams sp{};
        float h = static_cast<float>(params.cell_width);
        sp.h = h;
        sp.inv_h = 1.0f / h;
        sp.inv_d = static_cast<float>(4.0 / (params.cell_width * params.cell_width));
        sp.dt = static_cast<float>(dt);
        sp.gx = static_cast<float>(params.gravity[0]);
        sp.gy = static_cast<float>(params.gravity[1]);
        sp.gz = static_cast<float>(params.gravity[2]);
        sp.has_bounds = params.has_bounds ? 1 : 0;
        sp.wall_mode = params.wall_mode;
        for (int k = 0; k < 3; ++k) {
            sp.bmin[k] = static_cast<float>(params.bounds_min[k]);
            sp.bmax[k] = static_cast<float>(params.bounds_max[k]);
            // gpu.wgsl:962-965: floor(bound * inv_h - 0.5) -/+ 2 in f32
            float lo = std::floor(sp.bmin[k] * sp.inv_h - 0.5f), hi = std::floor(sp.bmax[k] * sp.inv_h - 0.5f);
            sp.first_base[k] = static_cast<int>(std::max(lo, -1.0e9f)) - 2;
            sp.last_base[k] = static_cast<int>(std::min(hi, 1.0e9f)) + 2;
        }
        sp.num_obstacles = static_cast<int>(obstacles.size());
        sp.reactions = 0;
        sp.apply_force = 0;
        sp.resident_checks = resident ? 1 : 0;
        sp.has_plastic = has_plastic ? 1 : 0;
        return sp;
    }

    // validate_resident_world (gpu.rs:664-677)
    TmpmStatus validate_resident(double dt) {
        if (!params_valid(params)) return fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM input");
        if (!std::isfinite(dt) || dt <= 0.0 || !std::isfinite(params.max_substep) || dt > stable_timestep(world, params))
            return fail(TMPM_ERR_INVALID_INPUT, "substep dt is not finite, not positive or above the CFL bound");
        for (const TmpmObstacle &o : obstacles)
            if (!obstacle_valid(o)) return fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM obstacle");
        return TMPM_OK;
    }

    // Pack and upload the world (the device half of GpuMpmTransfers::prepare,
    // gpu.rs:1091-1600).  Device buffers are reused when large enough.
    TmpmStatus upload(double dt) {
        float h32, dt32, inv_d32;
        if (!f32_ok(params.cell_width, h32) || !f32_ok(dt, dt32) ||
            !f32_ok(4.0 / (params.cell_width * params.cell_width), inv_d32) || h32 <= 0.0f || dt32 <= 0.0f)
            return fail(TMPM_ERR_INVALID_INPUT, "cell width or substep not representable in f32");
        float inv_h = 1.0f / h32;
        if (!std::isfinite(inv_h)) return fail(TMPM_ERR_INVALID_INPUT, "1 / cell width not representable in f32");

        // Packing runs in two parallel passes over contiguous particle chunks:
        // pass 1 validates, builds per-chunk class tables and block lists and
        // counts enabled particles; pass 2 writes the f32 arrays (component-
        // major with stride `cap`) straight into pinned memory at compacted
        // positions.  Results equal a serial pass in world order.
        const size_t N = world.n;
        struct ChunkOut {
            size_t first_bad = std::numeric_limits<size_t>::max();
            TmpmStatus st = TMPM_OK;
            const char *msg = "";
            size_t enabled = 0;
            std::vector<DevClass> classes;
            std::vector<unsigned long long> blocks;
        };
        const unsigned T = host_threads();
        std::vector<ChunkOut> co(T + 1);
        std::vector<uint32_t> lcls(std::max<size_t>(N, 1));
        parallel_chunks(N, [&](size_t c, size_t lo, size_t hi) {
            ChunkOut &o = co[c];
            std::unordered_map<std::string, uint32_t> index;
            DevClass last{};
            uint32_t last_ci = kClassMask;
            unsigned long long last_block = ~0ull;
            auto bad = [&](size_t i, TmpmStatus st, const char *msg) {
                o.first_bad = i;
                o.st = st;
                o.msg = msg;
            };
            for (size_t i = lo; i < hi; ++i) {
                float f4[4];
                for (int k = 0; k < 3; ++k)
                    if (!f32_ok(world.pos[3 * i + k], f4[k]) || !f32_ok(world.vel[3 * i + k], f4[3]) ||
                        !f32_ok(world.force[3 * i + k], f4[3]))
                        return bad(i, TMPM_ERR_INVALID_INPUT, "particle state not representable in f32");
                float m32, v32, r32, d32;
                if (!f32_ok(world.enabled[i] ? world.mass[i] : 0.0, m32) || !f32_ok(world.vol[i], v32) ||
                    !f32_ok(world.radius[i], r32) || !f32_ok(world.damping[i], d32))
                    return bad(i, TMPM_ERR_INVALID_INPUT, "particle scalars not representable in f32");
                if (world.enabled[i] && (m32 <= 0.0f || v32 <= 0.0f))
                    return bad(i, TMPM_ERR_INVALID_INPUT, "particle mass or volume underflows f32");
                if (r32 <= 0.0f || world.damping[i] < 0.0)
                    return bad(i, TMPM_ERR_INVALID_INPUT, "particle radius or damping invalid");
                for (int k = 0; k < 9; ++k) {
                    float t;
                    if (!f32_ok(world.F[9 * i + k], t) || !f32_ok(world.C[9 * i + k], t))
                        return bad(i, TMPM_ERR_INVALID_INPUT, "particle matrices not representable in f32");
                }
                if (!world.enabled[i]) continue;
                int base[3];
                for (int k = 0; k < 3; ++k) {
                    float xk = static_cast<float>(world.pos[3 * i + k]);
                    float cf = std::floor(xk * inv_h - 0.5f);
                    if (!std::isfinite(cf) || cf < -131000.0f || cf > 131000.0f)
                        return bad(i, TMPM_ERR_INVALID_INPUT, "particle cell outside the representable grid");
                    base[k] = static_cast<int>(cf);
                }
                int kind = class_kind(world.material[i]);
                const double *mp = &world.mparams[5 * i];
                if (kind == kMatCorotated || kind == kMatSand || kind == kMatSnow) {
                    // use_cpu_corotated (gpu.rs:1156-1170): ill-conditioned F is a CPU case
                    const double *Fm = &world.F[9 * i];
                    double nrm = fro9(Fm), inrm = std::numeric_limits<double>::infinity();
                    inverse_norm9(Fm, inrm);
                    if (std::fabs(det9(Fm)) < 1e-5 || !(nrm >= 1e-5 && nrm <= 20.0) || nrm * inrm > 100.0) kind = 0;
                }
                if (kind == 0)
                    return bad(i, TMPM_ERR_RESIDENT_UNAVAILABLE,
                               "particle material or deformation needs the CPU path (plastic material or "
                               "ill-conditioned F)");
                DevClass k{};
                k.mass = m32;
                k.volume = v32;
                k.radius = r32;
                k.damping = d32;
                k.kind = kind;
                k.color = world.color[i];
                float rho = std::max(m32 / v32, 1e-12f);
                if (kind == kMatFluid) {
                    float b, g, vi, te;
                    if (!f32_ok(mp[0], b) || !f32_ok(mp[1], g) || !f32_ok(mp[2], vi) || !f32_ok(mp[3], te))
                        return bad(i, TMPM_ERR_INVALID_INPUT, "fluid parameters not representable in f32");
                    k.p0 = b;
                    k.p1 = g;
                    k.p2 = vi;
                    k.p3 = te;
                    k.wave = std::sqrt(b * g / rho);
                } else {
                    double lambda, mu;
                    lame(mp[0], mp[1], lambda, mu);
                    float l32, m32b;
                    if (!f32_ok(lambda, l32) || !f32_ok(mu, m32b))
                        return bad(i, TMPM_ERR_INVALID_INPUT, "Lame parameters not representable in f32");
                    k.p0 = l32;
                    k.p1 = m32b;
                    k.wave = std::sqrt((l32 + 2.0f * m32b) / rho);
                    // sand / NH sand: friction angle, cohesion; snow: hardening, critical compression, stretch
                    bool ok = true;
                    if (kind == kMatSand || kind == kMatSandNeoHookean) {
                        ok = f32_ok(mp[2], k.p2) && f32_ok(mp[3], k.p3);
                    } else if (kind == kMatSnow) {
                        ok = f32_ok(mp[4], k.p2) && f32_ok(mp[2], k.p3) && f32_ok(mp[3], k.p4);
                    }
                    float t3;
                    if (kind >= kMatSnow)
                        for (int q = 0; q < 3; ++q) ok = ok && f32_ok(world.plastic[3 * i + q], t3);
                    if (!ok) return bad(i, TMPM_ERR_INVALID_INPUT, "plastic parameters not representable in f32");
                }
                uint32_t ci;
                if (last_ci != kClassMask && std::memcmp(&k, &last, sizeof(DevClass)) == 0) {
                    ci = last_ci;
                } else {
                    std::string key(reinterpret_cast<const char *>(&k), sizeof(DevClass));
                    auto it = index.find(key);
                    if (it == index.end()) {
                        ci = static_cast<uint32_t>(o.classes.size());
                        o.classes.push_back(k);
                        index.emplace(std::move(key), ci);
                    } else {
                        ci = it->second;
                    }
                    last = k;
                    last_ci = ci;
                }
                lcls[i] = ci;
                unsigned long long hb =
                    (static_cast<unsigned long long>(world.color[i]) << 48) |
                    (static_cast<unsigned long long>(static_cast<uint32_t>((base[0] >> 2) + kBlockBias) & 0xFFFF) << 32) |
                    (static_cast<unsigned long long>(static_cast<uint32_t>((base[1] >> 2) + kBlockBias) & 0xFFFF) << 16) |
                    static_cast<unsigned long long>(static_cast<uint32_t>((base[2] >> 2) + kBlockBias) & 0xFFFF);
                if (hb != last_block) {
                    o.blocks.push_back(hb);
                    last_block = hb;
                }
                ++o.enabled;
            }
            std::sort(o.blocks.begin(), o.blocks.end());
            o.blocks.erase(std::unique(o.blocks.begin(), o.blocks.end()), o.blocks.end());
        });
        size_t worst = std::numeric_limits<size_t>::max();
        const ChunkOut *failed = nullptr;
        for (const ChunkOut &o : co)
            if (o.first_bad < worst) {
                worst = o.first_bad;
                failed = &o;
            }
        if (failed) return fail(failed->st, failed->msg);
        // merge class tables and block lists (small), compute compacted offsets
        std::vector<DevClass> cls_table;
        std::unordered_map<std::string, uint32_t> cls_index;
        std::vector<std::vector<uint32_t>> remap(co.size());
        std::vector<size_t> offset(co.size(), 0);
        std::vector<unsigned long long> home_blocks;
        size_t n_enabled = 0;
        for (size_t c = 0; c < co.size(); ++c) {
            offset[c] = n_enabled;
            n_enabled += co[c].enabled;
            for (const DevClass &k : co[c].classes) {
                std::string key(reinterpret_cast<const char *>(&k), sizeof(DevClass));
                auto it = cls_index.find(key);
                uint32_t gi;
                if (it == cls_index.end()) {
                    gi = static_cast<uint32_t>(cls_table.size());
                    cls_table.push_back(k);
                    cls_index.emplace(std::move(key), gi);
                } else {
                    gi = it->second;
                }
                remap[c].push_back(gi);
            }
            home_blocks.insert(home_blocks.end(), co[c].blocks.begin(), co[c].blocks.end());
        }
        if (n_enabled > static_cast<size_t>(std::numeric_limits<int>::max() / 2))
            return fail(TMPM_ERR_CAPACITY, "too many particles for one session");
        bool plastic_classes = false;
        for (const DevClass &k : cls_table) plastic_classes = plastic_classes || k.kind >= kMatSnow;
        const size_t cap = std::max<size_t>(256, (n_enabled + 255) / 256 * 256);
        if (!upload_staging.ensure((27 * cap + 2 * cap) * sizeof(float)))
            return fail(TMPM_ERR_DEVICE, "cudaMallocHost upload staging failed");
        float *hx = static_cast<float *>(upload_staging.ptr);
        float *hv = hx + 3 * cap, *hC = hv + 3 * cap, *hF = hC + 9 * cap, *hpl = hF + 9 * cap;
        uint32_t *hcls = reinterpret_cast<uint32_t *>(hpl + 3 * cap), *hwidx = hcls + cap;
        parallel_chunks(N, [&](size_t c, size_t lo, size_t hi) {
            size_t j = offset[c];
            const std::vector<uint32_t> &rm = remap[c];
            for (size_t i = lo; i < hi; ++i) {
                if (!world.enabled[i]) continue;
                for (int k3 = 0; k3 < 3; ++k3) {
                    hx[k3 * cap + j] = static_cast<float>(world.pos[3 * i + k3]);
                    hv[k3 * cap + j] = static_cast<float>(world.vel[3 * i + k3]);
                }
                for (int k9 = 0; k9 < 9; ++k9) {
                    hC[k9 * cap + j] = static_cast<float>(world.C[9 * i + k9]);
                    hF[k9 * cap + j] = static_cast<float>(world.F[9 * i + k9]);
                }
                for (int k3 = 0; k3 < 3; ++k3) hpl[k3 * cap + j] = static_cast<float>(world.plastic[3 * i + k3]);
                hcls[j] = rm[lcls[i]] | (world.fixed[i] ? kFixedBit : 0u);
                hwidx[j] = static_cast<uint32_t>(i);
                ++j;
            }
        });
        // obstacles (pack_obstacle, gpu.rs:2025-2166)
        std::vector<DevObstacle> dobs;
        std::vector<float> dplanes;
        for (size_t oi = 0; oi < obstacles.size(); ++oi) {
            const TmpmObstacle &o = obstacles[oi];
            if (!obstacle_valid(o)) return fail(TMPM_ERR_INVALID_INPUT, "invalid obstacle");
            DevObstacle d{};
            d.shape = o.shape;
            d.boundary = o.boundary;
            d.cpic_group = o.cpic_group;
            bool ok = true;
            float t;
            for (int k = 0; k < 3; ++k) {
                ok = ok && f32_ok(o.center[k], d.center[k]) && f32_ok(o.linear_velocity[k], d.lin[k]) &&
                     f32_ok(o.angular_velocity[k], d.ang[k]) && f32_ok(o.dims[k], d.dims[k]);
            }
            for (int k = 0; k < 4; ++k) ok = ok && f32_ok(o.orientation[k], d.q[k]);
            ok = ok && f32_ok(o.friction, d.lin[3]);
            if (o.shape == TMPM_SHAPE_TRIANGLE_PRISM) {
                double rmax = 0.0;
                for (int vtx = 0; vtx < 3; ++vtx) {
                    double r2 = 0.0;
                    for (int k = 0; k < 3; ++k) {
                        ok = ok && f32_ok(o.vertices[3 * vtx + k], d.verts[4 * vtx + k]);
                        r2 += o.vertices[3 * vtx + k] * o.vertices[3 * vtx + k];
                    }
                    rmax = std::max(rmax, std::sqrt(r2));
                }
                ok = ok && f32_ok((rmax + o.dims[0]) * (1.0 + 1e-5), d.center[3]);
            } else if (o.shape == TMPM_SHAPE_CONVEX) {
                if (o.plane_count > 32) return fail(TMPM_ERR_CAPACITY, "convex obstacle has more than 32 planes");
                d.plane_offset = static_cast<int32_t>(dplanes.size() / 4);
                d.plane_count = static_cast<int32_t>(o.plane_count);
                for (uint32_t pi = 0; pi < 4 * o.plane_count; ++pi) {
                    ok = ok && f32_ok(o.planes[pi], t);
                    dplanes.push_back(t);
                }
                ok = ok && f32_ok(o.bound_radius * (1.0 + 1e-5), d.center[3]);
            }
            if (!ok) return fail(TMPM_ERR_INVALID_INPUT, "obstacle not representable in f32");
            dobs.push_back(d);
        }
        cudaError_t e;
        if ((e = cudaSetDevice(device))) return cuda_fail(e, "cudaSetDevice");
        // block pool sizing from the number of occupied home blocks
        std::sort(home_blocks.begin(), home_blocks.end());
        size_t unique_blocks = std::unique(home_blocks.begin(), home_blocks.end()) - home_blocks.begin();  // small
        uint64_t want_blocks = options.max_blocks ? options.max_blocks : std::max<uint64_t>(4096, 16 * unique_blocks + 4096);
        if (want_blocks > (1u << 27)) want_blocks = 1u << 27;
        for (int b = 0; b < 2; ++b)
            if (pbuf[b].cap != cap)
                if ((e = pbuf[b].alloc(cap))) return cuda_fail(e, "cudaMalloc particles");
        size_t ctas = (cap + kTransferThreads - 1) / kTransferThreads;
        if (cta_cache.count < ctas * kCacheStride)
            if ((e = cta_cache.alloc(ctas * kCacheStride))) return cuda_fail(e, "cudaMalloc cache");
        if (force.count < 3 * std::max<size_t>(world.n, 1)) {
            if ((e = force.alloc(3 * std::max<size_t>(world.n, 1)))) return cuda_fail(e, "cudaMalloc forces");
            cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
        }
        if (force_dirty) cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
        for (int g = 0; g < 2; ++g)
            if (grids[g].max_blocks != want_blocks)
                if ((e = grids[g].alloc(static_cast<uint32_t>(want_blocks)))) return cuda_fail(e, "cudaMalloc grid");
        size_t sort_cap = pbuf[0].cap;
        size_t tiles = (sort_cap + 4095) / 4096;
        if (sort_keys[0].count < sort_cap) {
            for (int b = 0; b < 2; ++b)
                if ((e = sort_keys[b].alloc(sort_cap)) || (e = sort_vals[b].alloc(sort_cap)))
                    return cuda_fail(e, "cudaMalloc sort");
            if ((e = sort_hist.alloc(256 * tiles)) || (e = sort_totals.alloc(256))) return cuda_fail(e, "cudaMalloc sort");
        }
        if ((e = classes.alloc(std::max<size_t>(cls_table.size(), 1)))) return cuda_fail(e, "cudaMalloc classes");
        if ((e = dev_obstacles.alloc(std::max<size_t>(dobs.size(), 1)))) return cuda_fail(e, "cudaMalloc obstacles");
        if ((e = dev_planes.alloc(std::max<size_t>(dplanes.size(), 4)))) return cuda_fail(e, "cudaMalloc planes");
        if (!status.ptr && (e = status.alloc(1))) return cuda_fail(e, "cudaMalloc status");
        if ((e = reactions.alloc(6 * std::max<size_t>(obstacles.size(), 1)))) return cuda_fail(e, "cudaMalloc reactions");

        n_dev = static_cast<int>(n_enabled);
        has_plastic = plastic_classes;
        cur = 0;
        ParticleBuffers &pb = pbuf[0];
        if (n_dev) {
            cudaMemcpyAsync(pb.x.ptr, hx, sizeof(float) * 3 * cap, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(pb.v.ptr, hv, sizeof(float) * 3 * cap, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(pb.C.ptr, hC, sizeof(float) * 9 * cap, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(pb.F.ptr, hF, sizeof(float) * 9 * cap, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(pb.pl.ptr, hpl, sizeof(float) * 3 * cap, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(pb.cls.ptr, hcls, sizeof(uint32_t) * cap, cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(pb.widx.ptr, hwidx, sizeof(uint32_t) * cap, cudaMemcpyHostToDevice, stream);
        }
        if (!cls_table.empty())
            cudaMemcpyAsync(classes.ptr, cls_table.data(), sizeof(DevClass) * cls_table.size(), cudaMemcpyHostToDevice, stream);
        if (!dobs.empty())
            cudaMemcpyAsync(dev_obstacles.ptr, dobs.data(), sizeof(DevObstacle) * dobs.size(), cudaMemcpyHostToDevice, stream);
        if (!dplanes.empty())
            cudaMemcpyAsync(dev_planes.ptr, dplanes.data(), sizeof(float) * dplanes.size(), cudaMemcpyHostToDevice, stream);
        cudaMemsetAsync(status.ptr, 0, sizeof(uint32_t), stream);
        if ((e = upload_forces())) return cuda_fail(e, "upload forces");
        if ((e = cudaStreamSynchronize(stream))) return cuda_fail(e, "upload");
        since_resort = std::numeric_limits<uint64_t>::max();
        return TMPM_OK;
    }

    cudaError_t upload_forces() {
        std::atomic<bool> any{false};
        parallel_for(world.n, [&](size_t lo, size_t hi) {
            for (size_t i = 3 * lo; i < 3 * hi; ++i)
                if (world.force[i] != 0.0) {
                    any = true;
                    break;
                }
        });
        force_dirty = any;
        if (!force_dirty) return cudaSuccess;  // the device array is zero after every consumption
        std::vector<float> f(3 * std::max<size_t>(world.n, 1), 0.0f);
        parallel_for(world.n, [&](size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i)
                for (int k = 0; k < 3; ++k) f[k * world.n + i] = static_cast<float>(world.force[3 * i + k]);
        });
        cudaError_t e = cudaMemcpyAsync(force.ptr, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice, stream);
        if (e) return e;
        return cudaStreamSynchronize(stream);
    }

    ParticleSoA soa() const { return pbuf[cur].view(force.ptr, std::max<size_t>(world.n, 1)); }

    // Grid views for one batch: both share grids[0]'s hash table and block
    // metadata (ids stay stable for the whole batch); they differ in the pool.
    void grid_views(GridTable g[2]) const {
        g[0] = grids[0].view();
        g[1] = g[0];
        g[1].pool = grids[1].pool.ptr;
    }

    // Queue `steps` resident substeps on the stream (encode_prepared, gpu.rs:1729-1777).
    TmpmStatus enqueue(uint32_t steps, double dt, bool resident, bool with_reactions, std::vector<float> *kernel_ms) {
        if (n_dev == 0) return TMPM_OK;
        SimParams sp = sim_params(dt, resident);
        sp.reactions = with_reactions ? 1 : 0;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        auto tick = [&](int slot) {
            if (!kernel_ms) return;
            cudaEventRecord(ev[slot], stream);
        };
        auto tock = [&](int which) {
            if (!kernel_ms) return;
            cudaEventRecord(ev[1], stream);
            cudaEventSynchronize(ev[1]);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            (*kernel_ms)[2 * which] += ms;
            (*kernel_ms)[2 * which + 1] += 1.0f;
        };
        if (kernel_ms) {
            cudaEventCreate(&ev[0]);
            cudaEventCreate(&ev[1]);
        }
        uint32_t interval = options.resort_interval;
        bool resort_now = interval == 0 ? true : since_resort >= interval;
        if (resort_now) {
            tick(0);
            ParticleSoA src = soa();
            ParticleSoA dst = pbuf[cur ^ 1].view(force.ptr, std::max<size_t>(world.n, 1));
            SortBuffers sb{};
            sb.keys[0] = sort_keys[0].ptr;
            sb.keys[1] = sort_keys[1].ptr;
            sb.vals[0] = sort_vals[0].ptr;
            sb.vals[1] = sort_vals[1].ptr;
            sb.hist = sort_hist.ptr;
            sb.totals = sort_totals.ptr;
            sb.cap = sort_keys[0].count;
            launch_resort(src, dst, n_dev, sp, sb, stream);
            cur ^= 1;
            since_resort = 0;
            tock(4);
        }
        GridTable g[2];
        grid_views(g);
        ParticleSoA P = soa();
        tick(0);
        launch_clear_table(g[0], stream);
        launch_transfer(kModeP2G, P, n_dev, classes.ptr, g[1], g[0], sp, dev_obstacles.ptr, dev_planes.ptr,
                        reactions.ptr, status.ptr, cta_cache.ptr, stream);
        tock(0);
        for (uint32_t s = 0; s < steps; ++s) {
            const GridTable &gc = g[s & 1], &gn = g[(s + 1) & 1];
            tick(0);
            launch_grid_update(gc, gn, sp, dev_obstacles.ptr, dev_planes.ptr, reactions.ptr, status.ptr, stream);
            tock(1);
            SimParams spk = sp;
            spk.apply_force = (s == 0 && force_dirty) ? 1 : 0;
            bool last = s + 1 == steps;
            tick(0);
            launch_transfer(last ? kModeG2P : kModeG2P2G, P, n_dev, classes.ptr, gc, gn, spk, dev_obstacles.ptr,
                            dev_planes.ptr, reactions.ptr, status.ptr, cta_cache.ptr, stream);
            tock(last ? 3 : 2);
            if (s == 0 && force_dirty) {
                cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
                force_dirty = false;
            }
        }
        since_resort += steps;
        if (kernel_ms) {
            cudaEventDestroy(ev[0]);
            cudaEventDestroy(ev[1]);
        }
        cudaError_t e = cudaGetLastError();
        if (e) return cuda_fail(e, "kernel launch");
        return TMPM_OK;
    }

    // Wait with a time limit (gpu.rs:1853-1862).
    TmpmStatus wait_done() {
        cudaError_t e = cudaEventRecord(done, stream);
        if (e) return cuda_fail(e, "cudaEventRecord");
        auto t0 = std::chrono::steady_clock::now();
        double limit = kSyncTimeoutSeconds;
        if (const char *env = std::getenv("TMPM_SYNC_TIMEOUT_S")) limit = std::max(0.1, std::atof(env));
        for (;;) {
            e = cudaEventQuery(done);
            if (e == cudaSuccess) return TMPM_OK;
            if (e != cudaErrorNotReady) return cuda_fail(e, "device work failed");
            double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (el > limit) {
                valid = false;
                return fail(TMPM_ERR_READBACK, "timed out waiting for submitted substeps");
            }
            std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 20 : 200));
        }
    }

    // Read the device state back, validate, and replace the host world
    // (read_prepared + collect_prepared + apply_gpu_transfers, gpu.rs:1821-1989, 2295-2329).
    TmpmStatus read_back_and_apply() {
        uint32_t st = 0;
        cudaError_t e = cudaMemcpy(&st, status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (e) return cuda_fail(e, "status readback");
        if (st & kStatusCapacity) {
            valid = false;
            return fail(TMPM_ERR_CAPACITY, "GPU MPM transfer exceeds the device capacity (grid block pool or hash table)");
        }
        if (st & kStatusTimeout) {
            valid = false;
            return fail(TMPM_ERR_READBACK, "a bounded device wait gave up");
        }
        if (st & kStatusResident) {
            valid = false;
            return fail(TMPM_ERR_RESIDENT_UNAVAILABLE,
                        "GPU MPM resident substeps require a CPU fallback; world state is unchanged");
        }
        const int n = n_dev;
        if (n > 0) {
            const size_t pc = pbuf[cur].cap;
            size_t floats = 27 * static_cast<size_t>(n);
            if (!staging.ensure(floats * sizeof(float) + sizeof(uint32_t) * n))
                return fail(TMPM_ERR_DEVICE, "cudaMallocHost staging failed");
            float *h = static_cast<float *>(staging.ptr);
            const ParticleBuffers &pb = pbuf[cur];
            for (int k = 0; k < 3; ++k) {
                cudaMemcpyAsync(h + (0 + k) * n, pb.x.ptr + k * pc, sizeof(float) * n, cudaMemcpyDeviceToHost, stream);
                cudaMemcpyAsync(h + (3 + k) * n, pb.v.ptr + k * pc, sizeof(float) * n, cudaMemcpyDeviceToHost, stream);
            }
            for (int k = 0; k < 9; ++k) {
                cudaMemcpyAsync(h + (6 + k) * n, pb.C.ptr + k * pc, sizeof(float) * n, cudaMemcpyDeviceToHost, stream);
                cudaMemcpyAsync(h + (15 + k) * n, pb.F.ptr + k * pc, sizeof(float) * n, cudaMemcpyDeviceToHost, stream);
            }
            for (int k = 0; k < 3; ++k)
                cudaMemcpyAsync(h + (24 + k) * n, pb.pl.ptr + k * pc, sizeof(float) * n, cudaMemcpyDeviceToHost, stream);
            uint32_t *widx = reinterpret_cast<uint32_t *>(h + floats);
            cudaMemcpyAsync(widx, pb.widx.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, stream);
            if ((e = cudaStreamSynchronize(stream))) return cuda_fail(e, "readback");
            // collect_prepared: non-finite transfers are an error before anything is applied
            std::atomic<bool> bad{false};
            parallel_for(static_cast<size_t>(n), [&](size_t a, size_t b) {
                for (size_t c = 0; c < 27 && !bad.load(std::memory_order_relaxed); ++c)
                    for (size_t j = a; j < b; ++j)
                        if (!std::isfinite(h[c * n + j])) {
                            bad = true;
                            break;
                        }
            });
            if (bad) {
                valid = false;
                return fail(TMPM_ERR_NON_FINITE_STATE, "MPM integration produced a non-finite state");
            }
            parallel_for(static_cast<size_t>(n), [&](size_t a, size_t b) {
                for (size_t j = a; j < b; ++j) {
                    size_t w = widx[j];
                    if (world.fixed[w]) {
                        for (int k = 0; k < 3; ++k) world.vel[3 * w + k] = 0.0;
                        for (int k = 0; k < 9; ++k) world.C[9 * w + k] = 0.0;
                        continue;
                    }
                    for (int k = 0; k < 3; ++k) {
                        world.pos[3 * w + k] = h[(0 + k) * n + j];
                        world.vel[3 * w + k] = h[(3 + k) * n + j];
                    }
                    for (int k = 0; k < 9; ++k) {
                        world.C[9 * w + k] = h[(6 + k) * n + j];
                        world.F[9 * w + k] = h[(15 + k) * n + j];
                    }
                    const int mat = world.material[w];
                    if (mat == TMPM_MAT_SAND || mat == TMPM_MAT_SNOW || mat == TMPM_MAT_SAND_NEO_HOOKEAN)
                        for (int k = 0; k < 3; ++k) world.plastic[3 * w + k] = h[(24 + k) * n + j];
                }
            });
        }
        std::fill(world.force.begin(), world.force.end(), 0.0);
        return TMPM_OK;
    }

    TmpmStatus synchronize() {
        if (!valid) return fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "session is invalid after an earlier error");
        if (pending == 0) return TMPM_OK;
        uint64_t steps = pending;
        pending = 0;
        TmpmStatus st = wait_done();
        if (st != TMPM_OK) return st;
        st = read_back_and_apply();
        if (st != TMPM_OK) return st;
        substeps += steps;
        return TMPM_OK;
    }
};

namespace {

TmpmStatus session_guard(TmpmSession *s, bool require_idle) {
    if (!s) {
        g_last_error = "null session";
        return TMPM_ERR_INVALID_INPUT;
    }
    if (!s->valid) return s->fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "session is invalid after an earlier error");
    if (require_idle && s->pending) return s->fail(TMPM_ERR_PENDING_STEPS, "GPU MPM steps are pending; synchronize first");
    return TMPM_OK;
}

TmpmStatus load_checked(const TmpmParticleArrays *particles, HostWorld &out, std::string &err) {
    if (!particles || particles->count == 0) {
        out.resize(0);
        return TMPM_OK;
    }
    if (!particles->position || !particles->velocity || !particles->mass || !particles->rest_volume ||
        !particles->radius || !particles->material || !particles->material_params) {
        err = "required particle arrays are missing";
        return TMPM_ERR_INVALID_INPUT;
    }
    out.load(*particles);
    std::atomic<bool> bad{false};
    parallel_for(out.n, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi && !bad.load(std::memory_order_relaxed); ++i)
            if (!valid_particle(out, i)) bad = true;
    });
    if (bad) {
        err = "invalid MPM input";
        return TMPM_ERR_MPM_INVALID_INPUT;
    }
    return TMPM_OK;
}

}  // namespace

extern "C" {

const char *tmpm_version(void) { return "tessera-b200 tmpm 0.1 (sm_100a)"; }

const char *tmpm_last_error(void) { return g_last_error.c_str(); }

const char *tmpm_last_error_message(const TmpmSession *s) { return s ? s->last_error.c_str() : g_last_error.c_str(); }

TmpmStatus tmpm_session_create(const TmpmParams *params, const TmpmParticleArrays *particles,
                               const TmpmObstacle *obstacles, size_t obstacle_count, int32_t use_cpic,
                               double substep_dt, const TmpmSessionOptions *options, TmpmSession **out) {
    if (!out || !params) {
        g_last_error = "null argument";
        return TMPM_ERR_INVALID_INPUT;
    }
    *out = nullptr;
    auto s = std::make_unique<TmpmSession>();
    s->params = *params;
    if (options) s->options = *options;
    s->device = s->options.device;
    s->use_cpic = use_cpic != 0;
    s->substep_dt = substep_dt;
    s->substeps = s->options.substeps;
    std::string err;
    if (!params_valid(*params)) {
        g_last_error = "invalid MPM input";
        return TMPM_ERR_MPM_INVALID_INPUT;
    }
    TmpmStatus st = load_checked(particles, s->world, err);
    if (st != TMPM_OK) {
        g_last_error = err;
        return st;
    }
    uint64_t max_chunk = 0;
    for (size_t i = 0; i < s->world.n; ++i) max_chunk = std::max(max_chunk, s->world.chunk[i]);
    s->next_chunk = s->options.next_chunk_id ? s->options.next_chunk_id : max_chunk + 1;
    for (size_t i = 0; i < obstacle_count; ++i) {
        s->obstacles.push_back(obstacles[i]);
        if (obstacles[i].shape == TMPM_SHAPE_CONVEX && obstacles[i].planes) {
            s->obstacle_planes.emplace_back(obstacles[i].planes, obstacles[i].planes + 4 * obstacles[i].plane_count);
            s->obstacles.back().planes = s->obstacle_planes.back().data();
        } else {
            s->obstacle_planes.emplace_back();
        }
    }
    // re-point plane storage after all vectors are in place
    for (size_t i = 0; i < s->obstacles.size(); ++i)
        if (!s->obstacle_planes[i].empty()) s->obstacles[i].planes = s->obstacle_planes[i].data();
    st = s->validate_resident(substep_dt);
    if (st != TMPM_OK) return st;
    cudaError_t e = cudaSetDevice(s->device);
    if (e) {
        g_last_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return TMPM_ERR_DEVICE;
    }
    if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming))) {
        g_last_error = std::string("stream setup: ") + cudaGetErrorString(e);
        return TMPM_ERR_DEVICE;
    }
    st = s->upload(substep_dt);
    if (st != TMPM_OK) return st;
    *out = s.release();
    return TMPM_OK;
}

void tmpm_session_destroy(TmpmSession *s) { delete s; }

TmpmStatus tmpm_submit_steps(TmpmSession *s, uint32_t steps) {
    TmpmStatus st = session_guard(s, false);
    if (st != TMPM_OK) return st;
    if (steps == 0 || steps > 64) return s->fail(TMPM_ERR_INVALID_INPUT, "substeps per submit must be 1..64");
    if (s->pending > std::numeric_limits<uint64_t>::max() - steps) return s->fail(TMPM_ERR_CAPACITY, "pending overflow");
    st = s->validate_resident(s->substep_dt);
    if (st != TMPM_OK) return st;
    cudaSetDevice(s->device);
    st = s->enqueue(steps, s->substep_dt, true, false, nullptr);
    if (st != TMPM_OK) return st;
    s->pending += steps;
    return TMPM_OK;
}

TmpmStatus tmpm_synchronize(TmpmSession *s) {
    if (!s) return TMPM_ERR_INVALID_INPUT;
    cudaSetDevice(s->device);
    return s->synchronize();
}

TmpmStatus tmpm_step(TmpmSession *s, uint32_t steps) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    st = tmpm_submit_steps(s, steps);
    if (st != TMPM_OK) return st;
    return tmpm_synchronize(s);
}

uint64_t tmpm_pending_substeps(const TmpmSession *s) { return s ? s->pending : 0; }
int32_t tmpm_has_pending_steps(const TmpmSession *s) { return s && s->pending ? 1 : 0; }
uint64_t tmpm_substeps(const TmpmSession *s) { return s ? s->substeps : 0; }
size_t tmpm_particle_count(const TmpmSession *s) { return s ? s->world.n : 0; }
size_t tmpm_device_count(const TmpmSession *s) { return s ? static_cast<size_t>(s->n_dev) : 0; }
double tmpm_substep_dt(const TmpmSession *s) { return s ? s->substep_dt : 0.0; }

double tmpm_stable_timestep(const TmpmSession *s) { return s ? stable_timestep(s->world, s->params) : 0.0; }

TmpmStatus tmpm_read_particles(const TmpmSession *s, TmpmParticleArrays *out) {
    if (!s || !out) return TMPM_ERR_INVALID_INPUT;
    if (out->count != s->world.n) {
        g_last_error = "output array count does not match the world";
        return TMPM_ERR_INVALID_INPUT;
    }
    s->world.store(*out);
    return TMPM_OK;
}

TmpmStatus tmpm_set_substep_dt(TmpmSession *s, double dt) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    st = s->validate_resident(dt);
    if (st != TMPM_OK) return st;
    s->substep_dt = dt;
    return TMPM_OK;
}

TmpmStatus tmpm_set_particle_force(TmpmSession *s, size_t index, const double force[3]) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    if (index >= s->world.n || !force) return s->fail(TMPM_ERR_INVALID_INPUT, "particle index out of range");
    float t;
    for (int k = 0; k < 3; ++k)
        if (!f32_ok(force[k], t)) return s->fail(TMPM_ERR_INVALID_INPUT, "force not representable in f32");
    if (!f32_ok(s->world.damping[index], t)) return s->fail(TMPM_ERR_INVALID_INPUT, "damping not representable");
    for (int k = 0; k < 3; ++k) s->world.force[3 * index + k] = force[k];
    cudaSetDevice(s->device);
    cudaError_t e = s->upload_forces();
    if (e) return s->cuda_fail(e, "force upload");
    return TMPM_OK;
}

TmpmStatus tmpm_set_obstacles(TmpmSession *s, const TmpmObstacle *obstacles, size_t count) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    for (size_t i = 0; i < count; ++i)
        if (!obstacle_valid(obstacles[i])) return s->fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM obstacle");
    std::vector<TmpmObstacle> old = s->obstacles;
    std::vector<std::vector<double>> old_planes = s->obstacle_planes;
    s->obstacles.assign(obstacles, obstacles + count);
    s->obstacle_planes.assign(count, {});
    for (size_t i = 0; i < count; ++i)
        if (obstacles[i].shape == TMPM_SHAPE_CONVEX && obstacles[i].planes) {
            s->obstacle_planes[i].assign(obstacles[i].planes, obstacles[i].planes + 4 * obstacles[i].plane_count);
            s->obstacles[i].planes = s->obstacle_planes[i].data();
        }
    cudaSetDevice(s->device);
    st = s->upload(s->substep_dt);
    if (st != TMPM_OK) {
        s->obstacles = old;
        s->obstacle_planes = old_planes;
        for (size_t i = 0; i < s->obstacles.size(); ++i)
            if (!s->obstacle_planes[i].empty()) s->obstacles[i].planes = s->obstacle_planes[i].data();
        if (s->valid) s->upload(s->substep_dt);
        return st;
    }
    return TMPM_OK;
}

TmpmStatus tmpm_add_particles(TmpmSession *s, const TmpmParticleArrays *particles, uint64_t *chunk_out) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    if (!particles || particles->count == 0) return s->fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM input");
    HostWorld add;
    std::string err;
    st = load_checked(particles, add, err);
    if (st != TMPM_OK) return s->fail(st, err);
    if (s->next_chunk == std::numeric_limits<uint64_t>::max())
        return s->fail(TMPM_ERR_PARTICLE_CAPACITY, "MPM particle capacity exceeded");
    uint64_t chunk = s->next_chunk;
    for (size_t i = 0; i < add.n; ++i) add.chunk[i] = chunk;
    HostWorld old = s->world;
    s->world.append(add);
    st = s->validate_resident(s->substep_dt);
    if (st == TMPM_OK) st = s->upload(s->substep_dt);
    if (st != TMPM_OK) {
        s->world = old;
        if (s->valid) s->upload(s->substep_dt);
        return st;
    }
    s->next_chunk += 1;
    if (chunk_out) *chunk_out = chunk;
    return TMPM_OK;
}

TmpmStatus tmpm_remove_chunk(TmpmSession *s, uint64_t chunk, size_t *removed_out) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    HostWorld old = s->world;
    size_t removed = s->world.remove_chunk(chunk);
    if (removed == 0) {
        s->world = old;
        return s->fail(TMPM_ERR_UNKNOWN_CHUNK, "MPM particle chunk was not found");
    }
    st = s->validate_resident(s->substep_dt);
    if (st == TMPM_OK) st = s->upload(s->substep_dt);
    if (st != TMPM_OK) {
        s->world = old;
        if (s->valid) s->upload(s->substep_dt);
        return st;
    }
    if (removed_out) *removed_out = removed;
    return TMPM_OK;
}

TmpmStatus tmpm_write_particles(TmpmSession *s, const TmpmParticleArrays *particles) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    // Load into the session's spare world (its storage is reused across calls)
    // and swap it in; the previous world comes back on any failure.
    HostWorld &nw = s->spare;
    std::string err;
    st = load_checked(particles, nw, err);
    if (st != TMPM_OK) return s->fail(st, err);
    if (!particles || !particles->chunk_id) {
        for (size_t i = 0; i < nw.n && i < s->world.n; ++i) nw.chunk[i] = s->world.chunk[i];
    }
    std::swap(s->world, s->spare);
    st = s->validate_resident(s->substep_dt);
    if (st == TMPM_OK) st = s->upload(s->substep_dt);
    if (st != TMPM_OK) {
        std::swap(s->world, s->spare);
        if (s->valid) s->upload(s->substep_dt);
        return st;
    }
    return TMPM_OK;
}

TmpmStatus tmpm_encode_particle_snapshot(TmpmSession *s, void *device_out, size_t capacity_bytes, uint32_t *written) {
    TmpmStatus st = session_guard(s, false);
    if (st != TMPM_OK) return st;
    if (written) *written = 0;
    if (s->n_dev == 0) return TMPM_OK;
    size_t bytes = 32 * s->world.n;
    if (!device_out || capacity_bytes < bytes) return s->fail(TMPM_ERR_CAPACITY, "snapshot buffer too small");
    cudaSetDevice(s->device);
    cudaMemsetAsync(device_out, 0, bytes, s->stream);
    launch_snapshot(s->soa(), s->n_dev, s->classes.ptr, static_cast<float4 *>(device_out), s->stream);
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e) return s->cuda_fail(e, "snapshot");
    if (written) *written = static_cast<uint32_t>(s->world.n);
    return TMPM_OK;
}

// MpmWorld::step_with_gpu_transfers / step_with_gpu_obstacle_reactions (gpu.rs:2208-2293)
static TmpmStatus step_cfl(TmpmSession *s, double dt, double *reactions_out, size_t obstacle_count) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    if (!std::isfinite(dt) || dt <= 0.0) return s->fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM input");
    for (const TmpmObstacle &o : s->obstacles)
        if (!obstacle_valid(o)) return s->fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM obstacle");
    if (reactions_out && obstacle_count != s->obstacles.size())
        return s->fail(TMPM_ERR_INVALID_INPUT, "reaction buffer does not match the obstacle count");
    std::vector<double> total(6 * s->obstacles.size(), 0.0);
    cudaSetDevice(s->device);
    double remaining = dt;
    size_t count = 0;
    while (remaining > 0.0) {
        double stable = stable_timestep(s->world, s->params);
        if (!std::isfinite(stable) || stable <= 1e-12 || count >= 100000)
            return s->fail(TMPM_ERR_EXCESSIVE_SUBSTEPS, "MPM timestep is too small for the requested duration");
        double sub = std::min(remaining, stable);
        float t;
        if (!f32_ok(sub, t) || t <= 0.0f) return s->fail(TMPM_ERR_INVALID_INPUT, "substep not representable in f32");
        if (reactions_out && !s->obstacles.empty())
            cudaMemsetAsync(s->reactions.ptr, 0, sizeof(double) * 6 * s->obstacles.size(), s->stream);
        st = s->enqueue(1, sub, false, reactions_out != nullptr, nullptr);
        if (st != TMPM_OK) return st;
        s->pending = 1;
        st = s->synchronize();
        if (st != TMPM_OK) return st;
        if (reactions_out && !s->obstacles.empty()) {
            std::vector<double> r(6 * s->obstacles.size());
            cudaMemcpy(r.data(), s->reactions.ptr, sizeof(double) * r.size(), cudaMemcpyDeviceToHost);
            for (size_t k = 0; k < r.size(); ++k) total[k] += r[k];
        }
        remaining = std::max(remaining - sub, 0.0);
        count += 1;
    }
    if (reactions_out) {
        for (size_t k = 0; k < total.size(); ++k) {
            if (!std::isfinite(total[k])) return s->fail(TMPM_ERR_NON_FINITE_STATE, "non-finite obstacle reaction");
            reactions_out[k] = total[k];
        }
    }
    return TMPM_OK;
}

TmpmStatus tmpm_step_cfl(TmpmSession *s, double dt) { return step_cfl(s, dt, nullptr, 0); }

TmpmStatus tmpm_step_cfl_with_reactions(TmpmSession *s, double dt, double *reactions_out, size_t obstacle_count) {
    if (!reactions_out) return TMPM_ERR_INVALID_INPUT;
    return step_cfl(s, dt, reactions_out, obstacle_count);
}

TmpmStatus tmpm_debug_binning(TmpmSession *s, uint32_t *world_index_out, int32_t *base_cell_out, uint32_t *key_out) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    int n = s->n_dev;
    if (n == 0) return TMPM_OK;
    cudaSetDevice(s->device);
    DevBuf<int32_t> cells;
    DevBuf<uint32_t> keys;
    cudaError_t e;
    if ((e = cells.alloc(3 * static_cast<size_t>(n))) || (e = keys.alloc(n))) return s->cuda_fail(e, "cudaMalloc");
    SimParams sp = s->sim_params(s->substep_dt, true);
    ParticleSoA P = s->soa();
    launch_bin_keys(P, n, sp, cells.ptr, keys.ptr, s->stream);
    if (world_index_out) cudaMemcpyAsync(world_index_out, P.widx, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream);
    if (base_cell_out) cudaMemcpyAsync(base_cell_out, cells.ptr, sizeof(int32_t) * 3 * n, cudaMemcpyDeviceToHost, s->stream);
    if (key_out) cudaMemcpyAsync(key_out, keys.ptr, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream);
    if ((e = cudaStreamSynchronize(s->stream))) return s->cuda_fail(e, "binning");
    return TMPM_OK;
}

TmpmStatus tmpm_debug_p2g(TmpmSession *s, int32_t *cells_out, float *mm_out, size_t capacity, size_t *count) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    if (count) *count = 0;
    if (s->n_dev == 0) return TMPM_OK;
    cudaSetDevice(s->device);
    SimParams sp = s->sim_params(s->substep_dt, true);
    GridTable gv[2];
    s->grid_views(gv);
    GridTable g0 = gv[0], g1 = gv[1];
    cudaMemsetAsync(s->status.ptr, 0, sizeof(uint32_t), s->stream);
    launch_clear_table(g0, s->stream);
    launch_transfer(kModeP2G, s->soa(), s->n_dev, s->classes.ptr, g1, g0, sp, s->dev_obstacles.ptr, s->dev_planes.ptr,
                    s->reactions.ptr, s->status.ptr, s->cta_cache.ptr, s->stream);
    DevBuf<int32_t> cells;
    DevBuf<float4> vals;
    DevBuf<uint32_t> cnt;
    size_t cap = std::max<size_t>(capacity, 1);
    cudaError_t e;
    if ((e = cells.alloc(3 * cap)) || (e = vals.alloc(cap)) || (e = cnt.alloc(1))) return s->cuda_fail(e, "cudaMalloc");
    cudaMemsetAsync(cnt.ptr, 0, sizeof(uint32_t), s->stream);
    launch_dump_grid(g0, cells.ptr, vals.ptr, cnt.ptr, static_cast<uint32_t>(cap), s->stream);
    uint32_t total = 0, stw = 0;
    cudaMemcpyAsync(&total, cnt.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    cudaMemcpyAsync(&stw, s->status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream);
    if ((e = cudaStreamSynchronize(s->stream))) return s->cuda_fail(e, "p2g dump");
    if (stw & kStatusCapacity) return s->fail(TMPM_ERR_CAPACITY, "grid capacity exceeded");
    size_t got = std::min<size_t>(total, capacity);
    if (cells_out && got) cudaMemcpy(cells_out, cells.ptr, sizeof(int32_t) * 3 * got, cudaMemcpyDeviceToHost);
    if (mm_out && got) cudaMemcpy(mm_out, vals.ptr, sizeof(float4) * got, cudaMemcpyDeviceToHost);
    if (count) *count = total;
    return TMPM_OK;
}

TmpmStatus tmpm_bench_substeps(TmpmSession *s, uint32_t steps, double *ms, double *kernel_ms, size_t kernel_count) {
    TmpmStatus st = session_guard(s, false);
    if (st != TMPM_OK) return st;
    if (steps == 0) return s->fail(TMPM_ERR_INVALID_INPUT, "steps must be positive");
    cudaSetDevice(s->device);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    std::vector<float> acc(10, 0.0f);
    cudaStreamSynchronize(s->stream);
    cudaEventRecord(a, s->stream);
    uint32_t left = steps;
    while (left) {
        uint32_t batch = std::min<uint32_t>(64, left);
        st = s->enqueue(batch, s->substep_dt, true, false, kernel_ms ? &acc : nullptr);
        if (st != TMPM_OK) break;
        left -= batch;
    }
    cudaEventRecord(b, s->stream);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (st != TMPM_OK) return st;
    s->pending += steps;
    if (ms) *ms = t;
    if (kernel_ms)
        for (size_t k = 0; k < kernel_count && k < 5; ++k) kernel_ms[k] = acc[2 * k + 1] > 0 ? acc[2 * k] / acc[2 * k + 1] : 0.0;
    return TMPM_OK;
}

}  // extern "C"
