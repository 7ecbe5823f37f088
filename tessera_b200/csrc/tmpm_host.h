// tmpm_host.h -- host-side pieces shared by the single-scene session
// (tmpm_session.cu) and the multi-scene batch (tmpm_batch.cu): the f64 host
// world, validation that mirrors the reference's MpmWorld checks, device and
// pinned buffers, and the f32 packing of a world for upload.
#pragma once

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tmpm.h"
#include "tmpm_internal.h"

namespace tmpm {

inline thread_local std::string g_last_error;  // reason reported by tmpm_last_error()

inline constexpr double kSyncTimeoutSeconds = 5.0;  // gpu.rs:1853-1862

// Host threads for the parallel host passes: the hardware threads (at most 32),
// or TMPM_HOST_THREADS (1-32) when set, read once per process.
inline unsigned host_threads() {
    static const unsigned t = [] {
        unsigned n = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        if (const char *e = std::getenv("TMPM_HOST_THREADS")) {
            const long v = std::strtol(e, nullptr, 10);
            if (v >= 1 && v <= 32) n = static_cast<unsigned>(v);
        }
        return n;
    }();
    return t;
}

// ------------------------------------------------------ host memory traffic

// Copy with non-temporal stores for the 16-byte-aligned middle: the destination
// lines are written without first being read into the cache (no
// read-for-ownership), a third of the traffic of a large state copy, and the
// copy does not evict the data a pass is working on.  Short copies use memcpy.
// A thread that stored this way calls stream_fence() before another thread or
// a DMA engine reads the destination.
inline void stream_copy(void *dst, const void *src, size_t bytes) {
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    if (bytes < 256) {
        std::memcpy(d, s, bytes);
        return;
    }
    const size_t head = (16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15;
    std::memcpy(d, s, head);
    d += head;
    s += head;
    bytes -= head;
    const size_t lines = bytes / 64;
    for (size_t i = 0; i < lines; ++i, d += 64, s += 64) {
        const __m128i a = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s));
        const __m128i b = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + 16));
        const __m128i c = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + 32));
        const __m128i e = _mm_loadu_si128(reinterpret_cast<const __m128i *>(s + 48));
        _mm_stream_si128(reinterpret_cast<__m128i *>(d), a);
        _mm_stream_si128(reinterpret_cast<__m128i *>(d + 16), b);
        _mm_stream_si128(reinterpret_cast<__m128i *>(d + 32), c);
        _mm_stream_si128(reinterpret_cast<__m128i *>(d + 48), e);
    }
    std::memcpy(d, s, bytes - 64 * lines);
}

// Zero `bytes` with non-temporal stores (see stream_copy).
inline void stream_zero(void *dst, size_t bytes) {
    char *d = static_cast<char *>(dst);
    if (bytes < 256) {
        std::memset(d, 0, bytes);
        return;
    }
    const size_t head = (16 - (reinterpret_cast<uintptr_t>(d) & 15)) & 15;
    std::memset(d, 0, head);
    d += head;
    bytes -= head;
    const __m128i z = _mm_setzero_si128();
    const size_t lines = bytes / 64;
    for (size_t i = 0; i < lines; ++i, d += 64) {
        _mm_stream_si128(reinterpret_cast<__m128i *>(d), z);
        _mm_stream_si128(reinterpret_cast<__m128i *>(d + 16), z);
        _mm_stream_si128(reinterpret_cast<__m128i *>(d + 32), z);
        _mm_stream_si128(reinterpret_cast<__m128i *>(d + 48), z);
    }
    std::memset(d, 0, bytes - 64 * lines);
}

inline void stream_fence() { _mm_sfence(); }

// Persistent workers for the parallel host passes (a pass over a few million
// particles takes milliseconds, and creating and joining 16 threads for each
// took ~0.23 ms).  One job runs at a time: the caller and the workers claim
// chunk indices from a shared counter, so the caller alone can finish any job;
// a caller that finds a job running (another thread, or a pass nested inside a
// chunk) runs its own job on threads of its own instead of waiting.  A child
// process forked between passes has no workers and runs each pass on its
// calling thread alone.
class HostPool {
  public:
    static HostPool &get() {
        static HostPool *pool = new HostPool(host_threads() - 1);  // never destroyed: workers may outlive statics
        return *pool;
    }

    // fn(c) for every c in [0, chunks), on the workers and the calling thread;
    // false (nothing run) when another job holds the pool.
    bool try_run(size_t chunks, const std::function<void(size_t)> &fn) {
        std::unique_lock<std::mutex> run(run_mu_, std::try_to_lock);
        if (!run.owns_lock()) return false;
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &fn;
            count_ = chunks;
            next_.store(0, std::memory_order_relaxed);
            completed_ = 0;
            ++gen_;
        }
        cv_.notify_all();
        const size_t did = drain(fn, chunks);
        std::unique_lock<std::mutex> lk(mu_);
        completed_ += did;
        // every chunk done and no worker still between claiming and leaving
        done_cv_.wait(lk, [&] { return completed_ == count_ && active_ == 0; });
        job_ = nullptr;
        return true;
    }

  private:
    explicit HostPool(unsigned workers) {
        for (unsigned w = 0; w < workers; ++w) std::thread([this] { loop(); }).detach();
    }

    size_t drain(const std::function<void(size_t)> &fn, size_t chunks) {
        size_t did = 0;
        for (size_t c; (c = next_.fetch_add(1, std::memory_order_relaxed)) < chunks; ++did) fn(c);
        return did;
    }

    void loop() {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            if (!job_) continue;
            const std::function<void(size_t)> *fn = job_;
            const size_t chunks = count_;
            ++active_;
            lk.unlock();
            const size_t did = drain(*fn, chunks);
            lk.lock();
            completed_ += did;
            --active_;
            if (completed_ == count_ && active_ == 0) done_cv_.notify_all();
        }
    }

    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(size_t)> *job_ = nullptr;
    size_t count_ = 0, completed_ = 0;
    unsigned active_ = 0;
    uint64_t gen_ = 0;
    std::atomic<size_t> next_{0};
};

// Run fn(chunk, begin, end) over [0, n) split into contiguous chunks, one per host thread.
template <typename Fn>
inline void parallel_chunks(size_t n, Fn fn, size_t min_per_chunk = 32768) {
    size_t chunks = std::min<size_t>(host_threads(), std::max<size_t>(1, n / min_per_chunk));
    if (chunks <= 1) {
        fn(size_t(0), size_t(0), n);
        return;
    }
    const size_t per = (n + chunks - 1) / chunks;
    chunks = (n + per - 1) / per;
    const std::function<void(size_t)> job = [&](size_t c) { fn(c, c * per, std::min(n, c * per + per)); };
    if (HostPool::get().try_run(chunks, job)) return;
    std::vector<std::thread> pool;
    for (size_t c = 0; c < chunks; ++c) pool.emplace_back([&, c]() { job(c); });
    for (auto &t : pool) t.join();
}

template <typename Fn>
inline void parallel_for(size_t n, Fn fn) {
    parallel_chunks(n, [&](size_t, size_t a, size_t b) { fn(a, b); });
}

// --------------------------------------------------------------- host world

// Allocator whose value-less construct leaves elements uninitialised: resizing a
// host-world array then neither zero-fills nor touches its pages on the calling
// thread; the parallel loaders write (and first-touch) every element.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept {
        ::new (static_cast<void *>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U *p, Args &&...args) {
        ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

struct HostWorld {
    size_t n = 0;
    // Any change of positions, velocities, deformation or materials bumps
    // `version`; stable_timestep() caches its result per version and params.
    uint64_t version = 0;
    mutable uint64_t cfl_version = ~0ull;
    mutable double cfl_h = 0.0, cfl_max = 0.0, cfl_value = 0.0;
    HostVec<double> pos, vel, F, C, force, mass, vol, radius, damping, plastic, mparams;
    HostVec<int32_t> material;
    HostVec<uint8_t> enabled, fixed;
    HostVec<uint16_t> color;
    HostVec<uint32_t> group;
    HostVec<uint64_t> chunk;

    // Sizes every field for `count` particles; existing storage is reused and
    // not cleared (load() writes every element).
    void resize(size_t count) {
        ++version;
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

    // Field by field (contiguous copies of [lo, hi) in the same layout), with the
    // defaults of absent optional arrays: F = I, C = 0, force 0, damping 0, the
    // plastic state (1, 1 for sand kinds else 0, 0), enabled, not fixed.
    void load_range(const TmpmParticleArrays &a, size_t lo, size_t hi) {
        const size_t m = hi - lo;
        auto copy = [&](auto *dst, const auto *src, int width) {
            std::memcpy(dst + width * lo, src + width * lo, sizeof(*dst) * width * m);
        };
        copy(pos.data(), a.position, 3);
        copy(vel.data(), a.velocity, 3);
        if (a.force) copy(force.data(), a.force, 3);
        else std::fill(force.begin() + 3 * lo, force.begin() + 3 * hi, 0.0);
        if (a.deformation) {
            copy(F.data(), a.deformation, 9);
        } else {
            for (size_t i = lo; i < hi; ++i)
                for (int k = 0; k < 9; ++k) F[9 * i + k] = (k % 4 == 0) ? 1.0 : 0.0;
        }
        if (a.affine) copy(C.data(), a.affine, 9);
        else std::fill(C.begin() + 9 * lo, C.begin() + 9 * hi, 0.0);
        copy(mass.data(), a.mass, 1);
        copy(vol.data(), a.rest_volume, 1);
        copy(radius.data(), a.radius, 1);
        if (a.damping) copy(damping.data(), a.damping, 1);
        else std::fill(damping.begin() + lo, damping.begin() + hi, 0.0);
        copy(material.data(), a.material, 1);
        copy(mparams.data(), a.material_params, 5);
        if (a.plastic) {
            copy(plastic.data(), a.plastic, 3);
        } else {
            for (size_t i = lo; i < hi; ++i) {
                plastic[3 * i] = 1.0;
                plastic[3 * i + 1] =
                    (material[i] == TMPM_MAT_SAND || material[i] == TMPM_MAT_SAND_NEO_HOOKEAN) ? 1.0 : 0.0;
                plastic[3 * i + 2] = 0.0;
            }
        }
        if (a.enabled) {
            for (size_t i = lo; i < hi; ++i) enabled[i] = a.enabled[i] != 0;
        } else {
            std::fill(enabled.begin() + lo, enabled.begin() + hi, uint8_t(1));
        }
        if (a.fixed) {
            for (size_t i = lo; i < hi; ++i) fixed[i] = a.fixed[i] != 0;
        } else {
            std::fill(fixed.begin() + lo, fixed.begin() + hi, uint8_t(0));
        }
        if (a.transfer_color) copy(color.data(), a.transfer_color, 1);
        else std::fill(color.begin() + lo, color.begin() + hi, uint16_t(0));
        if (a.group_id) copy(group.data(), a.group_id, 1);
        else std::fill(group.begin() + lo, group.begin() + hi, 0u);
        if (a.chunk_id) copy(chunk.data(), a.chunk_id, 1);
        else std::fill(chunk.begin() + lo, chunk.begin() + hi, uint64_t(0));
    }

    void store(TmpmParticleArrays &a) const {
        parallel_for(n, [&](size_t lo, size_t hi) {
            store_range(a, lo, hi);
            stream_fence();
        });
    }

    // Field by field, only the fields `a` asks for, with streaming stores (the
    // caller's arrays are written, not read: no read-for-ownership traffic);
    // the caller fences before the arrays are read on another thread.
    void store_range(TmpmParticleArrays &a, size_t lo, size_t hi) const {
        const size_t m = hi - lo;
        auto copy = [&](auto *dst, const auto *src, int width) {
            if (dst) stream_copy(dst + width * lo, src + width * lo, sizeof(*dst) * width * m);
        };
        copy(a.position, pos.data(), 3);
        copy(a.velocity, vel.data(), 3);
        copy(a.force, force.data(), 3);
        copy(a.plastic, plastic.data(), 3);
        copy(a.deformation, F.data(), 9);
        copy(a.affine, C.data(), 9);
        copy(a.mass, mass.data(), 1);
        copy(a.rest_volume, vol.data(), 1);
        copy(a.radius, radius.data(), 1);
        copy(a.damping, damping.data(), 1);
        copy(a.material, material.data(), 1);
        copy(a.material_params, mparams.data(), 5);
        copy(a.transfer_color, color.data(), 1);
        copy(a.group_id, group.data(), 1);
        copy(a.chunk_id, chunk.data(), 1);
        if (a.enabled)
            for (size_t i = lo; i < hi; ++i) a.enabled[i] = enabled[i];
        if (a.fixed)
            for (size_t i = lo; i < hi; ++i) a.fixed[i] = fixed[i];
    }

    void append(const HostWorld &o) {
        ++version;
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
        ++version;
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

inline double det9(const double *m) {  // column-major
    return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) + m[6] * (m[1] * m[5] - m[4] * m[2]);
}
inline double fro9(const double *m) {
    double s = 0;
    for (int k = 0; k < 9; ++k) s += m[k] * m[k];
    return std::sqrt(s);
}
inline bool inverse_norm9(const double *m, double &out) {
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

inline void lame(double young, double poisson, double &lambda, double &mu) {  // material.rs:433-438
    lambda = young * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson));
    mu = young / (2.0 * (1.0 + poisson));
}

inline bool valid_elasticity(double young, double poisson) {  // material.rs:429-431
    return std::isfinite(young) && young > 0.0 && std::isfinite(poisson) && poisson >= -1.0 && poisson < 0.5;
}

inline bool material_valid(int kind, const double *p) {  // material.rs:171-231
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
inline double timestep_bound(int kind, const double *p, double density, const double *v, double h, double det_f) {
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

inline bool finite_particle(const HostWorld &w, size_t i) {  // world.rs:505-515
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(w.pos[3 * i + k]) || !std::isfinite(w.vel[3 * i + k]) || !std::isfinite(w.force[3 * i + k]))
            return false;
    for (int k = 0; k < 9; ++k)
        if (!std::isfinite(w.F[9 * i + k]) || !std::isfinite(w.C[9 * i + k])) return false;
    return std::isfinite(w.mass[i]) && std::isfinite(w.vol[i]) && std::isfinite(w.radius[i]) &&
           std::isfinite(w.damping[i]);
}

inline bool valid_particle(const HostWorld &w, size_t i) {  // world.rs:492-503
    const double *pl = &w.plastic[3 * i];
    return finite_particle(w, i) && w.mass[i] > 0.0 && w.vol[i] > 0.0 && w.radius[i] > 0.0 &&
           material_valid(w.material[i], &w.mparams[5 * i]) && w.damping[i] >= 0.0 && std::isfinite(pl[0]) &&
           pl[0] > 0.0 && std::isfinite(pl[1]) && std::isfinite(pl[2]);
}

inline bool params_valid(const TmpmParams &p) {  // world.rs:51-65
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

inline double stable_timestep(const HostWorld &w, const TmpmParams &p) {  // world.rs:288-303
    if (w.cfl_version == w.version && w.cfl_h == p.cell_width && w.cfl_max == p.max_substep) return w.cfl_value;
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
    w.cfl_version = w.version;
    w.cfl_h = p.cell_width;
    w.cfl_max = p.max_substep;
    w.cfl_value = std::min(dt, p.max_substep);
    return w.cfl_value;
}

// RigidObstacle::is_valid (obstacle.rs:264-341)
inline bool obstacle_valid(const TmpmObstacle &o) {
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

inline bool f32_ok(double v, float &out) {  // finite_f32 (gpu.rs:1992-1999)
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
    void swap(DevBuf &o) {
        std::swap(ptr, o.ptr);
        std::swap(count, o.count);
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
    void swap(ParticleBuffers &o) {
        x.swap(o.x);
        v.swap(o.v);
        C.swap(o.C);
        F.swap(o.F);
        pl.swap(o.pl);
        cls.swap(o.cls);
        widx.swap(o.widx);
        std::swap(cap, o.cap);
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

// Hash table, block coordinates and node pool of one grid.  `max_blocks` counts
// 4^3 blocks; the pool holds `pool_nodes` nodes, at least max_blocks x 64, so
// a view for 8^3 blocks has pool_nodes / 512 blocks.
struct GridBuffers {
    DevBuf<unsigned long long> keys;
    DevBuf<uint32_t> vals, count;
    DevBuf<float4> pool;
    DevBuf<int4> coords;
    uint32_t capacity = 0, max_blocks = 0;
    size_t pool_nodes = 0;
    cudaError_t alloc(uint32_t blocks, size_t nodes = 0) {
        nodes = std::max(nodes, static_cast<size_t>(blocks) * kNodesPerBlock);
        uint32_t cap = 1024;
        while (cap < 2u * blocks) cap <<= 1;
        cudaError_t e;
        if ((e = keys.alloc(cap)) || (e = vals.alloc(cap)) || (e = count.alloc(1)) || (e = pool.alloc(nodes)) ||
            (e = coords.alloc(blocks)))
            return e;
        capacity = cap;
        max_blocks = blocks;
        pool_nodes = nodes;
        return cudaSuccess;
    }
    GridTable view(int block_shift = kBlockShift) const {
        GridTable g;
        g.keys = keys.ptr;
        g.vals = vals.ptr;
        g.count = count.ptr;
        g.pool = pool.ptr;
        g.coords = coords.ptr;
        g.mask = capacity - 1;
        g.max_blocks = static_cast<uint32_t>(std::min<size_t>(max_blocks, pool_nodes >> (3 * block_shift)));
        return g;
    }
};

// Occupied 8^3 home blocks from the sorted, distinct 4^3 home-block keys
// (namespace << 48 | biased bx << 32 | biased by << 16 | biased bz).
inline size_t big_home_blocks(const std::vector<unsigned long long> &blocks4) {
    std::vector<unsigned long long> big;
    big.reserve(blocks4.size());
    auto halve = [](unsigned long long key, int at) {
        const int c = static_cast<int>((key >> at) & 0xFFFFu) - kBlockBias;
        return static_cast<unsigned long long>(static_cast<uint32_t>((c >> 1) + kBlockBias) & 0xFFFFu) << at;
    };
    for (unsigned long long k : blocks4)
        big.push_back((k & 0xFFFF000000000000ull) | halve(k, 32) | halve(k, 16) | halve(k, 0));
    std::sort(big.begin(), big.end());
    return static_cast<size_t>(std::unique(big.begin(), big.end()) - big.begin());
}

// Block pool sizing: 16 pool blocks per occupied home block plus slack, in 4^3
// blocks (or the caller's fixed count).  8^3 blocks are a tuner candidate when
// the same rule for them needs at most twice the 4^3 pool's nodes (dense
// scenes); the pool then holds the larger of the two.
struct PoolPlan {
    uint64_t blocks = 0;  // 4^3 blocks
    size_t nodes = 0;
    bool big = false;
};
inline PoolPlan pool_plan(size_t home4, size_t home8, uint64_t fixed_blocks, uint64_t slack_num = 0) {
    PoolPlan p;
    uint64_t want = fixed_blocks ? fixed_blocks : std::max<uint64_t>(4096, 16 * home4 + 4096);
    if (!fixed_blocks) want += want * slack_num / 4;
    want = std::min<uint64_t>(want, 1u << 27);
    p.blocks = want;
    p.nodes = static_cast<size_t>(want) * kNodesPerBlock;
    if (!fixed_blocks) {
        uint64_t big_blocks = 16 * static_cast<uint64_t>(home8) + 512;
        big_blocks += big_blocks * slack_num / 4;
        const size_t big_nodes = static_cast<size_t>(big_blocks) * kBigNodesPerBlock;
        if (big_nodes <= 2 * p.nodes && big_blocks <= want) {
            p.big = true;
            p.nodes = std::max(p.nodes, big_nodes);
        }
    }
    return p;
}

// Launch-configuration tuner of the transfer kernels (a configuration is a
// launch shape and a grid block edge, see config_shape / config_block_shift).
// The first submitted segments (real work, not a rehearsal) run under each
// candidate in turn, timed with CUDA events on the submitting stream: one
// round in order and one in reverse order, so that a workload that gets
// slower or faster as the scene evolves weighs on every candidate alike, and
// the candidate with the least mean time per particle-substep is kept once
// every trial has completed.  The candidates' kernels are loaded before the
// first trial, so none pays a lazy module load.  Nothing waits for a trial:
// completed events are read when the next segment asks for its
// configuration.  Candidates are the 4^3-block configurations, and the
// 8^3-block ones too when the block pool can hold them (`allow_big` at the
// first request).
struct LaunchTuner {
    static constexpr int kRounds = 2;
    // Trials this long (particle-substeps; ~0.15 s of device time) are measured
    // well enough in one round: the second is skipped.
    static constexpr double kOneRoundWork = 1073741824.0;
    int rounds = kRounds;
    int fixed = -1;       // >= 0: the caller's configuration; no tuning
    int chosen = -1;      // the tuned configuration, -1 while trials are outstanding
    int candidates = 0;   // configurations under trial (0: not yet started)
    int issued = 0;       // trials started
    int read = 0;         // trials whose time has been read
    double best[kNumLaunchConfigs];  // mean ms per particle-substep of the trials read
    int rounds_read[kNumLaunchConfigs];
    struct Trial {
        int config = 0;
        double work = 0.0;
        cudaEvent_t a = nullptr, b = nullptr;
    };
    std::vector<Trial> trials;
    int open = -1;  // index of the trial being recorded

    // After the choice (single scenes, `watch`): a scene's cost per
    // particle-substep drifts as it evolves (a dam break's CTA boxes widen as
    // it spreads) and the best configuration can change with it, so every full
    // segment keeps being timed ("probes") and every kChallengeEvery-th one
    // runs the best other candidate by its latest time; the challenger takes
    // over when it beat the mean of the chosen configuration's segments since
    // the last challenge by more than kSwitchMargin.  Segments open with a
    // re-sort and a table clear either way, so a switch costs nothing extra.
    // A segment that first captures its graph is not probed (the capture would
    // count as device time); a challenge not probed is issued again.
    static constexpr int kChallengeEvery = 6;
    static constexpr double kSwitchMargin = 0.01;
    bool watch = false;
    struct Probe {
        int config = 0;
        double work = 0.0;
        cudaEvent_t a = nullptr, b = nullptr;
    };
    std::vector<Probe> probes;        // recorded, oldest first; read ones are removed
    std::vector<cudaEvent_t> spare;   // events of read probes, reused
    int probe_open = -1;
    double recent = 0.0;              // mean time of the chosen configuration's probes since the last challenge
    int recent_n = 0;
    int since_challenge = 0;          // probes of the chosen configuration since the last challenge
    bool challenge_pending = false;   // a challenger's probe is recorded but not read

    LaunchTuner() { reset(0); }
    ~LaunchTuner() {
        release();
        drop_probes();
    }
    LaunchTuner(const LaunchTuner &) = delete;
    LaunchTuner &operator=(const LaunchTuner &) = delete;

    void release() {
        for (Trial &t : trials) {
            if (t.a) cudaEventDestroy(t.a);
            if (t.b) cudaEventDestroy(t.b);
        }
        trials.clear();
        open = -1;
    }
    void drop_probes() {
        for (Probe &p : probes) {
            if (p.a) cudaEventDestroy(p.a);
            if (p.b) cudaEventDestroy(p.b);
        }
        probes.clear();
        for (cudaEvent_t e : spare) cudaEventDestroy(e);
        spare.clear();
        probe_open = -1;
        recent = 0.0;
        recent_n = since_challenge = 0;
        challenge_pending = false;
    }
    // `option`: 0 = tune, k > 0 = fixed configuration k - 1 (out of range: 0).
    void reset(uint32_t option) {
        release();
        drop_probes();
        fixed = option == 0 ? -1 : (option <= static_cast<uint32_t>(kNumLaunchConfigs) ? static_cast<int>(option) - 1 : 0);
        chosen = fixed;
        candidates = 0;
        rounds = kRounds;
        issued = read = 0;
        for (double &b : best) b = std::numeric_limits<double>::infinity();
        for (int &r : rounds_read) r = 0;
    }
    // Candidate of trial t: rounds alternate forward and reverse order.
    int trial_config(int t) const {
        const int pos = t % candidates;
        return (t / candidates) % 2 == 0 ? pos : candidates - 1 - pos;
    }
    bool tuning() const { return chosen < 0; }
    int trials_total() const { return rounds * candidates; }
    void poll() {
        while (read < static_cast<int>(trials.size()) && read != open) {
            Trial &t = trials[read];
            if (cudaEventQuery(t.b) != cudaSuccess) {
                cudaGetLastError();  // cudaErrorNotReady is not an error of the stream
                return;
            }
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess && t.work > 0) {
                const int c = t.config, r = rounds_read[c]++;
                best[c] = r == 0 ? ms / t.work : (best[c] * r + ms / t.work) / (r + 1);
            }
            ++read;
        }
        if (chosen < 0 && candidates > 0 && issued == trials_total() && read == issued) {
            int s = 0;
            for (int k = 1; k < candidates; ++k)
                if (best[k] < best[s]) s = k;
            chosen = s;
            release();
        }
    }
    // Configuration for the next segment.  Without room for 8^3 blocks
    // (`allow_big` false) an 8^3 choice falls back to the best 4^3 one.
    // `multi` and `obstacles` say which kernel variants the trials run;
    // `may_challenge`: the segment will be a full, probed one.
    int config(bool allow_big, bool multi, bool obstacles = false, bool may_challenge = false) {
        if (candidates == 0 && fixed < 0) {
            candidates = allow_big ? kNumLaunchConfigs : kNumLaunchShapes;
            preload_launch_shapes(multi, obstacles);
        }
        int c = chosen;
        if (c < 0) {
            poll();
            c = chosen;
        } else if (watching()) {
            poll_probes();
            c = chosen;
            if (may_challenge && !challenge_pending && recent_n >= 2 && since_challenge >= kChallengeEvery) {
                const int r = challenger(allow_big);
                if (r >= 0) return r;
            }
        }
        if (c < 0) c = issued < trials_total() ? trial_config(issued) : 0;
        return usable(c, allow_big);
    }
    // The configuration to report: the choice (or trial), as config() runs it.
    int current(bool allow_big) const { return chosen < 0 ? chosen : usable(chosen, allow_big); }
    int usable(int c, bool allow_big) const {
        if (!allow_big && c >= kNumLaunchShapes) {
            if (fixed >= 0) return config_shape(c);
            int s = 0;
            for (int k = 1; k < kNumLaunchShapes; ++k)
                if (best[k] < best[s]) s = k;
            return s;
        }
        return c;
    }
    bool watching() const { return watch && chosen >= 0 && fixed < 0 && candidates > 1; }
    // The best candidate other than the choice by its latest time (-1: none).
    int challenger(bool allow_big) const {
        int r = -1;
        const int limit = allow_big ? candidates : std::min(candidates, kNumLaunchShapes);
        for (int k = 0; k < limit; ++k)
            if (k != chosen && (r < 0 || best[k] < best[r])) r = k;
        return r;
    }
    // Brackets a full segment (re-sort included) of `work` particle-substeps
    // after the choice; no-ops unless watching.
    void probe_begin(int config_used, cudaStream_t stream) {
        if (!watching() || probe_open >= 0) return;
        Probe p;
        p.config = config_used;
        p.a = take_event();
        p.b = take_event();
        if (!p.a || !p.b || cudaEventRecord(p.a, stream)) {
            if (p.a) spare.push_back(p.a);
            if (p.b) spare.push_back(p.b);
            cudaGetLastError();
            return;
        }
        probes.push_back(p);
        probe_open = static_cast<int>(probes.size()) - 1;
        if (config_used == chosen) {
            ++since_challenge;
        } else {
            since_challenge = 0;
            challenge_pending = true;
        }
    }
    void probe_end(double work, cudaStream_t stream) {
        if (probe_open < 0) return;
        probes[probe_open].work = work;
        cudaEventRecord(probes[probe_open].b, stream);
        probe_open = -1;
    }
    cudaEvent_t take_event() {
        if (!spare.empty()) {
            cudaEvent_t e = spare.back();
            spare.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return e;
    }
    // Reads the finished probes in order and applies the switch rule.
    void poll_probes() {
        size_t done = 0;
        for (; done < probes.size() && static_cast<int>(done) != probe_open; ++done) {
            Probe &p = probes[done];
            if (cudaEventQuery(p.b) != cudaSuccess) {
                cudaGetLastError();
                break;
            }
            float ms = 0.f;
            const bool ok = cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess && p.work > 0;
            cudaGetLastError();
            spare.push_back(p.a);
            spare.push_back(p.b);
            if (!ok) continue;
            const double v = ms / p.work;
            if (p.config == chosen) {
                recent = (recent * recent_n + v) / (recent_n + 1);
                ++recent_n;
                continue;
            }
            best[p.config] = v;
            challenge_pending = false;
            if (recent_n >= 2 && v < recent * (1.0 - kSwitchMargin)) {
                best[chosen] = recent;
                chosen = p.config;
                recent = v;
                recent_n = 1;
            } else {
                if (recent_n > 0) best[chosen] = recent;
                recent = 0.0;
                recent_n = 0;
            }
        }
        if (done > 0) {
            probes.erase(probes.begin(), probes.begin() + done);
            if (probe_open >= 0) probe_open -= static_cast<int>(done);
        }
    }
    // Brackets one segment of `work` particle-substeps run under config();
    // only trials are recorded.
    void begin(int config_used, cudaStream_t stream) {
        if (chosen >= 0 || candidates == 0 || issued >= trials_total() || config_used != trial_config(issued)) return;
        Trial t;
        t.config = config_used;
        if (cudaEventCreate(&t.a) || cudaEventCreate(&t.b) || cudaEventRecord(t.a, stream)) {
            if (t.a) cudaEventDestroy(t.a);
            if (t.b) cudaEventDestroy(t.b);
            cudaGetLastError();
            return;
        }
        trials.push_back(t);
        open = static_cast<int>(trials.size()) - 1;
        ++issued;
    }
    void end(double work, cudaStream_t stream) {
        if (open < 0) return;
        if (issued == 1 && work >= kOneRoundWork) rounds = 1;
        trials[open].work = work;
        cudaEventRecord(trials[open].b, stream);
        open = -1;
    }
    // Measured ms per particle-substep of each configuration (infinity: not measured).
    void costs(double *out, uint32_t count) const {
        for (uint32_t k = 0; k < count && k < static_cast<uint32_t>(kNumLaunchConfigs); ++k) out[k] = best[k];
    }
};

// Device material codes, as the reference packs them (gpu.rs:1171-1276).
inline int class_kind(int material) {
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


// Node indices at the walls, with the f64 arithmetic of apply_grid_boundary
// (world.rs:561-575: node position i * h against bounds_min + h and
// bounds_max - h): the largest i with i * h <= bound, and the smallest i with
// i * h >= bound.  Clamped far beyond the representable cells.
inline int wall_index_le(double bound, double h) {
    double q = std::floor(bound / h);
    long long i = static_cast<long long>(std::min(std::max(q, -1.0e9), 1.0e9));
    while (static_cast<double>(i + 1) * h <= bound && i < 1000000000LL) ++i;
    while (static_cast<double>(i) * h > bound && i > -1000000000LL) --i;
    return static_cast<int>(i);
}
inline int wall_index_ge(double bound, double h) {
    double q = std::ceil(bound / h);
    long long i = static_cast<long long>(std::min(std::max(q, -1.0e9), 1.0e9));
    while (static_cast<double>(i - 1) * h >= bound && i > -1000000000LL) --i;
    while (static_cast<double>(i) * h < bound && i < 1000000000LL) ++i;
    return static_cast<int>(i);
}

// Per-scene f32 integration constants (MpmParams + the fixed substep).
inline SceneParams scene_params(const TmpmParams &params, double dt) {
    SceneParams sc{};
    float h = static_cast<float>(params.cell_width);
    sc.h = h;
    sc.inv_h = 1.0f / h;
    sc.inv_d = static_cast<float>(4.0 / (params.cell_width * params.cell_width));
    sc.dt = static_cast<float>(dt);
    sc.gx = static_cast<float>(params.gravity[0]);
    sc.gy = static_cast<float>(params.gravity[1]);
    sc.gz = static_cast<float>(params.gravity[2]);
    sc.has_bounds = params.has_bounds ? 1 : 0;
    sc.wall_mode = params.wall_mode;
    sc.live = 1;
    for (int k = 0; k < 3; ++k) {
        sc.bmin[k] = static_cast<float>(params.bounds_min[k]);
        sc.bmax[k] = static_cast<float>(params.bounds_max[k]);
        // gpu.wgsl:962-965: floor(bound * inv_h - 0.5) -/+ 2 in f32
        float lo = std::floor(sc.bmin[k] * sc.inv_h - 0.5f), hi = std::floor(sc.bmax[k] * sc.inv_h - 0.5f);
        sc.first_base[k] = static_cast<int>(std::max(lo, -1.0e9f)) - 2;
        sc.last_base[k] = static_cast<int>(std::min(hi, 1.0e9f)) + 2;
        if (params.has_bounds) {
            sc.wall_lo[k] = wall_index_le(params.bounds_min[k] + params.cell_width, params.cell_width);
            sc.wall_hi[k] = wall_index_ge(params.bounds_max[k] - params.cell_width, params.cell_width);
        }
    }
    return sc;
}

// Load and validate caller arrays (MpmWorld::add_particle checks, world.rs:492-503).
inline TmpmStatus load_checked(const TmpmParticleArrays *particles, HostWorld &out, std::string &err,
                               const TmpmParams *cfl_params = nullptr) {
    if (!particles || particles->count == 0) {
        out.resize(0);
        return TMPM_OK;
    }
    if (!particles->position || !particles->velocity || !particles->mass || !particles->rest_volume ||
        !particles->radius || !particles->material || !particles->material_params) {
        err = "required particle arrays are missing";
        return TMPM_ERR_INVALID_INPUT;
    }
    // Copy, validate and (with `cfl_params`) take the CFL bound in one parallel
    // pass; each particle is checked right after it is copied, while in cache.
    out.resize(particles->count);
    std::atomic<bool> bad{false};
    const double max_substep = cfl_params ? cfl_params->max_substep : 0.0;
    std::vector<double> part(host_threads() + 1, max_substep);
    parallel_chunks(out.n, [&](size_t c, size_t lo, size_t hi) {
        double dt = max_substep;
        constexpr size_t kStep = 256;
        for (size_t a = lo; a < hi && !bad.load(std::memory_order_relaxed); a += kStep) {
            const size_t b = std::min(hi, a + kStep);
            out.load_range(*particles, a, b);
            for (size_t i = a; i < b; ++i) {
                if (!valid_particle(out, i)) {
                    bad = true;
                    break;
                }
                if (cfl_params && out.enabled[i] && !out.fixed[i])
                    dt = std::min(dt, timestep_bound(out.material[i], &out.mparams[5 * i], out.mass[i] / out.vol[i],
                                                     &out.vel[3 * i], cfl_params->cell_width, det9(&out.F[9 * i])));
            }
        }
        part[c] = dt;
    });
    if (bad) {
        err = "invalid MPM input";
        return TMPM_ERR_MPM_INVALID_INPUT;
    }
    if (cfl_params) {  // the same value stable_timestep() computes for this world and params
        double dt = max_substep;
        for (double d : part) dt = std::min(dt, d);
        out.cfl_version = out.version;
        out.cfl_h = cfl_params->cell_width;
        out.cfl_max = cfl_params->max_substep;
        out.cfl_value = std::min(dt, max_substep);
    }
    return TMPM_OK;
}

// Deduplicated device material classes (one DevClass per distinct particle
// constant set; particles carry a class index).
struct ClassTable {
    std::vector<DevClass> table;
    std::unordered_map<std::string, uint32_t> index;
    uint32_t intern(const DevClass &k) {
        std::string key(reinterpret_cast<const char *>(&k), sizeof(DevClass));
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        uint32_t id = static_cast<uint32_t>(table.size());
        table.push_back(k);
        index.emplace(std::move(key), id);
        return id;
    }
    bool plastic() const {
        for (const DevClass &k : table)
            if (k.kind >= kMatSnow) return true;
        return false;
    }
};

// Where pack_world writes: `base` holds 27 component rows of `stride` floats
// (x 0-2, v 3-5, C 6-14, F 15-23, plastic 24-26, matrices column-major),
// `cls` and `widx` one entry per enabled particle.
struct PackTarget {
    float *base = nullptr;
    uint32_t *cls = nullptr;
    uint32_t *widx = nullptr;
    size_t stride = 0;
};

struct PackResult {
    TmpmStatus st = TMPM_OK;
    const char *msg = "";
    size_t enabled = 0;
    std::vector<unsigned long long> blocks;  // distinct occupied home blocks (namespace included), sorted
};

// Validate the world's f32 representation and pack its enabled particles (the
// device half of GpuMpmTransfers::prepare, gpu.rs:1091-1600).  Runs in two
// parallel passes over contiguous particle chunks: pass 1 validates, builds
// per-chunk class tables and block lists and counts enabled particles; then
// `alloc(n_enabled)` supplies the PackTarget and pass 2 writes the f32 rows
// at compacted positions.  Results equal a serial pass in world order.
// `ns_high` is OR-ed into every class's grid namespace (multi-scene batches).
// No work before a block of pass 1 (see pack_world's `before`).
struct PackNoHook {
    bool operator()(size_t, size_t, size_t) const { return true; }
};

// Nothing to do when a range of eager rows is complete (see pack_world's `ready`).
struct PackNoRows {
    void operator()(size_t, size_t) const {}
};

// With `eager_rows`, the f32 rows are written in the first pass, at each
// particle's world index, while its values are in cache (the target comes from
// alloc(world.n)); when every particle is enabled those are the final
// positions and the second pass writes only the class and index rows.  Each
// pass-1 thread calls `ready(begin, end)` whenever the eager rows of world
// indices [begin, end) are written (about every 32k particles), so they can be
// copied on while the pass goes on; they are final only if every particle
// turns out enabled and the pack succeeds.
template <typename Alloc, typename Before = PackNoHook, typename Ready = PackNoRows>
PackResult pack_world(const HostWorld &world, float inv_h, uint32_t ns_high, ClassTable &ct, Alloc alloc,
                      Before before = Before(), bool eager_rows = false, Ready ready = Ready()) {
    PackResult res;
    const size_t N = world.n;
    PackTarget tg0;
    if (eager_rows && N > 0) tg0 = alloc(N);
    const bool eager = tg0.base != nullptr;
    const size_t S0 = tg0.stride;
    struct ChunkOut {
        size_t first_bad = std::numeric_limits<size_t>::max();
        TmpmStatus st = TMPM_OK;
        const char *msg = "";
        size_t enabled = 0;
        bool aborted = false;  // `before` rejected a block
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
        // one particle; `return bad(...)` records the chunk's first error
        auto one = [&](size_t i) {
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
            if (!world.enabled[i]) return;
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
            k.color = ns_high | world.color[i];
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
                (static_cast<unsigned long long>(k.color & 0xFFFF) << 48) |
                (static_cast<unsigned long long>(static_cast<uint32_t>((base[0] >> 2) + kBlockBias) & 0xFFFF) << 32) |
                (static_cast<unsigned long long>(static_cast<uint32_t>((base[1] >> 2) + kBlockBias) & 0xFFFF) << 16) |
                static_cast<unsigned long long>(static_cast<uint32_t>((base[2] >> 2) + kBlockBias) & 0xFFFF);
            if (hb != last_block) {
                o.blocks.push_back(hb);
                last_block = hb;
            }
            if (eager) {
                float *r = tg0.base;
                for (int k3 = 0; k3 < 3; ++k3) {
                    r[k3 * S0 + i] = static_cast<float>(world.pos[3 * i + k3]);
                    r[(3 + k3) * S0 + i] = static_cast<float>(world.vel[3 * i + k3]);
                    r[(24 + k3) * S0 + i] = static_cast<float>(world.plastic[3 * i + k3]);
                }
                for (int k9 = 0; k9 < 9; ++k9) {
                    r[(6 + k9) * S0 + i] = static_cast<float>(world.C[9 * i + k9]);
                    r[(15 + k9) * S0 + i] = static_cast<float>(world.F[9 * i + k9]);
                }
            }
            ++o.enabled;
        };
        // blocks of 256: `before` (e.g. the load of these particles into `world`)
        // runs first, so the particles are checked and packed while in cache;
        // after an error of this pass the rest of the chunk still goes through
        // `before`, whose own errors come first
        constexpr size_t kBlock = 256, kReadyRows = 32768;
        size_t handed = lo;  // eager rows [lo, handed) went to `ready`
        for (size_t a0 = lo; a0 < hi; a0 += kBlock) {
            const size_t b0 = std::min(hi, a0 + kBlock);
            if (!before(c, a0, b0)) {
                o.aborted = true;
                return;
            }
            for (size_t i = a0; i < b0 && o.first_bad == std::numeric_limits<size_t>::max(); ++i) one(i);
            if (eager && o.first_bad == std::numeric_limits<size_t>::max() && (b0 - handed >= kReadyRows || b0 == hi)) {
                ready(handed, b0);
                handed = b0;
            }
        }
        std::sort(o.blocks.begin(), o.blocks.end());
        o.blocks.erase(std::unique(o.blocks.begin(), o.blocks.end()), o.blocks.end());
    });
    for (const ChunkOut &o : co)
        if (o.aborted) {
            res.st = TMPM_ERR_MPM_INVALID_INPUT;
            res.msg = "invalid MPM input";
            return res;
        }
    size_t worst = std::numeric_limits<size_t>::max();
    for (const ChunkOut &o : co)
        if (o.first_bad < worst) {
            worst = o.first_bad;
            res.st = o.st;
            res.msg = o.msg;
        }
    if (res.st != TMPM_OK) return res;
    // merge class tables and block lists (small), compute compacted offsets
    std::vector<std::vector<uint32_t>> remap(co.size());
    std::vector<size_t> offset(co.size(), 0);
    size_t n_enabled = 0;
    for (size_t c = 0; c < co.size(); ++c) {
        offset[c] = n_enabled;
        n_enabled += co[c].enabled;
        for (const DevClass &k : co[c].classes) remap[c].push_back(ct.intern(k));
        res.blocks.insert(res.blocks.end(), co[c].blocks.begin(), co[c].blocks.end());
    }
    std::sort(res.blocks.begin(), res.blocks.end());
    res.blocks.erase(std::unique(res.blocks.begin(), res.blocks.end()), res.blocks.end());
    if (ct.table.size() > kClassMask) {
        res.st = TMPM_ERR_CAPACITY;
        res.msg = "too many distinct particle classes";
        return res;
    }
    res.enabled = n_enabled;
    // every particle enabled: the rows of the first pass are in place
    const bool rows_done = eager && n_enabled == N;
    PackTarget tg = rows_done ? tg0 : alloc(n_enabled);
    if (!tg.base) {
        res.st = TMPM_ERR_DEVICE;
        res.msg = "pinned staging allocation failed";
        return res;
    }
    const size_t S = tg.stride;
    float *hx = tg.base, *hv = hx + 3 * S, *hC = hv + 3 * S, *hF = hC + 9 * S, *hpl = hF + 9 * S;
    parallel_chunks(N, [&](size_t c, size_t lo, size_t hi) {
        size_t j = offset[c];
        const std::vector<uint32_t> &rm = remap[c];
        for (size_t i = lo; i < hi; ++i) {
            if (!world.enabled[i]) continue;
            if (rows_done) {
                tg.cls[j] = rm[lcls[i]] | (world.fixed[i] ? kFixedBit : 0u);
                tg.widx[j] = static_cast<uint32_t>(i);
                ++j;
                continue;
            }
            for (int k3 = 0; k3 < 3; ++k3) {
                hx[k3 * S + j] = static_cast<float>(world.pos[3 * i + k3]);
                hv[k3 * S + j] = static_cast<float>(world.vel[3 * i + k3]);
            }
            for (int k9 = 0; k9 < 9; ++k9) {
                hC[k9 * S + j] = static_cast<float>(world.C[9 * i + k9]);
                hF[k9 * S + j] = static_cast<float>(world.F[9 * i + k9]);
            }
            for (int k3 = 0; k3 < 3; ++k3) hpl[k3 * S + j] = static_cast<float>(world.plastic[3 * i + k3]);
            tg.cls[j] = rm[lcls[i]] | (world.fixed[i] ? kFixedBit : 0u);
            tg.widx[j] = static_cast<uint32_t>(i);
            ++j;
        }
    });
    return res;
}

}  // namespace tmpm
