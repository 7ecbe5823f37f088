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
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tmpm.h"
#include "tmpm_host.h"
#include "tmpm_internal.h"

using namespace tmpm;


void tmpm::set_last_error(const std::string &msg) { g_last_error = msg; }

namespace {
// The local-frame box that holds an obstacle's surface (DevObstacle::reach),
// from the shape definitions of obstacle.rs:372-472, widened by 1e-4 of
// itself against the f32 rounding of the device's distance evaluations.
void obstacle_reach(const TmpmObstacle &o, DevObstacle &d) {
    const double *dm = o.dims;
    double r[3] = {0.0, 0.0, 0.0};
    double ground = 0.0;
    switch (o.shape) {
    case TMPM_SHAPE_SPHERE:
        r[0] = r[1] = r[2] = dm[0];
        break;
    case TMPM_SHAPE_BOX:
        r[0] = dm[0], r[1] = dm[1], r[2] = dm[2];
        break;
    case TMPM_SHAPE_CAPSULE:  // segment of half height dm[0] along z, radius dm[1]
        r[0] = r[1] = dm[1];
        r[2] = dm[0] + dm[1];
        break;
    case TMPM_SHAPE_CYLINDER:  // half height dm[0] along z, radius dm[1]
    case TMPM_SHAPE_CONE:      // base radius dm[1] at z = -dm[0], apex at z = dm[0]
        r[0] = r[1] = dm[1];
        r[2] = dm[0];
        break;
    case TMPM_SHAPE_GROUND:  // the plane z = 0 over |x| <= dm[0], |y| <= dm[1], solid below
        r[0] = dm[0], r[1] = dm[1];
        ground = 1.0;
        break;
    default:  // triangle prism, convex: the bounding radius
        r[0] = r[1] = r[2] = static_cast<double>(d.center[3]);
    }
    for (int k = 0; k < 3; ++k) d.reach[k] = static_cast<float>(r[k] * (1.0 + 1e-4));
    d.reach[3] = static_cast<float>(ground);
}
}  // namespace

// Segments of at least this many substeps are captured and replayed as CUDA
// graphs (shorter ones, e.g. the single substeps of tmpm_step_cfl, are
// launched: a capture costs more than it saves when not repeated).
constexpr uint32_t kGraphMinSubsteps = 8;

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
    DevBuf<DevRigid> rigid_bodies;  // two-way rigid coupling (tmpm_rigid_*)
    DevBuf<DevRigidMap> rigid_maps;
    size_t rigid_body_count = 0, rigid_map_count = 0;
    DevBuf<int> cta_cache;  // kCacheStride ints per transfer CTA
    DevBuf<uint32_t> defer;  // the fused transfer's deferred-chunk lists (defer_words of the chunk count)
    ForkJoin fj{};           // second stream and events of the fused transfer
    DevBuf<uint32_t> sort_keys[2], sort_vals[2], sort_hist, sort_totals;
    PinnedBuf staging;         // readback
    DevBuf<float> unsorted;    // readback rows in world order
    DevBuf<uint32_t> readback_flag;  // non-finite flag of a readback
    static constexpr int kReadChunks = 8;
    cudaEvent_t read_events[kReadChunks] = {};  // pipelined readback: copy chunk k+1 while chunk k is applied
    PinnedBuf upload_staging;  // packed f32 state for uploads
    bool force_dirty = false;
    bool has_plastic = false;  // class table holds a snow, sand or NH sand class
    uint64_t since_resort = 0;
    LaunchTuner tuner;       // transfer launch configuration (tuned on the first segments unless fixed)
    // Segments captured as CUDA graphs, keyed by everything their kernels bake
    // in (parameters, buffer pointers, sizes); replayed when a segment repeats.
    std::map<std::string, cudaGraphExec_t> seg_graphs;
    int stored_shape = -1;   // launch shape whose per-CTA interleave the device rows hold
    bool big_blocks_ok = false;  // the node pools hold the scene in 8^3 blocks too

    ~TmpmSession() {
        if (stream) {
            cudaStreamSynchronize(stream);
        }
        if (fj.side) cudaStreamSynchronize(fj.side);
        drop_graphs();
        if (done) cudaEventDestroy(done);
        if (fj.fork) cudaEventDestroy(fj.fork);
        if (fj.join) cudaEventDestroy(fj.join);
        if (fj.side) cudaStreamDestroy(fj.side);
        for (cudaEvent_t &ev : read_events)
            if (ev) cudaEventDestroy(ev);
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
        sp.s0 = scene_params(params, dt);
        sp.scenes = nullptr;
        sp.scene_status = nullptr;
        sp.multi = 0;
        sp.step_index = 0;
        sp.num_obstacles = static_cast<int>(obstacles.size());
        sp.reactions = 0;
        sp.apply_force = 0;
        sp.resident_checks = resident ? 1 : 0;
        sp.has_plastic = has_plastic ? 1 : 0;
        sp.cpic = cpic_active() ? 1 : 0;
        sp.shape = 0;
        sp.block_shift = kBlockShift;
        return sp;
    }

    // CPIC applies when enabled and some obstacle carries a CPIC group (world.rs:470-490).
    bool cpic_active() const {
        if (!use_cpic) return false;
        for (const TmpmObstacle &o : obstacles)
            if (o.cpic_group >= 0) return true;
        return false;
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
    // `before`, when given, runs on each block of particles just before the
    // packing pass validates and packs it (tmpm_write_particles loads the
    // particles into the world there, so they are checked and packed in cache).
    TmpmStatus upload(double dt, const std::function<bool(size_t, size_t, size_t)> *before = nullptr) {
        float h32, dt32, inv_d32;
        if (!f32_ok(params.cell_width, h32) || !f32_ok(dt, dt32) ||
            !f32_ok(4.0 / (params.cell_width * params.cell_width), inv_d32) || h32 <= 0.0f || dt32 <= 0.0f)
            return fail(TMPM_ERR_INVALID_INPUT, "cell width or substep not representable in f32");
        float inv_h = 1.0f / h32;
        if (!std::isfinite(inv_h)) return fail(TMPM_ERR_INVALID_INPUT, "1 / cell width not representable in f32");

        // CPIC on the device: groups below kMaxCpicGroups and colours below 256
        // (the namespace is colour << 8 | side mask); other cases need the CPU path.
        if (cpic_active()) {
            for (const TmpmObstacle &o : obstacles)
                if (o.cpic_group >= kMaxCpicGroups)
                    return fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "CPIC groups above 7 need the CPU path");
            for (size_t i = 0; i < world.n; ++i)
                if (world.enabled[i] && world.color[i] >= 256)
                    return fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "transfer colours above 255 with CPIC need the CPU path");
        }

        // Validate and pack the world straight into pinned staging (stride `cap`).
        // When the device rows already have this capacity, each range of rows
        // the packing completes is copied to the device at once, so the copy
        // runs while the rest is packed (the rows are final when every
        // particle is enabled; otherwise, or after a failure, the full copies
        // below or the re-upload overwrite them in stream order).
        ClassTable ct;
        size_t cap = 256;
        bool early = false;
        std::atomic<int> early_err{0};
        PackResult pr = pack_world(
            world, inv_h, 0u, ct,
            [&](size_t n_enabled) {
                PackTarget tg;
                cap = std::max<size_t>(256, (n_enabled + 255) / 256 * 256);
                if (n_enabled > static_cast<size_t>(std::numeric_limits<int>::max() / 2)) return tg;
                if (!upload_staging.ensure((27 * cap + 2 * cap) * sizeof(float))) return tg;
                tg.base = static_cast<float *>(upload_staging.ptr);
                tg.cls = reinterpret_cast<uint32_t *>(tg.base + 27 * cap);
                tg.widx = tg.cls + cap;
                tg.stride = cap;
                early = n_enabled == world.n && pbuf[0].cap == cap && pbuf[1].cap == cap;
                return tg;
            },
            [&](size_t c, size_t a, size_t b) { return !before || (*before)(c, a, b); }, true,
            [&](size_t lo, size_t hi) {
                if (!early) return;
                const float *h = static_cast<const float *>(upload_staging.ptr);
                const ParticleBuffers &pb = pbuf[0];
                const size_t pitch = cap * sizeof(float), w = (hi - lo) * sizeof(float);
                const struct {
                    float *dst;
                    int row, rows;
                } parts[5] = {{pb.x.ptr, 0, 3}, {pb.v.ptr, 3, 3}, {pb.C.ptr, 6, 9}, {pb.F.ptr, 15, 9}, {pb.pl.ptr, 24, 3}};
                cudaError_t e = cudaSetDevice(device);
                for (int k = 0; k < 5 && e == cudaSuccess; ++k)
                    e = cudaMemcpy2DAsync(parts[k].dst + lo, pitch, h + parts[k].row * cap + lo, pitch, w, parts[k].rows,
                                          cudaMemcpyHostToDevice, stream);
                if (e != cudaSuccess) early_err = static_cast<int>(e);
            });
        if (early_err.load()) return cuda_fail(static_cast<cudaError_t>(early_err.load()), "cudaMemcpy2DAsync rows");
        if (pr.st != TMPM_OK) {
            if (pr.st == TMPM_ERR_DEVICE && pr.enabled > static_cast<size_t>(std::numeric_limits<int>::max() / 2))
                return fail(TMPM_ERR_CAPACITY, "too many particles for one session");
            return fail(pr.st, pr.msg);
        }
        const size_t n_enabled = pr.enabled;
        const std::vector<DevClass> &cls_table = ct.table;
        const bool plastic_classes = ct.plastic();
        float *hx = static_cast<float *>(upload_staging.ptr);
        float *hv = hx + 3 * cap, *hC = hv + 3 * cap, *hF = hC + 9 * cap, *hpl = hF + 9 * cap;
        uint32_t *hcls = reinterpret_cast<uint32_t *>(hpl + 3 * cap), *hwidx = hcls + cap;
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
            obstacle_reach(o, d);
            if (!ok) return fail(TMPM_ERR_INVALID_INPUT, "obstacle not representable in f32");
            dobs.push_back(d);
        }
        cudaError_t e;
        if ((e = cudaSetDevice(device))) return cuda_fail(e, "cudaSetDevice");
        // block pool sizing from the number of occupied home blocks
        const PoolPlan plan = pool_plan(pr.blocks.size(), big_home_blocks(pr.blocks), options.max_blocks);
        big_blocks_ok = plan.big;
        for (int b = 0; b < 2; ++b)
            if (pbuf[b].cap != cap)
                if ((e = pbuf[b].alloc(cap))) return cuda_fail(e, "cudaMalloc particles");
        size_t ctas = (cap + kMinTransferThreads - 1) / kMinTransferThreads;
        if (cta_cache.count < ctas * kCacheStride)
            if ((e = cta_cache.alloc(ctas * kCacheStride))) return cuda_fail(e, "cudaMalloc cache");
        if (defer.count < defer_words(ctas))
            if ((e = defer.alloc(defer_words(ctas)))) return cuda_fail(e, "cudaMalloc deferred lists");
        if (force.count < 3 * std::max<size_t>(world.n, 1)) {
            if ((e = force.alloc(3 * std::max<size_t>(world.n, 1)))) return cuda_fail(e, "cudaMalloc forces");
            cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
        }
        if (force_dirty) cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
        for (int g = 0; g < 2; ++g)
            if (grids[g].max_blocks != plan.blocks || grids[g].pool_nodes != plan.nodes)
                if ((e = grids[g].alloc(static_cast<uint32_t>(plan.blocks), plan.nodes))) return cuda_fail(e, "cudaMalloc grid");
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
            if (!(early && n_enabled == world.n)) {  // else the rows are on their way already
                cudaMemcpyAsync(pb.x.ptr, hx, sizeof(float) * 3 * cap, cudaMemcpyHostToDevice, stream);
                cudaMemcpyAsync(pb.v.ptr, hv, sizeof(float) * 3 * cap, cudaMemcpyHostToDevice, stream);
                cudaMemcpyAsync(pb.C.ptr, hC, sizeof(float) * 9 * cap, cudaMemcpyHostToDevice, stream);
                cudaMemcpyAsync(pb.F.ptr, hF, sizeof(float) * 9 * cap, cudaMemcpyHostToDevice, stream);
                cudaMemcpyAsync(pb.pl.ptr, hpl, sizeof(float) * 3 * cap, cudaMemcpyHostToDevice, stream);
            }
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
    void grid_views(GridTable g[2], int block_shift) const {
        g[0] = grids[0].view(block_shift);
        g[1] = g[0];
        g[1].pool = grids[1].pool.ptr;
    }

    void drop_graphs() {
        for (auto &kv : seg_graphs) cudaGraphExecDestroy(kv.second);
        seg_graphs.clear();
    }

    SortBuffers sort_buffers() const {
        SortBuffers sb{};
        sb.keys[0] = sort_keys[0].ptr;
        sb.keys[1] = sort_keys[1].ptr;
        sb.vals[0] = sort_vals[0].ptr;
        sb.vals[1] = sort_vals[1].ptr;
        sb.hist = sort_hist.ptr;
        sb.totals = sort_totals.ptr;
        sb.cap = sort_keys[0].count;
        return sb;
    }

    // The kernels of one segment in stream order: re-sort from row buffer
    // `from` into the other (when `resort`), table clear, P2G, `seg` x (grid
    // update, transfer) with the last transfer G2P-only; the one-shot forces
    // act in the first substep and are cleared after it when `apply_force`.
    void launch_segment(const SimParams &sp, int from, bool resort, uint32_t seg, bool apply_force) {
        const int bs = sp.block_shift;
        const int rows = resort ? from ^ 1 : from;
        if (resort) {
            ParticleSoA src = pbuf[from].view(force.ptr, std::max<size_t>(world.n, 1));
            ParticleSoA dst = pbuf[rows].view(force.ptr, std::max<size_t>(world.n, 1));
            SortBuffers sb = sort_buffers();
            launch_resort(src, dst, n_dev, n_dev, classes.ptr, sp, sb, stream);
        }
        GridTable g[2];
        grid_views(g, bs);
        const ParticleSoA P = pbuf[rows].view(force.ptr, std::max<size_t>(world.n, 1));
        launch_clear_table(g[0], g[1], bs, stream);
        const SimParams sp0 = substep_params(sp, -1, false);
        open_defer_lists(sp0);
        launch_transfer(kModeP2G, P, n_dev, classes.ptr, g[1], g[0], sp0, dev_obstacles.ptr, dev_planes.ptr,
                        reactions.ptr, status.ptr, cta_cache.ptr, stream);
        for (uint32_t k = 0; k < seg; ++k) {
            const GridTable &gc = g[k & 1], &gn = g[(k + 1) & 1];
            const SimParams spk = substep_params(sp, static_cast<int>(k), apply_force && k == 0);
            launch_grid_update(gc, gn, spk, dev_obstacles.ptr, dev_planes.ptr, reactions.ptr, status.ptr, stream);
            launch_transfer(k + 1 == seg ? kModeG2P : kModeG2P2G, P, n_dev, classes.ptr, gc, gn, spk,
                            dev_obstacles.ptr, dev_planes.ptr, reactions.ptr, status.ptr, cta_cache.ptr, stream, &fj);
            if (apply_force && k == 0) cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
        }
    }

    // The parameters of one launch of a segment: the substep it completes
    // (-1: the opening P2G), which tags the per-CTA records and picks the
    // deferred-chunk lists, and the one-shot forces.
    SimParams substep_params(const SimParams &sp, int step_index, bool apply_force) const {
        SimParams spk = sp;
        spk.step_index = step_index;
        spk.apply_force = apply_force ? 1 : 0;
        spk.defer = defer.ptr;
        spk.defer_cap = static_cast<int>(defer.count >= static_cast<size_t>(kDeferHeader)
                                             ? (defer.count - kDeferHeader) / 4
                                             : 0);
        return spk;
    }
    // Empty the deferred-chunk list counts before a segment's opening P2G.
    void open_defer_lists(const SimParams &sp0) {
        if (sp0.defer) cudaMemsetAsync(sp0.defer, 0, sizeof(uint32_t) * kDeferHeader, stream);
    }

    // Everything launch_segment's kernels bake in, as a byte string.
    std::string segment_key(const SimParams &sp, int from, bool resort, uint32_t seg, bool apply_force) const {
        struct {
            SimParams sp;
            ParticleSoA rows[2];
            GridTable g[2];
            SortBuffers sb;
            const void *ptr[8];
            size_t force_count, n_world, defer_count;
            int64_t from, resort, seg, n_dev, apply_force;
        } k;
        std::memset(&k, 0, sizeof k);
        k.sp = sp;
        for (int b = 0; b < 2; ++b) k.rows[b] = pbuf[b].view(force.ptr, std::max<size_t>(world.n, 1));
        grid_views(k.g, sp.block_shift);
        k.sb = sort_buffers();
        const void *ptrs[8] = {classes.ptr, dev_obstacles.ptr, dev_planes.ptr, reactions.ptr, status.ptr,
                               cta_cache.ptr, force.ptr, defer.ptr};
        for (int i = 0; i < 8; ++i) k.ptr[i] = ptrs[i];
        k.force_count = force.count;
        k.defer_count = defer.count;
        k.n_world = world.n;
        k.from = from;
        k.resort = resort;
        k.seg = seg;
        k.n_dev = n_dev;
        k.apply_force = apply_force;
        return std::string(reinterpret_cast<const char *>(&k), sizeof k);
    }

    // One segment replayed from its captured graph (captured now if new).
    TmpmStatus run_segment_graph(const SimParams &sp, bool resort, uint32_t seg, bool apply_force) {
        const std::string key = segment_key(sp, cur, resort, seg, apply_force);
        auto it = seg_graphs.find(key);
        cudaError_t e;
        if (it == seg_graphs.end()) {
            if (seg_graphs.size() >= 16) drop_graphs();
            cudaGraph_t g = nullptr;
            if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)))
                return cuda_fail(e, "cudaStreamBeginCapture");
            launch_segment(sp, cur, resort, seg, apply_force);
            if ((e = cudaStreamEndCapture(stream, &g))) return cuda_fail(e, "cudaStreamEndCapture");
            cudaGraphExec_t exec = nullptr;
            e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (e) return cuda_fail(e, "cudaGraphInstantiate");
            it = seg_graphs.emplace(key, exec).first;
        }
        if ((e = cudaGraphLaunch(it->second, stream))) return cuda_fail(e, "cudaGraphLaunch");
        return TMPM_OK;
    }

    // Queue `steps` resident substeps on the stream (encode_prepared, gpu.rs:1729-1777).
    // With `kernel_ms`, each kernel is timed with CUDA events (bench hook).
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
        // The batch runs in segments ending at re-sort points: a re-sort every
        // `interval` substeps keeps each CTA's particles inside a compact box as
        // they move (the fused transfer slows as boxes widen).  A segment ends
        // with a G2P-only transfer (the fused one keeps v and C in registers)
        // and the next opens with re-sort, table clear and P2G.
        const uint32_t interval = options.resort_interval ? options.resort_interval : kResortSubsteps;
        // Plastic and CPIC variants run the default shape only.
        const bool tunable = !has_plastic && !sp.cpic;
        TmpmStatus st = TMPM_OK;
        for (uint32_t done = 0; done < steps && st == TMPM_OK;) {
            // a challenger only where the segment will be a full one replayed from its graph (timed)
            const bool full = kernel_ms == nullptr && steps - done >= interval && interval >= kGraphMinSubsteps;
            const int config = tunable ? tuner.config(big_blocks_ok, false, !obstacles.empty(), full) : 0;
            const int shape = config_shape(config), bs = config_block_shift(config);
            sp.shape = shape;
            sp.block_shift = bs;
            // the rows are re-sorted (and re-interleaved) when the shape changes
            const bool resort = since_resort >= interval || shape != stored_shape;
            const uint32_t seg = std::min<uint32_t>(steps - done, resort ? interval : interval - since_resort);
            const bool apply_force = done == 0 && force_dirty;
            // Replay a captured graph for a segment long enough to be worth it,
            // outside per-kernel timing and tuning trials; otherwise launch.
            if (kernel_ms == nullptr && !(tunable && tuner.tuning()) && seg >= kGraphMinSubsteps) {
                // after the choice, full segments are timed (re-sort included) for the
                // tuner's watch, once their graph exists: a segment that captures its
                // graph first would count the capture as device time.  A
                // challenger without a graph runs its kernels directly (probed:
                // the launches stay ahead of the device, so its device time is
                // the replay's) and gets no graph unless it takes over, so a
                // challenge never pays a capture.
                const bool cached = seg_graphs.count(segment_key(sp, cur, resort, seg, apply_force)) > 0;
                const bool challenge = tunable && tuner.watching() && config != tuner.current(big_blocks_ok);
                const bool probe = tunable && resort && seg == interval && tuner.watching() && (cached || challenge);
                if (probe) tuner.probe_begin(config, stream);
                if (challenge && !cached)
                    launch_segment(sp, cur, resort, seg, apply_force);
                else
                    st = run_segment_graph(sp, resort, seg, apply_force);
                if (probe) tuner.probe_end(static_cast<double>(n_dev) * seg, stream);
            } else {
                // launch_segment's kernels one by one, timed with `kernel_ms`
                if (resort) {
                    tick(0);
                    ParticleSoA src = soa();
                    ParticleSoA dst = pbuf[cur ^ 1].view(force.ptr, std::max<size_t>(world.n, 1));
                    SortBuffers sb = sort_buffers();
                    launch_resort(src, dst, n_dev, n_dev, classes.ptr, sp, sb, stream);
                    tock(4);
                }
                if (tunable) tuner.begin(config, stream);
                GridTable g[2];
                grid_views(g, bs);
                const ParticleSoA P = pbuf[resort ? cur ^ 1 : cur].view(force.ptr, std::max<size_t>(world.n, 1));
                tick(0);
                launch_clear_table(g[0], g[1], bs, stream);
                const SimParams sp0 = substep_params(sp, -1, false);
                open_defer_lists(sp0);
                launch_transfer(kModeP2G, P, n_dev, classes.ptr, g[1], g[0], sp0, dev_obstacles.ptr, dev_planes.ptr,
                                reactions.ptr, status.ptr, cta_cache.ptr, stream);
                tock(0);
                for (uint32_t k = 0; k < seg; ++k) {
                    const GridTable &gc = g[k & 1], &gn = g[(k + 1) & 1];
                    const SimParams spk = substep_params(sp, static_cast<int>(k), apply_force && k == 0);
                    tick(0);
                    launch_grid_update(gc, gn, spk, dev_obstacles.ptr, dev_planes.ptr, reactions.ptr, status.ptr,
                                       stream);
                    tock(1);
                    const bool last = k + 1 == seg;
                    tick(0);
                    launch_transfer(last ? kModeG2P : kModeG2P2G, P, n_dev, classes.ptr, gc, gn, spk,
                                    dev_obstacles.ptr, dev_planes.ptr, reactions.ptr, status.ptr, cta_cache.ptr,
                                    stream, &fj);
                    tock(last ? 3 : 2);
                    if (apply_force && k == 0) cudaMemsetAsync(force.ptr, 0, sizeof(float) * force.count, stream);
                }
                if (tunable) tuner.end(static_cast<double>(n_dev) * seg, stream);
            }
            if (resort) {
                cur ^= 1;
                since_resort = 0;
                stored_shape = shape;
            }
            if (apply_force) force_dirty = false;
            since_resort += seg;
            done += seg;
        }
        if (kernel_ms) {
            cudaEventDestroy(ev[0]);
            cudaEventDestroy(ev[1]);
        }
        if (st != TMPM_OK) return st;
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
            // rows back in world order on the device, one copy, then sequential host passes
            const size_t N = world.n, floats = 27 * N;
            if (unsorted.count < floats && (e = unsorted.alloc(floats))) return cuda_fail(e, "cudaMalloc readback");
            if (!readback_flag.count && (e = readback_flag.alloc(1))) return cuda_fail(e, "cudaMalloc readback");
            if (!staging.ensure(floats * sizeof(float))) return fail(TMPM_ERR_DEVICE, "cudaMallocHost staging failed");
            for (cudaEvent_t &ev : read_events)
                if (!ev && (e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming))) return cuda_fail(e, "cudaEventCreate");
            float *h = static_cast<float *>(staging.ptr);
            // collect_prepared: non-finite transfers are an error before anything is
            // applied; the un-sort kernel checks every component on the device
            uint32_t nonfinite = 0;
            if ((e = cudaMemsetAsync(readback_flag.ptr, 0, sizeof(uint32_t), stream))) return cuda_fail(e, "readback");
            launch_unsort(soa(), n, unsorted.ptr, N, stream, readback_flag.ptr);
            if ((e = cudaMemcpyAsync(&nonfinite, readback_flag.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) ||
                (e = cudaStreamSynchronize(stream)))
                return cuda_fail(e, "readback");
            if (nonfinite) {
                valid = false;
                return fail(TMPM_ERR_NON_FINITE_STATE, "MPM integration produced a non-finite state");
            }
            // world-index chunks: the copy of chunk k + 1 runs while chunk k is applied
            const size_t per = (N + kReadChunks - 1) / kReadChunks;
            int chunks = 0;
            const size_t rows = has_plastic ? 27 : 24;  // rows 24-26 (plastic state) are read for plastic classes only
            for (size_t a = 0; a < N; a += per, ++chunks) {
                const size_t w = std::min(per, N - a) * sizeof(float);
                if ((e = cudaMemcpy2DAsync(h + a, N * sizeof(float), unsorted.ptr + a, N * sizeof(float), w, rows,
                                           cudaMemcpyDeviceToHost, stream)) ||
                    (e = cudaEventRecord(read_events[chunks], stream)))
                    return cuda_fail(e, "readback");
            }
            ++world.version;
            for (int k = 0; k < chunks; ++k) {
                if ((e = cudaEventSynchronize(read_events[k]))) return cuda_fail(e, "readback");
                const size_t lo = k * per, hi = std::min(N, lo + per);
                parallel_for(hi - lo, [&](size_t a, size_t b) {
                for (size_t w = lo + a; w < lo + b; ++w) {
                    for (int c = 0; c < 3; ++c) world.force[3 * w + c] = 0.0;
                    if (!world.enabled[w]) continue;
                    if (world.fixed[w]) {
                        for (int k = 0; k < 3; ++k) world.vel[3 * w + k] = 0.0;
                        for (int k = 0; k < 9; ++k) world.C[9 * w + k] = 0.0;
                        continue;
                    }
                    for (int k = 0; k < 3; ++k) {
                        world.pos[3 * w + k] = h[(0 + k) * N + w];
                        world.vel[3 * w + k] = h[(3 + k) * N + w];
                    }
                    for (int k = 0; k < 9; ++k) {
                        world.C[9 * w + k] = h[(6 + k) * N + w];
                        world.F[9 * w + k] = h[(15 + k) * N + w];
                    }
                    const int mat = world.material[w];
                    if (mat == TMPM_MAT_SAND || mat == TMPM_MAT_SNOW || mat == TMPM_MAT_SAND_NEO_HOOKEAN)
                        for (int q = 0; q < 3; ++q) world.plastic[3 * w + q] = h[(24 + q) * N + w];
                }
                });
            }
            return TMPM_OK;
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
    s->tuner.reset(s->options.launch_shape);
    s->tuner.watch = true;  // one scene: its best configuration can change as it evolves
    std::string err;
    if (!params_valid(*params)) {
        g_last_error = "invalid MPM input";
        return TMPM_ERR_MPM_INVALID_INPUT;
    }
    TmpmStatus st = load_checked(particles, s->world, err, params);
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
        (e = cudaEventCreateWithFlags(&s->done, cudaEventDisableTiming)) ||
        (e = cudaStreamCreateWithFlags(&s->fj.side, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&s->fj.fork, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&s->fj.join, cudaEventDisableTiming))) {
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
    const bool fused = particles && particles->count > 0 && !s->cpic_active() && particles->position &&
                       particles->velocity && particles->mass && particles->rest_volume && particles->radius &&
                       particles->material && particles->material_params;
    if (fused) {
        // The particles are loaded into the world inside the packing pass, one
        // block at a time, so each is copied, validated (world.rs:492-503),
        // bounded for the CFL step and packed for upload while in cache.  The
        // errors keep the order of the two-pass path below: invalid input, then
        // the CFL bound, then what packing rejects.
        std::swap(s->world, s->spare);  // spare: the previous world, restored on failure
        HostWorld &nw = s->world;
        const HostWorld &old = s->spare;
        nw.resize(particles->count);
        const double max_substep = s->params.max_substep, h = s->params.cell_width;
        std::vector<double> part(host_threads() + 1, max_substep);
        std::atomic<bool> bad{false};
        const bool keep_chunks = !particles->chunk_id;
        std::function<bool(size_t, size_t, size_t)> load = [&](size_t c, size_t a, size_t b) {
            if (bad.load(std::memory_order_relaxed)) return false;
            nw.load_range(*particles, a, b);
            double dt = part[c];
            for (size_t i = a; i < b; ++i) {
                if (!valid_particle(nw, i)) {
                    bad = true;
                    return false;
                }
                if (nw.enabled[i] && !nw.fixed[i])
                    dt = std::min(dt, timestep_bound(nw.material[i], &nw.mparams[5 * i], nw.mass[i] / nw.vol[i],
                                                     &nw.vel[3 * i], h, det9(&nw.F[9 * i])));
                if (keep_chunks && i < old.n) nw.chunk[i] = old.chunk[i];
            }
            part[c] = dt;
            return true;
        };
        cudaSetDevice(s->device);
        st = s->upload(s->substep_dt, &load);
        if (bad) {
            st = s->fail(TMPM_ERR_MPM_INVALID_INPUT, "invalid MPM input");
        } else {
            double dt = max_substep;  // the CFL bound stable_timestep() would compute
            for (double d : part) dt = std::min(dt, d);
            nw.cfl_version = nw.version;
            nw.cfl_h = h;
            nw.cfl_max = max_substep;
            nw.cfl_value = std::min(dt, max_substep);
            const TmpmStatus v = s->validate_resident(s->substep_dt);
            if (v != TMPM_OK) st = v;
        }
        if (st != TMPM_OK) {
            std::swap(s->world, s->spare);
            if (s->valid) s->upload(s->substep_dt);
            return st;
        }
        return TMPM_OK;
    }
    // Load into the session's spare world (its storage is reused across calls)
    // and swap it in; the previous world comes back on any failure.
    HostWorld &nw = s->spare;
    std::string err;
    st = load_checked(particles, nw, err, &s->params);
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
    launch_bin_keys(P, n, s->classes.ptr, sp, cells.ptr, keys.ptr, s->stream);
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
    s->grid_views(gv, kBlockShift);
    GridTable g0 = gv[0], g1 = gv[1];
    cudaMemsetAsync(s->status.ptr, 0, sizeof(uint32_t), s->stream);
    launch_clear_table(g0, g1, kBlockShift, s->stream);
    launch_transfer(kModeP2G, s->soa(), s->n_dev, s->classes.ptr, g1, g0, sp, s->dev_obstacles.ptr, s->dev_planes.ptr,
                    s->reactions.ptr, s->status.ptr, s->cta_cache.ptr, s->stream);
    DevBuf<int32_t> cells;
    DevBuf<float4> vals;
    DevBuf<uint32_t> cnt;
    size_t cap = std::max<size_t>(capacity, 1);
    cudaError_t e;
    if ((e = cells.alloc(3 * cap)) || (e = vals.alloc(cap)) || (e = cnt.alloc(1))) return s->cuda_fail(e, "cudaMalloc");
    cudaMemsetAsync(cnt.ptr, 0, sizeof(uint32_t), s->stream);
    launch_dump_grid(g0, cells.ptr, vals.ptr, cnt.ptr, static_cast<uint32_t>(cap), kBlockShift, s->stream);
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
    cudaEvent_t a, b, seg;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventCreateWithFlags(&seg, cudaEventDisableTiming);
    std::vector<float> acc(10, 0.0f);
    cudaStreamSynchronize(s->stream);
    cudaEventRecord(a, s->stream);
    uint32_t left = steps;
    while (left) {
        // one submission of at most 64 substeps (the reference's per-submit
        // maximum) at a time, each waited for, as a caller stepping frame by
        // frame runs them: the tuner's watch reads each segment's time before
        // the next segment picks its launch configuration
        uint32_t batch = std::min<uint32_t>(64, left);
        st = s->enqueue(batch, s->substep_dt, true, false, kernel_ms ? &acc : nullptr);
        if (st != TMPM_OK) break;
        left -= batch;
        if (left) {
            cudaEventRecord(seg, s->stream);
            cudaEventSynchronize(seg);
        }
    }
    cudaEventRecord(b, s->stream);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaEventDestroy(seg);
    if (st != TMPM_OK) return st;
    s->pending += steps;
    if (ms) *ms = t;
    if (kernel_ms)
        for (size_t k = 0; k < kernel_count && k < 5; ++k) kernel_ms[k] = acc[2 * k + 1] > 0 ? acc[2 * k] / acc[2 * k + 1] : 0.0;
    return TMPM_OK;
}

}  // extern "C"

uint32_t tmpm_launch_shape_count(void) { return static_cast<uint32_t>(kNumLaunchConfigs); }

TmpmStatus tmpm_launch_shape_info(uint32_t shape, uint32_t *threads_per_cta, uint32_t *ctas_per_sm,
                                  uint32_t *block_edge) {
    if (shape >= static_cast<uint32_t>(kNumLaunchConfigs)) {
        g_last_error = "launch shape out of range";
        return TMPM_ERR_INVALID_INPUT;
    }
    const int c = static_cast<int>(shape);
    if (threads_per_cta) *threads_per_cta = static_cast<uint32_t>(kLaunchShapes[config_shape(c)].threads);
    if (ctas_per_sm) *ctas_per_sm = static_cast<uint32_t>(kLaunchShapes[config_shape(c)].min_blocks);
    if (block_edge) *block_edge = 1u << config_block_shift(c);
    return TMPM_OK;
}

int32_t tmpm_session_launch_shape(TmpmSession *s, double *ms_per_unit, size_t count) {
    if (!s) return -1;
    cudaSetDevice(s->device);
    if (s->tuner.tuning()) s->tuner.poll();
    else if (s->tuner.watching()) s->tuner.poll_probes();
    if (ms_per_unit) s->tuner.costs(ms_per_unit, static_cast<uint32_t>(count));
    if (s->has_plastic || s->cpic_active()) return 0;  // variants built for the default shape only
    return s->tuner.current(s->big_blocks_ok);  // 8^3 without room: the best 4^3
}

// ---------------------------------------------------------------- rigid coupling

TmpmStatus tmpm_rigid_attach(TmpmSession *s, const TmpmRigidBody *bodies, size_t body_count,
                             const TmpmRigidMapping *mappings, size_t mapping_count) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    if ((body_count && !bodies) || (mapping_count && !mappings))
        return s->fail(TMPM_ERR_INVALID_INPUT, "null rigid body or mapping array");
    if (mapping_count != s->obstacles.size())
        return s->fail(TMPM_ERR_INVALID_INPUT, "one rigid mapping per session obstacle is needed");
    if (body_count > (1u << 20)) return s->fail(TMPM_ERR_CAPACITY, "too many rigid bodies");
    std::vector<DevRigid> db(body_count);
    for (size_t i = 0; i < body_count; ++i) {
        const TmpmRigidBody &b = bodies[i];
        float v[16], im = 0.f;
        const double *src[5] = {b.position, b.orientation, b.linear_velocity, b.angular_velocity, b.inverse_inertia};
        const int width[5] = {3, 4, 3, 3, 3};
        bool ok = f32_ok(b.inverse_mass, im);
        int k = 0;
        for (int f = 0; f < 5; ++f)
            for (int c = 0; c < width[f]; ++c) ok = ok && f32_ok(src[f][c], v[k++]);
        const double qn = b.orientation[0] * b.orientation[0] + b.orientation[1] * b.orientation[1] +
                          b.orientation[2] * b.orientation[2] + b.orientation[3] * b.orientation[3];
        if (!ok || !(std::fabs(qn - 1.0) < 1e-3))
            return s->fail(TMPM_ERR_INVALID_INPUT, "rigid body not finite in f32 or orientation not a unit quaternion");
        db[i].pos_inv_mass = make_float4(v[0], v[1], v[2], im);
        db[i].q = make_float4(v[3], v[4], v[5], v[6]);
        db[i].lin = make_float4(v[7], v[8], v[9], 0.f);
        db[i].ang = make_float4(v[10], v[11], v[12], 0.f);
        db[i].inv_inertia = make_float4(v[13], v[14], v[15], 1.f);
    }
    std::vector<DevRigidMap> dm(mapping_count);
    for (size_t i = 0; i < mapping_count; ++i) {
        const TmpmRigidMapping &m = mappings[i];
        if (m.body >= 0 && static_cast<size_t>(m.body) >= body_count)
            return s->fail(TMPM_ERR_INVALID_INPUT, "rigid mapping names a body that does not exist");
        float c[7];
        bool ok = true;
        for (int k = 0; k < 3; ++k) ok = ok && f32_ok(m.local_center[k], c[k]);
        for (int k = 0; k < 4; ++k) ok = ok && f32_ok(m.local_orientation[k], c[3 + k]);
        if (!ok) return s->fail(TMPM_ERR_INVALID_INPUT, "rigid mapping not finite in f32");
        dm[i].body = m.body < 0 ? -1 : m.body;
        dm[i].local_center = make_float4(c[0], c[1], c[2], 0.f);
        dm[i].local_q = make_float4(c[3], c[4], c[5], c[6]);
    }
    cudaSetDevice(s->device);
    cudaError_t e;
    if ((e = s->rigid_bodies.alloc(std::max<size_t>(body_count, 1))) ||
        (e = s->rigid_maps.alloc(std::max<size_t>(mapping_count, 1))))
        return s->cuda_fail(e, "cudaMalloc rigid");
    if ((body_count && (e = cudaMemcpy(s->rigid_bodies.ptr, db.data(), sizeof(DevRigid) * body_count,
                                       cudaMemcpyHostToDevice))) ||
        (mapping_count && (e = cudaMemcpy(s->rigid_maps.ptr, dm.data(), sizeof(DevRigidMap) * mapping_count,
                                          cudaMemcpyHostToDevice))))
        return s->cuda_fail(e, "rigid upload");
    s->rigid_body_count = body_count;
    s->rigid_map_count = mapping_count;
    return TMPM_OK;
}

TmpmStatus tmpm_rigid_step(TmpmSession *s, uint32_t substeps, const double gravity[3], double max_linear_speed,
                           int32_t integrate_pose) {
    TmpmStatus st = session_guard(s, true);
    if (st != TMPM_OK) return st;
    if (substeps == 0 || substeps > 64) return s->fail(TMPM_ERR_INVALID_INPUT, "substeps per submit must be 1..64");
    if (s->rigid_map_count != s->obstacles.size() || (!s->rigid_body_count && s->rigid_map_count))
        return s->fail(TMPM_ERR_INVALID_INPUT, "rigid coupling not attached for the current obstacle set");
    if (s->cpic_active())
        return s->fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "rigid coupling with CPIC obstacles is not supported");
    RigidParams p{};
    bool ok = f32_ok(s->substep_dt, p.dt) && f32_ok(std::isfinite(max_linear_speed) ? max_linear_speed : -1.0, p.max_speed);
    for (int k = 0; k < 3; ++k) ok = ok && gravity && f32_ok(gravity[k], p.gravity[k]);
    if (!ok) return s->fail(TMPM_ERR_INVALID_INPUT, "rigid gravity or speed limit not finite in f32");
    p.integrate_pose = integrate_pose ? 1 : 0;
    st = s->validate_resident(s->substep_dt);
    if (st != TMPM_OK) return st;
    cudaSetDevice(s->device);
    const int nobs = static_cast<int>(s->obstacles.size());
    for (uint32_t k = 0; k < substeps; ++k) {
        if (nobs) {
            cudaMemsetAsync(s->reactions.ptr, 0, sizeof(double) * 6 * nobs, s->stream);
            launch_rigid_sync(s->rigid_bodies.ptr, s->rigid_maps.ptr, nobs, s->dev_obstacles.ptr, s->stream);
        }
        st = s->enqueue(1, s->substep_dt, true, nobs > 0, nullptr);
        if (st != TMPM_OK) return st;
        launch_rigid_apply(s->rigid_bodies.ptr, static_cast<int>(s->rigid_body_count), s->rigid_maps.ptr, nobs,
                           s->dev_obstacles.ptr, s->reactions.ptr, p, s->stream);
        s->pending += 1;
    }
    cudaError_t e = cudaGetLastError();
    if (e) return s->cuda_fail(e, "rigid coupling launch");
    return s->synchronize();
}

TmpmStatus tmpm_rigid_read(TmpmSession *s, TmpmRigidBody *bodies, size_t body_count) {
    if (!s || (body_count && !bodies)) return TMPM_ERR_INVALID_INPUT;
    if (body_count != s->rigid_body_count) return s->fail(TMPM_ERR_INVALID_INPUT, "body count does not match the attachment");
    if (!body_count) return TMPM_OK;
    std::vector<DevRigid> db(body_count);
    cudaSetDevice(s->device);
    cudaError_t e;
    if ((e = cudaStreamSynchronize(s->stream)) ||
        (e = cudaMemcpy(db.data(), s->rigid_bodies.ptr, sizeof(DevRigid) * body_count, cudaMemcpyDeviceToHost)))
        return s->cuda_fail(e, "rigid readback");
    for (size_t i = 0; i < body_count; ++i) {
        const DevRigid &d = db[i];
        TmpmRigidBody &b = bodies[i];
        const float4 *f[5] = {&d.pos_inv_mass, &d.q, &d.lin, &d.ang, &d.inv_inertia};
        double *dst[5] = {b.position, b.orientation, b.linear_velocity, b.angular_velocity, b.inverse_inertia};
        const int width[5] = {3, 4, 3, 3, 3};
        for (int k = 0; k < 5; ++k) {
            const float c[4] = {f[k]->x, f[k]->y, f[k]->z, f[k]->w};
            for (int j = 0; j < width[k]; ++j) dst[k][j] = c[j];
        }
        b.inverse_mass = d.pos_inv_mass.w;
    }
    return TMPM_OK;
}

void tmpm_rigid_detach(TmpmSession *s) {
    if (!s) return;
    s->rigid_body_count = s->rigid_map_count = 0;
}
