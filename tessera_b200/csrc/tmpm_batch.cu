// tmpm_batch.cu -- multi-scene batches (include/tmpm.h, "multi-scene batches").
//
// Many independent scenes share one set of device particle rows, one class
// table, one sparse grid (each scene in its own namespace of the block key:
// scene << 8 | transfer colour) and one stream.  A batch is one re-sort, one
// opening P2G and S x (grid update, fused G2P+P2G) launches over the rows of
// every scene, S being the largest substep count asked for; each scene takes
// part in its own first `steps` substeps only (the transfer kernel gates on
// the scene table) and writes its velocity and affine matrix back at its last
// substep.  The per-scene constants live in a device scene table that is
// copied once per batch.
//
// Device rows stay sorted by (scene, block) after every batch's re-sort, so a
// scene occupies one contiguous range and is read back with a few strided
// copies.  Admission is split for overlap with device work: a scene is
// validated and packed into host memory by tmpm_scene_prepare (any thread,
// no device work), attached to the batch by tmpm_batch_admit (allowed while a
// batch is in flight) and copied to the device at the next submit, appended
// after the resident rows.  A retired scene is marked removed: the next
// re-sort moves its rows past the live ones and drops them.  A batch re-sorts
// from one row buffer into the other and only reads the first, so while it
// runs, every scene it does not advance can still be read from the first
// buffer, on a side stream, concurrently with the batch.
//
// Prepared rows stay in ordinary (pageable) memory: pinning a scene-sized
// buffer per scene costs more than the staged copy it would speed up.  An
// admitted scene's rows are copied at once, on an upload stream, when the
// allocated rows have room, so the copy overlaps the batch in flight; reads go
// through one pinned buffer that the batch keeps and reuses.

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "tmpm_host.h"

using namespace tmpm;

namespace {

// Per-particle device bytes: two row sets of 27 floats + class + index, sort
// keys and values (double-buffered); per home block the pool sizing rule
// (16 blocks per occupied block) x two pools of 64 float4 nodes + coords +
// two hash slots.
constexpr size_t kBytesPerRow = 2 * (27 * 4 + 2 * 4) + 4 * 4;
constexpr size_t kBytesPerPoolBlock = 2 * kNodesPerBlock * 16 + 16 + 2 * (8 + 4);

// Rows of one scene in host memory: 27 f32 component rows of `stride`, then
// class and world-index rows (29 rows of 4-byte words).
using HostRows = HostVec<float>;
float *row_base(HostRows &l) { return l.data(); }
uint32_t *row_cls(HostRows &l, size_t stride) { return reinterpret_cast<uint32_t *>(row_base(l) + 27 * stride); }
uint32_t *row_widx(HostRows &l, size_t stride) { return row_cls(l, stride) + stride; }

}  // namespace

// A validated, packed scene waiting for admission (no device state).
struct TmpmPreparedScene {
    TmpmParams params{};
    double dt = 0.0;
    HostWorld world;
    ClassTable classes;     // local classes (namespace 0)
    HostRows rows;          // packed rows, class ids local
    size_t m = 0;           // enabled particles (device rows)
    size_t blocks = 0;      // occupied 4^3 home blocks
    size_t blocks8 = 0;     // occupied 8^3 home blocks
};

namespace {

TmpmStatus prepare_scene(const TmpmParams &params, const TmpmParticleArrays *particles, double dt,
                         TmpmPreparedScene &p) {
    if (!params_valid(params)) {
        g_last_error = "invalid MPM input";
        return TMPM_ERR_MPM_INVALID_INPUT;
    }
    std::string err;
    TmpmStatus st = load_checked(particles, p.world, err, &params);
    if (st != TMPM_OK) {
        g_last_error = err;
        return st;
    }
    if (p.world.n >= (1u << 31)) {
        g_last_error = "too many particles in one scene";
        return TMPM_ERR_CAPACITY;
    }
    for (size_t i = 0; i < p.world.n; ++i)
        if (p.world.color[i] >= kMaxBatchColors) {
            g_last_error = "transfer colours in a batch must be below 256";
            return TMPM_ERR_INVALID_INPUT;
        }
    // validate_resident_world (gpu.rs:664-677)
    if (!std::isfinite(dt) || dt <= 0.0 || dt > stable_timestep(p.world, params)) {
        g_last_error = "substep dt is not finite, not positive or above the CFL bound";
        return TMPM_ERR_INVALID_INPUT;
    }
    float h32, dt32, inv_d32;
    if (!f32_ok(params.cell_width, h32) || !f32_ok(dt, dt32) ||
        !f32_ok(4.0 / (params.cell_width * params.cell_width), inv_d32) || h32 <= 0.0f || dt32 <= 0.0f ||
        !std::isfinite(1.0f / h32)) {
        g_last_error = "cell width or substep not representable in f32";
        return TMPM_ERR_INVALID_INPUT;
    }
    size_t stride = 0;
    PackResult pr = pack_world(p.world, 1.0f / h32, 0u, p.classes, [&](size_t n_enabled) {
        PackTarget tg;
        stride = std::max<size_t>(n_enabled, 1);
        p.rows.resize(29 * stride);
        tg.base = row_base(p.rows);
        tg.cls = row_cls(p.rows, stride);
        tg.widx = row_widx(p.rows, stride);
        tg.stride = stride;
        return tg;
    }, PackNoHook(), true);
    if (pr.st != TMPM_OK) {
        g_last_error = pr.msg;
        return pr.st;
    }
    p.params = params;
    p.dt = dt;
    p.m = pr.enabled;
    p.blocks = pr.blocks.size();
    p.blocks8 = big_home_blocks(pr.blocks);
    return TMPM_OK;
}

struct BatchScene {
    bool live = false;
    bool draining = false;   // removed; its rows go at the next re-sort
    TmpmParams params{};
    double dt = 0.0;
    HostWorld world;         // admitted state, or the last state read back
    bool stale = false;      // the device holds substeps `world` lacks
    uint64_t substeps = 0;   // substeps completed on the device
    size_t dev_offset = 0;   // first device row
    size_t dev_count = 0;    // enabled particles (device rows)
    size_t blocks = 0;       // occupied 4^3 home blocks at admission (pool sizing)
    size_t blocks8 = 0;      // occupied 8^3 home blocks at admission
    uint32_t queued = 0;     // substeps in the batch in flight
    std::unique_ptr<TmpmPreparedScene> staged;  // admitted, rows not yet on the device
    size_t prev_offset = 0;  // first row in the buffer the batch in flight reads
    TmpmStatus status = TMPM_OK;
    std::string error;
};

}  // namespace

struct TmpmBatch {
    TmpmBatchOptions options{};
    int device = 0;
    bool valid = true;
    std::string last_error;
    std::vector<BatchScene> scenes;  // indexed by scene id
    ClassTable classes;
    size_t classes_uploaded = 0;

    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr, t_begin = nullptr, t_end = nullptr;
    ParticleBuffers pbuf[2];
    int cur = 0;
    size_t n_phys = 0;  // device rows in use (live + draining)
    size_t n_live = 0;  // rows of live scenes, staged ones included
    DevBuf<DevClass> dclasses;
    GridBuffers grids[2];
    DevBuf<uint32_t> status, scene_status;
    DevBuf<SceneParams> dscenes;
    DevBuf<int> cta_cache;
    DevBuf<uint32_t> defer;  // the fused transfer's deferred-chunk lists (defer_words of the chunk count)
    ForkJoin fj{};           // second stream and events of the fused transfer
    DevBuf<uint32_t> sort_keys[2], sort_vals[2], sort_hist, sort_totals;
    PinnedBuf table_staging;
    std::vector<std::unique_ptr<TmpmPreparedScene>> in_flight_uploads;  // kept until the copies complete
    cudaStream_t read_stream = nullptr;  // reads of scenes the batch in flight does not advance
    PinnedBuf read_pinned;               // readback staging, reused by every read
    HostRows read_pageable;              // fallback when pinned memory is unavailable
    DevBuf<float> read_unsorted;         // a read scene's rows in world order (27 x its world count)
    DevBuf<uint32_t> take_flag;          // non-finite flag of a take
    cudaStream_t upload_stream = nullptr;  // row copies issued at admission
    cudaEvent_t upload_done = nullptr;
    bool uploads_open = false;  // copies on upload_stream the batch stream has not waited for yet
    // Row copies go through two pinned staging buffers: host threads fill one
    // while the copy engine drains the other (pageable copies are staged by
    // the driver one small buffer at a time, several times slower).
    static constexpr size_t kStageBytes = size_t(64) << 20;
    PinnedBuf stage[2];
    cudaEvent_t stage_free[2] = {nullptr, nullptr};  // recorded after the copies out of each buffer
    bool stage_busy[2] = {false, false};
    std::vector<std::unique_ptr<TmpmPreparedScene>> early_uploads;  // their host rows
    uint64_t epoch = 1;  // bumps whenever a device pointer a graph holds changes
    bool pending = false;
    double last_ms = 0.0;
    LaunchTuner tuner;  // transfer launch configuration (tuned on the first batches unless fixed)
    bool big_blocks_ok = false;  // the node pools hold the live scenes in 8^3 blocks too

    struct GraphKey {
        uint32_t steps;
        size_t n_phys, n_live;
        int cur;
        uint64_t epoch;
        int shape;
        bool operator<(const GraphKey &o) const {
            return std::tie(steps, n_phys, n_live, cur, epoch, shape) <
                   std::tie(o.steps, o.n_phys, o.n_live, o.cur, o.epoch, o.shape);
        }
    };
    std::map<GraphKey, cudaGraphExec_t> graphs;

    ~TmpmBatch() {
        if (upload_worker.joinable()) {
            {
                std::lock_guard<std::mutex> lk(up_mu);
                up_stop = true;
            }
            up_cv.notify_all();
            upload_worker.join();
        }
        if (upload_stream) cudaStreamSynchronize(upload_stream);
        if (stream) cudaStreamSynchronize(stream);
        if (upload_done) cudaEventDestroy(upload_done);
        for (int k = 0; k < 2; ++k)
            if (stage_free[k]) cudaEventDestroy(stage_free[k]);
        if (upload_stream) cudaStreamDestroy(upload_stream);
        drop_graphs();
        if (done) cudaEventDestroy(done);
        if (t_begin) cudaEventDestroy(t_begin);
        if (t_end) cudaEventDestroy(t_end);
        if (read_stream) cudaStreamDestroy(read_stream);
        if (fj.side) cudaStreamSynchronize(fj.side);
        if (fj.fork) cudaEventDestroy(fj.fork);
        if (fj.join) cudaEventDestroy(fj.join);
        if (fj.side) cudaStreamDestroy(fj.side);
        if (stream) cudaStreamDestroy(stream);
    }

    void drop_graphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
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

    TmpmStatus guard(bool idle) {
        if (!valid) return fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "batch is invalid after an earlier error");
        if (idle && pending) return fail(TMPM_ERR_PENDING_STEPS, "a batch is in flight; synchronize first");
        return TMPM_OK;
    }

    BatchScene *scene_at(uint32_t id) {
        if (id >= scenes.size() || !scenes[id].live) return nullptr;
        return &scenes[id];
    }

    SimParams sim_params() const {
        SimParams sp{};
        sp.scenes = dscenes.ptr;
        sp.scene_status = scene_status.ptr;
        sp.multi = 1;
        sp.step_index = 0;
        sp.num_obstacles = 0;
        sp.reactions = 0;
        sp.apply_force = 0;
        sp.resident_checks = 1;
        sp.has_plastic = classes.plastic() ? 1 : 0;
        sp.shape = 0;
        sp.block_shift = kBlockShift;
        return sp;
    }

    size_t total_blocks() const {
        size_t b = 0;
        for (const BatchScene &s : scenes)
            if (s.live || s.draining) b += s.blocks;
        return b;
    }
    size_t total_blocks8() const {
        size_t b = 0;
        for (const BatchScene &s : scenes)
            if (s.live || s.draining) b += s.blocks8;
        return b;
    }

    SortBuffers sort_buffers() {
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

    // Grow the device rows to hold `need` rows, keeping rows [0, n_phys).  Idle only.
    TmpmStatus ensure_rows(size_t need) {
        cudaError_t e;
        if (need > pbuf[cur].cap) {
            size_t cap = std::max<size_t>(need, pbuf[cur].cap + pbuf[cur].cap / 2);
            cap = std::max<size_t>(256, (cap + 255) / 256 * 256);
            ParticleBuffers nb;
            if ((e = nb.alloc(cap))) return cuda_fail(e, "cudaMalloc particles");
            const ParticleBuffers &ob = pbuf[cur];
            if (n_phys) {
                auto copy_rows = [&](void *dst, const void *src, size_t elem, int rows) {
                    return cudaMemcpy2DAsync(dst, cap * elem, src, ob.cap * elem, n_phys * elem, rows,
                                             cudaMemcpyDeviceToDevice, stream);
                };
                if ((e = copy_rows(nb.x.ptr, ob.x.ptr, 4, 3)) || (e = copy_rows(nb.v.ptr, ob.v.ptr, 4, 3)) ||
                    (e = copy_rows(nb.C.ptr, ob.C.ptr, 4, 9)) || (e = copy_rows(nb.F.ptr, ob.F.ptr, 4, 9)) ||
                    (e = copy_rows(nb.pl.ptr, ob.pl.ptr, 4, 3)) || (e = copy_rows(nb.cls.ptr, ob.cls.ptr, 4, 1)) ||
                    (e = copy_rows(nb.widx.ptr, ob.widx.ptr, 4, 1)))
                    return cuda_fail(e, "grow particle rows");
            }
            if ((e = cudaStreamSynchronize(stream))) return cuda_fail(e, "grow particle rows");
            pbuf[cur].swap(nb);
            if ((e = pbuf[cur ^ 1].alloc(cap))) return cuda_fail(e, "cudaMalloc particles");
            ++epoch;
        }
        const size_t cap = pbuf[cur].cap;
        const size_t ctas = (cap + kMinTransferThreads - 1) / kMinTransferThreads;
        if (cta_cache.count < ctas * kCacheStride) {
            if ((e = cta_cache.alloc(ctas * kCacheStride))) return cuda_fail(e, "cudaMalloc cache");
            ++epoch;
        }
        if (defer.count < defer_words(ctas)) {
            if ((e = defer.alloc(defer_words(ctas)))) return cuda_fail(e, "cudaMalloc deferred lists");
            ++epoch;
        }
        if (sort_keys[0].count < cap) {
            const size_t tiles = (cap + 4095) / 4096;
            for (int b = 0; b < 2; ++b)
                if ((e = sort_keys[b].alloc(cap)) || (e = sort_vals[b].alloc(cap))) return cuda_fail(e, "cudaMalloc sort");
            if ((e = sort_hist.alloc(256 * tiles)) || (e = sort_totals.alloc(256))) return cuda_fail(e, "cudaMalloc sort");
            ++epoch;
        }
        return TMPM_OK;
    }

    TmpmStatus ensure_grid() {
        const PoolPlan need = pool_plan(total_blocks(), total_blocks8(), options.max_blocks);
        big_blocks_ok = need.big;
        if (grids[0].max_blocks >= need.blocks && grids[0].pool_nodes >= need.nodes) return TMPM_OK;
        // grow with slack: admissions come one by one
        const PoolPlan grow = pool_plan(total_blocks(), total_blocks8(), options.max_blocks, 1);
        const size_t nodes = std::max(grow.nodes, need.nodes);
        cudaError_t e;
        for (int g = 0; g < 2; ++g)
            if ((e = grids[g].alloc(static_cast<uint32_t>(std::max(grow.blocks, need.blocks)), nodes)))
                return cuda_fail(e, "cudaMalloc grid");
        ++epoch;
        return TMPM_OK;
    }

    // Idle only (synchronous copy from the host table).
    TmpmStatus upload_classes() {
        if (classes.table.size() == classes_uploaded) return TMPM_OK;
        cudaError_t e;
        if (dclasses.count < classes.table.size()) {
            if ((e = dclasses.alloc(std::max<size_t>(2 * classes.table.size(), 64)))) return cuda_fail(e, "cudaMalloc classes");
            ++epoch;
        }
        if ((e = cudaMemcpy(dclasses.ptr, classes.table.data(), sizeof(DevClass) * classes.table.size(),
                            cudaMemcpyHostToDevice)))
            return cuda_fail(e, "upload classes");
        classes_uploaded = classes.table.size();
        ++epoch;  // the transfer variant (plastic or not) captured in a graph follows the class table
        return TMPM_OK;
    }

    // Copy the scene table (with this batch's step counts) to the device.
    cudaError_t upload_table() {
        SceneParams *t = static_cast<SceneParams *>(table_staging.ptr);
        for (size_t id = 0; id < static_cast<size_t>(kMaxScenes); ++id) {
            if (id < scenes.size() && scenes[id].live) {
                const BatchScene &s = scenes[id];
                t[id] = scene_params(s.params, s.dt);
                t[id].steps = static_cast<int>(s.queued);
            } else {
                t[id] = SceneParams{};
                t[id].h = 1.0f;
                t[id].inv_h = 1.0f;
                t[id].live = 0;
            }
        }
        return cudaMemcpyAsync(dscenes.ptr, t, sizeof(SceneParams) * kMaxScenes, cudaMemcpyHostToDevice, stream);
    }

    // Device ranges after a re-sort: live scenes in id order, each contiguous.
    void assign_offsets() {
        size_t off = 0;
        for (BatchScene &s : scenes) {
            if (s.draining) s.draining = false;  // rows dropped by this re-sort: id free again
            if (!s.live) continue;
            s.dev_offset = off;
            off += s.dev_count;
        }
        n_phys = n_live;
    }

    // Copy scene `id`'s staged rows to rows [n_phys, n_phys + m) of the
    // buffer the next batch re-sorts from, and clear its failure word, on `st`.
    // Host-to-device copies of (device destination, host source, bytes)
    // pieces on `st` through the pinned staging buffers; pageable copies when
    // pinned memory cannot be had.  Returns once every host source has been
    // read (the device side may still be copying).
    struct CopyPiece {
        void *dst;
        const void *src;
        size_t bytes;
    };
    // Admission copies run on a worker thread, so that the thread admitting
    // scenes returns at once (the copies overlap the batch in flight and the
    // caller's own work); the next submit waits for them (join_uploads).
    struct UploadJob {
        std::vector<CopyPiece> pieces;
        size_t id;
    };
    std::thread upload_worker;
    std::mutex up_mu;
    std::condition_variable up_cv;
    std::deque<UploadJob> up_jobs;
    bool up_busy = false, up_stop = false;
    cudaError_t up_error = cudaSuccess;

    void upload_loop() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(up_mu);
        for (;;) {
            up_cv.wait(lk, [&] { return up_stop || !up_jobs.empty(); });
            if (up_jobs.empty()) return;  // stopping with nothing left
            UploadJob job = std::move(up_jobs.front());
            up_jobs.pop_front();
            up_busy = true;
            lk.unlock();
            cudaError_t e = copy_h2d(job.pieces, upload_stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(scene_status.ptr + job.id, 0, sizeof(uint32_t), upload_stream);
            lk.lock();
            if (e != cudaSuccess && up_error == cudaSuccess) up_error = e;
            up_busy = false;
            up_cv.notify_all();
        }
    }

    // Wait until the worker has issued every queued copy; its first error.
    cudaError_t drain_uploads() {
        std::unique_lock<std::mutex> lk(up_mu);
        up_cv.wait(lk, [&] { return up_jobs.empty() && !up_busy; });
        const cudaError_t e = up_error;
        up_error = cudaSuccess;
        return e;
    }
    cudaError_t copy_h2d(const std::vector<CopyPiece> &pieces, cudaStream_t st) {
        cudaError_t e;
        bool pinned = true;
        for (int k = 0; k < 2 && pinned; ++k) {
            if (!stage_free[k] && cudaEventCreateWithFlags(&stage_free[k], cudaEventDisableTiming) != cudaSuccess) {
                stage_free[k] = nullptr;
                pinned = false;
            }
            if (pinned && !stage[k].ensure(kStageBytes)) pinned = false;
        }
        if (!pinned) {
            cudaGetLastError();
            for (const CopyPiece &c : pieces)
                if ((e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, st))) return e;
            return cudaSuccess;
        }
        int b = 0;
        size_t fill = 0;
        // pieces packed into stage[b]: src = host source, dst = device destination,
        // bytes; staged at offset `at`
        struct Staged {
            CopyPiece c;
            size_t at;
        };
        std::vector<Staged> queued;
        auto wait_free = [&](int k) -> cudaError_t {
            if (!stage_busy[k]) return cudaSuccess;
            stage_busy[k] = false;
            return cudaEventSynchronize(stage_free[k]);
        };
        // fill stage[b] from the host sources (one parallel pass over its bytes),
        // queue the copies out of it and move to the other buffer
        auto flush = [&]() -> cudaError_t {
            char *base = static_cast<char *>(stage[b].ptr);
            parallel_chunks(fill, [&](size_t, size_t lo, size_t hi) {
                for (const Staged &q : queued) {
                    const size_t a = std::max(lo, q.at), z = std::min(hi, q.at + q.c.bytes);
                    if (a < z) std::memcpy(base + a, static_cast<const char *>(q.c.src) + (a - q.at), z - a);
                }
            }, size_t(4) << 20);
            cudaError_t err;
            for (const Staged &q : queued)
                if ((err = cudaMemcpyAsync(q.c.dst, base + q.at, q.c.bytes, cudaMemcpyHostToDevice, st))) return err;
            queued.clear();
            if ((err = cudaEventRecord(stage_free[b], st))) return err;
            stage_busy[b] = true;
            b ^= 1;
            fill = 0;
            return wait_free(b);
        };
        if ((e = wait_free(b))) return e;
        for (const CopyPiece &c : pieces) {
            size_t done = 0;
            while (done < c.bytes) {
                if (fill == kStageBytes && (e = flush())) return e;
                const size_t n = std::min(c.bytes - done, kStageBytes - fill);
                queued.push_back({{static_cast<char *>(c.dst) + done, static_cast<const char *>(c.src) + done, n}, fill});
                fill += n;
                done += n;
            }
        }
        if (!queued.empty() && (e = flush())) return e;
        return cudaSuccess;
    }

    // The copies that put scene `id`'s staged rows at rows [n_phys, n_phys + m)
    // of the buffer the next batch re-sorts from; assigns those rows.
    std::vector<CopyPiece> scene_pieces(size_t id) {
        TmpmPreparedScene &p = *scenes[id].staged;
        const size_t m = p.m, stride = std::max<size_t>(m, 1);
        const size_t pc = pbuf[cur].cap;
        const ParticleBuffers &pb = pbuf[cur];
        std::vector<CopyPiece> pieces;
        if (m) {
            const float *hb = row_base(p.rows);
            auto rows = [&](float *dst, int first, int count) {
                for (int r = 0; r < count; ++r)
                    pieces.push_back({dst + r * pc + n_phys, hb + (first + r) * stride, m * 4});
            };
            rows(pb.x.ptr, 0, 3);
            rows(pb.v.ptr, 3, 3);
            rows(pb.C.ptr, 6, 9);
            rows(pb.F.ptr, 15, 9);
            rows(pb.pl.ptr, 24, 3);
            pieces.push_back({pb.cls.ptr + n_phys, row_cls(p.rows, stride), m * 4});
            pieces.push_back({pb.widx.ptr + n_phys, row_widx(p.rows, stride), m * 4});
        }
        scenes[id].dev_offset = n_phys;
        n_phys += m;
        return pieces;
    }

    // Scene `id`'s staged rows to the device on `st` (see scene_pieces).
    cudaError_t copy_scene_rows(size_t id, cudaStream_t st) {
        const cudaError_t e = copy_h2d(scene_pieces(id), st);
        if (e != cudaSuccess) return e;
        return cudaMemsetAsync(scene_status.ptr + id, 0, sizeof(uint32_t), st);
    }

    // Copy an admitted scene's rows now, on the upload stream, if the
    // allocated rows have room: rows from n_phys on in the buffer the next
    // batch re-sorts from are free (a batch in flight writes only the first
    // n_phys rows of it), so the copy overlaps that batch.  Without room the
    // rows stay staged and the next submit grows the buffers and copies them.
    TmpmStatus upload_early(size_t id) {
        if (n_phys + scenes[id].staged->m > pbuf[cur].cap) return TMPM_OK;
        UploadJob job{scene_pieces(id), id};
        if (!upload_worker.joinable()) upload_worker = std::thread([this] { upload_loop(); });
        {
            std::lock_guard<std::mutex> lk(up_mu);
            up_jobs.push_back(std::move(job));
        }
        up_cv.notify_all();
        early_uploads.push_back(std::move(scenes[id].staged));  // rows stay alive until the copies are done
        uploads_open = true;
        return TMPM_OK;
    }

    // Order the batch stream after the copies admission issued.
    TmpmStatus join_uploads() {
        if (!uploads_open) return TMPM_OK;
        cudaError_t e;
        if ((e = drain_uploads())) return cuda_fail(e, "scene upload");
        if ((e = cudaEventRecord(upload_done, upload_stream)) || (e = cudaStreamWaitEvent(stream, upload_done, 0)))
            return cuda_fail(e, "scene upload");
        for (auto &p : early_uploads) in_flight_uploads.push_back(std::move(p));
        early_uploads.clear();
        uploads_open = false;
        return TMPM_OK;
    }

    // Copy the rows of admitted scenes still staged to the device (appended
    // after the resident rows), upload the class table and size the grid.
    // Idle only; the packed rows stay alive until the batch that follows
    // completes.
    TmpmStatus commit_staged() {
        TmpmStatus st;
        if ((st = join_uploads()) != TMPM_OK) return st;
        size_t add = 0;
        for (BatchScene &s : scenes)
            if (s.live && s.staged) add += s.staged->m;
        bool any = false;
        for (BatchScene &s : scenes) any = any || (s.live && s.staged);
        if (any && (st = ensure_rows(n_phys + add)) != TMPM_OK) return st;
        if ((st = upload_classes()) != TMPM_OK) return st;
        if ((st = ensure_grid()) != TMPM_OK) return st;
        if (!any) return TMPM_OK;
        cudaError_t e;
        for (size_t id = 0; id < scenes.size(); ++id) {
            BatchScene &s = scenes[id];
            if (!s.live || !s.staged) continue;
            if ((e = copy_scene_rows(id, stream))) return cuda_fail(e, "scene upload");
            in_flight_uploads.push_back(std::move(s.staged));
        }
        return TMPM_OK;
    }

    // The kernels of one batch of `steps` substeps (captured into a graph or launched directly).
    void launch_batch(uint32_t steps, int config) {
        SimParams sp = sim_params();
        sp.shape = config_shape(config);
        const int bs = config_block_shift(config);
        sp.block_shift = bs;
        ParticleSoA src = pbuf[cur].view(nullptr, 1), dst = pbuf[cur ^ 1].view(nullptr, 1);
        SortBuffers sb = sort_buffers();
        launch_resort(src, dst, static_cast<int>(n_phys), static_cast<int>(n_live), dclasses.ptr, sp, sb, stream);
        GridTable g[2];
        g[0] = grids[0].view(bs);
        g[1] = g[0];
        g[1].pool = grids[1].pool.ptr;
        const int n = static_cast<int>(n_live);
        launch_clear_table(g[0], g[1], bs, stream);
        // the fused transfer's deferred-chunk lists (as in a session): emptied
        // before the opening P2G, then by each grid update for its transfer
        sp.defer = defer.ptr;
        sp.defer_cap = static_cast<int>(defer.count >= static_cast<size_t>(kDeferHeader)
                                            ? (defer.count - kDeferHeader) / 4
                                            : 0);
        if (sp.defer) cudaMemsetAsync(sp.defer, 0, sizeof(uint32_t) * kDeferHeader, stream);
        SimParams sp0 = sp;
        sp0.step_index = -1;
        launch_transfer(kModeP2G, dst, n, dclasses.ptr, g[1], g[0], sp0, nullptr, nullptr, nullptr, status.ptr,
                        cta_cache.ptr, stream);
        for (uint32_t s = 0; s < steps; ++s) {
            const GridTable &gc = g[s & 1], &gn = g[(s + 1) & 1];
            SimParams spk = sp;
            spk.step_index = static_cast<int>(s);
            launch_grid_update(gc, gn, spk, nullptr, nullptr, nullptr, status.ptr, stream);
            launch_transfer(s + 1 == steps ? kModeG2P : kModeG2P2G, dst, n, dclasses.ptr, gc, gn, spk, nullptr,
                            nullptr, nullptr, status.ptr, cta_cache.ptr, stream, &fj);
        }
    }

    TmpmStatus enqueue(uint32_t steps) {
        cudaError_t e;
        TmpmStatus st;
        if ((st = commit_staged()) != TMPM_OK) return st;
        if ((e = upload_table())) return cuda_fail(e, "scene table upload");
        if ((e = cudaEventRecord(t_begin, stream))) return cuda_fail(e, "cudaEventRecord");
        for (BatchScene &s : scenes)
            if (s.live) s.prev_offset = s.dev_offset;
        prev_buf = cur;
        if (n_phys > 0) {
            // Plastic classes run the default shape only.
            const bool tunable = !classes.plastic();
            const int config = tunable ? tuner.config(big_blocks_ok, true) : 0;
            const double work = static_cast<double>(n_live) * steps;
            if (options.use_graphs) {
                GraphKey key{steps, n_phys, n_live, cur, epoch, config};
                auto it = graphs.find(key);
                if (it == graphs.end()) {
                    if (graphs.size() > 16) drop_graphs();
                    cudaGraph_t graph = nullptr;
                    if ((e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal)))
                        return cuda_fail(e, "cudaStreamBeginCapture");
                    launch_batch(steps, config);
                    if ((e = cudaStreamEndCapture(stream, &graph))) return cuda_fail(e, "cudaStreamEndCapture");
                    cudaGraphExec_t exec = nullptr;
                    e = cudaGraphInstantiate(&exec, graph, 0);
                    cudaGraphDestroy(graph);
                    if (e) return cuda_fail(e, "cudaGraphInstantiate");
                    it = graphs.emplace(key, exec).first;
                }
                if (tunable) tuner.begin(config, stream);
                if ((e = cudaGraphLaunch(it->second, stream))) return cuda_fail(e, "cudaGraphLaunch");
            } else {
                if (tunable) tuner.begin(config, stream);
                launch_batch(steps, config);
            }
            if (tunable) tuner.end(work, stream);
            cur ^= 1;
        }
        assign_offsets();
        if ((e = cudaEventRecord(t_end, stream))) return cuda_fail(e, "cudaEventRecord");
        if ((e = cudaGetLastError())) return cuda_fail(e, "kernel launch");
        return TMPM_OK;
    }
    int prev_buf = 0;  // row buffer the batch in flight re-sorts from (and only reads)

    // Host staging for a read of `m` rows: the pinned buffer (grown by half
    // again when too small), else pageable memory.
    float *read_staging(size_t floats) {
        const size_t bytes = std::max<size_t>(floats, 1) * sizeof(float);
        if (read_pinned.bytes >= bytes || read_pinned.ensure(std::max(bytes, read_pinned.bytes + read_pinned.bytes / 2)))
            return static_cast<float *>(read_pinned.ptr);
        read_pageable.resize(std::max<size_t>(floats, 1));
        return read_pageable.data();
    }

    // Put a scene's rows (m stored rows at row `off` of row buffer `buf`) in
    // world order on the device (27 f32 rows of stride N = its world count;
    // rows of disabled particles are left unwritten), copy them into `h` on
    // `st`, and wait: the host then applies them front to back instead of
    // scattering by world index.
    TmpmStatus read_rows(BatchScene &s, int buf, size_t off, cudaStream_t st, float *h) {
        const size_t m = s.dev_count, N = s.world.n;
        if (!m) return TMPM_OK;
        cudaError_t e;
        if (read_unsorted.count < 27 * N && (e = read_unsorted.alloc(27 * N))) return cuda_fail(e, "cudaMalloc readback");
        ParticleSoA P = pbuf[buf].view(nullptr, 1);
        P.x += off;
        P.v += off;
        P.C += off;
        P.F += off;
        P.pl += off;
        P.cls += off;
        P.widx += off;
        launch_unsort(P, static_cast<int>(m), read_unsorted.ptr, N, st);
        if ((e = cudaMemcpyAsync(h, read_unsorted.ptr, sizeof(float) * 27 * N, cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            return cuda_fail(e, "scene readback");
        return TMPM_OK;
    }

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
                return fail(TMPM_ERR_READBACK, "timed out waiting for the batch");
            }
            std::this_thread::sleep_for(std::chrono::microseconds(el < 0.01 ? 20 : 200));
        }
    }

    TmpmStatus synchronize() {
        if (!valid) return fail(TMPM_ERR_RESIDENT_UNAVAILABLE, "batch is invalid after an earlier error");
        if (!pending) return TMPM_OK;
        pending = false;
        TmpmStatus st = wait_done();
        if (st != TMPM_OK) return st;
        in_flight_uploads.clear();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t_begin, t_end);
        last_ms = ms;
        std::vector<uint32_t> flags(kMaxScenes + 1, 0);
        cudaError_t e;
        if ((e = cudaMemcpy(flags.data(), status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost)) ||
            (e = cudaMemcpy(flags.data() + 1, scene_status.ptr, sizeof(uint32_t) * kMaxScenes, cudaMemcpyDeviceToHost)))
            return cuda_fail(e, "status readback");
        if (flags[0] & kStatusCapacity) {
            valid = false;
            return fail(TMPM_ERR_CAPACITY, "GPU MPM batch exceeds the device capacity (grid block pool or hash table)");
        }
        if (flags[0] & kStatusTimeout) {
            valid = false;
            return fail(TMPM_ERR_READBACK, "a bounded device wait gave up");
        }
        for (size_t id = 0; id < scenes.size(); ++id) {
            BatchScene &s = scenes[id];
            if (!s.live || s.queued == 0) continue;
            if (flags[1 + id] & kStatusResident) {
                if (s.status == TMPM_OK) {
                    s.status = TMPM_ERR_RESIDENT_UNAVAILABLE;
                    s.error = "GPU MPM resident substeps require a CPU fallback; scene state is the last one read";
                }
            } else if (s.status == TMPM_OK) {
                s.substeps += s.queued;
                s.stale = true;
            }
            s.queued = 0;
        }
        return TMPM_OK;
    }

    // Apply world-order rows (27 f32 rows of stride N, as read_rows leaves
    // them) to a scene's host world (collect_prepared + apply_gpu_transfers,
    // gpu.rs:1821-1989, 2295-2329): a non-finite value of an enabled particle
    // fails the scene before anything is applied; fixed particles keep their
    // position and get zero velocity and affine field.
    TmpmStatus apply_rows(BatchScene &s, const float *h) {
        HostWorld &w = s.world;
        const size_t N = w.n;
        if (!s.dev_count) return TMPM_OK;
        std::atomic<bool> bad{false};
        parallel_for(N, [&](size_t a, size_t b) {
            for (size_t c = 0; c < 27 && !bad.load(std::memory_order_relaxed); ++c)
                for (size_t i = a; i < b; ++i)
                    if (w.enabled[i] && !std::isfinite(h[c * N + i])) {
                        bad = true;
                        break;
                    }
        });
        if (bad) {
            s.status = TMPM_ERR_NON_FINITE_STATE;
            s.error = "MPM integration produced a non-finite state";
            return s.status;
        }
        ++w.version;
        parallel_for(N, [&](size_t a, size_t b) {
            for (size_t i = a; i < b; ++i) {
                if (!w.enabled[i]) continue;
                if (w.fixed[i]) {
                    for (int k = 0; k < 3; ++k) w.vel[3 * i + k] = 0.0;
                    for (int k = 0; k < 9; ++k) w.C[9 * i + k] = 0.0;
                    continue;
                }
                for (int k = 0; k < 3; ++k) {
                    w.pos[3 * i + k] = h[(0 + k) * N + i];
                    w.vel[3 * i + k] = h[(3 + k) * N + i];
                }
                for (int k = 0; k < 9; ++k) {
                    w.C[9 * i + k] = h[(6 + k) * N + i];
                    w.F[9 * i + k] = h[(15 + k) * N + i];
                }
                const int mat = w.material[i];
                if (mat == TMPM_MAT_SAND || mat == TMPM_MAT_SNOW || mat == TMPM_MAT_SAND_NEO_HOOKEAN)
                    for (int k = 0; k < 3; ++k) w.plastic[3 * i + k] = h[(24 + k) * N + i];
            }
        });
        return TMPM_OK;
    }

    // Bring a scene's host world up to date from the device: from the current
    // rows when idle; while a batch runs, for a scene that batch does not
    // advance, from the buffer the batch re-sorts from, on the side stream.
    TmpmStatus refresh(BatchScene &s) {
        if (pending && s.queued) return fail(TMPM_ERR_PENDING_STEPS, "the scene is in the batch in flight");
        if (!s.stale) return TMPM_OK;
        TmpmStatus st;
        float *h = read_staging(27 * s.world.n);
        if (pending) {
            st = read_rows(s, prev_buf, s.prev_offset, read_stream, h);
        } else {
            st = read_rows(s, cur, s.dev_offset, stream, h);
        }
        if (st != TMPM_OK) return st;
        st = apply_rows(s, h);
        s.stale = false;
        return st;
    }

    int free_id() const {
        for (size_t id = 0; id < scenes.size(); ++id)
            if (!scenes[id].live && !scenes[id].draining) return static_cast<int>(id);
        return scenes.size() < static_cast<size_t>(kMaxScenes) ? static_cast<int>(scenes.size()) : -1;
    }

    // Attach a prepared scene (allowed while a batch is in flight: host work only).
    TmpmStatus admit(std::unique_ptr<TmpmPreparedScene> p, uint32_t *id_out) {
        int id = free_id();
        if (id < 0 && !pending && n_phys != n_live) {
            TmpmStatus st = compact();
            if (st != TMPM_OK) return st;
            id = free_id();
        }
        if (id < 0) return fail(TMPM_ERR_CAPACITY, "a batch holds at most 256 live scenes");
        if (n_live + p->m > static_cast<size_t>(std::numeric_limits<int>::max() / 2))
            return fail(TMPM_ERR_CAPACITY, "too many particles for one batch");
        // classes into the batch table, in this scene's grid namespace
        std::vector<uint32_t> remap(p->classes.table.size());
        const size_t before = classes.table.size();
        for (size_t k = 0; k < remap.size(); ++k) {
            DevClass c = p->classes.table[k];
            c.color |= static_cast<uint32_t>(id) << kSceneShift;
            remap[k] = classes.intern(c);
        }
        if (classes.table.size() > kClassMask) {
            classes.table.resize(before);
            for (auto it = classes.index.begin(); it != classes.index.end();)
                it = it->second >= before ? classes.index.erase(it) : std::next(it);
            return fail(TMPM_ERR_CAPACITY, "too many distinct particle classes");
        }
        const size_t stride = std::max<size_t>(p->m, 1);
        uint32_t *cls = row_cls(p->rows, stride);
        parallel_for(p->m, [&](size_t a, size_t b) {
            for (size_t j = a; j < b; ++j) cls[j] = remap[cls[j] & kClassMask] | (cls[j] & kFixedBit);
        });
        BatchScene sc;
        sc.live = true;
        sc.params = p->params;
        sc.dt = p->dt;
        sc.dev_count = p->m;
        sc.blocks = p->blocks;
        sc.blocks8 = p->blocks8;
        sc.world = std::move(p->world);
        sc.staged = std::move(p);
        if (static_cast<size_t>(id) == scenes.size()) scenes.emplace_back();
        scenes[id] = std::move(sc);
        n_live += scenes[id].dev_count;
        if (id_out) *id_out = static_cast<uint32_t>(id);
        return upload_early(static_cast<size_t>(id));
    }

    // The scene's state into the non-null fields of `out`, then its removal
    // (a server's retire step).  When the device holds newer state than the
    // host world, only the requested per-particle rows cross to the host, in
    // world order, and go straight into `out`; the host world is not updated,
    // since the scene goes.  The non-finite check covers every transferred
    // component, on the device (collect_prepared, gpu.rs:1940-1989); a
    // non-finite state fails the scene and keeps it, like a read.
    TmpmStatus take(uint32_t id, const TmpmParticleArrays &out) {
        BatchScene &s = scenes[id];
        if (pending && s.queued) return fail(TMPM_ERR_PENDING_STEPS, "the scene is in the batch in flight");
        HostWorld &w = s.world;
        if (!s.stale || !s.dev_count) {
            w.store(const_cast<TmpmParticleArrays &>(out));
            return remove(id);
        }
        const size_t m = s.dev_count, N = w.n;
        // device components: position 0-2, velocity 3-5, affine 6-14, deformation 15-23, plastic 24-26
        double *const dst[5] = {out.position, out.velocity, out.affine, out.deformation, out.plastic};
        const int first[5] = {0, 3, 6, 15, 24}, width[5] = {3, 3, 9, 9, 3};
        int at[5], rows = 0;
        for (int f = 0; f < 5; ++f) {
            at[f] = rows;
            if (dst[f]) rows += width[f];
        }
        cudaStream_t st = pending ? read_stream : stream;
        ParticleSoA P = pbuf[pending ? prev_buf : cur].view(nullptr, 1);
        const size_t off = pending ? s.prev_offset : s.dev_offset;
        P.x += off;
        P.v += off;
        P.C += off;
        P.F += off;
        P.pl += off;
        P.cls += off;
        P.widx += off;
        cudaError_t e;
        if (read_unsorted.count < 27 * N && (e = read_unsorted.alloc(27 * N))) return cuda_fail(e, "cudaMalloc readback");
        if (!take_flag.count && (e = take_flag.alloc(1))) return cuda_fail(e, "cudaMalloc readback");
        float *h = read_staging(static_cast<size_t>(rows) * N + 1);
        uint32_t *hflag = reinterpret_cast<uint32_t *>(h + static_cast<size_t>(rows) * N);
        if ((e = cudaMemsetAsync(take_flag.ptr, 0, sizeof(uint32_t), st))) return cuda_fail(e, "scene readback");
        launch_unsort(P, static_cast<int>(m), read_unsorted.ptr, N, st, take_flag.ptr);
        for (int f = 0; f < 5; ++f)
            if (dst[f] && (e = cudaMemcpyAsync(h + static_cast<size_t>(at[f]) * N, read_unsorted.ptr + first[f] * N,
                                               sizeof(float) * width[f] * N, cudaMemcpyDeviceToHost, st)))
                return cuda_fail(e, "scene readback");
        if ((e = cudaMemcpyAsync(hflag, take_flag.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) ||
            (e = cudaStreamSynchronize(st)))
            return cuda_fail(e, "scene readback");
        if (*hflag) {
            s.status = TMPM_ERR_NON_FINITE_STATE;
            s.error = "MPM integration produced a non-finite state";
            return s.status;
        }
        // fields the device does not hold come from the host world
        TmpmParticleArrays rest = out;
        rest.position = rest.velocity = rest.affine = rest.deformation = rest.plastic = nullptr;
        w.store(rest);
        parallel_for(N, [&](size_t a, size_t b) {
            for (size_t i = a; i < b; ++i) {
                const bool dev = w.enabled[i] && !w.fixed[i];
                const int mat = w.material[i];
                const bool plastic = mat == TMPM_MAT_SAND || mat == TMPM_MAT_SNOW || mat == TMPM_MAT_SAND_NEO_HOOKEAN;
                for (int f = 0; f < 5; ++f) {
                    if (!dst[f]) continue;
                    const int k = width[f];
                    double *d = dst[f] + k * i;
                    const float *src = h + static_cast<size_t>(at[f]) * N + i;
                    if (dev && (f != 4 || plastic)) {
                        for (int c = 0; c < k; ++c) d[c] = src[c * N];
                    } else if (w.enabled[i] && (f == 1 || f == 2)) {
                        for (int c = 0; c < k; ++c) d[c] = 0.0;  // fixed: zero velocity and affine field
                    } else {
                        const double *hw = f == 0 ? w.pos.data() : f == 1 ? w.vel.data() : f == 2 ? w.C.data()
                                         : f == 3 ? w.F.data() : w.plastic.data();
                        for (int c = 0; c < k; ++c) d[c] = hw[k * i + c];
                    }
                }
            }
        });
        return remove(id);
    }

    TmpmStatus remove(uint32_t id) {
        BatchScene *s = scene_at(id);
        if (!s) return fail(TMPM_ERR_INVALID_INPUT, "unknown scene id");
        n_live -= s->dev_count;
        const bool had_rows = !s->staged;
        scenes[id] = BatchScene();
        scenes[id].draining = had_rows;  // rows on the device go at the next re-sort
        return TMPM_OK;
    }

    // Drop the rows of removed scenes now (a re-sort without substeps).  Idle only.
    TmpmStatus compact() {
        for (BatchScene &s : scenes) s.queued = 0;
        // rows copied at admission take part in the re-sort: their copies and classes first
        TmpmStatus st;
        if ((st = join_uploads()) != TMPM_OK || (st = upload_classes()) != TMPM_OK) return st;
        cudaError_t e;
        if ((e = upload_table())) return cuda_fail(e, "scene table upload");
        if (n_phys) {
            SimParams sp = sim_params();
            ParticleSoA src = pbuf[cur].view(nullptr, 1), dst = pbuf[cur ^ 1].view(nullptr, 1);
            SortBuffers sb = sort_buffers();
            launch_resort(src, dst, static_cast<int>(n_phys), static_cast<int>(n_live_committed()), dclasses.ptr, sp, sb,
                          stream);
            cur ^= 1;
        }
        // rows of live committed scenes now lead, in id order; staged scenes follow at commit
        size_t off = 0;
        for (BatchScene &s : scenes) {
            if (s.draining) s.draining = false;
            if (!s.live || s.staged) continue;
            s.dev_offset = off;
            off += s.dev_count;
        }
        n_phys = off;
        if ((e = cudaStreamSynchronize(stream))) return cuda_fail(e, "compact");
        return TMPM_OK;
    }

    size_t n_live_committed() const {
        size_t n = 0;
        for (const BatchScene &s : scenes)
            if (s.live && !s.staged) n += s.dev_count;
        return n;
    }

    size_t device_bytes() const {
        size_t b = 0;
        for (int k = 0; k < 2; ++k) b += pbuf[k].cap * (27 * 4 + 2 * 4);
        b += (sort_keys[0].count + sort_keys[1].count + sort_vals[0].count + sort_vals[1].count + sort_hist.count) * 4;
        for (int g = 0; g < 2; ++g)
            b += grids[g].pool_nodes * 16 + static_cast<size_t>(grids[g].max_blocks) * 16 +
                 static_cast<size_t>(grids[g].capacity) * 12;
        b += (cta_cache.count + defer.count) * 4 + dclasses.count * sizeof(DevClass) +
             kMaxScenes * (sizeof(SceneParams) + 4);
        b += read_unsorted.count * 4;
        return b;
    }
};

extern "C" {

TmpmStatus tmpm_scene_prepare(const TmpmParams *params, const TmpmParticleArrays *particles, double substep_dt,
                              TmpmPreparedScene **out) {
    if (!out || !params) {
        g_last_error = "null argument";
        return TMPM_ERR_INVALID_INPUT;
    }
    *out = nullptr;
    auto p = std::make_unique<TmpmPreparedScene>();
    TmpmStatus st = prepare_scene(*params, particles, substep_dt, *p);
    if (st != TMPM_OK) return st;
    *out = p.release();
    return TMPM_OK;
}

void tmpm_scene_prepared_destroy(TmpmPreparedScene *p) { delete p; }

size_t tmpm_scene_prepared_particle_count(const TmpmPreparedScene *p) { return p ? p->world.n : 0; }

size_t tmpm_scene_prepared_bytes(const TmpmPreparedScene *p) {
    if (!p) return 0;
    // the pool share as pool_plan sizes it: 4^3 blocks, or 8^3 when they fit in twice the nodes
    const size_t nodes4 = 16 * p->blocks * kNodesPerBlock, nodes8 = 16 * p->blocks8 * kBigNodesPerBlock;
    const size_t extra = nodes8 <= 2 * nodes4 && nodes8 > nodes4 ? 2 * (nodes8 - nodes4) * 16 : 0;
    return p->m * kBytesPerRow + 16 * p->blocks * kBytesPerPoolBlock + extra;
}

// Reads of finished scenes run beside the batch in flight; at the highest
// stream priority their small un-sort kernel is scheduled ahead of the
// batch's queued CTAs instead of waiting for them.
static cudaError_t create_read_stream(cudaStream_t *s) {
    int least = 0, greatest = 0;
    cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e != cudaSuccess) return e;
    return cudaStreamCreateWithPriority(s, cudaStreamNonBlocking, greatest);
}

TmpmStatus tmpm_batch_create(const TmpmBatchOptions *options, TmpmBatch **out) {
    if (!out) {
        g_last_error = "null argument";
        return TMPM_ERR_INVALID_INPUT;
    }
    *out = nullptr;
    auto b = std::make_unique<TmpmBatch>();
    if (options) b->options = *options;
    else b->options.use_graphs = 1;
    b->device = b->options.device;
    b->tuner.reset(b->options.launch_shape);
    cudaError_t e;
    if ((e = cudaSetDevice(b->device)) || (e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) ||
        (e = create_read_stream(&b->read_stream)) ||
        (e = cudaStreamCreateWithFlags(&b->upload_stream, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&b->upload_done, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming)) || (e = cudaEventCreate(&b->t_begin)) ||
        (e = cudaStreamCreateWithFlags(&b->fj.side, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&b->fj.fork, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&b->fj.join, cudaEventDisableTiming)) ||
        (e = cudaEventCreate(&b->t_end)) || (e = b->status.alloc(1)) || (e = b->scene_status.alloc(kMaxScenes)) ||
        (e = b->dscenes.alloc(kMaxScenes))) {
        g_last_error = std::string("batch setup: ") + cudaGetErrorString(e);
        return TMPM_ERR_DEVICE;
    }
    if (!b->table_staging.ensure(sizeof(SceneParams) * kMaxScenes)) {
        g_last_error = "cudaMallocHost scene table failed";
        return TMPM_ERR_DEVICE;
    }
    cudaMemsetAsync(b->status.ptr, 0, sizeof(uint32_t), b->stream);
    cudaMemsetAsync(b->scene_status.ptr, 0, sizeof(uint32_t) * kMaxScenes, b->stream);
    if (b->options.particle_capacity) {
        TmpmStatus st = b->ensure_rows(b->options.particle_capacity);
        if (st != TMPM_OK) return st;
    }
    if (b->options.max_blocks) {
        TmpmStatus st = b->ensure_grid();
        if (st != TMPM_OK) return st;
    }
    if ((e = cudaStreamSynchronize(b->stream))) {
        g_last_error = std::string("batch setup: ") + cudaGetErrorString(e);
        return TMPM_ERR_DEVICE;
    }
    *out = b.release();
    return TMPM_OK;
}

void tmpm_batch_destroy(TmpmBatch *batch) { delete batch; }

TmpmStatus tmpm_batch_admit(TmpmBatch *b, TmpmPreparedScene *prepared, uint32_t *scene_out) {
    if (!b || !prepared) {
        g_last_error = "null argument";
        if (prepared) delete prepared;
        return TMPM_ERR_INVALID_INPUT;
    }
    std::unique_ptr<TmpmPreparedScene> p(prepared);
    TmpmStatus st = b->guard(false);
    if (st != TMPM_OK) return st;
    cudaSetDevice(b->device);
    return b->admit(std::move(p), scene_out);
}

TmpmStatus tmpm_batch_add_scene(TmpmBatch *b, const TmpmParams *params, const TmpmParticleArrays *particles,
                                double substep_dt, uint32_t *scene_out) {
    if (!b || !params) {
        g_last_error = "null argument";
        return TMPM_ERR_INVALID_INPUT;
    }
    TmpmStatus st = b->guard(false);
    if (st != TMPM_OK) return st;
    auto p = std::make_unique<TmpmPreparedScene>();
    st = prepare_scene(*params, particles, substep_dt, *p);
    if (st != TMPM_OK) return b->fail(st, g_last_error);
    cudaSetDevice(b->device);
    return b->admit(std::move(p), scene_out);
}

TmpmStatus tmpm_batch_take_scene(TmpmBatch *b, uint32_t scene, TmpmParticleArrays *out) {
    if (!b || !out) return TMPM_ERR_INVALID_INPUT;
    TmpmStatus st = b->guard(false);
    if (st != TMPM_OK) return st;
    BatchScene *s = b->scene_at(scene);
    if (!s) return b->fail(TMPM_ERR_INVALID_INPUT, "unknown scene id");
    if (s->status != TMPM_OK) return b->fail(s->status, s->error);
    if (out->count != s->world.n) return b->fail(TMPM_ERR_INVALID_INPUT, "output array count does not match the scene");
    cudaSetDevice(b->device);
    st = b->take(scene, *out);
    if (st != TMPM_OK) return b->fail(st, s->error.empty() ? b->last_error : s->error);
    return TMPM_OK;
}

TmpmStatus tmpm_batch_remove_scene(TmpmBatch *b, uint32_t scene) {
    if (!b) return TMPM_ERR_INVALID_INPUT;
    TmpmStatus st = b->guard(false);
    if (st != TMPM_OK) return st;
    return b->remove(scene);
}

TmpmStatus tmpm_batch_submit(TmpmBatch *b, const uint32_t *ids, const uint32_t *steps, size_t count) {
    if (!b) return TMPM_ERR_INVALID_INPUT;
    TmpmStatus st = b->guard(true);
    if (st != TMPM_OK) return st;
    if (count && (!ids || !steps)) return b->fail(TMPM_ERR_INVALID_INPUT, "null scene or step array");
    for (BatchScene &s : b->scenes) s.queued = 0;
    uint32_t S = 0;
    for (size_t k = 0; k < count; ++k) {
        BatchScene *s = b->scene_at(ids[k]);
        if (!s) return b->fail(TMPM_ERR_INVALID_INPUT, "unknown scene id");
        if (s->status != TMPM_OK) return b->fail(s->status, "scene failed earlier: " + s->error);
        if (steps[k] == 0 || steps[k] > 4096) return b->fail(TMPM_ERR_INVALID_INPUT, "substeps per scene must be 1..4096");
        if (s->queued) return b->fail(TMPM_ERR_INVALID_INPUT, "scene listed twice");
        s->queued = steps[k];
        S = std::max(S, steps[k]);
    }
    if (S == 0) return TMPM_OK;
    cudaSetDevice(b->device);
    st = b->enqueue(S);
    if (st != TMPM_OK) return st;
    b->pending = true;
    return TMPM_OK;
}

TmpmStatus tmpm_batch_synchronize(TmpmBatch *b) {
    if (!b) return TMPM_ERR_INVALID_INPUT;
    cudaSetDevice(b->device);
    return b->synchronize();
}

int32_t tmpm_batch_pending(const TmpmBatch *b) { return b && b->pending ? 1 : 0; }

TmpmStatus tmpm_batch_scene_status(const TmpmBatch *b, uint32_t scene) {
    if (!b || scene >= b->scenes.size() || !b->scenes[scene].live) return TMPM_ERR_INVALID_INPUT;
    return b->scenes[scene].status;
}

uint64_t tmpm_batch_scene_substeps(const TmpmBatch *b, uint32_t scene) {
    if (!b || scene >= b->scenes.size() || !b->scenes[scene].live) return 0;
    return b->scenes[scene].substeps;
}

size_t tmpm_batch_scene_particle_count(const TmpmBatch *b, uint32_t scene) {
    if (!b || scene >= b->scenes.size() || !b->scenes[scene].live) return 0;
    return b->scenes[scene].world.n;
}

TmpmStatus tmpm_batch_read_scene(TmpmBatch *b, uint32_t scene, TmpmParticleArrays *out) {
    if (!b || !out) return TMPM_ERR_INVALID_INPUT;
    TmpmStatus st = b->guard(false);
    if (st != TMPM_OK) return st;
    BatchScene *s = b->scene_at(scene);
    if (!s) return b->fail(TMPM_ERR_INVALID_INPUT, "unknown scene id");
    if (s->status != TMPM_OK) return b->fail(s->status, s->error);
    if (out->count != s->world.n) return b->fail(TMPM_ERR_INVALID_INPUT, "output array count does not match the scene");
    cudaSetDevice(b->device);
    st = b->refresh(*s);
    if (st != TMPM_OK) return b->fail(st, s->error.empty() ? b->last_error : s->error);
    s->world.store(*out);
    return TMPM_OK;
}

double tmpm_batch_last_ms(const TmpmBatch *b) { return b ? b->last_ms : 0.0; }

int32_t tmpm_batch_launch_shape(TmpmBatch *b, double *ms_per_unit, size_t count) {
    if (!b) return -1;
    if (b->tuner.tuning()) {
        cudaSetDevice(b->device);
        b->tuner.poll();
    }
    if (ms_per_unit) b->tuner.costs(ms_per_unit, static_cast<uint32_t>(count));
    if (b->classes.plastic()) return 0;  // variants built for the default shape only
    return b->tuner.current(b->big_blocks_ok);  // 8^3 without room: the best 4^3
}

size_t tmpm_batch_device_bytes(const TmpmBatch *b) { return b ? b->device_bytes() : 0; }

size_t tmpm_batch_scene_bytes(size_t particles, size_t home_blocks) {
    return particles * kBytesPerRow + 16 * home_blocks * kBytesPerPoolBlock;
}

const char *tmpm_batch_last_error_message(const TmpmBatch *b) { return b ? b->last_error.c_str() : g_last_error.c_str(); }

}  // extern "C"
