#!/usr/bin/env python3
"""Benchmark of the MLS-MPM substep (tessera-mpm's resident GPU path) on B200.

Workload: the single large scene of the benchmark configurations (~4.05M
particles: weakly compressible fluid column [0,0.4]x[0,0.8]x[0,1] plus three
elastic cubes, h = 2.2/256, 4^3 hashed blocks, dt = 5e-5, separating walls).
One bench step = one submitted batch of 64 substeps (the reference's per-submit
maximum, gpu.rs:303-322) over the whole scene.

  value  device-resident throughput: particle-substeps/s with the state in HBM,
         timed with CUDA events on the session stream (max over ranks).
  e2e    the same metric through the C ABI with host buffers: every step
         uploads the particle state from host arrays, runs 64 substeps and
         reads the state back into host f64 arrays (tmpm_write_particles +
         tmpm_step).
  batched  256 heterogeneous scenes (4k-256k particles, resolution 32-128,
         elastic or fluid, dt = 1e-4, 100 substeps) advanced in one multi-scene
         batch against the same scenes one at a time through single-scene
         sessions: device-timed and end to end (host arrays in, results out).
  serving  Poisson arrivals of dam-break-sized requests (50-400 substeps) into
         the continuous-batching server under a 120 GB footprint budget, against
         the one-scene-at-a-time loop: p50/p99 time-to-result and throughput.
  adjoint  the differentiable rollout (64k-particle corotated block, 256
         substeps, checkpoints every 16): forward and adjoint wall time through
         the C ABI (host arrays in and out).
  obstacle the benchmark scene with a rigid sphere in the flow: per-launch time
         of the fused transfer variant that carries the obstacle contact.

`--impl reference` times the reference's CPU path (its C++ restatement in
oracle/, f64, ordered-map grid) on the host cores for the same workload.
Multi-GPU (--gpus N under torchrun): independent replicas, one scene per rank
("replicas only": a single scene does not shard without a halo exchange).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BATCH = 64
# re-sort per batch: bin keys, 4 radix passes (27-bit keys) x (hist, scan, scatter), gather
RESORT_LAUNCHES = 1 + 4 * 3 + 1
# kernels of one 64-substep segment: re-sort, table clear, opening P2G, then per
# substep the grid update and the fused transfer (k_transfer_fast with the two
# k_transfer_deferred launches beside and after it), the last substep's
# transfer a single G2P launch
SEGMENT_LAUNCHES = RESORT_LAUNCHES + 2 + 4 * (BATCH - 1) + 2
METRIC = "particle-substeps/s"
# the fields a substep changes (--save-state / --load-state)
STATE_FIELDS = ("position", "velocity", "deformation", "affine", "plastic")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tessera", choices=["tessera", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0, help="column footprint scale (1.0 = full config)")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-scenes", type=int, default=256)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-rates", default="50,200,2000", help="comma-separated arrival rates (requests/s)")
    ap.add_argument("--serve-requests", type=int, default=100, help="requests per arrival rate")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-obstacle", action="store_true")
    ap.add_argument("--launch-shape", type=int, default=None,
                    help="fix the single-scene launch shape (index of _native.launch_shapes()) instead of tuning it")
    ap.add_argument("--only", choices=["batched", "serving", "adjoint", "obstacle"],
                    help="run one section alone and print its result (profiling; not the benchmark line)")
    ap.add_argument("--save-state", default=None,
                    help="after the single-scene timing, save the evolved particle state (.npz) for --load-state")
    ap.add_argument("--load-state", default=None,
                    help="start the single scene from a state saved by --save-state (profiling the evolved scene "
                         "with few launches before the captured one; not the benchmark line)")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def allreduce_max(value: float, world: int) -> float:
    from tessera_b200.replicas import Reducer

    return Reducer(world, "cuda").max(value)


def allreduce_sum(value: float, world: int) -> float:
    from tessera_b200.replicas import Reducer

    return Reducer(world, "cuda").sum(value)


def barrier(world: int):
    from tessera_b200.replicas import Reducer

    Reducer(world, "cuda").barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        import threading

        self.lines = []
        self.first = threading.Event()
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return self

        def reader():
            for ln in self.proc.stdout:
                if ln.strip():
                    self.lines.append(ln)
                    self.first.set()
            self.first.set()

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        self.first.wait(timeout=10.0)  # start timing once sampling runs
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(scene_fn, target_seconds=15.0):
    """The oracle (C++ f64 restatement of the reference CPU path) on a bounded
    sample of the workload, one independent copy per host core."""
    from oracle import oracle as O

    sample = scene_fn(scale=0.1)
    threads = os.cpu_count() or 1
    world = O.OracleWorld(sample.params, sample.particles)
    el = world.bench(threads, 1, sample.dt)
    substeps = max(1, int(target_seconds / max(el, 1e-3)))
    el = world.bench(threads, substeps, sample.dt)
    value = threads * sample.particles.count * substeps / el
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{sample.particles.count} particles of the same scene (column footprint x0.1, same h, dt, "
                      f"materials) x {substeps} substeps, {threads} independent copies in parallel, {el:.1f} s"}


def bench_small_configs(target_seconds=5.0) -> dict:
    """The CPU-runnable configurations beside the GPU: the corotated block of
    configuration 1 (h = 1/64, [0.3, 0.6]^3 at 8 per cell; dt = 5e-5, since
    1e-4 is above its CFL bound) through a single-scene session, and both it
    and the 64k-particle block of configuration 5 through the oracle, one
    independent copy per host core."""
    from oracle import oracle as O
    from tessera_b200 import scenes
    from tessera_b200.session import Session

    out = {}
    threads = os.cpu_count() or 1
    for name, sc in (("config1-corotated-block", scenes.elastic_block()), ("config5-corotated-block",
                                                                         scenes.adjoint_block())):
        n = sc.particles.count
        entry = {"particles": n, "dt": sc.dt, "unit": METRIC}
        ses = Session(sc.params, sc.particles, sc.dt)
        for _ in range(3):
            ses.bench_substeps(64)
        ses.synchronize()
        ms, _ = ses.bench_substeps(64 * 8)
        ses.synchronize()
        ses.close()
        entry["gpu"] = n * 64 * 8 / (ms / 1e3)
        world = O.OracleWorld(sc.params, sc.particles)
        el = world.bench(threads, 1, sc.dt)
        substeps = max(1, int(target_seconds / max(el, 1e-3)))
        el = world.bench(threads, substeps, sc.dt)
        entry["cpu"] = {"value": threads * n * substeps / el, "cores": threads, "kind": "port",
                        "sample": f"{substeps} substeps, {threads} independent copies in parallel, {el:.1f} s"}
        out[name] = entry
    return out


def shape_summary(info: dict) -> dict:
    """The tuned transfer launch shape and what each candidate measured."""
    k = info["shape"]
    out = {"tuned": k is not None}
    if k is not None:
        out["particles_per_cta"], out["ctas_per_sm"], out["block_edge"] = info["shapes"][k]
    out["ns_per_particle_substep"] = {f"{t}x{b}/{e}^3": (None if c is None else c * 1e6)
                                      for (t, b, e), c in zip(info["shapes"], info["ms_per_particle_substep"])}
    return out


def bench_batched(count: int) -> dict:
    """256 heterogeneous scenes x 100 substeps: one multi-scene batch against one
    session per scene, on the same device."""
    import torch

    from tessera_b200 import scenes
    from tessera_b200.batch import Batch, PreparedScene
    from tessera_b200.session import Session

    scs = scenes.batch_scenes(count)
    steps = scs[0].substeps
    n = sum(s.particles.count for s in scs)
    work = float(n) * steps
    # batched, end to end: host arrays -> admission -> 100 substeps -> positions/velocities back
    b = Batch()
    b.add_scene(scs[0].params, scs[0].particles, scs[0].dt)  # warm the pinned pool and the context
    b.close()
    torch.cuda.synchronize()
    from concurrent.futures import ThreadPoolExecutor

    t0 = time.perf_counter()
    b = Batch()
    with ThreadPoolExecutor(max_workers=8) as pool:  # preparation is host work, thread-safe
        prepared = list(pool.map(lambda s: PreparedScene(s.params, s.particles, s.dt), scs))
    ids = [b.admit(p) for p in prepared]
    b.run({i: steps for i in ids})
    outs = [b.read(i) for i in ids]
    e2e_batched = time.perf_counter() - t0
    assert all(np.all(np.isfinite(o["position"])) for o in outs)
    # the launch-shape tuner reads its trials (the first six batches) before the timed batches
    for _ in range(16):
        if b.launch_shape()["shape"] is not None:
            break
        b.run({i: steps for i in ids})
    shape_info = b.launch_shape()
    # batched, device-resident: further batches of the same scenes (graph replays)
    dev = []
    for _ in range(3):
        b.run({i: steps for i in ids})
        dev.append(b.last_ms())
    fails = sum(b.status(i) != 0 for i in ids)
    b.close()
    # plain: one scene at a time through a single-scene session each, at the
    # default launch shape (a 100-substep session ends before its tuner would)
    plain_dev = 0.0
    t0 = time.perf_counter()
    for s in scs:
        ses = Session(s.params, s.particles, s.dt, launch_shape=0)
        left = steps
        while left:
            k = min(BATCH, left)
            ms, _ = ses.bench_substeps(k)
            ses.synchronize()
            plain_dev += ms
            left -= k
        ses.read()
        ses.close()
    e2e_plain = time.perf_counter() - t0
    batched_dev = float(np.median(dev))
    return {
        "workload": "config3-heterogeneous-batch", "scenes": count, "particles": n, "substeps": steps, "dt": scs[0].dt,
        "materials": {"elastic": sum(s.info["material"] == "elastic" for s in scs),
                      "fluid": sum(s.info["material"] == "fluid" for s in scs)},
        "batched": {"value": work / (batched_dev / 1e3), "ms_per_batch": batched_dev, "failed_scenes": fails,
                    "e2e": work / e2e_batched, "e2e_seconds": e2e_batched, "graph_replay": True,
                    "launch_shape": shape_summary(shape_info)},
        "plain": {"value": work / (plain_dev / 1e3), "device_ms": plain_dev, "e2e": work / e2e_plain,
                  "e2e_seconds": e2e_plain},
        "speedup_device": plain_dev / batched_dev, "speedup_e2e": e2e_plain / e2e_batched, "unit": METRIC,
        "timing": "value: CUDA events around each batch (plain: sum over sessions of CUDA-event time of their "
                  "substeps); e2e: wall clock from host arrays to positions/velocities back on the host",
    }


def bench_batched_parallel(count: int, world: int, rank: int) -> dict:
    """The heterogeneous batch split across ranks by scene (no data-path
    collective): each rank advances the scenes that placement by device
    footprint assigns to it (largest first onto the least-loaded rank, the same
    on every rank) in its own multi-scene batch; throughput = all ranks' work
    over the slowest rank's device time."""
    import torch

    from tessera_b200 import scenes
    from tessera_b200.batch import Batch, home_blocks, scene_bytes
    from tessera_b200.replicas import my_items

    scs = scenes.batch_scenes(count)
    steps = scs[0].substeps
    sizes = [scene_bytes(s.particles.count, home_blocks(s.particles.position, s.params.cell_width)) for s in scs]
    mine = [scs[k] for k in my_items(sizes, world, rank)]
    b = Batch()
    ids = [b.add_scene(s.params, s.particles, s.dt) for s in mine]
    for _ in range(16):  # the launch-shape trials before the timed batches
        b.run({i: steps for i in ids})
        if b.launch_shape()["shape"] is not None:
            break
    barrier(world)
    torch.cuda.synchronize()
    dev = []
    for _ in range(3):
        b.run({i: steps for i in ids})
        dev.append(b.last_ms())
    fails = sum(b.status(i) != 0 for i in ids)
    b.close()
    ms = allreduce_max(float(np.median(dev)), world)
    work = allreduce_sum(float(sum(s.particles.count for s in mine)) * steps, world)
    fails = int(allreduce_sum(float(fails), world))
    return {"workload": "config3-heterogeneous-batch, scene-parallel", "scenes": count, "ranks": world,
            "placement": "by device footprint, largest first onto the least-loaded rank",
            "scenes_on_rank0": len(mine), "batched": {"value": work / (ms / 1e3), "ms_per_batch": ms,
                                                      "failed_scenes": fails}, "unit": METRIC,
            "timing": "CUDA events around each rank's batch, max over ranks"}


def bench_serving(rates, count: int) -> dict:
    """Poisson arrivals of dam-break requests (50-400 substeps) into the
    continuous-batching server (120 GB budget), one run per arrival rate, and
    the one-scene-at-a-time loop once (every listed rate saturates one GPU, so
    the plain loop's throughput does not depend on the rate; it runs on the
    first rate's arrivals)."""
    from tessera_b200 import scenes
    from tessera_b200.batch import Batch
    from tessera_b200.serve import Request, Server, poisson_arrivals, run_plain, summarize

    pool = [scenes.dam_break(seed=100 + k) for k in range(4)]  # distinct seeded cube positions
    rng = np.random.default_rng(7)
    steps = [int(rng.integers(50, 401)) for _ in range(count)]
    out = {"workload": "config4-serving", "requests_per_rate": count, "scene": "config2 dam break (4 seeded variants)",
           "particles_per_request": pool[0].particles.count, "substeps": "uniform 50-400 (seeded)",
           "hbm_budget_gb": 120, "chunk_substeps": 32, "unit": METRIC, "rates": []}

    def requests(rate):
        t = poisson_arrivals(rate, count, seed=int(rate))
        return [Request(k, float(t[k] - t[0]), pool[k % len(pool)], steps[k]) for k in range(count)]

    offered = float(sum(pool[k % len(pool)].particles.count * steps[k] for k in range(count)))
    for rate in rates:
        reqs = requests(rate)
        # rows for the scenes the 120 GB budget can hold at once (the batch grows on demand beyond)
        cap = min(sum(r.scene.particles.count for r in reqs), 60 * pool[0].particles.count)
        server = Server(batch=Batch(particle_capacity=cap), chunk=32, hbm_budget=120e9)
        served, span = server.run(reqs)
        s_served = summarize(served, span)
        s_served.update(batches=server.batches, peak_resident=server.peak_resident,
                        peak_gb=server.peak_bytes / 1e9, launch_shape=shape_summary(server.batch.launch_shape()),
                        offered_particle_substeps_per_s=offered / max(reqs[-1].arrival, 1e-9))
        tm = dict(server.timing)
        prep = tm.pop("prepare_s")
        tm.update(prepare_mean_s=float(np.mean(prep)) if prep else None, prepare_max_s=max(prep) if prep else None)
        s_served["timing"] = tm
        server.batch.close()
        out["rates"].append({"rate": rate, "served": s_served})
    # the plain loop is host-bound at ~0.7 G particle-substeps/s (a session per
    # request: upload, substeps, readback), so it runs the first half of the
    # requests; its throughput does not depend on how many it runs
    plain_n = max(1, count // 2)
    plain, span_p = run_plain(requests(rates[0])[:plain_n])
    s_plain = summarize(plain, span_p)
    s_plain["arrivals"] = f"the first {plain_n} arrivals of the {rates[0]} req/s run"
    out["plain"] = s_plain
    for r in out["rates"]:
        r["throughput_ratio"] = r["served"]["particle_substeps_per_s"] / s_plain["particle_substeps_per_s"]
    return out


def bench_obstacle(free_launch_ms: float) -> dict:
    """The benchmark scene with a rigid sphere just ahead of the column (the
    fluid reaches it within the first ~400 substeps): per-launch device time of
    the fused transfer in the variant that carries the obstacle contact, at the
    64-register (256 x 4) and 80-register (256 x 3) shapes on 8^3 blocks, after
    the same 18 warm-up segments of 64 substeps, beside the obstacle-free
    kernel's time from the single-scene section."""
    from tessera_b200 import scenes
    from tessera_b200.session import Session

    sc = scenes.dam_break_obstacle()
    c = np.asarray(sc.obstacles[0].center)
    r = sc.obstacles[0].dims[0]
    out = {"workload": "config2 dam break + sphere obstacle", "particles": sc.particles.count,
           "obstacle": sc.info["obstacle"], "obstacle_free_launch_ms": free_launch_ms, "launch_ms": {}}
    for cfg, name in ((3, "256x4/8^3"), (5, "256x3/8^3")):
        s = Session(sc.params, sc.particles, sc.dt, obstacles=sc.obstacles, launch_shape=cfg)
        for _ in range(18):
            s.bench_substeps(BATCH)
        s.synchronize()
        _, kms = s.bench_substeps(BATCH, per_kernel=True)
        s.synchronize()
        out["launch_ms"][name] = float(kms[2])
        pos = s.read(("position",))["position"]
        out.setdefault("particles_within_one_cell_of_the_sphere", {})[name] = int(
            np.count_nonzero(np.linalg.norm(pos - c, axis=1) < r + sc.params.cell_width))
        s.close()
    return out


def bench_adjoint() -> dict:
    """Forward + adjoint of the 64k-particle rollout (256 substeps, checkpoints every 16)."""
    from tessera_b200 import scenes
    from tessera_b200.adjoint import Rollout

    sc = scenes.adjoint_block()
    n = sc.particles.count
    sim = Rollout(sc.params, sc.particles, sc.dt, sc.substeps, checkpoint_every=16)
    v0 = sc.particles.velocity.copy()
    E = np.full(n, 5e3)
    target = np.asarray(sc.info["target"])
    fw, bw = [], []
    for it in range(4):
        t0 = time.perf_counter()
        x, _ = sim.forward(v0, E)
        t1 = time.perf_counter()
        sim.backward(np.tile(2.0 * (x.mean(0) - target) / n, (n, 1)))
        t2 = time.perf_counter()
        if it > 0:
            fw.append(t1 - t0)
            bw.append(t2 - t1)
    sim.close()
    work = float(n) * sc.substeps
    f, b = float(np.median(fw)), float(np.median(bw))
    # the dense node array of the rollout: cells floor(bound / h - 0.5) - 1 .. + 3 per axis
    h = sc.params.cell_width
    dims = [int(np.floor(np.float32(sc.params.bounds_max[k]) * np.float32(1.0 / h) - np.float32(0.5))) + 3 -
            (int(np.floor(np.float32(sc.params.bounds_min[k]) * np.float32(1.0 / h) - np.float32(0.5))) - 1) + 1
            for k in range(3)]
    nodes = int(np.prod(dims))
    peak, peak_kind = measured_peaks()

    def roof(bytes_particle, bytes_node, seconds):
        alg = (bytes_particle * n + bytes_node * nodes) * sc.substeps
        gbs = alg / seconds / 1e9
        return {"bound": "latency (every kernel is one partial wave of CTAs at 64k particles)",
                "alg_bytes_per_particle_substep": bytes_particle, "alg_bytes_per_node_substep": bytes_node,
                "nodes": nodes, "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                "peak_source": peak_kind}

    # algorithmic bytes per substep: forward P2G (state 96 + E 4 in, node 16 out), grid (32 per node),
    # G2P (state 96 in and out, node 16 in), node clear (16), checkpoint copies (12 per particle);
    # backward replay as the forward plus the polar factors (36), and the adjoint: G2P adjoint (state 96,
    # state adjoint 96, partials 48 out; node velocity 16 in, node adjoint 16 out, cleared 16), grid
    # adjoint (48 in, 16 out per node), P2G adjoint (state 96, E 4, partials 48, polar 36 in; node 16 in;
    # state adjoint 96 and E adjoint 4 out)
    roofline = {"forward": roof(304, 80, f), "backward": roof(852, 208, b)}
    return {"workload": "config5-differentiable", "particles": n, "substeps": sc.substeps, "checkpoint_every": 16,
            "forward_s": f, "backward_s": b, "forward": work / f, "backward": work / b,
            "forward_plus_backward": work / (f + b), "unit": METRIC, "roofline": roofline,
            "timing": "wall clock through the C ABI (host f64 arrays in and out, synchronous calls)",
            "parity": "gradients vs central differences of the oracle: tests/test_gpu_adjoint.py"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from tessera_b200 import scenes

    per_step = []
    for it in range(args.warmup + args.steps):
        res = cpu_baseline(scenes.dam_break, target_seconds=8.0)
        if it >= args.warmup:
            per_step.append(res["value"])
    value = float(np.median(per_step))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "config2-dam-break (bounded CPU sample, see cpu_baseline.sample)",
                   "particles_full": 4049637},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": res["cores"], "kind": res["kind"],
                         "sample": res["sample"]},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_tessera(args, world, rank, local):
    import torch

    from tessera_b200 import scenes
    from tessera_b200.session import Session

    torch.cuda.set_device(local)
    sc = scenes.dam_break(seed=2 + rank, scale=args.scale)
    if args.load_state:  # the evolved dynamic fields over the same seeded scene
        with np.load(args.load_state) as st:
            for f in STATE_FIELDS:
                getattr(sc.particles, f)[...] = st[f]
    n = sc.particles.count
    session = Session(sc.params, sc.particles, sc.dt, device=local, launch_shape=args.launch_shape)
    # active grid nodes G (nodes with mass after P2G) for the algorithmic bytes
    _, mm = session.debug_p2g()
    grid_nodes = int(mm.shape[0])

    # the launch-shape tuner's trials (two 64-substep segments per shape) come
    # before the warm-up, so the timed region starts on the chosen shape (the
    # session keeps timing its segments and may switch as the scene evolves)
    for _ in range(16):
        if session.launch_shape()["shape"] is not None:
            break
        session.bench_substeps(BATCH)
        session.synchronize()
    shape_info = session.launch_shape()
    for _ in range(args.warmup):
        session.bench_substeps(BATCH)
    session.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms, _ = session.bench_substeps(BATCH * args.steps)
    torch.cuda.synchronize()
    barrier(world)
    session.synchronize()  # validates the device result (raises on any failure flag)
    ms_max = allreduce_max(ms, world)
    units = allreduce_sum(float(n) * BATCH * args.steps, world)
    value = units / (ms_max / 1000.0)

    # per-kernel average launch durations (CUDA events on the session stream),
    # one segment under the configuration in use
    _, kms = session.bench_substeps(BATCH, per_kernel=True)
    session.synchronize()
    shape_end = session.launch_shape()
    if args.save_state:  # f32 is exact: the device state is f32
        st = session.particles()
        np.savez(args.save_state, **{f: getattr(st, f).astype(np.float32) for f in STATE_FIELDS})
    g2p2g_ms = float(kms[2])
    peak, peak_kind = measured_peaks()
    # algorithmic bytes of one fused G2P->P2G launch: 248 B per particle (P2G 104 + G2P 48 + 96 write) and
    # 32 B per active node (P2G write 16 + G2P read 16); the grid update's 32 B/node is the other kernel
    alg_bytes = 248.0 * n + 32.0 * grid_nodes
    achieved = alg_bytes / (g2p2g_ms / 1000.0) / 1e9
    roofline = {"kernel": "fused G2P of step n + P2G of step n+1: k_transfer_fast with k_transfer_deferred beside and "
                          "after it, timed together", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": None, "alg_bytes_per_launch": alg_bytes, "launch_ms": g2p2g_ms,
                "kernel_ms": {"p2g": float(kms[0]), "grid": float(kms[1]), "g2p2g": g2p2g_ms, "g2p": float(kms[3]),
                              "resort": float(kms[4])}}
    # DRAM traffic per particle of the fused launch, captured with ncu for a launch
    # configuration; used when the timed launches ran that configuration
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    k_end = shape_end["shape"]
    timed_config = None if k_end is None else "{}x{}/{}^3".format(*shape_end["shapes"][k_end])
    roofline["launch_config"] = timed_config
    if os.path.exists(prof):
        with open(prof) as f:
            tr = json.load(f)
        per = tr.get("g2p2g_bytes_per_particle", {})
        if timed_config in per:
            roofline["traffic"] = per[timed_config] * n
            roofline["traffic_source"] = tr.get("source")

    # e2e: host arrays -> device -> 64 substeps -> host arrays, through the C ABI
    host = sc.particles
    e2e = None
    if args.e2e_steps > 0:
        from tessera_b200._abi import ParticleArrays

        out = ParticleArrays(n)  # caller-owned host arrays, reused across steps

        def e2e_step():
            session.write_particles(host)
            session.step(BATCH)
            session.particles(out)

        # warm-up as for the device timing (the first calls also fault in the
        # session's host world buffers), then one timed region of e2e_steps steps
        for _ in range(max(args.warmup, 3)):
            e2e_step()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = allreduce_max((time.perf_counter() - t0) / args.e2e_steps, world)
        cap = (n + 255) // 256 * 256
        assert np.all(np.isfinite(out.position))
        e2e = {"value": allreduce_sum(float(n) * BATCH, world) / e2e_s, "unit": METRIC,
               # 27 f32 rows (x, v, C, F, plastic) per particle up with the class and
               # world-index rows; 24 back (no plastic materials in this scene) with the
               # status and non-finite flags
               "h2d_bytes_per_step": 4 * 27 * n + 8 * cap,
               "d2h_bytes_per_step": 4 * 24 * n + 8, "seconds_per_step": e2e_s,
               "timing": f"wall clock of {args.e2e_steps} consecutive steps after {max(args.warmup, 3)} warm-up steps"}

    cpu = small = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(scenes.dam_break)
    clk = clocks.summary()
    session.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        small = bench_small_configs()
    batched = serving = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = bench_batched(args.batched_scenes)
    elif world > 1 and not args.no_batched:  # every rank: its share of the scenes
        batched = bench_batched_parallel(args.batched_scenes, world, rank)
    if rank == 0 and world == 1 and not args.no_serving:
        serving = bench_serving([float(r) for r in args.serve_rates.split(",") if r], args.serve_requests)
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = bench_adjoint()
    obstacle = None
    if rank == 0 and world == 1 and not args.no_obstacle:
        obstacle = bench_obstacle(g2p2g_ms)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "config2-dam-break", "particles_per_gpu": n, "grid": "256^3 virtual, hashed blocks of 4^3 or 8^3 cells (tuned)",
                       "active_grid_nodes": grid_nodes, "dt": sc.dt, "substeps_per_step": BATCH,
                       "l2": "inputs larger than L2 (particle state ~0.4 GB per GPU)",
                       "launch_shape": shape_summary(shape_info),
                       "launch_shape_after_timing": shape_summary(shape_end),
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": SEGMENT_LAUNCHES * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "batched": batched,
            "serving": serving,
            "adjoint": adjoint,
            "obstacle": obstacle,
            "small_configs": small,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.only:
        if args.only == "batched":
            res = bench_batched(args.batched_scenes)
        elif args.only == "serving":
            res = bench_serving([float(r) for r in args.serve_rates.split(",") if r], args.serve_requests)
        elif args.only == "obstacle":
            res = bench_obstacle(float("nan"))
        else:
            res = bench_adjoint()
        print(json.dumps(res), flush=True)
        return
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_tessera(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
