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
# re-sort per batch: bin keys, 4 radix passes x (hist, scan, scatter), gather
RESORT_LAUNCHES = 1 + 4 * 3 + 1
METRIC = "particle-substeps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tessera", choices=["tessera", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0, help="column footprint scale (1.0 = full config)")
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
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

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
    n = sc.particles.count
    session = Session(sc.params, sc.particles, sc.dt, device=local)
    # active grid nodes G (nodes with mass after P2G) for the algorithmic bytes
    _, mm = session.debug_p2g()
    grid_nodes = int(mm.shape[0])

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

    # per-kernel average launch durations (CUDA events on the session stream)
    _, kms = session.bench_substeps(BATCH, per_kernel=True)
    session.synchronize()
    g2p2g_ms = float(kms[2])
    peak, peak_kind = measured_peaks()
    # algorithmic bytes of one fused G2P->P2G launch: 248 B per particle (P2G 104 + G2P 48 + 96 write) and
    # 32 B per active node (P2G write 16 + G2P read 16); the grid update's 32 B/node is the other kernel
    alg_bytes = 248.0 * n + 32.0 * grid_nodes
    achieved = alg_bytes / (g2p2g_ms / 1000.0) / 1e9
    roofline = {"kernel": "k_transfer<G2P2G> (fused G2P of step n + P2G of step n+1)", "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "traffic": None, "alg_bytes_per_launch": alg_bytes, "launch_ms": g2p2g_ms,
                "kernel_ms": {"p2g": float(kms[0]), "grid": float(kms[1]), "g2p2g": g2p2g_ms, "g2p": float(kms[3]),
                              "resort": float(kms[4])}}
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            tr = json.load(f)
        if "g2p2g_bytes_per_particle" in tr:
            roofline["traffic"] = tr["g2p2g_bytes_per_particle"] * n
            roofline["traffic_source"] = tr.get("source")

    # e2e: host arrays -> device -> 64 substeps -> host arrays, through the C ABI
    host = sc.particles
    e2e = None
    if args.e2e_steps > 0:
        from tessera_b200._abi import ParticleArrays

        e2e_times = []
        out = ParticleArrays(n)  # caller-owned host arrays, reused across steps
        for it in range(1 + args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            session.write_particles(host)
            session.step(BATCH)
            session.particles(out)
            t1 = time.perf_counter()
            if it > 0:
                e2e_times.append(t1 - t0)
        e2e_s = allreduce_max(max(e2e_times), world)
        cap = (n + 255) // 256 * 256
        assert np.all(np.isfinite(out.position))
        e2e = {"value": allreduce_sum(float(n) * BATCH, world) / e2e_s, "unit": METRIC,
               "h2d_bytes_per_step": 4 * 24 * cap + 8 * cap + 12 * n + 4,
               "d2h_bytes_per_step": 4 * 24 * n + 4 * n + 4, "seconds_per_step": e2e_s}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(scenes.dam_break)
    clk = clocks.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": "config2-dam-break", "particles_per_gpu": n, "grid": "256^3 virtual, 4^3 blocks",
                       "active_grid_nodes": grid_nodes, "dt": sc.dt, "substeps_per_step": BATCH,
                       "l2": "inputs larger than L2 (particle state ~0.4 GB per GPU)",
                       "parallelism": f"replicas x{world}"},
            "gpu_launches": (2 * BATCH + 2 + RESORT_LAUNCHES) * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    session.close()


def main():
    args = parse()
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
