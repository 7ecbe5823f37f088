"""Serving loop: continuous batching of MPM scenes on one device.

Requests (a scene and a substep count) arrive over time.  Arrived requests
are prepared (validated and packed for upload) on worker threads
while the device runs, admitted in arrival order while their device
footprint fits the HBM budget and a scene slot is free, and advanced
together: every batch moves each resident scene by up to `chunk` substeps
in one set of launches.  Admission happens while a batch runs, so a new
scene's rows are copied to the device during it and the scene joins the next
batch, or at once when the device has nothing else to run.  A scene that finishes in a batch is read while the
next batch runs (the batch does not touch it) and retired, which frees its
budget.  Requests that arrive while
others are on the device therefore join at the next batch boundary instead
of waiting for the device to drain.

Each result is the scene's state after its substeps, the same as a
single-scene session over that scene alone (GpuMpmResidentSession,
crates/tessera-mpm/src/gpu.rs:206-662) within f32 round-off.

`run_plain` is the one-scene-at-a-time loop on the same device, for
comparison: a session per request, in arrival order.
"""

from __future__ import annotations

import math
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from ._abi import TMPM_ERR_CAPACITY, TMPM_OK
from .scenes import Scene
from .session import TesseraError

OUTPUT_FIELDS = ("position", "velocity")


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the start of the run
    scene: Scene
    steps: int


@dataclass
class Outcome:
    rid: int
    arrival: float
    steps: int
    particles: int
    admitted: float = math.nan
    finished: float = math.nan
    status: int = TMPM_OK
    error: str = ""
    outputs: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def queueing(self) -> float:
        return self.admitted - self.arrival


def poisson_arrivals(rate: float, count: int, seed: int = 0) -> np.ndarray:
    """Arrival times of a Poisson process of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def summarize(outcomes: list[Outcome], makespan: float) -> dict:
    ok = [o for o in outcomes if o.status == TMPM_OK]
    lat = np.array([o.latency for o in ok]) if ok else np.zeros(0)
    work = float(sum(o.particles * o.steps for o in ok))
    arrivals = np.array([o.arrival for o in outcomes])
    span = float(arrivals.max() - arrivals.min()) if len(arrivals) > 1 else 0.0
    return dict(
        requests=len(outcomes), completed=len(ok), failed=len(outcomes) - len(ok),
        offered_req_per_s=(len(outcomes) - 1) / span if span > 0 else None,
        makespan_s=makespan,
        particle_substeps_per_s=work / makespan if makespan > 0 else 0.0,
        p50_s=float(np.percentile(lat, 50)) if len(lat) else None,
        p99_s=float(np.percentile(lat, 99)) if len(lat) else None,
        mean_queueing_s=float(np.mean([o.queueing for o in ok])) if ok else None,
    )


class Server:
    """Continuous-batching server over one multi-scene batch.

    `batch` is a tessera_b200.batch.Batch (or an object with the same
    methods); `prepare(params, particles, dt)` returns a prepared scene with
    `device_bytes()` (tessera_b200.batch.PreparedScene by default)."""

    def __init__(self, batch=None, hbm_budget: float = 120e9, chunk: int = 32, lookahead: int = 8,
                 prepare_workers: int = 1, keep_outputs: bool = False, max_scenes: int = 256, prepare=None,
                 clock=time.perf_counter):
        if batch is None or prepare is None:
            from .batch import Batch, PreparedScene
            batch = batch if batch is not None else Batch()
            prepare = prepare if prepare is not None else PreparedScene
        self.batch = batch
        self.prepare = prepare
        self.budget = float(hbm_budget)
        self.chunk = int(chunk)
        self.lookahead = int(lookahead)
        self.workers = int(prepare_workers)
        self.keep_outputs = keep_outputs
        self.max_scenes = int(max_scenes)
        self.clock = clock
        self.used = 0.0
        self.batches = 0
        self.peak_resident = 0
        self.peak_bytes = 0.0
        # where the run's time went (seconds): host time in submit (it copies
        # rows admitted without room), in admission (it copies rows while a
        # batch runs), in reading and retiring finished scenes, waiting
        # for a batch, idle waiting for a preparation; device time of the batches
        # (CUDA events); and each preparation's own duration on its worker
        self.timing = {"submit_s": 0.0, "admit_s": 0.0, "retire_s": 0.0, "sync_wait_s": 0.0, "prepare_wait_s": 0.0,
                       "device_s": 0.0, "first_submit_s": None, "prepare_s": []}

    def _prepare_timed(self, params, particles, dt):
        t = self.clock()
        try:
            return self.prepare(params, particles, dt)
        finally:
            self.timing["prepare_s"].append(self.clock() - t)

    def run(self, requests: list[Request]) -> tuple[list[Outcome], float]:
        reqs = sorted(requests, key=lambda r: r.arrival)
        outcomes = {r.rid: Outcome(r.rid, r.arrival, r.steps, r.scene.particles.count) for r in reqs}
        waiting: deque = deque()  # [request, future]
        resident: dict[int, list] = {}  # scene id -> [request, remaining, bytes]
        finished: list[int] = []  # finished in the last batch, to read and retire
        nxt = 0
        pool = ThreadPoolExecutor(max_workers=max(1, self.workers))
        t0 = self.clock()

        def now() -> float:
            return self.clock() - t0

        def arrivals():
            nonlocal nxt
            t = now()
            while nxt < len(reqs) and reqs[nxt].arrival <= t:
                waiting.append([reqs[nxt], None])
                nxt += 1
            for k, w in enumerate(waiting):
                if k >= self.lookahead:
                    break
                if w[1] is None:
                    sc = w[0].scene
                    w[1] = pool.submit(self._prepare_timed, sc.params, sc.particles, sc.dt)

        def retire(sid: int):
            t_r = self.clock()
            req, _, nbytes = resident.pop(sid)
            o = outcomes[req.rid]
            take = getattr(self.batch, "take", None)  # read + remove in one call, where the batch has it
            removed = False
            try:
                if take is not None:
                    out = take(sid, OUTPUT_FIELDS)
                    removed = True
                else:
                    out = self.batch.read(sid, OUTPUT_FIELDS)
                if self.keep_outputs:
                    o.outputs = out
            except TesseraError as e:
                o.status, o.error = e.status, e.reason
            o.finished = now()
            if not removed:
                self.batch.remove_scene(sid)
            self.used -= nbytes
            self.timing["retire_s"] += self.clock() - t_r

        def admit_ready(limit=None):
            # admission in arrival order, by device footprint (at most `limit` scenes)
            admitted = 0
            while waiting and waiting[0][1] is not None and waiting[0][1].done():
                if limit is not None and admitted >= limit:
                    break
                req, fut = waiting[0]
                o = outcomes[req.rid]
                try:
                    prepared = fut.result()
                except TesseraError as e:
                    waiting.popleft()
                    o.status, o.error, o.finished = e.status, e.reason, now()
                    continue
                need = float(prepared.device_bytes())
                if need > self.budget:
                    waiting.popleft()
                    o.status, o.error, o.finished = TMPM_ERR_CAPACITY, "scene exceeds the HBM budget", now()
                    continue
                if self.used + need > self.budget or len(resident) >= self.max_scenes:
                    break
                t_a = self.clock()
                sid = self.batch.admit(prepared)
                self.timing["admit_s"] += self.clock() - t_a
                admitted += 1
                waiting.popleft()
                self.used += need
                resident[sid] = [req, req.steps, need]
                o.admitted = now()
                arrivals()

        def pending_work():
            return {sid: min(self.chunk, st[1]) for sid, st in resident.items() if st[1] > 0}

        try:
            while True:
                arrivals()
                active = pending_work()
                if not active:
                    # nothing to run: admit one scene now and start on it (otherwise admission
                    # waits for the batch in flight, so rows are copied while the device works)
                    admit_ready(limit=1)
                    active = pending_work()
                if not active:
                    for sid in finished:
                        retire(sid)
                    finished = []
                    if nxt >= len(reqs) and not waiting and not resident:
                        break
                    # idle: the next arrival or a preparation in progress
                    if waiting and waiting[0][1] is not None:
                        t_w = self.clock()
                        waiting[0][1].result()
                        self.timing["prepare_wait_s"] += self.clock() - t_w
                    elif nxt < len(reqs):
                        time.sleep(max(0.0, min(reqs[nxt].arrival - now(), 0.005)))
                    continue
                t_s = self.clock()
                if self.timing["first_submit_s"] is None:
                    self.timing["first_submit_s"] = t_s - t0
                self.batch.submit(active)
                self.timing["submit_s"] += self.clock() - t_s
                self.batches += 1
                self.peak_resident = max(self.peak_resident, len(resident))
                self.peak_bytes = max(self.peak_bytes, self.used)
                # host work while the batch runs: results of the previous batch, arrivals
                for sid in finished:
                    retire(sid)
                finished = []
                arrivals()
                admit_ready()  # joins the next batch
                t_s = self.clock()
                self.batch.synchronize()
                self.timing["sync_wait_s"] += self.clock() - t_s
                last_ms = getattr(self.batch, "last_ms", None)
                if last_ms is not None:
                    self.timing["device_s"] += float(last_ms()) / 1e3
                for sid, k in active.items():
                    st = resident[sid]
                    status = self.batch.status(sid)
                    if status != TMPM_OK:
                        o = outcomes[st[0].rid]
                        o.status, o.error = status, "scene left the resident path"
                        st[1] = 0
                        finished.append(sid)
                        continue
                    st[1] -= k
                    if st[1] == 0:
                        finished.append(sid)
            makespan = now()
        finally:
            pool.shutdown(wait=True)
        return [outcomes[r.rid] for r in reqs], makespan


def run_plain(requests: list[Request], device: int = 0, keep_outputs: bool = False,
              clock=time.perf_counter) -> tuple[list[Outcome], float]:
    """One scene at a time in arrival order: a session per request."""
    from .session import Session
    reqs = sorted(requests, key=lambda r: r.arrival)
    outcomes = []
    t0 = clock()
    for r in reqs:
        o = Outcome(r.rid, r.arrival, r.steps, r.scene.particles.count)
        wait = r.arrival - (clock() - t0)
        if wait > 0:
            time.sleep(wait)
        o.admitted = clock() - t0
        try:
            s = Session(r.scene.params, r.scene.particles, r.scene.dt, device=device)
            left = r.steps
            while left:
                k = min(64, left)
                s.step(k)
                left -= k
            out = s.read(OUTPUT_FIELDS)
            if keep_outputs:
                o.outputs = out
            s.close()
        except TesseraError as e:
            o.status, o.error = e.status, e.reason
        o.finished = clock() - t0
        outcomes.append(o)
    return outcomes, clock() - t0
