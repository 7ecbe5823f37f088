"""CPU tests of the serving loop's host logic (admission by footprint, arrival
order, continuous batching, retirement) over a fake batch that advances each
scene with the f64 oracle, so the results can be compared with the oracle run
alone."""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200 import scenes
from tessera_b200._abi import TMPM_ERR_CAPACITY, TMPM_OK
from tessera_b200.serve import Request, Server, poisson_arrivals, summarize

ROW_BYTES = 264


class FakePrepared:
    def __init__(self, params, particles, dt):
        self.params, self.particles, self.dt = params, particles.copy(), dt

    def device_bytes(self):
        return self.particles.count * ROW_BYTES


class FakeBatch:
    """The Batch methods the server uses, with the oracle as the device."""

    def __init__(self, budget):
        self.budget = budget
        self.worlds = {}
        self.steps = {}
        self.used = 0
        self.peak = 0
        self.in_flight = None
        self.log = []

    def admit(self, p):
        sid = next(i for i in range(256) if i not in self.worlds)
        self.worlds[sid] = (O.OracleWorld(p.params, p.particles), p.dt, p.device_bytes())
        self.used += p.device_bytes()
        self.peak = max(self.peak, self.used)
        assert self.used <= self.budget
        self.log.append(("admit", sid))
        return sid

    def submit(self, steps):
        assert self.in_flight is None
        self.in_flight = dict(steps)
        self.log.append(("submit", tuple(sorted(steps.items()))))

    def synchronize(self):
        for sid, k in self.in_flight.items():
            w, dt, _ = self.worlds[sid]
            for _ in range(k):
                w.substep_fixed(dt)
        self.in_flight = None

    def status(self, sid):
        return TMPM_OK

    def read(self, sid, fields):
        assert self.in_flight is None or sid not in self.in_flight
        p = self.worlds[sid][0].particles()
        return {f: getattr(p, f).copy() for f in fields}

    def remove_scene(self, sid):
        self.used -= self.worlds.pop(sid)[2]
        self.log.append(("remove", sid))


def small_requests(n=6, seed=21, rate=400.0):
    t = poisson_arrivals(rate, n, seed)
    rng = np.random.default_rng(seed)
    return [Request(k, float(t[k]), scenes.batch_scene(seed * 100 + k, cells=3), int(rng.integers(3, 12)))
            for k in range(n)]


def oracle_alone(req):
    w = O.OracleWorld(req.scene.params, req.scene.particles)
    for _ in range(req.steps):
        w.substep_fixed(req.scene.dt)
    return w.particles()


def test_served_results_equal_each_scene_alone():
    reqs = small_requests()
    fb = FakeBatch(budget=1e12)
    server = Server(batch=fb, prepare=FakePrepared, chunk=4, keep_outputs=True, hbm_budget=1e12)
    outcomes, makespan = server.run(reqs)
    assert [o.rid for o in outcomes] == [r.rid for r in sorted(reqs, key=lambda r: r.arrival)]
    for r, o in zip(sorted(reqs, key=lambda r: r.arrival), outcomes):
        assert o.status == TMPM_OK
        ref = oracle_alone(r)
        assert np.array_equal(o.outputs["position"], ref.position)
        assert np.array_equal(o.outputs["velocity"], ref.velocity)
        assert o.arrival <= o.admitted <= o.finished
    s = summarize(outcomes, makespan)
    assert s["completed"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0
    assert fb.used == 0  # every scene retired


def test_admission_respects_the_budget_and_arrival_order():
    reqs = small_requests(n=8, seed=22, rate=5000.0)  # all arrive almost at once
    per_scene = reqs[0].scene.particles.count * ROW_BYTES
    budget = 2.5 * per_scene  # two scenes fit at a time
    fb = FakeBatch(budget=budget)
    server = Server(batch=fb, prepare=FakePrepared, chunk=3, hbm_budget=budget)
    outcomes, _ = server.run(reqs)
    assert all(o.status == TMPM_OK for o in outcomes)
    assert fb.peak <= budget and server.peak_resident == 2
    admitted = [sid for op, sid in fb.log if op == "admit"]
    assert len(admitted) == len(reqs)
    order = sorted(outcomes, key=lambda o: o.admitted)
    assert [o.rid for o in order] == [o.rid for o in outcomes]  # admitted in arrival order


def test_requests_join_while_others_are_running():
    # a long request first, then short ones: the short ones are admitted and
    # finish while the long one is still resident (continuous batching)
    reqs = small_requests(n=4, seed=23, rate=2000.0)
    reqs[0].steps = 40
    for r in reqs[1:]:
        r.steps = 3
    fb = FakeBatch(budget=1e12)
    outcomes, _ = Server(batch=fb, prepare=FakePrepared, chunk=4, hbm_budget=1e12).run(reqs)
    long = next(o for o in outcomes if o.rid == reqs[0].rid)
    for o in outcomes:
        if o.rid != long.rid:
            assert o.finished < long.finished
    multi = [ops for op, ops in fb.log if op == "submit" and len(ops) > 1]
    assert multi, "no batch carried more than one scene"


def test_oversized_scene_is_rejected_not_queued_forever():
    reqs = small_requests(n=3, seed=24)
    big = scenes.batch_scene(999, cells=5)
    reqs[1].scene = big
    budget = 2 * reqs[0].scene.particles.count * ROW_BYTES
    fb = FakeBatch(budget=budget)
    outcomes, _ = Server(batch=fb, prepare=FakePrepared, chunk=4, hbm_budget=budget).run(reqs)
    bad = next(o for o in outcomes if o.rid == reqs[1].rid)
    assert bad.status == TMPM_ERR_CAPACITY
    assert sum(o.status == TMPM_OK for o in outcomes) == 2


def test_poisson_arrivals_rate():
    t = poisson_arrivals(200.0, 4000, seed=1)
    assert np.all(np.diff(t) > 0)
    assert (len(t) - 1) / (t[-1] - t[0]) == pytest.approx(200.0, rel=0.05)
