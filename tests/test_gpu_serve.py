"""GPU test of the serving loop: every request's result, computed while other
requests share the device batch, equals the same scene run alone (a
single-scene session), within the resident-path FP32 tolerance
(gpu.rs:3699-3703: position 2e-5, velocity 2e-4)."""

import numpy as np
import pytest

from tessera_b200 import scenes
from tessera_b200._abi import TMPM_OK
from tessera_b200.batch import Batch
from tessera_b200.serve import Request, Server, poisson_arrivals, run_plain, summarize

pytestmark = pytest.mark.gpu


def requests(n=10, seed=31, rate=300.0):
    t = poisson_arrivals(rate, n, seed)
    rng = np.random.default_rng(seed)
    return [Request(k, float(t[k]), scenes.batch_scene(seed * 100 + k, cells=int(rng.integers(4, 9))),
                    int(rng.integers(5, 40))) for k in range(n)]


def test_each_result_is_the_same_alone_and_in_the_mix():
    reqs = requests()
    server = Server(batch=Batch(), chunk=8, keep_outputs=True, hbm_budget=64e9)
    mixed, makespan = server.run(reqs)
    alone, _ = run_plain(reqs, keep_outputs=True)
    assert server.batches > 0 and server.peak_resident > 1  # requests overlapped on the device
    for a, m in zip(alone, mixed):
        assert a.rid == m.rid and a.status == TMPM_OK and m.status == TMPM_OK
        dp = np.linalg.norm(a.outputs["position"] - m.outputs["position"], axis=1).max()
        dv = np.linalg.norm(a.outputs["velocity"] - m.outputs["velocity"], axis=1).max()
        assert dp < 2e-5, (m.rid, dp)
        assert dv < 2e-4, (m.rid, dv)
    s = summarize(mixed, makespan)
    assert s["completed"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0


def test_budget_limits_resident_scenes_on_the_device():
    from tessera_b200.batch import PreparedScene
    t = poisson_arrivals(5000.0, 8, seed=32)
    reqs = [Request(k, float(t[k]), scenes.batch_scene(3200 + k, cells=6), 12) for k in range(8)]
    one = PreparedScene(reqs[0].scene.params, reqs[0].scene.particles, reqs[0].scene.dt).device_bytes()
    budget = 2.5 * one  # footprints vary with the blocks each scene occupies: two or three fit at a time
    server = Server(batch=Batch(), chunk=6, hbm_budget=budget)
    outcomes, _ = server.run(reqs)
    assert all(o.status == TMPM_OK for o in outcomes)
    assert server.peak_bytes <= budget
    assert 2 <= server.peak_resident < len(reqs)
