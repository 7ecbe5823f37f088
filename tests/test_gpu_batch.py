"""GPU tests of multi-scene batches: every scene advanced inside a batch agrees
with the same scene run alone (a single-scene session) and with the f64 oracle.

Tolerances are the resident-path precedent (gpu.rs:3699-3703: position 2e-5,
velocity 2e-4, F 2e-4, affine 2e-3 after 8 substeps of FP32 device work against
the f64 CPU path).  Batch against alone compares two FP32 runs whose only
difference is the partition of particles into thread blocks (the fixed-point
scale of each block's shared accumulation), so it uses the same bounds.
"""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import (
    MAT_ELASTIC, TMPM_ERR_INVALID_INPUT, TMPM_ERR_PENDING_STEPS, TMPM_ERR_RESIDENT_UNAVAILABLE, ParticleArrays,
    density_particles, make_params,
)
from tessera_b200 import scenes
from tessera_b200.batch import Batch, home_blocks, scene_bytes
from tessera_b200.session import Session, TesseraError

pytestmark = pytest.mark.gpu


def mat_norm(a):
    return np.linalg.norm(a.reshape(-1, 9), axis=1)


def assert_close(expected: ParticleArrays, actual: ParticleArrays, pos=2e-5, vel=2e-4, F=2e-4, C=2e-3, what=""):
    dp = np.linalg.norm(expected.position - actual.position, axis=1).max()
    dv = np.linalg.norm(expected.velocity - actual.velocity, axis=1).max()
    dF = mat_norm(expected.deformation - actual.deformation).max()
    dC = mat_norm(expected.affine - actual.affine).max()
    assert dp < pos, f"{what} position {dp}"
    assert dv < vel, f"{what} velocity {dv}"
    assert dF < F, f"{what} deformation {dF}"
    assert dC < C, f"{what} affine {dC}"


def small_scenes(count=6, cells=6, seed=11):
    return [scenes.batch_scene(seed * 100 + k, cells=cells) for k in range(count)]


def alone(sc, steps):
    s = Session(sc.params, sc.particles, sc.dt)
    left = steps
    while left:
        k = min(64, left)
        s.step(k)
        left -= k
    out = s.particles()
    s.close()
    return out


def oracle_run(sc, steps):
    w = O.OracleWorld(sc.params, sc.particles)
    for _ in range(steps):
        w.substep_fixed(sc.dt)
    return w.particles()


def test_batch_scene_equals_scene_alone_and_oracle():
    scs = small_scenes()
    b = Batch()
    ids = [b.add_scene(sc.params, sc.particles, sc.dt) for sc in scs]
    assert ids == list(range(len(scs)))
    b.run({i: 16 for i in ids})
    for i, sc in zip(ids, scs):
        assert b.substeps(i) == 16
        got = b.particles(i)
        assert_close(alone(sc, 16), got, what=f"scene {i} vs alone")
        assert_close(oracle_run(sc, 16), got, what=f"scene {i} vs oracle")
    assert b.last_ms() > 0.0


def test_uneven_step_counts_in_one_batch():
    scs = small_scenes(count=4, cells=5, seed=12)
    b = Batch()
    ids = [b.add_scene(sc.params, sc.particles, sc.dt) for sc in scs]
    steps = {ids[0]: 3, ids[1]: 16, ids[2]: 9, ids[3]: 1}
    b.run(steps)
    for i, sc in zip(ids, scs):
        assert b.substeps(i) == steps[i]
        assert_close(alone(sc, steps[i]), b.particles(i), what=f"scene {i}")
    # a second batch continues each scene from where it stopped
    b.run({ids[0]: 13, ids[3]: 15})
    for i in (ids[0], ids[3]):
        assert b.substeps(i) == 16
        assert_close(alone(scs[i], 16), b.particles(i), what=f"scene {i} second batch")
    assert b.substeps(ids[2]) == 9


def test_batch_with_and_without_graph_replay_agree():
    scs = small_scenes(count=3, cells=5, seed=13)
    outs = []
    for graphs in (True, False):
        b = Batch(use_graphs=graphs)
        ids = [b.add_scene(sc.params, sc.particles, sc.dt) for sc in scs]
        for _ in range(3):  # replays the captured graph twice per buffer parity
            b.run({i: 4 for i in ids})
        outs.append([b.particles(i) for i in ids])
        b.close()
    for a, c in zip(*outs):
        assert_close(a, c, what="graph vs direct")


def test_admission_and_retirement_between_batches():
    scs = small_scenes(count=4, cells=5, seed=14)
    b = Batch()
    a0 = b.add_scene(scs[0].params, scs[0].particles, scs[0].dt)
    a1 = b.add_scene(scs[1].params, scs[1].particles, scs[1].dt)
    a2 = b.add_scene(scs[2].params, scs[2].particles, scs[2].dt)
    b.run({a0: 8, a1: 8, a2: 8})
    b.remove_scene(a1)
    a3 = b.add_scene(scs[3].params, scs[3].particles, scs[3].dt)
    assert a3 == 3  # the removed id frees up only after the next re-sort
    b.run({a0: 8, a2: 4, a3: 8})
    assert_close(alone(scs[0], 16), b.particles(a0), what="kept scene")
    assert_close(alone(scs[2], 12), b.particles(a2), what="kept scene 2")
    assert_close(alone(scs[3], 8), b.particles(a3), what="admitted scene")
    a4 = b.add_scene(scs[1].params, scs[1].particles, scs[1].dt)
    assert a4 == a1
    b.run({a4: 5})
    assert_close(alone(scs[1], 5), b.particles(a4), what="re-admitted scene")
    with pytest.raises(TesseraError) as e:
        b.particles(99)
    assert e.value.status == TMPM_ERR_INVALID_INPUT


def test_failed_scene_does_not_disturb_the_others():
    # a scene whose substep sits at its initial CFL bound and that gravity then
    # pushes over it fails the resident check on the device (gpu.wgsl:983-994)
    h = 1.0 / 32
    r = h / 4
    pos = scenes.lattice((0.4, 0.4, 0.6), (0.4 + 4 * h, 0.4 + 4 * h, 0.6 + 4 * h), 2 * r, np.random.default_rng(5))
    parts = density_particles(pos, r, 1000.0, MAT_ELASTIC, (1e4, 0.2))
    params = make_params(h, gravity=(0.0, 0.0, -2000.0), max_substep=1.0, bounds=((0, 0, 0), (1, 1, 1)))
    c = np.sqrt((1e4 * 0.2 / (1.2 * 0.6) + 2 * 1e4 / 2.4) / 1000.0)
    dt_edge = 0.4 * h / c * 0.9999
    good = small_scenes(count=2, cells=5, seed=15)
    b = Batch()
    g0 = b.add_scene(good[0].params, good[0].particles, good[0].dt)
    bad = b.add_scene(params, parts, dt_edge)
    g1 = b.add_scene(good[1].params, good[1].particles, good[1].dt)
    b.run({g0: 12, bad: 12, g1: 12})
    assert b.status(bad) == TMPM_ERR_RESIDENT_UNAVAILABLE
    assert b.substeps(bad) == 0
    with pytest.raises(TesseraError) as e:
        b.particles(bad)
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE
    with pytest.raises(TesseraError):
        b.submit({bad: 1})
    for i, sc in ((g0, good[0]), (g1, good[1])):
        assert b.status(i) == 0
        assert_close(alone(sc, 12), b.particles(i), what=f"healthy scene {i}")
    # run alone, the same scene fails the same way
    s = Session(params, parts, dt_edge)
    with pytest.raises(TesseraError) as e:
        s.step(12)
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE


def test_batch_rejects_invalid_requests():
    sc = small_scenes(count=1, cells=4, seed=16)[0]
    b = Batch()
    with pytest.raises(TesseraError) as e:
        b.add_scene(sc.params, sc.particles, 1.0)  # above the CFL bound
    assert e.value.status == TMPM_ERR_INVALID_INPUT
    colored = sc.particles.copy()
    colored.transfer_color[:] = 300
    with pytest.raises(TesseraError) as e:
        b.add_scene(sc.params, colored, sc.dt)
    assert e.value.status == TMPM_ERR_INVALID_INPUT
    i = b.add_scene(sc.params, sc.particles, sc.dt)
    with pytest.raises(TesseraError) as e:
        b.submit({i: 0})
    assert e.value.status == TMPM_ERR_INVALID_INPUT
    b.submit({i: 4})
    with pytest.raises(TesseraError) as e:
        b.submit({i: 4})
    assert e.value.status == TMPM_ERR_PENDING_STEPS
    b.synchronize()
    assert b.substeps(i) == 4
    assert b.device_bytes() > scene_bytes(sc.particles.count, home_blocks(sc.particles.position, 1.0 / 16)) // 4


def test_admission_and_reads_while_a_batch_is_in_flight():
    from tessera_b200.batch import PreparedScene
    scs = small_scenes(count=3, cells=5, seed=17)
    b = Batch()
    a = b.add_scene(scs[0].params, scs[0].particles, scs[0].dt)
    b.submit({a: 8})
    assert b.pending()
    prepared = PreparedScene(scs[1].params, scs[1].particles, scs[1].dt)  # no device work
    assert prepared.device_bytes() > 0
    c = b.admit(prepared)  # attached while the first batch runs; copied at the next submit
    with pytest.raises(TesseraError) as e:
        b.particles(a)  # in flight
    assert e.value.status == TMPM_ERR_PENDING_STEPS
    b.synchronize()
    b.run({a: 8, c: 8})
    b.submit({c: 4})
    # `a` is not in the batch in flight: it is read from the rows that batch re-sorts from
    assert_close(alone(scs[0], 16), b.particles(a), what="scene beside a running batch")
    with pytest.raises(TesseraError) as e:
        b.particles(c)
    assert e.value.status == TMPM_ERR_PENDING_STEPS
    b.synchronize()
    assert_close(alone(scs[1], 12), b.particles(c), what="admitted-in-flight scene")
    # retire while a batch is in flight
    d = b.admit(PreparedScene(scs[2].params, scs[2].particles, scs[2].dt))
    b.submit({a: 4, c: 4, d: 4})
    b.remove_scene(a)
    b.synchronize()
    assert_close(alone(scs[1], 16), b.particles(c), what="scene beside a retired one")
    assert_close(alone(scs[2], 4), b.particles(d), what="third scene")
    with pytest.raises(TesseraError):
        b.particles(a)
    # a prepared scene that is never admitted just goes away
    PreparedScene(scs[2].params, scs[2].particles, scs[2].dt).close()


def test_take_returns_what_a_read_returns_and_removes_the_scene():
    """Retiring through take (only the requested rows come back, the host world
    is not updated first) gives the state a read gives, fixed and disabled
    particles included, and frees the scene's slot."""
    sc = scenes.batch_scene(31, cells=6)
    parts = sc.particles.copy()
    parts.fixed[0] = 1
    parts.enabled[1] = 0
    runs = []
    for mode in ("read", "take"):
        b = Batch()
        sid = b.add_scene(sc.params, parts, sc.dt)
        other = b.add_scene(sc.params, sc.particles, sc.dt)  # a neighbour that stays
        b.run({sid: 8, other: 8})
        if mode == "read":
            got = b.particles(sid)
        else:
            fields = ("position", "velocity", "affine", "deformation", "mass", "material")
            arrays = b.take(sid, fields)
            with pytest.raises(TesseraError) as e:
                b.read(sid, ("position",))  # gone
            assert e.value.status == TMPM_ERR_INVALID_INPUT
            got = parts.copy()
            for f in fields:
                getattr(got, f)[:] = arrays[f]
            assert np.array_equal(arrays["mass"], parts.mass) and np.array_equal(arrays["material"], parts.material)
        runs.append(got)
        assert np.all(np.isfinite(b.particles(other).position))  # the neighbour is intact
        b.close()
    read, took = runs
    assert_close(read, took, pos=1e-6, vel=1e-5, F=1e-5, C=1e-4, what="take vs read")
    for arr in (took, read):
        assert np.array_equal(arr.position[0], parts.position[0])  # fixed: stays
        assert np.all(arr.velocity[0] == 0.0) and np.all(arr.affine[0] == 0.0)
        assert np.array_equal(arr.position[1], parts.position[1])  # disabled: untouched
        assert np.array_equal(arr.velocity[1], parts.velocity[1])


def test_config3_subset_at_size_matches_alone_and_oracle():
    """Scenes of the 256-scene heterogeneous batch at their real sizes: the
    largest (262,144 particles on a 128^3 grid, elastic), the largest fluid
    scene (238,328 particles, 124^3), the smallest (4,096, 32^3) and two
    mid-sized ones, advanced together as one batch for the workload's 100
    substeps.  Each scene is compared with the same scene run alone and with
    the f64 oracle under the relative drift bounds of the configuration-sized
    parity tests (parity_tol.py): position 1e-3 h, velocity 1e-3 of the largest
    speed, C 1e-2 of max(|C|, |v| / h), F 1e-4."""
    from concurrent.futures import ThreadPoolExecutor

    from parity_tol import assert_rel_close

    drift = dict(position=1e-3, velocity=1e-3, affine=1e-2, deformation=1e-4)
    every = scenes.batch_scenes(256)
    pick = [49, 174, 6, 0, 1]
    scs = [every[k] for k in pick]
    assert scs[0].particles.count == 262144 and scs[0].info["resolution"] == 128
    assert scs[1].info["material"] == "fluid" and scs[1].particles.count == 238328
    steps = 100
    with ThreadPoolExecutor(max_workers=len(scs)) as pool:  # the oracle releases the GIL in its C calls
        expected = list(pool.map(lambda sc: oracle_run(sc, steps), scs))
    b = Batch()
    ids = [b.add_scene(sc.params, sc.particles, sc.dt) for sc in scs]
    b.run({i: steps for i in ids})
    for i, k, sc, e in zip(ids, pick, scs, expected):
        assert b.substeps(i) == steps
        got = b.particles(i)
        h = sc.params.cell_width
        assert_rel_close(e, got, h, drift, f"batch scene {k} vs oracle")
        assert_rel_close(alone(sc, steps), got, h, drift, f"batch scene {k} vs alone")
    b.close()
