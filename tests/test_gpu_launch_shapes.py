"""GPU tests of the transfer kernels' launch shapes and of the tuner that picks
one (particles per CTA, CTAs per SM).

Every shape must give the oracle's answer within the resident tolerances of
the reference (FP32 device vs f64 CPU after 8 substeps: position 2e-5,
velocity 2e-4, F 2e-4, gpu.rs:3699-3703; the affine bound is the dam-break
parity test's 2e-2); shapes differ from one another only by the f32 summation
order of the per-CTA partial sums.  A tuned session or batch must settle on a
shape after its first segments and keep tracking the oracle while it tries
them, since the trials are real work.
"""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200 import _native, scenes
from tessera_b200.batch import Batch
from tessera_b200.session import Session

pytestmark = pytest.mark.gpu


def assert_tracks(expected, actual, pos=2e-5, vel=2e-4, F=2e-4, C=2e-2):
    dp = np.linalg.norm(expected.position - actual.position, axis=1).max()
    dv = np.linalg.norm(expected.velocity - actual.velocity, axis=1).max()
    dF = np.linalg.norm((expected.deformation - actual.deformation).reshape(-1, 9), axis=1).max()
    dC = np.linalg.norm((expected.affine - actual.affine).reshape(-1, 9), axis=1).max()
    assert dp < pos and dv < vel and dF < F and dC < C, (dp, dv, dF, dC)


@pytest.fixture(scope="module")
def dam_break_8():
    """Dam-break physics (fluid column + elastic cubes) on ~60k particles and the
    oracle's state after 8 substeps."""
    sc = scenes.dam_break(scale=0.15)
    cpu = O.OracleWorld(sc.params, sc.particles)
    for _ in range(8):
        cpu.substep_fixed(sc.dt)
    return sc, cpu.particles()


@pytest.mark.parametrize("shape", range(3))
def test_every_launch_shape_tracks_the_oracle(dam_break_8, shape):
    sc, expected = dam_break_8
    s = Session(sc.params, sc.particles, sc.dt, launch_shape=shape)
    s.step(8)
    assert_tracks(expected, s.particles())
    info = s.launch_shape()
    assert info["shape"] == shape and info["shapes"][shape] == _native.launch_shapes()[shape]


def test_tuned_session_settles_and_tracks_the_oracle(dam_break_8):
    sc, expected = dam_break_8
    s = Session(sc.params, sc.particles, sc.dt)
    assert s.launch_shape()["shape"] is None
    # one substep per submit: six trials (two per shape, each behind a re-sort
    # when the shape changes), then the chosen shape
    for _ in range(8):
        s.step(1)
    info = s.launch_shape()
    assert info["shape"] in range(3)
    costs = info["ms_per_particle_substep"]
    assert all(c is not None and c > 0 for c in costs)
    assert costs[info["shape"]] == min(costs)
    assert_tracks(expected, s.particles())


def test_batches_under_each_shape_and_tuned_match_the_oracle_per_scene():
    pair = [scenes.batch_scene(21, cells=6), scenes.batch_scene(22, cells=9)]
    steps = (6, 4)
    expected = []
    for p, k in zip(pair, steps):
        w = O.OracleWorld(p.params, p.particles)
        for _ in range(k):
            w.substep_fixed(p.dt)
        expected.append(w.particles())
    for shape in (0, 1, 2, None):
        b = Batch(launch_shape=shape)
        ids = [b.add_scene(p.params, p.particles, p.dt) for p in pair]
        b.run({ids[0]: steps[0], ids[1]: steps[1]})
        for sid, exp in zip(ids, expected):
            assert_tracks(exp, b.particles(sid))
        if shape is not None:
            assert b.launch_shape()["shape"] == shape
        else:
            # keep submitting (one substep each) until the tuner has read its six trials
            for _ in range(8):
                b.run({ids[0]: 1, ids[1]: 1})
            info = b.launch_shape()
            assert info["shape"] in range(3)
            assert all(c is not None for c in info["ms_per_particle_substep"])
        b.close()
