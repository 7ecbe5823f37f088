"""GPU tests of the transfer kernels' launch shapes and of the tuner that picks
one (particles per CTA, CTAs per SM, grid block edge 4 or 8 cells).

Every shape must give the oracle's answer within the resident tolerances of
the reference (FP32 device vs f64 CPU after 8 substeps: position 2e-5,
velocity 2e-4, F 2e-4, gpu.rs:3699-3703; the affine bound is the dam-break
parity test's 2e-2); shapes differ from one another only by the f32 summation
order of the per-CTA partial sums.  A tuned session or batch must settle on a
shape after its first segments and keep tracking the oracle while it tries
them, since the trials are real work (up to 16 substeps there: twice the
8-substep bounds).
"""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200 import _native, scenes
from tessera_b200._abi import Obstacle
from tessera_b200.batch import Batch
from tessera_b200.session import Session

pytestmark = pytest.mark.gpu

SHAPES = range(6)


def assert_tracks(expected, actual, pos=2e-5, vel=2e-4, F=2e-4, C=2e-2):
    dp = np.linalg.norm(expected.position - actual.position, axis=1).max()
    dv = np.linalg.norm(expected.velocity - actual.velocity, axis=1).max()
    dF = np.linalg.norm((expected.deformation - actual.deformation).reshape(-1, 9), axis=1).max()
    dC = np.linalg.norm((expected.affine - actual.affine).reshape(-1, 9), axis=1).max()
    assert dp < pos and dv < vel and dF < F and dC < C, (dp, dv, dF, dC)


@pytest.fixture(scope="module")
def dam_break():
    """Dam-break physics (fluid column + elastic cubes) on ~118k particles and
    the oracle's states after 1..16 substeps."""
    sc = scenes.dam_break(scale=0.15)
    cpu = O.OracleWorld(sc.params, sc.particles)
    states = {}
    for k in range(1, 17):
        cpu.substep_fixed(sc.dt)
        states[k] = cpu.particles()
    return sc, states


@pytest.mark.parametrize("shape", SHAPES)
def test_every_launch_shape_tracks_the_oracle(dam_break, shape):
    sc, states = dam_break
    s = Session(sc.params, sc.particles, sc.dt, launch_shape=shape)
    s.step(8)
    assert_tracks(states[8], s.particles())
    info = s.launch_shape()
    assert info["shape"] == shape and info["shapes"][shape] == _native.launch_shapes()[shape]


def test_obstacle_and_obstacle_free_variants_agree(dam_break):
    """A session with a rigid sphere far outside the scene runs the kernels with
    the obstacle contact compiled in; without obstacles, the obstacle-free
    variants. No particle or node comes near the sphere, so both track the
    oracle and agree with each other to f32 rounding."""
    sc, states = dam_break
    runs = []
    for obstacles in ([], [Obstacle.sphere((50.0, 50.0, 50.0), 0.5)]):
        for shape in (0, 3):
            s = Session(sc.params, sc.particles, sc.dt, obstacles=obstacles, launch_shape=shape)
            s.step(8)
            runs.append(s.particles())
            assert_tracks(states[8], runs[-1])
    for plain, obst in zip(runs[:2], runs[2:]):
        assert np.abs(plain.position - obst.position).max() < 1e-6
        assert np.abs(plain.velocity - obst.velocity).max() < 1e-5


def test_one_substep_agrees_between_block_edges(dam_break):
    """The same CTA shape on 4^3 and on 8^3 blocks: both track the oracle, and
    they agree with each other to f32 summation order."""
    sc, states = dam_break
    runs = []
    for shape in (0, 3):
        s = Session(sc.params, sc.particles, sc.dt, launch_shape=shape)
        s.step(1)
        runs.append(s.particles())
        assert_tracks(states[1], runs[-1])
    assert np.abs(runs[0].position - runs[1].position).max() < 1e-6
    assert np.abs(runs[0].velocity - runs[1].velocity).max() < 1e-5


def test_tuned_session_settles_and_tracks_the_oracle(dam_break):
    sc, states = dam_break
    s = Session(sc.params, sc.particles, sc.dt)
    assert s.launch_shape()["shape"] is None
    # one substep per submit: two trials per candidate (each behind a re-sort
    # when the CTA size changes), then the chosen shape
    done = 0
    while s.launch_shape()["shape"] is None and done < 16:
        s.step(1)
        done += 1
    info = s.launch_shape()
    assert info["shape"] in SHAPES
    costs = info["ms_per_particle_substep"]
    measured = [c for c in costs if c is not None]
    assert len(measured) in (3, 6) and all(c > 0 for c in measured)
    assert costs[info["shape"]] == min(measured)
    assert_tracks(states[done], s.particles(), pos=4e-5, vel=4e-4, F=4e-4, C=4e-2)


def test_session_keeps_timing_and_challenges_after_the_choice(dam_break):
    """After the choice, a session stepping one 64-substep frame at a time keeps
    timing its segments and every sixth runs the best other shape, so the
    reported times move on from the trials' (a challenger's, and the chosen
    shape's recent mean); the shape in use stays a valid one and the state
    stays finite through the switches."""
    sc, _ = dam_break
    s = Session(sc.params, sc.particles, sc.dt)
    frames = 0
    while s.launch_shape()["shape"] is None and frames < 16:
        s.step(64)
        frames += 1
    assert s.launch_shape()["shape"] is not None
    first = list(s.launch_shape()["ms_per_particle_substep"])
    # a shape's first segments on each row buffer capture their graphs and are
    # not timed, so a challenge can take three segments: 20 frames hold one
    for _ in range(20):
        s.step(64)
    info = s.launch_shape()
    costs = info["ms_per_particle_substep"]
    moved = [k for k, (a, b) in enumerate(zip(first, costs)) if a is not None and b is not None and a != b]
    assert len(moved) >= 2, (first, costs)
    assert info["shape"] in SHAPES and costs[info["shape"]] is not None
    p = s.particles()
    assert np.isfinite(p.position).all() and np.isfinite(p.velocity).all()


def test_batches_under_each_shape_and_tuned_match_the_oracle_per_scene():
    pair = [scenes.batch_scene(21, cells=6), scenes.batch_scene(22, cells=9)]
    steps = (6, 4)
    expected = []
    for p, k in zip(pair, steps):
        w = O.OracleWorld(p.params, p.particles)
        for _ in range(k):
            w.substep_fixed(p.dt)
        expected.append(w.particles())
    for shape in list(SHAPES) + [None]:
        b = Batch(launch_shape=shape)
        ids = [b.add_scene(p.params, p.particles, p.dt) for p in pair]
        b.run({ids[0]: steps[0], ids[1]: steps[1]})
        for sid, exp in zip(ids, expected):
            assert_tracks(exp, b.particles(sid))
        if shape is not None:
            info = b.launch_shape()
            # an 8^3 shape without room in the pool runs the same CTA shape on 4^3 blocks
            assert info["shape"] in (shape, shape % 3)
        else:
            # keep submitting (one substep each) until the tuner has read its trials
            for _ in range(16):
                if b.launch_shape()["shape"] is not None:
                    break
                b.run({ids[0]: 1, ids[1]: 1})
            info = b.launch_shape()
            assert info["shape"] in SHAPES
            assert sum(c is not None for c in info["ms_per_particle_substep"]) in (3, 6)
        b.close()
