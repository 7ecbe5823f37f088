"""GPU tests of the MPM-owned two-way rigid coupling (GpuRigidMpmCoupler::
step_mpm_owned, crates/tessera-mpm/src/gpu_rigid_sync.rs:187-214): an elastic
block pushes a sphere obstacle carried by a free body.  The device run is
compared with the f64 oracle driven substep by substep: obstacle pose from the
body (gpu_rigid_sync.wgsl:46-61), one substep with obstacle reactions, the
impulses applied to the body (gpu_rigid_reaction.wgsl:71-150).

Tolerances: particles as the resident parity tests after 8 substeps (position
2e-5, velocity 2e-4, gpu.rs:3699-3703); the body's velocity, the sum of the
impulses times 1/m, to 1e-3 of its change (f32 accumulation of the impulses on
the device against f64), its position to 5e-7 (a few f32 ulps at 0.5).
"""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200 import scenes
from tessera_b200._abi import (
    MAT_ELASTIC, TMPM_ERR_INVALID_INPUT, Obstacle, TmpmRigidBody, TmpmRigidMapping, density_particles, make_params,
)
from tessera_b200.session import Session, TesseraError

pytestmark = pytest.mark.gpu

DT = 1e-4


def scene(offset=(0.0, 0.0, 0.0)):
    h = 1.0 / 32
    r = h / 4
    rng = np.random.default_rng(4)
    pos = scenes.lattice((0.30, 0.42, 0.42), (0.385, 0.58, 0.58), 2 * r, rng, 0.5)
    parts = density_particles(pos, r, 1000.0, MAT_ELASTIC, (2e3, 0.25))
    parts.velocity[:, 0] = 0.5
    params = make_params(h, gravity=(0.0, 0.0, 0.0), max_substep=1e-3, bounds=((0, 0, 0), (1, 1, 1)))
    center = np.array([0.5, 0.5, 0.5]) + np.asarray(offset)
    return params, parts, center


def run_oracle(params, parts, obstacles, bodies, maps, steps, gravity=(0.0, 0.0, 0.0)):
    w = O.OracleWorld(params, parts)
    for _ in range(steps):
        obstacles = O.rigid_sync(bodies, maps, obstacles)
        w.set_obstacles(obstacles)
        r = w.substep_fixed(DT, reactions_count=len(obstacles))
        bodies = O.rigid_apply(bodies, maps, obstacles, r, DT, gravity=gravity)
    return w.particles(), bodies


def test_block_pushes_a_free_sphere_like_the_oracle():
    params, parts, center = scene(offset=(0.0, 0.01, 0.0))  # off-centre: the contact also spins the body
    sphere = Obstacle.sphere(tuple(center - [0.0, 0.01, 0.0]), 0.1)
    body = TmpmRigidBody.make(center, 2.0, inverse_inertia=(500.0, 500.0, 500.0))
    mapping = TmpmRigidMapping.make(0, local_center=(0.0, -0.01, 0.0))
    s = Session(params, parts, DT, obstacles=[sphere])
    s.rigid_attach([body], [mapping])
    s.rigid_step(8)
    got = s.particles()
    dev = s.rigid_bodies()[0].as_dict()
    exp_parts, exp_bodies = run_oracle(params, parts, [sphere], [body.as_dict()],
                                       [(0, np.array([0.0, -0.01, 0.0]), np.array([0.0, 0.0, 0.0, 1.0]))], 8)
    e = exp_bodies[0]
    assert e["linear_velocity"][0] > 0.1  # the block pushed the sphere along +x
    assert np.linalg.norm(got.position - exp_parts.position, axis=1).max() < 2e-5
    assert np.linalg.norm(got.velocity - exp_parts.velocity, axis=1).max() < 2e-4
    dv = np.abs(dev["linear_velocity"] - e["linear_velocity"]).max()
    assert dv <= 1e-3 * np.abs(e["linear_velocity"]).max(), (dev["linear_velocity"], e["linear_velocity"])
    assert np.abs(dev["angular_velocity"] - e["angular_velocity"]).max() <= 1e-3 * np.abs(
        e["angular_velocity"]).max() + 1e-6
    assert np.abs(dev["position"] - e["position"]).max() < 5e-7  # f32 positions near 0.5: ulp 6e-8
    assert abs(np.linalg.norm(dev["orientation"]) - 1.0) < 1e-6


def test_static_obstacle_and_body_under_gravity():
    """A body with no contact falls freely (v += g dt, x += v dt each substep);
    an obstacle mapped to no body keeps its pose, so the run equals the plain
    session with that obstacle."""
    params, parts, center = scene()
    fixed = Obstacle.sphere((0.5, 0.5, 0.5), 0.1)
    far = Obstacle.sphere((0.8, 0.8, 0.8), 0.02)
    body = TmpmRigidBody.make((0.8, 0.8, 0.8), 1.0, linear_velocity=(0.0, 0.0, 0.2),
                              inverse_inertia=(1.0, 1.0, 1.0))
    s = Session(params, parts, DT, obstacles=[fixed, far])
    s.rigid_attach([body], [TmpmRigidMapping.make(-1), TmpmRigidMapping.make(0)])
    s.rigid_step(10, gravity=(0.0, 0.0, -9.8))
    b = s.rigid_bodies()[0].as_dict()
    vz, z = 0.2, 0.8
    for _ in range(10):
        vz -= 9.8 * DT
        z += vz * DT
    assert abs(b["linear_velocity"][2] - vz) < 1e-6 and abs(b["position"][2] - z) < 1e-6
    plain = Session(params, parts, DT, obstacles=[fixed, far])
    plain.step(10)
    d = np.abs(plain.particles().position - s.particles().position).max()
    assert d < 1e-6, d


def test_attach_rejects_inconsistent_input():
    params, parts, center = scene()
    s = Session(params, parts, DT, obstacles=[Obstacle.sphere((0.5, 0.5, 0.5), 0.1)])
    body = TmpmRigidBody.make(center, 1.0, inverse_inertia=(1.0, 1.0, 1.0))
    for bodies, maps in (([body], []),  # one mapping per obstacle
                         ([body], [TmpmRigidMapping.make(3)]),  # no body 3
                         ([TmpmRigidBody.make(center, 1.0, orientation=(0.0, 0.0, 0.0, 2.0))],
                          [TmpmRigidMapping.make(0)])):  # not a unit quaternion
        with pytest.raises(TesseraError) as e:
            s.rigid_attach(bodies, maps)
        assert e.value.status == TMPM_ERR_INVALID_INPUT
    with pytest.raises(TesseraError) as e:
        s.rigid_step(1)  # nothing attached for this obstacle set
    assert e.value.status == TMPM_ERR_INVALID_INPUT


def one_particle(x, vx=0.0):
    p = density_particles([x], 0.04, 1000.0, MAT_ELASTIC, (1000.0, 0.2))
    p.velocity[0, 0] = vx
    return p


def unit_sphere_bodies(xs, **kw):
    bodies = [TmpmRigidBody.make((x, 0.0, 0.0), 1.0, inverse_inertia=(1.0, 1.0, 1.0), **kw) for x in xs]
    obstacles = [Obstacle.sphere((x, 0.0, 0.0), 1.0) for x in xs]
    maps = [TmpmRigidMapping.make(i) for i in range(len(xs))]
    return bodies, obstacles, maps


def test_mpm_owned_step_integrates_rigid_pose():  # gpu_rigid_sync.rs:607-668
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0))
    bodies, obstacles, maps = unit_sphere_bodies([0.0], linear_velocity=(1.0, 0.0, 0.0),
                                                 angular_velocity=(0.0, 0.0, 1.0))
    s = Session(params, one_particle((3.0, 0.0, 0.0)), 0.001, obstacles=obstacles)
    s.rigid_attach(bodies, maps)
    s.rigid_step(1, gravity=(0.0, 0.0, -9.81))
    first = s.rigid_bodies()[0].as_dict()
    assert abs(first["position"][0] - 0.001) < 1e-6
    assert abs(first["position"][2] + 9.81e-6) < 1e-7
    assert abs(first["orientation"][2] - 0.0005) < 1e-6
    s.rigid_step(1, gravity=(0.0, 0.0, -9.81))
    second = s.rigid_bodies()[0].as_dict()
    assert second["position"][0] > first["position"][0] and second["orientation"][2] > first["orientation"][2]


def test_mpm_owned_step_caps_speed_before_pose_integration():  # gpu_rigid_sync.rs:671-724
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0))
    bodies, obstacles, maps = unit_sphere_bodies([0.0], linear_velocity=(2.0, 0.0, 0.0))
    s = Session(params, one_particle((3.0, 0.0, 0.0)), 0.001, obstacles=obstacles)
    s.rigid_attach(bodies, maps)
    s.rigid_step(1, max_linear_speed=0.5)
    b = s.rigid_bodies()[0].as_dict()
    assert abs(b["linear_velocity"][0] - 0.5) < 1e-5 and abs(b["position"][0] - 0.0005) < 1e-6


@pytest.mark.parametrize("count", [1, 17, 70])
def test_two_way_reaction_reaches_its_body(count):  # gpu_rigid_sync.rs:727-858
    """A particle moving into the last of `count` unit spheres (the others far
    away): only that body takes the impulse; the particle slows down."""
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0))
    xs = [10.0 + 3.0 * k for k in range(count - 1)] + [0.0]
    bodies, obstacles, maps = unit_sphere_bodies(xs)
    s = Session(params, one_particle((1.02, 0.0, 0.0), vx=-1.0), 0.001, obstacles=obstacles)
    s.rigid_attach(bodies, maps)
    s.rigid_step(1, integrate_pose=False)
    states = [b.as_dict() for b in s.rigid_bodies()]
    assert all(abs(b["linear_velocity"][0]) < 1e-6 for b in states[:-1])
    assert states[-1]["linear_velocity"][0] < -0.01, states[-1]
    assert states[-1]["position"][0] == 0.0  # velocities only: the rigid solver integrates
    assert s.particles().velocity[0, 0] > -1.0
    assert s.substeps() == 1
