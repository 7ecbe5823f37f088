"""CPU tests of the rigid-coupling restatement the GPU tests check against
(the MPM-owned two-way coupling: gpu_rigid_sync.wgsl:46-61,
gpu_rigid_reaction.wgsl:71-150), on closed-form cases, and of the C structs."""

import ctypes as C

import numpy as np

from oracle import oracle as O
from tessera_b200._abi import Obstacle, TmpmRigidBody, TmpmRigidMapping


def body(**kw):
    b = dict(position=np.zeros(3), inverse_mass=1.0, orientation=np.array([0.0, 0.0, 0.0, 1.0]),
             linear_velocity=np.zeros(3), angular_velocity=np.zeros(3), inverse_inertia=np.ones(3))
    b.update({k: (np.asarray(v, dtype=np.float64) if not np.isscalar(v) else v) for k, v in kw.items()})
    return b


def test_struct_layouts_match_header():
    assert C.sizeof(TmpmRigidBody) == 17 * 8
    assert C.sizeof(TmpmRigidMapping) == 8 + 7 * 8


def test_free_body_integrates_gravity_then_pose():
    b = [body(linear_velocity=[1.0, 0.0, 0.0])]
    obs = [Obstacle.sphere((0.0, 0.0, 0.0), 0.1)]
    maps = [(0, np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))]
    out = O.rigid_apply(b, maps, obs, np.zeros((1, 6)), 0.01, gravity=(0.0, 0.0, -10.0))
    assert np.allclose(out[0]["linear_velocity"], [1.0, 0.0, -0.1])
    assert np.allclose(out[0]["position"], [0.01, 0.0, -0.001])
    assert np.allclose(out[0]["orientation"], [0.0, 0.0, 0.0, 1.0])


def test_impulses_change_linear_and_angular_velocity():
    # impulse J through an obstacle 0.5 m from the body centre along x, J along y
    b = [body(inverse_mass=0.5, inverse_inertia=[1.0, 2.0, 4.0])]
    obs = [Obstacle.sphere((0.5, 0.0, 0.0), 0.1)]
    maps = [(0, np.array([0.5, 0.0, 0.0]), np.array([0.0, 0.0, 0.0, 1.0]))]
    r = np.array([[0.0, 2.0, 0.0, 0.0, 0.0, 0.1]])
    out = O.rigid_apply(b, maps, obs, r, 0.01, integrate_pose=False)
    assert np.allclose(out[0]["linear_velocity"], [0.0, 1.0, 0.0])
    # torque (0, 0, 0.1 + 0.5 * 2) in an unrotated body: dw = I^-1 tau = 4 * 1.1
    assert np.allclose(out[0]["angular_velocity"], [0.0, 0.0, 4.4])
    assert np.allclose(out[0]["position"], 0.0)


def test_rotated_body_uses_world_frame_inertia():
    # a quarter turn about z maps the body's x axis to world y: world torque about y
    # meets the body-frame x inverse inertia
    s = np.sqrt(0.5)
    b = [body(orientation=[0.0, 0.0, s, s], inverse_inertia=[3.0, 5.0, 7.0])]
    obs = [Obstacle.sphere((0.0, 0.0, 0.0), 0.1)]
    maps = [(0, np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))]
    out = O.rigid_apply(b, maps, obs, np.array([[0.0, 0.0, 0.0, 0.0, 1.0, 0.0]]), 0.01, integrate_pose=False)
    assert np.allclose(out[0]["angular_velocity"], [0.0, 3.0, 0.0])


def test_static_and_unmapped_bodies_and_speed_limit():
    b = [body(inverse_mass=0.0), body(), body(linear_velocity=[3.0, 4.0, 0.0])]
    obs = [Obstacle.sphere((0.0, 0.0, 0.0), 0.1), Obstacle.sphere((1.0, 0.0, 0.0), 0.1)]
    maps = [(0, np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0])), (2, np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))]
    r = np.array([[1.0, 0.0, 0.0, 0.0, 0.0, 0.0], [0.0, 0.0, 0.0, 0.0, 0.0, 0.0]])
    out = O.rigid_apply(b, maps, obs, r, 0.1, max_speed=1.0)
    assert np.allclose(out[0]["linear_velocity"], 0.0)  # static: impulse ignored
    assert np.allclose(out[1]["position"], 0.0)  # unmapped: not integrated
    assert np.allclose(out[2]["linear_velocity"], [0.6, 0.8, 0.0])  # clamped to 1 m/s


def test_sync_places_obstacles_in_the_body_frame():
    s = np.sqrt(0.5)
    b = [body(position=[1.0, 2.0, 3.0], orientation=[0.0, 0.0, s, s], angular_velocity=[0.0, 0.0, 2.0],
              linear_velocity=[0.1, 0.0, 0.0])]
    obs = [Obstacle.sphere((0.0, 0.0, 0.0), 0.1), Obstacle.sphere((5.0, 5.0, 5.0), 0.1)]
    maps = [(0, np.array([1.0, 0.0, 0.0]), np.array([0.0, 0.0, 0.0, 1.0])),
            (-1, np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))]
    out = O.rigid_sync(b, maps, obs)
    assert np.allclose(out[0].center, [1.0, 3.0, 3.0])  # body x axis -> world y
    assert np.allclose(out[0].linear_velocity, [0.1 - 2.0, 0.0, 0.0])  # v + w x offset
    assert np.allclose(out[0].orientation, [0.0, 0.0, s, s])
    assert out[1].center == (5.0, 5.0, 5.0)
