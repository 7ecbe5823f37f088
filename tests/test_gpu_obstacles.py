"""GPU parity for every rigid-obstacle shape and boundary mode the device
compiles, and for sticky walls.

The reference defines the shapes and modes in obstacle.rs:10-77, the signed
surface distance per shape in obstacle.rs:373 (`surface`), the contact
velocity per boundary mode in obstacle.rs:507-540 (`contact_velocity`), the
grid contact with its reaction impulse in world.rs:561-603, and the shader
twins in gpu.wgsl:259-414.  Each test drives a small elastic block (h = 0.02,
8 particles per cell) into one obstacle through the resident session and
compares it with the f64 oracle:

* particles after 12 substeps under the reference's resident tolerances
  (gpu.rs:3699-3703: position 2e-5, velocity 2e-4, F 2e-4, affine 2e-3);
* one CFL-split step with obstacle reactions (linear impulse and moment about
  the obstacle centre) against `step_with_obstacle_reactions`, within 1e-4
  relative to the largest reaction component (the reference's reaction test
  uses 1e-4, gpu.rs:2602-2649).

Every obstacle is rotated and moving, so the body-frame transforms and the
obstacle's own velocity enter the contact.  Each scene is checked on the
oracle to actually touch the obstacle (non-zero reactions), so no test passes
by missing it.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import (
    BOUNDARY_FREE_SLIP, BOUNDARY_NON_REFLECTING, BOUNDARY_SEPARATE, BOUNDARY_SLIP, BOUNDARY_STICK, MAT_ELASTIC,
    Obstacle, density_particles, make_params,
)
from tessera_b200.session import Session

pytestmark = pytest.mark.gpu

H = 0.02
DT = 2e-4
BOUNDS = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))


def quat(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    s = math.sin(angle / 2.0)
    return (axis[0] * s, axis[1] * s, axis[2] * s, math.cos(angle / 2.0))


def falling_block(lo=(0.44, 0.44, 0.40), cells=(5, 5, 4), velocity=(0.3, -0.2, -1.5), seed=5):
    """An elastic block of 8 particles per cell moving down onto the obstacle below it."""
    rng = np.random.default_rng(seed)
    r = H / 4.0
    lo = np.asarray(lo)
    axes = [lo[a] + 2.0 * r * (np.arange(2 * cells[a]) + 0.5) for a in range(3)]
    pos = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    pos = pos + rng.uniform(-0.25 * r, 0.25 * r, size=pos.shape)
    p = density_particles(pos, r, 1000.0, MAT_ELASTIC, (1.0e4, 0.2), velocity=velocity)
    return p


ROT = quat((1.0, 2.0, 0.5), 0.35)
MOVING = dict(linear_velocity=(0.1, 0.05, 0.2), angular_velocity=(0.3, -0.2, 0.5))

# Each obstacle's top surface sits a little below the block's bottom face (z = 0.40).
SHAPES = {
    "sphere": lambda **kw: Obstacle.sphere((0.49, 0.49, 0.27), 0.12, **kw),
    "box": lambda **kw: Obstacle.cuboid((0.49, 0.49, 0.30), (0.15, 0.12, 0.085), orientation=ROT, **kw),
    "ground": lambda **kw: Obstacle.ground((0.49, 0.49, 0.385), (0.4, 0.4), orientation=quat((1, 0, 0), 0.1),
                                           **kw),
    "capsule": lambda **kw: Obstacle.capsule((0.49, 0.49, 0.33), 0.10, 0.06, orientation=quat((1, 0, 0), 1.4),
                                             **kw),
    "cylinder": lambda **kw: Obstacle.cylinder((0.49, 0.49, 0.32), 0.07, 0.15, orientation=ROT, **kw),
    "cone": lambda **kw: Obstacle.cone((0.49, 0.49, 0.32), 0.07, 0.15, orientation=quat((0, 1, 0), 0.2), **kw),
    "triangle_prism": lambda **kw: Obstacle.triangle_prism(
        (0.49, 0.49, 0.37), [(-0.2, -0.2, 0.0), (0.25, -0.15, 0.0), (0.0, 0.25, 0.0)], 0.012,
        orientation=quat((0, 1, 1), 0.15), **kw),
    "convex": lambda **kw: convex_wedge(**kw),
}


def convex_wedge(**kw):
    """A convex hull (a wedge: 6 vertices, 5 faces) through RigidObstacle::convex's planes."""
    verts = [(-0.15, -0.15, -0.06), (0.15, -0.15, -0.06), (-0.15, 0.15, -0.06), (0.15, 0.15, -0.06),
             (-0.15, 0.0, 0.05), (0.15, 0.0, 0.05)]
    n1 = np.array([0.0, -0.11, 0.15])
    n2 = np.array([0.0, 0.11, 0.15])
    normals = [(0, 0, -1), (1, 0, 0), (-1, 0, 0), tuple(n1 / np.linalg.norm(n1)), tuple(n2 / np.linalg.norm(n2))]
    return Obstacle.convex((0.49, 0.49, 0.335), verts, normals, orientation=quat((0, 0, 1), 0.3), **kw)


def run_pair(obstacle, params=None, parts=None, substeps=12):
    params = params or make_params(H, bounds=BOUNDS)
    parts = parts if parts is not None else falling_block()
    cpu = O.OracleWorld(params, parts)
    cpu.set_obstacles([obstacle])
    s = Session(params, parts, DT, obstacles=[obstacle])
    for _ in range(substeps):
        cpu.substep_fixed(DT)
    s.step(substeps)
    return cpu, s


def assert_resident_close(cpu, s):
    e, g = cpu.particles(), s.particles()
    dp = np.linalg.norm(e.position - g.position, axis=1).max()
    dv = np.linalg.norm(e.velocity - g.velocity, axis=1).max()
    dF = np.linalg.norm((e.deformation - g.deformation).reshape(-1, 9), axis=1).max()
    dC = np.linalg.norm((e.affine - g.affine).reshape(-1, 9), axis=1).max()
    assert dp < 2e-5 and dv < 2e-4 and dF < 2e-4 and dC < 2e-3, (dp, dv, dF, dC)


def assert_reactions_close(obstacle, params=None, parts=None, dt=1e-3):
    params = params or make_params(H, bounds=BOUNDS)
    parts = parts if parts is not None else falling_block()
    cpu = O.OracleWorld(params, parts)
    cpu.set_obstacles([obstacle])
    expected = cpu.step_with_obstacle_reactions(dt, 1)
    s = Session(params, parts, DT, obstacles=[obstacle])
    got = s.step_cfl_with_reactions(dt)
    assert s.substeps() == cpu.substeps()
    if obstacle.boundary == BOUNDARY_NON_REFLECTING:
        # the contact keeps the velocity (obstacle.rs:507-540): no impulse at all,
        # but the particles are still pushed out of the surface
        assert not np.any(expected) and not np.any(got)
        moved = np.linalg.norm(cpu.particles().position - parts.position - dt * parts.velocity, axis=1)
        assert moved.max() > 1e-4, "the scene does not touch the obstacle"
        return
    scale = np.abs(expected).max()
    assert scale > 0.0, "the scene does not touch the obstacle"
    assert np.abs(expected - got).max() < 1e-4 * scale, (expected, got)


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_obstacle_shape_matches_oracle(shape):
    obstacle = SHAPES[shape](friction=0.3, **MOVING)
    assert_reactions_close(obstacle)
    cpu, s = run_pair(obstacle)
    assert_resident_close(cpu, s)


@pytest.mark.parametrize("mode", [BOUNDARY_SLIP, BOUNDARY_STICK, BOUNDARY_SEPARATE, BOUNDARY_NON_REFLECTING,
                                  BOUNDARY_FREE_SLIP])
def test_obstacle_boundary_mode_matches_oracle(mode):
    obstacle = SHAPES["box"](friction=0.4, boundary=mode, **MOVING)
    assert_reactions_close(obstacle)
    cpu, s = run_pair(obstacle)
    assert_resident_close(cpu, s)


def test_sticky_walls_match_oracle():
    """wall_mode = 1: a node within one cell of a wall loses its whole velocity
    (separating walls, the reference's only kind, zero only the inward normal
    component, world.rs:561-575).  A block sliding along the floor and into the
    x wall under both modes: the modes differ, and each matches the oracle."""
    parts = falling_block(lo=(0.86, 0.44, 0.025), cells=(5, 5, 3), velocity=(1.0, 0.4, -0.5))
    got = {}
    for mode in (0, 1):
        params = make_params(H, bounds=BOUNDS, wall_mode=mode)
        cpu = O.OracleWorld(params, parts)
        s = Session(params, parts, DT)
        for _ in range(12):
            cpu.substep_fixed(DT)
        s.step(12)
        assert_resident_close(cpu, s)
        got[mode] = s.particles().velocity
    # sticky walls stop the tangential slide of the particles next to the walls
    assert np.abs(got[0] - got[1]).max() > 1e-2
