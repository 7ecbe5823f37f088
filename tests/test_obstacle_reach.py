"""The obstacle reach test of the fast fused transfer, checked on the CPU.

In a scene with rigid obstacles the fast transfer kernel keeps no contact code:
it tests each updated particle position against every obstacle's reach, a
local-frame box that holds the obstacle's surface (set per shape when the
obstacles are uploaded; the ground is a half-space below its plane), widened by
the particle radius, and defers a chunk with a particle inside some reach to
the general path, which has the contact.  That is only exact if a particle
outside every reach has no contact.  This test restates the rule and checks it
against the oracle's signed distance (RigidObstacle::surface, obstacle.rs:372-472)
for every shape, rotated, at points around and inside each obstacle: a point
outside the reach widened by r lies at least r from the surface.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import Obstacle


def quat(axis, angle):
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    s = math.sin(angle / 2)
    return (axis[0] * s, axis[1] * s, axis[2] * s, math.cos(angle / 2))


def rotate_inv(q, v):
    """v in the frame of the unit quaternion q (x, y, z, w)."""
    u = -np.asarray(q[:3])
    t = 2.0 * np.cross(u, v)
    return v + q[3] * t + np.cross(u, t)


def reach(o: Obstacle):
    """The local-frame half extents of the box that holds the surface, and whether
    the lower z bound is dropped (the ground)."""
    d = o.dims
    if o.shape == 0:  # sphere
        r = (d[0],) * 3
    elif o.shape == 1:  # box
        r = d
    elif o.shape == 2:  # capsule: segment of half height d0 along z, radius d1
        r = (d[1], d[1], d[0] + d[1])
    elif o.shape in (3, 4):  # cylinder, cone: half height d0 along z, radius d1
        r = (d[1], d[1], d[0])
    elif o.shape == 5:  # ground: the plane z = 0 over |x| <= d0, |y| <= d1, solid below
        return np.array([d[0], d[1], 0.0]) * (1 + 1e-4), True
    elif o.shape == 6:  # triangle prism: the vertices' radius plus the half thickness
        v = np.asarray(o.vertices).reshape(3, 3)
        r = (float(np.linalg.norm(v, axis=1).max()) + d[0],) * 3
    else:  # convex: the bounding radius
        r = (o.bound_radius,) * 3
    return np.asarray(r, dtype=np.float64) * (1 + 1e-4), False


def near(o: Obstacle, p, r):
    e, ground = reach(o)
    loc = rotate_inv(o.orientation, np.asarray(p) - np.asarray(o.center))
    return (abs(loc[0]) <= e[0] + r and abs(loc[1]) <= e[1] + r and loc[2] <= e[2] + r
            and (ground or loc[2] >= -e[2] - r))


def shapes():
    q = quat((1.0, 2.0, 0.5), 0.7)
    c = (0.3, -0.2, 0.5)
    cube = [(x, y, z) for x in (-0.2, 0.2) for y in (-0.2, 0.2) for z in (-0.2, 0.2)]
    normals = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    return [
        Obstacle.sphere(c, 0.25),
        Obstacle.cuboid(c, (0.3, 0.1, 0.2), q),
        Obstacle.capsule(c, 0.3, 0.1, q),
        Obstacle.cylinder(c, 0.25, 0.15, q),
        Obstacle.cone(c, 0.25, 0.2, q),
        Obstacle.ground(c, (0.4, 0.3), q),
        Obstacle.triangle_prism(c, [(0.0, -0.3, -0.2), (0.0, 0.3, -0.2), (0.0, 0.0, 0.3)], 0.05, q),
        Obstacle.convex(c, cube, normals, q),
    ]


@pytest.mark.parametrize("o", shapes(), ids=lambda o: f"shape{o.shape}")
def test_points_outside_the_reach_have_no_contact(o):
    rng = np.random.default_rng(o.shape)
    c = np.asarray(o.center)
    pts = c + rng.uniform(-0.8, 0.8, size=(3000, 3))
    outside = 0
    for p in pts:
        for r in (0.005, 0.02):
            if not near(o, p, r):
                outside += 1
                d, _ = O.obstacle_surface(o, p)
                assert d >= r, (o.shape, p, r, d)
    # the reach is not trivially everywhere
    assert outside > 500
