"""The P2G scatter where a per-CTA fixed-point scale can fail: one particle of
a CTA moving 10^3-10^4 times faster than its 255 neighbours.

The scatter accumulates each CTA's contributions in 32-bit fixed point with
one power-of-two scale per quantity, set by the sum of the CTA's particle
bounds.  A single fast particle would set that scale by itself and coarsen the
quantum of every node its slow neighbours reach; a CTA in which one particle's
mass or momentum bound exceeds 1/8 of the CTA's total therefore scatters
through the direct path instead (f32 global atomics per node, each node
accurate relative to its own magnitude, as in the reference's shader).  The
scene is one 256-particle CTA (a 16 x 8 x 2 lattice of 8 particles per cell,
h = 0.02) moving coherently at |u| ~ 1.1e-3 m/s, with one particle at the
x-low end moving 10^3 or 10^4 |u|.

Checks, against the f64 oracle's P2G (world.rs:378-399) and substep:
  * every grid node's mass and momentum within 1e-5 of the largest node value
    (the grid tolerance of the other P2G parity tests), and mass and momentum
    conserved;
  * after one substep, the velocity of every slow particle whose stencil does
    not reach the fast particle's within 1e-5 |u| of the oracle.  A per-CTA
    scale set by the fast particle misses this bar at 10^4 (an emulation of
    that scatter in f64 gives 3.4e-5 |u|).
"""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import MAT_ELASTIC, density_particles, make_params
from tessera_b200.session import Session

pytestmark = pytest.mark.gpu

H = 0.02
FAST = 5


def one_cta_scene(ratio, seed=3):
    rng = np.random.default_rng(seed)
    r = H / 4.0
    axes = [0.4 + 2.0 * r * (np.arange(n) + 0.5) for n in (16, 8, 2)]
    pos = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    pos = pos + rng.uniform(-0.25 * r, 0.25 * r, size=pos.shape)
    assert len(pos) == 256  # one CTA of the 256-particle launch shape
    u = np.array([1e-3, 5e-4, 0.0])
    vel = np.tile(u, (256, 1)) * (1.0 + rng.uniform(-0.1, 0.1, size=(256, 1)))
    vel[FAST] = ratio * np.linalg.norm(u) * np.array([0.6, -0.8, 0.0])
    p = density_particles(pos, r, 1000.0, MAT_ELASTIC, (1.0e4, 0.2))
    p.velocity[:] = vel
    return p, np.linalg.norm(u)


@pytest.mark.parametrize("ratio", [1e3, 1e4])
def test_fast_particle_does_not_coarsen_its_neighbours(ratio):
    params = make_params(H, gravity=(0.0, 0.0, 0.0), bounds=((0, 0, 0), (1, 1, 1)))
    parts, speed = one_cta_scene(ratio)
    dt = 1e-5
    s = Session(params, parts, dt, launch_shape=0)  # 256 particles per CTA: the whole scene is one CTA
    cells, mm = s.debug_p2g()
    cpu = O.OracleWorld(params, parts)
    keys, vals = cpu.p2g(dt)
    order = np.lexsort((cells[:, 2], cells[:, 1], cells[:, 0]))
    cells, mm = cells[order], mm[order].astype(np.float64)
    assert np.array_equal(cells, keys[:, :3].astype(np.int32))
    assert np.abs(mm[:, 0] - vals[:, 0]).max() < 1e-5 * vals[:, 0].max()
    assert np.abs(mm[:, 1:] - vals[:, 1:]).max() < 1e-5 * np.abs(vals[:, 1:]).max()
    assert abs(mm[:, 0].sum() - parts.mass.sum()) < 1e-6 * parts.mass.sum()
    momentum = (parts.mass[:, None] * parts.velocity).sum(axis=0)
    assert np.abs(mm[:, 1:].sum(axis=0) - momentum).max() < 1e-6 * np.abs(momentum).max()

    s.step(1)
    cpu.substep_fixed(dt)
    b = np.floor(parts.position / H - 0.5).astype(int)
    far = np.abs(b - b[FAST]).max(axis=1) > 2
    assert far.sum() > 150
    dv = np.linalg.norm(s.particles().velocity - cpu.particles().velocity, axis=1)
    assert dv[far].max() < 1e-5 * speed, dv[far].max() / speed
    assert dv[FAST] < 1e-5 * ratio * speed
