"""GPU tests of CPIC (compatible particle-in-cell) on the device: the grid
namespace of a particle includes the side mask of each CPIC group's closest
triangle prism (transfer_key, world.rs:470-490; the reference shader computes
the same mask per substep, gpu.wgsl:82-131), so material on opposite sides of a
thin sheet does not exchange momentum through shared grid nodes.

The first test is the reference's own scene (world.rs:720-781) run through the
resident path; the second compares a block straddling a sheet with the f64
oracle under the resident tolerances (gpu.rs:3699-3703).
"""

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200 import scenes
from tessera_b200._abi import (
    BOUNDARY_NON_REFLECTING, MAT_ELASTIC, TMPM_ERR_RESIDENT_UNAVAILABLE, Obstacle, ParticleArrays,
    density_particles, make_params,
)
from tessera_b200.session import Session, TesseraError

pytestmark = pytest.mark.gpu


def sheet(group, center=(0.5, 0.5, 0.5), half=0.001):
    return Obstacle.triangle_prism(center, [(0.0, -1.0, -1.0), (0.0, 1.0, -1.0), (0.0, 0.0, 1.0)], half,
                                   cpic_group=group, boundary=BOUNDARY_NON_REFLECTING)


def two_particles():
    left = density_particles([(0.48, 0.5, 0.5)], 0.005, 1000.0, MAT_ELASTIC, (1000.0, 0.2))
    left.velocity[0, 0] = -1.0
    right = left.copy()
    right.position[0, 0] = 0.52
    right.velocity[0, 0] = 1.0
    return ParticleArrays.concat([left, right])


def test_cpic_sheet_separates_opposite_sides_like_the_reference():  # world.rs:720-781
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0), max_substep=1e-3)
    parts = two_particles()
    separated = Session(params, parts, 1e-3, obstacles=[sheet(0)])
    separated.step_cfl(0.001)
    v = separated.particles().velocity
    assert v[0, 0] < -0.9 and v[1, 0] > 0.9
    disabled = Session(params, parts, 1e-3, obstacles=[sheet(0)], use_cpic=False)
    disabled.step_cfl(0.001)
    v = disabled.particles().velocity
    assert abs(v[0, 0]) < 0.5 and abs(v[1, 0]) < 0.5
    explicit = parts.copy()
    explicit.transfer_color[1] = 1
    coloured = Session(params, explicit, 1e-3, obstacles=[sheet(0)], use_cpic=False)
    coloured.step_cfl(0.001)
    v = coloured.particles().velocity
    assert v[0, 0] < -0.9 and v[1, 0] > 0.9
    mixed = Session(params, parts, 1e-3, obstacles=[sheet(-1)])
    mixed.step_cfl(0.001)
    v = mixed.particles().velocity
    assert abs(v[0, 0]) < 0.5 and abs(v[1, 0]) < 0.5
    # the oracle agrees on each case
    for obs, cpic, p, got in ((sheet(0), True, parts, separated), (sheet(0), False, parts, disabled),
                              (sheet(0), False, explicit, coloured), (sheet(-1), True, parts, mixed)):
        w = O.OracleWorld(params, p)
        w.set_obstacles([obs])
        w.set_use_cpic(cpic)
        w.step(0.001)
        d = np.abs(w.particles().velocity - got.particles().velocity).max()
        assert d < 2e-4, d


def test_block_across_a_cpic_sheet_matches_oracle():
    h = 1.0 / 32
    r = h / 4
    rng = np.random.default_rng(9)
    pos = scenes.lattice((0.40, 0.40, 0.40), (0.60, 0.52, 0.52), 2 * r, rng, 0.5)
    pos = pos[np.abs(pos[:, 0] - 0.5) > 0.004]  # nothing inside the sheet itself
    parts = density_particles(pos, r, 1000.0, MAT_ELASTIC, (2e3, 0.25))
    parts.velocity[:, 0] = np.where(pos[:, 0] < 0.5, 0.3, -0.3)  # both halves push against the sheet
    params = make_params(h, gravity=(0.0, 0.0, -9.81), max_substep=1e-3, bounds=((0, 0, 0), (1, 1, 1)))
    obstacles = [sheet(0, center=(0.5, 0.46, 0.46), half=0.002)]
    s = Session(params, parts, 1e-4, obstacles=obstacles)
    w = O.OracleWorld(params, parts)
    w.set_obstacles(obstacles)
    s.step(8)
    for _ in range(8):
        w.substep_fixed(1e-4)
    got, exp = s.particles(), w.particles()
    dp = np.linalg.norm(got.position - exp.position, axis=1).max()
    dv = np.linalg.norm(got.velocity - exp.velocity, axis=1).max()
    assert dp < 2e-5 and dv < 2e-4, (dp, dv)
    # without CPIC the two halves share grid nodes through the sheet: a different answer
    s2 = Session(params, parts, 1e-4, obstacles=obstacles, use_cpic=False)
    s2.step(8)
    assert np.linalg.norm(s2.particles().velocity - got.velocity, axis=1).max() > 1e-3


def test_cpic_cases_beyond_the_device_namespace_need_the_cpu_path():
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0), max_substep=1e-3)
    parts = two_particles()
    with pytest.raises(TesseraError) as e:
        Session(params, parts, 1e-3, obstacles=[sheet(9)])
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE
    coloured = parts.copy()
    coloured.transfer_color[:] = 300
    with pytest.raises(TesseraError) as e:
        Session(params, coloured, 1e-3, obstacles=[sheet(0)])
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE
    Session(params, coloured, 1e-3, obstacles=[sheet(0)], use_cpic=False)  # fine without CPIC
