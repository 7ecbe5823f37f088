"""Plastic materials on the device (snow, sand, Neo-Hookean sand) against the
CPU oracle, on the reference's own scenes and tolerances:
  * gpu_corotated_stress_tracks_cpu_for_elastic_sand_and_snow (gpu.rs:4423-4516):
    12 direct steps, position 2e-5, velocity 3e-4, F 2e-4, plastic_det 2e-4;
  * sand_neo_hookean_gpu_matches_cpu_direct_and_resident (gpu.rs:2339-2446):
    4 substeps direct and resident, position 2e-5, velocity 3e-4, affine 2e-3,
    F 2e-4, plastic state 2e-4.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import (
    MAT_ELASTIC, MAT_SAND, MAT_SAND_NEO_HOOKEAN, MAT_SNOW, ParticleArrays, density_particles, make_params,
)
from tessera_b200.session import Session

pytestmark = pytest.mark.gpu
DEG = math.pi / 180.0


def euler(roll, pitch, yaw):
    cr, sr, cp, sp, cy, sy = (math.cos(roll), math.sin(roll), math.cos(pitch), math.sin(pitch),
                              math.cos(yaw), math.sin(yaw))
    return (np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]]) @ np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
            @ np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]]))


def cm(m):
    return np.asarray(m, dtype=float).T.reshape(9)  # column-major


def check(expected, actual, pos, vel, F, plastic, C=None):
    assert np.linalg.norm(expected.position - actual.position, axis=1).max() < pos
    assert np.linalg.norm(expected.velocity - actual.velocity, axis=1).max() < vel
    assert np.linalg.norm((expected.deformation - actual.deformation), axis=1).max() < F
    if C is not None:
        assert np.linalg.norm((expected.affine - actual.affine), axis=1).max() < C
    assert np.abs(expected.plastic - actual.plastic).max() < plastic


def test_corotated_stress_tracks_cpu_for_elastic_sand_and_snow():  # gpu.rs:4423-4516
    mats = [(MAT_ELASTIC, (4000.0, 0.2)), (MAT_SAND, (4000.0, 0.2, 30.0 * DEG, 0.0)),
            (MAT_SNOW, (4000.0, 0.2, 2.5e-2, 7.5e-3, 10.0))]
    parts = []
    F0 = np.array([[1.1, 0.15, 0.02], [0.0, 0.88, 0.08], [0.0, 0.0, 1.04]])
    for i, (m, prm) in enumerate(mats):
        p = density_particles([(0.25 + 0.25 * i, 0.4, 0.5)], 0.04, 1000.0, m, prm)
        p.deformation[0] = cm(F0)
        if i == 2:
            p.plastic[0, 0] = 0.8
        parts.append(p)
    for x, diag in ((0.25, (0.95, 0.8, 0.75)), (0.5, (1.2, 0.9, 0.7))):
        p = density_particles([(x, 0.7, 0.5)], 0.04, 1000.0, MAT_SAND, (4000.0, 0.2, 30.0 * DEG, 0.0))
        p.deformation[0] = cm(np.diag(diag))
        parts.append(p)
    parts = ParticleArrays.concat(parts)
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0))
    cpu = O.OracleWorld(params, parts)
    gpu = Session(params, parts, 1e-4)
    for _ in range(12):
        cpu.step(0.001)
        gpu.step_cfl(0.001)
    assert cpu.substeps() == gpu.substeps() == 12
    e, a = cpu.particles(), gpu.particles()
    check(e, a, 2e-5, 3e-4, 2e-4, 2e-4)
    assert a.plastic[4, 1] > parts.plastic[4, 1]  # the stretched sand particle hardened


@pytest.mark.parametrize("resident", [False, True])
def test_sand_neo_hookean_matches_cpu_direct_and_resident(resident):  # gpu.rs:2339-2446
    rot = euler(0.2, -0.4, 0.7)
    defs = [np.eye(3), rot, np.eye(3) * 1.1, np.diag([0.8, 0.79, 0.81]),
            rot @ np.diag([math.exp(0.15), math.exp(-0.25), math.exp(-0.1)])]
    parts = []
    for i, Fm in enumerate(defs):
        p = density_particles([(0.5 + i * 0.4, 0.5, 0.5)], 0.04, 1000.0, MAT_SAND_NEO_HOOKEAN,
                              (4000.0, 0.2, 35.0 * DEG, 0.02))
        p.deformation[0] = cm(Fm)
        p.plastic[0, 1] += i * 0.2
        parts.append(p)
    parts = ParticleArrays.concat(parts)
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0), bounds=((0, 0, 0), (3, 3, 3)))
    cpu = O.OracleWorld(params, parts)
    for _ in range(4):
        cpu.step(1e-4)
    gpu = Session(params, parts, 1e-4)
    if resident:
        gpu.step(4)
    else:
        for _ in range(4):
            gpu.step_cfl(1e-4)
    assert gpu.substeps() == cpu.substeps() == 4
    e, a = cpu.particles(), gpu.particles()
    check(e, a, 2e-5, 3e-4, 2e-4, 2e-4, C=2e-3)
    assert a.plastic[2, 1] > parts.plastic[2, 1] and a.plastic[4, 1] > parts.plastic[4, 1]


def test_snow_block_resident_tracks_oracle():
    """A small snow block falling under gravity: resident substeps vs the oracle."""
    from tessera_b200 import scenes
    sc = scenes.elastic_block(lo=(0.45, 0.45, 0.45), hi=(0.53, 0.53, 0.53), young=1.4e5, density=400.0)
    p = sc.particles.copy()
    p.material[:] = MAT_SNOW
    p.material_params[:] = (1.4e5, 0.2, 2.5e-2, 7.5e-3, 10.0)
    cpu = O.OracleWorld(sc.params, p)
    gpu = Session(sc.params, p, 5e-5)
    for _ in range(16):
        cpu.substep_fixed(5e-5)
    gpu.step(16)
    check(cpu.particles(), gpu.particles(), 2e-5, 3e-4, 2e-4, 2e-4)
