"""The tessera3d-compatible MpmWorld binding: host-side behaviour on CPU, and
on GPU the reference's executable acceptance script (examples/mpm_resident.py)
against the CPU oracle."""

import math

import numpy as np
import pytest

from tessera_b200.mpm import (
    MpmBoundary, MpmMaterial, MpmObstacleInput, MpmObstacleShape, MpmParticleInput, MpmWorld, Quaternion,
    TesseraError, Vec3,
)


def vec(x, y, z):
    return Vec3(x=x, y=y, z=z)


FLUID = MpmMaterial.FLUID(bulk_modulus=2000.0, gamma=7.0, viscosity=0.1, tensile_stiffness=0.0)
PARTICLE = MpmParticleInput(position=vec(0.5, 0.5, 0.5), velocity=vec(0.0, 0.0, 0.0), radius=0.03, density=1000.0,
                            material=FLUID, enabled=True, fixed=False, damping=0.0)


def world(bounded=True):
    return MpmWorld(particles=[PARTICLE], gravity=vec(0.0, 0.0, -1.0), cell_width=0.1, max_substep=0.001,
                    bounds_min=vec(0, 0, 0) if bounded else None, bounds_max=vec(1, 1, 1) if bounded else None)


# ---------------------------------------------------------------- CPU (host logic)

def test_constructor_validates_like_mpm_world_new():
    with pytest.raises(TesseraError):
        MpmWorld([PARTICLE], vec(0, 0, -1), 0.0, 0.001)
    with pytest.raises(TesseraError, match="both MPM bounds"):
        MpmWorld([PARTICLE], vec(0, 0, -1), 0.1, 0.001, bounds_min=vec(0, 0, 0))
    bad = MpmParticleInput(position=vec(0.5, 0.5, 0.5), velocity=vec(0, 0, 0), radius=-0.03, density=1000.0,
                           material=FLUID)
    with pytest.raises(TesseraError):
        MpmWorld([bad], vec(0, 0, -1), 0.1, 0.001)
    w = world()
    assert w.substeps() == 0 and w.frame_substeps() == 1 and w.use_cpic()
    p = w.particles()[0]
    assert math.isclose(p.mass, 1000.0 * 0.06 ** 3)
    assert p.deformation == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_chunks_and_forces_without_device_state():
    w = world()
    chunk = w.add_particles([PARTICLE])
    assert chunk == 1 and len(w.particles()) == 2
    assert w.remove_chunk(chunk) == 1
    with pytest.raises(TesseraError, match="unknown MPM particle chunk"):
        w.remove_chunk(chunk)
    with pytest.raises(TesseraError, match="out of range"):
        w.set_particle_force(5, vec(1, 0, 0))
    with pytest.raises(TesseraError, match="finite"):
        w.set_particle_force(0, vec(float("nan"), 0, 0))
    w.set_particle_force(0, vec(0.1, 0.0, 0.0))
    assert w.particle_arrays().force[0, 0] == 0.1


def test_obstacle_inputs_are_validated():
    w = world()
    sphere = MpmObstacleInput(shape=MpmObstacleShape.SPHERE(radius=0.1), center=vec(0.5, 0.5, 0.2))
    w.set_obstacles([sphere])
    assert w.obstacle_count() == 1 and w.obstacle_boundaries() == [MpmBoundary.SLIP]
    with pytest.raises(TesseraError, match="unit quaternion"):
        w.set_obstacles([MpmObstacleInput(shape=MpmObstacleShape.SPHERE(radius=0.1), center=vec(0, 0, 0),
                                          orientation=Quaternion(0, 0, 0, 2))])
    with pytest.raises(TesseraError, match="invalid MPM obstacle"):
        w.set_obstacles([MpmObstacleInput(shape=MpmObstacleShape.SPHERE(radius=-1.0), center=vec(0, 0, 0))])
    with pytest.raises(TesseraError, match="three vertices"):
        w.set_obstacles([MpmObstacleInput(shape=MpmObstacleShape.TRIANGLE_PRISM(
            vertices=[vec(0, 0, 0), vec(1, 0, 0)], half_thickness=0.01), center=vec(0, 0, 0))])
    w.set_obstacle_boundaries([MpmBoundary.FREE_SLIP])
    assert w.obstacle_boundaries() == [MpmBoundary.FREE_SLIP]
    with pytest.raises(TesseraError, match="CPIC"):
        w.set_obstacle_cpic_groups([0])  # only triangle prisms carry CPIC groups


def test_fixed_step_input_validation():
    w = world()
    for dt, steps in ((0.0, 1), (float("nan"), 1), (1e-4, 0), (1e-4, 65)):
        with pytest.raises(TesseraError, match="invalid fixed GPU substep input"):
            w.step_gpu_fixed(dt, steps)
    with pytest.raises(TesseraError, match="invalid MPM frame timestep"):
        w.step(-1.0)


# --------------------------------------------------------------------- GPU

@pytest.mark.gpu
def test_mpm_resident_example_tracks_cpu():  # crates/tessera-python3d/examples/mpm_resident.py:1-91
    from oracle import oracle as O
    from tessera_b200._abi import MAT_FLUID, density_particles, make_params

    def oracle_world(bounded=True):
        p = density_particles([(0.5, 0.5, 0.5)], 0.03, 1000.0, MAT_FLUID, (2000.0, 7.0, 0.1, 0.0))
        return O.OracleWorld(make_params(0.1, gravity=(0, 0, -1.0), max_substep=0.001,
                                         bounds=((0, 0, 0), (1, 1, 1)) if bounded else None), p)

    cpu, gpu = oracle_world(), world()
    for step in range(20):
        if step == 4:
            cpu.set_particle_force(0, (0.1, 0.0, 0.0))
            gpu.set_particle_force(0, vec(0.1, 0.0, 0.0))
        if step == 8:
            cpu.step(0.0001)
            gpu.step(0.0001)
        if step == 12:
            chunk = gpu.add_particles([PARTICLE])
            assert gpu.remove_chunk(chunk) == 1
            ch = cpu.add_particles(density_particles([(0.5, 0.5, 0.5)], 0.03, 1000.0, MAT_FLUID,
                                                     (2000.0, 7.0, 0.1, 0.0)))
            assert cpu.remove_chunk(ch) == 1
        dt = 0.00005 if step >= 16 else 0.0001
        cpu.step(dt)
        gpu.step_gpu_fixed(dt, 1)
        assert cpu.substeps() == gpu.substeps()
        e, a = cpu.particles(), gpu.particle_arrays()
        assert np.abs(e.position - a.position).max() < 1e-5
        assert np.abs(e.velocity - a.velocity).max() < 1e-4
    before = gpu.substeps()
    with pytest.raises(TesseraError):
        gpu.step_gpu_fixed(0.0001, 0)
    assert gpu.substeps() == before
    gpu.step_gpu_fixed(0.00005, 1)

    # unbounded fixed steps keep the session while one-shot forces are updated
    far = MpmParticleInput(position=vec(10.5, 0.5, 0.5), velocity=vec(0, 0, 0), radius=0.03, density=1000.0,
                           material=FLUID)
    gpu2 = MpmWorld([PARTICLE, far], vec(0, 0, -1.0), 0.1, 0.001)
    p2 = density_particles([(0.5, 0.5, 0.5), (10.5, 0.5, 0.5)], 0.03, 1000.0, MAT_FLUID, (2000.0, 7.0, 0.1, 0.0))
    cpu2 = O.OracleWorld(make_params(0.1, gravity=(0, 0, -1.0), max_substep=0.001), p2)
    for _ in range(3):
        cpu2.step(0.0001)
        gpu2.step_gpu(0.0001)
        e, a = cpu2.particles(), gpu2.particle_arrays()
        assert np.abs(e.position - a.position).max() < 1e-5
        assert np.abs(e.velocity - a.velocity).max() < 1e-4
    for _ in range(8):
        cpu2.set_particle_force(0, (0.1, 0.0, 0.0))
        gpu2.set_particle_force(0, vec(0.1, 0.0, 0.0))
        for _ in range(4):
            cpu2.step(0.0001)
        gpu2.step_gpu_fixed(0.0001, 4)
        assert cpu2.substeps() == gpu2.substeps()
        e, a = cpu2.particles(), gpu2.particle_arrays()
        assert np.abs(e.position - a.position).max() < 1e-4
        assert np.abs(e.velocity - a.velocity).max() < 2e-3
