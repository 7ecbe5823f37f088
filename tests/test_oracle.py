"""Pins the CPU oracle to the reference's own known-answer tests.

The reference ships no golden vector files; its CPU-only tests construct
fixtures inline.  Each test here restates one of them with the same inputs and
the same assertions (tolerances included), citing the Rust test it follows.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import (
    BOUNDARY_FREE_SLIP, BOUNDARY_NON_REFLECTING, BOUNDARY_SEPARATE, BOUNDARY_SLIP, BOUNDARY_STICK,
    MAT_ELASTIC, MAT_FLUID, MAT_NEO_HOOKEAN, MAT_SAND, MAT_SAND_NEO_HOOKEAN, MAT_SNOW,
    TMPM_ERR_MPM_INVALID_INPUT, TMPM_ERR_UNKNOWN_CHUNK, Obstacle, ParticleArrays,
    density_particles, make_params,
)

DEG = math.pi / 180.0


def particle(pos, radius=0.04, density=1000.0, material=MAT_ELASTIC, params=(1000.0, 0.2)):
    """MpmParticle::new as used by world.rs tests (world.rs:650-657)."""
    return density_particles([pos], radius, density, material, params)


def default_params(**kw):
    """MpmParams::default (world.rs:40-49) with overrides."""
    args = dict(cell_width=0.1, gravity=(0.0, 0.0, -9.81), max_substep=1e-3, bounds=None)
    args.update(kw)
    return make_params(**args)


def euler(roll, pitch, yaw):
    """nalgebra UnitQuaternion::from_euler_angles rotation matrix Rz(yaw) Ry(pitch) Rx(roll)."""
    cr, sr, cp, sp, cy, sy = (math.cos(roll), math.sin(roll), math.cos(pitch), math.sin(pitch),
                              math.cos(yaw), math.sin(yaw))
    rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return rz @ ry @ rx


def quat_axis_angle(axis, angle):
    axis = np.asarray(axis, dtype=float)
    axis = axis / np.linalg.norm(axis)
    s = math.sin(angle / 2)
    return (axis[0] * s, axis[1] * s, axis[2] * s, math.cos(angle / 2))


# ------------------------------------------------------------------ world.rs


def test_one_particle_free_fall_matches_gravity():  # world.rs:659-672
    w = O.OracleWorld(default_params(max_substep=0.001), particle((0.5, 0.5, 0.5)))
    w.step(0.001)
    p = w.particles()
    assert abs(p.velocity[0, 2] + 0.00981) < 1e-10
    assert abs(p.position[0, 2] - (0.5 - 0.00000981)) < 1e-10


def test_apic_transfer_preserves_uniform_velocity_without_forces():  # world.rs:674-693
    a = particle((0.45, 0.5, 0.55))
    b = particle((0.55, 0.5, 0.45))
    parts = ParticleArrays.concat([a, b])
    parts.velocity[:] = (1.0, -2.0, 0.5)
    w = O.OracleWorld(default_params(gravity=(0, 0, 0), max_substep=0.001), parts)
    w.step(0.001)
    for v in w.particles().velocity:
        assert np.linalg.norm(v - np.array([1.0, -2.0, 0.5])) < 1e-10


def test_transfer_colors_keep_opposed_particles_on_separate_grid_nodes():  # world.rs:695-718
    left = particle((0.5, 0.5, 0.5))
    left.velocity[0, 0] = 1.0
    right = left.copy()
    right.velocity[0, 0] = -1.0
    right.transfer_color[0] = 1
    params = default_params(gravity=(0, 0, 0), max_substep=0.001)
    sep = O.OracleWorld(params, ParticleArrays.concat([left, right]))
    sep.step(0.001)
    v = sep.particles().velocity
    assert abs(v[0, 0] - 1.0) < 1e-10
    assert abs(v[1, 0] + 1.0) < 1e-10
    right.transfer_color[0] = 0
    mixed = O.OracleWorld(params, ParticleArrays.concat([left, right]))
    mixed.step(0.001)
    v = mixed.particles().velocity
    assert abs(v[0, 0]) < 1e-10
    assert abs(v[1, 0]) < 1e-10


def _sheet(group):
    return Obstacle.triangle_prism((0.5, 0.5, 0.5), [(0.0, -1.0, -1.0), (0.0, 1.0, -1.0), (0.0, 0.0, 1.0)],
                                   0.001, cpic_group=group, boundary=BOUNDARY_NON_REFLECTING)


def test_cpic_triangle_assigns_opposite_sides_to_separate_grid_regions():  # world.rs:720-781
    left = particle((0.48, 0.5, 0.5), radius=0.005)
    left.velocity[0, 0] = -1.0
    right = left.copy()
    right.position[0, 0] = 0.52
    right.velocity[0, 0] = 1.0
    params = default_params(gravity=(0, 0, 0))
    parts = ParticleArrays.concat([left, right])
    separated = O.OracleWorld(params, parts)
    separated.set_obstacles([_sheet(0)])
    disabled = separated.clone()
    disabled.set_use_cpic(False)
    disabled.step(0.001)
    v = disabled.particles().velocity
    assert abs(v[0, 0]) < 0.5 and abs(v[1, 0]) < 0.5
    explicit = separated.clone()
    explicit.set_use_cpic(False)
    ep = explicit.particles()
    ep.transfer_color[1] = 1
    explicit.write_particles(ep)
    explicit.step(0.001)
    v = explicit.particles().velocity
    assert v[0, 0] < -0.9 and v[1, 0] > 0.9
    separated.step(0.001)
    v = separated.particles().velocity
    assert v[0, 0] < -0.9 and v[1, 0] > 0.9
    mixed = O.OracleWorld(params, parts)
    mixed.set_obstacles([_sheet(-1)])
    mixed.step(0.001)
    v = mixed.particles().velocity
    assert abs(v[0, 0]) < 0.5 and abs(v[1, 0]) < 0.5


def test_obstacle_reaction_opposes_particle_impact():  # world.rs:783-807
    imp = particle((1.02, 0.0, 0.0))
    imp.velocity[0, 0] = -1.0
    initial = imp.velocity[0] * imp.mass[0]
    w = O.OracleWorld(default_params(gravity=(0, 0, 0)), imp)
    w.set_obstacles([Obstacle.sphere((0, 0, 0), 1.0)])
    r = w.step_with_obstacle_reactions(0.001, 1)
    assert r.shape == (1, 6)
    lin, ang = r[0, :3], r[0, 3:]
    assert lin[0] < 0.0
    assert abs(lin[1]) < 1e-10
    assert np.linalg.norm(ang) < 1e-10
    p = w.particles()
    assert p.velocity[0, 0] > -1.0
    final = p.velocity[0] * p.mass[0]
    assert np.linalg.norm(initial - final - lin) < 1e-10


def test_fixed_particle_does_not_move():  # world.rs:809-818
    f = particle((0.5, 0.5, 0.5))
    f.fixed[0] = 1
    f.velocity[0] = (1.0, 2.0, 3.0)
    w = O.OracleWorld(default_params(), f)
    w.step(0.01)
    p = w.particles()
    assert np.array_equal(p.position[0], [0.5, 0.5, 0.5])
    assert np.array_equal(p.velocity[0], [0.0, 0.0, 0.0])


def test_world_boundary_prevents_particle_escape():  # world.rs:820-840
    f = particle((0.5, 0.5, 0.05))
    f.velocity[0, 2] = -10.0
    w = O.OracleWorld(default_params(gravity=(0, 0, 0), max_substep=0.001, bounds=((0, 0, 0), (1, 1, 1))), f)
    w.step(0.01)
    p = w.particles()
    assert p.position[0, 2] >= 0.04
    assert p.velocity[0, 2] >= 0.0


def test_all_materials_complete_finite_steps():  # world.rs:842-866
    mats = [
        (MAT_ELASTIC, (1000.0, 0.2)),
        (MAT_NEO_HOOKEAN, (1000.0, 0.2)),
        (MAT_SAND, (1000.0, 0.2, 35.0 * DEG, 0.0)),
        (MAT_FLUID, (2000.0, 7.0, 0.01, 0.25)),
        (MAT_SNOW, (1000.0, 0.2, 2.5e-2, 7.5e-3, 10.0)),
    ]
    parts = ParticleArrays.concat(
        [density_particles([(0.3 + i * 0.1, 0.5, 0.5)], 0.03, 1000.0, m, prm) for i, (m, prm) in enumerate(mats)])
    w = O.OracleWorld(default_params(), parts)
    w.step(0.002)
    p = w.particles()
    for name in ("position", "velocity", "deformation", "affine"):
        assert np.all(np.isfinite(getattr(p, name)))


def test_cfl_bound_tightens_for_stiffer_material():  # world.rs:868-893
    params = default_params(max_substep=1.0)
    soft = O.OracleWorld(params, particle((0, 0, 0), params=(1000.0, 0.2))).stable_timestep()
    stiff = O.OracleWorld(params, particle((0, 0, 0), params=(100000.0, 0.2))).stable_timestep()
    assert stiff < soft


def test_rejects_invalid_particle_and_world_parameters():  # world.rs:895-914
    bad = particle((0, 0, 0))
    bad.mass[0] = 0.0
    with pytest.raises(O.OracleError) as e:
        O.OracleWorld(default_params(), bad)
    assert e.value.status == TMPM_ERR_MPM_INVALID_INPUT
    with pytest.raises(O.OracleError) as e:
        O.OracleWorld(default_params(cell_width=0.0))
    assert e.value.status == TMPM_ERR_MPM_INVALID_INPUT


def test_moving_sphere_pushes_particle_without_changing_obstacle():  # world.rs:916-932
    w = O.OracleWorld(default_params(gravity=(0, 0, 0)), particle((0.62, 0.5, 0.5)))
    ob = Obstacle.sphere((0.5, 0.5, 0.5), 0.1, linear_velocity=(1.0, 0.0, 0.0))
    w.set_obstacles([ob])
    w.step(0.001)
    p = w.particles()
    assert p.velocity[0, 0] > 0.0
    d, _ = O.obstacle_surface(ob, p.position[0])
    assert d >= p.radius[0] - 1e-12


def test_rejects_invalid_obstacle_without_replacing_current_set():  # world.rs:934-945
    w = O.OracleWorld(default_params())
    w.set_obstacles([Obstacle.sphere((0, 0, 0), 1.0)])
    with pytest.raises(O.OracleError) as e:
        w.set_obstacles([Obstacle.sphere((0, 0, 0), -1.0)])
    assert e.value.status == TMPM_ERR_MPM_INVALID_INPUT


def test_invalid_particle_batch_does_not_append_or_consume_chunk_id():  # world.rs:947-968
    w = O.OracleWorld(default_params(), particle((0.0, 0.0, 0.5)))
    bad = particle((0.2, 0.0, 0.5))
    bad.mass[0] = 0.0
    with pytest.raises(O.OracleError):
        w.add_particles(ParticleArrays.concat([particle((0.1, 0.0, 0.5)), bad]))
    assert w.count() == 1
    chunk = w.add_particles(particle((0.3, 0.0, 0.5)))
    assert chunk == 1
    assert w.particles().chunk_id[1] == chunk
    assert w.remove_chunk(0) == 1
    assert w.particles().chunk_id[0] == chunk
    with pytest.raises(O.OracleError) as e:
        w.remove_chunk(0)
    assert e.value.status == TMPM_ERR_UNKNOWN_CHUNK


# --------------------------------------------------------------- material.rs


@pytest.mark.parametrize("material", [MAT_SAND, MAT_SAND_NEO_HOOKEAN])
def test_sand_hardening_accumulates_across_shear_and_apex_loads(material):  # material.rs:547-595
    params = (4000.0, 0.2, 35.0 * DEG, 0.0)
    state = np.array([1.0, 1.0, 0.0])
    for load in [np.array([0.15, -0.25, -0.1])] * 3 + [np.full(3, math.log(1.2)), np.full(3, math.log(0.8))]:
        strain = load + state[2] / 3.0
        trace = strain.sum()
        dev = strain - trace / 3.0
        angle = 35.0 * DEG + (9.0 * DEG * state[1] - 10.0 * DEG) * math.exp(-0.2 * state[1])
        alpha = math.sqrt(2.0 / 3.0) * 2.0 * math.sin(angle) / (3.0 - math.sin(angle))
        if trace > 0.0 or np.linalg.norm(dev) < 1e-12:
            expected_log, inc = np.zeros(3), np.linalg.norm(strain)
        else:
            gamma = np.linalg.norm(dev) + 2.0 * trace * alpha
            assert gamma > 0
            expected_log, inc = strain - dev * (gamma / np.linalg.norm(dev)), gamma
        proj, nxt = O.project_deformation(material, params, np.diag(np.exp(load)), state)
        assert np.linalg.norm(proj - np.diag(np.exp(expected_log))) < 1e-12
        assert abs(nxt[1] - state[1] - inc) < 1e-12
        vol = load.sum() - expected_log.sum()
        assert abs(nxt[0] - state[0] * math.exp(vol)) < 1e-12
        assert abs(nxt[2] - state[2] - vol) < 1e-12
        state = nxt


def test_corotated_sand_isotropic_roundoff_and_disabled_plasticity():  # material.rs:597-620
    rot = euler(0.2, -0.4, 0.7)
    params = (4000.0, 0.2, 35.0 * DEG, 0.02)
    st = (1.0, 1.0, 0.0)
    exact, es = O.project_deformation(MAT_SAND, params, rot, st)
    rounded, rs = O.project_deformation(MAT_SAND, params, rot.astype(np.float32).astype(np.float64), st)
    assert np.linalg.norm(exact - rounded) < 2e-6
    assert np.all(np.abs(es - rs) < 2e-6)
    tension = np.eye(3) * 1.2
    out, os_ = O.project_deformation(MAT_SAND, (4000.0, 0.0, 0.5, 0.0), tension, st)
    assert np.array_equal(out, tension) and np.array_equal(os_, st)


def test_fluid_pressure_resists_compression_and_softly_resists_tension():  # material.rs:622-638
    prm = (1000.0, 7.0, 0.01, 0.25)
    comp = O.kirchhoff_stress(MAT_FLUID, prm, np.eye(3) * 0.9)
    exp_ = O.kirchhoff_stress(MAT_FLUID, prm, np.eye(3) * 1.1)
    assert np.trace(comp) < 0.0 < np.trace(exp_)
    assert abs(np.trace(comp)) > abs(np.trace(exp_))


def test_snow_projection_clamps_elastic_singular_values():  # material.rs:640-649
    prm = (1000.0, 0.2, 2.5e-2, 7.5e-3, 10.0)
    proj, st = O.project_deformation(MAT_SNOW, prm, np.diag([0.5, 1.0, 1.5]))
    s = np.linalg.svd(proj, compute_uv=False)
    assert np.all(s >= 0.975 - 1e-12) and np.all(s <= 1.0075 + 1e-12)
    assert st[0] != 1.0


def test_sand_projection_removes_unsupported_tension():  # material.rs:651-658
    proj, st = O.project_deformation(MAT_SAND, (5000.0, 0.2, 35.0 * DEG, 0.0), np.eye(3) * 1.2)
    assert np.linalg.norm(proj - np.eye(3)) < 1e-10
    assert st[0] > 1.0


def test_invalid_material_parameters_are_rejected_by_validation():  # material.rs:660-665
    assert not O.material_valid(MAT_ELASTIC, (-1.0, 0.2))
    assert not O.material_valid(MAT_FLUID, (1.0, 0.0, 0.0, 0.25))
    assert O.material_valid(MAT_NEO_HOOKEAN, (1000.0, 0.49))


# -------------------------------------------------- sand_neo_hookean_tests.rs

SNH = (4000.0, 0.2, 35.0 * DEG, 0.0)
SNH_STATE = (1.0, 1.0, 0.0)


def test_sand_neo_hookean_stress_vanishes_for_identity_and_rotation():  # :16-25
    for F in (np.eye(3), euler(0.3, -0.4, 0.7)):
        assert np.linalg.norm(O.kirchhoff_stress(MAT_SAND_NEO_HOOKEAN, SNH, F, None, SNH_STATE)) < 1e-10


def test_cohesive_rotation_projection_is_stable_after_f32_upload():  # :27-44
    rot = euler(0.2, -0.4, 0.7)
    prm = (4000.0, 0.2, 35.0 * DEG, 0.02)
    exact, es = O.project_deformation(MAT_SAND_NEO_HOOKEAN, prm, rot, SNH_STATE)
    rounded, rs = O.project_deformation(MAT_SAND_NEO_HOOKEAN, prm, rot.astype(np.float32).astype(np.float64),
                                        SNH_STATE)
    assert np.linalg.norm(exact - rounded) < 2e-6
    assert abs(es[0] - rs[0]) < 2e-6 and abs(es[2] - rs[2]) < 2e-6


def test_sand_neo_hookean_stress_matches_reference_under_deformation_and_rotation():  # :46-65
    F = np.array([[0.9, 0.2, 0.0], [0.0, 0.8, 0.0], [0.0, 0.0, 1.1]])
    rot = euler(0.2, -0.6, 0.3)
    expected = F @ F.T * (5000.0 / 3.0) + np.eye(3) * ((10000.0 / 9.0) * math.log(0.792) - 5000.0 / 3.0)
    stress = O.kirchhoff_stress(MAT_SAND_NEO_HOOKEAN, SNH, F, None, SNH_STATE)
    rotated = O.kirchhoff_stress(MAT_SAND_NEO_HOOKEAN, SNH, rot @ F, None, SNH_STATE)
    assert np.linalg.norm(stress - expected) < 1e-10
    assert np.linalg.norm(rotated - rot @ expected @ rot.T) < 1e-10
    linear = O.kirchhoff_stress(MAT_SAND, SNH, F, None, SNH_STATE)
    assert np.linalg.norm(stress - linear) > 100.0


def test_sand_neo_hookean_tensile_apex_updates_all_reference_plastic_state():  # :67-81
    prm = (4000.0, 0.2, 35.0 * DEG, 0.06)
    proj, pl = O.project_deformation(MAT_SAND_NEO_HOOKEAN, prm, np.eye(3) * 1.2, (2.0, 1.5, 0.03))
    assert np.linalg.norm(proj - np.eye(3) * math.exp(0.02)) < 1e-12
    assert abs(pl[0] - 2.0 * 1.2 ** 3 / math.exp(0.06)) < 1e-12
    assert abs(pl[2] - (0.03 + 3.0 * math.log(1.2) - 0.06)) < 1e-12
    assert abs(pl[1] - (1.5 + math.sqrt(3.0) * (math.log(1.2) + 0.01))) < 1e-12


def test_sand_neo_hookean_shear_return_uses_accumulated_hardening():  # :83-105
    strain = np.array([0.15, -0.25, -0.1])
    for q in (1.0, 4.0):
        proj, pl = O.project_deformation(MAT_SAND_NEO_HOOKEAN, SNH, np.diag(np.exp(strain)), (1.0, q, 0.0))
        trace = -0.2
        dev = strain - trace / 3.0
        angle = 35.0 * DEG + (9.0 * DEG * q - 10.0 * DEG) * math.exp(-0.2 * q)
        alpha = math.sqrt(2.0 / 3.0) * 2.0 * math.sin(angle) / (3.0 - math.sin(angle))
        gamma = np.linalg.norm(dev) + 2.0 * trace * alpha
        expected = np.exp(strain - dev * (gamma / np.linalg.norm(dev)))
        assert np.linalg.norm(proj - np.diag(expected)) < 1e-12
        assert abs(pl[1] - q - gamma) < 1e-12
        assert abs(pl[0] - 1.0) < 1e-12
        assert abs(pl[2]) < 1e-12


def test_sand_neo_hookean_elastic_region_and_disabled_plasticity_preserve_state():  # :107-120
    F = np.diag([0.8, 0.79, 0.81])
    out, st = O.project_deformation(MAT_SAND_NEO_HOOKEAN, SNH, F, SNH_STATE)
    assert np.array_equal(out, F) and np.array_equal(st, SNH_STATE)
    out, st = O.project_deformation(MAT_SAND_NEO_HOOKEAN, (4000.0, 0.0, 0.5, 0.0), np.eye(3) * 1.2, SNH_STATE)
    assert np.array_equal(out, np.eye(3) * 1.2) and np.array_equal(st, SNH_STATE)


def test_sand_neo_hookean_validation_rejects_nonphysical_parameters():  # :122-137
    for prm in [(-1.0, 0.2, 0.5, 0.0), (math.nan, 0.2, 0.5, 0.0), (1.0, 0.5, 0.5, 0.0), (1.0, 0.2, -0.1, 0.0),
                (1.0, 0.2, math.pi / 2, 0.0), (1.0, 0.2, math.nan, 0.0), (1.0, 0.2, 0.5, -0.1),
                (1.0, 0.2, 0.5, math.inf)]:
        assert not O.material_valid(MAT_SAND_NEO_HOOKEAN, prm)
    assert O.material_valid(MAT_SAND_NEO_HOOKEAN, SNH)


def test_sand_neo_hookean_particle_initialization_and_cfl_match_reference():  # :139-155
    p = density_particles([(0.5, 0.5, 0.5)], 0.04, 1000.0, MAT_SAND_NEO_HOOKEAN, SNH)
    assert np.array_equal(p.plastic[0], SNH_STATE)
    p.deformation[0] = (np.eye(3) * 2.0).T.reshape(9)
    w = O.OracleWorld(default_params(max_substep=1.0), p)
    expected_ws = math.sqrt((40000.0 / 9.0) / (1000.0 / 8.0))
    assert abs(w.stable_timestep() - 0.05 / expected_ws) < 1e-12
    moving = O.timestep_bound(MAT_SAND_NEO_HOOKEAN, SNH, 1000.0, (10.0, 0.0, 0.0), 0.1, 8.0)
    assert abs(moving - 0.005) < 1e-12


# --------------------------------------------------------------- obstacle.rs


def test_rotated_box_reports_world_normal_and_signed_distance():  # obstacle.rs:793-805
    box = Obstacle.cuboid((1.0, 2.0, 3.0), (0.2, 0.4, 0.6), quat_axis_angle((0, 0, 1), math.pi / 2))
    d, n = O.obstacle_surface(box, (1.5, 2.0, 3.0))
    assert abs(d - 0.1) < 1e-12
    assert np.linalg.norm(n - np.array([1, 0, 0])) < 1e-12
    d, _ = O.obstacle_surface(box, box.center)
    assert abs(d + 0.2) < 1e-12


def test_moving_surface_pushes_and_friction_reduces_sliding():  # obstacle.rs:807-818
    s = Obstacle.sphere((0, 0, 0), 1.0, linear_velocity=(1.0, 0, 0), friction=0.5)
    v = O.contact_velocity(s, (1.0, 0, 0), (0.0, 2.0, 0.0), (1, 0, 0))
    assert np.linalg.norm(v - np.array([1.0, 1.5, 0.0])) < 1e-12


def test_boundary_modes_apply_distinct_contact_velocities():  # obstacle.rs:820-843
    incoming = np.array([0.0, 2.0, 0.0])
    cases = [(BOUNDARY_SLIP, (1.0, 1.5, 0.0)), (BOUNDARY_STICK, (1.0, 0.0, 0.0)),
             (BOUNDARY_SEPARATE, (1.0, 2.0, 0.0)), (BOUNDARY_NON_REFLECTING, incoming),
             (BOUNDARY_FREE_SLIP, (1.0, 2.0, 0.0))]
    for boundary, expected in cases:
        s = Obstacle.sphere((0, 0, 0), 1.0, linear_velocity=(1.0, 0, 0), friction=0.5, boundary=boundary)
        v = O.contact_velocity(s, (1, 0, 0), incoming, (1, 0, 0))
        assert np.linalg.norm(v - np.asarray(expected)) < 1e-12, boundary


def test_free_slip_removes_both_signs_of_moving_surface_relative_normal_velocity():  # obstacle.rs:845-879
    base = dict(linear_velocity=(1.0, 2.0, 3.0), angular_velocity=(0.0, 0.0, 2.0), friction=10.0)
    point = np.array([1.0, 0.0, 0.0])
    surface = np.array([1.0, 2.0, 3.0]) + np.cross([0.0, 0.0, 2.0], point)
    for ns in (-2.0, 2.0):
        vel = surface + np.array([ns, 4.0, -3.0])
        s = Obstacle.sphere((0, 0, 0), 1.0, boundary=BOUNDARY_FREE_SLIP, **base)
        assert np.linalg.norm(O.contact_velocity(s, point, vel, (1, 0, 0)) - (surface + [0.0, 4.0, -3.0])) < 1e-12
        for boundary in (BOUNDARY_SLIP, BOUNDARY_SEPARATE):
            s = Obstacle.sphere((0, 0, 0), 1.0, boundary=boundary, **base)
            r = O.contact_velocity(s, point, vel, (1, 0, 0))
            if ns > 0:
                assert np.array_equal(r, vel)
            else:
                assert abs(r[0] - surface[0]) < 1e-12
                if boundary == BOUNDARY_SEPARATE:
                    assert abs(r[1] - vel[1]) < 1e-12 and abs(r[2] - vel[2]) < 1e-12


def test_capsule_cylinder_and_cone_report_signed_surfaces():  # obstacle.rs:881-915
    cap = Obstacle.capsule((0, 0, 0), 0.5, 0.2)
    d, n = O.obstacle_surface(cap, (0.3, 0, 0))
    assert abs(d - 0.1) < 1e-12 and np.linalg.norm(n - [1, 0, 0]) < 1e-12
    d, n = O.obstacle_surface(cap, (0, 0, 0.8))
    assert abs(d - 0.1) < 1e-12 and np.linalg.norm(n - [0, 0, 1]) < 1e-12
    assert abs(O.obstacle_surface(cap, (0, 0, 0))[0] + 0.2) < 1e-12
    line = Obstacle.capsule((0, 0, 0), 0.5, 0.0)
    assert O.obstacle_valid(line)
    assert O.may_contact(line, (0, 0, 0.54), 0.04)
    assert not O.may_contact(line, (0, 0, 0.55), 0.04)
    cyl = Obstacle.cylinder((0, 0, 0), 0.5, 0.2)
    d, n = O.obstacle_surface(cyl, (0.3, 0, 0.7))
    assert abs(d - math.hypot(0.1, 0.2)) < 1e-12
    assert np.linalg.norm(n - np.array([0.1, 0, 0.2]) / math.hypot(0.1, 0.2)) < 1e-12
    assert abs(O.obstacle_surface(cyl, (0, 0, 0))[0] + 0.2) < 1e-12
    cone = Obstacle.cone((0, 0, 0), 0.5, 0.4)
    d, n = O.obstacle_surface(cone, (0, 0, 0.7))
    assert abs(d - 0.2) < 1e-12 and np.linalg.norm(n - [0, 0, 1]) < 1e-12
    d, n = O.obstacle_surface(cone, (0, 0, -0.7))
    assert abs(d - 0.2) < 1e-12 and np.linalg.norm(n + np.array([0, 0, 1])) < 1e-12
    d, n = O.obstacle_surface(cone, (0, 0, 0))
    assert d < -0.1 and n[0] > 0 and n[2] > 0
    assert O.obstacle_valid(cone)


def test_rotated_capsule_and_invalid_primitives():  # obstacle.rs:917-933
    cap = Obstacle.capsule((0, 0, 0), 0.5, 0.2, quat_axis_angle((0, 1, 0), math.pi / 2))
    d, n = O.obstacle_surface(cap, (0.8, 0, 0))
    assert abs(d - 0.1) < 1e-12 and np.linalg.norm(n - [1, 0, 0]) < 1e-12
    assert not O.obstacle_valid(Obstacle.cylinder((0, 0, 0), 0.0, 0.2))
    assert not O.obstacle_valid(Obstacle.cone((0, 0, 0), 0.5, -0.2))


def test_finite_ground_has_one_sided_interior_and_finite_edges():  # obstacle.rs:935-957
    g = Obstacle.ground((0, 0, 0), (1.0, 1.0))
    d, n = O.obstacle_surface(g, (0, 0, 0.2))
    assert d == 0.2 and np.array_equal(n, [0, 0, 1])
    d, n = O.obstacle_surface(g, (0, 0, -0.2))
    assert d == -0.2 and np.array_equal(n, [0, 0, 1])
    d, n = O.obstacle_surface(g, (1.3, 0, 0))
    assert abs(d - 0.3) < 1e-12 and np.linalg.norm(n - [1, 0, 0]) < 1e-12
    d, n = O.obstacle_surface(g, (1.3, 0, -0.4))
    assert abs(d - 0.5) < 1e-12 and np.linalg.norm(n - [0.6, 0, -0.8]) < 1e-12
    assert O.obstacle_valid(g)


def test_triangle_prism_exposes_caps_sides_and_interior():  # obstacle.rs:959-984
    pr = Obstacle.triangle_prism((0, 0, 0), [(-0.2, -0.2, 0.0), (0.2, -0.2, 0.0), (0.0, 0.2, 0.0)], 0.01)
    assert O.obstacle_valid(pr)
    d, n = O.obstacle_surface(pr, (0, -0.05, 0.05))
    assert abs(d - 0.04) < 1e-12 and np.linalg.norm(n - [0, 0, 1]) < 1e-12
    d, n = O.obstacle_surface(pr, (0, -0.05, -0.05))
    assert abs(d - 0.04) < 1e-12 and np.linalg.norm(n + np.array([0, 0, 1])) < 1e-12
    d, _ = O.obstacle_surface(pr, (0, -0.05, 0.0))
    assert abs(d + 0.01) < 1e-12
    d, n = O.obstacle_surface(pr, (0, -0.3, 0.0))
    assert abs(d - 0.1) < 1e-12 and np.linalg.norm(n + np.array([0, 1, 0])) < 1e-12


def test_convex_planes_report_face_edge_vertex_and_interior():  # obstacle.rs:986-1018
    cx = Obstacle.convex((0, 0, 0), [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)],
                         [(-1, 0, 0), (0, -1, 0), (0, 0, -1), np.ones(3) / math.sqrt(3)])
    assert O.obstacle_valid(cx)
    d, n = O.obstacle_surface(cx, (0.1, 0.1, 0.1))
    assert abs(d + 0.1) < 1e-12 and np.linalg.norm(n + np.array([1, 0, 0])) < 1e-12
    d, n = O.obstacle_surface(cx, (-0.2, 0.1, 0.1))
    assert abs(d - 0.2) < 1e-9 and np.linalg.norm(n + np.array([1, 0, 0])) < 1e-9
    d, n = O.obstacle_surface(cx, (-0.2, -0.3, 0.1))
    assert abs(d - math.hypot(0.2, 0.3)) < 1e-8
    assert np.linalg.norm(n - np.array([-0.2, -0.3, 0.0]) / math.hypot(0.2, 0.3)) < 1e-8
    d, _ = O.obstacle_surface(cx, (1.2, 0.1, 0.1))
    assert abs(d - math.sqrt(0.06)) < 1e-7
    bad = Obstacle.convex((0, 0, 0), [(math.nan, 0, 0)], [(-1, 0, 0)] * 4)
    assert not O.obstacle_valid(bad)


def test_convex_plane_distance_matches_analytic_box():  # obstacle.rs:1020-1060
    half = np.array([0.2, 0.3, 0.4])
    verts = [(x * half[0], y * half[1], z * half[2]) for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)]
    cx = Obstacle.convex((0, 0, 0), verts, [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)])
    box = Obstacle.cuboid((0, 0, 0), half)
    for x in (-0.6, -0.2, -0.1, 0.0, 0.1, 0.2, 0.6):
        for y in (-0.7, -0.3, 0.0, 0.3, 0.7):
            for z in (-0.8, -0.4, 0.0, 0.4, 0.8):
                a = O.obstacle_surface(cx, (x, y, z))[0]
                b = O.obstacle_surface(box, (x, y, z))[0]
                assert abs(a - b) < 1e-7, (x, y, z, a, b)


# ------------------------------------------------------------ f32 binning


def test_binning_reference_is_stable_and_blocks_match_floor_division():
    rng = np.random.default_rng(7)
    pos = rng.uniform(-1.0, 1.0, size=(5000, 3)).astype(np.float32)
    cells, keys, perm = O.binning_reference(pos, 0.05)
    assert np.all(np.diff(keys[perm].astype(np.int64)) >= 0)
    same = keys[perm][1:] == keys[perm][:-1]
    assert np.all(perm[1:][same] > perm[:-1][same])  # stability
    blocks = np.floor_divide(cells, 4)
    assert np.array_equal(np.right_shift(cells, 2), blocks)
    # the key orders by block first, then by cell inside the block
    assert np.array_equal(keys >> 6, O.block_morton_keys(cells))
    inner = cells & 3
    assert np.array_equal(keys & 63 == 0, np.all(inner == 0, axis=1))
    # storage order: a permutation, transposed within full 256-chunks
    order = O.storage_order(perm)
    assert np.array_equal(np.sort(order), np.sort(perm))
    assert order[2] == perm[64] and order[8] == perm[128]  # quarter-warps take slabs of the cell group
    assert sorted(O.lane_cell(np.arange(32))) == list(range(32))
    assert order[1] == perm[8] and order[32] == perm[1] and np.array_equal(order[-(len(perm) % 256):],
                                                                            perm[-(len(perm) % 256):])
