"""GPU parity: the sm_100a path through the C ABI against the f64 CPU oracle.

Tolerances are the reference's own GPU-vs-CPU precedent (FP32 device vs f64
CPU, Frobenius / Euclidean norms as nalgebra's `.norm()`):
  * one direct step:      position 1e-5, velocity 1e-4, affine 1e-3, F 1e-5  (gpu.rs:4093-4096)
  * resident 8 substeps:  position 2e-5, velocity 2e-4, F 2e-4, affine 2e-3  (gpu.rs:3699-3703)
Scenes with other scales state their tolerance beside the assertion.

The configuration-sized scenes (configurations 1 and 2, the reduced elastic
block) are checked with relative FP32 bounds instead (parity_tol.py): position
error in cells, velocity relative to the largest speed, the affine matrix C
relative to max(max |C|, max |v| / h) and F relative to max |F|, at every
checkpoint:
  * per substep (1-8 substeps):  position 1e-4 h, velocity 1e-4, C 1e-3, F 1e-5
  * drift (49-200 substeps):      the DRIFT bounds below.
"""

import math

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200._abi import (
    MAT_ELASTIC, MAT_FLUID, MAT_NEO_HOOKEAN, TMPM_ERR_CAPACITY, TMPM_ERR_INVALID_INPUT,
    TMPM_ERR_NON_FINITE_STATE, TMPM_ERR_PENDING_STEPS, TMPM_ERR_RESIDENT_UNAVAILABLE, Obstacle, ParticleArrays,
    density_particles, make_params,
)
from tessera_b200 import scenes
from tessera_b200.session import Session, TesseraError

from parity_tol import PER_SUBSTEP, assert_grid_close, assert_rel_close

pytestmark = pytest.mark.gpu

# bounded FP32 drift over 49-200 substeps of the configuration-sized scenes
DRIFT = dict(position=1e-3, velocity=1e-3, affine=1e-2, deformation=1e-4)

REF_BOUNDS = ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))


def mat_norm(a):  # per-particle Frobenius norm of column-major 9-vectors
    return np.linalg.norm(a.reshape(-1, 9), axis=1)


def assert_close(expected: ParticleArrays, actual: ParticleArrays, pos, vel, F=None, C=None):
    dp = np.linalg.norm(expected.position - actual.position, axis=1).max()
    dv = np.linalg.norm(expected.velocity - actual.velocity, axis=1).max()
    assert dp < pos, f"position {dp}"
    assert dv < vel, f"velocity {dv}"
    if F is not None:
        dF = mat_norm(expected.deformation - actual.deformation).max()
        assert dF < F, f"deformation {dF}"
    if C is not None:
        dC = mat_norm(expected.affine - actual.affine).max()
        assert dC < C, f"affine {dC}"


def reference_resident_particles():
    """The three particles of resident_substeps_match_cpu_with_force_boundary_and_fixed_particles
    (gpu.rs:3634-3677)."""
    a = density_particles([(0.42, 0.48, 0.51)], 0.04, 1000.0, MAT_NEO_HOOKEAN, (2000.0, 0.2))
    b = density_particles([(0.48, 0.48, 0.0401)], 0.04, 1000.0, MAT_FLUID, (2000.0, 7.0, 0.1, 0.25))
    c = density_particles([(0.6, 0.5, 0.5)], 0.04, 1000.0, MAT_NEO_HOOKEAN, (2000.0, 0.2))
    p = ParticleArrays.concat([a, b, c])
    p.force[0] = (0.2, -0.1, 0.3)
    p.damping[0] = 0.4
    p.velocity[1, 2] = -2.0
    p.fixed[2] = 1
    p.velocity[2, 0] = 1.0
    return p


def test_resident_substeps_match_cpu_with_force_boundary_and_fixed_particles():  # gpu.rs:3634-3775
    params = make_params(0.1, bounds=REF_BOUNDS)
    parts = reference_resident_particles()
    cpu = O.OracleWorld(params, parts)
    session = Session(params, parts, 1e-4)
    for _ in range(2):
        for _ in range(4):
            cpu.step(1e-4)
        session.step(4)
    assert session.substeps() == 8 and cpu.substeps() == 8
    assert_close(cpu.particles(), session.particles(), 2e-5, 2e-4, F=2e-4, C=2e-3)
    # the fixed particle keeps its pose; the consumed force is zero again
    got = session.particles()
    assert np.array_equal(got.position[2], parts.position[2])
    assert np.array_equal(got.velocity[2], [0, 0, 0])
    assert np.array_equal(got.force[0], [0, 0, 0])

    obstacle = Obstacle.sphere((0.5, 0.5, 0.5), 0.1)
    cpu.set_obstacles([obstacle])
    session.set_obstacles([obstacle])
    for _ in range(4):
        cpu.step(1e-4)
    session.step(4)
    assert_close(cpu.particles(), session.particles(), 2e-5, 2e-4)


def test_resident_escape_is_unavailable_and_keeps_world():  # gpu.rs:3730-3745
    params = make_params(0.1, bounds=REF_BOUNDS)
    p = density_particles([(0.95, 0.5, 0.5)], 0.04, 1000.0, MAT_FLUID, (2000.0, 7.0, 0.1, 0.25))
    s = Session(params, p, 1e-4, obstacles=[Obstacle.sphere((0.9, 0.5, 0.5), 10.0)])
    before = s.particles()
    with pytest.raises(TesseraError) as e:
        s.step(4)
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE
    assert np.array_equal(s.particles().position, before.position)
    assert s.substeps() == 0


def test_resident_cfl_violation_is_unavailable_and_force_is_retained():  # gpu.rs:3747-3774
    params = make_params(0.1, bounds=REF_BOUNDS)
    p = density_particles([(0.5, 0.5, 0.5)], 0.04, 1000.0, MAT_NEO_HOOKEAN, (2000.0, 0.2))
    p.force[0, 0] = 4_000_000.0
    s = Session(params, p, 1e-4)
    with pytest.raises(TesseraError) as e:
        s.step(4)
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE
    assert s.substeps() == 0
    with pytest.raises(TesseraError) as e:
        s.step(1)
    assert e.value.status == TMPM_ERR_RESIDENT_UNAVAILABLE
    assert s.particles().force[0, 0] == 4_000_000.0
    ok = Session(params, p, 1e-6)
    ok.step(4)
    assert ok.substeps() == 4
    assert ok.particles().force[0, 0] == 0.0


def test_direct_transfers_track_cpu_for_elastic_particles():  # gpu.rs:4043-4099
    a = density_particles([(0.35, 0.43, 0.53)], 0.04, 1000.0, MAT_ELASTIC, (2000.0, 0.2))
    b = density_particles([(0.41, 0.47, 0.56)], 0.04, 1000.0, MAT_NEO_HOOKEAN, (2000.0, 0.2))
    p = ParticleArrays.concat([a, b])
    p.velocity[0] = (0.2, -0.1, -0.5)
    p.velocity[1] = (-0.1, 0.3, 0.2)
    p.deformation[0, 0] = 0.97  # (0, 0)
    p.deformation[1, 4] = 1.04  # (1, 1)
    params = make_params(0.1, bounds=REF_BOUNDS)
    cpu = O.OracleWorld(params, p)
    cpu.step(0.002)
    s = Session(params, p, 1e-4)
    s.step_cfl(0.002)
    assert s.substeps() == cpu.substeps()
    assert_close(cpu.particles(), s.particles(), 1e-5, 1e-4, F=1e-5, C=1e-3)


def test_obstacle_reactions_match_cpu_momentum_transfer():  # gpu.rs:2602-2649, world.rs:783-807
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0))
    p = density_particles([(1.02, 0.0, 0.0)], 0.04, 1000.0, MAT_ELASTIC, (1000.0, 0.2))
    p.velocity[0, 0] = -1.0
    sphere = Obstacle.sphere((0.0, 0.0, 0.0), 1.0)
    cpu = O.OracleWorld(params, p)
    cpu.set_obstacles([sphere])
    expected = cpu.step_with_obstacle_reactions(0.001, 1)
    s = Session(params, p, 1e-4, obstacles=[sphere])
    got = s.step_cfl_with_reactions(0.001)
    assert np.abs(expected - got).max() < 1e-4
    assert_close(cpu.particles(), s.particles(), 1e-5, 1e-4)
    m = p.mass[0]
    assert np.linalg.norm(p.velocity[0] * m - s.particles().velocity[0] * m - got[0, :3]) < 1e-4


def test_transfer_colors_separate_grid_momentum():  # world.rs:695-718, gpu.rs:4151-4199
    left = density_particles([(0.5, 0.5, 0.5)], 0.04, 1000.0, MAT_ELASTIC, (1000.0, 0.2))
    left.velocity[0, 0] = 1.0
    right = left.copy()
    right.velocity[0, 0] = -1.0
    right.transfer_color[0] = 1
    params = make_params(0.1, gravity=(0.0, 0.0, 0.0))
    s = Session(params, ParticleArrays.concat([left, right]), 1e-4)
    s.step(10)
    v = s.particles().velocity
    assert abs(v[0, 0] - 1.0) < 1e-5 and abs(v[1, 0] + 1.0) < 1e-5
    right.transfer_color[0] = 0
    mixed = Session(params, ParticleArrays.concat([left, right]), 1e-4)
    mixed.step(1)
    v = mixed.particles().velocity
    assert abs(v[0, 0]) < 1e-5 and abs(v[1, 0]) < 1e-5


def test_elastic_block_tracks_oracle_per_substep_and_drift():
    """Config 1 geometry at a reduced block ([0.40, 0.52]^3, ~14k particles)."""
    sc = scenes.elastic_block(lo=(0.40, 0.40, 0.40), hi=(0.52, 0.52, 0.52))
    cpu = O.OracleWorld(sc.params, sc.particles)
    s = Session(sc.params, sc.particles, sc.dt)
    # the stated config-1 dt = 1e-4 is above the CFL bound: the resident path rejects it
    with pytest.raises(TesseraError) as e:
        Session(sc.params, sc.particles, 1e-4)
    assert e.value.status == TMPM_ERR_INVALID_INPUT
    h = sc.params.cell_width
    cpu.substep_fixed(sc.dt)
    s.step(1)
    assert_rel_close(cpu.particles(), s.particles(), h, PER_SUBSTEP, "elastic_block 1")
    for k in range(3):
        for _ in range(16):
            cpu.substep_fixed(sc.dt)
        s.step(16)
        # drift up to 49 substeps of a stiff (c = 105 m/s) block, FP32 vs f64
        assert_rel_close(cpu.particles(), s.particles(), h, DRIFT, f"elastic_block {1 + 16 * (k + 1)}")
    e_v = cpu.particles().velocity
    g_v = s.particles().velocity
    assert np.abs(e_v.mean(axis=0) - g_v.mean(axis=0)).max() < 1e-5


def test_dam_break_subscene_tracks_oracle():
    """Config 2 physics (h = 2.2/256, fluid + elastic cubes) on a column scaled to ~60k particles."""
    sc = scenes.dam_break(scale=0.15)
    params = sc.params
    cpu = O.OracleWorld(params, sc.particles)
    s = Session(params, sc.particles, sc.dt)
    for k in range(4):
        for _ in range(2):
            cpu.substep_fixed(sc.dt)
        s.step(2)
        assert_rel_close(cpu.particles(), s.particles(), params.cell_width, PER_SUBSTEP, f"dam_break_0.15 {2 * k + 2}")


def test_binning_and_sort_order_are_bit_exact():
    sc = scenes.dam_break(scale=0.1)
    s = Session(sc.params, sc.particles, sc.dt)
    widx0, cells0, keys0 = s.debug_binning()
    pos32 = sc.particles.position.astype(np.float32)[widx0]
    ref_cells, ref_keys, ref_perm = O.binning_reference(pos32, sc.params.cell_width)
    assert np.array_equal(cells0, ref_cells)
    assert np.array_equal(keys0, ref_keys)
    s.submit_steps(1)  # the batch opens by re-sorting storage by (block, cell) key
    s.synchronize()
    widx1, cells1, keys1 = s.debug_binning()
    assert np.array_equal(widx1, widx0[O.storage_order(ref_perm)])
    # after one substep the device positions (read back exactly) re-bin identically
    pos1 = s.particles().position.astype(np.float32)[widx1]
    c1, k1, _ = O.binning_reference(pos1, sc.params.cell_width)
    assert np.array_equal(cells1, c1) and np.array_equal(keys1, k1)


def test_p2g_grid_matches_oracle_and_conserves_mass_and_momentum():
    sc = scenes.elastic_block(lo=(0.40, 0.40, 0.40), hi=(0.50, 0.50, 0.50))
    p = sc.particles.copy()
    rng = np.random.default_rng(11)
    p.velocity[:] = rng.normal(0.0, 0.1, size=p.velocity.shape)
    s = Session(sc.params, p, sc.dt)
    cells, mm = s.debug_p2g()
    cpu = O.OracleWorld(sc.params, p)
    keys, vals = cpu.p2g(sc.dt)
    order = np.lexsort((cells[:, 2], cells[:, 1], cells[:, 0]))
    cells, mm = cells[order], mm[order].astype(np.float64)
    assert np.array_equal(cells, keys[:, :3].astype(np.int32))
    scale_m = vals[:, 0].max()
    scale_p = np.abs(vals[:, 1:]).max()
    assert np.abs(mm[:, 0] - vals[:, 0]).max() < 1e-5 * scale_m
    assert np.abs(mm[:, 1:] - vals[:, 1:]).max() < 1e-4 * scale_p
    total_mass = p.mass.sum()
    assert abs(mm[:, 0].sum() - total_mass) < 1e-5 * total_mass
    momentum = (p.mass[:, None] * p.velocity).sum(axis=0)
    assert np.abs(mm[:, 1:].sum(axis=0) - momentum).max() < 1e-4 * np.abs(p.mass[:, None] * p.velocity).sum()


def test_full_size_dam_break_conserves_grid_mass_and_stays_finite():
    """Config 2 at full size (~4.05M particles): size-independent properties."""
    sc = scenes.dam_break()
    assert 3.9e6 < sc.particles.count < 4.2e6
    s = Session(sc.params, sc.particles, sc.dt)
    cells, mm = s.debug_p2g()
    total = sc.particles.mass.sum()
    assert abs(mm[:, 0].astype(np.float64).sum() - total) < 1e-5 * total
    # zero initial velocity and affine: total grid momentum is zero (APIC weights sum dpos to 0)
    assert np.abs(mm[:, 1:].astype(np.float64).sum(axis=0)).max() < 1e-6 * total
    s.step(64)
    got = s.particles()
    assert np.all(np.isfinite(got.position)) and np.all(np.isfinite(got.deformation))
    lo = np.asarray(REF_BOUNDS[0])
    assert np.all(got.position >= lo) and np.all(got.position <= 2.2)
    # after 64 substeps of free fall + pressure the centroid moved down, not up
    assert got.position[:, 2].mean() <= sc.particles.position[:, 2].mean()


def test_full_size_dam_break_per_substep_against_oracle():
    """Config 2 at full size (4,049,637 particles), substep by substep against
    the f64 oracle: before each of three substeps the grid after P2G of the
    current state, then the particles after the substep (x, v, C, F under the
    per-substep relative bounds).  Grid bounds: mass within 2e-5 and momentum
    within 1e-4 of the largest node value.  They are set by the f32 positions:
    at x ~ 2.2 m an f32 ulp is 2.4e-7 m, 2.8e-5 of a cell (h = 2.2/256), so
    each B-spline weight carries a relative error of that order (measured:
    mass 5e-6, momentum 3e-5)."""
    sc = scenes.dam_break()
    assert 3.9e6 < sc.particles.count < 4.2e6
    h = sc.params.cell_width
    cpu = O.OracleWorld(sc.params, sc.particles)
    s = Session(sc.params, sc.particles, sc.dt)
    for k in range(3):
        cells, mm = s.debug_p2g()
        keys, vals = cpu.p2g(sc.dt)
        assert_grid_close(cells, mm, keys, vals, tol_mass=2e-5, tol_momentum=1e-4, label=f"config2 p2g {k}")
        cpu.substep_fixed(sc.dt)
        s.step(1)
        assert_rel_close(cpu.particles(), s.particles(), h, PER_SUBSTEP, f"config2 {k + 1}")
        g = s.particles()
        assert abs(g.mass.sum() - sc.particles.mass.sum()) == 0.0  # masses are never rewritten


def test_capacity_exhaustion_reports_capacity_and_keeps_world():  # gpu.rs:2872-2961
    sc = scenes.sphere_drop()
    s = Session(sc.params, sc.particles, sc.dt, obstacles=sc.obstacles, max_blocks=1)
    before = s.particles()
    with pytest.raises(TesseraError) as e:
        s.step(2)
    assert e.value.status == TMPM_ERR_CAPACITY
    assert np.array_equal(s.particles().position, before.position)
    assert s.substeps() == 0


def test_non_finite_direct_step_reports_non_finite_and_keeps_world():
    # Unbounded: with walls the clamp would turn the infinite velocity into a finite state.
    params = make_params(0.1)
    p = density_particles([(0.5, 0.5, 0.5)], 0.04, 1000.0, MAT_NEO_HOOKEAN, (2000.0, 0.2))
    s = Session(params, p, 1e-4)
    s.set_particle_force(0, (3.0e38, 0.0, 0.0))  # force / mass overflows f32
    before = s.particles()
    with pytest.raises(TesseraError) as e:
        s.step_cfl(1e-4)
    assert e.value.status == TMPM_ERR_NON_FINITE_STATE
    assert np.array_equal(s.particles().position, before.position)
    # the f64 reference path fails too (its overflow comes one step later, in x += v dt)
    q = p.copy()
    q.force[0, 0] = 1.0e308
    cpu = O.OracleWorld(params, q)
    with pytest.raises(O.OracleError) as oe:
        cpu.step(1e-4)
    assert oe.value.status == TMPM_ERR_NON_FINITE_STATE


def test_pending_steps_block_edits_and_synchronize_applies():  # gpu.rs:3306-3409
    sc = scenes.sphere_drop()
    s = Session(sc.params, sc.particles, sc.dt, obstacles=sc.obstacles)
    s.submit_steps(3)
    s.submit_steps(2)
    assert s.pending_substeps() == 5 and s.has_pending_steps()
    with pytest.raises(TesseraError) as e:
        s.set_particle_force(0, (1.0, 0.0, 0.0))
    assert e.value.status == TMPM_ERR_PENDING_STEPS
    s.synchronize()
    assert s.substeps() == 5 and not s.has_pending_steps()
    cpu = O.OracleWorld(sc.params, sc.particles)
    cpu.set_obstacles(sc.obstacles)
    for _ in range(5):
        cpu.substep_fixed(sc.dt)
    assert_close(cpu.particles(), s.particles(), 2e-5, 2e-4, F=2e-4, C=2e-3)


def test_add_and_remove_chunks_keep_world_order():  # gpu.rs:3934-4041
    sc = scenes.sphere_drop()
    s = Session(sc.params, sc.particles, sc.dt)
    extra = density_particles([(0.7, 0.7, 0.7), (0.72, 0.7, 0.7)], 0.0125, 1000.0, MAT_ELASTIC, (3e3, 0.25))
    chunk = s.add_particles(extra)
    assert chunk == 1 and s.count() == sc.particles.count + 2
    s.step(2)
    assert s.remove_chunk(chunk) == 2
    assert s.count() == sc.particles.count
    with pytest.raises(TesseraError):
        s.remove_chunk(chunk)
    s.step(1)
    assert s.substeps() == 3


def test_snapshot_matches_synchronized_state():  # gpu.rs:2964-3161
    import torch
    sc = scenes.sphere_drop()
    s = Session(sc.params, sc.particles, sc.dt)
    s.step(3)
    n = s.count()
    out = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    written = s.encode_particle_snapshot(out.data_ptr(), out.numel() * 4)
    assert written == n
    snap = out.cpu().numpy().astype(np.float64)
    got = s.particles()
    assert np.abs(snap[:, :3] - got.position).max() < 1e-6
    assert np.abs(snap[:, 4:7] - got.velocity).max() < 1e-6
    assert np.allclose(snap[:, 3], got.mass, rtol=1e-6) and np.allclose(snap[:, 7], got.rest_volume, rtol=1e-6)


def test_write_particles_replaces_the_world_and_bad_input_leaves_it():
    """tmpm_write_particles (load, validation, CFL bound and packing in one pass):
    the written world is what the session then advances, like the oracle; an
    invalid particle, a step above the CFL bound or a state f32 cannot hold is
    rejected with the previous world and device state intact."""
    from tessera_b200._abi import TMPM_ERR_MPM_INVALID_INPUT

    sc = scenes.sphere_drop()
    s = Session(sc.params, sc.particles, sc.dt, obstacles=sc.obstacles)
    s.step(4)
    moved = sc.particles.copy()
    moved.position[:, 0] += 0.02
    moved.velocity[:, 1] = 0.3
    moved.chunk_id[:] = 7
    s.write_particles(moved)
    got = s.particles()
    assert np.array_equal(got.position, moved.position) and np.array_equal(got.velocity, moved.velocity)
    assert np.all(got.chunk_id == 7)
    s.step(8)
    w = O.OracleWorld(sc.params, moved)
    w.set_obstacles(sc.obstacles)
    for _ in range(8):
        w.substep_fixed(sc.dt)
    assert_close(w.particles(), s.particles(), 2e-5, 2e-4)
    keep = s.particles()
    bad_mass = moved.copy()
    bad_mass.mass[5] = -1.0
    too_fast = moved.copy()
    too_fast.velocity[9, 2] = 1e4
    no_f32 = moved.copy()
    no_f32.position[3, 0] = 1e39  # finite in f64, beyond f32
    for bad, status in ((bad_mass, TMPM_ERR_MPM_INVALID_INPUT), (too_fast, TMPM_ERR_INVALID_INPUT),
                        (no_f32, TMPM_ERR_INVALID_INPUT)):
        with pytest.raises(TesseraError) as e:
            s.write_particles(bad)
        assert e.value.status == status
        now = s.particles()
        assert np.array_equal(now.position, keep.position) and np.array_equal(now.velocity, keep.velocity)
    # the session still advances the kept world like the oracle
    s.step(2)
    for _ in range(2):
        w.substep_fixed(sc.dt)
    assert_close(w.particles(), s.particles(), 2e-5, 2e-4)


def test_config1_full_block_200_substeps_bounded_drift():
    """Configuration 1 at its stated size (corotated block [0.3, 0.6]^3, h = 1/64,
    8 per cell: 54,872 particles) for 200 substeps (dt = 5e-5: the stated 1e-4 is
    above this block's CFL bound, see test_elastic_block_tracks_oracle_per_substep_and_drift),
    checked against the f64 oracle every 50 substeps with the resident
    tolerances (gpu.rs:3699-3703): the FP32 drift stays bounded (measured
    ~1e-7 in position and ~4e-7 in velocity after 200 substeps)."""
    sc = scenes.elastic_block()
    assert sc.particles.count == 54872
    h = sc.params.cell_width
    cpu = O.OracleWorld(sc.params, sc.particles)
    s = Session(sc.params, sc.particles, sc.dt)
    done = 0
    for chunk in (1, 1, 2, 4, 8, 16, 18, 50, 50, 50):  # checkpoints at 1, 2, 4, 8, ..., 200 substeps
        for _ in range(chunk):
            cpu.substep_fixed(sc.dt)
        s.step(chunk)
        done += chunk
        e, g = cpu.particles(), s.particles()
        assert_rel_close(e, g, h, PER_SUBSTEP if done <= 8 else DRIFT, f"config1 {done}")
        assert_close(e, g, 2e-5, 2e-4, F=2e-4)
        assert np.abs(e.velocity.mean(axis=0) - g.velocity.mean(axis=0)).max() < 1e-6  # momentum per unit mass
    assert s.substeps() == done == 200
