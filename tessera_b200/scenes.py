"""Seeded synthetic MPM scenes with the shapes of the benchmark configurations.

Particles are placed as BoxEmitter does (crates/tessera-mpm/src/emitter.rs:165-224):
a lattice of spacing ``2 r``, rest volume ``(2 r)^3`` and mass ``rho (2 r)^3``
(world.rs:118-150).  With ``r = h / 4`` that is 8 particles per grid cell.  A
seeded uniform jitter (a fraction of the half spacing) moves each particle
inside its own lattice cell.  Gravity points along -z, the reference default
(world.rs:40-49).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from ._abi import MAT_ELASTIC, MAT_FLUID, Obstacle, ParticleArrays, TmpmParams, density_particles, make_params


@dataclass
class Scene:
    name: str
    params: TmpmParams
    particles: ParticleArrays
    dt: float
    substeps: int
    obstacles: list = field(default_factory=list)
    info: dict = field(default_factory=dict)


def lattice(lo, hi, spacing, rng=None, jitter=0.5):
    """Lattice points (cell centres of spacing `spacing`) inside the box [lo, hi]."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    counts = np.floor((hi - lo) / spacing + 1e-9).astype(int)
    axes = [lo[a] + spacing * (np.arange(counts[a]) + 0.5) for a in range(3)]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    if rng is not None and jitter > 0:
        g = g + rng.uniform(-0.5 * jitter * spacing, 0.5 * jitter * spacing, size=g.shape)
    return g


def elastic_block(seed=1, cell_width=1.0 / 64, lo=(0.3, 0.3, 0.3), hi=(0.6, 0.6, 0.6), young=1e4, poisson=0.2,
                  density=1.0, gravity=(0.0, 0.0, -9.8), dt=5e-5, substeps=400, wall_mode=0, jitter=0.5,
                  max_substep=1e-3, name="config1-corotated-block"):
    """Config 1: unit cube, h = 1/64, corotated block [0.3, 0.6]^3 at 8 particles per cell.

    The stated dt = 1e-4 exceeds this material's CFL bound 0.4 h / c = 5.9e-5
    (c = sqrt((lambda + 2 mu) / rho) = 105 m/s), which the resident path rejects
    (gpu.rs:664-677).  The default therefore takes 400 substeps of 5e-5, the
    same 0.02 s of simulated time.
    """
    rng = np.random.default_rng(seed)
    r = cell_width / 4.0
    pos = lattice(lo, hi, 2.0 * r, rng, jitter)
    parts = density_particles(pos, r, density, MAT_ELASTIC, (young, poisson))
    params = make_params(cell_width, gravity=gravity, max_substep=max_substep, bounds=((0, 0, 0), (1, 1, 1)),
                         wall_mode=wall_mode)
    return Scene(name, params, parts, dt, substeps, info=dict(particles=len(pos), cell_width=cell_width))


def dam_break(seed=2, side=2.2, resolution=256, column=(0.4, 0.8, 1.0), bulk=1e4, gamma=7.0, viscosity=0.01,
              fluid_density=1000.0, cube_side=0.1, cube_young=1e4, cube_poisson=0.2, cube_density=1000.0,
              dt=5e-5, substeps=500, jitter=0.5, scale=1.0, name="config2-dam-break"):
    """Config 2: 256^3 virtual domain of side 2.2 m (h = 2.2 / 256), weakly
    compressible fluid column [0, 0.4] x [0, 0.8] x [0, 1] (~4.0M particles at 8
    per cell) plus three elastic cubes of side 0.1 at seeded positions.

    `scale` < 1 shrinks the column's footprint (x and y) for small test cases
    while keeping h, dt and the materials.
    """
    rng = np.random.default_rng(seed)
    h = side / resolution
    r = h / 4.0
    col = np.array(column, dtype=np.float64)
    col[:2] *= scale
    fluid = lattice((0.0, 0.0, 0.0), col, 2.0 * r, rng, jitter)
    parts = [density_particles(fluid, r, fluid_density, MAT_FLUID, (bulk, gamma, viscosity, 0.25))]
    cubes = []
    for _ in range(3):
        lo = np.array([rng.uniform(col[0] + 0.2, side - 0.2 - cube_side),
                       rng.uniform(0.1, min(side - 0.1 - cube_side, max(col[1], 0.3) + 0.3)),
                       rng.uniform(0.1, 1.0)])
        cubes.append(lo)
        pts = lattice(lo, lo + cube_side, 2.0 * r, rng, jitter)
        parts.append(density_particles(pts, r, cube_density, MAT_ELASTIC, (cube_young, cube_poisson)))
    allp = ParticleArrays.concat(parts)
    params = make_params(h, gravity=(0.0, 0.0, -9.81), max_substep=1e-3, bounds=((0, 0, 0), (side, side, side)))
    return Scene(name, params, allp, dt, substeps,
                 info=dict(particles=allp.count, fluid=len(fluid), cubes=[c.tolist() for c in cubes], cell_width=h))


def dam_break_obstacle(seed=2, scale=1.0, center=(0.40, 0.40, 0.10), radius=0.12, friction=0.3):
    """Config 2 with a rigid sphere obstacle straddling the column's front face
    near the floor (the particles it would hold, and those within half a cell
    of its surface, are left out): the column collapses around and over it,
    so the particle and grid contact run from the first substep on."""
    sc = dam_break(seed=seed, scale=scale, name="config2-dam-break-sphere")
    c = np.asarray(center, dtype=np.float64)
    c[1] *= scale if scale < 1.0 else 1.0
    h = sc.params.cell_width
    keep = np.linalg.norm(sc.particles.position - c, axis=1) > radius + 0.5 * h
    sc.particles = sc.particles.select(np.nonzero(keep)[0])
    sc.obstacles = [Obstacle.sphere(tuple(c), radius, friction=friction)]
    sc.info["obstacle"] = dict(shape="sphere", center=c.tolist(), radius=radius, friction=friction)
    sc.info["particles"] = sc.particles.count
    return sc


def adjoint_block(seed=5, young=5e3, poisson=0.3, density=1000.0, dt=1e-4, substeps=256, jitter=0.5,
                  cells=20, velocity=None, name="config5-corotated-block"):
    """Config 5: 64k-particle corotated block (20^3 cells at 8 per cell) on a 64^3 grid
    of the unit cube, two cells above the floor, moving down onto it.

    The block position and initial velocity are not given with the workload.  A
    block that touches no wall conserves linear momentum exactly (the B-spline
    weights have zero first moment and gravity is uniform), so its final
    centroid - and the loss - would not depend on Young's modulus at all.  The
    block therefore starts next to the floor with a seeded downward velocity:
    the floor's separating wall acts from the first substep and the loss
    depends on E through the contact.
    """
    h = 1.0 / 64
    rng = np.random.default_rng(seed)
    lo = np.array([22.0, 22.0, 2.0]) * h
    sc = elastic_block(seed=seed, cell_width=h, lo=lo, hi=lo + cells * h, young=young, poisson=poisson,
                       density=density, dt=dt, substeps=substeps, jitter=jitter, name=name,
                       gravity=(0.0, 0.0, -9.81))
    if velocity is None:
        velocity = (rng.uniform(-0.2, 0.2), rng.uniform(-0.2, 0.2), -rng.uniform(0.3, 0.6))
    sc.particles.velocity[:] = np.asarray(velocity, dtype=np.float64)
    sc.info["target"] = (0.5 + rng.uniform(-0.1, 0.1), 0.5 + rng.uniform(-0.1, 0.1), 0.2 + rng.uniform(-0.05, 0.05))
    return sc


def sphere_drop(seed=3, n_side=8, cell_width=0.05, name="sphere-drop"):
    """Small mixed-material scene with a slip sphere obstacle (test case)."""
    rng = np.random.default_rng(seed)
    r = cell_width / 4.0
    pos = lattice((0.3, 0.3, 0.55), (0.3 + n_side * 2 * r, 0.3 + n_side * 2 * r, 0.55 + n_side * 2 * r), 2 * r,
                  rng, 0.5)
    parts = density_particles(pos, r, 1000.0, MAT_ELASTIC, (3e3, 0.25))
    params = make_params(cell_width, gravity=(0.0, 0.0, -9.81), max_substep=1e-3, bounds=((0, 0, 0), (1, 1, 1)))
    obstacles = [Obstacle.sphere((0.35, 0.35, 0.4), 0.1, friction=0.3)]
    return Scene(name, params, parts, 1e-4, 20, obstacles=obstacles)


def batch_scene(seed, cells=None, density=1000.0, dt=1e-4, substeps=100, jitter=0.5, name=None):
    """One scene of the heterogeneous batch: a block of `cells`^3 cells (8 particles
    per cell) in the unit cube at resolution 4 * `cells` (so the block spans a
    quarter of the domain side), at a seeded interior position; material drawn
    uniformly from corotated elastic (E log-uniform in [1e3, 1e5], nu = 0.2) and
    weakly compressible fluid (K = 1e4, gamma = 7).  Without `cells` the particle
    count is drawn log-uniform in [4096, 262144] (cells 8..32, resolution 32..128).

    The density is not given with the workload; rho = 1000 keeps dt = 1e-4 under
    the CFL bound 0.4 h / c for every draw (E = 1e5 at h = 1/128 needs rho > 114).
    """
    rng = np.random.default_rng(seed)
    if cells is None:
        n = float(np.exp(rng.uniform(np.log(4096.0), np.log(262144.0))))
        cells = int(np.clip(round((n / 8.0) ** (1.0 / 3.0)), 8, 32))
    res = 4 * cells
    h = 1.0 / res
    side = cells * h
    lo = np.array([rng.uniform(4 * h, 1.0 - side - 4 * h) for _ in range(3)])
    lo = np.round(lo / h) * h
    r = h / 4.0
    pos = lattice(lo, lo + side, 2.0 * r, rng, jitter)
    if rng.uniform() < 0.5:
        young = float(np.exp(rng.uniform(np.log(1e3), np.log(1e5))))
        parts = density_particles(pos, r, density, MAT_ELASTIC, (young, 0.2))
        material = dict(material="elastic", young=young)
    else:
        parts = density_particles(pos, r, density, MAT_FLUID, (1e4, 7.0, 0.01, 0.25))
        material = dict(material="fluid", bulk=1e4)
    params = make_params(h, gravity=(0.0, 0.0, -9.8), max_substep=1e-3, bounds=((0, 0, 0), (1, 1, 1)))
    return Scene(name or f"batch-scene-{seed}", params, parts, dt, substeps,
                 info=dict(particles=len(pos), resolution=res, **material))


def batch_scenes(count=256, seed=3, max_cells=None, dt=1e-4, substeps=100):
    """The heterogeneous batch: `count` independent scenes seeded seed*1000 + k.
    `max_cells` caps the block size (small test batches)."""
    out = []
    for k in range(count):
        sc = batch_scene(seed * 1000 + k, dt=dt, substeps=substeps)
        if max_cells is not None and sc.info["resolution"] // 4 > max_cells:
            sc = batch_scene(seed * 1000 + k, cells=max_cells, dt=dt, substeps=substeps)
        out.append(sc)
    return out
