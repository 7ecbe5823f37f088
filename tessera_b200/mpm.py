"""tessera3d-compatible MPM API backed by the B200 library.

Mirrors the UniFFI surface of ``tessera3d.MpmWorld`` and its records
(crates/tessera-python3d/src/mpm.rs:48-1283): the same class, method and field
names, argument meaning and error behaviour (every failure raises
``TesseraError`` with a reason, lib.rs:82-95).

One difference of mechanism, not of results: the reference's ``step`` runs its
CPU pipeline and ``step_gpu`` a per-substep upload/readback; here both run the
same CFL-limited substeps (world.rs:332-359) on the device through one resident
session, which also serves ``step_gpu_fixed``.  The session is rebuilt whenever
the reference would rebuild its resident buffers (parameter changes), and after
a device error the last synchronized world is kept, as in mpm.rs:839-842.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._abi import (
    BOUNDARY_FREE_SLIP, BOUNDARY_NON_REFLECTING, BOUNDARY_SEPARATE, BOUNDARY_SLIP, BOUNDARY_STICK,
    MAT_ELASTIC, MAT_FLUID, MAT_NEO_HOOKEAN, MAT_SAND, MAT_SAND_NEO_HOOKEAN, MAT_SNOW, Obstacle, ParticleArrays,
    make_params,
)
from .session import Session, TesseraError

__all__ = [
    "Vec3", "Quaternion", "MpmMaterial", "MpmParticleInput", "MpmParticleState", "MpmObstacleShape",
    "MpmObstacleInput", "MpmBoundary", "MpmWorld", "TesseraError",
]


@dataclass
class Vec3:
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0

    def tuple(self):
        return (float(self.x), float(self.y), float(self.z))


@dataclass
class Quaternion:
    """XYZW unit quaternion (mpm.rs:359-360)."""
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0
    w: float = 1.0


@dataclass
class _Material:
    kind: int
    params: tuple


class MpmMaterial:
    """Constitutive model variants (mpm.rs:48-111) as factory functions."""

    @staticmethod
    def ELASTIC(young_modulus, poisson_ratio):
        return _Material(MAT_ELASTIC, (young_modulus, poisson_ratio))

    @staticmethod
    def NEO_HOOKEAN(young_modulus, poisson_ratio):
        return _Material(MAT_NEO_HOOKEAN, (young_modulus, poisson_ratio))

    @staticmethod
    def SAND(young_modulus, poisson_ratio, friction_angle, cohesion):
        return _Material(MAT_SAND, (young_modulus, poisson_ratio, friction_angle, cohesion))

    @staticmethod
    def FLUID(bulk_modulus, gamma, viscosity, tensile_stiffness):
        return _Material(MAT_FLUID, (bulk_modulus, gamma, viscosity, tensile_stiffness))

    @staticmethod
    def SNOW(young_modulus, poisson_ratio, critical_compression, critical_stretch, hardening):
        return _Material(MAT_SNOW, (young_modulus, poisson_ratio, critical_compression, critical_stretch, hardening))

    @staticmethod
    def SAND_NEO_HOOKEAN(young_modulus, poisson_ratio, friction_angle, cohesion):
        return _Material(MAT_SAND_NEO_HOOKEAN, (young_modulus, poisson_ratio, friction_angle, cohesion))


@dataclass
class MpmParticleInput:
    """New material point (mpm.rs:180-199)."""
    position: Vec3
    velocity: Vec3
    radius: float
    density: float
    material: _Material
    enabled: bool = True
    fixed: bool = False
    damping: float = 0.0


@dataclass
class MpmParticleState:
    """Particle state in insertion order (mpm.rs:240-271); matrices column-major."""
    position: Vec3
    velocity: Vec3
    mass: float
    rest_volume: float
    radius: float
    deformation: list
    affine: list
    plastic_det: float
    hardening: float
    log_volume_gain: float
    chunk_id: int
    enabled: bool
    fixed: bool
    transfer_color: int


@dataclass
class _Shape:
    kind: str
    fields: dict = field(default_factory=dict)


class MpmObstacleShape:
    """Obstacle shape variants (mpm.rs:294-350)."""

    @staticmethod
    def SPHERE(radius):
        return _Shape("sphere", dict(radius=radius))

    @staticmethod
    def BOX(half_extents):
        return _Shape("box", dict(half_extents=half_extents))

    @staticmethod
    def CAPSULE(half_height, radius):
        return _Shape("capsule", dict(half_height=half_height, radius=radius))

    @staticmethod
    def CYLINDER(half_height, radius):
        return _Shape("cylinder", dict(half_height=half_height, radius=radius))

    @staticmethod
    def CONE(half_height, radius):
        return _Shape("cone", dict(half_height=half_height, radius=radius))

    @staticmethod
    def GROUND(half_extent_x, half_extent_y):
        return _Shape("ground", dict(half_extent_x=half_extent_x, half_extent_y=half_extent_y))

    @staticmethod
    def TRIANGLE_PRISM(vertices, half_thickness):
        return _Shape("triangle_prism", dict(vertices=vertices, half_thickness=half_thickness))

    @staticmethod
    def CONVEX(vertices, face_normals):
        return _Shape("convex", dict(vertices=vertices, face_normals=face_normals))


@dataclass
class MpmObstacleInput:
    """Prescribed obstacle pose, motion and friction (mpm.rs:352-367)."""
    shape: _Shape
    center: Vec3
    orientation: Quaternion = field(default_factory=Quaternion)
    linear_velocity: Vec3 = field(default_factory=Vec3)
    angular_velocity: Vec3 = field(default_factory=Vec3)
    friction: float = 0.0


class MpmBoundary:
    SLIP = BOUNDARY_SLIP
    STICK = BOUNDARY_STICK
    SEPARATE = BOUNDARY_SEPARATE
    NON_REFLECTING = BOUNDARY_NON_REFLECTING
    FREE_SLIP = BOUNDARY_FREE_SLIP


def _vec(v) -> tuple:
    if isinstance(v, Vec3):
        return v.tuple()
    return tuple(float(c) for c in v)


def _unit_orientation(q: Quaternion):
    """mpm.rs:408-417: |q|^2 must be within 1e-5 of one; then normalized."""
    n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w
    if not math.isfinite(n2) or abs(n2 - 1.0) > 1e-5:
        raise TesseraError("obstacle orientation must be a unit quaternion")
    n = math.sqrt(n2)
    return (q.x / n, q.y / n, q.z / n, q.w / n)


def _obstacle(inp: MpmObstacleInput) -> Obstacle:
    """mpm.rs:419-482."""
    c = _vec(inp.center)
    q = _unit_orientation(inp.orientation)
    f = inp.shape.fields
    kind = inp.shape.kind
    if kind == "sphere":
        ob = Obstacle.sphere(c, f["radius"])
    elif kind == "box":
        ob = Obstacle.cuboid(c, _vec(f["half_extents"]), q)
    elif kind == "capsule":
        ob = Obstacle.capsule(c, f["half_height"], f["radius"], q)
    elif kind == "cylinder":
        ob = Obstacle.cylinder(c, f["half_height"], f["radius"], q)
    elif kind == "cone":
        ob = Obstacle.cone(c, f["half_height"], f["radius"], q)
    elif kind == "ground":
        ob = Obstacle.ground(c, (f["half_extent_x"], f["half_extent_y"]), q)
    elif kind == "triangle_prism":
        verts = list(f["vertices"])
        if len(verts) != 3:
            raise TesseraError("triangle prism requires exactly three vertices")
        ob = Obstacle.triangle_prism(c, [_vec(v) for v in verts], f["half_thickness"], q)
    elif kind == "convex":
        ob = Obstacle.convex(c, [_vec(v) for v in f["vertices"]], [_vec(n) for n in f["face_normals"]], q)
    else:
        raise TesseraError(f"unknown obstacle shape {kind}")
    ob.orientation = q
    ob.linear_velocity = _vec(inp.linear_velocity)
    ob.angular_velocity = _vec(inp.angular_velocity)
    ob.friction = float(inp.friction)
    if not _obstacle_valid(ob):
        raise TesseraError("invalid MPM obstacle")
    return ob


def _finite(*vals) -> bool:
    return all(math.isfinite(float(v)) for v in vals)


def _obstacle_valid(o: Obstacle) -> bool:
    """RigidObstacle::is_valid (obstacle.rs:264-341)."""
    d = o.dims
    if o.shape == 0:
        ok = _finite(d[0]) and d[0] > 0
    elif o.shape == 1:
        ok = all(_finite(v) and v > 0 for v in d)
    elif o.shape == 2:
        ok = _finite(d[0], d[1]) and d[0] >= 0 and d[1] >= 0 and (d[0] > 0 or d[1] > 0)
    elif o.shape in (3, 4, 5):
        ok = _finite(d[0], d[1]) and d[0] > 0 and d[1] > 0
    elif o.shape == 6:
        v = np.asarray(o.vertices, dtype=float).reshape(3, 3)
        area = float(np.sum(np.cross(v[1] - v[0], v[2] - v[0]) ** 2))
        ok = _finite(d[0]) and d[0] > 0 and bool(np.all(np.isfinite(v))) and math.isfinite(area) and area > 1e-24
    elif o.shape == 7:
        pl = np.asarray(o.planes if o.planes is not None else np.zeros((0, 4)))
        ok = (len(pl) >= 4 and _finite(o.bound_radius) and o.bound_radius > 0 and bool(np.all(np.isfinite(pl)))
              and bool(np.all(np.abs((pl[:, :3] ** 2).sum(axis=1) - 1.0) <= 1e-4)))
    else:
        ok = False
    cpic = o.cpic_group < 0 or (o.cpic_group < 32 and o.shape == 6)
    return bool(ok and cpic and _finite(*o.center, *o.orientation, *o.linear_velocity, *o.angular_velocity)
                and _finite(o.friction) and o.friction >= 0)


def _valid_elasticity(e, nu):
    return np.isfinite(e) & (e > 0) & np.isfinite(nu) & (nu >= -1.0) & (nu < 0.5)


def _materials_valid(material: np.ndarray, p: np.ndarray) -> np.ndarray:
    """MaterialModel::is_valid (material.rs:171-231), vectorized."""
    ok = np.zeros(len(material), dtype=bool)
    e, nu = p[:, 0], p[:, 1]
    el = np.isin(material, (MAT_ELASTIC, MAT_NEO_HOOKEAN))
    ok[el] = _valid_elasticity(e, nu)[el]
    sand = np.isin(material, (MAT_SAND, MAT_SAND_NEO_HOOKEAN))
    ok[sand] = (_valid_elasticity(e, nu) & np.isfinite(p[:, 2]) & (p[:, 2] >= 0) & (p[:, 2] < math.pi / 2)
                & np.isfinite(p[:, 3]) & (p[:, 3] >= 0))[sand]
    fl = material == MAT_FLUID
    ok[fl] = (np.isfinite(p[:, 0]) & (p[:, 0] > 0) & np.isfinite(p[:, 1]) & (p[:, 1] > 0) & np.isfinite(p[:, 2])
              & (p[:, 2] >= 0) & np.isfinite(p[:, 3]) & (p[:, 3] >= 0))[fl]
    sn = material == MAT_SNOW
    ok[sn] = (_valid_elasticity(e, nu) & np.isfinite(p[:, 2]) & (p[:, 2] >= 0) & (p[:, 2] < 1) & np.isfinite(p[:, 3])
              & (p[:, 3] >= 0) & np.isfinite(p[:, 4]) & (p[:, 4] >= 0))[sn]
    return ok


def _particles_valid(a: ParticleArrays) -> bool:
    """valid_particle (world.rs:492-503) for every particle."""
    if a.count == 0:
        return True
    fin = all(np.all(np.isfinite(getattr(a, f))) for f in
              ("position", "velocity", "deformation", "affine", "force", "mass", "rest_volume", "radius", "damping"))
    return bool(fin and np.all(a.mass > 0) and np.all(a.rest_volume > 0) and np.all(a.radius > 0)
                and np.all(_materials_valid(a.material, a.material_params)) and np.all(a.damping >= 0)
                and np.all(np.isfinite(a.plastic)) and np.all(a.plastic[:, 0] > 0))


def _inputs_to_arrays(particles) -> ParticleArrays:
    """MpmParticleInput -> MpmParticle::new (mpm.rs:224-238, world.rs:118-150)."""
    particles = list(particles)
    out = ParticleArrays(len(particles))
    for i, p in enumerate(particles):
        v0 = (2.0 * float(p.radius)) ** 3
        out.position[i] = _vec(p.position)
        out.velocity[i] = _vec(p.velocity)
        out.radius[i] = float(p.radius)
        out.rest_volume[i] = v0
        out.mass[i] = float(p.density) * v0
        out.material[i] = p.material.kind
        prm = list(p.material.params) + [0.0] * (5 - len(p.material.params))
        out.material_params[i] = prm
        out.enabled[i] = 1 if p.enabled else 0
        out.fixed[i] = 1 if p.fixed else 0
        out.damping[i] = float(p.damping)
        out.plastic[i] = (1.0, 1.0 if p.material.kind in (MAT_SAND, MAT_SAND_NEO_HOOKEAN) else 0.0, 0.0)
    return out


def _params_valid(cell_width, gravity, max_substep, bounds) -> bool:
    """MpmParams::validate (world.rs:51-65)."""
    if not (_finite(cell_width) and cell_width > 0 and _finite(*gravity) and _finite(max_substep) and max_substep > 0):
        return False
    if bounds is not None:
        lo, hi = bounds
        if not _finite(*lo, *hi) or any(not (h - l > 0) for l, h in zip(lo, hi)):
            return False
    return True


def _bounds(bounds_min, bounds_max):
    if bounds_min is None and bounds_max is None:
        return None
    if bounds_min is None or bounds_max is None:
        raise TesseraError("both MPM bounds corners must be supplied")
    return (_vec(bounds_min), _vec(bounds_max))


class MpmWorld:
    """Three-dimensional MPM world (mpm.rs:630-1283), stepped on the B200."""

    def __init__(self, particles, gravity, cell_width, max_substep, bounds_min=None, bounds_max=None, *,
                 device: int = 0):
        bounds = _bounds(bounds_min, bounds_max)
        g = _vec(gravity)
        if not _params_valid(cell_width, g, max_substep, bounds):
            raise TesseraError("invalid MPM input")
        arrays = _inputs_to_arrays(particles)
        if not _particles_valid(arrays):
            raise TesseraError("invalid MPM input")
        self._device = device
        self._cell_width = float(cell_width)
        self._gravity = g
        self._max_substep = float(max_substep)
        self._bounds = bounds
        self._use_cpic = True
        self._frame_substeps = 1
        self._world = arrays
        self._obstacles: list[Obstacle] = []
        self._substeps = 0
        self._chunks = {0} if arrays.count else set()
        self._next_chunk = 1
        self._session: Session | None = None

    # ---------------------------------------------------------------- helpers
    def _tparams(self):
        return make_params(self._cell_width, self._gravity, self._max_substep, self._bounds)

    def _arrays(self) -> ParticleArrays:
        if self._session is not None:
            return self._session.particles()
        return self._world

    def _pending(self) -> int:
        return self._session.pending_substeps() if self._session is not None else 0

    def _reject_pending(self):
        if self._pending() > 0:
            raise TesseraError("synchronize pending GPU substeps before editing MPM state")

    def _drop_session(self):
        """Keep the last synchronized world and release the device session."""
        if self._session is not None:
            self._world = self._session.particles()
            self._substeps = self._session.substeps()
            self._session.close()
            self._session = None

    def _ensure_session(self, substep_dt=None) -> Session:
        if self._session is None:
            probe = substep_dt if substep_dt is not None else 1e-30
            self._session = Session(self._tparams(), self._world, probe, obstacles=self._obstacles,
                                    use_cpic=self._use_cpic, device=self._device, next_chunk_id=self._next_chunk,
                                    substeps=self._substeps)
        elif substep_dt is not None and self._session.substep_dt() != substep_dt:
            self._session.set_substep_dt(substep_dt)
        return self._session

    # ------------------------------------------------------------ parameters
    def _set_configuration(self, cell_width, gravity, max_substep, bounds, use_cpic):
        if not _params_valid(cell_width, gravity, max_substep, bounds):
            raise TesseraError("invalid MPM input")
        self._reject_pending()
        arrays = self._arrays()
        old = (self._cell_width, self._gravity, self._max_substep, self._bounds, self._use_cpic)
        self._cell_width, self._gravity, self._max_substep, self._bounds, self._use_cpic = (
            float(cell_width), tuple(gravity), float(max_substep), bounds, bool(use_cpic))
        if self._session is not None:
            # validate device representability by building the replacement first (mpm.rs:540-567)
            try:
                replacement = Session(self._tparams(), arrays, 1e-30, obstacles=self._obstacles,
                                      use_cpic=self._use_cpic, device=self._device, next_chunk_id=self._next_chunk,
                                      substeps=self._session.substeps())
            except TesseraError:
                self._cell_width, self._gravity, self._max_substep, self._bounds, self._use_cpic = old
                raise
            self._substeps = self._session.substeps()
            self._session.close()
            self._session = replacement
        self._world = arrays

    def set_gravity(self, gravity):
        self._set_configuration(self._cell_width, _vec(gravity), self._max_substep, self._bounds, self._use_cpic)

    def gravity(self) -> Vec3:
        return Vec3(*self._gravity)

    def set_params(self, gravity, cell_width, max_substep, bounds_min=None, bounds_max=None):
        self._set_configuration(cell_width, _vec(gravity), max_substep, _bounds(bounds_min, bounds_max),
                                self._use_cpic)

    def set_substeps(self, substeps: int):
        self._reject_pending()
        self._frame_substeps = max(int(substeps), 1)

    def frame_substeps(self) -> int:
        return self._frame_substeps

    def set_use_cpic(self, enabled: bool):
        self._set_configuration(self._cell_width, self._gravity, self._max_substep, self._bounds, bool(enabled))

    def use_cpic(self) -> bool:
        return self._use_cpic

    # ---------------------------------------------------------------- stepping
    def step(self, dt: float):
        """CFL-limited substeps of total `dt` / frame_substeps each (mpm.rs:758-772), on the device."""
        self._reject_pending()
        substep_dt = float(dt) / self._frame_substeps
        if not math.isfinite(dt) or substep_dt <= 0:
            raise TesseraError("invalid MPM frame timestep")
        session = self._ensure_session()
        for _ in range(self._frame_substeps):
            self._run(lambda: session.step_cfl(substep_dt))

    def step_gpu(self, dt: float):
        """MpmWorld.step_gpu (mpm.rs:774-799)."""
        self.step(dt)

    def step_gpu_fixed(self, substep_dt: float, steps: int):
        """Fixed resident substeps, session kept while dt and state agree (mpm.rs:801-853)."""
        if not math.isfinite(substep_dt) or substep_dt <= 0 or steps == 0 or steps > 64:
            raise TesseraError("invalid fixed GPU substep input")
        self._reject_pending()
        session = self._run(lambda: self._ensure_session(float(substep_dt)))
        self._run(lambda: session.step(int(steps)))

    def submit_gpu_fixed(self, substep_dt: float, steps: int):
        """Queue fixed substeps without synchronizing (GpuMpmResidentSession::submit_steps)."""
        if not math.isfinite(substep_dt) or substep_dt <= 0 or steps == 0 or steps > 64:
            raise TesseraError("invalid fixed GPU substep input")
        if self._pending() and self._session.substep_dt() != substep_dt:
            raise TesseraError("synchronize pending GPU substeps before changing the substep")
        session = self._run(lambda: self._ensure_session(float(substep_dt)))
        self._run(lambda: session.submit_steps(int(steps)))

    def _run(self, fn):
        try:
            return fn()
        except TesseraError:
            # a failed step invalidates the session; keep the last synchronized world
            if self._session is not None:
                world = self._session.particles()
                subs = self._session.substeps()
                self._session.close()
                self._session = None
                self._world = world
                self._substeps = subs
            raise

    def synchronize_gpu(self):
        if self._session is None:
            return
        self._run(self._session.synchronize)

    def pending_gpu_substeps(self) -> int:
        return self._pending()

    def substeps(self) -> int:
        return self._session.substeps() if self._session is not None else self._substeps

    # ------------------------------------------------------------------ state
    def particle_arrays(self) -> ParticleArrays:
        """All particles as numpy arrays (fast path; world order)."""
        return self._arrays()

    def particles(self):
        a = self._arrays()
        out = []
        for i in range(a.count):
            out.append(MpmParticleState(
                position=Vec3(*a.position[i]), velocity=Vec3(*a.velocity[i]), mass=float(a.mass[i]),
                rest_volume=float(a.rest_volume[i]), radius=float(a.radius[i]),
                deformation=a.deformation[i].tolist(), affine=a.affine[i].tolist(),
                plastic_det=float(a.plastic[i, 0]), hardening=float(a.plastic[i, 1]),
                log_volume_gain=float(a.plastic[i, 2]), chunk_id=int(a.chunk_id[i]), enabled=bool(a.enabled[i]),
                fixed=bool(a.fixed[i]), transfer_color=int(a.transfer_color[i])))
        return out

    def add_particles(self, particles) -> int:
        self._reject_pending()
        new = _inputs_to_arrays(particles)
        if new.count == 0 or not _particles_valid(new):
            raise TesseraError("invalid MPM input")
        if self._session is not None:
            chunk = self._session.add_particles(new)
        else:
            chunk = self._next_chunk
            new.chunk_id[:] = chunk
            self._world = ParticleArrays.concat([self._world, new]) if self._world.count else new
        self._next_chunk = chunk + 1
        self._chunks.add(chunk)
        return chunk

    def remove_chunk(self, chunk_id: int) -> int:
        self._reject_pending()
        if chunk_id not in self._chunks:
            raise TesseraError("unknown MPM particle chunk")
        if self._session is not None:
            removed = self._session.remove_chunk(chunk_id)
        else:
            keep = self._world.chunk_id != chunk_id
            removed = int(np.count_nonzero(~keep))
            if removed == 0:
                raise TesseraError("MPM particle chunk was not found")
            self._world = self._world.select(keep)
        self._chunks.discard(chunk_id)
        return removed

    def set_obstacles(self, obstacles):
        obs = [_obstacle(o) for o in obstacles]
        self._replace_obstacles(obs)

    def _replace_obstacles(self, obs):
        self._reject_pending()
        if self._session is not None:
            self._session.set_obstacles(obs)
        self._obstacles = obs

    def set_obstacle_boundaries(self, boundaries):
        if len(boundaries) != len(self._obstacles):
            raise TesseraError("MPM boundary count must match obstacle count")
        obs = [Obstacle(**{**o.__dict__, "boundary": int(b)}) for o, b in zip(self._obstacles, boundaries)]
        self._replace_obstacles(obs)

    def obstacle_boundaries(self):
        return [o.boundary for o in self._obstacles]

    def set_obstacle_cpic_groups(self, groups):
        if len(groups) != len(self._obstacles):
            raise TesseraError("MPM CPIC group count must match obstacle count")
        obs = []
        for o, g in zip(self._obstacles, groups):
            ob = Obstacle(**{**o.__dict__, "cpic_group": -1 if g is None else int(g)})
            if not _obstacle_valid(ob):
                raise TesseraError("invalid MPM CPIC group or obstacle shape")
            obs.append(ob)
        self._replace_obstacles(obs)

    def obstacle_cpic_groups(self):
        return [None if o.cpic_group < 0 else o.cpic_group for o in self._obstacles]

    def obstacle_count(self) -> int:
        return len(self._obstacles)

    def set_particle_force(self, index: int, force):
        """Force consumed by the next particle step (mpm.rs:1249-1264)."""
        f = _vec(force)
        n = self._session.count() if self._session is not None else self._world.count
        if index < 0 or index >= n:
            raise TesseraError("MPM particle index out of range")
        if not _finite(*f):
            raise TesseraError("MPM force must be finite")
        if self._session is not None:
            self._session.set_particle_force(index, f)
        else:
            self._world.force[index] = f

    def set_particle_transfer_color(self, index: int, color: int):
        """Independent particle-grid transfer region (mpm.rs:1266-1283)."""
        self._reject_pending()
        if not (0 <= int(color) <= 0xFFFF):
            raise TesseraError("MPM transfer color out of range")
        a = self._arrays()
        if index < 0 or index >= a.count:
            raise TesseraError("MPM particle index out of range")
        a = a.copy()
        a.transfer_color[index] = int(color)
        if self._session is not None:
            self._session.write_particles(a)
        self._world = a
