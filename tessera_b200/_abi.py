"""ctypes mirror of ``include/tmpm.h`` plus numpy-backed particle arrays.

The structures here are the plain-data half of the C ABI: parameters,
obstacles and a structure-of-arrays particle view.  They follow the reference
types ``MpmParams`` (crates/tessera-mpm/src/world.rs:27-49), ``MpmParticle``
(world.rs:67-102) and ``RigidObstacle`` (obstacle.rs:79-98).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

# ----------------------------------------------------------------- status codes
TMPM_OK = 0
TMPM_ERR_INVALID_INPUT = 1
TMPM_ERR_CAPACITY = 2
TMPM_ERR_PENDING_STEPS = 3
TMPM_ERR_READBACK = 4
TMPM_ERR_RESIDENT_UNAVAILABLE = 5
TMPM_ERR_MPM_INVALID_INPUT = 6
TMPM_ERR_EXCESSIVE_SUBSTEPS = 7
TMPM_ERR_NON_FINITE_STATE = 8
TMPM_ERR_UNKNOWN_CHUNK = 9
TMPM_ERR_PARTICLE_CAPACITY = 10
TMPM_ERR_DEVICE = 11

# Display strings of GpuMpmError / MpmError (gpu.rs:135-154, world.rs:164-181).
STATUS_MESSAGES = {
    TMPM_ERR_INVALID_INPUT: "invalid or unrepresentable GPU MPM input",
    TMPM_ERR_CAPACITY: "GPU MPM transfer exceeds the device capacity",
    TMPM_ERR_PENDING_STEPS: "GPU MPM steps are pending; synchronize before stepping or editing state",
    TMPM_ERR_READBACK: "GPU MPM readback failed",
    TMPM_ERR_RESIDENT_UNAVAILABLE: "GPU MPM resident substeps require a CPU fallback; world state is unchanged",
    TMPM_ERR_MPM_INVALID_INPUT: "invalid MPM input",
    TMPM_ERR_EXCESSIVE_SUBSTEPS: "MPM timestep is too small for the requested duration",
    TMPM_ERR_NON_FINITE_STATE: "MPM integration produced a non-finite state",
    TMPM_ERR_UNKNOWN_CHUNK: "MPM particle chunk was not found",
    TMPM_ERR_PARTICLE_CAPACITY: "MPM particle capacity exceeded",
    TMPM_ERR_DEVICE: "CUDA device failure",
}

# ------------------------------------------------------------------ enumerations
MAT_ELASTIC = 0
MAT_NEO_HOOKEAN = 1
MAT_SAND = 2
MAT_FLUID = 3
MAT_SNOW = 4
MAT_SAND_NEO_HOOKEAN = 5

SHAPE_SPHERE = 0
SHAPE_BOX = 1
SHAPE_CAPSULE = 2
SHAPE_CYLINDER = 3
SHAPE_CONE = 4
SHAPE_GROUND = 5
SHAPE_TRIANGLE_PRISM = 6
SHAPE_CONVEX = 7

BOUNDARY_SLIP = 0
BOUNDARY_STICK = 1
BOUNDARY_SEPARATE = 2
BOUNDARY_NON_REFLECTING = 3
BOUNDARY_FREE_SLIP = 4


class TmpmParams(C.Structure):
    _fields_ = [
        ("cell_width", C.c_double),
        ("gravity", C.c_double * 3),
        ("max_substep", C.c_double),
        ("has_bounds", C.c_int32),
        ("wall_mode", C.c_int32),
        ("bounds_min", C.c_double * 3),
        ("bounds_max", C.c_double * 3),
    ]


class TmpmParticleArrays(C.Structure):
    _fields_ = [
        ("count", C.c_size_t),
        ("position", C.c_void_p),
        ("velocity", C.c_void_p),
        ("deformation", C.c_void_p),
        ("affine", C.c_void_p),
        ("force", C.c_void_p),
        ("mass", C.c_void_p),
        ("rest_volume", C.c_void_p),
        ("radius", C.c_void_p),
        ("damping", C.c_void_p),
        ("plastic", C.c_void_p),
        ("material", C.c_void_p),
        ("material_params", C.c_void_p),
        ("enabled", C.c_void_p),
        ("fixed", C.c_void_p),
        ("transfer_color", C.c_void_p),
        ("group_id", C.c_void_p),
        ("chunk_id", C.c_void_p),
    ]


class TmpmObstacle(C.Structure):
    _fields_ = [
        ("shape", C.c_int32),
        ("boundary", C.c_int32),
        ("cpic_group", C.c_int32),
        ("plane_count", C.c_uint32),
        ("center", C.c_double * 3),
        ("orientation", C.c_double * 4),
        ("linear_velocity", C.c_double * 3),
        ("angular_velocity", C.c_double * 3),
        ("friction", C.c_double),
        ("dims", C.c_double * 3),
        ("vertices", C.c_double * 9),
        ("bound_radius", C.c_double),
        ("planes", C.c_void_p),
    ]


class TmpmSessionOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_blocks", C.c_uint32),
        ("resort_interval", C.c_uint32),
        ("launch_shape", C.c_uint32),
        ("next_chunk_id", C.c_uint64),
        ("substeps", C.c_uint64),
    ]


class TmpmRigidBody(C.Structure):
    """include/tmpm.h TmpmRigidBody: a rigid body of the two-way coupling."""
    _fields_ = [
        ("position", C.c_double * 3),
        ("inverse_mass", C.c_double),
        ("orientation", C.c_double * 4),  # x, y, z, w
        ("linear_velocity", C.c_double * 3),
        ("angular_velocity", C.c_double * 3),
        ("inverse_inertia", C.c_double * 3),  # body frame, principal
    ]

    @staticmethod
    def make(position, inverse_mass, orientation=(0.0, 0.0, 0.0, 1.0), linear_velocity=(0.0, 0.0, 0.0),
             angular_velocity=(0.0, 0.0, 0.0), inverse_inertia=(0.0, 0.0, 0.0)) -> "TmpmRigidBody":
        b = TmpmRigidBody()
        b.position[:] = [float(v) for v in position]
        b.inverse_mass = float(inverse_mass)
        b.orientation[:] = [float(v) for v in orientation]
        b.linear_velocity[:] = [float(v) for v in linear_velocity]
        b.angular_velocity[:] = [float(v) for v in angular_velocity]
        b.inverse_inertia[:] = [float(v) for v in inverse_inertia]
        return b

    def as_dict(self) -> dict:
        return {f: (float(getattr(self, f)) if f == "inverse_mass" else np.array(getattr(self, f)[:]))
                for f, _ in self._fields_}


class TmpmRigidMapping(C.Structure):
    """include/tmpm.h TmpmRigidMapping: obstacle -> body (-1: the obstacle keeps its pose)."""
    _fields_ = [
        ("body", C.c_int32),
        ("reserved", C.c_int32),
        ("local_center", C.c_double * 3),
        ("local_orientation", C.c_double * 4),
    ]

    @staticmethod
    def make(body, local_center=(0.0, 0.0, 0.0), local_orientation=(0.0, 0.0, 0.0, 1.0)) -> "TmpmRigidMapping":
        m = TmpmRigidMapping()
        m.body = int(body)
        m.local_center[:] = [float(v) for v in local_center]
        m.local_orientation[:] = [float(v) for v in local_orientation]
        return m


class TmpmBatchOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("max_blocks", C.c_uint32),
        ("use_graphs", C.c_uint32),
        ("launch_shape", C.c_uint32),
        ("particle_capacity", C.c_uint64),
    ]


def make_params(cell_width, gravity=(0.0, 0.0, -9.81), max_substep=1e-3,
                bounds=None, wall_mode=0) -> TmpmParams:
    p = TmpmParams()
    p.cell_width = float(cell_width)
    p.gravity[:] = [float(g) for g in gravity]
    p.max_substep = float(max_substep)
    p.wall_mode = int(wall_mode)
    if bounds is not None:
        p.has_bounds = 1
        p.bounds_min[:] = [float(v) for v in bounds[0]]
        p.bounds_max[:] = [float(v) for v in bounds[1]]
    return p


# Field name -> (dtype, per-particle width).  Matrices are column-major.
PARTICLE_FIELDS = {
    "position": (np.float64, 3),
    "velocity": (np.float64, 3),
    "deformation": (np.float64, 9),
    "affine": (np.float64, 9),
    "force": (np.float64, 3),
    "mass": (np.float64, 1),
    "rest_volume": (np.float64, 1),
    "radius": (np.float64, 1),
    "damping": (np.float64, 1),
    "plastic": (np.float64, 3),
    "material": (np.int32, 1),
    "material_params": (np.float64, 5),
    "enabled": (np.uint8, 1),
    "fixed": (np.uint8, 1),
    "transfer_color": (np.uint16, 1),
    "group_id": (np.uint32, 1),
    "chunk_id": (np.uint64, 1),
}

_IDENTITY_CM = np.eye(3).reshape(9)


class ParticleArrays:
    """Structure-of-arrays particle state in world order (all fields present)."""

    def __init__(self, count: int):
        self.count = int(count)
        for name, (dtype, width) in PARTICLE_FIELDS.items():
            shape = (self.count,) if width == 1 else (self.count, width)
            setattr(self, name, np.zeros(shape, dtype=dtype))
        self.deformation[:] = _IDENTITY_CM
        self.plastic[:, 0] = 1.0
        self.enabled[:] = 1

    @classmethod
    def from_fields(cls, **fields) -> "ParticleArrays":
        n = len(fields["position"])
        out = cls(n)
        for name, value in fields.items():
            arr = getattr(out, name)
            arr[...] = np.asarray(value, dtype=arr.dtype).reshape(arr.shape)
        if "plastic" not in fields:
            sand = np.isin(out.material, (MAT_SAND, MAT_SAND_NEO_HOOKEAN))
            out.plastic[:, 1] = np.where(sand, 1.0, 0.0)
        return out

    def copy(self) -> "ParticleArrays":
        out = ParticleArrays.__new__(ParticleArrays)
        out.count = self.count
        for name in PARTICLE_FIELDS:
            setattr(out, name, getattr(self, name).copy())
        return out

    def select(self, index) -> "ParticleArrays":
        out = ParticleArrays.__new__(ParticleArrays)
        for name in PARTICLE_FIELDS:
            setattr(out, name, np.ascontiguousarray(getattr(self, name)[index]))
        out.count = len(out.position)
        return out

    @staticmethod
    def concat(parts) -> "ParticleArrays":
        parts = list(parts)
        out = ParticleArrays.__new__(ParticleArrays)
        for name in PARTICLE_FIELDS:
            setattr(out, name, np.ascontiguousarray(np.concatenate([getattr(p, name) for p in parts])))
        out.count = len(out.position)
        return out

    def as_c(self) -> TmpmParticleArrays:
        c = TmpmParticleArrays()
        c.count = self.count
        for name in PARTICLE_FIELDS:
            arr = getattr(self, name)
            assert arr.flags["C_CONTIGUOUS"], name
            setattr(c, name, arr.ctypes.data if self.count else None)
        c._keep = self  # keep arrays alive with the view
        return c


def density_particles(positions, radius, density, material, params, velocity=None) -> ParticleArrays:
    """MpmParticle::new for many positions (world.rs:118-150): V0 = (2r)^3, m = rho V0."""
    positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    n = len(positions)
    v0 = (2.0 * float(radius)) ** 3
    fields = dict(
        position=positions,
        mass=np.full(n, density * v0),
        rest_volume=np.full(n, v0),
        radius=np.full(n, float(radius)),
        material=np.full(n, int(material), dtype=np.int32),
        material_params=np.tile(np.asarray(list(params) + [0.0] * (5 - len(params)), dtype=np.float64), (n, 1)),
    )
    if velocity is not None:
        fields["velocity"] = np.broadcast_to(np.asarray(velocity, dtype=np.float64), (n, 3))
    return ParticleArrays.from_fields(**fields)


@dataclass
class Obstacle:
    """Plain-data RigidObstacle (obstacle.rs:79-98) ready to pack into TmpmObstacle."""

    shape: int
    center: tuple = (0.0, 0.0, 0.0)
    orientation: tuple = (0.0, 0.0, 0.0, 1.0)  # x, y, z, w
    linear_velocity: tuple = (0.0, 0.0, 0.0)
    angular_velocity: tuple = (0.0, 0.0, 0.0)
    friction: float = 0.0
    boundary: int = BOUNDARY_SLIP
    cpic_group: int = -1
    dims: tuple = (0.0, 0.0, 0.0)
    vertices: tuple = (0.0,) * 9
    bound_radius: float = 0.0
    planes: np.ndarray | None = None

    @staticmethod
    def sphere(center, radius, **kw):
        return Obstacle(SHAPE_SPHERE, center=tuple(center), dims=(float(radius), 0.0, 0.0), **kw)

    @staticmethod
    def cuboid(center, half_extents, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        return Obstacle(SHAPE_BOX, center=tuple(center), orientation=tuple(orientation),
                        dims=tuple(float(v) for v in half_extents), **kw)

    @staticmethod
    def capsule(center, half_height, radius, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        return Obstacle(SHAPE_CAPSULE, center=tuple(center), orientation=tuple(orientation),
                        dims=(float(half_height), float(radius), 0.0), **kw)

    @staticmethod
    def cylinder(center, half_height, radius, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        return Obstacle(SHAPE_CYLINDER, center=tuple(center), orientation=tuple(orientation),
                        dims=(float(half_height), float(radius), 0.0), **kw)

    @staticmethod
    def cone(center, half_height, radius, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        return Obstacle(SHAPE_CONE, center=tuple(center), orientation=tuple(orientation),
                        dims=(float(half_height), float(radius), 0.0), **kw)

    @staticmethod
    def ground(center, half_extents_xy, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        return Obstacle(SHAPE_GROUND, center=tuple(center), orientation=tuple(orientation),
                        dims=(float(half_extents_xy[0]), float(half_extents_xy[1]), 0.0), **kw)

    @staticmethod
    def triangle_prism(center, vertices, half_thickness, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        verts = tuple(float(v) for vert in vertices for v in vert)
        return Obstacle(SHAPE_TRIANGLE_PRISM, center=tuple(center), orientation=tuple(orientation),
                        dims=(float(half_thickness), 0.0, 0.0), vertices=verts, **kw)

    @staticmethod
    def convex(center, vertices, face_normals, orientation=(0.0, 0.0, 0.0, 1.0), **kw):
        """RigidObstacle::convex (obstacle.rs:210-245): planes from hull vertices."""
        verts = np.asarray(vertices, dtype=np.float64).reshape(-1, 3)
        normals = np.asarray(face_normals, dtype=np.float64).reshape(-1, 3)
        planes = np.zeros((len(normals), 4))
        for i, n in enumerate(normals):
            offset = max((float(np.dot(n, v)) for v in verts), default=-np.inf)
            planes[i] = (n[0], n[1], n[2], offset)
        if len(verts) >= 4 and np.all(np.isfinite(verts)):
            bound = float(max(np.linalg.norm(v) for v in verts))
        else:
            bound = float("nan")
        return Obstacle(SHAPE_CONVEX, center=tuple(center), orientation=tuple(orientation),
                        bound_radius=bound, planes=planes, **kw)

    def to_c(self) -> TmpmObstacle:
        o = TmpmObstacle()
        o.shape = self.shape
        o.boundary = self.boundary
        o.cpic_group = self.cpic_group
        o.center[:] = [float(v) for v in self.center]
        o.orientation[:] = [float(v) for v in self.orientation]
        o.linear_velocity[:] = [float(v) for v in self.linear_velocity]
        o.angular_velocity[:] = [float(v) for v in self.angular_velocity]
        o.friction = float(self.friction)
        o.dims[:] = [float(v) for v in self.dims]
        o.vertices[:] = [float(v) for v in self.vertices]
        o.bound_radius = float(self.bound_radius)
        if self.planes is not None and len(self.planes):
            planes = np.ascontiguousarray(self.planes, dtype=np.float64)
            o.plane_count = len(planes)
            o.planes = planes.ctypes.data
            o._keep = planes
        return o


def obstacles_to_c(obstacles):
    arr_t = TmpmObstacle * max(1, len(obstacles))
    arr = arr_t()
    keep = []
    for i, ob in enumerate(obstacles):
        c = ob.to_c()
        keep.append(getattr(c, "_keep", None))
        arr[i] = c
    arr._keep = keep
    return arr, len(obstacles)


def partial_arrays(count: int, fields=("position", "velocity")):
    """A C view that receives only `fields` (other pointers NULL) and the numpy arrays behind it."""
    c = TmpmParticleArrays()
    c.count = count
    arrays = {}
    for name in fields:
        dtype, width = PARTICLE_FIELDS[name]
        a = np.zeros((count,) if width == 1 else (count, width), dtype=dtype)
        arrays[name] = a
        setattr(c, name, a.ctypes.data if count else None)
    c._keep = arrays
    return c, arrays
