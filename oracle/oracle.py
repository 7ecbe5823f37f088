"""TEST INFRASTRUCTURE ONLY: Python handle on the CPU oracle (``libmpm_oracle.so``).

The oracle is a C++ f64 restatement of tessera-mpm's CPU reference pipeline
(crates/tessera-mpm/src/world.rs, material.rs, obstacle.rs); see
``mpm_oracle.cpp`` for the line-by-line citations.  Only the tests, the smoke
check and the CPU-baseline leg of ``bench.py`` load it, always as the checker.

``binning_reference`` restates, with numpy float32 arithmetic, the device
binning: the f32 base cell of ``crates/tessera-mpm/src/gpu.rs:1145`` /
``gpu.wgsl:947`` (``floor(x * inv_h - 0.5)`` with no fused multiply-add), the 4^3
block it falls in, the Morton sort key and the stable sort order.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from tessera_b200._abi import (  # noqa: F401  (re-exported for tests)
    TMPM_OK, ParticleArrays, TmpmObstacle, TmpmParams, obstacles_to_c,
)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmpm_oracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (g++ only; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        L.orc_world_create.restype = P
        L.orc_world_create.argtypes = [C.POINTER(TmpmParams), P, C.POINTER(C.c_int32)]
        L.orc_world_destroy.argtypes = [P]
        L.orc_world_clone.restype = P
        L.orc_world_clone.argtypes = [P]
        L.orc_world_add_particles.argtypes = [P, P, C.POINTER(C.c_uint64)]
        L.orc_world_remove_chunk.argtypes = [P, C.c_uint64, C.POINTER(C.c_size_t)]
        L.orc_world_set_obstacles.argtypes = [P, P, C.c_size_t]
        L.orc_world_set_use_cpic.argtypes = [P, C.c_int32]
        L.orc_world_set_params.argtypes = [P, C.POINTER(TmpmParams)]
        L.orc_world_stable_timestep.restype = C.c_double
        L.orc_world_stable_timestep.argtypes = [P]
        L.orc_world_step.argtypes = [P, C.c_double]
        L.orc_world_step_reactions.argtypes = [P, C.c_double, P]
        L.orc_world_substep_fixed.argtypes = [P, C.c_double, P]
        L.orc_world_count.restype = C.c_size_t
        L.orc_world_count.argtypes = [P]
        L.orc_world_substeps.restype = C.c_uint64
        L.orc_world_substeps.argtypes = [P]
        L.orc_world_read.argtypes = [P, P]
        L.orc_world_write.argtypes = [P, P]
        L.orc_world_set_force.argtypes = [P, C.c_size_t, P]
        L.orc_world_p2g.restype = C.c_size_t
        L.orc_world_p2g.argtypes = [P, C.c_double, P, P, C.c_size_t]
        L.orc_kirchhoff_stress.argtypes = [C.c_int32, P, P, P, P, P]
        L.orc_project_deformation.argtypes = [C.c_int32, P, P, P, P, P]
        L.orc_timestep_bound.restype = C.c_double
        L.orc_timestep_bound.argtypes = [C.c_int32, P, C.c_double, P, C.c_double, C.c_double]
        L.orc_material_valid.argtypes = [C.c_int32, P]
        L.orc_obstacle_valid.argtypes = [P]
        L.orc_obstacle_surface.argtypes = [P, P, C.POINTER(C.c_double), P]
        L.orc_obstacle_contact_velocity.argtypes = [P, P, P, P, P]
        L.orc_obstacle_may_contact.argtypes = [P, P, C.c_double]
        L.orc_bench_threads.restype = C.c_double
        L.orc_bench_threads.argtypes = [P, C.c_int32, C.c_int32, C.c_double]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data


class OracleError(RuntimeError):
    def __init__(self, status: int):
        super().__init__(f"oracle status {status}")
        self.status = status


class OracleWorld:
    """MpmWorld (world.rs:206-468) restated on the CPU in f64."""

    def __init__(self, params: TmpmParams, particles: ParticleArrays | None = None):
        st = C.c_int32(0)
        arrays = particles.as_c() if particles is not None and particles.count else None
        self._h = lib().orc_world_create(C.byref(params), C.byref(arrays) if arrays else None, C.byref(st))
        if not self._h:
            raise OracleError(st.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_world_destroy(h)
            self._h = None

    def clone(self) -> "OracleWorld":
        out = OracleWorld.__new__(OracleWorld)
        out._h = lib().orc_world_clone(self._h)
        return out

    def _check(self, status):
        if status != TMPM_OK:
            raise OracleError(status)

    def add_particles(self, particles: ParticleArrays) -> int:
        chunk = C.c_uint64(0)
        arrays = particles.as_c()
        self._check(lib().orc_world_add_particles(self._h, C.byref(arrays), C.byref(chunk)))
        return chunk.value

    def remove_chunk(self, chunk: int) -> int:
        removed = C.c_size_t(0)
        self._check(lib().orc_world_remove_chunk(self._h, chunk, C.byref(removed)))
        return removed.value

    def set_obstacles(self, obstacles) -> None:
        arr, n = obstacles_to_c(obstacles)
        self._check(lib().orc_world_set_obstacles(self._h, arr, n))

    def set_use_cpic(self, enabled: bool) -> None:
        lib().orc_world_set_use_cpic(self._h, int(bool(enabled)))

    def set_params(self, params: TmpmParams) -> None:
        self._check(lib().orc_world_set_params(self._h, C.byref(params)))

    def stable_timestep(self) -> float:
        return lib().orc_world_stable_timestep(self._h)

    def step(self, dt: float) -> None:
        self._check(lib().orc_world_step(self._h, dt))

    def step_with_obstacle_reactions(self, dt: float, count: int) -> np.ndarray:
        out = np.zeros((max(count, 1), 6))
        self._check(lib().orc_world_step_reactions(self._h, dt, _ptr(out)))
        return out[:count]

    def substep_fixed(self, dt: float, reactions_count: int | None = None):
        if reactions_count is None:
            self._check(lib().orc_world_substep_fixed(self._h, dt, None))
            return None
        out = np.zeros((max(reactions_count, 1), 6))
        self._check(lib().orc_world_substep_fixed(self._h, dt, _ptr(out)))
        return out[:reactions_count]

    def count(self) -> int:
        return lib().orc_world_count(self._h)

    def substeps(self) -> int:
        return lib().orc_world_substeps(self._h)

    def particles(self) -> ParticleArrays:
        out = ParticleArrays(self.count())
        arrays = out.as_c()
        self._check(lib().orc_world_read(self._h, C.byref(arrays)))
        return out

    def write_particles(self, particles: ParticleArrays) -> None:
        arrays = particles.as_c()
        self._check(lib().orc_world_write(self._h, C.byref(arrays)))

    def set_particle_force(self, index: int, force) -> None:
        f = np.asarray(force, dtype=np.float64)
        self._check(lib().orc_world_set_force(self._h, index, _ptr(f)))

    def p2g(self, dt: float):
        """Grid after P2G only: (keys (G,4) int64 = i,j,k,transfer key; values (G,4) = m, p)."""
        n = lib().orc_world_p2g(self._h, dt, None, None, 0)
        keys = np.zeros((max(n, 1), 4), dtype=np.int64)
        vals = np.zeros((max(n, 1), 4), dtype=np.float64)
        lib().orc_world_p2g(self._h, dt, _ptr(keys), _ptr(vals), n)
        return keys[:n], vals[:n]

    def bench(self, threads: int, substeps: int, dt: float) -> float:
        """Wall seconds for `threads` concurrent copies each taking `substeps` substeps."""
        return lib().orc_bench_threads(self._h, threads, substeps, dt)


def _mat_params(params):
    p = np.zeros(5)
    p[: len(params)] = params
    return p


def kirchhoff_stress(material, params, F, C_=None, plastic=(1.0, 0.0, 0.0)):
    F = np.asarray(F, dtype=np.float64).reshape(3, 3)
    Cm = np.zeros((3, 3)) if C_ is None else np.asarray(C_, dtype=np.float64).reshape(3, 3)
    out = np.zeros(9)
    fcm = np.ascontiguousarray(F.T.reshape(9))
    ccm = np.ascontiguousarray(Cm.T.reshape(9))
    pl = np.asarray(plastic, dtype=np.float64)
    mp = _mat_params(params)
    lib().orc_kirchhoff_stress(material, _ptr(mp), _ptr(fcm), _ptr(ccm), _ptr(pl), _ptr(out))
    return out.reshape(3, 3).T


def project_deformation(material, params, F, plastic=(1.0, 0.0, 0.0)):
    F = np.asarray(F, dtype=np.float64).reshape(3, 3)
    fcm = np.ascontiguousarray(F.T.reshape(9))
    pl = np.asarray(plastic, dtype=np.float64)
    fo = np.zeros(9)
    po = np.zeros(3)
    mp = _mat_params(params)
    lib().orc_project_deformation(material, _ptr(mp), _ptr(fcm), _ptr(pl), _ptr(fo), _ptr(po))
    return fo.reshape(3, 3).T, po


def timestep_bound(material, params, density, velocity, cell_width, det=1.0):
    v = np.asarray(velocity, dtype=np.float64)
    mp = _mat_params(params)
    return lib().orc_timestep_bound(material, _ptr(mp), density, _ptr(v), cell_width, det)


def material_valid(material, params) -> bool:
    mp = _mat_params(params)
    return bool(lib().orc_material_valid(material, _ptr(mp)))


def obstacle_valid(obstacle) -> bool:
    c = obstacle.to_c()
    return bool(lib().orc_obstacle_valid(C.byref(c)))


def obstacle_surface(obstacle, point):
    c = obstacle.to_c()
    p = np.asarray(point, dtype=np.float64)
    d = C.c_double(0.0)
    n = np.zeros(3)
    lib().orc_obstacle_surface(C.byref(c), _ptr(p), C.byref(d), _ptr(n))
    return d.value, n


def contact_velocity(obstacle, point, velocity, normal):
    c = obstacle.to_c()
    p = np.asarray(point, dtype=np.float64)
    v = np.asarray(velocity, dtype=np.float64)
    n = np.asarray(normal, dtype=np.float64)
    out = np.zeros(3)
    lib().orc_obstacle_contact_velocity(C.byref(c), _ptr(p), _ptr(v), _ptr(n), _ptr(out))
    return out


def may_contact(obstacle, point, margin) -> bool:
    c = obstacle.to_c()
    p = np.asarray(point, dtype=np.float64)
    return bool(lib().orc_obstacle_may_contact(C.byref(c), _ptr(p), margin))


# ----------------------------------------------------------------- f32 binning

BLOCK_SHIFT = 2  # 4^3 cells per block


def base_cells_f32(position_f32: np.ndarray, cell_width: float) -> np.ndarray:
    """floor(x * inv_h - 0.5) in IEEE f32, inv_h = 1/(f32)h (gpu.rs:1118-1152)."""
    x = np.asarray(position_f32, dtype=np.float32)
    inv_h = np.float32(1.0) / np.float32(cell_width)
    return np.floor((x * inv_h) - np.float32(0.5)).astype(np.int32)


def _spread10(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint32) & np.uint32(0x3FF)
    v = (v | (v << np.uint32(16))) & np.uint32(0x030000FF)
    v = (v | (v << np.uint32(8))) & np.uint32(0x0300F00F)
    v = (v | (v << np.uint32(4))) & np.uint32(0x030C30C3)
    v = (v | (v << np.uint32(2))) & np.uint32(0x09249249)
    return v


def block_morton_keys(base_cells: np.ndarray, scene: int = 0) -> np.ndarray:
    """Sort key of the 4^3 block holding each base cell: scene << 21 | 21-bit Morton
    code of the block coordinates taken modulo 128."""
    b = np.right_shift(np.asarray(base_cells, dtype=np.int32), BLOCK_SHIFT)
    bu = b.astype(np.uint32) & np.uint32(0x7F)
    m = (_spread10(bu[:, 0]) << np.uint32(2)) | (_spread10(bu[:, 1]) << np.uint32(1)) | _spread10(bu[:, 2])
    return (np.uint32(scene & 0xFF) << np.uint32(21)) | m


def cell_sort_keys(base_cells: np.ndarray) -> np.ndarray:
    """Single-scene sort key: the block's 21-bit Morton code << 6 | the 6-bit Morton
    code of the cell inside its 4^3 block."""
    c = np.asarray(base_cells, dtype=np.int32).astype(np.uint32) & np.uint32(3)
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    cell = (((x & 2) << 4) | ((y & 2) << 3) | ((z & 2) << 2) | ((x & 1) << 2) | ((y & 1) << 1) | (z & 1))
    return (block_morton_keys(base_cells) << np.uint32(6)) | cell.astype(np.uint32)


def binning_reference(position_f32: np.ndarray, cell_width: float):
    """(base cells, sort keys, stable sort permutation) for device-order positions."""
    cells = base_cells_f32(position_f32, cell_width)
    keys = cell_sort_keys(cells)
    perm = np.argsort(keys, kind="stable").astype(np.uint32)
    return cells, keys, perm


def lane_cell(lane):
    """Cell group of a transfer warp's lane (the device's lane_cell): quarter-warp
    p = lane // 8 takes a 1 x 2 x 4 slab of the chunk's 2 x 4 x 4 Morton group."""
    lane = np.asarray(lane)
    p, q = lane >> 3, lane & 7
    return (p & 1) * 16 + ((q >> 1) & 1) * 8 + (p >> 1) * 4 + (q >> 2) * 2 + (q & 1)


def storage_order(perm: np.ndarray, chunk: int = 256, group: int = 8) -> np.ndarray:
    """Device storage order after a single-scene re-sort: each full chunk of 256
    sorted particles is stored transposed (position kk holds sorted element
    lane_cell(kk % 32) * 8 + kk // 32 of its chunk); the last partial chunk is in
    order."""
    perm = np.asarray(perm)
    n = len(perm)
    src = np.arange(n)
    full = (n // chunk) * chunk
    kk = np.arange(full) % chunk
    src[:full] = (np.arange(full) // chunk) * chunk + lane_cell(kk % 32) * group + kk // 32
    return perm[src]


# -------------------------------------------------------- rigid coupling (f64)
# Restatement of the MPM-owned two-way rigid coupling: obstacle pose from its
# body (crates/tessera-mpm/src/gpu_rigid_sync.wgsl:46-61) and obstacle impulses
# applied to the bodies (gpu_rigid_reaction.wgsl:71-150), in f64.  Bodies are
# dicts with numpy arrays: position, inverse_mass, orientation (x, y, z, w),
# linear_velocity, angular_velocity, inverse_inertia (body frame).  Mappings
# are (body, local_center, local_orientation) with body -1 for a fixed obstacle.

def quat_rotate(q, v):
    """v rotated by the unit quaternion q (gpu_rigid_sync.wgsl:32-35)."""
    q = np.asarray(q, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    t = 2.0 * np.cross(q[:3], v)
    return v + q[3] * t + np.cross(q[:3], t)


def quat_mul(a, b):
    """Hamilton product (gpu_rigid_sync.wgsl:37-42)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    v = a[3] * b[:3] + b[3] * a[:3] + np.cross(a[:3], b[:3])
    return np.array([v[0], v[1], v[2], a[3] * b[3] - np.dot(a[:3], b[:3])])


def quat_from_rotation(r):
    """Rotation by vector r; first order below 1e-5 rad (gpu_rigid_reaction.wgsl:62-69)."""
    r = np.asarray(r, dtype=np.float64)
    angle = float(np.linalg.norm(r))
    if angle < 1e-5:
        q = np.array([0.5 * r[0], 0.5 * r[1], 0.5 * r[2], 1.0])
        return q / np.linalg.norm(q)
    s = np.sin(0.5 * angle) / angle
    return np.array([r[0] * s, r[1] * s, r[2] * s, np.cos(0.5 * angle)])


def rigid_sync(bodies, mappings, obstacles):
    """Obstacles with the pose and velocity of their bodies (gpu_rigid_sync.wgsl:46-61)."""
    import dataclasses

    out = []
    for (body, local_center, local_q), o in zip(mappings, obstacles):
        if body < 0:
            out.append(o)
            continue
        b = bodies[body]
        offset = quat_rotate(b["orientation"], local_center)
        center = b["position"] + offset
        out.append(dataclasses.replace(
            o, center=tuple(center), orientation=tuple(quat_mul(b["orientation"], local_q)),
            linear_velocity=tuple(b["linear_velocity"] + np.cross(b["angular_velocity"], offset)),
            angular_velocity=tuple(b["angular_velocity"])))
    return out


def rigid_apply(bodies, mappings, obstacles, reactions, dt, gravity=(0.0, 0.0, 0.0), max_speed=0.0,
                integrate_pose=True):
    """Bodies after the obstacle impulses of one substep (gpu_rigid_reaction.wgsl:71-150):
    reactions[i] = (linear impulse, angular impulse about obstacle i's centre)."""
    out = []
    for bi, b in enumerate(bodies):
        b = {k: (np.array(v, dtype=np.float64) if not np.isscalar(v) else v) for k, v in b.items()}
        if b["inverse_mass"] <= 0.0:
            out.append(b)
            continue
        lin = np.zeros(3)
        ang = np.zeros(3)
        mapped = False
        for oi, (body, _, _) in enumerate(mappings):
            if body != bi:
                continue
            mapped = True
            imp = np.asarray(reactions[oi][:3], dtype=np.float64)
            lin += imp
            ang += np.asarray(reactions[oi][3:6], dtype=np.float64) + np.cross(
                np.asarray(obstacles[oi].center) - b["position"], imp)
        finite = np.all(np.abs(lin) < 1e30) and np.all(np.abs(ang) < 1e30)
        if not finite or not mapped or (not lin.any() and not ang.any() and not integrate_pose):
            out.append(b)
            continue
        q = b["orientation"]
        conj = np.array([-q[0], -q[1], -q[2], q[3]])
        dw = quat_rotate(q, quat_rotate(conj, ang) * b["inverse_inertia"])
        v = b["linear_velocity"] + lin * b["inverse_mass"]
        w = b["angular_velocity"] + dw
        if integrate_pose:
            v = v + np.asarray(gravity, dtype=np.float64) * dt
        if max_speed > 0.0:
            speed = float(np.linalg.norm(v))
            if speed > max_speed:
                v = v * (max_speed / speed)
        b["linear_velocity"] = v
        b["angular_velocity"] = w
        if integrate_pose:
            b["position"] = b["position"] + v * dt
            nq = quat_mul(quat_from_rotation(w * dt), q)
            b["orientation"] = nq / np.linalg.norm(nq)
        out.append(b)
    return out
