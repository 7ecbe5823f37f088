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


def storage_order(perm: np.ndarray, chunk: int = 256, group: int = 8) -> np.ndarray:
    """Device storage order after a single-scene re-sort: each full chunk of 256
    sorted particles is stored transposed (position kk holds sorted element
    (kk % 32) * 8 + kk // 32 of its chunk); the last partial chunk is in order."""
    perm = np.asarray(perm)
    n = len(perm)
    src = np.arange(n)
    full = (n // chunk) * chunk
    kk = np.arange(full) % chunk
    src[:full] = (np.arange(full) // chunk) * chunk + (kk % 32) * group + kk // 32
    return perm[src]
