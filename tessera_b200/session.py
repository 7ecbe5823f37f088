"""Python handle on the C-ABI session (``GpuMpmResidentSession`` counterpart).

Method names follow the reference's ``GpuMpmResidentSession``
(crates/tessera-mpm/src/gpu.rs:206-662).  Every failing call raises
``TesseraError`` carrying the ``TmpmStatus`` code and the library's reason,
as tessera-python3d maps every error to ``TesseraError.Failed(reason)``
(crates/tessera-python3d/src/lib.rs:82-95).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from ._abi import (
    STATUS_MESSAGES, TMPM_OK, ParticleArrays, TmpmParams, TmpmSessionOptions, obstacles_to_c, partial_arrays,
)


class TesseraError(Exception):
    """Mirror of tessera3d.TesseraError.Failed: `reason` is the diagnostic."""

    def __init__(self, reason: str, status: int = 0):
        super().__init__(reason)
        self.reason = reason
        self.status = status


def _check(status: int, handle=None) -> None:
    if status == TMPM_OK:
        return
    L = _native.lib()
    msg = (L.tmpm_last_error_message(handle) if handle else L.tmpm_last_error()) or b""
    reason = msg.decode() or STATUS_MESSAGES.get(status, f"status {status}")
    raise TesseraError(reason, status)


class Session:
    """Resident device session holding one world's particles and grids."""

    def __init__(self, params: TmpmParams, particles: ParticleArrays, substep_dt: float, obstacles=(),
                 use_cpic: bool = True, device: int = 0, max_blocks: int = 0, resort_interval: int = 0,
                 next_chunk_id: int = 0, substeps: int = 0, launch_shape: int | None = None):
        L = _native.lib()
        self._params = params
        arrays = particles.as_c()
        obs, nobs = obstacles_to_c(list(obstacles))
        opts = TmpmSessionOptions()
        opts.device = device
        opts.max_blocks = max_blocks
        opts.resort_interval = resort_interval
        opts.next_chunk_id = next_chunk_id
        opts.substeps = substeps
        # None: tuned on the first submits; k: launch shape k (see _native.launch_shapes())
        opts.launch_shape = 0 if launch_shape is None else int(launch_shape) + 1
        handle = C.c_void_p()
        self._h = None
        st = L.tmpm_session_create(C.byref(params), C.byref(arrays), obs, nobs, int(bool(use_cpic)),
                                   float(substep_dt), C.byref(opts), C.byref(handle))
        _check(st)
        self._h = handle
        self._obstacle_count = nobs

    def close(self) -> None:
        if self._h:
            _native.lib().tmpm_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    # --------------------------------------------------------------- stepping
    def submit_steps(self, steps: int) -> None:
        _check(_native.lib().tmpm_submit_steps(self._h, int(steps)), self._h)

    def step(self, steps: int) -> None:
        _check(_native.lib().tmpm_step(self._h, int(steps)), self._h)

    def synchronize(self) -> None:
        _check(_native.lib().tmpm_synchronize(self._h), self._h)

    def step_cfl(self, dt: float) -> None:
        _check(_native.lib().tmpm_step_cfl(self._h, float(dt)), self._h)

    def step_cfl_with_reactions(self, dt: float) -> np.ndarray:
        out = np.zeros((max(self._obstacle_count, 1), 6))
        _check(_native.lib().tmpm_step_cfl_with_reactions(self._h, float(dt), out.ctypes.data,
                                                          self._obstacle_count), self._h)
        return out[: self._obstacle_count]

    # ------------------------------------------------------------------ state
    def pending_substeps(self) -> int:
        return int(_native.lib().tmpm_pending_substeps(self._h))

    def has_pending_steps(self) -> bool:
        return bool(_native.lib().tmpm_has_pending_steps(self._h))

    def substeps(self) -> int:
        return int(_native.lib().tmpm_substeps(self._h))

    def count(self) -> int:
        return int(_native.lib().tmpm_particle_count(self._h))

    def device_count(self) -> int:
        return int(_native.lib().tmpm_device_count(self._h))

    def substep_dt(self) -> float:
        return float(_native.lib().tmpm_substep_dt(self._h))

    def set_substep_dt(self, dt: float) -> None:
        _check(_native.lib().tmpm_set_substep_dt(self._h, float(dt)), self._h)

    def stable_timestep(self) -> float:
        return float(_native.lib().tmpm_stable_timestep(self._h))

    def particles(self, out: ParticleArrays | None = None) -> ParticleArrays:
        if out is None:
            out = ParticleArrays(self.count())
        arrays = out.as_c()
        _check(_native.lib().tmpm_read_particles(self._h, C.byref(arrays)), self._h)
        return out

    def read(self, fields=("position", "velocity")) -> dict:
        """Only the named fields of the world's particles, as numpy arrays."""
        c, arrays = partial_arrays(self.count(), fields)
        _check(_native.lib().tmpm_read_particles(self._h, C.byref(c)), self._h)
        return arrays

    def write_particles(self, particles: ParticleArrays) -> None:
        arrays = particles.as_c()
        _check(_native.lib().tmpm_write_particles(self._h, C.byref(arrays)), self._h)

    # ------------------------------------------------------------------ edits
    def set_particle_force(self, index: int, force) -> None:
        f = np.ascontiguousarray(force, dtype=np.float64)
        _check(_native.lib().tmpm_set_particle_force(self._h, int(index), f.ctypes.data), self._h)

    def set_obstacles(self, obstacles) -> None:
        obs, n = obstacles_to_c(list(obstacles))
        _check(_native.lib().tmpm_set_obstacles(self._h, obs, n), self._h)
        self._obstacle_count = n

    def add_particles(self, particles: ParticleArrays) -> int:
        chunk = C.c_uint64(0)
        arrays = particles.as_c()
        _check(_native.lib().tmpm_add_particles(self._h, C.byref(arrays), C.byref(chunk)), self._h)
        return int(chunk.value)

    def remove_chunk(self, chunk: int) -> int:
        removed = C.c_size_t(0)
        _check(_native.lib().tmpm_remove_chunk(self._h, int(chunk), C.byref(removed)), self._h)
        return int(removed.value)

    def encode_particle_snapshot(self, device_ptr: int, capacity_bytes: int) -> int:
        written = C.c_uint32(0)
        _check(_native.lib().tmpm_encode_particle_snapshot(self._h, C.c_void_p(device_ptr), int(capacity_bytes),
                                                           C.byref(written)), self._h)
        return int(written.value)

    # ------------------------------------------------------------ diagnostics
    def debug_binning(self):
        """(world index, f32 base cells, Morton keys) of the device particles, in storage order."""
        n = self.device_count()
        widx = np.zeros(n, dtype=np.uint32)
        cells = np.zeros((n, 3), dtype=np.int32)
        keys = np.zeros(n, dtype=np.uint32)
        _check(_native.lib().tmpm_debug_binning(self._h, widx.ctypes.data, cells.ctypes.data, keys.ctypes.data),
               self._h)
        return widx, cells, keys

    def debug_p2g(self, capacity: int | None = None):
        """Grid nodes with non-zero mass after P2G only: (cells (G,3) int32, mass+momentum (G,4) float32)."""
        count = C.c_size_t(0)
        if capacity is None:
            _check(_native.lib().tmpm_debug_p2g(self._h, None, None, 0, C.byref(count)), self._h)
            capacity = int(count.value)
        cells = np.zeros((max(capacity, 1), 3), dtype=np.int32)
        vals = np.zeros((max(capacity, 1), 4), dtype=np.float32)
        _check(_native.lib().tmpm_debug_p2g(self._h, cells.ctypes.data, vals.ctypes.data, capacity,
                                            C.byref(count)), self._h)
        n = min(int(count.value), capacity)
        return cells[:n], vals[:n]

    # ------------------------------------------------------- rigid coupling
    def rigid_attach(self, bodies, mappings) -> None:
        """Rigid bodies (TmpmRigidBody) and one mapping (TmpmRigidMapping) per
        obstacle, in obstacle order, for MPM-owned two-way coupling."""
        from ._abi import TmpmRigidBody, TmpmRigidMapping

        b = (TmpmRigidBody * max(len(bodies), 1))(*bodies)
        m = (TmpmRigidMapping * max(len(mappings), 1))(*mappings)
        self._rigid_count = len(bodies)
        _check(_native.lib().tmpm_rigid_attach(self._h, b, len(bodies), m, len(mappings)), self._h)

    def rigid_step(self, substeps: int, gravity=(0.0, 0.0, 0.0), max_linear_speed: float = 0.0,
                   integrate_pose: bool = True) -> None:
        """`substeps` coupled substeps (obstacles follow their bodies; impulses
        change the bodies' velocities and, with integrate_pose, gravity acts and
        the poses advance), then a synchronize."""
        g = (C.c_double * 3)(*[float(v) for v in gravity])
        _check(_native.lib().tmpm_rigid_step(self._h, int(substeps), g, float(max_linear_speed),
                                             1 if integrate_pose else 0), self._h)

    def rigid_bodies(self) -> list:
        from ._abi import TmpmRigidBody

        n = getattr(self, "_rigid_count", 0)
        out = (TmpmRigidBody * max(n, 1))()
        _check(_native.lib().tmpm_rigid_read(self._h, out, n), self._h)
        return [out[i] for i in range(n)]

    def launch_shape(self) -> dict:
        """Transfer launch shape in use (None while trials are outstanding) and
        the measured cost of each shape."""
        return _native.query_launch_shape(_native.lib().tmpm_session_launch_shape, self._h)

    def bench_substeps(self, steps: int, per_kernel: bool = False):
        """Device-timed substeps (CUDA events on the session stream): (ms total, per-kernel ms or None)."""
        ms = C.c_double(0.0)
        kms = np.zeros(5) if per_kernel else None
        _check(_native.lib().tmpm_bench_substeps(self._h, int(steps), C.byref(ms),
                                                 kms.ctypes.data if per_kernel else None, 5), self._h)
        return ms.value, kms
