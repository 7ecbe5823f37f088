"""Python handle on a multi-scene batch (``tmpm_batch_*`` in include/tmpm.h).

A batch keeps many independent scenes resident on one device and advances them
together, one launch per kernel per substep for all scenes.  Each scene keeps
the reference's single-world semantics (``GpuMpmResidentSession`` over that
scene alone, crates/tessera-mpm/src/gpu.rs:206-662) within f32 round-off;
failures are per scene.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native
from ._abi import STATUS_MESSAGES, TMPM_OK, ParticleArrays, TmpmBatchOptions, TmpmParams, partial_arrays
from .session import TesseraError

MAX_SCENES = 256


def _check(status: int, handle=None) -> None:
    if status == TMPM_OK:
        return
    L = _native.lib()
    msg = (L.tmpm_batch_last_error_message(handle) if handle else L.tmpm_last_error()) or b""
    raise TesseraError(msg.decode() or STATUS_MESSAGES.get(status, f"status {status}"), status)


def scene_bytes(particles: int, home_blocks: int) -> int:
    """Device bytes one scene adds to a batch (admission control)."""
    return int(_native.lib().tmpm_batch_scene_bytes(int(particles), int(home_blocks)))


def home_blocks(position: np.ndarray, cell_width: float) -> int:
    """Occupied 4^3 blocks of a scene (the block-pool sizing input), from f32 base cells."""
    x = np.asarray(position, dtype=np.float32)
    inv_h = np.float32(1.0) / np.float32(cell_width)
    base = (np.floor(x * inv_h - np.float32(0.5)).astype(np.int64) >> 2) + (1 << 20)
    keys = (base[:, 0] << 42) | (base[:, 1] << 21) | base[:, 2]
    return int(len(np.unique(keys)))


class PreparedScene:
    """A scene validated and packed for admission (no device state).  Preparing
    releases the GIL inside the library, so it overlaps device work when run on
    a worker thread."""

    def __init__(self, params: TmpmParams, particles: ParticleArrays, substep_dt: float):
        handle = C.c_void_p()
        self._h = None
        arrays = particles.as_c()
        _check(_native.lib().tmpm_scene_prepare(C.byref(params), C.byref(arrays), float(substep_dt), C.byref(handle)))
        self._h = handle
        self.count = particles.count

    def device_bytes(self) -> int:
        return int(_native.lib().tmpm_scene_prepared_bytes(self._h))

    def _take(self):
        h, self._h = self._h, None
        return h

    def close(self) -> None:
        if self._h:
            _native.lib().tmpm_scene_prepared_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


class Batch:
    """Resident multi-scene batch on one device."""

    def __init__(self, device: int = 0, max_blocks: int = 0, use_graphs: bool = True, particle_capacity: int = 0,
                 launch_shape: int | None = None):
        L = _native.lib()
        opts = TmpmBatchOptions()
        opts.device = device
        opts.max_blocks = max_blocks
        opts.use_graphs = 1 if use_graphs else 0
        opts.particle_capacity = particle_capacity
        # None: tuned on the first batches; k: launch shape k (see _native.launch_shapes())
        opts.launch_shape = 0 if launch_shape is None else int(launch_shape) + 1
        handle = C.c_void_p()
        self._h = None
        _check(L.tmpm_batch_create(C.byref(opts), C.byref(handle)))
        self._h = handle
        self._counts: dict[int, int] = {}

    def close(self) -> None:
        if self._h:
            _native.lib().tmpm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def add_scene(self, params: TmpmParams, particles: ParticleArrays, substep_dt: float) -> int:
        sid = C.c_uint32(0)
        arrays = particles.as_c()
        _check(_native.lib().tmpm_batch_add_scene(self._h, C.byref(params), C.byref(arrays), float(substep_dt),
                                                   C.byref(sid)), self._h)
        self._counts[int(sid.value)] = particles.count
        return int(sid.value)

    def admit(self, prepared: PreparedScene) -> int:
        """Attach a prepared scene (allowed while a batch is in flight)."""
        sid = C.c_uint32(0)
        count = prepared.count
        h = prepared._take()
        if h is None:
            raise ValueError("prepared scene was already admitted")
        _check(_native.lib().tmpm_batch_admit(self._h, h, C.byref(sid)), self._h)
        self._counts[int(sid.value)] = count
        return int(sid.value)

    def remove_scene(self, scene: int) -> None:
        _check(_native.lib().tmpm_batch_remove_scene(self._h, int(scene)), self._h)
        self._counts.pop(int(scene), None)

    def submit(self, steps: dict[int, int]) -> None:
        """Queue one batch: scene -> substeps.  Scenes not in it stay readable while it runs."""
        ids = np.ascontiguousarray(list(steps.keys()), dtype=np.uint32)
        n = np.ascontiguousarray(list(steps.values()), dtype=np.uint32)
        _check(_native.lib().tmpm_batch_submit(self._h, ids.ctypes.data, n.ctypes.data, len(ids)), self._h)

    def synchronize(self) -> None:
        _check(_native.lib().tmpm_batch_synchronize(self._h), self._h)

    def run(self, steps: dict[int, int]) -> None:
        self.submit(steps)
        self.synchronize()

    def pending(self) -> bool:
        return bool(_native.lib().tmpm_batch_pending(self._h))

    def status(self, scene: int) -> int:
        return int(_native.lib().tmpm_batch_scene_status(self._h, int(scene)))

    def substeps(self, scene: int) -> int:
        return int(_native.lib().tmpm_batch_scene_substeps(self._h, int(scene)))

    def count(self, scene: int) -> int:
        return int(_native.lib().tmpm_batch_scene_particle_count(self._h, int(scene)))

    def particles(self, scene: int, out: ParticleArrays | None = None) -> ParticleArrays:
        if out is None:
            out = ParticleArrays(self.count(scene))
        arrays = out.as_c()
        _check(_native.lib().tmpm_batch_read_scene(self._h, int(scene), C.byref(arrays)), self._h)
        return out

    def read(self, scene: int, fields=("position", "velocity")) -> dict:
        """Only the named fields of a scene's particles (world order), as numpy arrays."""
        c, arrays = partial_arrays(self.count(scene), fields)
        _check(_native.lib().tmpm_batch_read_scene(self._h, int(scene), C.byref(c)), self._h)
        return arrays

    def take(self, scene: int, fields=("position", "velocity")) -> dict:
        """Read + remove: the named fields of a finished scene (world order), and
        the scene leaves the batch.  Only those fields are copied from the device."""
        c, arrays = partial_arrays(self.count(scene), fields)
        _check(_native.lib().tmpm_batch_take_scene(self._h, int(scene), C.byref(c)), self._h)
        self._counts.pop(int(scene), None)
        return arrays

    def last_ms(self) -> float:
        return float(_native.lib().tmpm_batch_last_ms(self._h))

    def launch_shape(self) -> dict:
        """Transfer launch shape in use (None while trials are outstanding) and
        the measured cost of each shape."""
        return _native.query_launch_shape(_native.lib().tmpm_batch_launch_shape, self._h)

    def device_bytes(self) -> int:
        return int(_native.lib().tmpm_batch_device_bytes(self._h))

    def scenes(self) -> list[int]:
        return sorted(self._counts)
