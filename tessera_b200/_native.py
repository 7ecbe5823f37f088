"""Loads ``libtmpm.so`` (built in-tree for sm_100a) and declares its C signatures.

The device path has no fallback: if the library is missing or no CUDA device is
present, the calls that need it raise.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

from ._abi import (
    TmpmBatchOptions, TmpmObstacle, TmpmParams, TmpmParticleArrays, TmpmRigidBody, TmpmRigidMapping,
    TmpmSessionOptions,
)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("TMPM_LIB_PATH") or os.path.join(_HERE, "libtmpm.so")
_lib = None


def build() -> str:
    """Compile libtmpm.so with nvcc (cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "csrc"), "-j4"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libtmpm.so is not built ({LIB_PATH}); run tessera_b200._native.build()")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    S = C.c_int32
    L.tmpm_version.restype = C.c_char_p
    L.tmpm_last_error.restype = C.c_char_p
    L.tmpm_last_error_message.restype = C.c_char_p
    L.tmpm_last_error_message.argtypes = [P]
    L.tmpm_session_create.restype = S
    L.tmpm_session_create.argtypes = [C.POINTER(TmpmParams), C.POINTER(TmpmParticleArrays), P, C.c_size_t,
                                      C.c_int32, C.c_double, C.POINTER(TmpmSessionOptions), C.POINTER(P)]
    L.tmpm_session_destroy.argtypes = [P]
    L.tmpm_session_destroy.restype = None
    for name in ("tmpm_submit_steps", "tmpm_step"):
        getattr(L, name).argtypes = [P, C.c_uint32]
        getattr(L, name).restype = S
    L.tmpm_synchronize.argtypes = [P]
    L.tmpm_synchronize.restype = S
    L.tmpm_pending_substeps.argtypes = [P]
    L.tmpm_pending_substeps.restype = C.c_uint64
    L.tmpm_has_pending_steps.argtypes = [P]
    L.tmpm_has_pending_steps.restype = C.c_int32
    L.tmpm_substeps.argtypes = [P]
    L.tmpm_substeps.restype = C.c_uint64
    L.tmpm_particle_count.argtypes = [P]
    L.tmpm_particle_count.restype = C.c_size_t
    L.tmpm_device_count.argtypes = [P]
    L.tmpm_device_count.restype = C.c_size_t
    L.tmpm_read_particles.argtypes = [P, C.POINTER(TmpmParticleArrays)]
    L.tmpm_read_particles.restype = S
    L.tmpm_stable_timestep.argtypes = [P]
    L.tmpm_stable_timestep.restype = C.c_double
    L.tmpm_set_particle_force.argtypes = [P, C.c_size_t, P]
    L.tmpm_set_particle_force.restype = S
    L.tmpm_set_obstacles.argtypes = [P, P, C.c_size_t]
    L.tmpm_set_obstacles.restype = S
    L.tmpm_add_particles.argtypes = [P, C.POINTER(TmpmParticleArrays), C.POINTER(C.c_uint64)]
    L.tmpm_add_particles.restype = S
    L.tmpm_remove_chunk.argtypes = [P, C.c_uint64, C.POINTER(C.c_size_t)]
    L.tmpm_remove_chunk.restype = S
    L.tmpm_write_particles.argtypes = [P, C.POINTER(TmpmParticleArrays)]
    L.tmpm_write_particles.restype = S
    L.tmpm_encode_particle_snapshot.argtypes = [P, P, C.c_size_t, C.POINTER(C.c_uint32)]
    L.tmpm_encode_particle_snapshot.restype = S
    L.tmpm_substep_dt.argtypes = [P]
    L.tmpm_substep_dt.restype = C.c_double
    L.tmpm_set_substep_dt.argtypes = [P, C.c_double]
    L.tmpm_set_substep_dt.restype = S
    L.tmpm_step_cfl.argtypes = [P, C.c_double]
    L.tmpm_step_cfl.restype = S
    L.tmpm_step_cfl_with_reactions.argtypes = [P, C.c_double, P, C.c_size_t]
    L.tmpm_step_cfl_with_reactions.restype = S
    L.tmpm_debug_binning.argtypes = [P, P, P, P]
    L.tmpm_debug_binning.restype = S
    L.tmpm_debug_p2g.argtypes = [P, P, P, C.c_size_t, C.POINTER(C.c_size_t)]
    L.tmpm_debug_p2g.restype = S
    L.tmpm_bench_substeps.argtypes = [P, C.c_uint32, C.POINTER(C.c_double), P, C.c_size_t]
    L.tmpm_bench_substeps.restype = S
    L.tmpm_sort_by_block_noalloc.argtypes = [P, C.c_size_t, C.c_size_t, C.c_double, P, P, P]
    L.tmpm_sort_by_block_noalloc.restype = S
    U32 = C.c_uint32
    L.tmpm_batch_create.argtypes = [C.POINTER(TmpmBatchOptions), C.POINTER(P)]
    L.tmpm_batch_create.restype = S
    L.tmpm_batch_destroy.argtypes = [P]
    L.tmpm_batch_destroy.restype = None
    L.tmpm_batch_add_scene.argtypes = [P, C.POINTER(TmpmParams), C.POINTER(TmpmParticleArrays), C.c_double,
                                       C.POINTER(U32)]
    L.tmpm_batch_add_scene.restype = S
    L.tmpm_batch_remove_scene.argtypes = [P, U32]
    L.tmpm_batch_remove_scene.restype = S
    L.tmpm_batch_submit.argtypes = [P, P, P, C.c_size_t]
    L.tmpm_batch_submit.restype = S
    L.tmpm_batch_synchronize.argtypes = [P]
    L.tmpm_batch_synchronize.restype = S
    L.tmpm_batch_pending.argtypes = [P]
    L.tmpm_batch_pending.restype = C.c_int32
    L.tmpm_batch_scene_status.argtypes = [P, U32]
    L.tmpm_batch_scene_status.restype = S
    L.tmpm_batch_scene_substeps.argtypes = [P, U32]
    L.tmpm_batch_scene_substeps.restype = C.c_uint64
    L.tmpm_batch_scene_particle_count.argtypes = [P, U32]
    L.tmpm_batch_scene_particle_count.restype = C.c_size_t
    L.tmpm_batch_read_scene.argtypes = [P, U32, C.POINTER(TmpmParticleArrays)]
    L.tmpm_batch_read_scene.restype = S
    L.tmpm_batch_take_scene.argtypes = [P, U32, C.POINTER(TmpmParticleArrays)]
    L.tmpm_batch_take_scene.restype = S
    L.tmpm_batch_last_ms.argtypes = [P]
    L.tmpm_batch_last_ms.restype = C.c_double
    L.tmpm_batch_device_bytes.argtypes = [P]
    L.tmpm_batch_device_bytes.restype = C.c_size_t
    L.tmpm_batch_scene_bytes.argtypes = [C.c_size_t, C.c_size_t]
    L.tmpm_batch_scene_bytes.restype = C.c_size_t
    L.tmpm_scene_prepare.argtypes = [C.POINTER(TmpmParams), C.POINTER(TmpmParticleArrays), C.c_double, C.POINTER(P)]
    L.tmpm_scene_prepare.restype = S
    L.tmpm_scene_prepared_destroy.argtypes = [P]
    L.tmpm_scene_prepared_destroy.restype = None
    L.tmpm_scene_prepared_particle_count.argtypes = [P]
    L.tmpm_scene_prepared_particle_count.restype = C.c_size_t
    L.tmpm_scene_prepared_bytes.argtypes = [P]
    L.tmpm_scene_prepared_bytes.restype = C.c_size_t
    L.tmpm_batch_admit.argtypes = [P, P, C.POINTER(U32)]
    L.tmpm_batch_admit.restype = S
    L.tmpm_adjoint_create.argtypes = [C.POINTER(TmpmParams), C.POINTER(TmpmParticleArrays), C.c_double, U32, U32,
                                      C.c_int32, C.POINTER(P)]
    L.tmpm_adjoint_create.restype = S
    L.tmpm_adjoint_destroy.argtypes = [P]
    L.tmpm_adjoint_destroy.restype = None
    L.tmpm_adjoint_particle_count.argtypes = [P]
    L.tmpm_adjoint_particle_count.restype = C.c_size_t
    L.tmpm_adjoint_forward.argtypes = [P, P, P, P, P]
    L.tmpm_adjoint_forward.restype = S
    L.tmpm_adjoint_backward.argtypes = [P, P, P, P, P]
    L.tmpm_adjoint_backward.restype = S
    L.tmpm_adjoint_last_error_message.argtypes = [P]
    L.tmpm_adjoint_last_error_message.restype = C.c_char_p
    L.tmpm_batch_last_error_message.argtypes = [P]
    L.tmpm_batch_last_error_message.restype = C.c_char_p
    L.tmpm_rigid_attach.argtypes = [P, C.POINTER(TmpmRigidBody), C.c_size_t, C.POINTER(TmpmRigidMapping), C.c_size_t]
    L.tmpm_rigid_attach.restype = S
    L.tmpm_rigid_step.argtypes = [P, C.c_uint32, C.POINTER(C.c_double), C.c_double, C.c_int32]
    L.tmpm_rigid_step.restype = S
    L.tmpm_rigid_read.argtypes = [P, C.POINTER(TmpmRigidBody), C.c_size_t]
    L.tmpm_rigid_read.restype = S
    L.tmpm_rigid_detach.argtypes = [P]
    L.tmpm_rigid_detach.restype = None
    L.tmpm_launch_shape_count.argtypes = []
    L.tmpm_launch_shape_count.restype = U32
    L.tmpm_launch_shape_info.argtypes = [U32, C.POINTER(U32), C.POINTER(U32), C.POINTER(U32)]
    L.tmpm_launch_shape_info.restype = S
    L.tmpm_session_launch_shape.argtypes = [P, P, C.c_size_t]
    L.tmpm_session_launch_shape.restype = C.c_int32
    L.tmpm_batch_launch_shape.argtypes = [P, P, C.c_size_t]
    L.tmpm_batch_launch_shape.restype = C.c_int32
    _lib = L
    return L


def version() -> str:
    return lib().tmpm_version().decode()


def launch_shapes() -> list[tuple[int, int, int]]:
    """(particles per CTA, CTAs per SM, grid block edge in cells) of each launch shape, by index."""
    L = lib()
    out = []
    for k in range(int(L.tmpm_launch_shape_count())):
        t, b, e = C.c_uint32(0), C.c_uint32(0), C.c_uint32(0)
        if L.tmpm_launch_shape_info(k, C.byref(t), C.byref(b), C.byref(e)) != 0:
            raise RuntimeError(f"launch shape {k}: {L.tmpm_last_error().decode()}")
        out.append((int(t.value), int(b.value), int(e.value)))
    return out


def query_launch_shape(fn, handle) -> dict:
    """The shape in use (None while tuning) and the measured ms per
    particle-substep of each shape (None where not measured)."""
    import numpy as np

    n = int(lib().tmpm_launch_shape_count())
    costs = np.full(n, np.inf)
    shape = int(fn(handle, costs.ctypes.data, n))
    return {"shape": None if shape < 0 else shape, "shapes": launch_shapes(),
            "ms_per_particle_substep": [None if not np.isfinite(c) else float(c) for c in costs]}
