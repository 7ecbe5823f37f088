"""The allocation-free binning entry point (tmpm_sort_by_block_noalloc).

It is for callers that cannot allocate device memory mid-call (frame-budgeted
loops, hosts that own every device buffer, graph-recording code).  The test
calls it through the C ABI on two scenes in a row, with caller-owned device
buffers, and checks it against the session path: the block keys must equal
tmpm_debug_binning's keys, and the order must equal the storage order the
session's re-sort produces (each full chunk of 256 sorted particles stored
transposed; the session is pinned to the 256-particle launch shape).  Both are
integer results, so the match is exact.  The variants cover no key output, a
position buffer whose component stride is larger than the count, and a
non-default stream.
This file sorts last so that a run stopping at the first failure has already
run every other test.
"""

import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tessera_b200 import _native, scenes
from tessera_b200._abi import TMPM_ERR_CAPACITY, TMPM_OK
from tessera_b200.session import Session

pytestmark = pytest.mark.gpu


def noalloc_sort(positions_f32: np.ndarray, cell_width: float, want_keys=True, pad=0, side_stream=False):
    import torch

    n = positions_f32.shape[0]
    stride = n + pad
    host = np.full((3, stride), np.nan, dtype=np.float32)  # the padding must never be read
    host[:, :n] = positions_f32.T
    pos = torch.from_numpy(host).cuda()  # component-major, `stride` floats apart
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    keys = torch.empty(n, dtype=torch.int32, device="cuda") if want_keys else None
    stream = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    stream.wait_stream(torch.cuda.current_stream())  # the positions' upload comes first
    st = _native.lib().tmpm_sort_by_block_noalloc(C.c_void_p(pos.data_ptr()), n, stride, cell_width,
                                                  C.c_void_p(order.data_ptr()),
                                                  C.c_void_p(keys.data_ptr()) if want_keys else None,
                                                  C.c_void_p(stream.cuda_stream))
    assert st == TMPM_OK, _native.lib().tmpm_last_error()
    stream.synchronize()
    return order.cpu().numpy().view(np.uint32), (keys.cpu().numpy().view(np.uint32) if want_keys else None)


def session_binning(scene):
    s = Session(scene.params, scene.particles, scene.dt, launch_shape=0)  # 256-particle CTAs
    widx0, _, keys0 = s.debug_binning()  # storage order = world order before any step
    s.submit_steps(1)  # each batch opens with the re-sort by block key
    s.synchronize()
    widx1, _, _ = s.debug_binning()
    s.close()
    assert np.array_equal(widx0, np.arange(len(widx0)))
    return widx1, keys0


@pytest.mark.parametrize("want_keys,pad,side_stream", [(True, 0, False), (False, 0, False), (True, 37, True)])
def test_noalloc_binning_matches_session_on_two_calls(want_keys, pad, side_stream):
    # two calls in a row on different scenes reuse the same scratch
    for scene in (scenes.dam_break(seed=7, scale=0.12), scenes.elastic_block(seed=3, lo=(0.4, 0.4, 0.4),
                                                                          hi=(0.55, 0.55, 0.55))):
        assert scene.particles.count <= 262144
        order, keys = noalloc_sort(scene.particles.position.astype(np.float32), scene.params.cell_width,
                                   want_keys=want_keys, pad=pad, side_stream=side_stream)
        ref_order, ref_keys = session_binning(scene)
        if want_keys:
            assert np.array_equal(keys, np.sort(ref_keys, kind="stable"))
        # the session stores each full 256-particle chunk of the sorted order transposed
        assert np.array_equal(O.storage_order(order), ref_order)


def test_noalloc_rejects_counts_beyond_the_scratch_limit():
    st = _native.lib().tmpm_sort_by_block_noalloc(None, 262145, 262145, 0.01, None, None, None)
    assert st == TMPM_ERR_CAPACITY
    assert b"262144" in _native.lib().tmpm_last_error()
