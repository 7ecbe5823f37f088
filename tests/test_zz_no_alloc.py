"""The allocation-free binning entry point (tmpm_sort_by_block_noalloc).

It is for callers that cannot allocate device memory mid-call (frame-budgeted
loops, hosts that own every device buffer, graph-recording code).  The test
calls it through the C ABI on two scenes in a row, with caller-owned device
buffers, and checks it against the session path: the block keys must equal
tmpm_debug_binning's keys, and the order must equal the storage order the
session's re-sort produces (each full chunk of 256 sorted particles stored
transposed).  Both are integer results, so the match is exact.
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


def noalloc_sort(positions_f32: np.ndarray, cell_width: float):
    import torch

    n = positions_f32.shape[0]
    pos = torch.from_numpy(np.ascontiguousarray(positions_f32.T)).cuda()  # component-major, stride n
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _native.lib().tmpm_sort_by_block_noalloc(C.c_void_p(pos.data_ptr()), n, n, cell_width,
                                                  C.c_void_p(order.data_ptr()), C.c_void_p(keys.data_ptr()),
                                                  C.c_void_p(stream))
    assert st == TMPM_OK, _native.lib().tmpm_last_error()
    torch.cuda.synchronize()
    return order.cpu().numpy().view(np.uint32), keys.cpu().numpy().view(np.uint32)


def session_binning(scene):
    s = Session(scene.params, scene.particles, scene.dt)
    widx0, _, keys0 = s.debug_binning()  # storage order = world order before any step
    s.submit_steps(1)  # each batch opens with the re-sort by block key
    s.synchronize()
    widx1, _, _ = s.debug_binning()
    s.close()
    assert np.array_equal(widx0, np.arange(len(widx0)))
    return widx1, keys0


@pytest.mark.parametrize("call", [0, 1])
def test_noalloc_binning_matches_session_on_two_calls(call):
    # two calls in a row on different scenes reuse the same scratch
    for scene in (scenes.dam_break(seed=7, scale=0.12), scenes.elastic_block(seed=3, lo=(0.4, 0.4, 0.4),
                                                                          hi=(0.55, 0.55, 0.55))):
        assert scene.particles.count <= 262144
        order, keys = noalloc_sort(scene.particles.position.astype(np.float32), scene.params.cell_width)
        ref_order, ref_keys = session_binning(scene)
        assert np.array_equal(keys, np.sort(ref_keys, kind="stable"))
        # the session stores each full 256-particle chunk of the sorted order transposed
        assert np.array_equal(O.storage_order(order), ref_order)


def test_noalloc_rejects_counts_beyond_the_scratch_limit():
    st = _native.lib().tmpm_sort_by_block_noalloc(None, 262145, 262145, 0.01, None, None, None)
    assert st == TMPM_ERR_CAPACITY
    assert b"262144" in _native.lib().tmpm_last_error()
