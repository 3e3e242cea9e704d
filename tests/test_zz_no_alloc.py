"""The allocation-free scene cost, through the C ABI, against the allocating operator.

`tba_scene_cost_noalloc` serves callers that cannot call cudaMalloc (their device memory belongs
to their own allocator, or they run on a thread where a synchronising allocation is not allowed):
it reads the packed scene from the caller's device buffers and keeps its scratch in a fixed array
inside the library.  This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

import typecv_b200 as tb
from typecv_b200 import _lib
from typecv_b200 import synthetic as S

pytestmark = pytest.mark.gpu

COST_REL = 1e-9  # the FP64 cost tolerance of the parity tests
RMS_PX = 1e-6


def _noalloc(lib, control, scene_ptr, index_ptr, result_ptr, scene_len=None, index_len=None, result_len=4):
    """One call through the C ABI; pointers are device addresses (ints), lengths default to the control's."""
    msg = ctypes.create_string_buffer(512)
    scene_len = lib.tba_scene_size(ctypes.byref(control)) if scene_len is None else scene_len
    index_len = lib.tba_index_size(ctypes.byref(control)) if index_len is None else index_len
    status = lib.tba_scene_cost_noalloc(ctypes.byref(control), scene_ptr, scene_len, index_ptr, index_len,
                                        result_ptr, result_len, None, msg, len(msg))
    return status, msg.value.decode()


def test_noalloc_cost_matches_the_allocating_entry_point_on_two_calls():
    import torch
    lib = _lib.load()
    # The larger scene first: the second, smaller call reuses the scratch rows of the first.
    scenes = [S.helix_scene(cameras=60, points=20_000), S.ring_scene(cameras=8, points=700)]
    with tb.ShadeDevice.open(0) as device:
        for scene in scenes:
            s, i = scene.packed()
            control = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=0,
                                      shared_focal=True, huber=2.0)
            out, _ = tb.solve_packed(device, control, s, i)
            base = 12 * scene.C + 3 * scene.P
            want_cost, want_rmse = out[base + 8], out[base + 24]
            scene_dev = torch.from_numpy(s).cuda()
            index_dev = torch.from_numpy(i.view(np.int32)).cuda()
            result_dev = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
            status, msg = _noalloc(lib, control, scene_dev.data_ptr(), index_dev.data_ptr(), result_dev.data_ptr())
            assert status == _lib.TBA_OK, msg
            torch.cuda.synchronize()
            cost, squares, failed, bad = result_dev.cpu().numpy()
            assert failed == 0 and bad == 0
            assert abs(cost - want_cost) <= COST_REL * want_cost, (cost, want_cost)
            assert abs(np.sqrt(squares / scene.M) - want_rmse) <= RMS_PX


def test_noalloc_refuses_scenes_beyond_its_scratch():
    import torch
    lib = _lib.load()
    big = tb.make_control(2, 1, 16_777_217, anchor=0, scale_view=1, huber=2.0)
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    status, msg = _noalloc(lib, big, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr())
    assert status == _lib.TBA_ERROR_ARGUMENT and "16777216" in msg


def test_noalloc_refuses_host_memory_and_short_buffers_before_any_launch():
    # Each refused call returns before launching anything, so the result buffer keeps its marker
    # and the context stays usable for the valid call at the end.
    import torch
    lib = _lib.load()
    scene = S.ring_scene(cameras=6, points=300)
    s, i = scene.packed()
    control = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, huber=2.0)
    scene_dev = torch.from_numpy(s).cuda()
    index_dev = torch.from_numpy(i.view(np.int32)).cuda()
    result_dev = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    host_result = np.full(4, -1.0)
    cases = [
        # host memory in place of each device buffer
        ((s.ctypes.data, index_dev.data_ptr(), result_dev.data_ptr()), {}, "scene is host memory"),
        ((scene_dev.data_ptr(), i.ctypes.data, result_dev.data_ptr()), {}, "index is host memory"),
        ((scene_dev.data_ptr(), index_dev.data_ptr(), host_result.ctypes.data), {}, "result is host memory"),
        # lengths that differ from the control's
        ((scene_dev.data_ptr(), index_dev.data_ptr(), result_dev.data_ptr()), {"scene_len": s.size - 1}, "lengths"),
        ((scene_dev.data_ptr(), index_dev.data_ptr(), result_dev.data_ptr()), {"index_len": i.size + 1}, "lengths"),
        ((scene_dev.data_ptr(), index_dev.data_ptr(), result_dev.data_ptr()), {"result_len": 3}, "lengths"),
    ]
    for ptrs, lens, text in cases:
        status, msg = _noalloc(lib, control, *ptrs, **lens)
        assert status == _lib.TBA_ERROR_ARGUMENT and text in msg, (text, msg)
    # A control claiming far more observations than the caller's device buffers hold: the lengths
    # agree with the control, the allocations do not.
    big = tb.make_control(scene.C, scene.P, 8_000_000, anchor=0, scale_view=1, huber=2.0)
    small = torch.zeros(1024, dtype=torch.float64, device="cuda")
    status, msg = _noalloc(lib, big, small.data_ptr(), small.data_ptr(), result_dev.data_ptr())
    assert status == _lib.TBA_ERROR_ARGUMENT and "allocation holds" in msg, msg
    torch.cuda.synchronize()
    assert np.all(result_dev.cpu().numpy() == -1.0) and np.all(host_result == -1.0)
    status, msg = _noalloc(lib, control, scene_dev.data_ptr(), index_dev.data_ptr(), result_dev.data_ptr())
    assert status == _lib.TBA_OK, msg
    torch.cuda.synchronize()
    assert result_dev.cpu().numpy()[0] > 0
