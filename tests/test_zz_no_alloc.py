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


def _noalloc(lib, control, scene_dev, index_dev, result_dev):
    msg = ctypes.create_string_buffer(512)
    status = lib.tba_scene_cost_noalloc(ctypes.byref(control), scene_dev.data_ptr(), index_dev.data_ptr(),
                                        result_dev.data_ptr(), None, msg, len(msg))
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
            status, msg = _noalloc(lib, control, scene_dev, index_dev, result_dev)
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
    status, msg = _noalloc(lib, big, dummy, dummy, dummy)
    assert status == _lib.TBA_ERROR_ARGUMENT and "16777216" in msg
