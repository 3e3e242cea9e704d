"""The reference's `budget` RangeError (src/sfm/bundle/gpu/bundle.ts:235-242): a problem whose device
workspace does not fit is refused before any kernel runs, with a message the reference's tests match
(/budget/), as TBA_ERROR_BUDGET through the C ABI and a RangeError through the operator.  The device
memory is taken by another allocation in the same process, as an application sharing the GPU would."""
import numpy as np
import pytest

import typecv_b200 as tb
from typecv_b200 import _lib
from typecv_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def test_a_problem_beyond_the_free_device_memory_raises_the_budget_error():
    import torch
    scene = S.helix_scene(seed=9, cameras=60, points=150_000)
    s, i = scene.packed()
    ctl = tb.make_control(scene.C, scene.P, scene.M, anchor=0, scale_view=1, iterations=2, shared_focal=True)
    with tb.ShadeDevice.open(0) as dev:  # a fresh handle: no workspace yet
        free, _ = torch.cuda.mem_get_info(0)
        # Leave 8 MiB free: the problem's workspace (1.1M observations: pixels, index, camera-major
        # copies and point blocks, before its 100 MB of Jacobian factors) needs far more.
        hog = torch.empty(max(0, free - (8 << 20)), dtype=torch.uint8, device="cuda:0")
        try:
            with pytest.raises(tb.RangeError, match="budget"):
                tb.solve_packed(dev, ctl, s, i)
            lib = _lib.load()
            assert "budget" in lib.tba_last_error(dev.handle).decode()
        finally:
            del hog
            torch.cuda.empty_cache()
        # With the memory back the same handle solves the problem.
        out, rep = tb.solve_packed(dev, ctl, s, i)
        assert rep["lm_iterations"] >= 1 and np.isfinite(out[12 * scene.C + 3 * scene.P + 6])
