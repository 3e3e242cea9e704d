"""The resident scene (tba_scene_*): an adjustment on device-resident arrays gives the result of
tba_bundle_adjust on the same arrays, leaves its solution in the scene for the next adjustment,
and uploads nothing of the problem per call."""
import numpy as np
import pytest

import typecv_b200 as tb
from typecv_b200 import synthetic as S
from typecv_b200.resident import ResidentScene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    dev = tb.ShadeDevice.open(0)
    yield dev
    dev.close()


def test_resident_adjustments_chain_like_separate_calls(device):
    sc = S.helix_scene(seed=41, cameras=30, points=3000)
    s, i = sc.packed()
    n = 12 * sc.C + 3 * sc.P
    ctl = tb.make_control(sc.C, sc.P, sc.M, anchor=0, scale_view=1, iterations=4, shared_focal=False)
    with ResidentScene(device, ctl, s, i) as rs:
        out1, st1, rep1 = rs.adjust(output=True)
        want1, _ = tb.solve_packed(device, ctl, s, i)
        assert abs(out1[n + 6] - want1[n + 6]) <= 1e-9 * want1[n + 6]
        assert np.allclose(st1, out1[n:n + 26])
        assert rep1["h2d_bytes"] < 0.05 * s.nbytes and rep1["check_ms"] == 0
        poses, points = rs.read()
        assert np.array_equal(poses, out1[:12 * sc.C]) and np.array_equal(points, out1[12 * sc.C:n])
        _, st2, _ = rs.adjust()
        s2 = s.copy()
        s2[:n] = out1[:n]
        want2, _ = tb.solve_packed(device, ctl, s2, i)
        assert abs(st2[6] - want2[n + 6]) <= 1e-9 * want2[n + 6]
        assert st2[6] <= st1[6]


def test_resident_write_read_and_shape_checks(device):
    sc = S.ring_scene(seed=3, cameras=8, points=400)
    s, i = sc.packed()
    ctl = tb.make_control(sc.C, sc.P, sc.M, anchor=0, scale_view=1, iterations=2, shared_focal=True)
    with ResidentScene(device, ctl, s, i) as rs:
        poses, points = rs.read()
        assert np.array_equal(poses, s[:12 * sc.C]) and np.array_equal(points, s[12 * sc.C:12 * sc.C + 3 * sc.P])
        moved = points + 0.001
        rs.write(points=moved)
        assert np.array_equal(rs.read()[1], moved)
        other = tb.make_control(sc.C, sc.P, sc.M, anchor=1, scale_view=2, iterations=2)
        with pytest.raises(tb.RangeError, match="differ"):
            rs.adjust(other)
        bad = points.copy()
        bad[0] = np.nan
        with pytest.raises(tb.RangeError, match="bounds"):
            rs.write(points=bad)
        out, st, _ = rs.adjust(output=True)
        assert st.size == 27 and out.size == 12 * sc.C + 3 * sc.P + 27
