"""The resident scene (tba_scene_*): an adjustment on device-resident arrays gives the result of
tba_bundle_adjust on the same arrays and of the reference operator's algorithm restated on the CPU
(the oracle, as packBundleScene feeds it: src/sfm/bundle/gpu/bundle-host.ts:177-218), leaves its
solution in the scene for the next adjustment, and uploads nothing of the problem per call."""
import numpy as np
import pytest

import typecv_b200 as tb
from oracle import bundle_adjust as ob
from typecv_b200 import synthetic as S
from typecv_b200.resident import ResidentScene

COST_REL = 1e-9  # final robust cost, FP64 form
POSE_TOL = 1e-7

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


@pytest.mark.parametrize("shared", [False, True])
def test_resident_chain_matches_the_operator_oracle(device, shared):
    # Two chained adjustments of one resident scene against the oracle run twice, the second time
    # on the oracle's own first solution: same accepted steps, costs within 1e-9, poses within 1e-7.
    # A resident scene carries poses and points from one adjustment to the next; its camera records
    # (and so the focal scale's starting point) stay as created, as they do here for the oracle.
    sc = S.helix_scene(seed=43, cameras=24, points=2500)
    s, i = sc.packed()
    C, P = sc.C, sc.P
    n = 12 * C + 3 * P
    ctl = tb.make_control(C, P, sc.M, anchor=0, scale_view=1, iterations=5, shared_focal=shared)
    kw = dict(iterations=5, huber=2.0, max_cg=ctl.max_cg, shared=shared)
    ref1 = ob.gpu_operator_packed({"C": C, "P": P, "M": sc.M, "scene": s, "index": i}, 0, 1, **kw)
    s_ref = s.copy()
    s_ref[:n] = ref1[:n]
    ref2 = ob.gpu_operator_packed({"C": C, "P": P, "M": sc.M, "scene": s_ref, "index": i}, 0, 1, **kw)
    with ResidentScene(device, ctl, s, i) as rs:
        out1, _, _ = rs.adjust(output=True)
        _, st2, _ = rs.adjust()
        poses2, points2 = rs.read()
    for got, want in ((out1[n:n + 26], ref1[n:n + 26]), (st2[:26], ref2[n:n + 26])):
        assert abs(got[6] - want[6]) <= COST_REL * want[6], (got[6], want[6])
        assert got[10] == want[10] and got[11] == want[11]  # accepted, rejected
    assert np.max(np.abs(out1[:12 * C] - ref1[:12 * C])) < POSE_TOL
    assert np.max(np.abs(poses2 - ref2[:12 * C])) < POSE_TOL


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
