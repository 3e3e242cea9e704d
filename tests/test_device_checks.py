"""The structural checks of tba_bundle_adjust, which run on the device after the upload, against
the host checks of tba_scene_create (the same checks on the host, in the same order): every
corruption of the packed arrays gets the same message from both, including the first of several
failures, and no solver kernel runs on a failing problem.
"""
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


@pytest.fixture(scope="module")
def problem():
    sc = S.ring_scene(cameras=6, points=300)
    s, i = sc.packed()
    return sc, s, i


def sections(sc, i):
    C, P, M = sc.C, sc.P, sc.M
    return {"obs_camera": (0, M), "obs_point": (M, 2 * M), "ps": (2 * M, 2 * M + P + 1),
            "cs": (2 * M + P + 1, 2 * M + P + C + 2), "cam_obs": (2 * M + P + C + 2, 3 * M + P + C + 2),
            "active": (3 * M + P + C + 2, 3 * M + P + 2 * C + 2)}


def corrupt(sc, s, i, kind):
    s, i = s.copy(), i.copy()
    sec = sections(sc, i)
    at = lambda name, k: sec[name][0] + k
    if kind == "point_ends":
        i[at("ps", sc.P)] -= 1
    elif kind == "short_track":
        # point 3 keeps one observation (its successor's list starts one after its own)
        i[at("ps", 4)] = i[at("ps", 3)] + 1
    elif kind == "point_mismatch":
        i[at("obs_point", 5)] += 1
    elif kind == "camera_range":
        i[at("obs_camera", sc.M - 2)] = sc.C + 3
    elif kind == "camera_ends":
        i[at("cs", sc.C)] -= 1
    elif kind == "camera_offsets":
        i[at("cs", 2)], i[at("cs", 3)] = i[at("cs", 3)], i[at("cs", 2)]
    elif kind == "lists_duplicate":
        b = sec["cam_obs"][0] + i[at("cs", 1)]
        i[b + 1] = i[b]
    elif kind == "lists_foreign":
        b0, b1 = sec["cam_obs"][0] + i[at("cs", 1)], sec["cam_obs"][0] + i[at("cs", 2)]
        i[b0], i[b1] = i[b1], i[b0]
    elif kind == "activity":
        i[at("active", 2)] = 2
    elif kind == "anchor":
        i[at("active", 0)] = 1
    elif kind == "scene_nan":
        s[12 * sc.C + 7] = np.nan
    elif kind == "scene_tiny":
        s[18 * sc.C + 3 * sc.P + 11] = 1e-31
    elif kind == "camera_bounds":
        s[12 * sc.C + 3 * sc.P + 6 * 2 + 4] = 2.0
    elif kind == "two_failures":
        s[12 * sc.C + 7] = np.nan
        i[at("obs_point", 5)] += 1
    elif kind == "late_and_early":
        i[at("active", 2)] = 2
        i[at("obs_camera", 1)] = sc.C
    return s, i


KINDS = ["point_ends", "short_track", "point_mismatch", "camera_range", "camera_ends", "camera_offsets",
         "lists_duplicate", "lists_foreign", "activity", "anchor", "scene_nan", "scene_tiny", "camera_bounds",
         "two_failures", "late_and_early"]


@pytest.mark.parametrize("kind", KINDS)
def test_device_checks_match_the_host_checks(device, problem, kind):
    sc, s0, i0 = problem
    s, i = corrupt(sc, s0, i0, kind)
    ctl = tb.make_control(sc.C, sc.P, sc.M, anchor=0, scale_view=1, iterations=3)
    with pytest.raises(tb.RangeError) as host:
        ResidentScene(device, ctl, s, i)
    with pytest.raises(tb.RangeError) as dev:
        tb.solve_packed(device, ctl, s, i)
    assert str(dev.value) == str(host.value), kind


def test_a_valid_problem_passes_and_reports_its_check_time(device, problem):
    sc, s, i = problem
    ctl = tb.make_control(sc.C, sc.P, sc.M, anchor=0, scale_view=1, iterations=3)
    out, rep = tb.solve_packed(device, ctl, s, i)
    assert rep["lm_iterations"] >= 1 and rep["check_ms"] > 0
    # The handle stays usable after a refused call.
    bad_s, bad_i = corrupt(sc, s, i, "point_mismatch")
    with pytest.raises(tb.RangeError):
        tb.solve_packed(device, ctl, bad_s, bad_i)
    out2, _ = tb.solve_packed(device, ctl, s, i)
    # Same solve: the shared-memory atomics of the product commute only up to rounding.
    base = 12 * sc.C + 3 * sc.P
    assert abs(out2[base + 6] - out[base + 6]) <= 1e-9 * out[base + 6]
    assert np.max(np.abs(out2[:base] - out[:base])) < 1e-7
