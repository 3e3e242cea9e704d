"""Inverse-depth linearisation: host packing, the oracle and its pins (CPU).

The reference checks its device linearisation against the CPU `inverseDepthJacobian`
(tests/typeshade/inverse-depth-cases.mjs:126-165).  The oracle restates that function
(oracle/inverse_depth.py); it is pinned here by the fixture's own pixels (inverseDepthScene projects
every point exactly, so the anchored point seeded from its XYZ must reproduce them) and by central
differences of every derivative column.
"""
import math

import numpy as np
import pytest

from oracle import inverse_depth as oid
from reference_cases import inverse_depth_long_scene, inverse_depth_scene, update_pose
from typecv_b200 import inverse_depth as ID
from typecv_b200.bundle import RangeError


def anchored(model, track=0, rho=None):
    p = model["landmarks"][track]
    view = model["views"][0]
    point = oid.initialize_inverse_depth(view, p["observations"][0]["pixel"], p["xyz"])
    if rho is not None:
        point["parameters"] = np.array([point["parameters"][0], point["parameters"][1], rho])
    return point


def test_packing_follows_the_reference_row_layout():
    model = inverse_depth_scene()
    point = anchored(model)
    view = model["views"][2]
    row = ID.pack_measurements([{"view": view, "point": point}])
    assert row.shape == (34,)
    assert np.array_equal(row[0:3], point["parameters"])
    assert np.array_equal(row[3:12], point["reference"]["R"]) and np.array_equal(row[12:15], point["reference"]["t"])
    assert np.array_equal(row[15:24], view["pose"]["R"]) and np.array_equal(row[24:27], view["pose"]["t"])
    assert list(row[27:33]) == [800, 760, 320, 240, -0.03, 0]
    assert row[33] == -1 / (3 * -0.03)
    free = {**view, "camera": {"fx": 500, "fy": 500, "cx": 1, "cy": 2}}
    assert ID.pack_measurements([{"view": free, "point": point}])[33] == 1e30


@pytest.mark.parametrize("k1,k2", [(0, 0), (-0.03, 0), (0.1, 0), (-0.2, 0.05), (0.1, -0.02), (-0.3, 0.01),
                                   (0.2, 0.3), (0, -0.1)])
def test_radial_limit_matches_the_oracle(k1, k2):
    assert ID.radial_limit_squared(k1, k2) == oid.radial_limit_squared(k1, k2)


def test_unpacking_keeps_flagged_rows_only():
    out = np.arange(46, dtype=float)
    out[0], out[23] = 1, 0.5
    rows = ID.unpack_linearizations(out, 2)
    assert rows[1] is None
    assert rows[0]["pixel"] == (1.0, 2.0)
    assert np.array_equal(rows[0]["point"], np.arange(3, 9)) and np.array_equal(rows[0]["pose"], np.arange(9, 21))
    assert np.array_equal(rows[0]["focal"], [21, 22])


def test_oracle_reproduces_the_fixture_pixels():
    for model in (inverse_depth_scene(), inverse_depth_long_scene()):
        views = {v["id"]: v for v in model["views"]}
        worst = 0.0
        for p in model["landmarks"][:40]:
            first = views[p["observations"][0]["viewId"]]
            point = oid.initialize_inverse_depth(first, p["observations"][0]["pixel"], p["xyz"])
            for o in p["observations"]:
                v = views[o["viewId"]]
                j = oid.inverse_depth_jacobian(v["camera"], v["pose"], point)
                worst = max(worst, abs(j["pixel"][0] - o["pixel"][0]), abs(j["pixel"][1] - o["pixel"][1]))
        assert worst < 1e-9


def test_bearing_only_anchor_projects_onto_its_own_pixel():
    model = inverse_depth_scene()
    v = model["views"][0]
    o = model["landmarks"][3]["observations"][0]
    point = oid.initialize_inverse_depth(v, o["pixel"])
    assert point["parameters"][2] == 0
    j = oid.inverse_depth_jacobian(v["camera"], v["pose"], point)
    assert abs(j["pixel"][0] - o["pixel"][0]) < 1e-9 and abs(j["pixel"][1] - o["pixel"][1]) < 1e-9
    # At rho = 0 the translation sensitivity is exactly zero.
    assert np.all(j["pose"][[3, 4, 5, 9, 10, 11]] == 0)


@pytest.mark.parametrize("rho_scale", [1.0, 0.0, 3.0])
def test_oracle_derivatives_match_central_differences(rho_scale):
    model = inverse_depth_scene()
    base = anchored(model, track=5)
    point = {**base, "parameters": base["parameters"] * np.array([1, 1, rho_scale])}
    v = model["views"][3]
    j = oid.inverse_depth_jacobian(v["camera"], v["pose"], point)
    h = 1e-6

    def pixel(camera, pose, pt):
        return np.array(oid.inverse_depth_jacobian(camera, pose, pt)["pixel"])

    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        plus = pixel(v["camera"], v["pose"], {**point, "parameters": point["parameters"] + e})
        minus = pixel(v["camera"], v["pose"], {**point, "parameters": point["parameters"] - e})
        fd = (plus - minus) / (2 * h)
        assert np.allclose(fd, j["point"][[k, 3 + k]], rtol=1e-6, atol=1e-4)
    for k in range(6):
        d = [0.0] * 6
        d[k] = h
        Rp, tp = update_pose(list(v["pose"]["R"]), list(v["pose"]["t"]), d)
        d[k] = -h
        Rm, tm = update_pose(list(v["pose"]["R"]), list(v["pose"]["t"]), d)
        fd = (pixel(v["camera"], {"R": Rp, "t": tp}, point) - pixel(v["camera"], {"R": Rm, "t": tm}, point)) / (2 * h)
        # The point is carried scaled by rho, so rho times the scaled point's derivative is the
        # metric translation derivative; at rho = 0 (a point at infinity) it is exactly zero.
        if k >= 3 and point["parameters"][2] == 0:
            assert np.all(j["pose"][[k, 6 + k]] == 0)
        assert np.allclose(fd, j["pose"][[k, 6 + k]], rtol=1e-6, atol=1e-4)
    s = 1e-7
    cam_p = {**v["camera"], "fx": v["camera"]["fx"] * math.exp(s), "fy": v["camera"]["fy"] * math.exp(s)}
    cam_m = {**v["camera"], "fx": v["camera"]["fx"] * math.exp(-s), "fy": v["camera"]["fy"] * math.exp(-s)}
    fd = (pixel(cam_p, v["pose"], point) - pixel(cam_m, v["pose"], point)) / (2 * s)
    assert np.allclose(fd, j["focal"], rtol=1e-6, atol=1e-4)


def test_a_strongly_negative_inverse_depth_leaves_the_far_views_invalid():
    model = inverse_depth_scene()
    for rho in (0, 1e-9, 0.2, -0.01):
        assert all(oid.inverse_depth_jacobian(v["camera"], v["pose"], anchored(model, rho=rho)) is not None
                   for v in model["views"])
    valid = [oid.inverse_depth_jacobian(v["camera"], v["pose"], anchored(model, rho=-5)) is not None
             for v in model["views"]]
    # The anchor view sees the bearing whatever rho is; the point sits behind the later views.
    assert valid == [True, True, False, False]


def test_batch_controls_are_checked_before_any_device_work():
    class NoDevice:
        working_bytes = None

        @property
        def handle(self):
            raise AssertionError("no device call expected")

    job = {"measurements": [{"view": inverse_depth_scene()["views"][1], "point": anchored(inverse_depth_scene())}]}
    for bad in (0, -1, 1.5, True):
        with pytest.raises(RangeError, match="batch"):
            ID.linearize_batches(NoDevice(), job, bad)
    small = NoDevice()
    small.working_bytes = 1
    with pytest.raises(RangeError, match="budget"):
        ID.linearize_batches(small, job)
    assert ID.linearize_batches(NoDevice(), {"measurements": []}) == {"rows": [], "batches": 0, "batchSize": 0,
                                                                      "reports": []}


def test_cpp_restatement_is_bit_identical_to_the_python_one():
    """oracle_linearize_inverse_depth (ba_oracle.cpp, no FMA) against inverse_depth_jacobian on the
    fixture's measurements, rows outside the model's domain included."""
    model = inverse_depth_scene()
    wide = {**model["views"][1], "camera": {"fx": 800, "fy": 760, "cx": 320, "cy": 240, "k1": -10.0}}
    ms = [{"view": v, "point": anchored(model, track=t, rho=rho)} for t in (0, 7, 13) for rho in (0, 0.2, -5)
          for v in model["views"] + [wide]]
    rows = ID.pack_measurements(ms).reshape(-1, 34)
    out = oid.linearize_rows(rows)
    invalid = 0
    for m, r in zip(ms, out):
        p = oid.inverse_depth_jacobian(m["view"]["camera"], m["view"]["pose"], m["point"])
        if p is None:
            invalid += 1
            assert not r.any()
            continue
        assert np.array_equal(np.concatenate([[1], p["pixel"], p["point"], p["pose"], p["focal"]]), r)
    assert 0 < invalid < len(ms)
