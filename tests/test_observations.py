"""Observation evaluation (typecv_b200/observations.py, tba_evaluate_observations).

The cases restate the reference's fixed-scene observation fixtures
(tests/typeshade/indexed-observations-cases.mjs:1-131): an empty scene, an unreferenced view outside
the GPU bounds, a radial tail of 129 observations, shuffled view/point/observation order, per-view
calibration with rotated poses, an outlier and a point behind the cameras, far points whose depth
is unstable, and a 65-observation track.  The oracle restates the reference kernels
(oracle/observations.py); the CUDA path must give the same masks, rejections and counts, and the
same mean error within 1e-12.
"""
import math

import numpy as np
import pytest

from oracle import observations as OO
from typecv_b200 import RangeError
from typecv_b200 import observations as OB


def observation_model(points=43, views=3, depth=10, baseline=0.35, radial=True):
    """observationModel (indexed-observations-cases.mjs:8-50)."""
    camera = {"fx": 730, "fy": 710, "cx": 312.5, "cy": 247.25, "k1": 0.08 if radial else 0, "k2": -0.01 if radial else 0}
    registered = [{"id": 10 + 7 * i, "camera": dict(camera),
                   "pose": {"R": np.array([1.0, 0, 0, 0, 1, 0, 0, 0, 1]), "t": np.array([-i * baseline, -0.0, 0])}}
                  for i in range(views)]
    landmarks = []
    for p in range(points):
        X = [-0.7 + 0.04 * p, 0.2 * math.sin(p), depth + 0.03 * p]
        obs = []
        for i, v in enumerate(registered):
            x, y = (X[0] - i * baseline) / X[2], X[1] / X[2]
            r2 = x * x + y * y
            d = 1 + camera["k1"] * r2 + camera["k2"] * r2 * r2
            obs.append({"viewId": v["id"], "featureId": p,
                        "pixel": [camera["fx"] * x * d + camera["cx"] + ((p + i) % 4) * 0.03,
                                  camera["fy"] * y * d + camera["cy"]]})
        landmarks.append({"trackId": 1000 + p, "xyz": np.array(X), "observations": obs})
    return {"views": registered, "landmarks": landmarks}


def observation_cases():
    """observationCases (indexed-observations-cases.mjs:52-131)."""
    mixed = observation_model(points=5)
    mixed["landmarks"][1]["observations"][2]["pixel"][0] += 40
    mixed["landmarks"][2]["xyz"][2] = -10
    unused = observation_model(points=2)
    unused["views"].append({**unused["views"][0], "id": 9999, "camera": {**unused["views"][0]["camera"], "fx": 1e8}})
    shuffled = observation_model(points=5, views=4)
    shuffled["views"].reverse()
    shuffled["landmarks"].reverse()
    for p in shuffled["landmarks"]:
        p["observations"] = [p["observations"][i] for i in (2, 0, 3, 1)]
    calibrated = observation_model(points=5, views=4)
    for i, v in enumerate(calibrated["views"]):
        a = i * 0.025
        c, s = math.cos(a), math.sin(a)
        v["pose"]["R"] = np.array([c, 0, s, 0, 1, 0, -s, 0, c])
        v["camera"].update({"fx": 600 + 41 * i, "fy": 640 + 27 * i, "cx": 301 + 3 * i, "k1": -0.03 + i * 0.025,
                            "k2": 0.001 * i})
    for p in calibrated["landmarks"]:
        for i, o in enumerate(p["observations"]):
            v = calibrated["views"][i]
            k, X, R, t = v["camera"], p["xyz"], v["pose"]["R"], v["pose"]["t"]
            q = [R[3 * r] * X[0] + R[3 * r + 1] * X[1] + R[3 * r + 2] * X[2] + t[r] for r in range(3)]
            x, y = q[0] / q[2], q[1] / q[2]
            r2 = x * x + y * y
            d = 1 + k["k1"] * r2 + k["k2"] * r2 * r2
            o["pixel"] = [k["fx"] * x * d + k["cx"] + 0.02, k["fy"] * y * d + k["cy"]]
    guard = {"maxRelativeDepthStdDev": 0.1}
    return [
        ("empty", {"views": [], "landmarks": []}, None),
        ("empty-guarded", {"views": [], "landmarks": []}, guard),
        ("unused-view-outside-gpu-bounds", unused, None),
        ("radial-tail-129", observation_model(), None),
        ("shuffled-view-point-observation-indices", shuffled, guard),
        ("different-calibration-and-rotated-poses", calibrated, guard),
        ("radial-tail-129-guarded", observation_model(), guard),
        ("mixed-inliers-behind-camera", mixed, guard),
        ("far-depth-rejected", observation_model(points=3, baseline=0.0001, depth=2000), {"maxRelativeDepthStdDev": 0.01}),
        ("long-track-65", observation_model(points=1, views=65, baseline=0.01), guard),
    ]


def oracle_result(model, options=None, max_error=3, last_only=False):
    req = OB.observation_request(model, max_error, options, last_only)
    o = OO.evaluate(req)
    return OB.unpack_observations(o["summary"], o["flags"], req["lengths"], req["count"], req["guarded"])


def test_oracle_known_answers():
    res = {name: oracle_result(m, opt) for name, m, opt in observation_cases()}
    assert res["empty"]["masks"] == [] and res["empty"]["inlierCount"] == 0 and res["empty"]["meanErrorPx"] == math.inf
    assert list(res["empty-guarded"]["depthRejected"]) == []
    assert res["radial-tail-129"]["inlierCount"] == 129
    assert 0 < res["radial-tail-129"]["meanErrorPx"] < 0.09
    mixed = res["mixed-inliers-behind-camera"]
    assert list(mixed["masks"][1]) == [1, 1, 0]          # the 40 px outlier
    assert list(mixed["masks"][2]) == [0, 0, 0]          # behind every camera
    assert list(mixed["depthRejected"]) == [0, 0, 0, 0, 0]
    far = res["far-depth-rejected"]
    assert list(far["depthRejected"]) == [1, 1, 1] and far["inlierCount"] == 0
    assert res["long-track-65"]["inlierCount"] == 65
    assert res["unused-view-outside-gpu-bounds"]["inlierCount"] == 6


def test_request_checks_and_messages():
    m = observation_model(points=2)
    with pytest.raises(RangeError, match="Invalid GPU observation threshold"):
        OB.observation_request(m, 0.0, None, False)
    with pytest.raises(RangeError, match="Invalid conditional depth sensitivity options"):
        OB.observation_request(m, 3, {"maxRelativeDepthStdDev": -1}, False)
    with pytest.raises(RangeError, match="Invalid conditional depth sensitivity options"):
        OB.observation_request(m, 3, {"pixelNoiseStdDevPx": 0}, False)
    bad = observation_model(points=2)
    bad["landmarks"][0]["xyz"][0] = 2e9
    with pytest.raises(RangeError, match="Invalid GPU scene coordinate bounds"):
        OB.observation_request(bad, 3, None, False)
    cam = observation_model(points=2)
    cam["views"][0]["camera"]["fx"] = 1e7
    with pytest.raises(RangeError, match="Camera exceeds the supported GPU geometry bounds"):
        OB.observation_request(cam, 3, None, False)


def test_continued_request_keeps_only_last_observations():
    m = observation_model(points=4)
    req = OB.observation_request(m, 3, None, True)
    assert req["count"] == 4 and req["lengths"] == [1, 1, 1, 1] and req["C"] == 1
    assert list(req["indices"][1::2]) == [0, 1, 2, 3]


@pytest.mark.gpu
def test_cuda_evaluation_matches_the_oracle_on_every_case():
    import typecv_b200 as tb
    with tb.ShadeDevice.open(0) as dev:
        for name, model, options in observation_cases():
            want = oracle_result(model, options)
            got = OB.evaluate_observations_gpu(dev, model, 3, options)
            assert [list(x) for x in got["masks"]] == [list(x) for x in want["masks"]], name
            assert got["inlierCount"] == want["inlierCount"], name
            if "depthRejected" in want:
                assert list(got["depthRejected"]) == list(want["depthRejected"]), name
            if math.isinf(want["meanErrorPx"]):
                assert math.isinf(got["meanErrorPx"]), name
            else:
                assert abs(got["meanErrorPx"] - want["meanErrorPx"]) <= 1e-12 * want["meanErrorPx"], name


@pytest.mark.gpu
def test_cuda_evaluation_of_a_solved_scene_and_its_last_observations():
    import typecv_b200 as tb
    from typecv_b200 import synthetic as S
    scene = S.helix_scene(seed=31, cameras=20, points=2000).as_reconstruction()
    with tb.ShadeDevice.open(0) as dev:
        for options, threshold in ((None, 3.0), ({"maxRelativeDepthStdDev": 0.05}, 4.0)):
            want = oracle_result(scene, options, threshold)
            got = OB.evaluate_observations_gpu(dev, scene, threshold, options)
            assert got["inlierCount"] == want["inlierCount"] and got["inlierCount"] > 0
            assert all(np.array_equal(a, b) for a, b in zip(got["masks"], want["masks"]))
            assert abs(got["meanErrorPx"] - want["meanErrorPx"]) <= 1e-12 * want["meanErrorPx"]
            if options:
                assert np.array_equal(got["depthRejected"], want["depthRejected"])
        last = OB.evaluate_continued_observations_gpu(dev, scene, 3.0)
        want = oracle_result(scene, None, 3.0, last_only=True)
        assert last["inlierCount"] == want["inlierCount"]
        assert all(len(m) == 1 for m in last["masks"])


def test_cpp_restatement_matches_the_python_one():
    """oracle_evaluate_observations (ba_oracle.cpp) against oracle/observations.py: identical flags,
    errors and summary on a guarded and an unguarded request of a synthetic scene with outliers."""
    import bench
    from oracle import observations as oo
    sc = bench.make_scene("cfg2", 0.01)
    for limit in (0.05, 0.0):
        req = bench.observation_request(sc, limit=limit)
        a, b = oo.evaluate(req), oo.evaluate_cpp(req)
        assert np.array_equal(a["flags"], b["flags"]) and np.array_equal(a["errors"], b["errors"])
        assert np.array_equal(a["summary"], b["summary"])
        assert 0 < a["summary"][1] < req["count"]
