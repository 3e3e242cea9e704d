"""Joint inverse-depth bundle adjustment on the CPU: the restated host steps
(oracle/inverse_depth_steps.py) driven by the oracle's CPU linearisation, i.e. the reference's CPU
`bundleAdjustInverseDepth`, and the package's own host steps (typecv_b200/inverse_depth_bundle.py)
held to it.

Restates tests/inverse-depth-bundle.test.ts:9-139 and tests/inverse-depth-sparse.test.ts:7-164 on the
same fixtures (tests/scene.ts restated in reference_cases.scene), plus the control checks of
inverseDepthBundleSteps (src/sfm/depth/inverse-depth-bundle.ts:214-263).
"""
import copy
import math

import numpy as np
import pytest

from oracle import inverse_depth as oid
from reference_cases import scene, seeded_random, update_pose
RangeError = ValueError  # both the package's and the oracle's RangeError derive from it
from typecv_b200.inverse_depth import camera_center

BA = oid.bundle_adjust_inverse_depth


def project_point(camera, pose, X):
    return list(oid.camera_projection(camera, oid.transform_point(pose, X))[0])


def fit_for(model, observations):
    by_id = {v["id"]: v for v in model["views"]}
    return oid.fit_inverse_depth([{"camera": by_id[o["viewId"]]["camera"], "pose": by_id[o["viewId"]]["pose"],
                                   "pixel": o["pixel"]} for o in observations])


def test_anchored_joint_ba_improves_keeps_gauge_and_marginalizes_cameras():
    reconstruction, rng = scene(count=30, views=4, noise=0.1)
    views = []
    for i, v in enumerate(reconstruction["views"]):
        if i == 0:
            views.append(v)
            continue
        delta = [(rng() - 0.5) * s for s in (0.002, 0.002, 0.002, 0.01, 0.01, 0.01)]
        R, t = update_pose(list(v["pose"]["R"]), list(v["pose"]["t"]), delta)
        views.append({**v, "pose": {"R": np.array(R), "t": np.array(t)}})
    landmarks = [{**p, "xyz": np.array([x + (rng() - 0.5) * 0.03 for x in p["xyz"]])} for p in reconstruction["landmarks"]]
    inp = {"views": views, "landmarks": landmarks}
    before = copy.deepcopy(inp)
    result = BA(inp, [], {"iterations": 12})
    d = result["diagnostics"]
    assert d["finalCost"] < d["initialCost"] * 0.1
    assert result["uncertainty"]["observable"] and result["uncertainty"]["poses"] == "joint"
    assert repr(inp) == repr(before)
    out0 = result["reconstruction"]["views"][0]["pose"]
    assert np.array_equal(out0["R"], inp["views"][0]["pose"]["R"]) and np.array_equal(out0["t"], inp["views"][0]["pose"]["t"])

    def baseline(m):
        a, b = camera_center(m["views"][0]["pose"]), camera_center(m["views"][1]["pose"])
        return math.hypot(*[x - b[i] for i, x in enumerate(a)])

    assert abs(baseline(inp) - baseline(result["reconstruction"])) < 1e-10
    p = result["estimates"][0]
    fixed = fit_for(result["reconstruction"], p["observations"])
    assert p.get("covariance") is not None and fixed["covariance"] is not None
    assert p["covariance"][8] > fixed["covariance"][8] * 1.01


def test_joint_uncertainty_agrees_with_repeated_image_noise_trials():
    reconstruction, _ = scene(count=20, views=4, noise=0)
    rng = seeded_random(3862)
    sigma = 0.2

    def gaussian():
        a = math.sqrt(-2 * math.log(max(1e-12, rng())))
        return a * math.cos(2 * math.pi * rng())

    truth = fit_for(reconstruction, reconstruction["landmarks"][0]["observations"])["point"]["parameters"][2]
    z = []
    for _ in range(80):
        noisy = {**reconstruction, "landmarks": [
            {**p, "observations": [{**o, "pixel": [o["pixel"][0] + sigma * gaussian(), o["pixel"][1] + sigma * gaussian()]}
                                   for o in p["observations"]]} for p in reconstruction["landmarks"]]}
        r = BA(noisy, [], {"iterations": 8, "pixelNoiseStdDevPx": sigma})
        p = r["estimates"][0]
        assert p.get("covariance") is not None
        z.append((p["point"]["parameters"][2] - truth) / math.sqrt(p["covariance"][8]))
    within2 = sum(abs(x) <= 2 for x in z) / len(z)
    rms = math.sqrt(sum(x * x for x in z) / len(z))
    assert 0.85 <= within2 <= 1
    assert 0.65 < rms < 1.35


def test_uncertainty_excludes_damping_scales_with_noise_and_nuisance_focal():
    reconstruction, _ = scene(count=25, views=4, noise=0)
    a = BA(reconstruction, [], {"iterations": 0})
    b = BA(reconstruction, [], {"iterations": 0, "pixelNoiseStdDevPx": 2})
    focal = BA(reconstruction, [], {"iterations": 0, "refineSharedFocal": True})
    assert a["uncertainty"]["observable"] and focal["uncertainty"]["observable"]
    assert abs(b["estimates"][0]["covariance"][8] / a["estimates"][0]["covariance"][8] - 4) < 1e-8
    assert focal["estimates"][0]["covariance"][8] > a["estimates"][0]["covariance"][8]
    two = reconstruction["views"][:2]
    ids = {v["id"] for v in two}
    degenerate = {"views": two, "landmarks": [{**p, "observations": [o for o in p["observations"] if o["viewId"] in ids]}
                                              for p in reconstruction["landmarks"][:2]]}
    unknown = BA(degenerate, [], {"iterations": 0})
    assert unknown["uncertainty"]["observable"] is False
    assert all(p.get("covariance") is None for p in unknown["estimates"])


def test_joint_solve_recovers_a_shared_focal_error():
    reconstruction, _ = scene(count=30, views=5, noise=0)
    inp = {**reconstruction, "views": [{**v, "camera": {**v["camera"], "fx": v["camera"]["fx"] * 0.9,
                                                          "fy": v["camera"]["fy"] * 0.9}} for v in reconstruction["views"]]}
    result = BA(inp, [], {"iterations": 30, "refineSharedFocal": True})
    assert result["diagnostics"]["finalCost"] < result["diagnostics"]["initialCost"] * 1e-8
    assert abs(result["reconstruction"]["views"][0]["camera"]["fx"] / reconstruction["views"][0]["camera"]["fx"] - 1) < 1e-6
    assert result["uncertainty"]["intrinsics"] == "joint-focal"


@pytest.mark.parametrize("shared_focal", [False, True])
def test_sparse_and_dense_solves_agree_on_objective_and_marginals(shared_focal):
    reconstruction, _ = scene(count=40, views=6, noise=0.15)
    dense = BA(reconstruction, [], {"solver": "dense", "iterations": 2, "refineSharedFocal": shared_focal})
    sparse = BA(reconstruction, [], {"solver": "sparse", "iterations": 2, "refineSharedFocal": shared_focal})
    assert dense["uncertainty"]["observable"] and sparse["uncertainty"]["observable"]
    assert abs(sparse["diagnostics"]["finalCost"] - dense["diagnostics"]["finalCost"]) < 1e-7
    for a, b in zip(dense["estimates"], sparse["estimates"]):
        for k in range(3):
            assert abs(b["covariance"][4 * k] / a["covariance"][4 * k] - 1) < 1e-6
    assert sparse["diagnostics"]["linearSolver"] == "sparse"
    assert sparse["diagnostics"]["cameraCovarianceEntries"] < dense["diagnostics"]["cameraCovarianceEntries"]


@pytest.mark.parametrize("solver", ["dense", "sparse"])
def test_zero_parallax_seed_is_deferred_without_removing_other_uncertainty(solver):
    reconstruction, _ = scene(count=30, views=4, noise=0)
    base = reconstruction["views"][0]
    repeated = {**base, "id": 100}
    good = [{**p, "observations": p["observations"] + [
        {"viewId": 100, "featureId": p["trackId"], "pixel": project_point(base["camera"], base["pose"], p["xyz"])}]}
        for p in reconstruction["landmarks"]]
    xyz = np.array([0.2, 0.1, 8.0])
    pixel = project_point(base["camera"], base["pose"], xyz)
    bad = {"trackId": 1000, "xyz": xyz, "observations": [{"viewId": base["id"], "featureId": 1000, "pixel": pixel},
                                                         {"viewId": 100, "featureId": 1000, "pixel": pixel}]}
    views = reconstruction["views"] + [repeated]
    clean = BA({"views": views, "landmarks": good}, [], {"solver": solver, "iterations": 1})
    result = BA({"views": views, "landmarks": good + [bad]}, [], {"solver": solver, "iterations": 1})
    assert result["uncertainty"]["observable"]
    assert result["diagnostics"]["deferredTrackIds"] == [1000]
    assert all(p.get("covariance") is not None for p in result["estimates"][:30])
    for i in range(30):
        assert abs(result["estimates"][i]["covariance"][8] / clean["estimates"][i]["covariance"][8] - 1) < 1e-10
    assert result["estimates"][30].get("covariance") is None
    assert result["estimates"][30]["informationDeferred"] is True
    assert len(result["reconstruction"]["landmarks"]) == 30
    assert result["diagnostics"]["inputObservations"] - result["diagnostics"]["observations"] == 2
    third = reconstruction["views"][1]
    recovered = BA({"views": views, "landmarks": good + [{**bad, "observations": bad["observations"] + [
        {"viewId": third["id"], "featureId": 1000, "pixel": project_point(third["camera"], third["pose"], xyz)}]}]},
        [], {"solver": solver, "iterations": 1})
    assert recovered["diagnostics"]["deferredTrackIds"] == []
    assert recovered["estimates"][30].get("covariance") is not None
    assert len(recovered["reconstruction"]["landmarks"]) == 31


def long_scene(count):
    """longScene (tests/inverse-depth-sparse.test.ts:107-133)."""
    f, _ = scene(count=12, views=4, noise=0)
    camera = f["views"][0]["camera"]
    views = [{"id": i, "camera": camera, "pose": {"R": np.eye(3).ravel(),
                                                  "t": np.array([-0.03 * i, -0.04 * math.sin(i), -0.02 * math.sin(i * 0.2)])}}
             for i in range(count)]
    points = [p["xyz"] for p in f["landmarks"]]
    return {"views": views, "landmarks": [
        {"trackId": start * 12 + j, "xyz": xyz,
         "observations": [{"viewId": v["id"], "featureId": start * 12 + j, "pixel": project_point(v["camera"], v["pose"], xyz)}
                          for v in views[start:start + 4]]}
        for start in range(count - 3) for j, xyz in enumerate(points)]}


def test_large_camera_graph_uses_compact_cross_blocks_and_selected_inverse():
    inp = long_scene(40)
    result = BA(inp, [], {"iterations": 0})
    d = result["diagnostics"]
    assert d["cameraParameters"] == 233 and d["linearSolver"] == "sparse"
    assert result["uncertainty"]["observable"]
    assert all(p.get("covariance") is not None for p in result["estimates"])
    assert d["pointCrossEntries"] < d["denseEquivalentCrossEntries"] / 5
    assert d["cameraCovarianceEntries"] < d["cameraParameters"] ** 2 / 3
    with pytest.raises(RangeError, match="budget"):
        BA(inp, [], {"iterations": 0, "maxSchurEntries": 10})
    with pytest.raises(RangeError, match="budget"):
        BA(inp, [], {"iterations": 0, "solver": "sparse", "maxFactorEntries": 10})


def test_controls_are_checked():
    reconstruction, _ = scene(count=12, views=3, noise=0)
    for bad in ({"iterations": -1}, {"iterations": 101}, {"huberPx": 0}, {"pixelNoiseStdDevPx": math.inf},
                {"maxCameraParameters": 0}):
        with pytest.raises(RangeError, match="Invalid inverse-depth bundle controls"):
            BA(reconstruction, [], bad)
    for bad in ({"maxSchurEntries": 0}, {"measurementBatchSize": 0}, {"solver": "qr"}):
        with pytest.raises(RangeError, match="sparse/batch controls"):
            BA(reconstruction, [], bad)
    with pytest.raises(RangeError, match="gauge"):
        BA(reconstruction, [], {"anchorViewId": 10, "scaleViewId": 10})
    with pytest.raises(RangeError, match="variable cameras"):
        BA(reconstruction, [], {"variableViewIds": [10, 20]})
    with pytest.raises(RangeError, match="camera parameter budget"):
        BA(reconstruction, [], {"maxCameraParameters": 5})
    moved = {**reconstruction, "views": [reconstruction["views"][0], {**reconstruction["views"][1],
                                                                      "pose": reconstruction["views"][0]["pose"]},
                                         reconstruction["views"][2]]}
    with pytest.raises(RangeError, match="pure rotation"):
        BA(moved, [], {})
