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


# ---- the package's array-wise host steps held to the oracle's loop restatement ----------------------

def product_ba(inp, constraints=(), options=None):
    """typecv_b200's host steps answered by the oracle's C++ linearisation (no device)."""
    from typecv_b200 import inverse_depth_bundle as IDB
    return IDB.drive(IDB.inverse_depth_bundle_steps(inp, constraints, options),
                     lambda job: oid.linearize_rows(job["rows"]))


EXACT = ("acceptedSteps", "observations", "cameraParameters", "linearSolver", "schurEntries", "factorEntries",
         "cameraCovarianceEntries", "pointCrossEntries", "denseEquivalentCrossEntries", "inputObservations",
         "deferredTrackIds")


def assert_same_solve(got, want, cost=1e-9, state=1e-8, covariance=1e-7, converged=False):
    """Same diagnostics, costs, poses, points and covariances.  Once the solve has converged a
    candidate's cost differs from the current one by rounding only, and which of those steps are
    taken is not part of the comparison (``converged``)."""
    dg, dw = got["diagnostics"], want["diagnostics"]
    for key in EXACT:
        if key == "acceptedSteps" and converged:
            continue
        assert dg[key] == dw[key], (key, dg[key], dw[key])
    for key in ("initialCost", "finalCost"):
        assert abs(dg[key] - dw[key]) <= cost * max(1.0, abs(dw[key])), (key, dg[key], dw[key])
    assert got["uncertainty"] == want["uncertainty"]
    for a, b in zip(got["reconstruction"]["views"], want["reconstruction"]["views"]):
        assert a["id"] == b["id"]
        assert np.max(np.abs(np.asarray(a["pose"]["R"]) - np.asarray(b["pose"]["R"]))) < state
        assert np.max(np.abs(np.asarray(a["pose"]["t"]) - np.asarray(b["pose"]["t"]))) < state
        assert abs(a["camera"]["fx"] / b["camera"]["fx"] - 1) < state
    assert [p["trackId"] for p in got["reconstruction"]["landmarks"]] == \
        [p["trackId"] for p in want["reconstruction"]["landmarks"]]
    for a, b in zip(got["reconstruction"]["landmarks"], want["reconstruction"]["landmarks"]):
        assert np.max(np.abs(np.asarray(a["xyz"]) - np.asarray(b["xyz"]))) < state * max(1.0, np.max(np.abs(b["xyz"])))
    assert len(got["estimates"]) == len(want["estimates"])
    for a, b in zip(got["estimates"], want["estimates"]):
        assert a["trackId"] == b["trackId"] and a.get("informationDeferred") == b.get("informationDeferred")
        assert np.max(np.abs(np.asarray(a["point"]["parameters"]) - np.asarray(b["point"]["parameters"]))) < state
        assert np.max(np.abs(np.asarray(a["point"]["reference"]["t"]) - np.asarray(b["point"]["reference"]["t"]))) < state
        for key in ("covariance", "bearingCovariance"):
            assert (a.get(key) is None) == (b.get(key) is None), key
            if b.get(key) is not None:
                ca, cb = np.asarray(a[key]), np.asarray(b[key])
                scale = np.sqrt(np.outer(np.abs(np.diag(cb.reshape(int(math.isqrt(cb.size)), -1))),
                                         np.abs(np.diag(cb.reshape(int(math.isqrt(cb.size)), -1))))).ravel()
                assert np.max(np.abs(ca - cb) / scale) < covariance, key


def perturbed_scene(count=30, views=4, seed_noise=0.1):
    reconstruction, rng = scene(count=count, views=views, noise=seed_noise)
    out = []
    for i, v in enumerate(reconstruction["views"]):
        if i == 0:
            out.append(v)
            continue
        delta = [(rng() - 0.5) * s for s in (0.002, 0.002, 0.002, 0.01, 0.01, 0.01)]
        R, t = update_pose(list(v["pose"]["R"]), list(v["pose"]["t"]), delta)
        out.append({**v, "pose": {"R": np.array(R), "t": np.array(t)}})
    landmarks = [{**p, "xyz": np.array([x + (rng() - 0.5) * 0.03 for x in p["xyz"]])} for p in reconstruction["landmarks"]]
    return {"views": out, "landmarks": landmarks}


@pytest.mark.parametrize("options", [
    {"iterations": 4},
    {"iterations": 6, "refineSharedFocal": True},
    {"iterations": 4, "solver": "sparse"},
    {"iterations": 4, "solver": "sparse", "refineSharedFocal": True, "huberPx": 0.05},
    {"iterations": 3, "variableViewIds": [30, 40]},
    {"iterations": 0, "pixelNoiseStdDevPx": 2},
])
def test_package_steps_match_the_oracle_steps(options):
    inp = perturbed_scene()
    before = copy.deepcopy(inp)
    got = product_ba(inp, [], options)
    assert repr(inp) == repr(before)
    assert_same_solve(got, BA(inp, [], options))


def test_package_steps_match_past_convergence():
    inp = perturbed_scene()
    got, want = product_ba(inp, [], {"iterations": 12}), BA(inp, [], {"iterations": 12})
    assert got["diagnostics"]["finalCost"] < got["diagnostics"]["initialCost"] * 1e-2
    assert_same_solve(got, want, converged=True)


def test_package_steps_match_on_a_shared_focal_error_and_focal_groups():
    reconstruction, _ = scene(count=30, views=5, noise=0)
    inp = {**reconstruction, "views": [{**v, "camera": {**v["camera"], "fx": v["camera"]["fx"] * 0.9,
                                                          "fy": v["camera"]["fy"] * 0.9}} for v in reconstruction["views"]]}
    options = {"iterations": 30, "refineSharedFocal": True}
    assert_same_solve(product_ba(inp, [], options), BA(inp, [], options), cost=1e-7, converged=True)
    groups = {"iterations": 5, "refineSharedFocal": True, "focalGroups": {v["id"]: v["id"] % 2 for v in inp["views"]}}
    assert_same_solve(product_ba(inp, [], groups), BA(inp, [], groups))


@pytest.mark.parametrize("solver", ["dense", "sparse"])
def test_package_steps_match_with_a_deferred_track(solver):
    reconstruction, _ = scene(count=30, views=4, noise=0)
    base = reconstruction["views"][0]
    views = reconstruction["views"] + [{**base, "id": 100}]
    good = [{**p, "observations": p["observations"] + [
        {"viewId": 100, "featureId": p["trackId"], "pixel": project_point(base["camera"], base["pose"], p["xyz"])}]}
        for p in reconstruction["landmarks"]]
    xyz = np.array([0.2, 0.1, 8.0])
    pixel = project_point(base["camera"], base["pose"], xyz)
    bad = {"trackId": 1000, "xyz": xyz, "observations": [{"viewId": base["id"], "featureId": 1000, "pixel": pixel},
                                                         {"viewId": 100, "featureId": 1000, "pixel": pixel}]}
    inp = {"views": views, "landmarks": good + [bad]}
    got = product_ba(inp, [], {"solver": solver, "iterations": 2})
    assert got["diagnostics"]["deferredTrackIds"] == [1000]
    assert_same_solve(got, BA(inp, [], {"solver": solver, "iterations": 2}))


def test_package_steps_match_with_constraints():
    """Bearing-only and inverse-depth constraint tracks beside the landmarks (the 2 x 2 blocks and
    the constraint checks of inverse-depth-bundle.ts:264-303)."""
    inp = perturbed_scene(count=20)
    views = inp["views"]
    rng = seeded_random(77)
    constraints = []
    for k in range(6):
        X = np.array([(rng() - 0.5) * 2, (rng() - 0.5) * 1.5, 6 + 2 * rng()])
        obs = [{"viewId": v["id"], "featureId": 5000 + k, "pixel": project_point(v["camera"], v["pose"], X)}
               for v in views[:3 if k % 2 else 4]]
        ref = views[0]["pose"]
        q = oid.transform_point(ref, X)
        direction = k % 2 == 0
        constraints.append({"trackId": 9000 + k, "observations": obs, "directionOnly": direction,
                            "point": {"reference": {"R": ref["R"], "t": ref["t"]},
                                      "parameters": [q[0] / q[2] + 0.001, q[1] / q[2] - 0.002,
                                                     0.0 if direction else 1 / q[2] * 1.05]}})
    for options in ({"iterations": 5}, {"iterations": 3, "solver": "sparse", "refineSharedFocal": True}):
        got = product_ba(inp, constraints, options)
        assert_same_solve(got, BA(inp, constraints, options))
        assert all(e.get("bearingCovariance") is not None for e in got["estimates"][-6:])
        assert all(e.get("covariance") is None for e in got["estimates"][-6::2])
    with pytest.raises(RangeError, match="Bearing-only"):
        product_ba(inp, [{**constraints[0], "point": {**constraints[0]["point"], "parameters": [0, 0, 1]}}])
    with pytest.raises(RangeError, match="Multiply owned"):
        product_ba(inp, [{**constraints[1], "observations": [inp["landmarks"][0]["observations"][0],
                                                              *constraints[1]["observations"][1:]]}])


def test_package_steps_match_on_the_long_camera_graph():
    inp = long_scene(40)
    got = product_ba(inp, [], {"iterations": 2})
    assert got["diagnostics"]["linearSolver"] == "sparse"
    assert_same_solve(got, BA(inp, [], {"iterations": 2}))
    for options in ({"iterations": 0, "maxSchurEntries": 10}, {"iterations": 0, "solver": "sparse", "maxFactorEntries": 10},
                    {"iterations": 0, "solver": "sparse", "maxFactorEntries": 2000}):
        with pytest.raises(RangeError) as want:
            BA(inp, [], options)
        with pytest.raises(RangeError) as have:
            product_ba(inp, [], options)
        assert str(have.value) == str(want.value)


def test_package_steps_match_on_the_noisy_corridor():
    """The seeded corridor of the joint inverse-depth benchmark (noisy pixels, perturbed start)."""
    from typecv_b200.synthetic import inverse_depth_corridor
    inp = inverse_depth_corridor(views=24)
    got, want = product_ba(inp, [], {"iterations": 3}), BA(inp, [], {"iterations": 3})
    assert got["diagnostics"]["finalCost"] < got["diagnostics"]["initialCost"] * 0.1
    assert_same_solve(got, want)


def test_package_steps_match_with_small_point_chunks(monkeypatch):
    """The point elimination and the marginals in chunks of one or a few points (the chunk bound
    lowered) give the same solve."""
    from typecv_b200 import inverse_depth_bundle as IDB
    inp = long_scene(16)
    want = BA(inp, [], {"iterations": 2})
    monkeypatch.setattr(IDB, "CHUNK_ELEMENTS", 64)
    assert_same_solve(product_ba(inp, [], {"iterations": 2}), want)


@pytest.mark.parametrize("seed", range(6))
def test_minimum_degree_fill_matches_the_sparse_factor(seed):
    """The elimination order and factor entries of the pattern-only minimum degree equal the
    oracle's numeric sparse factor on random SPD systems with random sparsity."""
    from oracle import inverse_depth_steps as OS
    from typecv_b200 import inverse_depth_bundle as IDB
    rng = np.random.default_rng(seed)
    n = int(rng.integers(5, 40))
    pattern = np.triu(rng.random((n, n)) < rng.uniform(0.05, 0.4), 1)
    pattern = pattern | pattern.T | np.eye(n, dtype=bool)
    A = np.where(pattern, rng.normal(size=(n, n)), 0.0)
    A = np.triu(A, 1) + np.triu(A, 1).T
    A += np.diag(np.abs(A).sum(axis=1) + 1.0)
    S = OS.SparseSymmetric(n, 10**9)
    for i in range(n):
        for j in range(i, n):
            if pattern[i, j]:
                S.add(i, j, A[i, j])
    f = OS.factor_sparse_schur(S, 10**9)
    order, entries = IDB._minimum_degree(pattern, S.entries, 10**9)
    assert entries == f.entries and list(order) == list(f.order)
    inv = IDB._factor_inverse(A, order)
    assert np.allclose(inv, np.linalg.inv(A), rtol=1e-10, atol=1e-12)
    for i in range(n):
        assert abs(f.covariance(i, i) - inv[i, i]) <= 1e-10 * inv[i, i]
