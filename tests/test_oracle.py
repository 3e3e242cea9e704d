"""The oracle, pinned: restated fixtures against the reference's input hashes, the operator
restatement against the reference's recorded GPU results, and the reference's own test assertions
(tests/bundle-adjustment.test.ts, tests/typeshade/focal.test.mjs, tests/typeshade/cpu.test.mjs)
against the CPU restatement."""
import json
import math
import os

import numpy as np
import pytest

from oracle import bundle_adjust as ob
from reference_cases import (bundle_fixture, bundle_metrics, input_sha256, joint_focal_fixture, perturbed,
                             scene, skew_bundle_fixture)

RECORDS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_records.json")))["records"]


def record_fixture(rec):
    f = rec["fixture"]
    return skew_bundle_fixture(f["views"], f["count"]) if f["skew"] else bundle_fixture(views=f["views"], count=f["count"])


@pytest.mark.parametrize("rec", RECORDS, ids=lambda r: r["name"] + "/" + str(r["options"]["iterations"]))
def test_restated_fixture_matches_reference_input_hash(rec):
    assert input_sha256(record_fixture(rec)) == rec["inputSha256"]


@pytest.mark.parametrize("rec", RECORDS, ids=lambda r: r["name"] + "/" + str(r["options"]["iterations"]))
def test_operator_oracle_reproduces_reference_gpu_records(rec):
    out = ob.gpu_operator(record_fixture(rec), rec["options"])
    serial = rec["variants"][0]
    costs = [v["finalCost"] for v in rec["variants"]]
    cg = [v["cgIterations"] for v in rec["variants"]]
    final = out["diagnostics"]["finalCost"]
    # The reference's own variants (emulated f64) spread by up to 5e-11 relative.
    assert abs(final - serial["finalCost"]) <= 1e-9 * serial["finalCost"]
    assert min(costs) * (1 - 1e-10) <= final <= max(costs) * (1 + 1e-10)
    assert min(cg) - 2 <= out["cgIterations"] <= max(cg) + 2
    assert out["linearSolverFailures"] == serial["failures"] == 0


def test_cpu_joint_schur_ba_decreases_objective_and_preserves_gauge():
    # tests/bundle-adjustment.test.ts:31-51
    inp = perturbed()
    snapshot = json.dumps([[list(v["pose"]["R"]), list(v["pose"]["t"])] for v in inp["views"]])
    out = ob.cpu_bundle_adjust(inp, {"iterations": 25})
    d = out["diagnostics"]
    assert d["acceptedSteps"] > 0
    assert d["finalCost"] < d["initialCost"] * 0.05
    assert d["finalRmsePx"] < 0.3
    assert d["observations"] == 350
    assert json.dumps([[list(v["pose"]["R"]), list(v["pose"]["t"])] for v in inp["views"]]) == snapshot
    v0 = out["reconstruction"]["views"][0]["pose"]
    assert np.array_equal(v0["R"], inp["views"][0]["pose"]["R"]) and np.array_equal(v0["t"], inp["views"][0]["pose"]["t"])
    a = ob.camera_center(out["reconstruction"]["views"][0]["pose"])
    b = ob.camera_center(out["reconstruction"]["views"][1]["pose"])
    assert abs(np.linalg.norm(a - b) - d["baseline"]) < 1e-10


def test_cpu_zero_iterations_is_identity():
    # tests/bundle-adjustment.test.ts:52-58
    inp = perturbed()
    out = ob.cpu_bundle_adjust(inp, {"iterations": 0})
    for a, b in zip(out["reconstruction"]["landmarks"], inp["landmarks"]):
        assert np.array_equal(a["xyz"], b["xyz"])
    assert out["diagnostics"]["initialCost"] == out["diagnostics"]["finalCost"]


def test_cpu_robust_objective_keeps_outlier():
    # tests/bundle-adjustment.test.ts:59-78
    inp = perturbed()
    lm0 = dict(inp["landmarks"][0])
    obs = [dict(o) for o in lm0["observations"]]
    obs[2]["pixel"] = [obs[2]["pixel"][0] + 40, obs[2]["pixel"][1] - 20]
    lm0["observations"] = obs
    out = ob.cpu_bundle_adjust({**inp, "landmarks": [lm0] + inp["landmarks"][1:]}, {"iterations": 20, "huberPx": 1})
    assert out["diagnostics"]["finalCost"] < out["diagnostics"]["initialCost"] * 0.2
    assert out["diagnostics"]["observations"] == 350


def test_cpu_rejects_ownership_gauge_baseline_cheirality():
    # tests/bundle-adjustment.test.ts:79-111
    inp = perturbed()
    with pytest.raises(ob.RangeError, match="owned"):
        ob.cpu_bundle_adjust({**inp, "landmarks": [inp["landmarks"][0], {**inp["landmarks"][1],
                                                   "observations": inp["landmarks"][0]["observations"]}]})
    with pytest.raises(ob.RangeError, match="gauge"):
        ob.cpu_bundle_adjust(inp, {"anchorViewId": 999})
    with pytest.raises(ob.RangeError, match="baseline"):
        ob.cpu_bundle_adjust({**inp, "views": [v if i != 1 else {**v, "pose": inp["views"][0]["pose"]}
                                               for i, v in enumerate(inp["views"])]})
    with pytest.raises(ob.RangeError, match="in front"):
        ob.cpu_bundle_adjust({**inp, "landmarks": [p if i else {**p, "xyz": np.array([0.0, 0, -10])}
                                                   for i, p in enumerate(inp["landmarks"])]})


def test_cpu_gauge_with_translated_world_and_local_window():
    # tests/bundle-adjustment.test.ts:113-152
    rec, _ = scene(count=30, views=4, noise=0.1)
    D = np.array([7.0, -3, 2])
    shifted = {"views": [{**v, "pose": {"R": v["pose"]["R"], "t": np.array(
        [v["pose"]["t"][i] - v["pose"]["R"][i * 3] * D[0] - v["pose"]["R"][i * 3 + 1] * D[1]
         - v["pose"]["R"][i * 3 + 2] * D[2] for i in range(3)])}} for v in rec["views"]],
        "landmarks": [{**p, "xyz": np.asarray(p["xyz"]) + D} for p in rec["landmarks"]]}
    out = ob.cpu_bundle_adjust(shifted, {"iterations": 15, "anchorViewId": 20, "scaleViewId": 40})
    assert out["diagnostics"]["finalCost"] <= out["diagnostics"]["initialCost"]
    a = ob.camera_center(out["reconstruction"]["views"][1]["pose"])
    b = ob.camera_center(out["reconstruction"]["views"][3]["pose"])
    assert abs(np.linalg.norm(a - b) - out["diagnostics"]["baseline"]) < 1e-9
    inp = perturbed()
    local = ob.cpu_bundle_adjust(inp, {"iterations": 15, "variableViewIds": [30, 40, 50]})
    assert local["diagnostics"]["finalCost"] < local["diagnostics"]["initialCost"]
    for i in (0, 1):
        assert np.array_equal(local["reconstruction"]["views"][i]["pose"]["t"], inp["views"][i]["pose"]["t"])
    with pytest.raises(ob.RangeError, match="window"):
        ob.cpu_bundle_adjust(inp, {"variableViewIds": [10]})
    with pytest.raises(ob.RangeError, match="scale camera"):
        ob.cpu_bundle_adjust(inp, {"variableViewIds": [20]})
    with pytest.raises(ob.RangeError, match="connected observation graph"):
        ob.cpu_bundle_adjust({**inp, "landmarks": [{**p, "observations": [o for o in p["observations"] if o["viewId"] != 50]}
                                                   for p in inp["landmarks"]]})


FOCAL = {"iterations": 40, "refineSharedFocal": True, "maxCgIterations": 256, "cgRelativeTolerance": 1e-10}


def test_joint_focal_recovers_ground_truth_cpu_and_operator_agree():
    # tests/typeshade/focal.test.mjs:13-45
    jf = joint_focal_fixture()
    inp, truth = jf["input"], jf["truth"]
    expected = ob.cpu_bundle_adjust(inp, FOCAL)
    actual = ob.gpu_operator(inp, FOCAL)
    for res in (expected, actual):
        d = res["diagnostics"]
        assert d["finalCost"] < 1e-7 and d["finalRmsePx"] < 1e-4 and d["initialCost"] > 50000
        views = res["reconstruction"]["views"]
        scale = views[0]["camera"]["fx"] / inp["views"][0]["camera"]["fx"]
        assert abs(views[0]["camera"]["fx"] - truth["views"][0]["camera"]["fx"]) < 0.001
        for v, v0 in zip(views, inp["views"]):
            assert abs(v["camera"]["fx"] / v0["camera"]["fx"] - scale) < 1e-12
            assert abs(v["camera"]["fy"] / v0["camera"]["fy"] - scale) < 1e-12
            assert v["camera"]["k1"] == v0["camera"]["k1"] and v["camera"]["k2"] == v0["camera"]["k2"]
        assert np.array_equal(views[0]["pose"]["R"], inp["views"][0]["pose"]["R"])
    assert abs(actual["diagnostics"]["finalCost"] - expected["diagnostics"]["finalCost"]) < 1e-7


def test_operator_oracle_cpu_tier_cases():
    # tests/typeshade/cpu.test.mjs:533-607
    for settings in ({}, {"outlier": True}, {"shift": (7, -3, 2)}):
        inp = bundle_fixture(**settings)
        initial = bundle_metrics(inp, 1)
        shifted = "shift" in settings
        anchor, scale_view = (1, 3) if shifted else (0, 1)
        r = ob.gpu_operator(inp, {"iterations": 15, "huberPx": 1,
                                  **({"anchorViewId": 20, "scaleViewId": 40} if shifted else {})})
        actual = bundle_metrics(r["reconstruction"], 1)
        assert r["diagnostics"]["acceptedSteps"] > 0
        assert actual["cost"] < initial["cost"] * 0.05
        assert abs(actual["cost"] - r["diagnostics"]["finalCost"]) < 1e-6
        a = ob.camera_center(r["reconstruction"]["views"][anchor]["pose"])
        b = ob.camera_center(r["reconstruction"]["views"][scale_view]["pose"])
        assert abs(np.linalg.norm(a - b) - r["diagnostics"]["baseline"]) < 1e-9
        assert actual["observations"] == 160
    inp = bundle_fixture()
    rejected = ob.gpu_operator(inp, {"iterations": 1, "maxCgIterations": 1, "cgRelativeTolerance": 1e-12})
    assert rejected["diagnostics"]["acceptedSteps"] == 0 and rejected["linearSolverFailures"] > 0
