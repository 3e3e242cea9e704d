"""Local and partitioned adjustments through the batched solver (typecv_b200/local_bundle.py).

The reference solves each connected component of a window with its own `bundleAdjustGpu` call
(src/sfm/mapper/mapper.ts:886-905); here the components go to the device in one batched launch.
Each result must equal the one-call result, and the reference's own assertions on the merged map
(tests/bundle-partitions.test.ts:36-86, tests/local-bundle.test.ts:60-98) must hold.
"""
import numpy as np
import pytest

import typecv_b200 as tb
from oracle import bundle_adjust as ob
from test_local_bundle import disconnected, local_scene
from typecv_b200 import local_bundle as L
from typecv_b200.bundle import validate_reconstruction

pytestmark = pytest.mark.gpu

COST_REL = 1e-9


@pytest.fixture(scope="module")
def device():
    dev = tb.ShadeDevice.open(0)
    yield dev
    dev.close()


def huber_cost(model, h=2.0):
    views = {v["id"]: v for v in model["views"]}
    total = 0.0
    for p in model["landmarks"]:
        X = np.asarray(p["xyz"], float)
        for o in p["observations"]:
            v = views[o["viewId"]]
            R = np.asarray(v["pose"]["R"], float).reshape(3, 3)
            q = R @ X + np.asarray(v["pose"]["t"], float)
            k = v["camera"]
            x, y = q[0] / q[2], q[1] / q[2]
            r2 = x * x + y * y
            d = 1 + (k.get("k1") or 0) * r2 + (k.get("k2") or 0) * r2 * r2
            e = np.hypot(k["fx"] * x * d + k["cx"] - o["pixel"][0], k["fy"] * y * d + k["cy"] - o["pixel"][1])
            total += e * e if e <= h else 2 * h * e - h * h
    return total


def test_components_in_one_launch_match_one_call_each(device):
    model = disconnected()
    plan = L.plan_connected_bundles(model, {"iterations": 8, "anchorViewId": 10, "scaleViewId": 20,
                                            "refineSharedFocal": True})
    many = L.bundle_adjust_gpu_many(device, [(p["reconstruction"], p["options"]) for p in plan["problems"]])
    assert len(many) == 2
    for p, r in zip(plan["problems"], many):
        one = tb.bundle_adjust_gpu(device, p["reconstruction"], p["options"])
        assert r["execution"]["report"]["batched"] == 2
        d, e = r["diagnostics"], one["diagnostics"]
        assert abs(d["finalCost"] - e["finalCost"]) <= COST_REL * e["finalCost"]
        # The last step of a converged solve changes the cost by about the stall threshold, where the
        # summation order of the two engines can decide whether it is taken.
        assert abs(d["acceptedSteps"] - e["acceptedSteps"]) <= 1
        assert d["finalCost"] < d["initialCost"]
        for a, b in zip(r["reconstruction"]["views"], one["reconstruction"]["views"]):
            assert np.max(np.abs(np.asarray(a["pose"]["t"]) - np.asarray(b["pose"]["t"]))) < 1e-9
    merged = L.merge_bundle_refinements(model, [r["reconstruction"] for r in many])
    assert len(merged["views"]) == 7 and len(merged["landmarks"]) == 48
    assert merged["views"][6] is model["views"][6]
    by_id = {v["id"]: v for v in model["views"]}
    for v in merged["views"]:
        if v["id"] in plan["partition"]["fixedViewIds"]:
            assert np.array_equal(v["pose"]["R"], by_id[v["id"]]["pose"]["R"])
            assert np.array_equal(v["pose"]["t"], by_id[v["id"]]["pose"]["t"])
        assert v["camera"] == by_id[v["id"]]["camera"]
    for a, b in zip(merged["landmarks"], model["landmarks"]):
        assert a["observations"] is b["observations"]


def test_local_adjustment_improves_the_window_and_keeps_the_rest(device):
    inp = local_scene()
    options = {"iterations": 20, "huberPx": 2, "cgRelativeTolerance": 1e-12, "maxCgIterations": 256}
    out = L.adjust_local(device, inp, [40, 50], options)
    merged = out["reconstruction"]
    validate_reconstruction(merged)
    assert len(out["results"]) == 1
    res = out["results"][0]["diagnostics"]
    assert res["acceptedSteps"] > 0 and res["finalCost"] < res["initialCost"]
    for old, new in zip(inp["views"], merged["views"]):
        assert new["camera"] is old["camera"]
        if old["id"] not in (40, 50):
            assert new is old
    for i, (old, new) in enumerate(zip(inp["landmarks"], merged["landmarks"])):
        assert new["observations"] is old["observations"]
        if i >= 24:
            assert new is old
    assert huber_cost(merged) <= huber_cost(inp)
    # The same window through the reference's CPU bundle adjustment (exact reduced solve).
    local = L.extract_local_bundle(inp, [40, 50])
    want = ob.cpu_bundle_adjust(local["reconstruction"], {
        "iterations": 20, "huberPx": 2, "variableViewIds": local["variableViewIds"],
        "anchorViewId": local["anchorViewId"], "scaleViewId": local["scaleViewId"]})
    assert abs(res["finalCost"] - want["diagnostics"]["finalCost"]) <= COST_REL * want["diagnostics"]["finalCost"]
