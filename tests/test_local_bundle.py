"""Local and partitioned problems of a map (typecv_b200/local_bundle.py) on the CPU.

Restates the reference's tests of its local-bundle planning (tests/local-bundle.test.ts:10-150 and
tests/bundle-partitions.test.ts:13-102) on the same fixtures (tests/scene.ts, restated in
reference_cases.scene): window extraction and its fallbacks, connected-component planning and
deferral, and what each merge takes from a result.
"""
import copy

import numpy as np
import pytest

from reference_cases import f64, scene, update_pose
from typecv_b200 import local_bundle as L
from typecv_b200.bundle import validate_reconstruction


def local_scene():
    """localScene (tests/local-bundle.test.ts:10-30)."""
    reconstruction, rng = scene(count=48, views=7, noise=0.1)
    variable = {40, 50}
    views = []
    for v in reconstruction["views"]:
        if v["id"] in variable:
            R, t = update_pose(v["pose"]["R"], v["pose"]["t"], [0.001, -0.002, 0.001, 0.02, -0.01, 0.01])
            views.append({**v, "pose": {"R": f64(R), "t": f64(t)}})
        else:
            views.append(v)
    landmarks = []
    for i, p in enumerate(reconstruction["landmarks"]):
        xyz = f64([x + (rng() - 0.5) * 0.08 for x in p["xyz"]]) if i < 24 else p["xyz"]
        keep = [20, 30, 40, 50] if i < 24 else [10, 20, 60, 70]
        landmarks.append({**p, "xyz": xyz, "observations": [o for o in p["observations"] if o["viewId"] in keep]})
    return {"views": views, "landmarks": landmarks}


def disconnected():
    """disconnected (tests/bundle-partitions.test.ts:13-34), its model only."""
    reconstruction, _ = scene(count=48, views=7, noise=0.15)
    return {"views": reconstruction["views"],
            "landmarks": [{**p, "xyz": f64([x + 0.015 for x in p["xyz"]]),
                           "observations": [o for o in p["observations"]
                                            if o["viewId"] in ([10, 20, 30] if i < 24 else [40, 50, 60])]}
                          for i, p in enumerate(reconstruction["landmarks"])]}


def test_local_extraction_keeps_selected_observations_and_connected_cameras():
    inp = local_scene()
    snapshot = copy.deepcopy(inp)
    local = L.extract_local_bundle(inp, [40, 50])
    assert local is not None
    validate_reconstruction(local["reconstruction"])
    assert [v["id"] for v in local["reconstruction"]["views"]] == [20, 30, 40, 50]
    assert len(local["reconstruction"]["landmarks"]) == 24
    assert local["anchorViewId"] == 20 and local["scaleViewId"] == 30
    assert local["anchorViewId"] not in local["variableViewIds"]
    assert local["scaleViewId"] not in local["variableViewIds"]
    for p in local["reconstruction"]["landmarks"]:
        assert p is inp["landmarks"][p["trackId"]]
        assert len(p["observations"]) == 4
    assert sum(len(p["observations"]) for p in local["reconstruction"]["landmarks"]) == 96
    assert repr(inp) == repr(snapshot)


def test_merging_takes_only_selected_coordinates_and_variable_poses():
    inp = local_scene()
    local = L.extract_local_bundle(inp, [40, 50])
    identity = {"R": f64([1, 0, 0, 0, 1, 0, 0, 0, 1]), "t": f64([0, 0, 0])}
    changed = {"views": [{**v, "camera": {**v["camera"], "fx": v["camera"]["fx"] * 2}, "pose": identity}
                         for v in inp["views"]],
               "landmarks": [{**p, "xyz": f64([1, 2, 3]), "observations": []} for p in inp["landmarks"]]}
    merged = L.merge_local_bundle(inp, local, changed)
    for old, cur in zip(inp["views"], merged["views"]):
        assert cur["camera"] is old["camera"]
        assert cur["pose"] is (identity if old["id"] in (40, 50) else old["pose"])
    for i, (old, cur) in enumerate(zip(inp["landmarks"], merged["landmarks"])):
        assert cur["observations"] is old["observations"]
        assert np.array_equal(cur["xyz"], [1, 2, 3] if i < 24 else old["xyz"])


def test_unsafe_windows_fall_back():
    inp = local_scene()
    assert L.extract_local_bundle(inp, []) is None
    assert L.extract_local_bundle(inp, [40, 40]) is None
    assert L.extract_local_bundle(inp, [40, 999]) is None
    ids = [v["id"] for v in inp["views"]]
    assert L.extract_local_bundle(inp, ids[1:]) is None
    assert L.extract_local_bundle(inp, ids) is None
    coincident = {**inp, "views": [{**v, "pose": inp["views"][1]["pose"]} if v["id"] == 30 else v
                                   for v in inp["views"]]}
    assert L.extract_local_bundle(coincident, [40, 50]) is None
    split = {**inp, "landmarks": [{**p, "observations": [
        o for o in p["observations"]
        if (o["viewId"] in (20, 40) if i < 12 else o["viewId"] in (30, 50) if i < 24 else True)]}
        for i, p in enumerate(inp["landmarks"])]}
    validate_reconstruction(split)
    assert L.extract_local_bundle(split, [40, 50]) is None


def test_connected_problem_is_planned_unchanged():
    reconstruction, _ = scene(count=24, views=3)
    options = {"iterations": 2, "refineSharedFocal": True}
    plan = L.plan_connected_bundles(reconstruction, options)
    assert "partition" not in plan
    assert len(plan["problems"]) == 1
    assert plan["problems"][0]["reconstruction"] is reconstruction
    assert plan["problems"][0]["options"] is options


def test_disconnected_components_get_their_own_gauges():
    model = disconnected()
    plan = L.plan_connected_bundles(model, {"iterations": 8, "anchorViewId": 10, "scaleViewId": 20,
                                            "refineSharedFocal": True})
    part = plan["partition"]
    assert part["components"] == [[10, 20, 30], [40, 50, 60], [70]]
    assert part["deferredViewIds"] == [70]
    assert part["sharedFocalDeferred"] is True
    assert len(plan["problems"]) == 2
    for p in plan["problems"]:
        o = p["options"]
        assert o["refineSharedFocal"] is False
        assert o["anchorViewId"] not in o["variableViewIds"] and o["scaleViewId"] not in o["variableViewIds"]
    merged = L.merge_bundle_refinements(model, [p["reconstruction"] for p in plan["problems"]])
    assert len(merged["views"]) == 7 and len(merged["landmarks"]) == 48
    assert merged["views"][6] is model["views"][6]


def test_windows_without_two_fixed_cameras_and_collapsed_components_are_deferred():
    model = disconnected()
    local = L.plan_connected_bundles(model, {"variableViewIds": [30, 40, 50, 60]})
    assert len(local["problems"]) == 1
    assert local["partition"]["deferredViewIds"] == [40, 50, 60, 70]
    collapsed = {**model, "views": [{**v, "pose": model["views"][3]["pose"]} if v["id"] in (40, 50, 60) else v
                                    for v in model["views"]]}
    plan = L.plan_connected_bundles(collapsed, {})
    assert len(plan["problems"]) == 1
    assert plan["partition"]["deferredViewIds"] == [40, 50, 60, 70]
