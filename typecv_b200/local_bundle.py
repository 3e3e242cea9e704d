"""Local and partitioned bundle adjustments of a map, solved together in one batched launch.

The reference's mapper adjusts a window of recently registered cameras (`adjust`,
src/sfm/mapper/mapper.ts:859-925): it extracts the window's local problem
(`extractLocalBundle`), splits the problem into its connected observation components
(`planConnectedBundles`), runs one `bundleAdjustGpu` call per component and merges the results
back (`mergeBundleRefinements`, `mergeLocalBundle`; src/sfm/bundle/local-bundle.ts:17-208).
This module restates those four functions over the same object model and replaces the per-component
calls by ``bundle_adjust_gpu_many``: every problem is prepared exactly as ``bundle_adjust_gpu``
prepares it (the reference host's validation, packing and control block), problems that share
their solver options go to the device in one ``tba_batch_adjust`` launch, and each result is read
exactly as ``bundle_adjust_gpu`` reads it.  A problem the batched solver does not take (bearings,
more cameras than its on-chip limit) falls back to its own ``bundle_adjust_gpu`` call.
"""
from __future__ import annotations

import math
from typing import Any

import numpy as np

from . import _lib
from .batch import PackedProblem, batch_adjust, max_cameras
from .bundle import ShadeDevice, camera_center_of, finish_bundle, prepare_bundle, solve_packed


def _root(parent: dict, v: int) -> int:
    r = v
    while parent[r] != r:
        r = parent[r]
    while v != r:  # path compression, as the reference's union-find
        parent[v], v = r, parent[v]
    return r


def _farthest_pair(ids, by_id, floor):
    """The pair of views whose camera centres are farthest apart (first found on ties), and that
    distance, over distances above `floor`."""
    best, pair = floor, None
    centres = [camera_center_of(by_id[i]["pose"]) for i in ids]
    for a in range(len(ids)):
        for b in range(a + 1, len(ids)):
            d = math.hypot(*(centres[a][k] - centres[b][k] for k in range(3)))
            if d > best:
                best, pair = d, (a, b)
    return pair, best


def plan_connected_bundles(model: dict, options: dict) -> dict:
    """planConnectedBundles (local-bundle.ts:17-112): one problem per connected component of the
    observation graph, each with its farthest pair of fixed ("boundary") cameras as the gauge;
    components without points or without a usable gauge are deferred."""
    parent = {v["id"]: v["id"] for v in model["views"]}
    for p in model["landmarks"]:
        first = _root(parent, p["observations"][0]["viewId"])
        for o in p["observations"]:
            parent[_root(parent, o["viewId"])] = first
    groups: dict[int, list[int]] = {}
    for v in model["views"]:
        groups.setdefault(_root(parent, v["id"]), []).append(v["id"])
    if len(groups) == 1:
        return {"problems": [{"reconstruction": model, "options": options}]}
    points: dict[int, list] = {}
    for p in model["landmarks"]:
        points.setdefault(_root(parent, p["observations"][0]["viewId"]), []).append(p)
    by_id = {v["id"]: v for v in model["views"]}
    variable = set(options["variableViewIds"]) if options.get("variableViewIds") else None
    problems, fixed, deferred = [], [], []
    for r, ids in groups.items():
        landmarks = points.get(r, [])
        boundary = [i for i in ids if not (variable and i in variable)]
        pair, _ = _farthest_pair(boundary, by_id, 1e-10)
        if not landmarks or pair is None:
            deferred.extend(ids)
            continue
        anchor, scale = boundary[pair[0]], boundary[pair[1]]
        fixed.extend(i for i in ids if i == anchor or i == scale or (variable and i not in variable))
        problems.append({
            "reconstruction": {"views": [by_id[i] for i in ids], "landmarks": landmarks},
            "options": {**options, "anchorViewId": anchor, "scaleViewId": scale,
                        "variableViewIds": [i for i in ids if i != anchor and i != scale
                                            and (not variable or i in variable)],
                        "refineSharedFocal": False, "focalGroups": None},
        })
    return {"problems": problems,
            "partition": {"components": list(groups.values()), "fixedViewIds": fixed, "deferredViewIds": deferred,
                          "sharedFocalDeferred": bool(options.get("refineSharedFocal"))}}


def merge_bundle_refinements(model: dict, refined: list[dict]) -> dict:
    """mergeBundleRefinements (local-bundle.ts:114-125): solved values replace their originals;
    isolated or deferred cameras and unrelated points stay."""
    views = {v["id"]: v for m in refined for v in m["views"]}
    points = {p["trackId"]: p for m in refined for p in m["landmarks"]}
    return {"views": [views.get(v["id"], v) for v in model["views"]],
            "landmarks": [points.get(p["trackId"], p) for p in model["landmarks"]]}


def extract_local_bundle(model: dict, variable_view_ids: list[int]) -> dict | None:
    """extractLocalBundle (local-bundle.ts:131-185): the landmarks seen by a variable camera with
    every one of their observations, the cameras observing them, and as gauge the farthest pair of
    the fixed cameras among them.  None when the window has no fixed, connected, non-degenerate
    gauge."""
    variable = set(variable_view_ids)
    if not variable or len(variable) != len(variable_view_ids):
        return None
    landmarks = [p for p in model["landmarks"] if any(o["viewId"] in variable for o in p["observations"])]
    neighbors: dict[int, list[int]] = {}
    for p in landmarks:
        first = p["observations"][0]["viewId"]
        for o in p["observations"]:
            neighbors.setdefault(o["viewId"], [])
            if o["viewId"] != first:
                neighbors[o["viewId"]].append(first)
                neighbors[first].append(o["viewId"])
    if any(i not in neighbors for i in variable_view_ids):
        return None
    views = [v for v in model["views"] if v["id"] in neighbors]
    boundary = [v for v in views if v["id"] not in variable]
    if len(views) != len(neighbors) or len(boundary) < 2:
        return None
    by_id = {v["id"]: v for v in boundary}
    pair, baseline = _farthest_pair([v["id"] for v in boundary], by_id, 0.0)
    if pair is None or not baseline > 1e-10:
        return None
    anchor = boundary[pair[0]]["id"]
    connected, pending = {anchor}, [anchor]
    i = 0
    while i < len(pending):
        for j in neighbors[pending[i]]:
            if j not in connected:
                connected.add(j)
                pending.append(j)
        i += 1
    if len(connected) != len(views):
        return None
    return {"reconstruction": {"views": views, "landmarks": landmarks}, "variableViewIds": list(variable_view_ids),
            "anchorViewId": anchor, "scaleViewId": boundary[pair[1]]["id"]}


def merge_local_bundle(model: dict, problem: dict, refined: dict) -> dict:
    """mergeLocalBundle (local-bundle.ts:188-208): the variable cameras' poses and the selected
    landmarks' coordinates from the local result; everything else, and every observation, as it was."""
    variable = set(problem["variableViewIds"])
    selected = {p["trackId"] for p in problem["reconstruction"]["landmarks"]}
    views = {v["id"]: v for v in refined["views"]}
    points = {p["trackId"]: p for p in refined["landmarks"] if p["trackId"] in selected}
    return {"views": [{**v, "pose": views[v["id"]]["pose"]} if v["id"] in variable else v for v in model["views"]],
            "landmarks": [{**p, "xyz": points[p["trackId"]]["xyz"]} if p["trackId"] in points else p
                          for p in model["landmarks"]]}


def _batch_key(prepared: dict) -> tuple:
    c = prepared["control"]
    return (c.iterations, c.max_cg, c.shared_focal, c.precision, c.huber, c.cg_tolerance, c.stall_tolerance)


def bundle_adjust_gpu_many(device: ShadeDevice, problems: list[tuple[dict, dict | None]], *,
                           precision: str = "fp64", schedule: int = 0) -> list[dict[str, Any]]:
    """``bundle_adjust_gpu`` for every (input, options) pair, in as few launches as possible:
    problems with the same solver options share one batched launch.  Results in input order."""
    prepared = [prepare_bundle(inp, opts, precision=precision) for inp, opts in problems]
    results: list[dict | None] = [None] * len(prepared)
    limit = max_cameras()
    groups: dict[tuple, list[int]] = {}
    for k, pr in enumerate(prepared):
        if pr["control"].directional_points == 0 and pr["C"] <= limit:
            groups.setdefault(_batch_key(pr), []).append(k)
        else:
            values, report = solve_packed(device, pr["control"], pr["scene"], pr["index"])
            results[k] = finish_bundle(values, report, pr)
    for key, members in groups.items():
        c = prepared[members[0]]["control"]
        packed = [PackedProblem(prepared[k]["C"], prepared[k]["P"], prepared[k]["M"], prepared[k]["scene"],
                                prepared[k]["index"], prepared[k]["control"].anchor,
                                prepared[k]["control"].scale_view) for k in members]
        records, report = batch_adjust(device, packed, iterations=c.iterations, max_cg=c.max_cg,
                                       shared_focal=bool(c.shared_focal),
                                       precision="mixed" if c.precision == _lib.TBA_PRECISION_MIXED else "fp64",
                                       huber=c.huber, tolerance=c.cg_tolerance, stall=c.stall_tolerance,
                                       schedule=schedule)
        for k, rec in zip(members, records):
            results[k] = finish_bundle(np.asarray(rec), {**report, "batched": len(members)}, prepared[k])
    return results


def adjust_local(device: ShadeDevice, model: dict, window: list[int], options: dict, *,
                 precision: str = "fp64") -> dict:
    """One local adjustment of the mapper (`adjust` with a local window, mapper.ts:866-908): the
    window's local problem, its connected components solved in one batched launch, the results
    merged back into the map.  Returns {"reconstruction", "partition", "results"}; when the window
    has no usable local problem, the whole map is planned instead, as the reference does."""
    subset = extract_local_bundle(model, window)
    problem = subset["reconstruction"] if subset else model
    opts = {**options, "variableViewIds": window}
    if subset:
        opts["anchorViewId"] = subset["anchorViewId"]
        opts["scaleViewId"] = subset["scaleViewId"]
    plan = plan_connected_bundles(problem, opts)
    results = bundle_adjust_gpu_many(device, [(p["reconstruction"], p["options"]) for p in plan["problems"]],
                                     precision=precision)
    refinements = [r["reconstruction"] for r in results]
    if not refinements:
        return {"reconstruction": model, "partition": plan.get("partition"), "results": []}
    solved = merge_bundle_refinements(problem, refinements) if plan.get("partition") else refinements[0]
    refined = merge_local_bundle(model, subset, solved) if subset else solved
    return {"reconstruction": refined, "partition": plan.get("partition"), "results": results}
