"""Joint inverse-depth bundle adjustment: the Python mirror of TypeCV's ``bundleAdjustInverseDepthGpu``
(src/sfm/depth/gpu/inverse-depth.ts:115-141) and the host steps it drives,
``inverseDepthBundleSteps`` (src/sfm/depth/inverse-depth-bundle.ts:196-565).

Each landmark becomes an anchored inverse-depth point in the chart of its first observing view
(explicit constraints add bearing-only or inverse-depth tracks).  Every Levenberg-Marquardt step
linearises all measurements on the device (``tba_linearize_inverse_depth``), builds the reduced
camera system on the host in FP64 (Huber-weighted point blocks eliminated by their 3x3 or 2x2
inverses; camera blocks of 6 parameters, 5 for a scale-free gauge's scale view, plus one log-focal
parameter per shared focal group), factors it densely or by the sparse minimum-degree Cholesky and
takes the step when the robust cost of the candidate, projected on the device, is lower.  After the
last step the undamped system gives each point's marginal covariance.

``inverse_depth_bundle_steps`` is a generator: it yields measurement jobs and receives one
linearisation (or None) per measurement.  A job with ``"purpose": "cost"`` asks for the candidate's
projections only; the reference evaluates those with its CPU ``inverseDepthJacobian``, here they go
to the device like the linearisations.
"""
from __future__ import annotations

import copy
import math
from typing import Any, Generator

import numpy as np

from .bundle import RangeError, ShadeDevice, validate_reconstruction, _safe_int
from .inverse_depth import (camera_center, initialize_inverse_depth, inverse_depth_covariance, inverse_depth_point,
                            linearize_batches, rescale_inverse_depth, update_pose, validate_pose)
from .sparse_schur import SparseSymmetric, dense_schur_factor, factor_sparse_schur, multiply_vector, positive_inverse


def _dot(a, b) -> float:
    s = 0.0
    for i in range(3):
        s += float(a[i]) * float(b[i])
    return s


def camera_blocks(model, active, scale_id, origin) -> tuple[dict[int, dict], int]:
    """cameraBlocks (inverse-depth-bundle.ts:135-177): each active view's parameter block and its
    6 x dim basis; the scale view of a scale-free gauge drops the translation along its baseline."""
    blocks: dict[int, dict] = {}
    n = 0
    for v in model["views"]:
        if v["id"] not in active:
            continue
        dim = 5 if v["id"] == scale_id else 6
        basis = [0.0] * (6 * dim)
        for i in range(3):
            basis[i * dim + i] = 1.0
        if dim == 6:
            for i in range(3, 6):
                basis[i * dim + i] = 1.0
        else:
            world = [x - origin[i] for i, x in enumerate(camera_center(v["pose"]))]
            length = math.hypot(*world)
            R = v["pose"]["R"]
            d = [_dot([R[3 * i], R[3 * i + 1], R[3 * i + 2]], world) / length for i in range(3)]
            axis = min(range(3), key=lambda a: abs(d[a]))
            u = [0.0, 0.0, 0.0]
            u[axis] = 1.0
            along = d[axis]
            for i in range(3):
                u[i] -= along * d[i]
            norm = math.hypot(*u)
            u = [x / norm for x in u]
            w = [d[1] * u[2] - d[2] * u[1], d[2] * u[0] - d[0] * u[2], d[0] * u[1] - d[1] * u[0]]
            for i in range(3):
                basis[(i + 3) * dim + 3] = u[i]
                basis[(i + 3) * dim + 4] = w[i]
        blocks[v["id"]] = {"offset": n, "dimension": dim, "basis": basis}
        n += dim
    return blocks, n


def choose_schur_solver(points, active, groups, options, parameters: int, max_factor_entries: int) -> str:
    """chooseSchurSolver (inverse-depth-bundle.ts:618-654): dense for small or well-filled camera
    graphs, sparse otherwise."""
    solver = options.get("solver")
    if solver and solver != "auto":
        return solver
    if parameters <= 96:
        return "dense"
    if parameters * parameters > max_factor_entries:
        return "sparse"
    cameras = {vid: index for index, vid in enumerate(active)}
    n = len(active) + len(groups)
    edges: set[int] = set()
    threshold = 0.35 * n * (n + 1) / 2
    focal_groups = options.get("focalGroups")
    for p in points:
        involved: dict[int, None] = {}
        for o in p["observations"]:
            c = cameras.get(o["viewId"])
            if c is not None:
                involved[c] = None
            if groups:
                involved[len(active) + groups[(focal_groups or {}).get(o["viewId"], 0)]] = None
        indices = list(involved)
        for a in range(len(indices)):
            for b in range(a, len(indices)):
                edges.add(min(indices[a], indices[b]) * n + max(indices[a], indices[b]))
        if len(edges) >= threshold:
            return "dense"
    return "sparse"


def reduce_system(eq: dict, m: int, lam: float) -> dict | None:
    """reduce (inverse-depth-bundle.ts:582-616): damp, eliminate every observable point block and
    return the reduced camera system with each block's inverse and W V^-1."""
    S = eq["A"].copy()
    b = list(eq["b"])
    points = []
    for i in range(m):
        S.add(i, i, lam * max(S.get(i, i), 1e-10))
    for block in eq["points"]:
        if block["deferred"]:
            points.append(block)
            continue
        d = block["d"]
        V = list(block["V"])
        for i in range(d):
            V[i * d + i] += lam * max(V[i * d + i], 1e-10)
        inverse = inverse_depth_covariance(V) if d == 3 else positive_inverse(V, d)
        if inverse is None:
            return None
        inverse = [float(x) for x in inverse]
        W, idx = block["W"], block["indices"]
        T = [0.0] * len(W)
        for row in range(len(idx)):
            for j in range(d):
                for k in range(d):
                    T[row * d + j] += W[row * d + k] * inverse[k * d + j]
        for row in range(len(idx)):
            i = idx[row]
            for k in range(d):
                b[i] -= T[row * d + k] * block["b"][k]
            for col in range(len(idx)):
                if i <= idx[col]:
                    for k in range(d):
                        S.add(i, idx[col], -T[col * d + k] * W[row * d + k])
        points.append({**block, "inverse": inverse, "T": T})
    return {"S": S, "b": b, "points": points}


def point_marginal(block: dict, factor) -> list[float]:
    """pointMarginal (inverse-depth-bundle.ts:669-700): V^-1 + T^T C T over the block's cameras."""
    result = list(block["inverse"])
    d, T, idx = block["d"], block["T"], block["indices"]
    if factor.storage == "dense":
        for a in range(len(idx)):
            for b in range(len(idx)):
                c = factor.covariance(idx[a], idx[b])
                for i in range(d):
                    left = T[a * d + i] * c
                    for j in range(d):
                        result[i * d + j] += left * T[b * d + j]
        return result
    for a in range(len(idx)):
        for b in range(a, len(idx)):
            c = factor.covariance(idx[a], idx[b])
            for i in range(d):
                for j in range(d):
                    value = T[a * d + i] * T[b * d + j] + (0 if a == b else T[b * d + i] * T[a * d + j])
                    result[i * d + j] += c * value
    return result


def _huber(e: float, h: float) -> float:
    return e * e if e <= h else 2 * h * e - h * h


def inverse_depth_bundle_steps(inp: dict, constraints=(), options: dict | None = None
                               ) -> Generator[dict, list, dict[str, Any]]:
    """inverseDepthBundleSteps (inverse-depth-bundle.ts:196-565)."""
    options = dict(options or {})
    inp = copy.deepcopy(inp)
    constraints = copy.deepcopy(list(constraints))
    if options.get("variableViewIds") is not None:
        options["variableViewIds"] = list(options["variableViewIds"])
    if options.get("focalGroups") is not None:
        options["focalGroups"] = dict(options["focalGroups"])
    validate_reconstruction(inp)
    views_in = inp["views"]
    iterations = options.get("iterations", 8)
    huber = options.get("huberPx", 3)
    sigma = options.get("pixelNoiseStdDevPx", 1)
    anchor_id = options.get("anchorViewId", views_in[0]["id"] if views_in else None)
    scale_id = options.get("scaleViewId")
    if scale_id is None:
        scale_id = next((v["id"] for v in views_in if v["id"] != anchor_id), None)
    limit = options.get("maxCameraParameters", 1536)
    max_schur = options.get("maxSchurEntries", 300000)
    max_factor = options.get("maxFactorEntries", 600000)
    if (not _safe_int(iterations) or iterations < 0 or iterations > 100
            or not (huber > 0 and math.isfinite(huber) and sigma > 0 and math.isfinite(sigma))
            or not _safe_int(limit) or limit < 1):
        raise RangeError("Invalid inverse-depth bundle controls")
    batch = options.get("measurementBatchSize", 1)
    if (not all(_safe_int(v) and v > 0 for v in (max_schur, max_factor, batch))
            or (options.get("solver") or "auto") not in ("auto", "dense", "sparse")):
        raise RangeError("Invalid inverse-depth sparse/batch controls")
    anchor = next((v for v in views_in if v["id"] == anchor_id), None)
    scale = next((v for v in views_in if v["id"] == scale_id), None)
    if anchor is None or scale is None or anchor_id == scale_id or not inp["landmarks"]:
        raise RangeError("Inverse-depth BA needs a connected finite map and gauge")
    origin = camera_center(anchor["pose"])
    baseline = math.hypot(*[x - origin[i] for i, x in enumerate(camera_center(scale["pose"]))])
    if not baseline > 1e-10:
        raise RangeError("Inverse-depth BA cannot initialize from pure rotation")
    connected = {anchor_id}
    for _ in range(len(views_in)):
        for p in inp["landmarks"]:
            if any(o["viewId"] in connected for o in p["observations"]):
                for o in p["observations"]:
                    connected.add(o["viewId"])
    if any(v["id"] not in connected for v in views_in):
        raise RangeError("Inverse-depth BA requires one connected finite observation graph")
    variable = options.get("variableViewIds")
    active_list = list(variable) if variable is not None else [v["id"] for v in views_in if v["id"] != anchor_id]
    active = dict.fromkeys(active_list)
    view_ids = {v["id"] for v in views_in}
    if anchor_id in active or any(i not in view_ids for i in active):
        raise RangeError("Invalid inverse-depth variable cameras")
    fixed = [v for v in views_in if v["id"] not in active]
    scale_free = len(fixed) == 1 and scale_id in active
    view_map = {v["id"]: v for v in views_in}
    ids = {p["trackId"] for p in inp["landmarks"]}
    owned = {(o["viewId"], o["featureId"]) for p in inp["landmarks"] for o in p["observations"]}
    points = []
    for p in inp["landmarks"]:
        first = p["observations"][0]
        points.append({"trackId": p["trackId"], "observations": p["observations"], "referenceViewId": first["viewId"],
                       "point": initialize_inverse_depth(view_map[first["viewId"]], first["pixel"], p["xyz"])})
    for p in constraints:
        validate_pose(p["point"]["reference"])
        params = np.asarray(p["point"]["parameters"], float)
        if p.get("directionOnly") and params[2] != 0:
            raise RangeError("Bearing-only constraints cannot assert finite inverse depth")
        if (p["trackId"] in ids or not _safe_int(p["trackId"]) or p["trackId"] < 0 or len(p["observations"]) < 2
                or params.size != 3 or not np.all(np.isfinite(params))):
            raise RangeError("Invalid inverse-depth constraint")
        seen = set()
        ids.add(p["trackId"])
        for o in p["observations"]:
            key = (o["viewId"], o["featureId"])
            if (not _safe_int(o["featureId"]) or o["featureId"] < 0 or o["viewId"] not in view_map
                    or o["viewId"] in seen or key in owned or not all(math.isfinite(x) for x in o["pixel"])):
                raise RangeError("Multiply owned/invalid inverse-depth observation")
            seen.add(o["viewId"])
            owned.add(key)
        points.append({**p, "point": {"reference": {"R": np.array(p["point"]["reference"]["R"], float).ravel(),
                                                    "t": np.array(p["point"]["reference"]["t"], float).ravel()},
                                      "parameters": params.copy()}})
    model = {"views": [{**v, "camera": dict(v["camera"]),
                        "pose": {"R": np.array(v["pose"]["R"], float).ravel(), "t": np.array(v["pose"]["t"], float).ravel()}}
                       for v in views_in],
             "landmarks": inp["landmarks"]}
    current = points
    focal_groups = options.get("focalGroups")
    groups: dict[int, int] = {}
    if options.get("refineSharedFocal"):
        for v in model["views"]:
            g = focal_groups.get(v["id"]) if focal_groups is not None else 0
            if g is None or not _safe_int(g) or g < 0:
                raise RangeError("Invalid inverse-depth focal groups")
            if g not in groups:
                groups[g] = len(groups)
    lam = 1e-3
    accepted_steps = 0
    initial_cost = final_cost = 0.0

    def job(views, pts, purpose="linearize"):
        by_id = {v["id"]: v for v in views}
        out = {"measurements": [{"view": by_id[o["viewId"]], "point": p["point"]} for p in pts
                                for o in p["observations"]]}
        if purpose != "linearize":
            out["purpose"] = purpose
        return out

    _, planned_n = camera_blocks(model, active, scale_id if scale_free else None, origin)
    planned = planned_n + len(groups)
    if planned > limit:
        raise RangeError("Inverse-depth camera parameter budget exceeded")
    linear_solver = choose_schur_solver(current, list(active), groups, options, planned, max_factor)
    if (planned ** 2 if linear_solver == "dense" else planned) > max_factor:
        raise RangeError("Schur factor budget exceeded before measurement allocation")

    def factorize(S):
        return factor_sparse_schur(S, max_factor) if linear_solver == "sparse" else dense_schur_factor(S, max_factor)

    group_of = (lambda vid: groups[(focal_groups or {}).get(vid, 0)]) if groups else None
    last = None
    for iteration in range(iterations + 1):
        blocks, n_cam = camera_blocks(model, active, scale_id if scale_free else None, origin)
        m = n_cam + len(groups)
        if m > limit:
            raise RangeError("Inverse-depth camera parameter budget exceeded")
        measurements = yield job(model["views"], current)
        A = SparseSymmetric(m, max_schur, linear_solver == "dense")
        bc = [0.0] * m
        point_blocks = []
        cross = [0.0] * (3 * m)
        touched = bytearray(m)
        row_index = 0
        cost = 0.0
        w2 = sigma ** 2
        for p in current:
            d = 2 if p.get("directionOnly") else 3
            V = [0.0] * (d * d)
            bp = [0.0] * d
            first_row = row_index
            for o in p["observations"]:
                j = measurements[row_index]
                row_index += 1
                if j is None:
                    raise RangeError("Inverse-depth bundle projection is behind a camera")
                pt = j["point"]
                res = (j["pixel"][0] - o["pixel"][0], j["pixel"][1] - o["pixel"][1])
                norm = math.hypot(*res)
                weight = (1 if norm <= huber else huber / norm) / w2
                for row in range(2):
                    for k in range(d):
                        bp[k] -= weight * pt[3 * row + k] * res[row]
                        for l in range(d):
                            V[k * d + l] += weight * pt[3 * row + k] * pt[3 * row + l]
            observable = inverse_depth_covariance(V) if d == 3 else positive_inverse(V, d)
            active_indices: list[int] = []
            if observable is not None:
                at = first_row
                for o in p["observations"]:
                    j = measurements[at]
                    at += 1
                    pt, pose_j, focal_j = j["point"], j["pose"], j["focal"]
                    res = (j["pixel"][0] - o["pixel"][0], j["pixel"][1] - o["pixel"][1])
                    norm = math.hypot(*res)
                    weight = (1 if norm <= huber else huber / norm) / w2
                    camera = blocks.get(o["viewId"])
                    cost += _huber(norm, huber)
                    for row in range(2):
                        columns, values = [], []
                        if camera is not None:
                            dim, basis, offset = camera["dimension"], camera["basis"], camera["offset"]
                            for k in range(dim):
                                value = 0.0
                                for l in range(6):
                                    value += pose_j[6 * row + l] * basis[l * dim + k]
                                columns.append(offset + k)
                                values.append(value)
                        if groups:
                            columns.append(n_cam + group_of(o["viewId"]))
                            values.append(focal_j[row])
                        for column in range(len(columns)):
                            i, a = columns[column], values[column]
                            if not touched[i]:
                                touched[i] = 1
                                active_indices.append(i)
                            for k in range(d):
                                cross[3 * i + k] += weight * a * pt[3 * row + k]
                            bc[i] -= weight * a * res[row]
                            for other in range(len(columns)):
                                k = columns[other]
                                if i <= k:
                                    A.add(i, k, weight * a * values[other])
            indices = sorted(i for i in active_indices if any(cross[3 * i + k] != 0 for k in range(d)))
            W = [cross[3 * i + k] for i in indices for k in range(d)]
            for i in active_indices:
                touched[i] = 0
                cross[3 * i] = cross[3 * i + 1] = cross[3 * i + 2] = 0.0
            point_blocks.append({"V": V, "b": bp, "W": W, "d": d, "indices": indices, "deferred": observable is None})
        eq = {"A": A, "b": bc, "points": point_blocks, "cost": cost}
        last = (eq, m)
        if not iteration:
            initial_cost = cost
        final_cost = cost
        if iteration == iterations:
            break
        reduced = reduce_system(eq, m, lam)
        if reduced is None:
            lam *= 10
            continue
        factor = factorize(reduced["S"])
        if factor is None:
            lam *= 10
            continue
        delta = factor.solve(reduced["b"])
        next_views = []
        for v in model["views"]:
            c = blocks.get(v["id"])
            step = [0.0] * 6
            if c is not None:
                dim, basis, offset = c["dimension"], c["basis"], c["offset"]
                for i in range(6):
                    for k in range(dim):
                        step[i] += basis[i * dim + k] * delta[offset + k]
            focal = math.exp(delta[n_cam + group_of(v["id"])]) if groups else 1
            next_views.append({**v, "camera": {**v["camera"], "fx": v["camera"]["fx"] * focal,
                                               "fy": v["camera"]["fy"] * focal},
                               "pose": update_pose(v["pose"], step) if c is not None else v["pose"]})
        next_points = []
        for i, p in enumerate(current):
            block = reduced["points"][i]
            if block["deferred"]:
                next_points.append(p)
                continue
            d = block["d"]
            rhs = list(block["b"])
            for row in range(len(block["indices"])):
                for j in range(d):
                    rhs[j] -= block["W"][row * d + j] * delta[block["indices"][row]]
            dp = multiply_vector(block["inverse"], rhs, d)
            params = np.array([x + (dp[k] if k < d else 0) for k, x in enumerate(p["point"]["parameters"])])
            next_points.append({**p, "point": {**p["point"], "parameters": params}})
        candidate_views = next_views
        if scale_free:
            moved = next(v for v in next_views if v["id"] == scale_id)
            length = math.hypot(*[x - origin[i] for i, x in enumerate(camera_center(moved["pose"]))])
            s = baseline / length if length else math.inf
            if not (s > 0 and math.isfinite(s)):
                lam *= 10
                continue
            candidate_views = []
            for v in next_views:
                if v["id"] == anchor_id:
                    candidate_views.append(v)
                    continue
                R = v["pose"]["R"]
                ro = [_dot([R[3 * i], R[3 * i + 1], R[3 * i + 2]], origin) for i in range(3)]
                candidate_views.append({**v, "pose": {"R": R, "t": np.array([s * float(t) + (s - 1) * ro[i]
                                                                            for i, t in enumerate(v["pose"]["t"])])}})
            next_points = [{**p, "point": rescale_inverse_depth(p["point"], s, origin)} for p in next_points]
        # The candidate's robust cost over the points that were not deferred, projected on the device.
        live = [p for i, p in enumerate(next_points) if not reduced["points"][i]["deferred"]]
        rows = yield job(candidate_views, live, "cost")
        next_cost, at = 0.0, 0
        for p in live:
            for o in p["observations"]:
                j = rows[at]
                at += 1
                if j is None:
                    next_cost = math.inf
                    break
                next_cost += _huber(math.hypot(j["pixel"][0] - o["pixel"][0], j["pixel"][1] - o["pixel"][1]), huber)
            if next_cost == math.inf:
                break
        if any(not p["point"]["parameters"][2] > 0 for p in next_points[:len(inp["landmarks"])]):
            next_cost = math.inf
        if next_cost < cost:
            model = {**model, "views": candidate_views}
            current = next_points
            lam = max(1e-12, lam / 3)
            accepted_steps += 1
        else:
            lam *= 10
    eq, m = last
    undamped = reduce_system(eq, m, 0)
    camera_factor = factorize(undamped["S"]) if undamped is not None else None
    estimates = []
    for index, p in enumerate(current):
        block = undamped["points"][index] if undamped is not None else None
        entry = dict(p)
        if block is not None and not block["deferred"] and camera_factor is not None:
            marginal = point_marginal(block, camera_factor)
            if block["d"] == 3:
                entry["covariance"] = np.array(marginal)
                entry["bearingCovariance"] = np.array([marginal[0], marginal[1], marginal[3], marginal[4]])
            else:
                entry["bearingCovariance"] = np.array(marginal)
        if eq["points"][index]["deferred"]:
            entry["informationDeferred"] = True
        estimates.append(entry)
    landmarks = []
    for i, p in enumerate(inp["landmarks"]):
        if estimates[i].get("informationDeferred"):
            continue
        landmarks.append({**p, "xyz": inverse_depth_point(estimates[i]["point"])})
    if any(p["xyz"] is None for p in landmarks):
        raise RangeError("Joint BA invalidated a finite input point")
    deferred = [eq["points"][i]["deferred"] for i in range(len(current))]
    return {
        "reconstruction": {"views": model["views"], "landmarks": landmarks},
        "estimates": estimates,
        "uncertainty": {"poses": "joint" if len(fixed) == 1 else "fixed-exterior",
                        "intrinsics": "joint-focal" if groups else "fixed", "anchorViewId": anchor_id,
                        "scaleViewId": scale_id, "observable": camera_factor is not None,
                        "approximation": "local-robust-Gaussian"},
        "diagnostics": {
            "initialCost": initial_cost, "finalCost": final_cost, "acceptedSteps": accepted_steps,
            "observations": sum(0 if deferred[i] else len(p["observations"]) for i, p in enumerate(current)),
            "cameraParameters": m, "backend": "cpu", "linearSolver": linear_solver,
            "schurEntries": undamped["S"].entries if undamped is not None else 0,
            "factorEntries": camera_factor.entries if camera_factor is not None else 0,
            "cameraCovarianceEntries": camera_factor.selected_entries if camera_factor is not None else 0,
            "pointCrossEntries": sum(len(b["W"]) for b in eq["points"]),
            "denseEquivalentCrossEntries": sum(m * b["d"] for b in eq["points"]),
            "inputObservations": sum(len(p["observations"]) for p in current),
            "deferredTrackIds": [p["trackId"] for i, p in enumerate(current) if deferred[i]],
        },
    }


def drive(steps: Generator, answer) -> dict[str, Any]:
    """Run a steps generator to its result, answering each job with ``answer(job)``."""
    try:
        job = next(steps)
        while True:
            job = steps.send(answer(job))
    except StopIteration as stop:
        return stop.value


def bundle_adjust_inverse_depth_gpu(device: ShadeDevice, model: dict, constraints=(),
                                    options: dict | None = None) -> dict[str, Any]:
    """bundleAdjustInverseDepthGpu (src/sfm/depth/gpu/inverse-depth.ts:115-141): device
    linearisations and projections, host FP64 reduced solve and covariance."""
    options = options or {}
    requested = options.get("measurementBatchSize")
    stats = {"batches": 0, "batchSize": 0, "costBatches": 0, "launches": 0, "device_ms": 0.0}

    def answer(job):
        out = linearize_batches(device, job, requested)
        if job.get("purpose") == "cost":
            stats["costBatches"] += out["batches"]
        else:
            stats["batches"] += out["batches"]
            stats["batchSize"] = max(stats["batchSize"], out["batchSize"])
        for rep in out["reports"]:
            stats["launches"] += rep["kernel_launches"]
            stats["device_ms"] += rep["upload_ms"] + rep["evaluate_ms"] + rep["download_ms"]
        return out["rows"]

    result = drive(inverse_depth_bundle_steps(model, constraints, options), answer)
    result["diagnostics"] = {**result["diagnostics"], "backend": f"{device.backend}-jacobians/host-f64-Schur",
                             "measurementBatches": stats["batches"], "measurementBatchSize": stats["batchSize"],
                             "costBatches": stats["costBatches"], "kernelLaunches": stats["launches"],
                             "deviceMs": stats["device_ms"]}
    return result
