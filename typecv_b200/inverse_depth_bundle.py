"""Joint inverse-depth bundle adjustment: the Python mirror of TypeCV's ``bundleAdjustInverseDepthGpu``
(src/sfm/depth/gpu/inverse-depth.ts:115-141) and the host steps it drives,
``inverseDepthBundleSteps`` (src/sfm/depth/inverse-depth-bundle.ts:196-565).

Each landmark becomes an anchored inverse-depth point in the chart of its first observing view
(explicit constraints add bearing-only or inverse-depth tracks).  Every Levenberg-Marquardt step
linearises all measurements on the device (``tba_linearize_inverse_depth``), builds the reduced
camera system on the host in FP64 (Huber-weighted point blocks eliminated by their 3x3 or 2x2
inverses; camera blocks of 6 parameters, 5 for a scale-free gauge's scale view, plus one log-focal
parameter per shared focal group), factors it and takes the step when the robust cost of the
candidate, projected on the device, is lower.  After the last step the undamped system gives each
point's marginal covariance.

The host work is array-wise rather than one measurement at a time.  The point blocks are segment
sums over each point's measurements; the camera system is a dense matrix of at most
``maxCameraParameters`` unknowns with the reference's sparsity pattern kept beside it (its entry
counts and budget errors); the point elimination scatters each point's block of camera columns,
in chunks of points with similar column counts.  The factor is the Cholesky factor of the
diagonally equilibrated system with the reference's pivot floor (1e-10): in the natural order for
the dense solver, and for the sparse solver in the order of the reference's greedy minimum-degree
elimination, which is run on the pattern for that order, its fill counts and its budgets — so the
pivots tested are the sparse factor's.  The camera covariance is the factor's inverse; the
reference's selected inverse holds the same values on the factor's pattern.

``inverse_depth_bundle_steps`` is a generator: it yields measurement jobs ({"rows": n x 34 packed
rows, "measurements": the same as records}) and receives one linearisation per measurement (an
n x 23 array, or a list of records / None).  A job with ``"purpose": "cost"`` asks for the
candidate's projections only; the reference evaluates those with its CPU ``inverseDepthJacobian``,
here they go to the device like the linearisations.
"""
from __future__ import annotations

import math
from typing import Any, Generator

import numpy as np

from .bundle import RangeError, ShadeDevice, _safe_int, validate_reconstruction
from .inverse_depth import (camera_center, initialize_inverse_depth, linearize_rows, radial_limit_squared,
                            update_pose, validate_pose)

#: Elements of one chunk of padded per-point column blocks (points x columns^2).
CHUNK_ELEMENTS = 1 << 22


# ---- small dense blocks, many at a time ------------------------------------------------------------

def _inverse3(a: np.ndarray):
    """inverse3 (src/geometry/numerics.ts:103-131) over (n, 3, 3): adjugate over the determinant."""
    a00, a01, a02 = a[:, 0, 0], a[:, 0, 1], a[:, 0, 2]
    a10, a11, a12 = a[:, 1, 0], a[:, 1, 1], a[:, 1, 2]
    a20, a21, a22 = a[:, 2, 0], a[:, 2, 1], a[:, 2, 2]
    c00, c01, c02 = a11 * a22 - a12 * a21, a02 * a21 - a01 * a22, a01 * a12 - a02 * a11
    det = a00 * c00 + a10 * c01 + a20 * c02
    with np.errstate(divide="ignore", invalid="ignore"):
        out = np.stack([c00, c01, c02, a12 * a20 - a10 * a22, a00 * a22 - a02 * a20, a02 * a10 - a00 * a12,
                        a10 * a21 - a11 * a20, a01 * a20 - a00 * a21, a00 * a11 - a01 * a10], axis=1) / det[:, None]
    ok = np.isfinite(det) & (det != 0) & np.all(np.isfinite(out), axis=1)
    return out.reshape(-1, 3, 3), ok


def _covariance3(info: np.ndarray):
    """inverseDepthCovariance (src/geometry/inverse-depth.ts:157-164) over (n, 3, 3): the inverse
    through the diagonally scaled form, and which blocks are observable."""
    with np.errstate(invalid="ignore", divide="ignore"):
        diag = np.sqrt(np.stack([info[:, 0, 0], info[:, 1, 1], info[:, 2, 2]], axis=1))
        ok = np.all((diag > 0) & np.isfinite(diag), axis=1)
        d = np.where(ok[:, None], diag, 1.0)
        scale = d[:, :, None] * d[:, None, :]
        inv, ok3 = _inverse3(info / scale)
        ok &= ok3 & (inv[:, 0, 0] > 0) & (inv[:, 1, 1] > 0) & (inv[:, 2, 2] > 0)
        return inv / scale, ok


def _positive_inverse2(a: np.ndarray):
    """positiveInverse (inverse-depth-bundle.ts:91-121) over (n, 2, 2): the equilibrated Cholesky
    factor's second pivot must exceed 1e-10."""
    with np.errstate(invalid="ignore", divide="ignore"):
        d = np.sqrt(np.stack([a[:, 0, 0], a[:, 1, 1]], axis=1))
        ok = np.all((d > 0) & np.isfinite(d), axis=1)
        d = np.where(ok[:, None], d, 1.0)
        l10 = a[:, 1, 0] / (d[:, 1] * d[:, 0])
        pivot = 1 - l10 * l10
        ok &= pivot > 1e-10
        inv = np.empty((len(a), 2, 2))
        inv[:, 0, 0] = inv[:, 1, 1] = 1 / pivot
        inv[:, 0, 1] = inv[:, 1, 0] = -l10 / pivot
        inv /= d[:, :, None] * d[:, None, :]
    return inv, ok & np.all(np.isfinite(inv.reshape(-1, 4)), axis=1)


def _factor_inverse(A: np.ndarray, order: np.ndarray | None = None):
    """positiveInverse's factor of an m x m system: the Cholesky factor of D^-1 A D^-1 (D the root of
    the diagonal) taken in ``order`` (natural when None), then its inverse; None unless every
    diagonal is positive and every pivot exceeds 1e-10."""
    n = len(A)
    if n == 0:
        return np.zeros((0, 0))
    with np.errstate(invalid="ignore"):
        d = np.sqrt(np.diag(A))
    if not np.all((d > 0) & np.isfinite(d)):
        return None
    B = A / np.outer(d, d)
    if order is not None:
        B = B[np.ix_(order, order)]
    if not np.all(np.isfinite(B)):
        return None
    try:
        L = np.linalg.cholesky(B)
    except np.linalg.LinAlgError:
        return None
    if not np.all(np.diag(L) ** 2 > 1e-10):
        return None
    Linv = np.linalg.inv(L)
    inv = Linv.T @ Linv
    if order is not None:
        out = np.empty_like(inv)
        out[np.ix_(order, order)] = inv
        inv = out
    inv /= np.outer(d, d)
    return inv if np.all(np.isfinite(inv)) else None


def _minimum_degree(pattern: np.ndarray, structural: int, max_factor: int) -> tuple[np.ndarray, int]:
    """The elimination of factorSparseSchur (src/sfm/depth/sparse-schur.ts:89-178) on the pattern:
    each step takes the uneliminated unknown with the fewest neighbours (the lowest index on ties),
    counts its column into the factor and its neighbours' new couplings into the fill, with the
    reference's budget errors.  Returns the order and the factor's entries (n + the columns)."""
    n = len(pattern)
    adj = pattern.copy()
    np.fill_diagonal(adj, False)
    degree = adj.sum(axis=1).astype(np.int64)
    done = np.zeros(n, dtype=bool)
    order = np.empty(n, dtype=np.int64)
    entries = n
    if entries > max_factor:
        raise RangeError("Schur factor nonzero budget exceeded")
    big = np.iinfo(np.int64).max
    for step in range(n):
        pivot = int(np.argmin(np.where(done, big, degree)))
        order[step] = pivot
        done[pivot] = True
        nb = np.nonzero(adj[pivot])[0]
        entries += len(nb)
        if entries > max_factor:
            raise RangeError("Schur factor nonzero budget exceeded")
        if len(nb) > 1:
            block = np.ix_(nb, nb)
            structural += int(np.count_nonzero(np.triu(~adj[block], 1)))
            if structural > max_factor:
                raise RangeError("Schur fill nonzero budget exceeded")
            adj[block] = True
            adj[nb, nb] = False
        adj[pivot, :] = False
        adj[:, pivot] = False
        degree[nb] = adj[nb].sum(axis=1)
    return order, entries


def _chunks(starts: np.ndarray):
    """Points with at least one column, in chunks of similar column counts: (points, K, entry
    indices (n x K, clipped), valid (n x K)) with n K^2 at most CHUNK_ELEMENTS (one point at least)."""
    counts = np.diff(starts)
    order = np.argsort(counts, kind="stable")
    order = order[counts[order] > 0]
    i = 0
    while i < len(order):
        j = i + 1
        while j < len(order) and (j + 1 - i) * int(counts[order[j]]) ** 2 <= CHUNK_ELEMENTS:
            j += 1
        pts = order[i:j]
        K = int(counts[pts].max())
        slot = np.arange(K)
        valid = slot[None, :] < counts[pts][:, None]
        index = np.where(valid, starts[pts][:, None] + slot[None, :], starts[pts][:, None])
        yield pts, K, index, valid
        i = j


def _huber_cost(e: np.ndarray, h: float) -> np.ndarray:
    return np.where(e <= h, e * e, 2 * h * e - h * h)


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
        basis = np.zeros((6, dim))
        for i in range(6 if dim == 6 else 3):
            basis[i, i] = 1.0
        if dim == 5:
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
                basis[3 + i, 3] = u[i]
                basis[3 + i, 4] = w[i]
        blocks[v["id"]] = {"offset": n, "dimension": dim, "basis": basis}
        n += dim
    return blocks, n


def choose_schur_solver(points, active, groups, options, parameters: int, max_factor_entries: int) -> str:
    """chooseSchurSolver (inverse-depth-bundle.ts:618-654): dense for small camera systems or when
    the camera graph (cameras and focal groups coupled by a common point, self-pairs included) has at
    least 35% of the n(n+1)/2 possible pairs, sparse otherwise.  The reference stops counting once
    that share is reached; the count only grows, so the whole graph decides the same way."""
    solver = options.get("solver")
    if solver and solver != "auto":
        return solver
    if parameters <= 96:
        return "dense"
    if parameters * parameters > max_factor_entries:
        return "sparse"
    cameras = {vid: index for index, vid in enumerate(active)}
    n = len(active) + len(groups)
    focal_groups = options.get("focalGroups") or {}
    point_of, node = [], []
    for k, p in enumerate(points):
        for o in p["observations"]:
            c = cameras.get(o["viewId"])
            if c is not None:
                point_of.append(k)
                node.append(c)
            if groups:
                point_of.append(k)
                node.append(len(active) + groups[focal_groups.get(o["viewId"], 0)])
    involved = np.zeros((len(points), max(n, 1)), dtype=np.float32)
    involved[np.asarray(point_of, dtype=np.int64), np.asarray(node, dtype=np.int64)] = 1
    coupled = np.zeros((max(n, 1), max(n, 1)), dtype=np.float32)
    for first in range(0, len(points), 4096):
        block = involved[first:first + 4096]
        coupled += block.T @ block
    edges = int(np.count_nonzero(np.triu(coupled[:n, :n] > 0)))
    return "dense" if edges >= 0.35 * n * (n + 1) / 2 else "sparse"


class _Measurements:
    """A job's measurement records ({"view", "point"}), built on demand from its packed rows."""

    def __init__(self, rows: np.ndarray):
        self.rows = rows

    def __len__(self):
        return len(self.rows)

    def __getitem__(self, k):
        r = self.rows[k]
        camera = {"fx": r[27], "fy": r[28], "cx": r[29], "cy": r[30], "k1": r[31], "k2": r[32]}
        return {"view": {"camera": camera, "pose": {"R": r[15:24], "t": r[24:27]}},
                "point": {"reference": {"R": r[3:12], "t": r[12:15]}, "parameters": r[0:3]}}

    def __iter__(self):
        for k in range(len(self.rows)):
            yield self[k]


def _as_rows(answer, n: int) -> np.ndarray:
    """An answer to a job as n x 23 result rows (flag 0 where a record is None)."""
    if isinstance(answer, np.ndarray):
        return answer.reshape(n, 23)
    if len(answer) != n:
        raise RangeError("Inverse-depth linearisation count does not match the job")
    out = np.zeros((n, 23))
    for k, j in enumerate(answer):
        if j is None:
            continue
        out[k, 0] = 1
        out[k, 1:3] = j["pixel"]
        out[k, 3:9] = j["point"]
        out[k, 9:21] = j["pose"]
        out[k, 21:23] = j["focal"]
    return out


def inverse_depth_bundle_steps(inp: dict, constraints=(), options: dict | None = None
                               ) -> Generator[dict, Any, dict[str, Any]]:
    """inverseDepthBundleSteps (inverse-depth-bundle.ts:196-565)."""
    # The input is read, never written: results are new records (sharing the input's observation
    # lists, as the reference's object spreads do).
    options = dict(options or {})
    constraints = list(constraints)
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
    # The views reachable from the anchor through shared landmarks (the closure that the
    # reference's repeated passes over the landmarks reach).
    tracks_of: dict[Any, list[int]] = {}
    for k, p in enumerate(inp["landmarks"]):
        for o in p["observations"]:
            tracks_of.setdefault(o["viewId"], []).append(k)
    connected, frontier, seen_tracks = {anchor_id}, [anchor_id], set()
    while frontier:
        for k in tracks_of.get(frontier.pop(), ()):
            if k not in seen_tracks:
                seen_tracks.add(k)
                for o in inp["landmarks"][k]["observations"]:
                    if o["viewId"] not in connected:
                        connected.add(o["viewId"])
                        frontier.append(o["viewId"])
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
    views = [{**v, "camera": dict(v["camera"]),
              "pose": {"R": np.array(v["pose"]["R"], float).ravel(), "t": np.array(v["pose"]["t"], float).ravel()}}
             for v in views_in]
    focal_groups = options.get("focalGroups")
    groups: dict[int, int] = {}
    if options.get("refineSharedFocal"):
        for v in views:
            g = focal_groups.get(v["id"]) if focal_groups is not None else 0
            if g is None or not _safe_int(g) or g < 0:
                raise RangeError("Invalid inverse-depth focal groups")
            if g not in groups:
                groups[g] = len(groups)
    _, planned_n = camera_blocks({"views": views}, active, scale_id if scale_free else None, origin)
    planned = planned_n + len(groups)
    if planned > limit:
        raise RangeError("Inverse-depth camera parameter budget exceeded")
    linear_solver = choose_schur_solver(points, list(active), groups, options, planned, max_factor)
    if (planned ** 2 if linear_solver == "dense" else planned) > max_factor:
        raise RangeError("Schur factor budget exceeded before measurement allocation")

    # The problem as arrays: observations point-major, as the reference walks them.
    vindex = {v["id"]: k for k, v in enumerate(views)}
    P = len(points)
    n_land = len(inp["landmarks"])
    obs_view = np.array([vindex[o["viewId"]] for p in points for o in p["observations"]], dtype=np.int64)
    obs_pix = np.array([o["pixel"] for p in points for o in p["observations"]], dtype=np.float64).reshape(-1, 2)
    counts = np.array([len(p["observations"]) for p in points], dtype=np.int64)
    offsets = np.zeros(P + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    obs_pt = np.repeat(np.arange(P), counts)
    N = len(obs_view)
    dims = np.array([2 if p.get("directionOnly") else 3 for p in points], dtype=np.int64)
    params = np.array([p["point"]["parameters"] for p in points], dtype=np.float64)
    refs = np.array([np.concatenate([np.asarray(p["point"]["reference"]["R"], float).ravel(),
                                     np.asarray(p["point"]["reference"]["t"], float).ravel()]) for p in points])
    group_of_view = np.array([groups[(focal_groups or {}).get(v["id"], 0)] if groups else 0 for v in views],
                             dtype=np.int64)
    lens = np.array([[v["camera"]["cx"], v["camera"]["cy"], v["camera"].get("k1") or 0, v["camera"].get("k2") or 0]
                     for v in views], dtype=np.float64)
    rlim = np.array([min(1e30, radial_limit_squared(k[2], k[3])) for k in lens])
    problem = {"obs_view": obs_view, "obs_pix": obs_pix, "obs_pt": obs_pt, "offsets": offsets, "dims": dims,
               "huber": huber, "sigma": sigma, "groups": groups, "group_of_view": group_of_view,
               "max_schur": max_schur}

    def pack(views_now, prm, rf, live=None):
        """The 34-word rows of linearizeBatches (inverse-depth.ts:51-62) for every observation, or
        for the ``live`` ones."""
        pose = np.array([np.concatenate([np.asarray(v["pose"]["R"], float).ravel(),
                                         np.asarray(v["pose"]["t"], float).ravel()]) for v in views_now])
        fxy = np.array([[v["camera"]["fx"], v["camera"]["fy"]] for v in views_now], dtype=np.float64)
        sel = slice(None) if live is None else live
        pt, vw = obs_pt[sel], obs_view[sel]
        rows = np.empty((len(pt), 34))
        rows[:, 0:3] = prm[pt]
        rows[:, 3:15] = rf[pt]
        rows[:, 15:27] = pose[vw]
        rows[:, 27:29] = fxy[vw]
        rows[:, 29:33] = lens[vw]
        rows[:, 33] = rlim[vw]
        return rows

    def job(rows, purpose="linearize"):
        out = {"rows": rows, "measurements": _Measurements(rows)}
        if purpose != "linearize":
            out["purpose"] = purpose
        return out

    lam = 1e-3
    accepted_steps = 0
    initial_cost = final_cost = 0.0
    last = None
    orders: dict = {}
    for iteration in range(iterations + 1):
        blocks, n_cam = camera_blocks({"views": views}, active, scale_id if scale_free else None, origin)
        m = n_cam + len(groups)
        if m > limit:
            raise RangeError("Inverse-depth camera parameter budget exceeded")
        lin = _as_rows((yield job(pack(views, params, refs))), N)
        if N and np.any(lin[:, 0] != 1):
            raise RangeError("Inverse-depth bundle projection is behind a camera")
        eq = _equations(problem, lin, blocks, views, n_cam, m)
        last = (eq, m)
        if not iteration:
            initial_cost = eq["cost"]
        final_cost = eq["cost"]
        if iteration == iterations:
            break
        reduced = _reduce(eq, m, lam, dims, max_schur)
        if reduced is None:
            lam *= 10
            continue
        factor = _factorize(reduced, linear_solver, max_factor, orders)
        if factor is None:
            lam *= 10
            continue
        delta = factor["inverse"] @ reduced["b"]
        next_views = []
        for k, v in enumerate(views):
            c = blocks.get(v["id"])
            focal = math.exp(delta[n_cam + group_of_view[k]]) if groups else 1
            pose = v["pose"]
            if c is not None:
                step = c["basis"] @ delta[c["offset"]:c["offset"] + c["dimension"]]
                pose = update_pose(v["pose"], [float(x) for x in step])
            next_views.append({**v, "camera": {**v["camera"], "fx": v["camera"]["fx"] * focal,
                                               "fy": v["camera"]["fy"] * focal}, "pose": pose})
        next_params = params + _point_steps(eq, reduced, delta, dims)
        next_refs = refs
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
            next_refs, next_params = _rescale(refs, next_params, s, origin)
        # The candidate's robust cost over the points that were not deferred, projected on the device.
        live = ~eq["deferred"][obs_pt]
        n_live = int(np.count_nonzero(live))
        rows = _as_rows((yield job(pack(candidate_views, next_params, next_refs, live), "cost")), n_live)
        if n_live and np.any(rows[:, 0] != 1):
            next_cost = math.inf
        else:
            e = np.hypot(rows[:, 1] - obs_pix[live, 0], rows[:, 2] - obs_pix[live, 1])
            next_cost = float(np.sum(_huber_cost(e, huber)))
        if np.any(~(next_params[:n_land, 2] > 0)):
            next_cost = math.inf
        if next_cost < eq["cost"]:
            views = candidate_views
            params, refs = next_params, next_refs
            lam = max(1e-12, lam / 3)
            accepted_steps += 1
        else:
            lam *= 10
    eq, m = last
    deferred = eq["deferred"]
    undamped = _reduce(eq, m, 0, dims, max_schur)
    camera_factor = _factorize(undamped, linear_solver, max_factor, orders) if undamped is not None else None
    marginals = _marginals(undamped, camera_factor["inverse"], m) if camera_factor is not None else None
    estimates = []
    for index, p in enumerate(points):
        entry = {**p, "point": {"reference": {"R": refs[index, :9].copy(), "t": refs[index, 9:].copy()},
                                "parameters": params[index].copy()}}
        if marginals is not None and not deferred[index]:
            mg = marginals[index]
            if dims[index] == 3:
                entry["covariance"] = mg.ravel().copy()
                entry["bearingCovariance"] = np.array([mg[0, 0], mg[0, 1], mg[1, 0], mg[1, 1]])
            else:
                entry["bearingCovariance"] = mg[:2, :2].ravel().copy()
        if deferred[index]:
            entry["informationDeferred"] = True
        estimates.append(entry)
    landmarks = []
    for i, p in enumerate(inp["landmarks"]):
        if deferred[i]:
            continue
        landmarks.append({**p, "xyz": _point_of(refs[i], params[i])})
    if any(p["xyz"] is None for p in landmarks):
        raise RangeError("Joint BA invalidated a finite input point")
    # The sparse factor's selected inverse is formed when some observable point has camera columns.
    column_counts = np.diff(eq["starts"])
    selected = linear_solver == "dense" or bool(np.any(column_counts[~deferred] > 0))
    return {
        "reconstruction": {"views": views, "landmarks": landmarks},
        "estimates": estimates,
        "uncertainty": {"poses": "joint" if len(fixed) == 1 else "fixed-exterior",
                        "intrinsics": "joint-focal" if groups else "fixed", "anchorViewId": anchor_id,
                        "scaleViewId": scale_id, "observable": camera_factor is not None,
                        "approximation": "local-robust-Gaussian"},
        "diagnostics": {
            "initialCost": initial_cost, "finalCost": final_cost, "acceptedSteps": accepted_steps,
            "observations": int(np.sum(counts[~deferred])),
            "cameraParameters": m, "backend": "cpu", "linearSolver": linear_solver,
            "schurEntries": undamped["entries"] if undamped is not None else 0,
            "factorEntries": camera_factor["entries"] if camera_factor is not None else 0,
            "cameraCovarianceEntries": camera_factor["entries"] if camera_factor is not None and selected else 0,
            "pointCrossEntries": int(np.sum(column_counts * dims)),
            "denseEquivalentCrossEntries": int(m * np.sum(dims)),
            "inputObservations": int(np.sum(counts)),
            "deferredTrackIds": [p["trackId"] for i, p in enumerate(points) if deferred[i]],
        },
    }


def _point_of(ref: np.ndarray, prm: np.ndarray):
    """inverseDepthPoint (src/geometry/inverse-depth.ts:77-87): the world point, for rho > 0."""
    a, b, rho = (float(v) for v in prm)
    if not rho > 0:
        return None
    R, t = ref[:9], ref[9:]
    C = [-R[i] * t[0] - R[i + 3] * t[1] - R[i + 6] * t[2] for i in range(3)]
    X = np.array([C[i] + (R[i] * a + R[3 + i] * b + R[6 + i]) / rho for i in range(3)])
    return X if np.all(np.isfinite(X)) else None


def _rescale(refs: np.ndarray, prm: np.ndarray, s: float, origin) -> tuple[np.ndarray, np.ndarray]:
    """rescaleInverseDepth (src/geometry/inverse-depth.ts:133-154) of every chart: the reference
    centre scaled about ``origin`` and the inverse depth divided by the scale."""
    R = refs[:, :9].reshape(-1, 3, 3)
    centre = -np.einsum("nji,nj->ni", R, refs[:, 9:])
    o = np.asarray(origin, float)
    out = refs.copy()
    out[:, 9:] = -np.einsum("nij,nj->ni", R, o + s * (centre - o))
    p2 = prm.copy()
    p2[:, 2] /= s
    return out, p2


def _equations(problem: dict, lin: np.ndarray, blocks: dict, views: list, n_cam: int, m: int) -> dict:
    """One pass of inverseDepthBundleSteps over the measurements (inverse-depth-bundle.ts:353-455):
    every point's block V and right-hand side, which points are observable, and over the observable
    ones the robust cost, the camera system A (with its pattern) and right-hand side, and each
    point's cross block W over its camera columns (entries sorted by point, then column; a column
    whose cross block is zero is dropped)."""
    obs_view, obs_pt, offsets, dims = problem["obs_view"], problem["obs_pt"], problem["offsets"], problem["dims"]
    huber, sigma, groups = problem["huber"], problem["sigma"], problem["groups"]
    P, N = len(dims), len(lin)
    Jp = lin[:, 3:9].reshape(N, 2, 3)
    res = lin[:, 1:3] - problem["obs_pix"]
    norm = np.hypot(res[:, 0], res[:, 1])
    with np.errstate(divide="ignore"):
        w = np.where(norm <= huber, 1.0, huber / norm) / sigma ** 2
    V = np.add.reduceat(w[:, None, None] * np.einsum("nrk,nrl->nkl", Jp, Jp), offsets[:-1], axis=0)
    bp = np.add.reduceat(-w[:, None] * np.einsum("nrk,nr->nk", Jp, res), offsets[:-1], axis=0)
    two = dims == 2
    ok = np.zeros(P, dtype=bool)
    if np.any(~two):
        ok[~two] = _covariance3(V[~two])[1]
    if np.any(two):
        ok[two] = _positive_inverse2(V[two][:, :2, :2])[1]
    live = ok[obs_pt]
    cost = float(np.sum(_huber_cost(norm[live], huber)))
    # Each measurement's camera columns (6 through the view's basis) and focal column; -1: none.
    basis = np.zeros((len(views), 6, 6))
    colbase = np.full((len(views), 6), -1, dtype=np.int64)
    for k, v in enumerate(views):
        c = blocks.get(v["id"])
        if c is not None:
            basis[k, :, :c["dimension"]] = c["basis"]
            colbase[k, :c["dimension"]] = c["offset"] + np.arange(c["dimension"])
    E = np.zeros((N, 2, 7))
    E[:, :, :6] = np.einsum("nra,nak->nrk", lin[:, 9:21].reshape(N, 2, 6), basis[obs_view])
    cols = np.full((N, 7), -1, dtype=np.int64)
    cols[:, :6] = colbase[obs_view]
    if groups:
        E[:, :, 6] = lin[:, 21:23]
        cols[:, 6] = n_cam + problem["group_of_view"][obs_view]
    cols[~live] = -1
    ci = np.where(cols >= 0, cols, m)  # column m collects what belongs to no unknown
    pair = (ci[:, :, None] * (m + 1) + ci[:, None, :]).ravel()
    size = (m + 1) * (m + 1)
    A = np.bincount(pair, weights=(w[:, None, None] * np.einsum("nra,nrb->nab", E, E)).ravel(),
                    minlength=size).reshape(m + 1, m + 1)[:m, :m]
    pattern = (np.bincount(pair, minlength=size) > 0).reshape(m + 1, m + 1)[:m, :m]
    bc = np.bincount(ci.ravel(), weights=(-w[:, None] * np.einsum("nra,nr->na", E, res)).ravel(),
                     minlength=m + 1)[:m]
    entries = int(np.count_nonzero(np.triu(pattern)))
    if entries > problem["max_schur"]:
        raise RangeError("Schur nonzero budget exceeded")
    Wn = w[:, None, None] * np.einsum("nra,nrk->nak", E, Jp)
    sel = cols >= 0
    keys, inverse = np.unique((obs_pt[:, None] * (m + 1) + cols)[sel], return_inverse=True)
    Wsel = Wn[sel]
    Ws = np.stack([np.bincount(inverse, weights=Wsel[:, k], minlength=len(keys)) for k in range(3)], axis=1)
    kpt, kcol = keys // (m + 1), keys % (m + 1)
    Ws = Ws * (np.arange(3)[None, :] < dims[kpt][:, None])
    keep = np.any(Ws != 0, axis=1)
    kpt, kcol, Ws = kpt[keep], kcol[keep], Ws[keep]
    return {"V": V, "b": bp, "A": A, "bc": bc, "pattern": pattern, "entries": entries, "cost": cost,
            "deferred": ~ok, "kpt": kpt, "kcol": kcol, "W": Ws, "starts": np.searchsorted(kpt, np.arange(P + 1))}


def _reduce(eq: dict, m: int, lam: float, dims: np.ndarray, max_schur: int):
    """reduce (inverse-depth-bundle.ts:582-616): damp the camera diagonal and every observable
    point block, invert the blocks and eliminate them: S = A - sum W V^-1 W^T, b_c - sum W V^-1 b_p.
    None when a damped block is not invertible."""
    S = eq["A"].copy()
    pattern = eq["pattern"].copy()
    b = eq["bc"].copy()
    di = np.arange(m)
    S[di, di] += lam * np.maximum(S[di, di], 1e-10)
    pattern[di, di] = True
    if int(np.count_nonzero(np.triu(pattern))) > max_schur:
        raise RangeError("Schur nonzero budget exceeded")
    P = len(dims)
    live = ~eq["deferred"]
    inv = np.zeros((P, 3, 3))
    three, two = live & (dims == 3), live & (dims == 2)
    if np.any(three):
        V3 = eq["V"][three].copy()
        for k in range(3):
            V3[:, k, k] += lam * np.maximum(V3[:, k, k], 1e-10)
        i3, ok3 = _covariance3(V3)
        if not np.all(ok3):
            return None
        inv[three] = i3
    if np.any(two):
        V2 = eq["V"][two][:, :2, :2].copy()
        for k in range(2):
            V2[:, k, k] += lam * np.maximum(V2[:, k, k], 1e-10)
        i2, ok2 = _positive_inverse2(V2)
        if not np.all(ok2):
            return None
        inv[two, :2, :2] = i2
    kpt, kcol, W = eq["kpt"], eq["kcol"], eq["W"]
    T = np.einsum("nk,nkj->nj", W, inv[kpt])  # W V^-1, one row per (point, column)
    b -= np.bincount(kcol, weights=np.einsum("nk,nk->n", T, eq["b"][kpt]), minlength=m)[:m]
    update = np.zeros((m + 1) * (m + 1))
    touched = np.zeros((m + 1) * (m + 1), dtype=bool)
    for _, _, index, valid in _chunks(eq["starts"]):
        Tp = T[index] * valid[:, :, None]
        cp = np.where(valid, kcol[index], m)
        pair = (cp[:, :, None] * (m + 1) + cp[:, None, :]).ravel()
        update += np.bincount(pair, weights=np.einsum("pak,pbk->pab", Tp, W[index]).ravel(), minlength=update.size)
        touched[pair] = True
    # The reference adds T_j . W_i to the entry (i, j), i <= j: the lower triangle of sum T W^T.
    U = np.tril(update.reshape(m + 1, m + 1)[:m, :m])
    S -= U + np.tril(U, -1).T
    pattern |= touched.reshape(m + 1, m + 1)[:m, :m]
    entries = int(np.count_nonzero(np.triu(pattern)))
    if entries > max_schur:
        raise RangeError("Schur nonzero budget exceeded")
    return {"S": S, "b": b, "pattern": pattern, "entries": entries, "inv": inv, "T": T, "kcol": kcol,
            "starts": eq["starts"], "m": m}


def _factorize(reduced: dict, solver: str, max_factor: int, orders: dict | None = None):
    """denseSchurFactor (inverse-depth-bundle.ts:655-668) or factorSparseSchur
    (sparse-schur.ts:89-208): {"inverse", "entries"}, or None when a pivot fails.  The elimination
    order is a function of the pattern alone; ``orders`` keeps it by pattern across the LM
    iterations of one solve, whose reduced systems mostly share their pattern."""
    m = reduced["m"]
    if solver == "dense":
        if m * m > max_factor:
            raise RangeError("Dense Schur factor budget exceeded")
        inv = _factor_inverse(reduced["S"])
        return None if inv is None else {"inverse": inv, "entries": m * m}
    if reduced["entries"] > max_factor:
        raise RangeError("Schur factor nonzero budget exceeded")
    diagonal = np.diag(reduced["S"])
    if not np.all((diagonal > 0) & np.isfinite(diagonal)):
        return None
    key = np.packbits(reduced["pattern"]).tobytes()
    if orders is not None and key in orders:
        order, entries = orders[key]
    else:
        order, entries = _minimum_degree(reduced["pattern"], reduced["entries"], max_factor)
        if orders is not None:
            orders[key] = (order, entries)
    inv = _factor_inverse(reduced["S"], order)
    return None if inv is None else {"inverse": inv, "entries": entries}


def _point_steps(eq: dict, reduced: dict, delta: np.ndarray, dims: np.ndarray) -> np.ndarray:
    """Every observable point's step V^-1 (b_p - W^T delta) (inverse-depth-bundle.ts:486-495);
    zero for the deferred ones and in a bearing-only point's depth."""
    kpt, kcol, W = eq["kpt"], eq["kcol"], eq["W"]
    P = len(dims)
    rhs = eq["b"].copy()
    for k in range(3):
        rhs[:, k] -= np.bincount(kpt, weights=W[:, k] * delta[kcol], minlength=P)
    component = (np.arange(3)[None, :] < dims[:, None]) & ~eq["deferred"][:, None]
    return np.einsum("pjk,pk->pj", reduced["inv"], rhs * component) * component


def _marginals(reduced: dict, C: np.ndarray, m: int) -> np.ndarray:
    """pointMarginal (inverse-depth-bundle.ts:669-700) of every point: V^-1 + T^T C T over its
    camera columns (T = W V^-1), C the camera covariance."""
    out = reduced["inv"].copy()
    Cext = np.zeros((m + 1, m + 1))
    Cext[:m, :m] = C
    T, kcol = reduced["T"], reduced["kcol"]
    for pts, _, index, valid in _chunks(reduced["starts"]):
        Tp = T[index] * valid[:, :, None]
        cp = np.where(valid, kcol[index], m)
        CT = np.einsum("pab,pbj->paj", Cext[cp[:, :, None], cp[:, None, :]], Tp)
        out[pts] += np.einsum("pai,paj->pij", Tp, CT)
    return out


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
        out = linearize_rows(device, job["rows"], requested)
        if job.get("purpose") == "cost":
            stats["costBatches"] += out["batches"]
        else:
            stats["batches"] += out["batches"]
            stats["batchSize"] = max(stats["batchSize"], out["batchSize"])
        for rep in out["reports"]:
            stats["launches"] += rep["kernel_launches"]
            stats["device_ms"] += rep["upload_ms"] + rep["evaluate_ms"] + rep["download_ms"]
        return out["out"]

    result = drive(inverse_depth_bundle_steps(model, constraints, options), answer)
    result["diagnostics"] = {**result["diagnostics"], "backend": f"{device.backend}-jacobians/host-f64-Schur",
                             "measurementBatches": stats["batches"], "measurementBatchSize": stats["batchSize"],
                             "costBatches": stats["costBatches"], "kernelLaunches": stats["launches"],
                             "deviceMs": stats["device_ms"]}
    return result
