"""The oracle's Python face (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module, and
only as the checker; the product package never does.  It wraps ``ba_oracle.cpp``:

* ``cpu_bundle_adjust(input, options)`` mirrors the reference's CPU ``bundleAdjust``
  (src/sfm/bundle/bundle-adjustment.ts:294-301): the host checks of
  bundle-adjustment.ts:84-142 / joint-focal.ts:49-110, validateReconstruction
  (src/geometry/validation.ts:6-46) and appendBundleDirections
  (src/sfm/bundle/bundle-directions.ts:19-72), then the dense LM in C++.
* ``gpu_operator(packed, options)`` runs the reference GPU operator's algorithm (matrix-free
  Schur PCG, bundle.shade.ts / joint-focal.shade.ts) on a packed problem and returns its output
  array (the layout of the reference's ``packBundleResult``).
* ``pack(input, ...)`` restates packBundleScene (src/sfm/bundle/gpu/bundle-host.ts:177-218).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libtba_oracle.so")
SOURCE = os.path.join(HERE, "ba_oracle.cpp")


class RangeError(ValueError):
    """The reference throws RangeError for invalid problems and options."""


class Control(ctypes.Structure):
    _fields_ = [
        ("cameras", ctypes.c_uint32), ("points", ctypes.c_uint32),
        ("observations", ctypes.c_uint32), ("directional_points", ctypes.c_uint32),
        ("anchor", ctypes.c_uint32), ("scale_view", ctypes.c_uint32),
        ("iterations", ctypes.c_uint32), ("max_cg", ctypes.c_uint32),
        ("shared_focal", ctypes.c_uint32), ("focal_groups", ctypes.c_uint32),
        ("huber", ctypes.c_double), ("cg_tolerance", ctypes.c_double),
        ("stall_tolerance", ctypes.c_double),
    ]


def build(force: bool = False) -> str:
    """Compile the restatement with gcc (no FMA, no contraction: JavaScript's rounding)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SOURCE):
        os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
        tmp = LIB_PATH + f".{os.getpid()}.tmp"
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
                               "-o", tmp, SOURCE])
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        P = ctypes.POINTER
        _lib.oracle_output_size.restype = ctypes.c_size_t
        _lib.oracle_output_size.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib.oracle_cpu_bundle_adjust.restype = ctypes.c_int
        _lib.oracle_cpu_bundle_adjust.argtypes = [P(Control), P(ctypes.c_double), P(ctypes.c_uint32),
                                                  P(ctypes.c_uint32), P(ctypes.c_double)]
        _lib.oracle_gpu_operator.restype = ctypes.c_int
        _lib.oracle_gpu_operator.argtypes = [P(Control), P(ctypes.c_double), P(ctypes.c_uint32),
                                             P(ctypes.c_double)]
        _lib.oracle_linearize_inverse_depth.restype = None
        _lib.oracle_linearize_inverse_depth.argtypes = [ctypes.c_uint32, P(ctypes.c_double), P(ctypes.c_double)]
        _lib.oracle_evaluate_observations.restype = None
        _lib.oracle_evaluate_observations.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                                      ctypes.c_double, ctypes.c_double, P(ctypes.c_double),
                                                      P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_uint32),
                                                      P(ctypes.c_uint32), P(ctypes.c_uint32), P(ctypes.c_double),
                                                      P(ctypes.c_double)]
        _lib.oracle_metrics.restype = None
        _lib.oracle_metrics.argtypes = [P(Control), P(ctypes.c_double), P(ctypes.c_uint32), P(ctypes.c_double)]
    return _lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _uptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


# ---- validation (src/geometry/validation.ts, camera.ts, pose.ts) --------------------------------

def _safe_int(v) -> bool:
    return isinstance(v, (int, np.integer)) and not isinstance(v, bool) and abs(int(v)) <= 2**53 - 1


def validate_camera(k) -> None:
    vals = [k["fx"], k["fy"], k["cx"], k["cy"], k.get("k1", 0) or 0, k.get("k2", 0) or 0]
    if not all(math.isfinite(v) for v in vals) or k["fx"] <= 0 or k["fy"] <= 0:
        raise RangeError("Invalid camera: finite parameters and positive focal lengths required")


def validate_pose(p) -> None:
    R, t = np.asarray(p["R"], float), np.asarray(p["t"], float)
    if R.size != 9 or t.size != 3 or not np.all(np.isfinite(R)) or not np.all(np.isfinite(t)):
        raise RangeError("Invalid pose dimensions or values")
    M = R.reshape(3, 3)
    q = M @ M.T
    if np.any(np.abs(q - np.eye(3)) > 1e-6) or abs(np.linalg.det(M) - 1) > 1e-6:
        raise RangeError("Pose rotation must belong to SO(3)")


def validate_reconstruction(inp) -> None:
    views = {}
    for v in inp["views"]:
        if not _safe_int(v["id"]) or v["id"] < 0 or v["id"] in views:
            raise RangeError("Invalid/duplicate registered view id")
        validate_camera(v["camera"])
        validate_pose(v["pose"])
        views[v["id"]] = v
    points, owned = set(), set()
    for p in inp["landmarks"]:
        xyz = np.asarray(p["xyz"], float)
        if (not _safe_int(p["trackId"]) or p["trackId"] < 0 or p["trackId"] in points or xyz.size != 3
                or not np.all(np.isfinite(xyz))):
            raise RangeError("Invalid/duplicate landmark")
        points.add(p["trackId"])
        if len(p["observations"]) < 2:
            raise RangeError("Landmarks require at least two observations")
        seen = set()
        for o in p["observations"]:
            key = (o["viewId"], o["featureId"])
            if (o["viewId"] not in views or o["viewId"] in seen or not _safe_int(o["featureId"])
                    or o["featureId"] < 0 or len(o["pixel"]) != 2
                    or not all(math.isfinite(x) for x in o["pixel"]) or key in owned):
                raise RangeError("Invalid or multiply owned landmark observation")
            seen.add(o["viewId"])
            owned.add(key)


def append_directions(inp, options):
    """appendBundleDirections, bundle-directions.ts:19-72: bearings become trailing points."""
    cons = options.get("directionalConstraints")
    if cons is None:
        return inp
    if not isinstance(cons, (list, tuple)):
        raise RangeError("directionalConstraints must be an array")
    ids = {p["trackId"] for p in inp["landmarks"]}
    views = {v["id"] for v in inp["views"]}
    features = {(o["viewId"], o["featureId"]) for p in inp["landmarks"] for o in p["observations"]}
    extra = []
    for c in cons:
        d = np.asarray(c.get("direction", []), float)
        norm = math.hypot(*d) if d.size == 3 else math.nan
        if (not _safe_int(c.get("trackId")) or c["trackId"] < 0 or c["trackId"] in ids or d.size != 3
                or not math.isfinite(norm) or norm <= 1e-12 or len(c.get("observations", [])) < 2):
            raise RangeError("Invalid or multiply owned directional constraint")
        ids.add(c["trackId"])
        seen = set()
        for o in c["observations"]:
            key = (o["viewId"], o["featureId"])
            if (o["viewId"] not in views or o["viewId"] in seen or not _safe_int(o["featureId"])
                    or o["featureId"] < 0 or len(o["pixel"]) != 2
                    or not all(math.isfinite(x) for x in o["pixel"]) or key in features):
                raise RangeError("Invalid or multiply owned directional observation")
            seen.add(o["viewId"])
            features.add(key)
        extra.append({"trackId": c["trackId"], "xyz": d / norm, "observations": c["observations"]})
    return {"views": inp["views"], "landmarks": list(inp["landmarks"]) + extra} if extra else inp


def _connected(inp, anchor_id) -> bool:
    connected = {anchor_id}
    grew = True
    while grew:
        grew = False
        for p in inp["landmarks"]:
            if any(o["viewId"] in connected for o in p["observations"]):
                for o in p["observations"]:
                    if o["viewId"] not in connected:
                        connected.add(o["viewId"])
                        grew = True
    return all(v["id"] in connected for v in inp["views"])


def pack(inp, active=None):
    """packBundleScene, bundle-host.ts:177-218: scene [poses|points|cameras|pixels], index
    [obsCamera|obsPoint|pointStart|cameraStart|cameraObservations|cameraActive]."""
    views, lms = inp["views"], inp["landmarks"]
    C, P = len(views), len(lms)
    M = sum(len(p["observations"]) for p in lms)
    by_id = {v["id"]: i for i, v in enumerate(views)}
    scene = np.zeros(18 * C + 3 * P + 2 * M)
    index = np.zeros(3 * M + P + 2 * C + 2, dtype=np.uint32)
    for c, v in enumerate(views):
        k = v["camera"]
        scene[12 * c:12 * c + 9] = v["pose"]["R"]
        scene[12 * c + 9:12 * c + 12] = v["pose"]["t"]
        scene[12 * C + 3 * P + 6 * c:12 * C + 3 * P + 6 * c + 6] = [
            k["fx"], k["fy"], k["cx"], k["cy"], k.get("k1", 0) or 0, k.get("k2", 0) or 0]
    a_off = 3 * M + P + C + 2
    if active is not None:
        index[a_off:a_off + C] = active
    lists = [[] for _ in range(C)]
    obs = 0
    pix_off = 18 * C + 3 * P
    for p, lm in enumerate(lms):
        scene[12 * C + 3 * p:12 * C + 3 * p + 3] = lm["xyz"]
        index[2 * M + p] = obs
        for o in lm["observations"]:
            c = by_id[o["viewId"]]
            index[obs] = c
            index[M + obs] = p
            scene[pix_off + 2 * obs:pix_off + 2 * obs + 2] = o["pixel"]
            lists[c].append(obs)
            obs += 1
    index[2 * M + P] = obs
    cur = 0
    for c in range(C):
        index[2 * M + P + 1 + c] = cur
        index[2 * M + P + C + 2 + cur:2 * M + P + C + 2 + cur + len(lists[c])] = lists[c]
        cur += len(lists[c])
    index[2 * M + P + 1 + C] = cur
    return {"C": C, "P": P, "M": M, "scene": scene, "index": index, "by_id": by_id}


def control(packed, anchor, scale_view, iterations, huber, *, max_cg=1, tolerance=1e-6, stall=1e-9,
            shared=False, groups=1, directional=0) -> Control:
    return Control(packed["C"], packed["P"], packed["M"], directional, anchor, scale_view, iterations,
                   max_cg, int(bool(shared)), groups, huber, tolerance, stall)


def _stall(options) -> float:
    tol = options.get("stallTolerance", 1e-9)
    if not math.isfinite(tol) or tol < 0 or tol >= 1:
        raise RangeError("stallTolerance must be in [0, 1)")
    return tol


def _group_index(inp, groups):
    """focalGroupIndex, joint-focal.ts:30-42."""
    if groups is None:
        return [0] * len(inp["views"])
    numbers = [groups.get(v["id"]) for v in inp["views"]]
    if any(g is None or not _safe_int(g) for g in numbers):
        raise RangeError("Every view needs a focal group")
    rank = {g: i for i, g in enumerate(sorted(set(numbers)))}
    return [rank[g] for g in numbers]


def cpu_bundle_adjust(inp, options=None):
    """bundleAdjust (bundle-adjustment.ts:294-301) on the CPU restatement."""
    options = dict(options or {})
    shared = bool(options.get("refineSharedFocal"))
    validate_reconstruction(inp)
    iterations = options.get("iterations", 20)
    huber = options.get("huberPx", 2)
    stall = _stall(options)
    bad_opts = not _safe_int(iterations) or iterations < 0 or not math.isfinite(huber) or huber <= 0
    if not shared:
        if len(inp["views"]) < 2 or not inp["landmarks"]:
            raise RangeError("Bundle adjustment needs two views and landmarks")
        if bad_opts:
            raise RangeError("Invalid bundle adjustment options")
    elif len(inp["views"]) < 2 or not inp["landmarks"] or bad_opts:
        raise RangeError("Invalid joint focal bundle scene/options")
    anchor_id = options.get("anchorViewId", inp["views"][0]["id"])
    scale_id = options.get("scaleViewId", inp["views"][1]["id"])
    ids = [v["id"] for v in inp["views"]]
    if anchor_id not in ids or scale_id not in ids or anchor_id == scale_id:
        raise RangeError("Invalid bundle adjustment gauge cameras")
    a, s = inp["views"][ids.index(anchor_id)]["pose"], inp["views"][ids.index(scale_id)]["pose"]
    o, sc = camera_center(a), camera_center(s)
    if not math.hypot(*(o - sc)) > 1e-10:
        raise RangeError("Bundle adjustment gauge requires a nonzero baseline")
    if not _connected(inp, anchor_id):
        raise RangeError("Bundle adjustment requires one connected observation graph")
    finite_points = len(inp["landmarks"])
    inp = append_directions(inp, options)
    variable = options.get("variableViewIds")

    def check_window():
        if variable is not None and (len(set(variable)) != len(variable)
                                     or any(i == anchor_id or i not in ids for i in variable)):
            raise RangeError("Invalid variable camera window")
        fixed = [i for i in ids if i == anchor_id or (variable is not None and i not in variable)]
        if len(fixed) > 1 and variable is not None and scale_id in variable:
            raise RangeError("Local BA scale camera must be fixed")

    packed = pack(inp, [int(i != anchor_id and (variable is None or i in variable)) for i in ids])
    group_of = None
    ngroups = 1
    if shared:
        check_window()
        g = _group_index(inp, options.get("focalGroups"))
        ngroups = max(g) + 1
        group_of = np.asarray(g, dtype=np.uint32)
        nact = sum(1 for i in ids if i != anchor_id and (variable is None or i in variable))
        n = 6 * nact + ngroups
        if n * n > 16 * 1024**2:
            raise RangeError("Joint focal CPU reduced system is too large")
    ctl = control(packed, ids.index(anchor_id), ids.index(scale_id), iterations, huber, stall=stall,
                  shared=shared, groups=ngroups, directional=len(inp["landmarks"]) - finite_points)
    out = np.zeros(lib().oracle_output_size(packed["C"], packed["P"]))
    if not shared:
        m3 = np.zeros(3)
        lib().oracle_metrics(ctypes.byref(ctl), _dptr(packed["scene"]), _uptr(packed["index"]), _dptr(m3))
        if not math.isfinite(m3[0]):
            raise RangeError("Bundle adjustment observations must initially project in front of their cameras")
        check_window()
    status = lib().oracle_cpu_bundle_adjust(ctypes.byref(ctl), _dptr(packed["scene"]), _uptr(packed["index"]),
                                            None if group_of is None else _uptr(group_of), _dptr(out))
    if status == 2:
        raise RangeError("Bundle adjustment observations must initially project in front of their cameras")
    return unpack(inp, packed, out, finite_points, cpu=True)


def camera_center(pose):
    R, t = np.asarray(pose["R"], float), np.asarray(pose["t"], float)
    return np.array([-R[i] * t[0] - R[i + 3] * t[1] - R[i + 6] * t[2] for i in range(3)])


def unpack(inp, packed, out, finite_points, cpu):
    C, P = packed["C"], packed["P"]
    st = out[12 * C + 3 * P:12 * C + 3 * P + 26]
    views = []
    for c, v in enumerate(inp["views"]):
        cam = dict(v["camera"])
        if cpu:
            cam["fx"], cam["fy"] = out[12 * C + 3 * P + 27 + c], out[12 * C + 3 * P + 27 + C + c]
        views.append({**v, "camera": cam, "pose": {"R": out[12 * c:12 * c + 9].copy(),
                                                   "t": out[12 * c + 9:12 * c + 12].copy()}})
    lms = [{**p, "xyz": out[12 * C + 3 * i:12 * C + 3 * i + 3].copy()} for i, p in enumerate(inp["landmarks"])]
    diag = {"initialCost": st[8], "finalCost": st[6], "initialRmsePx": st[24], "finalRmsePx": st[25],
            "acceptedSteps": int(st[10]), "rejectedSteps": int(st[11]), "observations": packed["M"],
            "baseline": st[2]}
    result = {"reconstruction": {"views": views, "landmarks": lms[:finite_points]}, "diagnostics": diag}
    if not cpu:
        result["cgIterations"] = int(st[16])
        result["linearSolverFailures"] = int(st[17])
        result["logFocalScale"] = out[12 * C + 3 * P + 26]
    if len(lms) > finite_points:
        result["directionalConstraints"] = [{"trackId": p["trackId"], "direction": p["xyz"],
                                             "observations": p["observations"]} for p in lms[finite_points:]]
    return result


def gpu_operator_packed(packed, anchor, scale_view, *, iterations=20, huber=2.0, max_cg=None, tolerance=1e-6,
                        stall=1e-9, shared=False, directional=0):
    """The reference operator's algorithm on a packed problem; returns its output array."""
    C = packed["C"]
    if max_cg is None:
        max_cg = min(256, max(32, 12 * C + 1)) if shared else min(96, max(24, 12 * C))
    ctl = control(packed, anchor, scale_view, iterations, huber, max_cg=max_cg, tolerance=tolerance,
                  stall=stall, shared=shared, directional=directional)
    out = np.zeros(lib().oracle_output_size(packed["C"], packed["P"]))
    lib().oracle_gpu_operator(ctypes.byref(ctl), _dptr(packed["scene"]), _uptr(packed["index"]), _dptr(out))
    return out[:12 * C + 3 * packed["P"] + 27]


def gpu_operator(inp, options=None):
    """The reference operator's algorithm with its host (bundle-host.ts bundleProblem subset)."""
    options = dict(options or {})
    shared = bool(options.get("refineSharedFocal"))
    finite_points = len(inp["landmarks"])
    inp2 = append_directions(inp, options)
    ids = [v["id"] for v in inp2["views"]]
    anchor_id = options.get("anchorViewId", ids[0])
    scale_id = options.get("scaleViewId", ids[1])
    variable = options.get("variableViewIds")
    active = [int(i != anchor_id and (variable is None or i in variable)) for i in ids]
    packed = pack(inp2, active)
    out = gpu_operator_packed(packed, ids.index(anchor_id), ids.index(scale_id),
                              iterations=options.get("iterations", 20), huber=options.get("huberPx", 2),
                              max_cg=options.get("maxCgIterations"),
                              tolerance=options.get("cgRelativeTolerance", 1e-6),
                              stall=_stall(options), shared=shared,
                              directional=len(inp2["landmarks"]) - finite_points)
    C, P = packed["C"], packed["P"]
    st = out[12 * C + 3 * P:]
    if st[14] == 1:
        raise RangeError("GPU BA gauge requires a nonzero baseline")
    if st[14] == 2:
        raise RangeError("GPU BA observations must initially project in front of their cameras")
    full = np.zeros(lib().oracle_output_size(C, P))
    full[:out.size] = out
    res = unpack(inp2, packed, full, finite_points, cpu=False)
    changed = st[10] > 0
    scale = math.exp(st[26]) if (changed and shared) else 1.0
    for c, v in enumerate(res["reconstruction"]["views"]):
        src = inp2["views"][c]
        if not (changed and active[c]):
            v["pose"] = {"R": np.asarray(src["pose"]["R"], float).copy(), "t": np.asarray(src["pose"]["t"], float).copy()}
        v["camera"] = dict(src["camera"])
        if changed and shared:
            v["camera"]["fx"] = src["camera"]["fx"] * scale
            v["camera"]["fy"] = src["camera"]["fy"] * scale
    if not changed:
        for lm, src in zip(res["reconstruction"]["landmarks"], inp2["landmarks"]):
            lm["xyz"] = np.asarray(src["xyz"], float).copy()
    return res


def metrics_packed(packed, huber, directional=0):
    ctl = control(packed, 0, 1, 0, huber, directional=directional)
    m3 = np.zeros(3)
    lib().oracle_metrics(ctypes.byref(ctl), _dptr(packed["scene"]), _uptr(packed["index"]), _dptr(m3))
    return {"cost": m3[0], "rmse": m3[1], "observations": int(m3[2])}
