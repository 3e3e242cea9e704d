"""Host side of the GPU bundle adjustment: the Python mirror of TypeCV's ``bundleAdjustGpu``.

``bundle_adjust_gpu(device, input, options)`` keeps the reference operator's contract
(src/sfm/bundle/gpu/bundle.ts:803-839): the same option names and defaults, the same synchronous
``RangeError`` checks with the same message substrings, the same packed arrays handed to the
device (packBundleScene, bundle-host.ts:177-218), the same reading of the output array
(checkBundleOutput / bundleOutputPose / bundleOutputLandmarks / bundleOutputReport,
bundle-host.ts:274-332) and the same result object.  The device work is one call of
``tba_bundle_adjust`` in libtba.so; there is no other implementation.

Objects follow the reference's contracts (src/contracts/scene.ts:22-40, camera.ts:1-20): a scene is
``{"views": [{"id", "camera": {fx, fy, cx, cy, k1?, k2?}, "pose": {"R": 9, "t": 3}}],
"landmarks": [{"trackId", "xyz": 3, "observations": [{"viewId", "featureId", "pixel": [u, v]}]}]}``.
"""
from __future__ import annotations

import ctypes
import math
from typing import Any

import numpy as np

from . import _lib

# src/sfm/config/defaults.ts:51-59
BUNDLE_DEFAULTS = {"iterations": 20, "huberPx": 2.0, "cgRelativeTolerance": 1e-6}
BUNDLE_SOLVER_STALL_TOLERANCE = 1e-9
# BUNDLE_STATE, src/sfm/bundle/gpu/bundle-shared.ts:370-386
BUNDLE_STATE = {"baseline": 2, "cost": 6, "initialCost": 8, "accepted": 10, "rejected": 11, "commit": 12,
                "inputError": 14, "cgSteps": 16, "failedSolves": 17, "initialRmsePx": 24, "finalRmsePx": 25,
                "size": 26, "focalScale": 26}


class RangeError(ValueError):
    """An invalid problem or option (the reference throws RangeError)."""


class DeviceError(RuntimeError):
    """The device failed (a CUDA error); the device should be closed."""


class ShadeDevice:
    """An open CUDA device for the operator (the role of the reference's ShadeDevice,
    src/device/gpu/device.ts:240-360): one stream and a reusable workspace."""

    def __init__(self, handle: int, ordinal: int):
        self._handle = ctypes.c_void_p(handle)
        self.ordinal = ordinal
        self.backend = "cuda"
        # An optional bound on one call's device working set in bytes (the reference device's
        # workingBytes); None leaves the bound to the device's free memory.
        self.working_bytes: int | None = None

    @classmethod
    def open(cls, ordinal: int = 0) -> "ShadeDevice":
        lib = _lib.load()
        h = ctypes.c_void_p()
        status = lib.tba_device_open(ordinal, ctypes.byref(h))
        if status != _lib.TBA_OK:
            raise DeviceError(f"tba_device_open failed ({status}): {lib.tba_last_error(None).decode()}")
        return cls(h.value, ordinal)

    @property
    def handle(self) -> ctypes.c_void_p:
        if not self._handle:
            raise DeviceError("device is closed")
        return self._handle

    def close(self) -> None:
        if self._handle:
            _lib.load().tba_device_close(self._handle)
            self._handle = None

    dispose = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---- validation (src/geometry/validation.ts:6-46, camera.ts:5-12, pose.ts:18-31) ---------------

def camera_center_of(pose) -> list[float]:
    """cameraCenter (src/geometry/pose.ts:34-39): -R^T t, in the reference's order of operations."""
    R, t = pose["R"], pose["t"]
    return [-float(R[i]) * float(t[0]) - float(R[i + 3]) * float(t[1]) - float(R[i + 6]) * float(t[2]) for i in range(3)]


def _safe_int(v) -> bool:
    return isinstance(v, (int, np.integer)) and not isinstance(v, bool) and abs(int(v)) <= 2**53 - 1


def validate_reconstruction(inp) -> None:
    views = set()
    for v in inp["views"]:
        if not _safe_int(v["id"]) or v["id"] < 0 or v["id"] in views:
            raise RangeError("Invalid/duplicate registered view id")
        k = v["camera"]
        vals = [k["fx"], k["fy"], k["cx"], k["cy"], k.get("k1") or 0, k.get("k2") or 0]
        if not all(math.isfinite(x) for x in vals) or k["fx"] <= 0 or k["fy"] <= 0:
            raise RangeError("Invalid camera: finite parameters and positive focal lengths required")
        R, t = np.asarray(v["pose"]["R"], float), np.asarray(v["pose"]["t"], float)
        if R.size != 9 or t.size != 3 or not (np.all(np.isfinite(R)) and np.all(np.isfinite(t))):
            raise RangeError("Invalid pose dimensions or values")
        Rm = R.reshape(3, 3)
        if np.any(np.abs(Rm @ Rm.T - np.eye(3)) > 1e-6) or abs(np.linalg.det(Rm) - 1) > 1e-6:
            raise RangeError("Pose rotation must belong to SO(3)")
        views.add(v["id"])
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


def append_bundle_directions(inp, options):
    """appendBundleDirections (src/sfm/bundle/bundle-directions.ts:19-72): world bearings with
    unresolved depth become trailing points that the kernels treat without translation."""
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


def bundle_problem(inp, options, default_max_cg):
    """bundleProblem (src/sfm/bundle/gpu/bundle-host.ts:31-113)."""
    validate_reconstruction(inp)
    finite_landmarks = inp["landmarks"]
    finite_points = len(finite_landmarks)
    inp = append_bundle_directions(inp, options)
    C, P = len(inp["views"]), len(inp["landmarks"])
    M = sum(len(p["observations"]) for p in inp["landmarks"])
    if not all(0 <= n <= 0xFFFFFFFF for n in (C, P, M)):
        raise RangeError("GPU BA scene dimensions exceed integer index bounds")
    iterations = options.get("iterations", BUNDLE_DEFAULTS["iterations"])
    huber = options.get("huberPx", BUNDLE_DEFAULTS["huberPx"])
    max_cg = options.get("maxCgIterations", default_max_cg(C))
    tolerance = options.get("cgRelativeTolerance", BUNDLE_DEFAULTS["cgRelativeTolerance"])
    if (C < 2 or finite_points < 1 or not _safe_int(iterations) or iterations < 0 or iterations > 100
            or not _finite(huber) or huber < 1e-12 or huber > 1e6 or not _safe_int(max_cg) or max_cg < 1
            or max_cg > 256 or not _finite(tolerance) or tolerance < 1e-12 or tolerance > 1e-2):
        raise RangeError("Invalid GPU BA scene/options")
    ids = [v["id"] for v in inp["views"]]
    by_id = {v: i for i, v in enumerate(ids)}
    anchor_id = options.get("anchorViewId", ids[0])
    scale_id = options.get("scaleViewId", ids[1])
    if anchor_id not in by_id or scale_id not in by_id or anchor_id == scale_id:
        raise RangeError("Invalid GPU BA gauge cameras")
    variable = options.get("variableViewIds")
    if variable is not None and (len(set(variable)) != len(variable)
                                 or any(i == anchor_id or i not in by_id for i in variable)):
        raise RangeError("Invalid GPU BA variable camera window")
    variable_set = None if variable is None else set(variable)
    active = [v != anchor_id and (variable_set is None or v in variable_set) for v in ids]
    fixed = sum(1 for a in active if not a)
    if fixed > 1 and variable_set is not None and scale_id in variable_set:
        raise RangeError("Local GPU BA scale camera must be fixed")
    connected = {anchor_id}
    grew = True
    while grew:
        grew = False
        for p in finite_landmarks:
            if any(o["viewId"] in connected for o in p["observations"]):
                for o in p["observations"]:
                    if o["viewId"] not in connected:
                        connected.add(o["viewId"])
                        grew = True
    if any(v not in connected for v in ids):
        raise RangeError("GPU BA requires one connected observation graph")
    return {"input": inp, "finitePoints": finite_points, "C": C, "P": P, "M": M, "iterations": iterations,
            "huber": float(huber), "maxCg": max_cg, "tolerance": float(tolerance), "byId": by_id,
            "anchorId": anchor_id, "scaleId": scale_id, "active": active, "fixed": fixed}


def _finite(x) -> bool:
    return isinstance(x, (int, float, np.floating, np.integer)) and math.isfinite(x)


def stall_tolerance(options) -> float:
    """bundleStallTolerance (src/sfm/bundle/bundle-shared.ts:8-14)."""
    tol = options.get("stallTolerance", BUNDLE_SOLVER_STALL_TOLERANCE)
    if not _finite(tol) or tol < 0 or tol >= 1:
        raise RangeError("stallTolerance must be in [0, 1)")
    return float(tol)


def validate_gpu_camera(k) -> None:
    """validateGpuCamera (src/geometry/gpu/bounds.ts:5-17)."""
    if (k["fx"] < 1e-6 or k["fy"] < 1e-6 or k["fx"] > 1e6 or k["fy"] > 1e6
            or max(abs(k["cx"]), abs(k["cy"])) > 1e9 or max(abs(k.get("k1") or 0), abs(k.get("k2") or 0)) > 1):
        raise RangeError("Camera exceeds the supported GPU geometry bounds")


def finite_gpu_array(a: np.ndarray) -> bool:
    """finiteGpuArray (src/geometry/gpu/bounds.ts:19-26)."""
    ab = np.abs(a)
    return bool(np.all(np.isfinite(a)) and np.all(ab <= 1e9) and np.all((a == 0) | (ab >= 1e-30)))


def pack_bundle_scene(model, by_id, active):
    """packBundleScene (bundle-host.ts:177-218): scene [poses 12C | points 3P | cameras 6C |
    pixels 2M] and index [obsCamera M | obsPoint M | pointStart P+1 | cameraStart C+1 |
    cameraObservations M | cameraActive C] (bundleIndexLayout, bundle-host.ts:121-131)."""
    views, lms = model["views"], model["landmarks"]
    C, P = len(views), len(lms)
    counts = np.fromiter((len(p["observations"]) for p in lms), dtype=np.int64, count=P)
    M = int(counts.sum())
    scene = np.empty(18 * C + 3 * P + 2 * M)
    index = np.empty(3 * M + P + 2 * C + 2, dtype=np.uint32)
    for c, v in enumerate(views):
        validate_gpu_camera(v["camera"])
        k = v["camera"]
        scene[12 * c:12 * c + 9] = v["pose"]["R"]
        scene[12 * c + 9:12 * c + 12] = v["pose"]["t"]
        scene[12 * C + 3 * P + 6 * c:12 * C + 3 * P + 6 * c + 6] = (
            k["fx"], k["fy"], k["cx"], k["cy"], k.get("k1") or 0, k.get("k2") or 0)
    obs_cam = np.fromiter((by_id[o["viewId"]] for p in lms for o in p["observations"]), dtype=np.uint32, count=M)
    pix = np.fromiter((x for p in lms for o in p["observations"] for x in o["pixel"]), dtype=np.float64, count=2 * M)
    pts = np.fromiter((x for p in lms for x in p["xyz"]), dtype=np.float64, count=3 * P)
    scene[12 * C:12 * C + 3 * P] = pts
    scene[18 * C + 3 * P:] = pix
    point_start = np.zeros(P + 1, dtype=np.int64)
    np.cumsum(counts, out=point_start[1:])
    index[:M] = obs_cam
    index[M:2 * M] = np.repeat(np.arange(P, dtype=np.uint32), counts)
    index[2 * M:2 * M + P + 1] = point_start
    return scene, _finish_index(index, obs_cam, C, P, M, active)


def _finish_index(index, obs_cam, C, P, M, active):
    """The camera-major part of the index: each camera's observations in ascending order."""
    order = np.argsort(obs_cam, kind="stable").astype(np.uint32)
    cam_counts = np.bincount(obs_cam, minlength=C).astype(np.int64)
    camera_start = np.zeros(C + 1, dtype=np.int64)
    np.cumsum(cam_counts, out=camera_start[1:])
    base = 2 * M + P + 1
    index[base:base + C + 1] = camera_start
    index[base + C + 1:base + C + 1 + M] = order
    index[base + C + 1 + M:] = np.asarray(active, dtype=np.uint32)
    return index


def pack_arrays(poses, points, cameras, obs_camera, obs_point, pixels, active):
    """Packed arrays from SoA inputs already in point-major observation order (obs_point
    non-decreasing): the fast path for large scenes, same layout as pack_bundle_scene."""
    C, P, M = len(poses), len(points), len(obs_camera)
    scene = np.empty(18 * C + 3 * P + 2 * M)
    scene[:12 * C] = np.asarray(poses, float).reshape(-1)
    scene[12 * C:12 * C + 3 * P] = np.asarray(points, float).reshape(-1)
    scene[12 * C + 3 * P:18 * C + 3 * P] = np.asarray(cameras, float).reshape(-1)
    scene[18 * C + 3 * P:] = np.asarray(pixels, float).reshape(-1)
    obs_camera = np.asarray(obs_camera, dtype=np.uint32)
    obs_point = np.asarray(obs_point, dtype=np.uint32)
    index = np.empty(3 * M + P + 2 * C + 2, dtype=np.uint32)
    index[:M] = obs_camera
    index[M:2 * M] = obs_point
    counts = np.bincount(obs_point, minlength=P)
    ps = np.zeros(P + 1, dtype=np.int64)
    np.cumsum(counts, out=ps[1:])
    index[2 * M:2 * M + P + 1] = ps
    return scene, _finish_index(index, obs_camera, C, P, M, active)


def make_control(C, P, M, *, anchor, scale_view, iterations=20, max_cg=None, shared_focal=False, huber=2.0,
                 tolerance=1e-6, stall=BUNDLE_SOLVER_STALL_TOLERANCE, directional=0, precision=0, flags=0):
    if max_cg is None:
        max_cg = min(256, max(32, 12 * C + 1)) if shared_focal else min(96, max(24, 12 * C))
    return _lib.Control(C, P, directional, M, anchor, scale_view, iterations, max_cg, int(bool(shared_focal)),
                        precision, flags, huber, tolerance, stall)


def solve_packed(device: ShadeDevice, control: _lib.Control, scene: np.ndarray, index: np.ndarray,
                 output: np.ndarray | None = None):
    """One ``tba_bundle_adjust`` call on packed arrays; returns (output array, report dict)."""
    lib = _lib.load()
    scene = np.ascontiguousarray(scene, dtype=np.float64)
    index = np.ascontiguousarray(index, dtype=np.uint32)
    n_out = lib.tba_output_size(ctypes.byref(control))
    if output is None:
        output = np.zeros(n_out)
    report = _lib.Report()
    status = lib.tba_bundle_adjust(device.handle, ctypes.byref(control), _lib.dptr(scene), scene.size,
                                   _lib.uptr(index), index.size, _lib.dptr(output), output.size, ctypes.byref(report))
    if status != _lib.TBA_OK:
        message = lib.tba_last_error(device.handle).decode()
        if status in (_lib.TBA_ERROR_ARGUMENT, _lib.TBA_ERROR_BUDGET):
            raise RangeError(message)
        raise DeviceError(f"tba_bundle_adjust failed ({status}): {message}")
    return output[:n_out], report.as_dict()


def check_bundle_output(values: np.ndarray, base: int) -> None:
    """checkBundleOutput (bundle-host.ts:278-283)."""
    if values[base + BUNDLE_STATE["inputError"]] == 1:
        raise RangeError("GPU BA gauge requires a nonzero baseline")
    if values[base + BUNDLE_STATE["inputError"]] == 2:
        raise RangeError("GPU BA observations must initially project in front of their cameras")


_WG = (32, 64, 128, 256, "auto")


def prepare_bundle(inp: dict, options: dict | None = None, *, precision: str = "fp64") -> dict[str, Any]:
    """The host half of bundleAdjustGpu before the device plan (bundle.ts:803-839 up to the
    upload): option checks, bundleProblem, packBundleScene, finiteGpuArray and the control block.
    Returns the packed problem with what `finish_bundle` needs to read the result."""
    options = dict(options or {})
    if options.get("cameraProductWorkgroupSize") is not None and options["cameraProductWorkgroupSize"] not in _WG:
        raise RangeError("cameraProductWorkgroupSize must be 32, 64, 128, 256 or auto")
    tile = options.get("cameraProductTileSize")
    if tile is not None and (not _safe_int(tile) or tile < 1 or tile > 0xFFFFFFFF):
        raise RangeError("cameraProductTileSize must be a positive u32 integer")
    if options.get("cameraProduct") is not None and options["cameraProduct"] not in ("workgroups", "rows"):
        raise RangeError("cameraProduct must be 'workgroups' or 'rows'")
    if options.get("schurCache") is not None and not isinstance(options["schurCache"], bool):
        raise RangeError("schurCache must be a boolean")
    if options.get("schurReduction") is not None and options["schurReduction"] not in ("auto", "serial", "cooperative"):
        raise RangeError("Invalid Schur reduction mode")
    shared = bool(options.get("refineSharedFocal"))
    if shared and options.get("focalGroups") and len({options["focalGroups"].get(v["id"]) for v in inp["views"]}) > 1:
        raise RangeError("Per-group focal refinement is not implemented on the GPU")
    if precision not in ("fp64", "mixed"):
        raise RangeError("precision must be 'fp64' or 'mixed'")
    default_max_cg = ((lambda C: min(256, max(32, C * 12 + 1))) if shared else (lambda C: min(96, max(24, C * 12))))
    pb = bundle_problem(inp, options, default_max_cg)
    stall = stall_tolerance(options)
    model = pb["input"]
    scene, index = pack_bundle_scene(model, pb["byId"], pb["active"])
    if not finite_gpu_array(scene):
        raise RangeError("GPU BA input exceeds supported coordinate bounds")
    C, P, M = pb["C"], pb["P"], pb["M"]
    control = make_control(C, P, M, anchor=pb["byId"][pb["anchorId"]], scale_view=pb["byId"][pb["scaleId"]],
                           iterations=pb["iterations"], max_cg=pb["maxCg"], shared_focal=shared, huber=pb["huber"],
                           tolerance=pb["tolerance"], stall=stall, directional=P - pb["finitePoints"],
                           precision=_lib.TBA_PRECISION_MIXED if precision == "mixed" else _lib.TBA_PRECISION_FP64)
    return {"pb": pb, "model": model, "scene": scene, "index": index, "control": control, "shared": shared,
            "C": C, "P": P, "M": M}


def finish_bundle(values: np.ndarray, report: dict, prepared: dict) -> dict[str, Any]:
    """The host half of bundleAdjustGpu after the device plan (bundle.ts:773-800): checkBundleOutput,
    bundleOutputPose / bundleOutputLandmarks / bundleOutputReport, separateBundleDirections."""
    pb, model, shared = prepared["pb"], prepared["model"], prepared["shared"]
    C, P, M = prepared["C"], prepared["P"], prepared["M"]
    base = 12 * C + 3 * P
    check_bundle_output(values, base)
    # Preserve fixed host constants exactly (bundle.ts:776-784; joint-focal.ts:902-910).
    changed = values[base + BUNDLE_STATE["accepted"]] > 0
    focal_scale = math.exp(values[base + BUNDLE_STATE["focalScale"]]) if (changed and shared) else 1.0
    views = []
    for c, v in enumerate(model["views"]):
        cam = dict(v["camera"])
        if changed and shared:
            cam["fx"] = v["camera"]["fx"] * focal_scale
            cam["fy"] = v["camera"]["fy"] * focal_scale
        pose = ({"R": values[12 * c:12 * c + 9].copy(), "t": values[12 * c + 9:12 * c + 12].copy()}
                if changed and pb["active"][c] else v["pose"])
        views.append({**v, "camera": cam, "pose": pose})
    landmarks = [{**p, "xyz": values[12 * C + 3 * i:12 * C + 3 * i + 3].copy() if changed else p["xyz"]}
                 for i, p in enumerate(model["landmarks"])]
    st = values[base:base + 26]
    result = {
        "reconstruction": {"views": views, "landmarks": landmarks},
        "diagnostics": {"initialCost": float(st[8]), "finalCost": float(st[6]), "initialRmsePx": float(st[24]),
                        "finalRmsePx": float(st[25]), "acceptedSteps": int(st[10]), "rejectedSteps": int(st[11]),
                        "observations": M, "baseline": float(st[2])},
        "cgIterations": int(st[16]),
        "linearSolverFailures": int(st[17]),
        "execution": {"backend": "cuda", "report": report, "applicationUploadBytes": report.get("h2d_bytes", 0),
                      "applicationReadbackBytes": report.get("d2h_bytes", 0), "cpuStages": []},
    }
    return separate_bundle_directions(result, pb["finitePoints"])


def bundle_adjust_gpu(device: ShadeDevice, inp: dict, options: dict | None = None, *,
                      precision: str = "fp64") -> dict[str, Any]:
    """Jointly optimise camera poses, points and (with ``refineSharedFocal``) one shared
    log-focal scale on the GPU (bundleAdjustGpu, src/sfm/bundle/gpu/bundle.ts:803-839).

    ``precision="mixed"`` selects the mixed-precision form (no reference counterpart)."""
    prepared = prepare_bundle(inp, options, precision=precision)
    values, report = solve_packed(device, prepared["control"], prepared["scene"], prepared["index"])
    return finish_bundle(values, report, prepared)


def separate_bundle_directions(result, finite_points):
    """separateBundleDirections (bundle-directions.ts:75-98)."""
    lms = result["reconstruction"]["landmarks"]
    if len(lms) == finite_points:
        return result
    directions = lms[finite_points:]
    out = dict(result)
    out["reconstruction"] = {"views": result["reconstruction"]["views"], "landmarks": lms[:finite_points]}
    out["directionalConstraints"] = [{"trackId": p["trackId"], "direction": p["xyz"], "observations": p["observations"]}
                                     for p in directions]
    out["diagnostics"] = {**result["diagnostics"],
                          "directionalObservations": sum(len(p["observations"]) for p in directions),
                          "pointParameters": 3 * finite_points + 2 * len(directions)}
    return out
