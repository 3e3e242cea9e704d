"""Inverse-depth measurement linearisation on the GPU: the Python mirror of TypeCV's
``linearizeInverseDepthGpu`` and its batching (src/sfm/depth/gpu/inverse-depth.ts:15-114).

Each measurement is an anchored inverse-depth point ``{"reference": pose, "parameters": (a, b, rho)}``
seen by a registered view.  The host packs one 34-word row per measurement (the point's parameters,
the reference pose record, the observing pose record, the camera record and its squared radial
limit, capped at 1e30), ``tba_linearize_inverse_depth`` evaluates every row on the device, and the
23-word result rows are unpacked into ``{"pixel", "point", "pose", "focal"}`` or None where the
projection leaves the camera model's domain.  Splitting the measurements into batches changes only
how much is resident at once: every row is evaluated exactly once and independently.
"""
from __future__ import annotations

import copy
import ctypes
import math
from typing import Any

import numpy as np

from . import _lib
from .bundle import DeviceError, RangeError, ShadeDevice

#: Device words held per measurement while a batch is resident (34 in, 23 out).
WORDS_PER_MEASUREMENT = 57
#: The largest batch one launch takes (one thread per measurement, 34-word rows addressed in 32 bits).
MAX_KERNEL_ELEMENTS = 0xFFFFFFFF // 34


def radial_limit_squared(k1: float, k2: float) -> float:
    """radialLimitSquared (src/geometry/camera.ts:15-24): the squared normalised radius where the
    radial model's first derivative vanishes (infinite when it never does)."""
    if k2 == 0:
        return -1 / (3 * k1) if k1 < 0 else math.inf
    a, b = 5 * k2, 3 * k1
    d = b * b - 4 * a
    if d < 0:
        return math.inf
    q = -0.5 * (b + (1.0 if b >= 0 else -1.0) * math.sqrt(d))
    roots = [x for x in ((q / a) if a else math.inf, (1 / q) if q else math.inf) if x > 0 and math.isfinite(x)]
    return min(roots) if roots else math.inf


def pose_record(pose) -> list[float]:
    """poseRecord (src/contracts/camera-record.ts:12-14): R row-major, then t."""
    return [float(x) for x in np.asarray(pose["R"], float).ravel()] + [float(x) for x in np.asarray(pose["t"], float).ravel()]


def camera_record(camera) -> list[float]:
    """cameraRecord (src/contracts/camera-record.ts:17-19): fx, fy, cx, cy, k1, k2."""
    return [camera["fx"], camera["fy"], camera["cx"], camera["cy"], camera.get("k1") or 0, camera.get("k2") or 0]


def pack_measurements(measurements) -> np.ndarray:
    """The 34-word input rows of linearizeBatches (inverse-depth.ts:51-62)."""
    out = np.zeros(34 * len(measurements))
    for i, m in enumerate(measurements):
        point, view = m["point"], m["view"]
        k = view["camera"]
        row = out[34 * i:34 * i + 34]
        row[0:3] = np.asarray(point["parameters"], float)
        row[3:15] = pose_record(point["reference"])
        row[15:27] = pose_record(view["pose"])
        row[27:33] = camera_record(k)
        row[33] = min(1e30, radial_limit_squared(k.get("k1") or 0, k.get("k2") or 0))
    return out


def unpack_linearizations(result: np.ndarray, n: int) -> list[dict[str, Any] | None]:
    """The 23-word result rows (inverse-depth.ts:80-91): None unless the valid flag is 1."""
    rows: list[dict[str, Any] | None] = []
    for i in range(n):
        r = result[23 * i:23 * i + 23]
        rows.append(None if r[0] != 1 else {"pixel": (float(r[1]), float(r[2])), "point": r[3:9].copy(),
                                            "pose": r[9:21].copy(), "focal": r[21:23].copy()})
    return rows


def _linearize(device: ShadeDevice, packed: np.ndarray, n: int) -> tuple[np.ndarray, dict]:
    lib = _lib.load()
    out = np.zeros(max(1, 23 * n))
    report = _lib.ObservationReport()
    src = np.ascontiguousarray(packed[:34 * n]) if n else np.zeros(1)
    status = lib.tba_linearize_inverse_depth(device.handle, n, _lib.dptr(src), 34 * n, _lib.dptr(out), 23 * n,
                                             ctypes.byref(report))
    if status != _lib.TBA_OK:
        message = lib.tba_last_error(device.handle).decode()
        if status in (_lib.TBA_ERROR_ARGUMENT, _lib.TBA_ERROR_BUDGET):
            raise RangeError(message)
        raise DeviceError(f"tba_linearize_inverse_depth failed ({status}): {message}")
    return out, report.as_dict()


def linearize_batches(device: ShadeDevice, job: dict, requested: int | None = None) -> dict[str, Any]:
    """linearizeBatches (inverse-depth.ts:16-106): {rows, batches, batchSize, reports}."""
    if requested is not None and (isinstance(requested, bool) or not isinstance(requested, int) or requested < 1):
        raise RangeError("Invalid inverse-depth measurement batch size")
    snapshot = copy.deepcopy(list(job["measurements"]))
    count = len(snapshot)
    if not count:
        return {"rows": [], "batches": 0, "batchSize": 0, "reports": []}
    available = device.working_bytes if device.working_bytes is not None else 1 << 62
    batch = min(count, requested if requested is not None else count, available // (8 * WORDS_PER_MEASUREMENT),
                MAX_KERNEL_ELEMENTS)
    if not batch >= 1:
        raise RangeError("Inverse-depth measurement budget cannot fit one observation")
    rows: list[dict[str, Any] | None] = []
    reports = []
    batches = 0
    for first in range(0, count, batch):
        n = min(batch, count - first)
        out, rep = _linearize(device, pack_measurements(snapshot[first:first + n]), n)
        batches += 1
        reports.append(rep)
        rows.extend(unpack_linearizations(out, n))
    return {"rows": rows, "batches": batches, "batchSize": batch, "reports": reports}


def linearize_rows(device: ShadeDevice, rows: np.ndarray, requested: int | None = None) -> dict[str, Any]:
    """The same batching on rows already packed (n x 34): {"out": n x 23, batches, batchSize, reports}."""
    if requested is not None and (isinstance(requested, bool) or not isinstance(requested, int) or requested < 1):
        raise RangeError("Invalid inverse-depth measurement batch size")
    rows = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 34)
    count = len(rows)
    if not count:
        return {"out": np.zeros((0, 23)), "batches": 0, "batchSize": 0, "reports": []}
    available = device.working_bytes if device.working_bytes is not None else 1 << 62
    batch = min(count, requested if requested is not None else count, available // (8 * WORDS_PER_MEASUREMENT),
                MAX_KERNEL_ELEMENTS)
    if not batch >= 1:
        raise RangeError("Inverse-depth measurement budget cannot fit one observation")
    out = np.empty((count, 23))
    reports, batches = [], 0
    for first in range(0, count, batch):
        n = min(batch, count - first)
        o, rep = _linearize(device, rows[first:first + n].ravel(), n)
        out[first:first + n] = o[:23 * n].reshape(n, 23)
        reports.append(rep)
        batches += 1
    return {"out": out, "batches": batches, "batchSize": batch, "reports": reports}


def linearize_inverse_depth_gpu(device: ShadeDevice, job: dict, batch_size: int | None = None):
    """linearizeInverseDepthGpu (inverse-depth.ts:108-114): one linearisation or None per measurement,
    in order."""
    return linearize_batches(device, job, batch_size)["rows"]


# ---- host geometry of the anchored inverse-depth chart (src/geometry/inverse-depth.ts, pose.ts) ----

def multiply3(a, b) -> list[float]:
    """multiply (src/geometry/linear.ts:8-17) for 3x3, row-major, sums in index order."""
    out = []
    for r in range(3):
        for c in range(3):
            s = 0.0
            for k in range(3):
                s += a[r * 3 + k] * b[k * 3 + c]
            out.append(s)
    return out


def rotation_exp(w) -> list[float]:
    """rotationExp (src/geometry/pose.ts:40-51)."""
    x, y, z = (float(v) for v in w[:3])
    if not all(math.isfinite(v) for v in (x, y, z)):
        raise RangeError("Invalid rotation vector")
    theta = math.hypot(x, y, z)
    a = 1 - theta * theta / 6 if theta < 1e-7 else math.sin(theta) / theta
    b = 0.5 - theta * theta / 24 if theta < 1e-7 else (1 - math.cos(theta)) / (theta * theta)
    W = [0.0, -z, y, z, 0.0, -x, -y, x, 0.0]
    W2 = multiply3(W, W)
    return [(1 if i % 4 == 0 else 0) + a * W[i] + b * W2[i] for i in range(9)]


def transform_point(pose, X) -> list[float]:
    """transformPoint (src/geometry/pose.ts:28-33)."""
    R, t = pose["R"], pose["t"]
    return [float(R[i * 3]) * X[0] + float(R[i * 3 + 1]) * X[1] + float(R[i * 3 + 2]) * X[2] + float(t[i])
            for i in range(3)]


def camera_center(pose) -> list[float]:
    """cameraCenter (src/geometry/pose.ts:34-39)."""
    R, t = pose["R"], pose["t"]
    return [-float(R[i]) * float(t[0]) - float(R[i + 3]) * float(t[1]) - float(R[i + 6]) * float(t[2]) for i in range(3)]


def update_pose(pose, delta) -> dict:
    """updatePose (src/geometry/pose.ts:52-57): left rotation, additive camera translation."""
    dR = rotation_exp(delta)
    rotated = transform_point({"R": dR, "t": [0.0, 0.0, 0.0]}, [float(v) for v in pose["t"]])
    return {"R": np.array(multiply3(dR, [float(v) for v in pose["R"]])),
            "t": np.array([rotated[i] + delta[i + 3] for i in range(3)])}


def validate_pose(p) -> None:
    """validatePose (src/geometry/pose.ts:13-27)."""
    R, t = np.asarray(p["R"], float).ravel(), np.asarray(p["t"], float).ravel()
    if R.size != 9 or t.size != 3 or not (np.all(np.isfinite(R)) and np.all(np.isfinite(t))):
        raise RangeError("Invalid pose dimensions or values")
    q = multiply3(list(R), [R[0], R[3], R[6], R[1], R[4], R[7], R[2], R[5], R[8]])
    det = (R[0] * (R[4] * R[8] - R[5] * R[7]) - R[1] * (R[3] * R[8] - R[5] * R[6])
           + R[2] * (R[3] * R[7] - R[4] * R[6]))
    if any(abs(v - (1 if i % 4 == 0 else 0)) > 1e-6 for i, v in enumerate(q)) or abs(det - 1) > 1e-6:
        raise RangeError("Pose rotation must belong to SO(3)")


def validate_camera(k) -> None:
    """validateCamera (src/geometry/camera.ts:5-12)."""
    vals = [k["fx"], k["fy"], k["cx"], k["cy"], k.get("k1") or 0, k.get("k2") or 0]
    if not all(math.isfinite(v) for v in vals) or k["fx"] <= 0 or k["fy"] <= 0:
        raise RangeError("Invalid camera: finite parameters and positive focal lengths required")


def unproject_pixel(k, pixel):
    """unprojectPixel (src/geometry/camera.ts:64-105): the normalised bearing of a pixel on the
    radial model's monotone branch, by backtracking Newton steps; None when it has none."""
    validate_camera(k)
    xd, yd = (pixel[0] - k["cx"]) / k["fx"], (pixel[1] - k["cy"]) / k["fy"]
    rd = math.hypot(xd, yd)
    if not math.isfinite(rd):
        return None
    if rd == 0:
        return (0.0, 0.0)
    k1, k2 = k.get("k1") or 0, k.get("k2") or 0
    limit2 = radial_limit_squared(k1, k2)
    if math.isfinite(limit2) and rd >= math.sqrt(limit2) * (1 + k1 * limit2 + k2 * limit2 * limit2):
        return None
    r = rd
    for _ in range(50):
        r2 = r * r
        d = 1 + k1 * r2 + k2 * r2 * r2
        slope = 1 + 3 * k1 * r2 + 5 * k2 * r2 * r2
        if not (slope > 1e-10 and d > 0):
            return None
        residual = r * d - rd
        if abs(residual) <= 1e-12 * max(1, rd):
            return (xd * r / rd, yd * r / rd)
        step, accepted = residual / slope, False
        for _ in range(25):
            nxt = r - step
            n2 = nxt * nxt
            if (nxt >= 0 and n2 < limit2 and 1 + 3 * k1 * n2 + 5 * k2 * n2 * n2 > 0
                    and abs(nxt * (1 + k1 * n2 + k2 * n2 * n2) - rd) < abs(residual)):
                r, accepted = nxt, True
                break
            step *= 0.5
        if not accepted:
            return None
    return None


def initialize_inverse_depth(view: dict, pixel, xyz=None) -> dict:
    """initializeInverseDepth (src/geometry/inverse-depth.ts:19-35): the chart anchored at the
    view, (a, b) the pixel's bearing and rho the inverse depth of xyz (0 without it)."""
    validate_camera(view["camera"])
    validate_pose(view["pose"])
    ray = unproject_pixel(view["camera"], pixel)
    if ray is None:
        raise RangeError("Inverse-depth anchor cannot be unprojected")
    params = [ray[0], ray[1], 0.0]
    if xyz is not None:
        q = transform_point(view["pose"], [float(v) for v in xyz])
        if not q[2] > 0 or not all(math.isfinite(v) for v in q):
            raise RangeError("Invalid finite inverse-depth seed")
        params = [q[0] / q[2], q[1] / q[2], 1 / q[2]]
    return {"reference": {"R": np.array(view["pose"]["R"], float).ravel(), "t": np.array(view["pose"]["t"], float).ravel()},
            "parameters": np.array(params, float)}


def inverse3(a) -> list[float] | None:
    """inverse3 (src/geometry/numerics.ts:103-131): adjugate over the determinant."""
    a00, a01, a02, a10, a11, a12, a20, a21, a22 = (float(v) for v in a)
    c00, c01, c02 = a11 * a22 - a12 * a21, a02 * a21 - a01 * a22, a01 * a12 - a02 * a11
    det = a00 * c00 + a10 * c01 + a20 * c02
    if not math.isfinite(det) or det == 0:
        return None
    out = [c00 / det, c01 / det, c02 / det, (a12 * a20 - a10 * a22) / det, (a00 * a22 - a02 * a20) / det,
           (a02 * a10 - a00 * a12) / det, (a10 * a21 - a11 * a20) / det, (a01 * a20 - a00 * a21) / det,
           (a00 * a11 - a01 * a10) / det]
    return out if all(math.isfinite(v) for v in out) else None


def inverse_depth_covariance(information) -> list[float] | None:
    """inverseDepthCovariance (src/geometry/inverse-depth.ts:157-164): the inverse of a 3x3
    information matrix through its diagonally scaled form; None where it is not observable."""
    info = [float(v) for v in information]
    diagonal = [math.sqrt(info[i]) if info[i] >= 0 else math.nan for i in (0, 4, 8)]
    if any(not (x > 0 and math.isfinite(x)) for x in diagonal):
        return None
    scaled = [x / (diagonal[i // 3] * diagonal[i % 3]) for i, x in enumerate(info)]
    inv = inverse3(scaled)
    if inv is None or any(not inv[i] > 0 for i in (0, 4, 8)):
        return None
    return [x / (diagonal[i // 3] * diagonal[i % 3]) for i, x in enumerate(inv)]


def inverse_depth_point(p) -> np.ndarray | None:
    """inverseDepthPoint (src/geometry/inverse-depth.ts:77-87): the world point, for rho > 0."""
    a, b, rho = (float(v) for v in p["parameters"])
    if not rho > 0:
        return None
    C = camera_center(p["reference"])
    R = p["reference"]["R"]
    X = np.array([C[i] + (float(R[i]) * a + float(R[3 + i]) * b + float(R[6 + i])) / rho for i in range(3)])
    return X if np.all(np.isfinite(X)) else None


def rescale_inverse_depth(p, scale: float, origin) -> dict:
    """rescaleInverseDepth (src/geometry/inverse-depth.ts:133-154) without a covariance: the chart of
    the same bearing after the map is scaled about `origin`."""
    if not (scale > 0 and math.isfinite(scale)):
        raise RangeError("Invalid inverse-depth map scale")
    C = [origin[i] + scale * (c - origin[i]) for i, c in enumerate(camera_center(p["reference"]))]
    R = np.array(p["reference"]["R"], float)
    t = np.array([-R[3 * i] * C[0] - R[3 * i + 1] * C[1] - R[3 * i + 2] * C[2] for i in range(3)])
    parameters = np.array(p["parameters"], float)
    parameters[2] /= scale
    return {"reference": {"R": R, "t": t}, "parameters": parameters}
