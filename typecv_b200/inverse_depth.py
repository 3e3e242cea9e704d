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


def linearize_inverse_depth_gpu(device: ShadeDevice, job: dict, batch_size: int | None = None):
    """linearizeInverseDepthGpu (inverse-depth.ts:108-114): one linearisation or None per measurement,
    in order."""
    return linearize_batches(device, job, batch_size)["rows"]
