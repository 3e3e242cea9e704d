"""Observation evaluation of a fixed scene on the GPU: the Python mirror of TypeCV's
``evaluateObservationsGpu`` and ``evaluateContinuedObservationsGpu``
(src/geometry/gpu/observations.ts:34-58), which the mapper runs after each bundle adjustment to
measure and filter observations (src/sfm/mapper/mapper.ts:837-858).

The host side keeps the reference's request checks and messages (`observationRequest`, :138-213),
its packing into the observation layout and its unpacking of the flags (`unpackObservations`,
:274-297); the device work is one ``tba_evaluate_observations`` call in libtba.so.
"""
from __future__ import annotations

import ctypes
import math
from typing import Any

import numpy as np

from . import _lib
from .bundle import DeviceError, RangeError, ShadeDevice, finite_gpu_array, validate_gpu_camera, validate_reconstruction


def depth_sensitivity_controls(options: dict | None) -> tuple[float, float]:
    """depthSensitivityControls (src/geometry/multiview.ts:26-36): (bound or 0, pixel noise)."""
    options = options or {}
    limit = options.get("maxRelativeDepthStdDev")
    noise = options.get("pixelNoiseStdDevPx", 1)
    if noise is None:
        noise = 1
    if ((limit is not None and (not math.isfinite(limit) or limit <= 0)) or not math.isfinite(noise) or noise <= 0):
        raise RangeError("Invalid conditional depth sensitivity options")
    return (limit or 0.0), float(noise)


def _supported(x: float) -> bool:
    if not math.isfinite(x):
        return False
    m = abs(x)
    return m <= 1e9 and (x == 0 or m >= 1e-30)


def observation_request(model: dict, max_error_px: float, options: dict | None, last_only: bool) -> dict[str, Any]:
    """observationRequest (observations.ts:138-213): checks, then the packed arrays."""
    limit, noise = depth_sensitivity_controls(options)
    guarded = limit > 0
    validate_reconstruction(model)
    if (not finite_gpu_array(np.array([limit, noise])) or not math.isfinite(max_error_px) or max_error_px < 1e-12
            or max_error_px > 1e6):
        raise RangeError("Invalid GPU observation threshold")
    lengths = [1 if last_only else len(p["observations"]) for p in model["landmarks"]]
    count = sum(lengths)
    original: dict[int, int] = {}
    for p in model["landmarks"]:
        for o in p["observations"]:
            original.setdefault(o["viewId"], len(original))
            if last_only and (not _supported(o["pixel"][0]) or not _supported(o["pixel"][1])):
                raise RangeError("Invalid GPU scene coordinate bounds")
    used = original
    if last_only:
        used = {}
        for p in model["landmarks"]:
            used.setdefault(p["observations"][-1]["viewId"], len(used))
    if 2 * count + len(model["landmarks"]) + 1 > 0xFFFFFFFF:
        raise RangeError("GPU observation evaluation exceeds budget")
    views = {v["id"]: v for v in model["views"]}
    cameras = np.zeros(18 * len(used))
    for vid in original:
        v = views[vid]
        k = v["camera"]
        validate_gpu_camera(k)
        row = np.concatenate([np.asarray(v["pose"]["R"], float).ravel(), np.asarray(v["pose"]["t"], float).ravel(),
                              [k["fx"], k["fy"], k["cx"], k["cy"], k.get("k1") or 0, k.get("k2") or 0]])
        if not finite_gpu_array(row):
            raise RangeError("Invalid GPU scene coordinate bounds")
        if vid in used:
            cameras[18 * used[vid]:18 * used[vid] + 18] = row
    P = len(model["landmarks"])
    points = np.zeros(3 * P)
    pixels = np.zeros(2 * count)
    indices = np.zeros(2 * count, dtype=np.uint32)
    at = 0
    for i, p in enumerate(model["landmarks"]):
        xyz = np.asarray(p["xyz"], float)
        if not finite_gpu_array(xyz):
            raise RangeError("Invalid GPU scene coordinate bounds")
        points[3 * i:3 * i + 3] = xyz
        for o in (p["observations"][-1:] if last_only else p["observations"]):
            pixels[2 * at:2 * at + 2] = o["pixel"]
            indices[2 * at] = used[o["viewId"]]
            indices[2 * at + 1] = i
            at += 1
    if not finite_gpu_array(pixels):
        raise RangeError("Invalid GPU scene coordinate bounds")
    offsets = np.zeros(P + 1, dtype=np.uint32)
    np.cumsum(lengths, out=offsets[1:])
    return {"limit": limit, "noise": noise, "guarded": guarded, "lengths": lengths, "count": count,
            "max_error": float(max_error_px),
            "cameras": cameras, "points": points, "pixels": pixels, "indices": indices, "offsets": offsets,
            "C": len(used), "P": P}


def unpack_observations(summary: np.ndarray, flags: np.ndarray, lengths: list[int], count: int,
                        guarded: bool) -> dict[str, Any]:
    """unpackObservations (observations.ts:274-297)."""
    masks, at = [], 0
    for n in lengths:
        masks.append(flags[at:at + n].astype(np.uint8))
        at += n
    out: dict[str, Any] = {}
    if guarded:
        out["depthRejected"] = flags[count:count + len(lengths)].astype(np.uint8)
    out["masks"] = masks
    out["inlierCount"] = float(summary[1])
    out["meanErrorPx"] = float(summary[0] / summary[1]) if summary[1] > 0 else math.inf
    return out


def _evaluate(device: ShadeDevice, model: dict, max_error_px: float, options: dict | None,
              last_only: bool) -> dict[str, Any]:
    req = observation_request(model, max_error_px, options, last_only)
    lib = _lib.load()
    C, P, M = req["C"], req["P"], req["count"]
    ctl = _lib.ObservationControl(C, P, M, 0, float(max_error_px), float(req["limit"]), float(req["noise"]))
    flags = np.zeros(max(1, M + (P if req["guarded"] else 0)), dtype=np.uint32)
    summary = np.zeros(2)
    report = _lib.ObservationReport()
    cams = np.ascontiguousarray(req["cameras"]) if C else np.zeros(1)
    pts = np.ascontiguousarray(req["points"]) if P else np.zeros(1)
    pix = np.ascontiguousarray(req["pixels"]) if M else np.zeros(1)
    idx = np.ascontiguousarray(req["indices"]) if M else np.zeros(1, dtype=np.uint32)
    off = np.ascontiguousarray(req["offsets"])
    status = lib.tba_evaluate_observations(device.handle, ctypes.byref(ctl), _lib.dptr(cams), req["cameras"].size,
                                           _lib.dptr(pts), req["points"].size, _lib.dptr(pix), req["pixels"].size,
                                           _lib.uptr(idx), req["indices"].size, _lib.uptr(off), off.size,
                                           _lib.uptr(flags), flags.size, _lib.dptr(summary), ctypes.byref(report))
    if status != _lib.TBA_OK:
        message = lib.tba_last_error(device.handle).decode()
        if status in (_lib.TBA_ERROR_ARGUMENT, _lib.TBA_ERROR_BUDGET):
            raise RangeError(message)
        raise DeviceError(f"tba_evaluate_observations failed ({status}): {message}")
    result = unpack_observations(summary, flags, req["lengths"], M, req["guarded"])
    rep = report.as_dict()
    result["execution"] = {"backend": "cuda", "report": rep, "applicationUploadBytes": rep["h2d_bytes"],
                           "applicationReadbackBytes": rep["d2h_bytes"]}
    return result


def evaluate_observations_gpu(device: ShadeDevice, model: dict, max_error_px: float = 3,
                              options: dict | None = None) -> dict[str, Any]:
    """Project and filter every observation of a fixed scene; masks in landmark order."""
    return _evaluate(device, model, max_error_px, options, False)


def evaluate_continued_observations_gpu(device: ShadeDevice, model: dict, max_error_px: float = 3,
                                        options: dict | None = None) -> dict[str, Any]:
    """evaluateContinuedObservationsGpu (observations.ts:50-58): only each landmark's last
    observation, unless the depth bound needs every original observation."""
    limit, _ = depth_sensitivity_controls(options)
    return _evaluate(device, model, max_error_px, options, not (limit > 0))
