"""CPU restatement of the reference's observation-evaluation kernels (test infrastructure only).

Follows src/geometry/gpu/observation-evaluation.shade.ts: `projectIndexedObservations` (:40-51),
`stableDepth` / `filterIndexedObservationDepth` (:53-98), the per-64 partials in order
(`indexedObservationPartialsOracle`, :125-138) and `observationSummary`
(src/geometry/gpu/triangulation.shade.ts:134-143), with the projection of
src/device/gpu/numerics.shade.ts (`radialLimit` :79-99, `project` :141-176, `solve3` :25-45).
Input is the packed request of typecv_b200.observations.observation_request.
"""
from __future__ import annotations

import math

import numpy as np


def radial_limit(k1: float, k2: float) -> float:
    if k2 == 0:
        return -1 / (3 * k1) if k1 < 0 else 1e30
    a, b = 5 * k2, 3 * k1
    d = b * b - 4 * a
    if d < 0:
        return 1e30
    q = -0.5 * (b + (-1.0 if b < 0 else 1.0) * math.sqrt(d))
    limit = 1e30
    first = q / a
    if first > 0:
        limit = min(limit, first)
    if q != 0:
        second = 1 / q
        if second > 0:
            limit = min(limit, second)
    return limit


def project(k, q):
    """(ok, pixel, du, dv) of the camera record k = (fx, fy, cx, cy, k1, k2) at camera point q."""
    fx, fy, cx, cy, k1, k2 = k
    if not q[2] > 1e-12:
        return False, None, None, None
    x, y = q[0] / q[2], q[1] / q[2]
    r2 = x * x + y * y
    if not (r2 < radial_limit(k1, k2) and r2 < 1e8):
        return False, None, None, None
    d = 1 + k1 * r2 + k2 * r2 * r2
    g = 2 * (k1 + 2 * k2 * r2)
    if not (d > 0 and 1 + 3 * k1 * r2 + 5 * k2 * r2 * r2 > 0):
        return False, None, None, None
    xx, xy, yy = d + g * x * x, g * x * y, d + g * y * y
    pixel = (fx * x * d + cx, fy * y * d + cy)
    du = ((fx * xx) / q[2], (fx * xy) / q[2], (-fx * (xx * x + xy * y)) / q[2])
    dv = ((fy * xy) / q[2], (fy * yy) / q[2], (-fy * (xy * x + yy * y)) / q[2])
    if not (max(abs(pixel[0]), abs(pixel[1])) < 1e12 and max(map(abs, du)) < 1e12 and max(map(abs, dv)) < 1e12):
        return False, None, None, None
    return True, pixel, du, dv


def solve3(a, b):
    if not min(a[0], a[4], a[8]) > 0:
        return None
    d = (1 / math.sqrt(a[0]), 1 / math.sqrt(a[4]), 1 / math.sqrt(a[8]))
    l10, l20 = a[3] * d[0] * d[1], a[6] * d[0] * d[2]
    p1 = 1 - l10 * l10
    if not p1 > 1e-14:
        return None
    l11 = math.sqrt(p1)
    l21 = (a[7] * d[1] * d[2] - l20 * l10) / l11
    p2 = 1 - l20 * l20 - l21 * l21
    if not p2 > 1e-14:
        return None
    l22 = math.sqrt(p2)
    y0 = b[0] * d[0]
    y1 = (b[1] * d[1] - l10 * y0) / l11
    y2 = (b[2] * d[2] - l20 * y0 - l21 * y1) / l22
    x2 = y2 / l22
    x1 = (y1 - l21 * x2) / l11
    x0 = y0 - l10 * x1 - l20 * x2
    return (x0 * d[0], x1 * d[1], x2 * d[2])


def _record(req, i):
    r = req["cameras"][18 * int(req["indices"][2 * i]):18 * int(req["indices"][2 * i]) + 18]
    return r[:12], r[12:18]


def _transform(pose, X):
    return [pose[3 * r] * X[0] + pose[3 * r + 1] * X[1] + pose[3 * r + 2] * X[2] + pose[9 + r] for r in range(3)]


def _stable_depth(req, flags, start, end, X):
    A = [0.0] * 9
    count = 0
    for i in range(start, end):
        if flags[i] == 0:
            continue
        count += 1
        pose, k = _record(req, i)
        ok, _, du, dv = project(k, _transform(pose, X))
        if not ok:
            return False
        for g in (du, dv):
            J = [g[0] * pose[0] + g[1] * pose[3] + g[2] * pose[6], g[0] * pose[1] + g[1] * pose[4] + g[2] * pose[7],
                 g[0] * pose[2] + g[1] * pose[5] + g[2] * pose[8]]
            for r in range(3):
                for c in range(3):
                    A[3 * r + c] += J[r] * J[c]
    if count < 2:
        return False
    for i in range(start, end):
        if flags[i] == 0:
            continue
        pose, _ = _record(req, i)
        axis = (pose[6], pose[7], pose[8])
        q = _transform(pose, X)
        s = solve3(A, axis)
        if s is None or not q[2] > 0:
            return False
        variance = axis[0] * s[0] + axis[1] * s[1] + axis[2] * s[2]
        if not variance >= 0:
            return False
        if not (req["noise"] * math.sqrt(variance) / q[2] <= req["limit"]):
            return False
    return True


def evaluate(req) -> dict:
    """flags (M [+ P]), errors, summary (error sum, inlier count) of a packed request."""
    M, P = req["count"], req["P"]
    flags = np.zeros(M + (P if req["guarded"] else 0), dtype=np.uint32)
    errors = np.zeros(M)
    for i in range(M):
        pose, k = _record(req, i)
        pt = int(req["indices"][2 * i + 1])
        ok, pixel, _, _ = project(k, _transform(pose, req["points"][3 * pt:3 * pt + 3]))
        if not ok:
            continue
        x, y = pixel[0] - req["pixels"][2 * i], pixel[1] - req["pixels"][2 * i + 1]
        e = math.sqrt(x * x + y * y)
        if e <= req["max_error"]:
            flags[i] = 1
            errors[i] = e
    if req["guarded"]:
        off = req["offsets"]
        for h in range(P):
            start, end = int(off[h]), int(off[h + 1])
            if end <= start or sum(flags[start:end] != 0) < 2:
                continue
            pt = int(req["indices"][2 * start + 1])
            if not _stable_depth(req, flags, start, end, req["points"][3 * pt:3 * pt + 3]):
                flags[M + h] = 1
                flags[start:end] = 0
                errors[start:end] = 0
    partials = []
    for b in range(0, M, 64):
        e = n = 0.0
        for i in range(b, min(M, b + 64)):
            if flags[i]:
                e += errors[i]
                n += 1
        partials.append((e, n))
    total_e = total_n = 0.0
    for e, n in partials:
        total_e += e
        total_n += n
    return {"flags": flags, "errors": errors, "summary": np.array([total_e, total_n])}


def evaluate_cpp(req) -> dict:
    """The same evaluation by the C++ restatement (oracle/ba_oracle.cpp, OpenMP over the host cores)."""
    from oracle import bundle_adjust as ob
    M, P = req["count"], req["P"]
    flags = np.zeros(max(1, M + (P if req["guarded"] else 0)), dtype=np.uint32)
    errors = np.zeros(max(1, M))
    summary = np.zeros(2)
    arr = {k: np.ascontiguousarray(req[k]) for k in ("cameras", "points", "pixels")}
    idx = np.ascontiguousarray(req["indices"], dtype=np.uint32)
    off = np.ascontiguousarray(req["offsets"], dtype=np.uint32)
    ob.lib().oracle_evaluate_observations(P, M, 1 if req["guarded"] else 0, float(req["max_error"]),
                                          float(req["noise"]), float(req["limit"]), ob._dptr(arr["cameras"]),
                                          ob._dptr(arr["points"]), ob._dptr(arr["pixels"]), ob._uptr(idx),
                                          ob._uptr(off), ob._uptr(flags), ob._dptr(errors), ob._dptr(summary))
    return {"flags": flags[:M + (P if req["guarded"] else 0)], "errors": errors[:M], "summary": summary}

