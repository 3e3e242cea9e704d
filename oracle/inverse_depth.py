"""CPU restatement of the reference's inverse-depth geometry (test infrastructure only).

Follows src/geometry/inverse-depth.ts: `initializeInverseDepth` (:19-35) and `inverseDepthJacobian`
(:38-74), with the CPU projection of src/geometry/camera.ts (`radialLimitSquared` :15-24,
`cameraProjection` :27-61, `unprojectPixel` :64-105) and the pose helpers of src/geometry/pose.ts
(`transformPoint` :28-33, `cameraCenter` :34-39).  These are the functions the reference's own test
compares its device linearisation with (tests/typeshade/inverse-depth-cases.mjs:126-165).

`bundle_adjust_inverse_depth` is the reference's CPU `bundleAdjustInverseDepth`
(src/sfm/depth/inverse-depth-bundle.ts:717-729): the host steps restated loop for loop
(oracle/inverse_depth_steps.py), answered with this file's CPU linearisation.  `fit_inverse_depth` restates
`fitInverseDepth` (src/geometry/inverse-depth.ts:184-249) with `solveSystem`
(src/geometry/numerics.ts:71-100), which the reference's bundle tests use as the fixed-pose baseline.
"""
from __future__ import annotations

import math

import numpy as np


def radial_limit_squared(k1: float, k2: float) -> float:
    if k2 == 0:
        return -1 / (3 * k1) if k1 < 0 else math.inf
    a, b = 5 * k2, 3 * k1
    d = b * b - 4 * a
    if d < 0:
        return math.inf
    q = -0.5 * (b + (1.0 if b >= 0 else -1.0) * math.sqrt(d))
    roots = []
    for x in (q / a, (1 / q) if q != 0 else math.inf):
        if x > 0 and math.isfinite(x):
            roots.append(x)
    return min(roots) if roots else math.inf


def camera_projection(k: dict, q):
    """(pixel, 2x3 jacobian row-major) or None."""
    X, Y, Z = float(q[0]), float(q[1]), float(q[2])
    if not Z > 1e-12 or not all(math.isfinite(v) for v in (X, Y, Z)):
        return None
    x, y = X / Z, Y / Z
    r2 = x * x + y * y
    k1, k2 = k.get("k1") or 0, k.get("k2") or 0
    if r2 >= radial_limit_squared(k1, k2):
        return None
    d = 1 + k1 * r2 + k2 * r2 * r2
    g = 2 * (k1 + 2 * k2 * r2)
    xx, xy, yy = d + g * x * x, g * x * y, d + g * y * y
    if not (d > 0 and 1 + 3 * k1 * r2 + 5 * k2 * r2 * r2 > 0):
        return None
    pixel = (k["fx"] * x * d + k["cx"], k["fy"] * y * d + k["cy"])
    jac = [k["fx"] * xx / Z, k["fx"] * xy / Z, -k["fx"] * (xx * x + xy * y) / Z,
           k["fy"] * xy / Z, k["fy"] * yy / Z, -k["fy"] * (xy * x + yy * y) / Z]
    if not all(math.isfinite(v) for v in (*pixel, *jac)):
        return None
    return pixel, jac


def unproject_pixel(k: dict, pixel):
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


def transform_point(pose, X):
    R, t = np.asarray(pose["R"], float).ravel(), np.asarray(pose["t"], float).ravel()
    return [R[3 * i] * X[0] + R[3 * i + 1] * X[1] + R[3 * i + 2] * X[2] + t[i] for i in range(3)]


def camera_center(pose):
    R, t = np.asarray(pose["R"], float).ravel(), np.asarray(pose["t"], float).ravel()
    return [-R[i] * t[0] - R[i + 3] * t[1] - R[i + 6] * t[2] for i in range(3)]


def initialize_inverse_depth(view: dict, pixel, xyz=None) -> dict:
    ray = unproject_pixel(view["camera"], pixel)
    if ray is None:
        raise ValueError("Inverse-depth anchor cannot be unprojected")
    params = [ray[0], ray[1], 0.0]
    if xyz is not None:
        q = transform_point(view["pose"], xyz)
        if not (q[2] > 0) or not all(math.isfinite(v) for v in q):
            raise ValueError("Invalid finite inverse-depth seed")
        params = [q[0] / q[2], q[1] / q[2], 1 / q[2]]
    pose = view["pose"]
    return {"reference": {"R": np.array(pose["R"], float).ravel(), "t": np.array(pose["t"], float).ravel()},
            "parameters": np.array(params, float)}


def inverse_depth_jacobian(camera: dict, pose: dict, point: dict):
    """{pixel, point (2x3), pose (2x6), focal (2)} or None, in the reference's summation order."""
    r = np.asarray(point["parameters"], float)
    Rv, Rr = np.asarray(pose["R"], float).ravel(), np.asarray(point["reference"]["R"], float).ravel()
    A = [0.0] * 9
    C = camera_center(point["reference"])
    T = transform_point(pose, C)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                A[3 * i + j] += Rv[3 * i + k] * Rr[3 * j + k]
    q = [A[3 * i] * r[0] + A[3 * i + 1] * r[1] + A[3 * i + 2] + r[2] * T[i] for i in range(3)]
    proj = camera_projection(camera, q)
    if proj is None:
        return None
    pixel, J = proj
    pt, cam = [0.0] * 6, [0.0] * 12
    B = [0, q[2], -q[1], -q[2], 0, q[0], q[1], -q[0], 0]
    for row in range(2):
        for col in range(3):
            for k in range(3):
                pt[3 * row + col] += J[3 * row + k] * (A[3 * k + col] if col < 2 else T[k])
                cam[6 * row + col] += J[3 * row + k] * B[3 * k + col]
            cam[6 * row + col + 3] = r[2] * J[3 * row + col]
    return {"pixel": pixel, "point": np.array(pt), "pose": np.array(cam),
            "focal": np.array([pixel[0] - camera["cx"], pixel[1] - camera["cy"]])}


def linearize_rows(rows: np.ndarray) -> np.ndarray:
    """The C++ restatement of inverseDepthJacobian (oracle/ba_oracle.cpp, OpenMP over the host
    cores) over (n x 34) rows; (n x 23) rows in the device layout, flag 0 where invalid."""
    from oracle import bundle_adjust as ob
    rows = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 34)
    out = np.zeros((len(rows), 23))
    if len(rows):
        ob.lib().oracle_linearize_inverse_depth(len(rows), ob._dptr(rows), ob._dptr(out))
    return out


def linearize_job(job):
    """linearizeInverseDepthJob (src/sfm/depth/inverse-depth-bundle.ts:717-719)."""
    return [inverse_depth_jacobian(m["view"]["camera"], m["view"]["pose"], m["point"]) for m in job["measurements"]]


def bundle_adjust_inverse_depth(inp, constraints=(), options=None):
    """The reference's CPU `bundleAdjustInverseDepth` (inverse-depth-bundle.ts:720-729): the restated
    host steps (oracle/inverse_depth_steps.py) answered with this file's CPU linearisation."""
    from oracle.inverse_depth_steps import drive, inverse_depth_bundle_steps
    return drive(inverse_depth_bundle_steps(inp, constraints, options), linearize_job)


def solve_system(matrix, rhs):
    n = len(rhs)
    a = [[float(matrix[i * n + j]) for j in range(n)] + [float(rhs[i])] for i in range(n)]
    if any(not all(math.isfinite(v) for v in row) for row in a):
        return None
    scale = max([0.0] + [max(abs(v) for v in row[:n]) for row in a])
    if not scale > 0:
        return [] if n == 0 else None
    for j in range(n):
        p = j
        for i in range(j + 1, n):
            if abs(a[i][j]) > abs(a[p][j]):
                p = i
        if abs(a[p][j]) < 1e-14 * scale:
            return None
        a[p], a[j] = a[j], a[p]
        for i in range(j + 1, n):
            f = a[i][j] / a[j][j]
            for k in range(j, n + 1):
                a[i][k] -= f * a[j][k]
    out = [0.0] * n
    for i in range(n - 1, -1, -1):
        b = a[i][n]
        for j in range(i + 1, n):
            b -= a[i][j] * out[j]
        out[i] = b / a[i][i]
    return out if all(math.isfinite(v) for v in out) else None


def fit_inverse_depth(observations, iterations=12, sigma=1.0, huber=3.0):
    """observations: [{camera, pose, pixel}], the first one the anchor."""
    from typecv_b200.inverse_depth import inverse_depth_covariance
    point = initialize_inverse_depth({"camera": observations[0]["camera"], "pose": observations[0]["pose"]},
                                     observations[0]["pixel"])
    lam = 1e-3

    def linearize(p):
        H, b = [0.0] * 9, [0.0] * 3
        cost = 0.0
        for o in observations:
            j = inverse_depth_jacobian(o["camera"], o["pose"], p)
            if j is None:
                return None
            r = (j["pixel"][0] - o["pixel"][0], j["pixel"][1] - o["pixel"][1])
            e = math.hypot(*r)
            w = (1 if e <= huber else huber / e) / sigma ** 2
            cost += e * e if e <= huber else 2 * huber * e - huber * huber
            for row in range(2):
                for k in range(3):
                    b[k] -= w * j["point"][3 * row + k] * r[row]
                    for l in range(3):
                        H[3 * k + l] += w * j["point"][3 * row + k] * j["point"][3 * row + l]
        return {"H": H, "b": b, "cost": cost}

    current = linearize(point)
    for _ in range(iterations):
        if current is None:
            break
        H = list(current["H"])
        for k in range(3):
            H[4 * k] += lam * max(H[4 * k], 1e-10)
        d = solve_system(H, current["b"])
        if d is None:
            break
        candidate = {**point, "parameters": np.array([x + d[k] for k, x in enumerate(point["parameters"])])}
        nxt = linearize(candidate)
        if nxt is not None and nxt["cost"] < current["cost"]:
            point, current = candidate, nxt
            lam /= 3
        else:
            lam *= 10
    if current is None:
        raise ValueError("Invalid inverse-depth observations")
    return {"point": point, "covariance": inverse_depth_covariance(current["H"])}
