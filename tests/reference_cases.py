"""Restatements of the reference's deterministic test fixtures (test infrastructure).

Each generator follows the reference's own fixture code step by step, in the same order of
floating-point operations and random draws, so that the scenes are bit-identical:

* ``pose_fixture``            tests/typeshade/geometry-cases.mjs:2-64   (poseFixture)
* ``bundle_fixture``          tests/typeshade/geometry-cases.mjs:166-218 (bundleFixture)
* ``ring_bundle_fixture``     tests/typeshade/geometry-cases.mjs:252-316 (ringBundleFixture)
* ``joint_focal_fixture``     tests/typeshade/joint-focal-cases.mjs:2-80 (jointFocalFixture)
* ``scene``                   tests/scene.ts:10-61                       (scene)
* ``perturbed``               tests/bundle-adjustment.test.ts:7-30       (perturbed)
* ``inverse_depth_scene``     tests/typeshade/inverse-depth-cases.mjs:1-56  (inverseDepthScene)
* ``inverse_depth_long_scene`` tests/typeshade/inverse-depth-cases.mjs:58-85 (inverseDepthLongScene)

The reference hashes ``JSON.stringify(input)`` of some of these scenes in its benchmark records
(docs/experiments/gpu/*.json, ``inputSha256``).  ``js_json`` restates JSON.stringify (ECMAScript
Number::toString for numbers, Float64Array as an object with index keys) so those hashes pin the
restated fixtures bit for bit.
"""
from __future__ import annotations

import hashlib
import math
from decimal import Decimal

import numpy as np


class F64(np.ndarray):
    """A Float64Array: JSON.stringify writes it as {"0": .., "1": ..}."""


def f64(values) -> F64:
    return np.asarray(values, dtype=np.float64).copy().view(F64)


# ---- JSON.stringify ----------------------------------------------------------------------------

def js_number(x: float) -> str:
    """ECMAScript Number::toString (radix 10) of a finite double; JSON writes NaN/inf as null."""
    x = float(x)
    if x != x or x in (math.inf, -math.inf):
        return "null"
    if x == 0:
        return "0"
    sign = "-" if x < 0 else ""
    t = Decimal(repr(abs(x))).as_tuple()  # repr is the shortest round-trip digit string
    digits = "".join(map(str, t.digits)).rstrip("0")
    exp = t.exponent + (len("".join(map(str, t.digits))) - len(digits))
    digits = digits.lstrip("0") or "0"
    k = len(digits)
    n = exp + k
    if k <= n <= 21:
        s = digits + "0" * (n - k)
    elif 0 < n <= 21:
        s = digits[:n] + "." + digits[n:]
    elif -6 < n <= 0:
        s = "0." + "0" * (-n) + digits
    else:
        e = n - 1
        mant = digits if k == 1 else digits[0] + "." + digits[1:]
        s = f"{mant}e{'+' if e >= 0 else '-'}{abs(e)}"
    return sign + s


def js_json(v) -> str:
    if isinstance(v, F64):
        return "{" + ",".join(f'"{i}":{js_number(x)}' for i, x in enumerate(v)) + "}"
    if isinstance(v, dict):
        return "{" + ",".join(f'"{k}":{js_json(x)}' for k, x in v.items()) + "}"
    if isinstance(v, (list, tuple)):
        return "[" + ",".join(js_json(x) for x in v) + "]"
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return js_number(float(v))
    if isinstance(v, (float, np.floating)):
        return js_number(float(v))
    if isinstance(v, str):
        return '"' + v + '"'
    raise TypeError(type(v))


def input_sha256(scene) -> str:
    return hashlib.sha256(js_json(scene).encode()).hexdigest()


# ---- random number generators ------------------------------------------------------------------

def _i32(v: int) -> int:
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


class XorShift32:
    """The fixtures' inline xorshift32 (geometry-cases.mjs:10-16) and seededRandom
    (src/geometry/numerics.ts:133-141): JS int32 shifts, result (s >>> 0) / 2**32."""

    def __init__(self, seed: int):
        self.s = _i32(seed)

    def __call__(self) -> float:
        s = self.s
        s = _i32(s ^ _i32(s << 13))
        s = _i32(s ^ ((s & 0xFFFFFFFF) >> 17))
        s = _i32(s ^ _i32(s << 5))
        self.s = s
        return (s & 0xFFFFFFFF) / 2**32


def seeded_random(seed: int) -> XorShift32:
    s = seed & 0xFFFFFFFF
    return XorShift32(s if s else 0x9E3779B9)


class Lcg:
    """joint-focal-cases.mjs:55-59: seed = (imul(seed, 1664525) + 1013904223) >>> 0."""

    def __init__(self, seed: int):
        self.s = seed

    def __call__(self) -> float:
        self.s = (self.s * 1664525 + 1013904223) & 0xFFFFFFFF
        return self.s / 2**32


# ---- geometry-cases.mjs ------------------------------------------------------------------------

def pose_fixture(count=97, noise=0.3, outliers=0.25, planar=False, scale=1, radial=True):
    nxt = XorShift32(731)
    a, b = 0.11, -0.03
    ca, sa, cb, sb = math.cos(a), math.sin(a), math.cos(b), math.sin(b)
    R = [ca, sa * sb, sa * cb, 0, cb, -sb, -sa, ca * sb, ca * cb]
    t = [0.3 * scale, -0.1 * scale, 0.2 * scale]
    camera = {"fx": 900, "fy": 920, "cx": 480, "cy": 270,
              "k1": -0.05 if radial else 0, "k2": 0.005 if radial else 0}
    world = np.zeros(count * 3)
    pixels = np.zeros(count * 2)
    for i in range(count):
        X0 = (nxt() - 0.5) * 4 * scale
        X1 = (nxt() - 0.5) * 3 * scale
        X2 = (6 if planar else 4 + nxt() * 5) * scale
        X = [X0, X1, X2]
        q = [t[j] + R[j * 3] * X[0] + R[j * 3 + 1] * X[1] + R[j * 3 + 2] * X[2] for j in range(3)]
        x, y = q[0] / q[2], q[1] / q[2]
        r2 = x * x + y * y
        d = 1 + camera["k1"] * r2 + camera["k2"] * r2 * r2
        world[3 * i:3 * i + 3] = X
        px = camera["fx"] * x * d + camera["cx"] + (nxt() - 0.5) * noise * 2
        py = camera["fy"] * y * d + camera["cy"] + (nxt() - 0.5) * noise * 2
        pixels[2 * i:2 * i + 2] = [px, py]
        if i < math.floor(count * outliers):
            pixels[2 * i:2 * i + 2] = [50 + i * 17, 100 + i * 7]
    return {"world": world, "pixels": pixels, "camera": camera, "truth": {"R": R, "t": t}}


def _project_fixture(camera, R, t, X):
    q = [t[j] + R[j * 3] * X[0] + R[j * 3 + 1] * X[1] + R[j * 3 + 2] * X[2] for j in range(3)]
    x, y = q[0] / q[2], q[1] / q[2]
    r2 = x * x + y * y
    d = 1 + camera["k1"] * r2 + camera["k2"] * r2 * r2
    return camera["fx"] * x * d + camera["cx"], camera["fy"] * y * d + camera["cy"]


def bundle_fixture(count=40, views=4, outlier=False, shift=(0, 0, 0)):
    data = pose_fixture(count=count, noise=0, outliers=0)
    cam = data["camera"]
    model = {"views": [], "landmarks": []}
    truth = []
    for c in range(views):
        a = 0.02 * c
        ca, sa = math.cos(a), math.sin(a)
        R = [ca, 0, sa, 0, 1, 0, -sa, 0, ca]
        t = [-0.32 * c, 0.02 * math.sin(c), 0.015 * c]
        truth.append((R, t))
        perturbed_angle = a + (0.004 * math.sin(c) if c else 0)
        cp, sp = math.cos(perturbed_angle), math.sin(perturbed_angle)
        Rp = [cp, 0, sp, 0, 1, 0, -sp, 0, cp]
        tp = [t[j] + (0.015 * math.sin(c + j) if c else 0)
              - Rp[j * 3] * shift[0] - Rp[j * 3 + 1] * shift[1] - Rp[j * 3 + 2] * shift[2]
              for j in range(3)]
        model["views"].append({"id": 10 + 10 * c, "camera": dict(cam),
                               "pose": {"R": f64(Rp), "t": f64(tp)}})
    for p in range(count):
        X = list(data["world"][p * 3:p * 3 + 3])
        observations = []
        for c, (R, t) in enumerate(truth):
            q = [t[j] + R[j * 3] * X[0] + R[j * 3 + 1] * X[1] + R[j * 3 + 2] * X[2] for j in range(3)]
            x, y = q[0] / q[2], q[1] / q[2]
            r2 = x * x + y * y
            d = 1 + cam["k1"] * r2 + cam["k2"] * r2 * r2
            pixel = [cam["fx"] * x * d + cam["cx"] + 0.1 * math.sin(p * 3 + c),
                     cam["fy"] * y * d + cam["cy"] + 0.1 * math.cos(p + c * 3)]
            if outlier and p == 0 and c == 2:
                pixel = [pixel[0] + 40, pixel[1] - 20]
            observations.append({"viewId": model["views"][c]["id"], "featureId": p, "pixel": pixel})
        model["landmarks"].append({
            "trackId": p,
            "xyz": f64([X[j] + shift[j] + 0.035 * math.sin(p + j) for j in range(3)]),
            "observations": observations,
        })
    return model


def skew_bundle_fixture(views=17, count=512):
    """scripts/benchmark-ba-camera-products.mjs:80-85: keep cameras 0, 1 and one more."""
    model = bundle_fixture(count=count, views=views)
    for i, p in enumerate(model["landmarks"]):
        extra = 2 + (i % (views - 2))
        p["observations"] = [o for c, o in enumerate(p["observations"]) if c < 2 or c == extra]
    return model


def ring_bundle_fixture(views=320, points=4800, track=5, global_points=0):
    nxt = XorShift32(977)
    camera = {"fx": 900, "fy": 920, "cx": 480, "cy": 270, "k1": -0.05, "k2": 0.005}

    def rotation(a):
        return [math.cos(a), 0, math.sin(a), 0, 1, 0, -math.sin(a), 0, math.cos(a)]

    truth, model = [], {"views": [], "landmarks": []}
    for c in range(views):
        a = (2 * math.pi * c) / views
        R, t = rotation(a), [0, 0, 10]
        truth.append((R, t))
        Rp = rotation(a + (0.002 * math.sin(c) if c else 0))
        tp = [t[j] + (0.01 * math.sin(c + j) if c else 0) for j in range(3)]
        model["views"].append({"id": 1000 + c, "camera": dict(camera),
                               "pose": {"R": f64(Rp), "t": f64(tp)}})
    features = [0] * views
    for p in range(points):
        X = [(nxt() - 0.5) * 3, (nxt() - 0.5) * 3, (nxt() - 0.5) * 3]
        observations = []
        for k in range(views if p < global_points else track):
            c = (p + k) % views
            px, py = _project_fixture(camera, truth[c][0], truth[c][1], X)
            observations.append({"viewId": model["views"][c]["id"], "featureId": features[c],
                                 "pixel": [px + 0.1 * math.sin(p * 3 + c), py + 0.1 * math.cos(p + c * 3)]})
            features[c] += 1
        model["landmarks"].append({"trackId": p, "xyz": f64([X[j] + 0.02 * math.sin(p + j) for j in range(3)]),
                                   "observations": observations})
    return model


def bundle_metrics(model, huber=2.0):
    """bundleMetrics of geometry-cases.mjs:220-249 (the tests' independent cost)."""
    views = {v["id"]: v for v in model["views"]}
    cost = squares = 0.0
    count = 0
    for p in model["landmarks"]:
        for o in p["observations"]:
            v = views[o["viewId"]]
            k, pose, X = v["camera"], v["pose"], p["xyz"]
            q = [pose["R"][j * 3] * X[0] + pose["R"][j * 3 + 1] * X[1] + pose["R"][j * 3 + 2] * X[2] + pose["t"][j]
                 for j in range(3)]
            if not q[2] > 0:
                return {"cost": math.inf, "rmse": math.inf}
            x, y = q[0] / q[2], q[1] / q[2]
            r2 = x * x + y * y
            d = 1 + k.get("k1", 0) * r2 + k.get("k2", 0) * r2 * r2
            error = math.hypot(k["fx"] * x * d + k["cx"] - o["pixel"][0], k["fy"] * y * d + k["cy"] - o["pixel"][1])
            squares += error * error
            cost += error * error if error <= huber else 2 * huber * error - huber * huber
            count += 1
    return {"cost": cost, "rmse": math.sqrt(squares / count), "observations": count}


# ---- joint-focal-cases.mjs ---------------------------------------------------------------------

def joint_focal_fixture(views=6, points=60, focal_scale=0.75, noise=0, radial=True):
    def multiply(a, b):
        return [sum_js([a[(i // 3) * 3 + k] * b[k * 3 + (i % 3)] for k in range(3)]) for i in range(9)]

    def rotation(x, y, z):
        cx, sx, cy, sy, cz, sz = math.cos(x), math.sin(x), math.cos(y), math.sin(y), math.cos(z), math.sin(z)
        return multiply([cz, -sz, 0, sz, cz, 0, 0, 0, 1],
                        multiply([cy, 0, sy, 0, 1, 0, -sy, 0, cy], [1, 0, 0, 0, cx, -sx, 0, sx, cx]))

    camera = {"fx": 800, "fy": 840, "cx": 511.5, "cy": 383.5,
              "k1": -0.04 if radial else 0, "k2": 0.004 if radial else 0}
    truth = {"views": [], "landmarks": []}
    inp = {"views": [], "landmarks": []}
    for c in range(views):
        angles = [0.03 * math.sin(c), 0.075 * c, 0.035 * math.sin(c * 0.7)]
        R = rotation(*angles)
        t = [-0.4 * c, 0.12 * math.sin(c * 1.3), 0.08 * (math.cos(c) - 1)]
        truth["views"].append({"id": 10 + 10 * c, "camera": dict(camera), "pose": {"R": f64(R), "t": f64(t)}})
        pa = [v + (0.003 * math.sin(c + j) if c else 0) for j, v in enumerate(angles)]
        inp["views"].append({
            "id": 10 + 10 * c,
            "camera": {**camera, "fx": camera["fx"] * focal_scale, "fy": camera["fy"] * focal_scale},
            "pose": {"R": f64(rotation(*pa)),
                     "t": f64([v + (0.012 * math.sin(c + j) if c else 0) for j, v in enumerate(t)])},
        })
    nxt = Lcg(117)
    for p in range(points):
        X = [(nxt() - 0.5) * 3, (nxt() - 0.5) * 2, 3 + nxt() * 6]
        observations = []
        for c, v in enumerate(truth["views"]):
            R, t = v["pose"]["R"], v["pose"]["t"]
            q = [t[j] + sum_js([R[j * 3 + k] * X[k] for k in range(3)]) for j in range(3)]
            x, y = q[0] / q[2], q[1] / q[2]
            r = x * x + y * y
            d = 1 + camera["k1"] * r + camera["k2"] * r * r
            observations.append({"viewId": v["id"], "featureId": p, "pixel": [
                camera["fx"] * x * d + camera["cx"] + noise * math.sin(p + c),
                camera["fy"] * y * d + camera["cy"] + noise * math.cos(p * 2 + c)]})
        truth["landmarks"].append({"trackId": p, "xyz": f64(X), "observations": observations})
        inp["landmarks"].append({"trackId": p, "xyz": f64([v + 0.025 * math.sin(p + j) for j, v in enumerate(X)]),
                                 "observations": observations})
    return {"input": inp, "truth": truth, "expectedScale": 1 / focal_scale}


def sum_js(values):
    """[..].reduce((s, v) => s + v, 0): left to right from 0."""
    s = 0.0
    for v in values:
        s = s + v
    return s


# ---- tests/scene.ts and tests/bundle-adjustment.test.ts ----------------------------------------

def _multiply3(a, b):
    return [sum_js([a[r * 3 + k] * b[k * 3 + c] for k in range(3)]) for r in range(3) for c in range(3)]


def rotation_exp(w):
    """rotationExp, src/geometry/pose.ts:46-56."""
    x, y, z = w
    theta = math.hypot(x, y, z)
    a = 1 - (theta * theta) / 6 if theta < 1e-7 else math.sin(theta) / theta
    b = 0.5 - (theta * theta) / 24 if theta < 1e-7 else (1 - math.cos(theta)) / (theta * theta)
    W = [0, -z, y, z, 0, -x, -y, x, 0]
    W2 = _multiply3(W, W)
    return [(1 if i % 4 == 0 else 0) + a * W[i] + b * W2[i] for i in range(9)]


def transform_point(R, t, X):
    """transformPoint, src/geometry/pose.ts:34-39."""
    return [R[i * 3] * X[0] + R[i * 3 + 1] * X[1] + R[i * 3 + 2] * X[2] + t[i] for i in range(3)]


def update_pose(R, t, delta):
    """updatePose, src/geometry/pose.ts:58-62."""
    dR = rotation_exp(delta[:3])
    rotated = transform_point(dR, [0, 0, 0], t)
    return _multiply3(dR, R), [rotated[i] + delta[i + 3] for i in range(3)]


def camera_center(R, t):
    return [-R[i] * t[0] - R[i + 3] * t[1] - R[i + 6] * t[2] for i in range(3)]


def scene(count=90, views=6, noise=0, seed=731, camera=None):
    camera = dict(camera or {"fx": 850, "fy": 870, "cx": 480, "cy": 270})
    rng = seeded_random(seed)
    points = [[(rng() - 0.5) * 4, (rng() - 0.5) * 3, 4 + rng() * 5] for _ in range(count)]
    registered = []
    for i in range(views):
        R = rotation_exp([0.008 * i, -0.018 * i, 0.003 * i])
        C = [i * 0.32, math.sin(i) * 0.04, 0.02 * i]
        t = [-x for x in transform_point(R, [0, 0, 0], C)]
        registered.append({"id": i * 10 + 10, "camera": dict(camera), "pose": {"R": f64(R), "t": f64(t)}})
    k = {"k1": 0, "k2": 0, **camera}
    keypoints = []
    for v in registered:
        kp = []
        for X in points:
            q = transform_point(v["pose"]["R"], v["pose"]["t"], X)
            x, y = q[0] / q[2], q[1] / q[2]
            r2 = x * x + y * y
            d = 1 + k["k1"] * r2 + k["k2"] * r2 * r2
            px, py = k["fx"] * x * d + k["cx"], k["fy"] * y * d + k["cy"]
            kp.append((px + (rng() - 0.5) * noise * 2, py + (rng() - 0.5) * noise * 2))
        keypoints.append(kp)
    reconstruction = {
        "views": registered,
        "landmarks": [{"trackId": i, "xyz": f64(X), "observations": [
            {"viewId": v["id"], "featureId": i, "pixel": [keypoints[c][i][0], keypoints[c][i][1]]}
            for c, v in enumerate(registered)]} for i, X in enumerate(points)],
    }
    return reconstruction, rng


def perturbed():
    reconstruction, rng = scene(count=70, views=5, noise=0.2)
    views = []
    for i, v in enumerate(reconstruction["views"]):
        if i == 0:
            views.append(v)
            continue
        delta = [(rng() - 0.5) * s * 2 for s in [0.005, 0.005, 0.005, 0.02, 0.02, 0.02]]
        R, t = update_pose(v["pose"]["R"], v["pose"]["t"], delta)
        views.append({**v, "pose": {"R": f64(R), "t": f64(t)}})
    landmarks = [{**p, "xyz": f64([x + (rng() - 0.5) * 0.08 for x in p["xyz"]])} for p in reconstruction["landmarks"]]
    return {"views": views, "landmarks": landmarks}


def inverse_depth_scene(count=4):
    """inverseDepthScene (tests/typeshade/inverse-depth-cases.mjs:1-56): `count` views turning about
    y along a slightly curved path, 25 points 5-7.4 in front, every point seen by every view,
    pixels projected exactly (k1 = -0.03)."""
    camera = {"fx": 800, "fy": 760, "cx": 320, "cy": 240, "k1": -0.03}
    views = []
    for i in range(count):
        y = i * 0.07
        c, s = math.cos(y), math.sin(y)
        R = f64([c, 0, s, 0, 1, 0, -s, 0, c])
        C = [i * 0.32, math.sin(i) * 0.04, 0.02 * i * i]
        t = f64([-R[3 * r] * C[0] - R[3 * r + 1] * C[1] - R[3 * r + 2] * C[2] for r in range(3)])
        views.append({"id": i, "camera": camera, "pose": {"R": R, "t": t}})
    points = [[math.sin(i * 1.3), math.cos(i * 1.7) * 0.8, 5 + (i % 7) * 0.4] for i in range(25)]

    def project(v, X):
        R, t = v["pose"]["R"], v["pose"]["t"]
        q = [R[3 * r] * X[0] + R[3 * r + 1] * X[1] + R[3 * r + 2] * X[2] + t[r] for r in range(3)]
        x, y = q[0] / q[2], q[1] / q[2]
        d = 1 + camera["k1"] * (x * x + y * y)
        return [camera["fx"] * x * d + camera["cx"], camera["fy"] * y * d + camera["cy"]]

    return {"views": views,
            "landmarks": [{"trackId": tid, "xyz": f64(xyz),
                           "observations": [{"viewId": v["id"], "featureId": tid, "pixel": project(v, xyz)}
                                            for v in views]}
                          for tid, xyz in enumerate(points)]}


def inverse_depth_long_scene(count=24):
    """inverseDepthLongScene (tests/typeshade/inverse-depth-cases.mjs:58-85): `count` translated views
    with identity rotation; each run of 4 consecutive views sees its own copy of the first 12 points
    of inverse_depth_scene."""
    source = inverse_depth_scene()
    camera = source["views"][0]["camera"]
    views = [{"id": i, "camera": camera,
              "pose": {"R": f64([1, 0, 0, 0, 1, 0, 0, 0, 1]),
                       "t": f64([-0.03 * i, -0.04 * math.sin(i), -0.02 * math.sin(i * 0.2)])}}
             for i in range(count)]
    landmarks = []
    for start in range(count - 3):
        for j, p in enumerate(source["landmarks"][:12]):
            obs = []
            for v in views[start:start + 4]:
                q = [x + v["pose"]["t"][k] for k, x in enumerate(p["xyz"])]
                x, y = q[0] / q[2], q[1] / q[2]
                d = 1 + camera["k1"] * (x * x + y * y)
                obs.append({"viewId": v["id"], "featureId": start * 12 + j,
                            "pixel": [camera["fx"] * x * d + camera["cx"], camera["fy"] * y * d + camera["cy"]]})
            landmarks.append({"trackId": start * 12 + j, "xyz": p["xyz"], "observations": obs})
    return {"views": views, "landmarks": landmarks}

