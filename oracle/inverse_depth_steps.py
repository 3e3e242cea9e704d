"""CPU restatement of the reference's inverse-depth bundle adjustment host steps (test
infrastructure only; nothing in typecv_b200 imports it).

Follows, loop for loop and in the reference's order of operations, `inverseDepthBundleSteps`
(src/sfm/depth/inverse-depth-bundle.ts:196-565) with `cameraBlocks` (:135-177), `reduce` (:582-616),
`chooseSchurSolver` (:618-654), `denseSchurFactor` (:655-668), `pointMarginal` (:669-700) and
`positiveInverse` (:91-121); `SparseSymmetric` and `factorSparseSchur`
(src/sfm/depth/sparse-schur.ts:1-208); and the chart helpers of src/geometry/inverse-depth.ts
(`inverseDepthCovariance` :157-164, `inverseDepthPoint` :77-87, `rescaleInverseDepth` :133-154) and
src/geometry/pose.ts (`rotationExp`, `updatePose`, `validatePose`).  The steps are a generator that
yields measurement jobs and takes one linearisation (or None) per measurement, as the reference's
does; `oracle.inverse_depth.bundle_adjust_inverse_depth` answers them with the CPU linearisation
(the reference's CPU `bundleAdjustInverseDepth`).
"""
from __future__ import annotations

import copy
import math
from typing import Any, Generator

import numpy as np

from oracle.bundle_adjust import RangeError, _safe_int, validate_reconstruction
from oracle.inverse_depth import camera_center, initialize_inverse_depth, transform_point


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


class SparseSymmetric:
    """SparseSymmetric (sparse-schur.ts:2-70)."""

    def __init__(self, size: int, max_entries: int, dense: bool = False):
        self.size = size
        self.max_entries = max_entries
        self.entries = 0
        self.rows: list[dict[int, float]] = [dict() for _ in range(size)]
        self.values: list[float] | None = [0.0] * (size * size) if dense else None
        self.pattern: bytearray | None = bytearray(size * size) if dense else None

    @property
    def dense_storage(self) -> bool:
        return self.values is not None

    def add(self, i: int, j: int, value: float) -> None:
        if i > j:
            i, j = j, i
        if self.values is not None:
            at = i * self.size + j
            if not self.pattern[at]:
                if self.entries >= self.max_entries:
                    raise RangeError("Schur nonzero budget exceeded")
                self.pattern[at] = 1
                self.entries += 1
            self.values[at] += value
            return
        row = self.rows[i]
        old = row.get(j)
        if old is None:
            if self.entries >= self.max_entries:
                raise RangeError("Schur nonzero budget exceeded")
            self.entries += 1
            row[j] = 0.0 + value
        else:
            row[j] = old + value

    def get(self, i: int, j: int) -> float:
        if i > j:
            i, j = j, i
        if self.values is not None:
            return self.values[i * self.size + j]
        return self.rows[i].get(j, 0.0)

    def copy(self) -> "SparseSymmetric":
        out = SparseSymmetric(self.size, self.max_entries)
        if self.values is not None:
            out.values = list(self.values)
            out.pattern = bytearray(self.pattern)
            out.entries = self.entries
            return out
        for i in range(self.size):
            for j, v in self.rows[i].items():
                out.add(i, j, v)
        return out

    def dense(self) -> np.ndarray:
        n = self.size
        if self.values is not None:
            out = np.array(self.values, dtype=np.float64).reshape(n, n)
            upper = np.triu(out)
            return upper + np.triu(upper, 1).T
        out = np.zeros((n, n))
        for i in range(n):
            for j, v in self.rows[i].items():
                out[i, j] = out[j, i] = v
        return out


def positive_inverse(A, n: int) -> np.ndarray | None:
    """positiveInverse (inverse-depth-bundle.ts:91-121): the inverse of an SPD matrix (row-major,
    n x n) by a Cholesky factor of its diagonally equilibrated form; None unless every pivot
    exceeds 1e-10."""
    if not n:
        return np.zeros(0)
    A = [float(x) for x in np.asarray(A, dtype=np.float64).ravel()]
    d = [math.sqrt(A[i * n + i]) if A[i * n + i] >= 0 else math.nan for i in range(n)]
    if any(not (v > 0 and math.isfinite(v)) for v in d):
        return None
    L = [0.0] * (n * n)
    for i in range(n):
        for j in range(i + 1):
            a = A[i * n + j] / (d[i] * d[j])
            for k in range(j):
                a -= L[i * n + k] * L[j * n + k]
            if i == j:
                if not a > 1e-10:
                    return None
                L[i * n + i] = math.sqrt(a)
            else:
                L[i * n + j] = a / L[j * n + j]
    inv = [0.0] * (n * n)
    for c in range(n):
        x = [0.0] * n
        for i in range(n):
            v = 1.0 if i == c else 0.0
            for j in range(i):
                v -= L[i * n + j] * x[j]
            x[i] = v / L[i * n + i]
        for i in range(n - 1, -1, -1):
            v = x[i]
            for j in range(i + 1, n):
                v -= L[j * n + i] * x[j]
            x[i] = v / L[i * n + i]
        for i in range(n):
            inv[i * n + c] = x[i] / (d[i] * d[c])
    return np.array(inv)


def multiply_vector(A, b, n: int) -> list[float]:
    out = []
    for i in range(n):
        v = 0.0
        for j in range(n):
            v += A[i * n + j] * b[j]
        out.append(v)
    return out


class DenseFactor:
    """denseSchurFactor (inverse-depth-bundle.ts:655-668)."""
    storage = "dense"

    def __init__(self, inverse: np.ndarray, n: int):
        self.inverse = [float(x) for x in inverse]
        self.n = n
        self.entries = len(self.inverse)
        self.selected_entries = len(self.inverse)

    def solve(self, rhs) -> list[float]:
        return multiply_vector(self.inverse, rhs, self.n)

    def covariance(self, i: int, j: int) -> float:
        return self.inverse[i * self.n + j]


def dense_schur_factor(S: SparseSymmetric, max_entries: int) -> DenseFactor | None:
    if S.size * S.size > max_entries:
        raise RangeError("Dense Schur factor budget exceeded")
    inverse = positive_inverse(S.dense(), S.size)
    return None if inverse is None else DenseFactor(inverse, S.size)


class SparseFactor:
    """The factor returned by factorSparseSchur (sparse-schur.ts:179-207)."""
    storage = "sparse"

    def __init__(self, n, scale, order, position, pivots, columns, entries):
        self.n, self.scale, self.order, self.position = n, scale, order, position
        self.pivots, self.columns, self.entries = pivots, columns, entries
        self._selected: list[dict[int, float]] | None = None

    @property
    def selected_entries(self) -> int:
        return self.entries if self._selected is not None else 0

    def _raw(self, i: int, j: int) -> float:
        if self.position[i] > self.position[j]:
            i, j = j, i
        value = self._selected[i].get(j)
        if value is None:
            raise RuntimeError("Selected inverse request is outside the factor pattern")
        return value

    def _select(self) -> None:
        if self._selected is not None:
            return
        self._selected = [dict() for _ in range(self.n)]
        for step in range(self.n - 1, -1, -1):
            pivot = self.order[step]
            rows, values = self.columns[step]
            root = self.pivots[step]
            for j in rows:
                value = 0.0
                for k in range(len(rows)):
                    value -= (values[k] * self._raw(rows[k], j)) / root
                self._selected[pivot][j] = value
            value = 1 / (root * root)
            for k in range(len(rows)):
                value -= (values[k] * self._raw(pivot, rows[k])) / root
            if not (value > 0 and math.isfinite(value)):
                raise RangeError("Selected Schur inverse is numerically invalid")
            self._selected[pivot][pivot] = value

    def solve(self, rhs) -> list[float]:
        x = [float(v) / self.scale[i] for i, v in enumerate(rhs)]
        for step in range(self.n):
            pivot = self.order[step]
            rows, values = self.columns[step]
            x[pivot] /= self.pivots[step]
            for j in range(len(rows)):
                x[rows[j]] -= values[j] * x[pivot]
        for step in range(self.n - 1, -1, -1):
            pivot = self.order[step]
            rows, values = self.columns[step]
            for j in range(len(rows)):
                x[pivot] -= values[j] * x[rows[j]]
            x[pivot] /= self.pivots[step]
        return [v / self.scale[i] for i, v in enumerate(x)]

    def covariance(self, i: int, j: int) -> float:
        self._select()
        return self._raw(i, j) / (self.scale[i] * self.scale[j])


def factor_sparse_schur(A: SparseSymmetric, max_factor_entries: int) -> SparseFactor | None:
    """factorSparseSchur (sparse-schur.ts:89-208)."""
    if A.dense_storage:
        raise RuntimeError("Sparse factor requires sparse matrix storage")
    if A.entries > max_factor_entries:
        raise RangeError("Schur factor nonzero budget exceeded")
    n = A.size
    scale = []
    for i in range(n):
        g = A.get(i, i)
        scale.append(math.sqrt(g) if g >= 0 else math.nan)
    if any(not (v > 0 and math.isfinite(v)) for v in scale):
        return None
    work: list[dict[int, float]] = [dict() for _ in range(n)]
    diagonal = [1.0] * n
    for i in range(n):
        for j, value in A.rows[i].items():
            if i != j:
                v = value / (scale[i] * scale[j])
                work[i][j] = v
                work[j][i] = v
    order = [0] * n
    position = [-1] * n
    pivots = [0.0] * n
    columns: list[tuple[list[int], list[float]]] = []
    entries = n
    structural = A.entries
    if entries > max_factor_entries:
        raise RangeError("Schur factor nonzero budget exceeded")
    for step in range(n):
        pivot, degree = -1, math.inf
        for i in range(n):
            if position[i] == -1 and len(work[i]) < degree:
                degree = len(work[i])
                pivot = i
        if pivot < 0 or not (diagonal[pivot] > 1e-10 and math.isfinite(diagonal[pivot])):
            return None
        order[step] = pivot
        position[pivot] = step
        root = math.sqrt(diagonal[pivot])
        neighbors = sorted(work[pivot].keys())
        values = [work[pivot][j] / root for j in neighbors]
        entries += len(neighbors)
        if entries > max_factor_entries:
            raise RangeError("Schur factor nonzero budget exceeded")
        pivots[step] = root
        columns.append((neighbors, values))
        for a in range(len(neighbors)):
            i, li = neighbors[a], values[a]
            diagonal[i] -= li * li
            work[i].pop(pivot, None)
            for b in range(a + 1, len(neighbors)):
                j = neighbors[b]
                old = work[i].get(j)
                if old is None:
                    structural += 1
                    if structural > max_factor_entries:
                        raise RangeError("Schur fill nonzero budget exceeded")
                v = (old if old is not None else 0.0) - li * values[b]
                work[i][j] = v
                work[j][i] = v
        work[pivot].clear()
    return SparseFactor(n, scale, order, position, pivots, columns, entries)


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
