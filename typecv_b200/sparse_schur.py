"""Host FP64 reduced-camera-system storage and factorisations of the inverse-depth bundle
adjustment (src/sfm/depth/sparse-schur.ts:1-208 and the dense helpers of
src/sfm/depth/inverse-depth-bundle.ts:91-128, 655-676).

``SparseSymmetric`` keeps the upper triangle, either as one ordered map per row or, for the dense
solver, as a full array with a pattern of touched entries; both count entries against a budget.
``factor_sparse_schur`` is an exact sparse Cholesky on the diagonally equilibrated matrix with a
greedy minimum-degree order and Takahashi selected inversion for covariances;
``dense_schur_factor`` inverts the whole matrix by an equilibrated Cholesky.  The camera systems
here have at most a few thousand unknowns and are solved once per Levenberg-Marquardt step on the
host, as in the reference, where the order of every sum is kept.
"""
from __future__ import annotations

import math

import numpy as np

from .bundle import RangeError


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
