"""Batched local-window bundle adjustment: many independent problems in one persistent launch.

The reference's mapper adjusts its local windows one ``bundleAdjustGpu`` call at a time
(src/sfm/mapper/mapper.ts:859-925 over the windows planned by src/sfm/bundle/local-bundle.ts:17-208).
``batch_adjust`` hands a whole list of such problems, each already packed as the reference packs one
call (packBundleScene / bundleIndexLayout, src/sfm/bundle/gpu/bundle-host.ts:121-218), to
``tba_batch_adjust`` in libtba.so and returns each problem's result record exactly as
``tba_bundle_adjust`` (``solve_packed``) would for the same arrays and options.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .bundle import BUNDLE_SOLVER_STALL_TOLERANCE, DeviceError, RangeError, ShadeDevice

_PRECISION = {"fp64": _lib.TBA_PRECISION_FP64, "mixed": _lib.TBA_PRECISION_MIXED}


@dataclass
class PackedProblem:
    """One problem in the reference's packed layout."""
    C: int
    P: int
    M: int
    scene: np.ndarray  # 18C + 3P + 2M doubles
    index: np.ndarray  # 3M + P + 2C + 2 words
    anchor: int = 0
    scale_view: int = 1


def output_size(C: int, P: int, shared_focal: bool) -> int:
    return 12 * C + 3 * P + 26 + (1 if shared_focal else 0)


@dataclass
class PackedBatch:
    """The concatenated arrays and the problem table of a batch (reusable across calls)."""
    scene: np.ndarray
    index: np.ndarray
    table: ctypes.Array
    output_offsets: np.ndarray
    output_len: int
    sizes: list


def pack_batch(problems: list[PackedProblem], shared_focal: bool, *, scene: np.ndarray | None = None,
               index: np.ndarray | None = None) -> PackedBatch:
    """Concatenate the problems' arrays (into `scene` / `index` when given, e.g. pinned buffers)."""
    n_scene = sum(p.scene.size for p in problems)
    n_index = sum(p.index.size for p in problems)
    scene = np.empty(n_scene) if scene is None else scene[:n_scene]
    index = np.empty(n_index, dtype=np.uint32) if index is None else index[:n_index]
    table = (_lib.BatchProblem * len(problems))()
    out_offsets = np.zeros(len(problems), dtype=np.int64)
    s = x = o = 0
    for k, p in enumerate(problems):
        scene[s:s + p.scene.size] = p.scene
        index[x:x + p.index.size] = p.index
        table[k] = _lib.BatchProblem(p.C, p.P, p.M, p.anchor, p.scale_view, 0, s, x, o)
        out_offsets[k] = o
        s += p.scene.size
        x += p.index.size
        o += output_size(p.C, p.P, shared_focal)
    return PackedBatch(scene, index, table, out_offsets, o, [(p.C, p.P) for p in problems])


def batch_shapes() -> list[tuple[int, int]]:
    """The solver's launch shapes: (threads per block, compiled blocks per SM)."""
    lib = _lib.load()
    out = []
    for k in range(lib.tba_batch_shapes()):
        t, b = ctypes.c_uint32(), ctypes.c_uint32()
        lib.tba_batch_shape(k, ctypes.byref(t), ctypes.byref(b))
        out.append((t.value, b.value))
    return out


def max_cameras() -> int:
    return int(_lib.load().tba_batch_max_cameras())


def batch_adjust(device: ShadeDevice, problems: list[PackedProblem] | PackedBatch, *, iterations: int = 10,
                 max_cg: int | None = None, shared_focal: bool = False, precision: str = "mixed",
                 huber: float = 2.0, tolerance: float = 1e-6, stall: float = BUNDLE_SOLVER_STALL_TOLERANCE,
                 schedule: int = 0, output: np.ndarray | None = None):
    """Solve every problem; returns (list of result records, report dict).

    ``schedule`` 0 lets the library's autotuner pick the launch shape; k >= 1 forces shape k - 1.
    ``max_cg`` defaults to the reference's default for the largest problem (bundle-host.ts:49-65).
    """
    lib = _lib.load()
    packed = problems if isinstance(problems, PackedBatch) else pack_batch(problems, shared_focal)
    if max_cg is None:
        cmax = max(C for C, _ in packed.sizes)
        max_cg = min(256, max(32, 12 * cmax + 1)) if shared_focal else min(96, max(24, 12 * cmax))
    if precision not in _PRECISION:
        raise RangeError("precision must be 'fp64' or 'mixed'")
    control = _lib.BatchControl(iterations, max_cg, int(bool(shared_focal)), _PRECISION[precision], schedule, 0,
                                huber, tolerance, stall)
    if output is None:
        output = np.zeros(packed.output_len)
    report = _lib.BatchReport()
    status = lib.tba_batch_adjust(device.handle, ctypes.byref(control), packed.table, len(packed.sizes),
                                  _lib.dptr(packed.scene), packed.scene.size, _lib.uptr(packed.index),
                                  packed.index.size, _lib.dptr(output), output.size, ctypes.byref(report))
    if status != _lib.TBA_OK:
        message = lib.tba_last_error(device.handle).decode()
        if status in (_lib.TBA_ERROR_ARGUMENT, _lib.TBA_ERROR_BUDGET):
            raise RangeError(message)
        raise DeviceError(f"tba_batch_adjust failed ({status}): {message}")
    records = [output[o:o + output_size(C, P, shared_focal)] for o, (C, P) in zip(packed.output_offsets, packed.sizes)]
    return records, report.as_dict()
