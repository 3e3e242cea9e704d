"""The adjoint of a converged bundle adjustment (``tba_bundle_vjp``): the vector-Jacobian product
of the solution with respect to the observed pixels and two shared intrinsics, by implicit
differentiation through the exact Hessian, and the exact-Newton steps that share its solver.

No counterpart in the reference.  The solution it differentiates is the one ``bundle_adjust_gpu``
/ ``solve_packed`` returns with fixed intrinsics (refineSharedFocal off): poses (R row-major, t)
and points, in the gauge the solver keeps (fixed cameras, and with one fixed camera the
anchor-to-scale-camera baseline).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .bundle import DeviceError, RangeError, ShadeDevice


def bundle_vjp(device: ShadeDevice, C: int, P: int, M: int, scene: np.ndarray, index: np.ndarray,
               cotangent: np.ndarray | None, *, anchor: int = 0, scale_view: int = 1, newton_steps: int = 0,
               max_cg: int = 5000, tolerance: float = 1e-12, huber: float = 2.0, want_solution: bool = False,
               time_products: bool = False):
    """Returns (pixels_bar (M x 2) or None, intrinsics_bar (d/ds, d/dk1) or None, solution or None,
    report dict).  `scene` holds the evaluation point (poses and points) and the observations.
    `time_products` brackets each one-pass Schur product with CUDA events (report product_ms)."""
    lib = _lib.load()
    scene = np.ascontiguousarray(scene, dtype=np.float64)
    index = np.ascontiguousarray(index, dtype=np.uint32)
    flags = _lib.TBA_VJP_FLAG_TIME_PRODUCTS if time_products else 0
    ctl = _lib.VjpControl(C, P, M, anchor, scale_view, newton_steps, max_cg, flags, huber, tolerance)
    n_theta = 12 * C + 3 * P
    report = _lib.VjpReport()
    ybar = np.zeros(2 * M) if cotangent is not None else None
    kbar = np.zeros(2) if cotangent is not None else None
    sol = np.zeros(n_theta) if want_solution else None
    cot = None if cotangent is None else np.ascontiguousarray(cotangent, dtype=np.float64)
    null_d = ctypes.POINTER(ctypes.c_double)()
    status = lib.tba_bundle_vjp(device.handle, ctypes.byref(ctl), _lib.dptr(scene), scene.size, _lib.uptr(index),
                                index.size, _lib.dptr(cot) if cot is not None else null_d,
                                cot.size if cot is not None else 0, _lib.dptr(ybar) if ybar is not None else null_d,
                                ybar.size if ybar is not None else 0, _lib.dptr(kbar) if kbar is not None else null_d,
                                _lib.dptr(sol) if sol is not None else null_d, sol.size if sol is not None else 0,
                                ctypes.byref(report))
    if status != _lib.TBA_OK:
        message = lib.tba_last_error(device.handle).decode()
        if status in (_lib.TBA_ERROR_ARGUMENT, _lib.TBA_ERROR_BUDGET):
            raise RangeError(message)
        raise DeviceError(f"tba_bundle_vjp failed ({status}): {message}")
    return (None if ybar is None else ybar.reshape(M, 2)), kbar, sol, report.as_dict()


def newton_solution(device: ShadeDevice, C: int, P: int, M: int, scene: np.ndarray, index: np.ndarray, *,
                    anchor: int = 0, scale_view: int = 1, steps: int = 3, max_cg: int = 5000,
                    tolerance: float = 1e-13, huber: float = 2.0):
    """`steps` exact-Newton steps from the scene's poses and points; returns (solution, report)."""
    _, _, sol, rep = bundle_vjp(device, C, P, M, scene, index, None, anchor=anchor, scale_view=scale_view,
                                newton_steps=steps, max_cg=max_cg, tolerance=tolerance, huber=huber,
                                want_solution=True)
    return sol, rep
