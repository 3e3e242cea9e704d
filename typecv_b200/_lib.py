"""ctypes binding of libtba.so (include/tba.h).

The library is loaded from this package's directory only.  There is no fallback: when the
library is missing or fails to load, every entry point raises ``LibraryError``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtba.so")

TBA_OK, TBA_ERROR_ARGUMENT, TBA_ERROR_BUDGET, TBA_ERROR_CUDA, TBA_ERROR_INTERNAL = range(5)
TBA_PRECISION_FP64, TBA_PRECISION_MIXED = 0, 1
TBA_FLAG_TIME_PRODUCTS = 1
TBA_FLAG_PRODUCT_ERROR = 2
TBA_FLAG_HOST_PCG_LOOP = 4
TBA_VJP_FLAG_TIME_PRODUCTS = 1
TBA_WAIT_LIMIT_DEFAULT = 4194304

# Every symbol include/tba.h declares.
EXPORTS = ("tba_scene_size", "tba_index_size", "tba_output_size", "tba_device_open", "tba_device_close",
           "tba_last_error", "tba_bundle_adjust", "tba_scene_cost_noalloc", "tba_batch_max_cameras",
           "tba_batch_shapes", "tba_batch_shape", "tba_batch_adjust", "tba_bundle_vjp",
           "tba_evaluate_observations", "tba_scene_create", "tba_scene_destroy", "tba_scene_adjust",
           "tba_scene_write", "tba_scene_read", "tba_linearize_inverse_depth", "tba_device_set_wait_limit")


class LibraryError(RuntimeError):
    """libtba.so is missing or unusable: the operator has no other implementation."""


class Control(ctypes.Structure):
    _fields_ = [
        ("cameras", ctypes.c_uint32), ("points", ctypes.c_uint32),
        ("directional_points", ctypes.c_uint32), ("observations", ctypes.c_uint32),
        ("anchor", ctypes.c_uint32), ("scale_view", ctypes.c_uint32),
        ("iterations", ctypes.c_uint32), ("max_cg", ctypes.c_uint32),
        ("shared_focal", ctypes.c_uint32), ("precision", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("huber", ctypes.c_double), ("cg_tolerance", ctypes.c_double), ("stall_tolerance", ctypes.c_double),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("solve_ms", ctypes.c_double), ("upload_ms", ctypes.c_double), ("download_ms", ctypes.c_double),
        ("wall_ms", ctypes.c_double), ("product_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint32), ("lm_iterations", ctypes.c_uint32),
        ("cg_iterations", ctypes.c_uint32), ("product_launches", ctypes.c_uint32), ("engine", ctypes.c_uint32),
        ("product_blocks", ctypes.c_uint32), ("refinements", ctypes.c_uint32),
        ("fp64_iterations", ctypes.c_uint32), ("check_ms", ctypes.c_double),
        ("product_error_max", ctypes.c_double), ("product_error_norm", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchProblem(ctypes.Structure):
    _fields_ = [
        ("cameras", ctypes.c_uint32), ("points", ctypes.c_uint32), ("observations", ctypes.c_uint32),
        ("anchor", ctypes.c_uint32), ("scale_view", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
        ("scene_offset", ctypes.c_uint64), ("index_offset", ctypes.c_uint64), ("output_offset", ctypes.c_uint64),
    ]


class BatchControl(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_uint32), ("max_cg", ctypes.c_uint32), ("shared_focal", ctypes.c_uint32),
        ("precision", ctypes.c_uint32), ("schedule", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("huber", ctypes.c_double), ("cg_tolerance", ctypes.c_double), ("stall_tolerance", ctypes.c_double),
    ]


class BatchReport(ctypes.Structure):
    _fields_ = [
        ("solve_ms", ctypes.c_double), ("upload_ms", ctypes.c_double), ("download_ms", ctypes.c_double),
        ("wall_ms", ctypes.c_double), ("tune_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("lm_iterations", ctypes.c_uint64), ("cg_iterations", ctypes.c_uint64),
        ("problems", ctypes.c_uint32), ("schedule", ctypes.c_uint32), ("threads", ctypes.c_uint32),
        ("blocks", ctypes.c_uint32), ("graph_replayed", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
        ("form", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class VjpControl(ctypes.Structure):
    _fields_ = [
        ("cameras", ctypes.c_uint32), ("points", ctypes.c_uint32), ("observations", ctypes.c_uint32),
        ("anchor", ctypes.c_uint32), ("scale_view", ctypes.c_uint32), ("newton_steps", ctypes.c_uint32),
        ("max_cg", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("huber", ctypes.c_double), ("cg_tolerance", ctypes.c_double),
    ]


class VjpReport(ctypes.Structure):
    _fields_ = [
        ("solve_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
        ("gradient_norm_initial", ctypes.c_double), ("gradient_norm_final", ctypes.c_double),
        ("adjoint_residual", ctypes.c_double),
        ("cg_iterations", ctypes.c_uint32), ("newton_steps", ctypes.c_uint32), ("failed", ctypes.c_uint32),
        ("invalid", ctypes.c_uint32), ("point_failures", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
        ("product_ms", ctypes.c_double), ("product_launches", ctypes.c_uint32), ("product_blocks", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ObservationControl(ctypes.Structure):
    _fields_ = [
        ("cameras", ctypes.c_uint32), ("points", ctypes.c_uint32), ("observations", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32), ("max_error_px", ctypes.c_double),
        ("max_relative_depth_std", ctypes.c_double), ("pixel_noise_std_px", ctypes.c_double),
    ]


class ObservationReport(ctypes.Structure):
    _fields_ = [
        ("upload_ms", ctypes.c_double), ("evaluate_ms", ctypes.c_double), ("download_ms", ctypes.c_double),
        ("wall_ms", ctypes.c_double), ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LibraryError(f"libtba.so is not built ({path}); run `python -m typecv_b200.build`")
    try:
        lib = ctypes.CDLL(path)
    except OSError as e:
        raise LibraryError(f"libtba.so failed to load: {e}") from e
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    lib.tba_scene_size.restype = ctypes.c_size_t
    lib.tba_scene_size.argtypes = [P(Control)]
    lib.tba_index_size.restype = ctypes.c_size_t
    lib.tba_index_size.argtypes = [P(Control)]
    lib.tba_output_size.restype = ctypes.c_size_t
    lib.tba_output_size.argtypes = [P(Control)]
    lib.tba_device_open.restype = ctypes.c_int
    lib.tba_device_open.argtypes = [ctypes.c_int, P(vp)]
    lib.tba_device_close.restype = None
    lib.tba_device_close.argtypes = [vp]
    lib.tba_last_error.restype = ctypes.c_char_p
    lib.tba_last_error.argtypes = [vp]
    lib.tba_bundle_adjust.restype = ctypes.c_int
    lib.tba_bundle_adjust.argtypes = [vp, P(Control), P(ctypes.c_double), ctypes.c_size_t, P(ctypes.c_uint32),
                                      ctypes.c_size_t, P(ctypes.c_double), ctypes.c_size_t, P(Report)]
    lib.tba_scene_cost_noalloc.restype = ctypes.c_int
    lib.tba_scene_cost_noalloc.argtypes = [P(Control), vp, ctypes.c_size_t, vp, ctypes.c_size_t, vp, ctypes.c_size_t,
                                           vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.tba_batch_max_cameras.restype = ctypes.c_uint32
    lib.tba_batch_max_cameras.argtypes = []
    lib.tba_batch_shapes.restype = ctypes.c_uint32
    lib.tba_batch_shapes.argtypes = []
    lib.tba_batch_shape.restype = ctypes.c_int
    lib.tba_batch_shape.argtypes = [ctypes.c_uint32, P(ctypes.c_uint32), P(ctypes.c_uint32)]
    lib.tba_batch_adjust.restype = ctypes.c_int
    lib.tba_batch_adjust.argtypes = [vp, P(BatchControl), P(BatchProblem), ctypes.c_uint32, P(ctypes.c_double),
                                     ctypes.c_size_t, P(ctypes.c_uint32), ctypes.c_size_t, P(ctypes.c_double),
                                     ctypes.c_size_t, P(BatchReport)]
    lib.tba_bundle_vjp.restype = ctypes.c_int
    lib.tba_bundle_vjp.argtypes = [vp, P(VjpControl), P(ctypes.c_double), ctypes.c_size_t, P(ctypes.c_uint32),
                                   ctypes.c_size_t, P(ctypes.c_double), ctypes.c_size_t, P(ctypes.c_double),
                                   ctypes.c_size_t, P(ctypes.c_double), P(ctypes.c_double), ctypes.c_size_t,
                                   P(VjpReport)]
    lib.tba_evaluate_observations.restype = ctypes.c_int
    lib.tba_evaluate_observations.argtypes = [vp, P(ObservationControl), P(ctypes.c_double), ctypes.c_size_t,
                                              P(ctypes.c_double), ctypes.c_size_t, P(ctypes.c_double), ctypes.c_size_t,
                                              P(ctypes.c_uint32), ctypes.c_size_t, P(ctypes.c_uint32), ctypes.c_size_t,
                                              P(ctypes.c_uint32), ctypes.c_size_t, P(ctypes.c_double),
                                              P(ObservationReport)]
    lib.tba_scene_create.restype = ctypes.c_int
    lib.tba_scene_create.argtypes = [vp, P(Control), P(ctypes.c_double), ctypes.c_size_t, P(ctypes.c_uint32),
                                     ctypes.c_size_t, P(vp)]
    lib.tba_scene_destroy.restype = None
    lib.tba_scene_destroy.argtypes = [vp]
    lib.tba_scene_adjust.restype = ctypes.c_int
    lib.tba_scene_adjust.argtypes = [vp, vp, P(Control), P(ctypes.c_double), ctypes.c_size_t, P(ctypes.c_double),
                                     ctypes.c_size_t, P(Report)]
    lib.tba_scene_write.restype = ctypes.c_int
    lib.tba_scene_write.argtypes = [vp, vp, P(ctypes.c_double), P(ctypes.c_double)]
    lib.tba_scene_read.restype = ctypes.c_int
    lib.tba_scene_read.argtypes = [vp, vp, P(ctypes.c_double), P(ctypes.c_double)]
    lib.tba_linearize_inverse_depth.restype = ctypes.c_int
    lib.tba_linearize_inverse_depth.argtypes = [vp, ctypes.c_uint32, P(ctypes.c_double), ctypes.c_size_t,
                                                P(ctypes.c_double), ctypes.c_size_t, P(ObservationReport)]
    lib.tba_device_set_wait_limit.restype = ctypes.c_int
    lib.tba_device_set_wait_limit.argtypes = [vp, ctypes.c_uint32]
    _lib = lib
    return lib


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def uptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
