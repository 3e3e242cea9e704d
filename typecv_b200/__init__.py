"""typecv_b200 — TypeCV's joint bundle adjustment (the `bundleAdjustGpu` operator) for B200.

The device work lives in libtba.so (hand-written CUDA for sm_100a behind the C ABI of
include/tba.h); this package holds its ctypes binding and the host mirror of the reference
operator's TypeScript side (validation, packing, result reading).
"""
from .bundle import (BUNDLE_DEFAULTS, DeviceError, RangeError, ShadeDevice, bundle_adjust_gpu, make_control,
                     pack_arrays, pack_bundle_scene, solve_packed)

__all__ = ["BUNDLE_DEFAULTS", "DeviceError", "RangeError", "ShadeDevice", "bundle_adjust_gpu", "make_control",
           "pack_arrays", "pack_bundle_scene", "solve_packed"]
