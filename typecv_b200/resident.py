"""A scene resident on the device between bundle adjustments (``tba_scene_*`` in libtba.so).

The reference packs and uploads the whole problem for every `bundleAdjustGpu` call
(packBundleScene, src/sfm/bundle/gpu/bundle-host.ts:177-218; bundle.ts:267-271), while its mapper
keeps the map in packed typed arrays between calls (HostScene, src/sfm/scene/scene.ts:8-131).  A
``ResidentScene`` keeps those packed arrays in device memory: they are checked and uploaded once,
each ``adjust`` solves on them and leaves the solution's poses and points in place for the next.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .bundle import DeviceError, RangeError, ShadeDevice


def _raise(lib, device, status, what):
    message = lib.tba_last_error(device.handle).decode()
    if status in (_lib.TBA_ERROR_ARGUMENT, _lib.TBA_ERROR_BUDGET):
        raise RangeError(message)
    raise DeviceError(f"{what} failed ({status}): {message}")


class ResidentScene:
    """The packed scene and index of one problem, resident on `device`."""

    def __init__(self, device: ShadeDevice, control: _lib.Control, scene: np.ndarray, index: np.ndarray):
        lib = _lib.load()
        self.device = device
        self.control = control
        self.C, self.P = control.cameras, control.points
        scene = np.ascontiguousarray(scene, dtype=np.float64)
        index = np.ascontiguousarray(index, dtype=np.uint32)
        handle = ctypes.c_void_p()
        status = lib.tba_scene_create(device.handle, ctypes.byref(control), _lib.dptr(scene), scene.size,
                                      _lib.uptr(index), index.size, ctypes.byref(handle))
        if status != _lib.TBA_OK:
            _raise(lib, device, status, "tba_scene_create")
        self._handle = handle

    def adjust(self, control: _lib.Control | None = None, *, output: bool = False):
        """One bundle adjustment on the resident arrays; returns (output record or None, state
        words, report dict).  The solution stays in the scene."""
        lib = _lib.load()
        control = control or self.control
        out = np.zeros(lib.tba_output_size(ctypes.byref(control))) if output else None
        state = np.zeros(27)
        report = _lib.Report()
        null = ctypes.POINTER(ctypes.c_double)()
        status = lib.tba_scene_adjust(self.device.handle, self._handle, ctypes.byref(control),
                                      _lib.dptr(out) if out is not None else null, out.size if out is not None else 0,
                                      _lib.dptr(state), state.size, ctypes.byref(report))
        if status != _lib.TBA_OK:
            _raise(lib, self.device, status, "tba_scene_adjust")
        return out, state[:26 + (1 if control.shared_focal else 0)], report.as_dict()

    def write(self, poses: np.ndarray | None = None, points: np.ndarray | None = None) -> None:
        lib = _lib.load()
        null = ctypes.POINTER(ctypes.c_double)()
        pz = None if poses is None else np.ascontiguousarray(poses, dtype=np.float64).ravel()
        pt = None if points is None else np.ascontiguousarray(points, dtype=np.float64).ravel()
        if pz is not None and pz.size != 12 * self.C or pt is not None and pt.size != 3 * self.P:
            raise RangeError("Invalid GPU BA resident scene: poses need 12C values and points 3P")
        status = lib.tba_scene_write(self.device.handle, self._handle, _lib.dptr(pz) if pz is not None else null,
                                     _lib.dptr(pt) if pt is not None else null)
        if status != _lib.TBA_OK:
            _raise(lib, self.device, status, "tba_scene_write")

    def read(self) -> tuple[np.ndarray, np.ndarray]:
        lib = _lib.load()
        poses, points = np.zeros(12 * self.C), np.zeros(3 * self.P)
        status = lib.tba_scene_read(self.device.handle, self._handle, _lib.dptr(poses), _lib.dptr(points))
        if status != _lib.TBA_OK:
            _raise(lib, self.device, status, "tba_scene_read")
        return poses, points

    def close(self) -> None:
        if getattr(self, "_handle", None) is not None and self._handle.value:
            _lib.load().tba_scene_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
