"""Pinhole camera records (``Camera``, bajo/bvh/camera.mojo:19-154).

A camera is 20 floats: origin, forward, right, up, fov_scale, focus distance,
defocus disk u, defocus disk v (Camera.STRIDE = 20).  The record is computed
by the library's host code (``bajo_camera_make`` / ``bajo_camera_from_vfov``)
so that it is bit-identical to what the kernels and the oracle expect.
"""
from __future__ import annotations

import numpy as np

from . import _lib

STRIDE = 20


def _vec(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float32).reshape(3))


def camera(origin, target, world_up, fov_scale: float) -> np.ndarray:
    """Camera.__init__ (camera.mojo:77-97) with a zero defocus angle."""
    out = np.zeros(STRIDE, np.float32)
    o, t, u = _vec(origin), _vec(target), _vec(world_up)
    _lib.check(_lib.load().bajo_camera_make(o.ctypes.data, t.ctypes.data, u.ctypes.data, float(fov_scale),
                                            out.ctypes.data), "bajo_camera_make")
    return out


def camera_from_vfov(origin, target, world_up, vfov_deg: float) -> np.ndarray:
    """Camera.from_vfov (camera.mojo:100-116)."""
    out = np.zeros(STRIDE, np.float32)
    o, t, u = _vec(origin), _vec(target), _vec(world_up)
    _lib.check(_lib.load().bajo_camera_from_vfov(o.ctypes.data, t.ctypes.data, u.ctypes.data, float(vfov_deg),
                                                 out.ctypes.data), "bajo_camera_from_vfov")
    return out


def plain_lbvh_camera() -> np.ndarray:
    """The plain LBVH workload's camera: eye (0.5, 0.5, -1.5) looking +z,
    60 degree vertical field of view."""
    return camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, -0.5], [0.0, 1.0, 0.0], 60.0)
