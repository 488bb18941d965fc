"""Two-level trees: instances of the BLASes of a segmented triangle build.

Mirrors the reference's TLAS (``build_triangle_tlas`` / ``GpuTriangleTlas``,
bajo/bvh/gpu/tlas.mojo:482-645; ``Instance``, bajo/bvh/types.mojo:153): a
BLAS set is a segmented ``GpuTriangleBvh`` (segment b = BLAS b), an instance
is a BLAS index and an affine transform (3x4 row-major, BLAS space to world
space) with its inverse.  The top-level tree is an LBVH over the instances'
world boxes; tracing takes each ray through the instances it reaches.
Device work is ``bajo_tlas_instance_boxes``, ``bajo_lbvh_build`` and
``bajo_trace_tlas_*`` in the C ABI.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, bvh


def invert_affine(transforms: np.ndarray) -> np.ndarray:
    """Inverses of (n, 12) row-major affine transforms, in float64 then float32."""
    t = np.asarray(transforms, np.float64).reshape(-1, 3, 4)
    m, tr = t[:, :, :3], t[:, :, 3]
    mi = np.linalg.inv(m)
    ti = -np.einsum("nij,nj->ni", mi, tr)
    return np.concatenate([mi, ti[:, :, None]], axis=2).reshape(-1, 12).astype(np.float32)


class GpuTriangleTlas:
    """Top-level tree over instances of ``blas_set`` (a segmented
    ``GpuTriangleBvh``).  ``transforms`` (n, 12) map BLAS space to world
    space; ``inv_transforms`` default to their float64 inverses."""

    def __init__(self, blas_set: bvh.GpuTriangleBvh, transforms, blas_idx, inv_transforms=None, stream=None):
        dev = blas_set.node_meta.device
        xf = np.ascontiguousarray(transforms, np.float32).reshape(-1, 12)
        self.n_instances = xf.shape[0]
        inv = invert_affine(xf) if inv_transforms is None else np.asarray(inv_transforms, np.float32).reshape(-1, 12)
        self.blas_set = blas_set
        self.transforms = torch.from_numpy(xf.copy()).to(dev)
        self.inv_transforms = torch.from_numpy(np.ascontiguousarray(inv)).to(dev)
        self.blas_idx = torch.from_numpy(np.ascontiguousarray(blas_idx, np.uint32).view(np.int32)).to(dev)
        if self.blas_idx.numel() != self.n_instances:
            raise ValueError("one BLAS index per instance")
        self.boxes = torch.empty(max(self.n_instances, 1) * 9, dtype=torch.float32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.top = None
        self.build(stream)

    def build(self, stream=None) -> "GpuTriangleTlas":
        b = self.blas_set.c_struct(False)
        _lib.check(_lib.load().bajo_tlas_instance_boxes(ctypes.byref(b), self.transforms.data_ptr(),
                                                        self.blas_idx.data_ptr(), self.n_instances,
                                                        self.boxes.data_ptr(), self.status.data_ptr(),
                                                        _lib.stream_handle(stream)), "bajo_tlas_instance_boxes")
        self.top = bvh.build_triangle_bvh(self.boxes[:self.n_instances * 9], stream=stream, out=self.top)
        return self

    def _args(self):
        return (ctypes.byref(self.top.c_struct(False)), ctypes.byref(self.blas_set.c_struct(False)),
                self.inv_transforms.data_ptr(), self.blas_idx.data_ptr(), self.n_instances)

    def launch_rays(self, d_rays, d_hits, ray_count, any_hit=False, tri_mode=_lib.TRI_WATERTIGHT, d_status=None,
                    stream=None):
        st = d_status if d_status is not None else torch.zeros(1, dtype=torch.int32, device=d_rays.device)
        _lib.check(_lib.load().bajo_trace_tlas_rays(*self._args(), d_rays.data_ptr(), ray_count, int(any_hit),
                                                    tri_mode, d_hits.data_ptr(), st.data_ptr(),
                                                    _lib.stream_handle(stream)), "bajo_trace_tlas_rays")
        return st

    def launch_camera(self, d_camera, d_hits, ray_count, width, height, any_hit=False, tri_mode=_lib.TRI_WATERTIGHT,
                      d_status=None, stream=None):
        st = d_status if d_status is not None else torch.zeros(1, dtype=torch.int32, device=d_camera.device)
        _lib.check(_lib.load().bajo_trace_tlas_camera(*self._args(), d_camera.data_ptr(), ray_count, width, height,
                                                      int(any_hit), tri_mode, d_hits.data_ptr(), st.data_ptr(),
                                                      _lib.stream_handle(stream)), "bajo_trace_tlas_camera")
        return st


def build_triangle_tlas(blas_set: bvh.GpuTriangleBvh, transforms, blas_idx, inv_transforms=None,
                        stream=None) -> GpuTriangleTlas:
    """Build the top-level tree over the given instances."""
    return GpuTriangleTlas(blas_set, transforms, blas_idx, inv_transforms, stream)
