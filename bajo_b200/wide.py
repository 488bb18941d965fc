"""Wide BVH (W = 4 or 8) collapsed from a built binary LBVH.

Mirrors the reference's ordinary wide layout (``GpuWideBoundsBvh``,
bajo/bvh/gpu/wide_layout.mojo:119; collapse ``hploc_literature_to_wide_kernel``,
bajo/bvh/gpu/builder/wide_collapse.mojo:148; triangle leaf packing
``pack_segmented_triangle_leaf_lanes_kernel``, bajo/bvh/gpu/triangle_bvh.mojo:81)
with deterministic node and leaf ids (a node's internal children are
consecutive nodes, its leaf blocks consecutive blocks), and the compressed
8-wide CWBVH8 layout built from it (``GpuBvhLayout.CWBVH8``,
bajo/bvh/gpu/compressed_bounds_bvh.mojo; ``build_triangle_blas_set``,
bajo/bvh/gpu/triangle_bvh.mojo:466).  Device work is ``bajo_wide_build`` /
``bajo_cwbvh8_build`` / ``bajo_trace_wide_*`` / ``bajo_trace_cwbvh8_*`` in the
C ABI.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import BajoCwbvh8C, BajoCwbvh8SizesC, BajoWideBvhC, BajoWideSizesC, CWBVH8_ARRAYS, WIDE_ARRAYS

_DTYPES = {"node_offsets": torch.int32, "leaf_offsets": torch.int32, "nodes": torch.float32,
           "leaf_indices": torch.int32, "leaf_tris": torch.float32, "leaf_sorted": torch.int32}


def wide_sizes(n_tris: int, n_segments: int, width: int) -> dict:
    s = BajoWideSizesC()
    _lib.check(_lib.load().bajo_wide_sizes(n_tris, n_segments, width, ctypes.byref(s)), "bajo_wide_sizes")
    return {name: getattr(s, name) for name in WIDE_ARRAYS + ("workspace",)}


class GpuWideBvh:
    """Wide tree of a ``GpuTriangleBvh``; ``n_nodes`` / ``n_leaf_blocks``
    are read back after the build (one synchronisation)."""

    def __init__(self, tree, width: int = 4, max_leaf: int = 4):
        if width not in (4, 8):
            raise ValueError("width must be 4 or 8")
        if not 1 <= max_leaf <= 4:
            raise ValueError("max_leaf must be 1..4")
        self.max_leaf = max_leaf
        dev = tree.node_meta.device
        sizes = wide_sizes(tree.n_leaves, tree.n_segments, width)
        self.width = width
        self.tree = tree
        for name in WIDE_ARRAYS:
            dt = _DTYPES[name]
            item = torch.empty(0, dtype=dt).element_size()
            setattr(self, name, torch.empty(max(sizes[name] // item, 1), dtype=dt, device=dev))
        self.workspace = torch.zeros(sizes["workspace"], dtype=torch.uint8, device=dev)
        self._c = None
        self.n_nodes = 0
        self.n_leaf_blocks = 0

    def c_struct(self) -> BajoWideBvhC:
        c = BajoWideBvhC()
        c.width = self.width
        c.max_leaf = self.max_leaf
        c.n_segments = self.tree.n_segments
        for name in WIDE_ARRAYS:
            setattr(c, name, getattr(self, name).data_ptr())
        c.bvh2_leaf_tris = self.tree.leaf_tris.data_ptr()
        self._c = c
        return c

    def build(self, stream=None, read_counts: bool = True) -> "GpuWideBvh":
        t = self.tree.c_struct()
        c = self.c_struct()
        _lib.check(_lib.load().bajo_wide_build(ctypes.byref(t), ctypes.byref(c), self.workspace.data_ptr(),
                                               self.workspace.numel(), _lib.stream_handle(stream)),
                   "bajo_wide_build")
        self._c = c
        if read_counts:
            self.read_counts(stream)
        return self

    def read_counts(self, stream=None):
        a, b = ctypes.c_uint32(0), ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_wide_counts(ctypes.byref(self._c), _lib.stream_handle(stream), ctypes.byref(a),
                                                ctypes.byref(b)), "bajo_wide_counts")
        self.n_nodes, self.n_leaf_blocks = a.value, b.value
        return self.n_nodes, self.n_leaf_blocks

    def status(self, stream=None) -> int:
        st = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_workspace_status(self.workspace.data_ptr(), _lib.stream_handle(stream),
                                                     ctypes.byref(st)), "bajo_workspace_status")
        return st.value

    def seg0_counts(self):
        """(wide nodes, leaf blocks) of segment 0, the tree the traversal
        entry points trace."""
        if self.tree.n_segments == 1:
            return self.n_nodes, self.n_leaf_blocks
        return int(self.node_offsets[1].item()), int(self.leaf_offsets[1].item())

    def launch_rays(self, d_rays, d_hits, ray_count, tri_mode=_lib.TRI_WATERTIGHT, d_t=None, d_prim=None,
                    d_status=None, stream=None):
        _lib.require_cuda(d_rays)
        st = d_status if d_status is not None else torch.zeros(1, dtype=torch.int32, device=d_rays.device)
        rc = _lib.load().bajo_trace_wide_rays(ctypes.byref(self._c), *self.seg0_counts(), d_rays.data_ptr(),
                                              ray_count, tri_mode, _ptr(d_hits), _ptr(d_t), _ptr(d_prim),
                                              st.data_ptr(), _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_wide_rays")
        return st

    def launch_camera(self, d_camera, d_hits, ray_count, width, height, tri_mode=_lib.TRI_WATERTIGHT, d_t=None,
                      d_prim=None, d_status=None, d_stats=None, stream=None):
        _lib.require_cuda(d_camera)
        st = d_status if d_status is not None else torch.zeros(1, dtype=torch.int32, device=d_camera.device)
        rc = _lib.load().bajo_trace_wide_camera(ctypes.byref(self._c), *self.seg0_counts(), d_camera.data_ptr(),
                                                ray_count, width, height, tri_mode, _ptr(d_hits), _ptr(d_t),
                                                _ptr(d_prim), st.data_ptr(), _ptr(d_stats),
                                                _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_wide_camera")
        return st


def _ptr(t):
    return None if t is None else t.data_ptr()


def build_wide_bvh(tree, width: int = 4, max_leaf: int = 4, stream=None) -> GpuWideBvh:
    """Collapse a built ``GpuTriangleBvh`` into a ``GpuWideBvh`` (leaf blocks
    of up to ``max_leaf`` triangles; 4 = the reference's fat leaves)."""
    return GpuWideBvh(tree, width, max_leaf).build(stream)


def cwbvh8_sizes(n_tris: int, n_segments: int) -> dict:
    s = BajoCwbvh8SizesC()
    _lib.check(_lib.load().bajo_cwbvh8_sizes(n_tris, n_segments, ctypes.byref(s)), "bajo_cwbvh8_sizes")
    return {name: getattr(s, name) for name in CWBVH8_ARRAYS + ("workspace",)}


class GpuCwbvh8:
    """Compressed 8-wide tree (80-byte nodes, 48-byte triangle records) of a
    ``GpuTriangleBvh``; ``n_nodes`` is read back after the build (one
    synchronisation)."""

    def __init__(self, tree):
        dev = tree.node_meta.device
        sizes = cwbvh8_sizes(tree.n_leaves, tree.n_segments)
        self.tree = tree
        self.node_offsets = torch.empty(max(sizes["node_offsets"] // 4, 1), dtype=torch.int32, device=dev)
        self.nodes = torch.empty(max(sizes["nodes"] // 4, 1), dtype=torch.float32, device=dev)
        self.triangles = torch.empty(max(sizes["triangles"] // 4, 1), dtype=torch.float32, device=dev)
        self.workspace = torch.zeros(sizes["workspace"], dtype=torch.uint8, device=dev)
        self._c = self.c_struct()
        self.n_nodes = 0

    def c_struct(self) -> BajoCwbvh8C:
        c = BajoCwbvh8C()
        c.n_segments = self.tree.n_segments
        c.n_tris = self.tree.n_leaves
        for name in CWBVH8_ARRAYS:
            setattr(c, name, getattr(self, name).data_ptr())
        return c

    def build(self, stream=None, read_count: bool = True) -> "GpuCwbvh8":
        t = self.tree.c_struct()
        _lib.check(_lib.load().bajo_cwbvh8_build(ctypes.byref(t), ctypes.byref(self._c), self.workspace.data_ptr(),
                                                 self.workspace.numel(), _lib.stream_handle(stream)),
                   "bajo_cwbvh8_build")
        if read_count:
            self.read_count(stream)
        return self

    def read_count(self, stream=None) -> int:
        a = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_cwbvh8_count(ctypes.byref(self._c), _lib.stream_handle(stream), ctypes.byref(a)),
                   "bajo_cwbvh8_count")
        self.n_nodes = a.value
        return self.n_nodes

    def status(self, stream=None) -> int:
        st = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_workspace_status(self.workspace.data_ptr(), _lib.stream_handle(stream),
                                                     ctypes.byref(st)), "bajo_workspace_status")
        return st.value

    def launch_rays(self, d_rays, d_hits, ray_count, any_hit: bool = False, d_t=None, d_prim=None, d_status=None,
                    stream=None):
        _lib.require_cuda(d_rays)
        st = d_status if d_status is not None else torch.zeros(1, dtype=torch.int32, device=d_rays.device)
        rc = _lib.load().bajo_trace_cwbvh8_rays(ctypes.byref(self._c), self.n_nodes, d_rays.data_ptr(), ray_count,
                                                int(any_hit), _ptr(d_hits), _ptr(d_t), _ptr(d_prim), st.data_ptr(),
                                                _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_cwbvh8_rays")
        return st

    def launch_camera(self, d_camera, d_hits, ray_count, width, height, any_hit: bool = False, d_t=None, d_prim=None,
                      d_status=None, stream=None):
        _lib.require_cuda(d_camera)
        st = d_status if d_status is not None else torch.zeros(1, dtype=torch.int32, device=d_camera.device)
        rc = _lib.load().bajo_trace_cwbvh8_camera(ctypes.byref(self._c), self.n_nodes, d_camera.data_ptr(), ray_count,
                                                  width, height, int(any_hit), _ptr(d_hits), _ptr(d_t), _ptr(d_prim),
                                                  st.data_ptr(), _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_cwbvh8_camera")
        return st


def build_cwbvh8(tree, stream=None) -> GpuCwbvh8:
    """Collapse and compress a built ``GpuTriangleBvh`` into a ``GpuCwbvh8``
    (8-wide, leaves of at most 3 triangles, octant child slots)."""
    return GpuCwbvh8(tree).build(stream)
