"""GPU LBVH build and closest-hit traversal, mirroring ``bajo.bvh.gpu``.

Reference entry points (jgsimard/bajo):
  - ``build_triangle_bvh`` (bajo/bvh/gpu/triangle_bvh.mojo:617) and the
    segmented driver (bajo/bvh/gpu/builder/segmented_build.mojo:89) down to
    ``build_binary_bvh_with_lbvh`` (bajo/bvh/gpu/builder/lbvh.mojo:332);
  - ``GpuTriangleBvh.launch_rays`` / ``launch_camera``
    (bajo/bvh/gpu/triangle_bvh.mojo:587, :520);
  - ``validate_topology`` / ``validate_refit_bounds``
    (bajo/bvh/gpu/validate.mojo:62, :127).

Device work goes through the C ABI in ``libbajo_b200.so``; torch tensors are
the device allocations.  The result object owns every array of the binary
LBVH in the reference's layouts (see ``include/bajo_b200.h``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import BajoLbvhC, BajoLbvhSizesC, LBVH_ARRAYS

CLOSEST_HIT = 0  # TRACE.CLOSEST_HIT, bajo/bvh/constants.mojo:10
TRI_MT = _lib.TRI_MT
TRI_WATERTIGHT = _lib.TRI_WATERTIGHT
SENTINEL = 0xFFFFFFFF
LEAF_FLAG = 0x80000000
HIT_STRIDE = 8   # Hit.STRIDE, bajo/bvh/types.mojo:23
RAY_STRIDE = 8   # Ray.STRIDE, bajo/core/ray.mojo:10
STATS_WORDS = 5  # GpuTraversalStats.STRIDE, bajo/bvh/gpu/trace.mojo:68

_DTYPES = {
    "internal_offsets": torch.int32, "leaf_bounds": torch.float32, "seg_bounds": torch.float32,
    "sort_keys": torch.int64, "leaf_ids": torch.int32, "morton_codes": torch.int32, "node_meta": torch.int32,
    "node_bounds": torch.float32, "node_leaf_counts": torch.int32, "node_flags": torch.int32,
    "leaf_parent": torch.int32, "roots": torch.int32, "leaf_tris": torch.float32,
}


def lbvh_sizes(n_tris: int, n_segments: int = 1) -> dict:
    s = BajoLbvhSizesC()
    _lib.check(_lib.load().bajo_lbvh_sizes(n_tris, n_segments, ctypes.byref(s)), "bajo_lbvh_sizes")
    return {name: getattr(s, name) for name in LBVH_ARRAYS + ("workspace",)}


# GpuBvhBuildMethod (bajo/bvh/gpu/builder): LBVH (Karras topology + refit) or
# HPLOC (hierarchical PLOC clustering over the same sorted keys)
BUILD_METHODS = ("lbvh", "hploc")


class GpuBvhBuildWorkspace:
    """Reusable build scratch for one (N, S) shape (GpuBinaryBuildWorkspace,
    bajo/bvh/gpu/builder/binary_layout.mojo:252)."""

    def __init__(self, n_tris: int, n_segments: int = 1, device="cuda", method: str = "lbvh"):
        if method not in BUILD_METHODS:
            raise ValueError(f"method must be one of {BUILD_METHODS}")
        self.n_tris, self.n_segments, self.method = n_tris, n_segments, method
        if method == "hploc":
            b = ctypes.c_size_t(0)
            _lib.check(_lib.load().bajo_hploc_workspace_size(n_tris, n_segments, ctypes.byref(b)),
                       "bajo_hploc_workspace_size")
            nbytes = b.value
        else:
            nbytes = lbvh_sizes(n_tris, n_segments)["workspace"]
        self.buffer = torch.zeros(max(nbytes, 256), dtype=torch.uint8, device=device)

    def status(self, stream=None) -> int:
        st = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_workspace_status(self.buffer.data_ptr(), _lib.stream_handle(stream),
                                                     ctypes.byref(st)), "bajo_workspace_status")
        return st.value


class GpuTriangleBvh:
    """Binary LBVH over triangles plus its traversal entry points.

    With ``stage_top`` the tree also carries ``top_nodes``, the first
    BAJO_TOP_NODES nodes of segment 0 in breadth-first order, which the build
    writes and the closest-hit kernels read from shared memory."""

    def __init__(self, n_tris: int, seg_offsets: torch.Tensor, device="cuda", stage_top: bool = False):
        self.n_leaves = n_tris
        self.n_segments = seg_offsets.numel() - 1
        self.seg_offsets = seg_offsets
        sizes = lbvh_sizes(n_tris, self.n_segments)
        for name in LBVH_ARRAYS:
            dt = _DTYPES[name]
            itemsize = torch.empty(0, dtype=dt).element_size()
            setattr(self, name, torch.empty(sizes[name] // itemsize, dtype=dt, device=device))
        self.top_nodes = torch.zeros(_lib.TOP_BYTES // 4, dtype=torch.float32, device=device) if stage_top else None
        self.vertices = None
        self._c = None

    def c_struct(self, stage_top: bool = True) -> BajoLbvhC:
        """The C record of this tree; ``stage_top=False`` leaves top_nodes
        NULL (builds through it do not stage, traces through it read the
        whole tree from global memory)."""
        c = BajoLbvhC()
        c.n_leaves, c.n_segments = self.n_leaves, self.n_segments
        c.seg_offsets = self.seg_offsets.data_ptr()
        for name in LBVH_ARRAYS:
            setattr(c, name, getattr(self, name).data_ptr())
        c.top_nodes = self.top_nodes.data_ptr() if stage_top and self.top_nodes is not None else None
        self._c = c
        return c

    def restage_top(self, stream=None) -> None:
        """Rewrite top_nodes from the current nodes (bajo_lbvh_stage_top)."""
        if self.top_nodes is None:
            raise ValueError("this tree was created without stage_top")
        c = self.c_struct()
        _lib.check(_lib.load().bajo_lbvh_stage_top(ctypes.byref(c), _lib.stream_handle(stream)),
                   "bajo_lbvh_stage_top")

    def top_header(self) -> tuple[int, int]:
        """(staged node count, root ref) of top_nodes."""
        h = self.top_nodes[:2].view(torch.int32).cpu().numpy().view(np.uint32)
        return int(h[0]), int(h[1])

    @property
    def internal_count(self) -> int:
        return int(self.internal_offsets[-1].item())

    # ---- traversal ---------------------------------------------------------
    def launch_rays(self, d_rays: torch.Tensor, d_hits: torch.Tensor | None, ray_count: int, mode: int = CLOSEST_HIT,
                    tri_mode: int = TRI_WATERTIGHT, d_t: torch.Tensor | None = None,
                    d_prim: torch.Tensor | None = None, d_status: torch.Tensor | None = None, stream=None) -> None:
        """Trace a field-major ray buffer (8 planes x ray_count) and write
        8-word hits (GpuTriangleBvh.launch_rays, triangle_bvh.mojo:587)."""
        if mode != CLOSEST_HIT:
            raise NotImplementedError("only CLOSEST_HIT traversal is provided")
        _lib.require_cuda(d_rays)
        if d_rays.numel() < ray_count * RAY_STRIDE:
            raise ValueError("packed ray input buffer is too short")
        if d_hits is not None and d_hits.numel() < ray_count * HIT_STRIDE:
            raise ValueError("hit output buffer is too short")
        c = self.c_struct()
        rc = _lib.load().bajo_trace_rays(ctypes.byref(c), d_rays.data_ptr(), ray_count, tri_mode,
                                         _ptr(d_hits), _ptr(d_t), _ptr(d_prim), _ptr(d_status),
                                         _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_rays")

    def launch_camera(self, d_camera_params: torch.Tensor, d_hits: torch.Tensor | None, ray_count: int, width: int,
                      height: int, tri_mode: int = TRI_WATERTIGHT, d_t: torch.Tensor | None = None,
                      d_prim: torch.Tensor | None = None, d_status: torch.Tensor | None = None, stream=None) -> None:
        """Primary rays from 20-float camera records, one camera per
        width*height rays (GpuTriangleBvh.launch_camera, triangle_bvh.mojo:520)."""
        _lib.require_cuda(d_camera_params)
        views = -(-ray_count // (width * height))
        if d_camera_params.numel() < views * 20:
            raise ValueError("camera parameter buffer is too short")
        if d_hits is not None and d_hits.numel() < ray_count * HIT_STRIDE:
            raise ValueError("hit output buffer is too short")
        c = self.c_struct()
        rc = _lib.load().bajo_trace_camera(ctypes.byref(c), d_camera_params.data_ptr(), ray_count, width, height,
                                           tri_mode, _ptr(d_hits), _ptr(d_t), _ptr(d_prim), _ptr(d_status),
                                           _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_camera")

    def launch_camera_instrumented(self, d_camera_params: torch.Tensor, d_hits: torch.Tensor | None,
                                   d_stats: torch.Tensor, ray_count: int, width: int, height: int,
                                   tri_mode: int = TRI_WATERTIGHT, stream=None) -> None:
        """launch_camera plus STATS_WORDS counters per ray in the layout of
        GpuTraversalStats (bajo/bvh/gpu/trace.mojo:62-90): node visits,
        internal child hits, leaf blocks, triangle tests, deepest stack
        (launch_camera_instrumented, triangle_bvh.mojo:550)."""
        _lib.require_cuda(d_stats)
        if d_stats.numel() < STATS_WORDS * ray_count or d_stats.element_size() != 4:
            raise ValueError("traversal stats output buffer is too short")
        c = self.c_struct()
        rc = _lib.load().bajo_trace_camera_stats(ctypes.byref(c), d_camera_params.data_ptr(), ray_count, width,
                                                 height, tri_mode, _ptr(d_hits), d_stats.data_ptr(),
                                                 _lib.stream_handle(stream))
        _lib.check(rc, "bajo_trace_camera_stats")


def _ptr(t):
    return None if t is None else t.data_ptr()


def build_triangle_bvh(vertices: torch.Tensor, seg_offsets=None, workspace: GpuBvhBuildWorkspace | None = None,
                       out: GpuTriangleBvh | None = None, stream=None,
                       stage_top: bool | None = None, method: str = "lbvh") -> GpuTriangleBvh:
    """Build the binary LBVH of `vertices` (9 floats per triangle, CUDA).

    `seg_offsets` (optional, S+1 item offsets) builds one independent tree per
    segment in the same launches (the batched BLAS path,
    bajo/bvh/gpu/triangle_bvh.mojo:469).  `stage_top` also writes the staged
    top levels for the traversal (off by default: on B200 the top of the tree
    stays in L1 and the staged kernels were measured no faster).  `method`
    "hploc" builds the tree by H-PLOC (the reference's default builder,
    GpuBvhBuildMethod.HPLOC) instead of the LBVH topology and refit."""
    _lib.require_cuda(vertices)
    if vertices.dtype != torch.float32 or not vertices.is_contiguous() or vertices.numel() % 9:
        raise ValueError("triangle vertex buffer must be contiguous float32 with 9 floats per triangle")
    n = vertices.numel() // 9
    if seg_offsets is None and out is not None and out.n_leaves == n and out.n_segments == 1:
        seg = out.seg_offsets  # reuse: no host-to-device copy per rebuild
    elif seg_offsets is None:
        seg = torch.tensor([0, n], dtype=torch.int32, device=vertices.device)
    elif isinstance(seg_offsets, torch.Tensor):
        seg = seg_offsets.to(device=vertices.device, dtype=torch.int32).contiguous()
    else:
        so = np.asarray(seg_offsets, dtype=np.int64)
        if so[0] != 0 or so[-1] != n or np.any(np.diff(so) < 0):
            raise ValueError("segment offsets must start at 0, end at the triangle count and not decrease")
        seg = torch.tensor(so.astype(np.int32), device=vertices.device)
    S = seg.numel() - 1
    if S < 1:
        raise ValueError("at least one segment is required")
    if stage_top is None:
        stage_top = False
    if (workspace is None or workspace.n_tris != n or workspace.n_segments != S or
            getattr(workspace, "method", "lbvh") != method):
        workspace = GpuBvhBuildWorkspace(n, S, device=vertices.device, method=method)
    reuse = out is not None and out.n_leaves == n and out.n_segments == S and (out.top_nodes is not None or not stage_top)
    bvh = out if reuse else GpuTriangleBvh(n, seg, vertices.device, stage_top=stage_top)
    bvh.seg_offsets = seg
    bvh.vertices = vertices
    bvh.workspace = workspace
    c = bvh.c_struct(stage_top)
    entry = "bajo_hploc_build" if method == "hploc" else "bajo_lbvh_build"
    rc = getattr(_lib.load(), entry)(vertices.data_ptr(), ctypes.byref(c), workspace.buffer.data_ptr(),
                                     workspace.buffer.numel(), _lib.stream_handle(stream))
    _lib.check(rc, entry)
    return bvh


# ---- host-side validators (bajo/bvh/gpu/validate.mojo) ---------------------
@dataclass
class TopologyValidation:
    ok: bool
    root_count: int
    root_idx: int
    checksum: int


@dataclass
class RefitBoundsValidation:
    ok: bool
    diff: float
    root_idx: int
    checksum: int


def validate_topology(node_meta: np.ndarray, leaf_parent: np.ndarray, leaf_count: int) -> TopologyValidation:
    """validate.mojo:62-124: one root, parent/child links consistent, every
    leaf has an in-range parent (single segment, leaf_count >= 2)."""
    m = np.asarray(node_meta, dtype=np.uint32).reshape(-1)[: 4 * (leaf_count - 1)].reshape(-1, 4)
    lp = np.asarray(leaf_parent, dtype=np.uint32).reshape(-1)[:leaf_count]
    ic = leaf_count - 1
    ok = True
    parent, left, right = m[:, 0].astype(np.int64), m[:, 1].astype(np.int64), m[:, 2].astype(np.int64)
    checksum = int(m.astype(np.uint64).sum()) + int(lp.astype(np.uint64).sum())
    roots = np.nonzero(parent == SENTINEL)[0]
    if np.any((parent != SENTINEL) & (parent >= ic)):
        ok = False
    for child in (left, right):
        is_leaf = (child & LEAF_FLAG) != 0
        idx = child & 0x7FFFFFFF
        if np.any(is_leaf & (idx >= leaf_count)):
            ok = False
        internal = ~is_leaf
        if np.any(internal & (idx >= ic)):
            ok = False
        else:
            ii = idx[internal]
            if np.any(parent[ii] != np.nonzero(internal)[0]):
                ok = False
    if np.any((lp == SENTINEL) | (lp >= ic)):
        ok = False
    if roots.size != 1:
        ok = False
    return TopologyValidation(ok, int(roots.size), int(roots[-1]) if roots.size else SENTINEL, checksum)


def validate_refit_bounds(node_bounds: np.ndarray, node_flags: np.ndarray, node_meta: np.ndarray, leaf_count: int,
                          scene_min, scene_max) -> RefitBoundsValidation:
    """validate.mojo:127-192: every arrival counter is 2 and the root's merged
    box matches the scene box within 1e-4."""
    ic = leaf_count - 1
    m = np.asarray(node_meta, dtype=np.uint32).reshape(-1)[: 4 * ic].reshape(-1, 4)
    flags = np.asarray(node_flags, dtype=np.uint32).reshape(-1)[:ic]
    b = np.asarray(node_bounds, dtype=np.float32).reshape(-1)[: 12 * ic].reshape(-1, 12)
    ok = bool(np.all(flags == 2))
    roots = np.nonzero(m[:, 0] == SENTINEL)[0]
    checksum = int(flags.astype(np.uint64).sum())
    if roots.size == 0:
        return RefitBoundsValidation(False, 1e30, SENTINEL, checksum)
    r = int(roots[-1])
    mn = np.minimum(b[r, 0:3], b[r, 6:9])
    mx = np.maximum(b[r, 3:6], b[r, 9:12])
    diff = float(max(np.abs(mn.astype(np.float64) - np.asarray(scene_min, np.float64)).max(),
                     np.abs(mx.astype(np.float64) - np.asarray(scene_max, np.float64)).max()))
    checksum += int(sum(abs(float(x)) * 1000.0 for x in list(mn) + list(mx)))
    if diff > 1e-4:
        ok = False
    return RefitBoundsValidation(ok, diff, r, checksum)
