"""Batched build + trace of many independent scenes.

One segmented LBVH holds every scene (the segment id is the top word of the
sort key, bajo/bvh/gpu/builder/lbvh.mojo:59); one batched trace launch shoots
width x height primary rays per scene plus one cosine-weighted bounce ray per
primary hit.  ``BatchedGraph`` captures the whole build + trace in one CUDA
graph so a frame is a single graph launch; the sort's tile shapes come from
the autotuner's table.

Reference: the BLAS-set build and trace (``build_triangle_blas_set``,
bajo/bvh/gpu/triangle_bvh.mojo:469; ``enqueue_segmented_wide_build``,
bajo/bvh/gpu/builder/segmented_build.mojo:89).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, bvh


class BatchResult:
    def __init__(self, n_rays: int, device):
        self.t0 = torch.empty(n_rays, dtype=torch.float32, device=device)
        self.p0 = torch.empty(n_rays, dtype=torch.int32, device=device)
        self.t1 = torch.empty(n_rays, dtype=torch.float32, device=device)
        self.p1 = torch.empty(n_rays, dtype=torch.int32, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.tree = None

    def outputs(self):
        """(primary t, primary prim, bounce t, bounce prim) as numpy."""
        return (self.t0.cpu().numpy(), self.p0.cpu().numpy().view(np.uint32), self.t1.cpu().numpy(),
                self.p1.cpu().numpy().view(np.uint32))


def _cameras(camera, device):
    cam = torch.from_numpy(np.ascontiguousarray(camera, np.float32).reshape(-1)).to(device)
    stride = 0 if cam.numel() == 20 else 20
    return cam, stride


def _launch_trace(tree_c, cam, stride, width, height, seed, res, tri_mode, stream=None):
    rc = _lib.load().bajo_trace_batch(ctypes.byref(tree_c), cam.data_ptr(), stride, width, height, seed, tri_mode,
                                      res.t0.data_ptr(), res.p0.data_ptr(), res.t1.data_ptr(), res.p1.data_ptr(),
                                      res.status.data_ptr(), _lib.stream_handle(stream))
    _lib.check(rc, "bajo_trace_batch")


def build_and_trace(vertices: torch.Tensor, seg_offsets, camera, width: int, height: int, seed: int = 7,
                    tri_mode: int = _lib.TRI_WATERTIGHT) -> BatchResult:
    """Build every scene's LBVH and trace its rays (eager launches)."""
    tree = bvh.build_triangle_bvh(vertices, seg_offsets)
    n_rays = tree.n_segments * width * height
    res = BatchResult(n_rays, vertices.device)
    res.tree = tree
    cam, stride = _cameras(camera, vertices.device)
    res.cam = cam
    _launch_trace(tree.c_struct(), cam, stride, width, height, seed, res, tri_mode)
    return res


class BatchedGraph:
    """Build + trace of a fixed batch captured once in a CUDA graph;
    ``replay()`` rebuilds every tree from the current vertex buffer and traces
    all rays with one graph launch."""

    def __init__(self, vertices: torch.Tensor, seg_offsets, camera, width: int, height: int, seed: int = 7,
                 tri_mode: int = _lib.TRI_WATERTIGHT):
        dev = vertices.device
        self.vertices = vertices
        so = torch.as_tensor(np.asarray(seg_offsets, dtype=np.int64).astype(np.int32), device=dev)
        n = vertices.numel() // 9
        S = so.numel() - 1
        self.workspace = bvh.GpuBvhBuildWorkspace(n, S, device=dev)
        self.tree = bvh.GpuTriangleBvh(n, so, dev)
        self.tree.vertices = vertices
        self.tree_c = self.tree.c_struct()
        self.result = BatchResult(S * width * height, dev)
        self.cam, self.stride = _cameras(camera, dev)
        self.args = (width, height, seed, tri_mode)
        # warm-up outside capture: kernel attributes, tuning table, lazy init
        self._enqueue()
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._enqueue()
        torch.cuda.synchronize()

    def _enqueue(self):
        L = _lib.load()
        ws = self.workspace.buffer
        _lib.check(L.bajo_lbvh_build(self.vertices.data_ptr(), ctypes.byref(self.tree_c), ws.data_ptr(), ws.numel(),
                                     _lib.stream_handle()), "bajo_lbvh_build")
        w, h, seed, mode = self.args
        _launch_trace(self.tree_c, self.cam, self.stride, w, h, seed, self.result, mode)

    def replay(self):
        self.graph.replay()

    def status(self) -> int:
        torch.cuda.synchronize()
        return int(self.result.status.item()) | self.workspace.status()
