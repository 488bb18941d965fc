"""Wavefront path tracing on the GPU, mirroring ``bajo.rt.gpu``.

Reference entry points (jgsimard/bajo): ``render_gpu_triangles`` /
``enqueue_render_gpu_triangles`` (bajo/rt/gpu/triangle_path.mojo:143,172)
with ``RenderSettings`` and the PATH / NEE / MIS algorithms
(``RENDER``, bajo/rt/types.mojo:53).  Scenes are Lambertian, emissive,
metal and dielectric triangles.  Device work is
``bajo_render`` in the C ABI; the light table is built by the library's host
code (``bajo_rt_build_lights``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, bvh, wide

PATH = 0
NEE = 3
MIS = 4
LIGHT_STRIDE = 16


class BajoRtSceneC(ctypes.Structure):
    _fields_ = [("bvh", ctypes.POINTER(_lib.BajoLbvhC)), ("surfaces", ctypes.c_void_p),
                ("lambertians", ctypes.c_void_p), ("emissives", ctypes.c_void_p), ("lights", ctypes.c_void_p),
                ("n_lights", ctypes.c_uint32), ("total_light_weight", ctypes.c_float),
                ("metals", ctypes.c_void_p), ("dielectrics", ctypes.c_void_p),
                ("cwbvh8", ctypes.POINTER(_lib.BajoCwbvh8C)), ("cwbvh8_nodes", ctypes.c_uint32)]

# Acceleration structure of the path tracer's rays (the reference's
# GPU_RT_BVH_* policies, bajo/rt/gpu/prepared_scene.mojo:29-33):
#  "cwbvh8_hploc"  the compressed 8-wide tree collapsed from an H-PLOC tree:
#                  the reference's default (GPU_RT_BVH_CWBVH8_HPLOC) and the
#                  fastest here (64-sphere workload, 64 spp: 379 ms against
#                  410 ms for "cwbvh8" and 573 ms for "lbvh" on B200)
#  "cwbvh8"        the compressed 8-wide tree collapsed from the LBVH
#  "lbvh"          the binary LBVH (watertight test, ties to the lowest id)
# The CWBVH8 walk keeps the reference's own hit rules (Moller-Trumbore,
# first of equal-distance hits in visiting order), so its images differ
# from the binary tree's on shared edges and ties, far below the noise.
BVH_POLICIES = ("cwbvh8_hploc", "cwbvh8", "lbvh")
DEFAULT_BVH_POLICY = "cwbvh8_hploc"


class BajoRenderSettingsC(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("seed", ctypes.c_uint64), ("algorithm", ctypes.c_int32),
                ("chunk_paths", ctypes.c_uint32)]


@dataclass
class RenderSettings:
    """RenderSettings (bajo/rt/types.mojo): image size, samples per pixel,
    Philox seed, maximum path depth."""
    width: int
    height: int
    samples_per_pixel: int
    rng_seed: int = 2026
    max_depth: int = 8
    chunk_paths: int = 0

    def c(self, algorithm: int) -> BajoRenderSettingsC:
        return BajoRenderSettingsC(self.width, self.height, self.samples_per_pixel, self.max_depth, self.rng_seed,
                                   algorithm, self.chunk_paths)


def build_lights(scene):
    """Emissive-triangle light records + alias table (host, C ABI)."""
    L = _lib.load()
    max_lights = int(np.count_nonzero((scene.surfaces >> 28) == 3))
    out = np.zeros(max(max_lights, 1) * LIGHT_STRIDE, np.float32)
    n = ctypes.c_uint32(0)
    w = ctypes.c_float(0.0)
    _lib.check(L.bajo_rt_build_lights(scene.vertices.ctypes.data, scene.surfaces.ctypes.data, scene.n_tris,
                                      scene.emissives.ctypes.data, scene.emissives.size // 3, out.ctypes.data,
                                      max_lights, ctypes.byref(n), ctypes.byref(w)), "bajo_rt_build_lights")
    return out, n.value, w.value


class GpuRtTriangleScene:
    """A scene resident on the GPU: LBVH, surfaces, materials, lights
    (GpuRtTriangleScene, bajo/rt/gpu/triangle_path.mojo:57)."""

    def __init__(self, scene, device="cuda", bvh_policy: str = DEFAULT_BVH_POLICY):
        if bvh_policy not in BVH_POLICIES:
            raise ValueError(f"bvh_policy must be one of {BVH_POLICIES}")
        self.host = scene
        self.bvh_policy = bvh_policy
        self.vertices = torch.from_numpy(scene.vertices).to(device)
        self.tree = bvh.build_triangle_bvh(self.vertices, method="hploc" if bvh_policy == "cwbvh8_hploc" else "lbvh")
        self.cwbvh8 = wide.build_cwbvh8(self.tree) if bvh_policy.startswith("cwbvh8") else None
        self.surfaces = torch.from_numpy(scene.surfaces.view(np.int32)).to(device)
        self.lambertians = torch.from_numpy(scene.lambertians).to(device)
        self.emissives = torch.from_numpy(scene.emissives).to(device)
        metals, dielectrics = getattr(scene, "metals", None), getattr(scene, "dielectrics", None)
        self.metals = None if metals is None or metals.size == 0 else torch.from_numpy(metals).to(device)
        self.dielectrics = (None if dielectrics is None or dielectrics.size == 0
                            else torch.from_numpy(dielectrics).to(device))
        lights, self.n_lights, self.total_light_weight = build_lights(scene)
        self.lights_host = lights
        self.lights = torch.from_numpy(lights).to(device)
        self._tree_c = self.tree.c_struct()

    def c(self) -> BajoRtSceneC:
        s = BajoRtSceneC()
        s.bvh = ctypes.pointer(self._tree_c)
        s.surfaces = self.surfaces.data_ptr()
        s.lambertians = self.lambertians.data_ptr()
        s.emissives = self.emissives.data_ptr()
        s.lights = self.lights.data_ptr()
        s.n_lights = self.n_lights
        s.total_light_weight = self.total_light_weight
        s.metals = None if self.metals is None else self.metals.data_ptr()
        s.dielectrics = None if self.dielectrics is None else self.dielectrics.data_ptr()
        if self.cwbvh8 is not None:
            s.cwbvh8 = ctypes.pointer(self.cwbvh8._c)
            s.cwbvh8_nodes = self.cwbvh8.n_nodes
        return s


class RenderWorkspace:
    def __init__(self, settings: RenderSettings, algorithm: int, device="cuda"):
        nbytes = ctypes.c_size_t(0)
        c = settings.c(algorithm)
        _lib.check(_lib.load().bajo_render_workspace_size(ctypes.byref(c), ctypes.byref(nbytes)),
                   "bajo_render_workspace_size")
        self.buffer = torch.zeros(nbytes.value, dtype=torch.uint8, device=device)

    def ray_counts(self):
        """(closest-hit rays, shadow rays) traced by the last render."""
        a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        _lib.check(_lib.load().bajo_render_stats(self.buffer.data_ptr(), _lib.stream_handle(), ctypes.byref(a),
                                                 ctypes.byref(b)), "bajo_render_stats")
        return a.value, b.value

    def status(self) -> int:
        st = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_workspace_status(self.buffer.data_ptr(), _lib.stream_handle(),
                                                     ctypes.byref(st)), "bajo_workspace_status")
        return st.value


def render_gpu_triangles(settings: RenderSettings, camera, scene: GpuRtTriangleScene, algorithm: int = MIS,
                         workspace: RenderWorkspace | None = None, pixels: torch.Tensor | None = None,
                         pixels64: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """Render and return a (height, width, 3) float32 CUDA tensor of mean
    radiance.  `pixels64` (optional, float64) accumulates per-pixel sums."""
    dev = scene.vertices.device
    cam = camera if isinstance(camera, torch.Tensor) else torch.from_numpy(np.asarray(camera, np.float32)).to(dev)
    if workspace is None:
        workspace = RenderWorkspace(settings, algorithm, dev)
    if pixels is None:
        pixels = torch.empty((settings.height, settings.width, 3), dtype=torch.float32, device=dev)
    c = settings.c(algorithm)
    sc = scene.c()
    rc = _lib.load().bajo_render(ctypes.byref(sc), cam.data_ptr(), ctypes.byref(c), pixels.data_ptr(),
                                 None if pixels64 is None else pixels64.data_ptr(), workspace.buffer.data_ptr(),
                                 workspace.buffer.numel(), _lib.stream_handle(stream))
    _lib.check(rc, "bajo_render")
    return pixels


class Renderer:
    """Handle-based rendering (bajo_render_create / enqueue / download /
    destroy): the settings and workspace are fixed at creation; the first
    enqueue on a non-default stream records the render into a CUDA graph,
    later enqueues with the same buffers replay it with one launch."""

    def __init__(self, settings: RenderSettings, algorithm: int = MIS, device="cuda"):
        self.settings, self.algorithm = settings, algorithm
        self.workspace = RenderWorkspace(settings, algorithm, device)
        self._c = settings.c(algorithm)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().bajo_render_create(ctypes.byref(self._c), self.workspace.buffer.data_ptr(),
                                                  self.workspace.buffer.numel(), ctypes.byref(h)),
                   "bajo_render_create")
        self._h = h
        self._scene_c = None

    def enqueue(self, scene: GpuRtTriangleScene, camera: torch.Tensor, pixels: torch.Tensor,
                pixels64: torch.Tensor | None = None, guide=None, stream=None) -> None:
        self._scene_c = scene.c()  # kept alive: the graph was recorded with its pointers
        rc = _lib.load().bajo_render_enqueue(self._h, ctypes.byref(self._scene_c), camera.data_ptr(),
                                             None if guide is None else ctypes.byref(guide), pixels.data_ptr(),
                                             None if pixels64 is None else pixels64.data_ptr(),
                                             _lib.stream_handle(stream))
        _lib.check(rc, "bajo_render_enqueue")

    def download(self, pixels: torch.Tensor, stream=None):
        """(host float32 image, closest-hit rays, shadow rays, status)."""
        out = np.empty((self.settings.height, self.settings.width, 3), np.float32)
        a, b, st = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_render_download(self._h, pixels.data_ptr(), out.ctypes.data, ctypes.byref(a),
                                                    ctypes.byref(b), ctypes.byref(st), _lib.stream_handle(stream)),
                   "bajo_render_download")
        return out, a.value, b.value, st.value

    def graph_launches(self) -> int:
        n = ctypes.c_uint32(0)
        _lib.check(_lib.load().bajo_render_graph_launches(self._h, ctypes.byref(n)), "bajo_render_graph_launches")
        return n.value

    def close(self) -> None:
        if self._h:
            _lib.load().bajo_render_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass
