"""Learned path guiding: a small MLP proposal trained online by the tracer.

The network maps an encoded surface point (one-blob position in the scene
box, 3 x 16 bins, and one-blob octahedral normal, 2 x 8 bins) through three
ReLU layers of 64 to a mixture of 4 von Mises-Fisher lobes.  Its FP16
forward, backward and Adam kernels run on the tensor cores
(``bajo_mlp_*`` in the C ABI); the guided tracer
(``bajo_render_guided``) evaluates it inside its shading kernel and draws
each continuation by one-sample MIS between the cosine BSDF and the mixture,
so the image stays unbiased whatever the network has learnt.  Training
records (vertex, sampled direction, weight L_i cos / pdf) come from the
tracer's own paths; ``GuidedRenderer`` alternates render passes with Adam
steps on them.

The reference has no guiding; the rendering it wraps is the MIS tracer of
``render_gpu_triangles`` (bajo/rt/gpu/triangle_path.mojo:143), which is also
the fallback (``guide_fraction = 0``) and the judge of its error.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, rt

GUIDED = 5
N_OUT = 20
IN, HID, OUT_PAD = 64, 64, 32
LAYER = HID * IN + HID


def param_count() -> int:
    n = ctypes.c_uint32(0)
    _lib.check(_lib.load().bajo_mlp_param_count(ctypes.byref(n)), "bajo_mlp_param_count")
    return n.value


N_PARAMS = 3 * LAYER + OUT_PAD * HID + OUT_PAD  # 14560, checked against the library in the tests


def offsets():
    """(weight offset, bias offset, rows, cols) of the four layers."""
    out = []
    for l in range(3):
        out.append((l * LAYER, l * LAYER + HID * IN, HID, IN))
    out.append((3 * LAYER, 3 * LAYER + OUT_PAD * HID, OUT_PAD, HID))
    return out


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform hidden layers, small output layer (broad lobes: log kappa
    bias 1), zero biases elsewhere; padded output rows zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for l, (w, b, rows, cols) in enumerate(offsets()):
        bound = np.sqrt(6.0 / cols) * (1.0 if l < 3 else 0.1)
        W = rng.uniform(-bound, bound, size=(rows, cols)).astype(np.float32)
        if l == 3:
            W[N_OUT:] = 0.0
        p[w:w + rows * cols] = W.reshape(-1)
    b4 = 3 * LAYER + OUT_PAD * HID
    p[b4 + 3:b4 + N_OUT:5] = 1.0  # log kappa of each lobe
    return p


class BajoGuideC(ctypes.Structure):
    _fields_ = [("params16", ctypes.c_void_p), ("box6", ctypes.c_void_p), ("guide_fraction", ctypes.c_float),
                ("record_fraction", ctypes.c_float), ("record_capacity", ctypes.c_uint32),
                ("records", ctypes.c_void_p)]


class BajoGuideNetC(ctypes.Structure):
    _fields_ = [("params32", ctypes.c_void_p), ("params16", ctypes.c_void_p), ("adam_m", ctypes.c_void_p),
                ("adam_v", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("loss", ctypes.c_void_p),
                ("step", ctypes.c_uint32), ("status", ctypes.c_void_p)]


class GuideNetwork:
    """FP32 master weights + FP16 copy + Adam moments on the device."""

    def __init__(self, device="cuda", seed: int = 0, params: np.ndarray | None = None):
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.params32 = torch.from_numpy(p.copy()).to(device)
        self.params16 = self.params32.to(torch.float16)
        self.adam_m = torch.zeros_like(self.params32)
        self.adam_v = torch.zeros_like(self.params32)
        self.grad_buf = torch.zeros_like(self.params32)
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)  # timeout bit of the gradient kernel
        self.step = 0

    def c(self) -> BajoGuideNetC:
        return BajoGuideNetC(self.params32.data_ptr(), self.params16.data_ptr(), self.adam_m.data_ptr(),
                             self.adam_v.data_ptr(), self.grad_buf.data_ptr(), self.loss_buf.data_ptr(), self.step,
                             self.status.data_ptr())

    def forward(self, pos: torch.Tensor, nrm: torch.Tensor, box: torch.Tensor, stream=None,
                tensor_memory: bool = False, status: torch.Tensor | None = None) -> torch.Tensor:
        """Raw outputs [n, 20]; ``tensor_memory`` runs the tcgen05 kernel
        (``status``: an optional int32 device word for its timeout bit)."""
        n = pos.numel() // 3
        out = torch.empty((n, N_OUT), dtype=torch.float32, device=pos.device)
        L = _lib.load()
        if tensor_memory:
            _lib.check(L.bajo_mlp_forward_tc(self.params16.data_ptr(), pos.data_ptr(), nrm.data_ptr(), n,
                                             box.data_ptr(), out.data_ptr(),
                                             status.data_ptr() if status is not None else None,
                                             _lib.stream_handle(stream)), "bajo_mlp_forward_tc")
        else:
            _lib.check(L.bajo_mlp_forward(self.params16.data_ptr(), pos.data_ptr(), nrm.data_ptr(), n,
                                          box.data_ptr(), out.data_ptr(), _lib.stream_handle(stream)),
                       "bajo_mlp_forward")
        return out

    def gradient(self, pos, nrm, dirs, weights, box, stream=None, tensor_memory: bool = True):
        """(gradient tensor, loss tensor) of sum -w log pdf(dir); the
        tcgen05 kernel (the one training uses) unless ``tensor_memory`` is
        false, then the mma.sync kernel."""
        n = pos.numel() // 3
        L = _lib.load()
        if tensor_memory:
            _lib.check(L.bajo_mlp_grad_tc(self.params16.data_ptr(), pos.data_ptr(), nrm.data_ptr(), dirs.data_ptr(),
                                          weights.data_ptr(), n, box.data_ptr(), self.grad_buf.data_ptr(),
                                          self.loss_buf.data_ptr(), self.status.data_ptr(),
                                          _lib.stream_handle(stream)), "bajo_mlp_grad_tc")
        else:
            _lib.check(L.bajo_mlp_grad(self.params16.data_ptr(), pos.data_ptr(), nrm.data_ptr(), dirs.data_ptr(),
                                       weights.data_ptr(), n, box.data_ptr(), self.grad_buf.data_ptr(),
                                       self.loss_buf.data_ptr(), _lib.stream_handle(stream)), "bajo_mlp_grad")
        return self.grad_buf, self.loss_buf

    def adam(self, lr: float = 1e-2, grad_scale: float = 1.0, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.step += 1
        _lib.check(_lib.load().bajo_mlp_adam(self.params32.data_ptr(), self.params16.data_ptr(),
                                             self.grad_buf.data_ptr(), self.adam_m.data_ptr(),
                                             self.adam_v.data_ptr(), self.step, lr, beta1, beta2, eps, grad_scale,
                                             _lib.stream_handle(stream)), "bajo_mlp_adam")

    # ---- checkpoint ---------------------------------------------------------
    # A plain dump of the training state: FP32 master weights, their FP16
    # copy, both Adam moments and the step count, so that training resumes
    # exactly where it stopped (the next Adam step sees the same state).
    def state(self) -> dict:
        torch.cuda.synchronize()
        return {"params32": self.params32.cpu().numpy(), "params16": self.params16.cpu().numpy(),
                "adam_m": self.adam_m.cpu().numpy(), "adam_v": self.adam_v.cpu().numpy(),
                "step": np.int64(self.step), "n_params": np.int64(N_PARAMS)}

    def save(self, path: str) -> None:
        np.savez(path, **self.state())

    @classmethod
    def load(cls, path: str, device="cuda") -> "GuideNetwork":
        with np.load(path) as z:
            if int(z["n_params"]) != N_PARAMS:
                raise ValueError(f"checkpoint holds {int(z['n_params'])} parameters, the network has {N_PARAMS}")
            net = cls(device, params=z["params32"])
            net.params16.copy_(torch.from_numpy(z["params16"]).to(device))
            net.adam_m.copy_(torch.from_numpy(z["adam_m"]).to(device))
            net.adam_v.copy_(torch.from_numpy(z["adam_v"]).to(device))
            net.step = int(z["step"])
        return net

    def train_records(self, records: "GuideRecords", box: torch.Tensor, batch: int, steps: int, lr: float = 1e-2,
                      stream=None):
        """`steps` Adam steps on `batch` records each (count read on device)."""
        c = self.c()
        _lib.check(_lib.load().bajo_guide_train(ctypes.byref(c), records.buffer.data_ptr(), records.capacity,
                                                box.data_ptr(), batch, steps, lr, _lib.stream_handle(stream)),
                   "bajo_guide_train")
        self.step = c.step


def _a256(x: int) -> int:
    return (x + 255) & ~255


class GuideRecords:
    """Training-record buffer written by the guided tracer."""

    def __init__(self, capacity: int, device="cuda"):
        nbytes = ctypes.c_size_t(0)
        _lib.check(_lib.load().bajo_guide_records_size(capacity, ctypes.byref(nbytes)), "bajo_guide_records_size")
        self.capacity = capacity
        self.buffer = torch.zeros(nbytes.value, dtype=torch.uint8, device=device)
        c = capacity
        o = 256
        self._off = {}
        for name, nb in (("pos", 12 * c), ("nrm", 12 * c), ("dir", 12 * c), ("weight", 4 * c)):
            self._off[name] = o
            o = _a256(o + nb)

    def reset(self):
        self.buffer[:8].zero_()

    def count(self) -> int:
        return min(int(self.buffer[:4].view(torch.int32).item()) & 0xFFFFFFFF, self.capacity)

    def arrays(self):
        """(pos [n,3], nrm [n,3], dir [n,3], weight [n]) views of the stored records."""
        n = self.count()
        f = self.buffer.view(torch.float32)
        out = []
        for name, k in (("pos", 3), ("nrm", 3), ("dir", 3), ("weight", 1)):
            s = self._off[name] // 4
            a = f[s:s + k * n]
            out.append(a.view(n, k) if k > 1 else a)
        return tuple(out)


class GuidedRenderer:
    """Progressive guided rendering: each pass renders `spp_per_pass`
    samples per pixel with the current network (and collects records);
    passes up to `train_passes` are each followed by `steps` Adam steps."""

    def __init__(self, scene: rt.GpuRtTriangleScene, camera, width: int, height: int, max_depth: int = 8,
                 guide_fraction: float = 0.5, record_capacity: int = 1 << 18, record_fraction: float | None = None,
                 network: GuideNetwork | None = None, lr: float = 1e-2, batch: int = 1 << 14, steps: int = 8,
                 chunk_paths: int = 0, spp_per_pass: int = 1):
        dev = scene.vertices.device
        self.scene = scene
        self.cam = camera if isinstance(camera, torch.Tensor) else torch.from_numpy(
            np.asarray(camera, np.float32)).to(dev)
        self.width, self.height, self.max_depth = width, height, max_depth
        self.spp_per_pass = spp_per_pass
        self.guide_fraction = guide_fraction
        self.net = network or GuideNetwork(dev)
        self.records = GuideRecords(record_capacity, dev)
        # expect about two continued vertices per path
        paths = width * height * spp_per_pass
        self.record_fraction = record_fraction if record_fraction is not None else min(
            1.0, record_capacity / max(1.0, 2.0 * paths))
        self.lr, self.batch, self.steps = lr, batch, steps
        self.box = scene.tree.seg_bounds[:6]
        self.settings = rt.RenderSettings(width, height, spp_per_pass, max_depth=max_depth, chunk_paths=chunk_paths)
        self.workspace = rt.RenderWorkspace(self.settings, GUIDED, dev)
        self._chunk_paths = chunk_paths
        self._by_spp = {spp_per_pass: (self.settings, self.workspace)}
        self.pixels = torch.empty((height, width, 3), dtype=torch.float32, device=dev)
        self.sum64 = torch.zeros((height, width, 3), dtype=torch.float64, device=dev)
        self.samples = 0
        self.passes = 0

    def guide_c(self, fraction: float, collect: bool) -> BajoGuideC:
        return BajoGuideC(self.net.params16.data_ptr(), self.box.data_ptr(), fraction, self.record_fraction,
                          self.records.capacity if collect else 0, self.records.buffer.data_ptr() if collect else None)

    def prepare_pass(self, spp: int) -> None:
        """Allocate the workspace of passes of `spp` samples per pixel now,
        so that the first such pass does not pay for the allocation."""
        self._settings_for(spp)

    def _settings_for(self, spp: int):
        """Settings and workspace of a pass of `spp` samples per pixel (the
        workspace's path capacity depends on it)."""
        if spp not in self._by_spp:
            s = rt.RenderSettings(self.width, self.height, spp, max_depth=self.max_depth,
                                  chunk_paths=self._chunk_paths)
            self._by_spp[spp] = (s, rt.RenderWorkspace(s, GUIDED, self.workspace.buffer.device))
        return self._by_spp[spp]

    def render_pass(self, seed: int, train: bool = True, guide_fraction: float | None = None, stream=None,
                    spp: int | None = None):
        """One pass of `spp` samples per pixel (default spp_per_pass) added
        into the FP64 sum; trains afterwards when asked.  Larger passes after
        training use the GPU better: the later bounces' kernels of a small
        pass run with few paths."""
        f = self.guide_fraction if guide_fraction is None else guide_fraction
        spp = self.spp_per_pass if spp is None else spp
        settings, workspace = self._settings_for(spp)
        self.workspace = workspace
        settings.rng_seed = seed
        c = settings.c(GUIDED)
        if train:
            self.records.reset()
        g = self.guide_c(f, train)
        sc = self.scene.c()
        L = _lib.load()
        _lib.check(L.bajo_render_guided(ctypes.byref(sc), self.cam.data_ptr(), ctypes.byref(c), ctypes.byref(g),
                                        self.pixels.data_ptr(), self.sum64.data_ptr(),
                                        self.workspace.buffer.data_ptr(), self.workspace.buffer.numel(),
                                        _lib.stream_handle(stream)), "bajo_render_guided")
        if train:
            self.net.train_records(self.records, self.box, self.batch, self.steps, self.lr, stream)
        self.samples += spp
        self.passes += 1

    def render(self, passes: int, train_passes: int, seed: int = 2026) -> torch.Tensor:
        """`passes` passes, training after the first `train_passes`; returns
        the FP64 mean image."""
        for k in range(passes):
            self.render_pass(seed + 7919 * (self.passes + 1), train=k < train_passes)
        return self.image()

    def image(self) -> torch.Tensor:
        return self.sum64 / max(self.samples, 1)

    def reset_image(self):
        self.sum64.zero_()
        self.samples = 0
