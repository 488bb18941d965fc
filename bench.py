#!/usr/bin/env python
"""Benchmark of the LBVH build + closest-hit path on B200.

Workload (plain LBVH): 65,536 triangles, each a centroid uniform in [0,1]^3
plus three vertex offsets uniform in +-0.01 per axis (seed 0, FP32); 30-bit
Morton codes; one LBVH build per step.  The closest-hit figure traces
1024x1024 pinhole rays from (0.5, 0.5, -1.5) looking +z with a 60 degree
vertical field of view against the built tree.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl bajo|reference]

One JSON line on rank 0.  `value` is the device-timed LBVH build throughput
(Mtri/s, inputs resident in HBM, L2 flushed before every timed step); `e2e`
is the same metric through the public API with the vertex upload from pinned
host memory and the read-back of the root bounds + status inside the timed
region; `closest_hit` reports MRays/s of the traversal.  With --impl
reference the restated reference CPU builder runs on the host cores.
Multi-GPU runs are replicas: every rank builds its own copy of the scene.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_TRIS = 65536
WIDTH = HEIGHT = 1024
METRIC = "LBVH build Mtri/s"
UNIT = "Mtri/s"
WORKLOAD = "plain LBVH build of 65,536 random triangles (seed 0) + 1024x1024 closest-hit camera rays"
# Algorithmic bytes of one onesweep digit pass over the LBVH sort (the
# per-stage build): read and write one u64 key and one u32 payload per key.
PASS_BYTES_PER_KEY = 24
# Algorithmic bytes per triangle of the build kernels.
#  lbvh_fused_kernel (the one-launch build): bounds (vertices 36 read, leaf
#    bounds 24 written, arrival counter 4 cleared), bucket sort of u32 code +
#    u32 id (8 written to the buckets, 8 read back, 16 written as sorted
#    codes, ids and u64 keys), hierarchy (codes 4, ids 4 and vertices 36
#    read; triangle record 48, node meta 16, node boxes 48, leaf count 4,
#    arrival counter 4 and parent link 4 written).
#  hierarchy_kernel (per-stage build): the hierarchy part alone.
_HIER_BYTES = 4 + 4 + 36 + 48 + 16 + 48 + 4 + 4 + 4
KERNEL_BYTES_PER_TRI = {"lbvh_fused_kernel": 36 + 24 + 4 + 8 + 8 + 16 + _HIER_BYTES,
                        "hierarchy_kernel": _HIER_BYTES}
# digit passes of the single-scene LBVH sort: 8-bit digits over the 30-bit
# Morton code, bits [0, 32) (the reference CPU builder's four byte passes,
# bajo/bvh/cpu/builder/lbvh.mojo:56-62)
CPU_SORT_PASSES = 4
HIT_BYTES = 32      # 8-word hit written per ray
NODE_BYTES = 64     # 48 B child boxes + 16 B child refs per visited node
TRI_BYTES = 48      # packed triangle record per triangle test


def workload_triangles(n: int = N_TRIS, seed: int = 0, spread: float = 0.01):
    """The plain LBVH workload's triangles: centroids uniform in [0,1]^3 plus
    three vertex offsets uniform in +-spread per axis, FP32, seeded.  The same
    numpy calls as bajo_b200.scenes.random_triangles, repeated here so the
    reference arm imports nothing from bajo_b200."""
    import numpy as np
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3), dtype=np.float32)
    off = rng.uniform(-spread, spread, size=(n, 3, 3)).astype(np.float32)
    return np.ascontiguousarray((c + off).reshape(n * 9), dtype=np.float32)


def workload_camera():
    """The workload's pinhole camera through the oracle's restatement of
    Camera.from_vfov (bajo/bvh/camera.mojo): eye (0.5, 0.5, -1.5) looking +z,
    60 degree vertical field of view."""
    from oracle import oracle as O
    return O.camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, -0.5], [0.0, 1.0, 0.0], 60.0)


def workload_config() -> dict:
    """The `config` both arms print (identical dicts)."""
    return {"workload": WORKLOAD, "triangles": N_TRIS, "rays": WIDTH * HEIGHT, "seed": 0, "morton_bits": 30,
            "l2": "GPU arm: 256 MiB device write before every timed build and trace; CPU arm: host caches as they are"}


def parse(argv=None):
    return parse_args(argv)


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="bajo", choices=["bajo", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample length")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-sweep", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the render, batched and guided workloads")
    p.add_argument("--case", default=None,
                   choices=["sort", "build", "trace", "wide", "cwbvh8", "hploc", "tlas", "tune", "render",
                            "batched", "guided", "guided_pass", "mlp_forward", "mlp_train"],
                   help="time one piece alone (profiling runs) instead of the benchmark line")
    p.add_argument("--n", type=int, default=1 << 24, help="--case size (keys or triangles)")
    p.add_argument("--bits", type=int, default=32, choices=[32, 64], help="--case sort key width")
    p.add_argument("--end-bit", type=int, default=None, help="--case sort: sort bits [0, end-bit)")
    p.add_argument("--keys-only", action="store_true", help="--case sort without payload")
    p.add_argument("--node-width", type=int, default=4, choices=[4, 8], help="--case wide node width")
    p.add_argument("--method", default="lbvh", choices=["lbvh", "hploc"],
                   help="--case wide / cwbvh8: binary builder under the wide tree")
    p.add_argument("--max-leaf", type=int, default=4, choices=[1, 2, 3, 4], help="--case wide leaf block size")
    p.add_argument("--scene", default="spheres", choices=["spheres", "indirect", "spheres_up", "door"],
                   help="--case guided scene (spheres_up: the path-tracing workload with its light facing the "
                        "ceiling)")
    p.add_argument("--width", type=int, default=1280, help="--case guided image width")
    p.add_argument("--height", type=int, default=720, help="--case guided image height")
    p.add_argument("--ref-spp", type=int, default=4096, help="--case guided reference samples per pixel")
    p.add_argument("--spp-per-pass", type=int, default=2, help="--case guided samples per pixel per pass")
    p.add_argument("--spp", type=int, default=64, help="--case render samples per pixel")
    p.add_argument("--scenes", type=int, default=4096, help="--case batched scene count")
    p.add_argument("--train-passes", type=int, default=8, help="--case guided passes followed by training")
    p.add_argument("--first-guided", action="store_true",
                   help="--case guided: guide the first pass too (by default it samples the BSDF only, since the "
                        "network is untrained)")
    p.add_argument("--train-steps", type=int, default=64, help="--case guided Adam steps per training pass")
    p.add_argument("--late-spp", type=int, default=4,
                   help="--case guided samples per pixel of the passes after the training passes")
    p.add_argument("--records", type=int, default=1 << 20,
                   help="--case guided training records kept per pass (batches of 2^14 are drawn from them)")
    return p.parse_args(argv)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per launch of the onesweep pass from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML every 5 ms while
    the timed region runs (nvidia-smi's 200 ms loop is longer than the
    region itself)."""
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, device_index=0, period=0.005):
        self.device_index = device_index
        self.period = period
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self._h = None
        self._nvml = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        self._nvml = pynvml
        try:
            props = torch.cuda.get_device_properties(self.device_index)
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.device_index)

    def _sample(self):
        n = self._nvml
        sm = n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM)
        try:
            reasons = n.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        except Exception:
            reasons = n.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
        self.samples.append((sm, reasons))

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            time.sleep(self.period)

    def __enter__(self):
        try:
            self._h = self._handle()
            self.max_mhz = self._nvml.nvmlDeviceGetMaxClockInfo(self._h, self._nvml.NVML_CLOCK_SM)
            self._sample()
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        except Exception:
            self._h = None
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=1)
        if self._h is not None:
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples]
        reasons = sorted(name for name, bit in self.BITS.items() if any(r & bit for _, r in self.samples))
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples), "source": "nvml"}


# ----------------------------------------------------------------- distributed
def dist_setup(args):
    """One process per GPU over NCCL (torchrun sets RANK / WORLD_SIZE /
    LOCAL_RANK / MASTER_*); see bajo_b200/dist.py."""
    from bajo_b200 import dist
    return dist.init()


def barrier(world):
    from bajo_b200 import dist
    dist.barrier(world)


def max_over_ranks(world, x: float) -> float:
    from bajo_b200 import dist
    return dist.max_over_ranks(world, x)


# ----------------------------------------------------------------- CPU baseline
def cpu_baseline(verts, seconds):
    """The restated reference CPU LBVH builder (bajo/bvh/cpu/builder/lbvh.mojo)
    on every host thread: a bounded sample of repeated 65,536-tri builds."""
    from oracle import oracle as O
    O.build()
    cb = O.CpuLbvh(verts)
    cb.build()
    t0 = time.perf_counter()
    builds = 0
    while time.perf_counter() - t0 < seconds:
        cb.build()
        builds += 1
    dt = time.perf_counter() - t0
    return {"value": round(N_TRIS * builds / dt / 1e6, 3), "unit": UNIT, "cores": cb.threads, "kind": "port",
            "sample": f"{builds} builds of the 65,536-triangle scene in {dt:.1f} s (C restatement of the "
                      "reference CPU LBVH builder, all host threads)"}


def cpu_trace_sample(verts, stride=16):
    from oracle import oracle as O
    cb = O.CpuLbvh(verts)
    cb.build()
    rays = O.camera_rays(workload_camera(), WIDTH * HEIGHT, WIDTH, HEIGHT).reshape(8, -1)
    sub = rays[:, ::stride].copy().reshape(-1)
    n = sub.size // 8
    cb.trace(sub)
    seconds = float(os.environ.get("BENCH_CPU_TRACE_SECONDS", "2.0"))
    t0 = time.perf_counter()
    reps = 0
    while True:
        cb.trace(sub)
        reps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = (time.perf_counter() - t0) / reps
    return n / dt / 1e6, cb.threads, n


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    verts = workload_triangles()
    cb = O.CpuLbvh(verts)
    for _ in range(max(args.warmup, 1)):
        cb.build()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cb.build()
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = N_TRIS * args.steps / total / 1e6
    mrays, cores, nsample = cpu_trace_sample(verts)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(), "parallelism": f"{cb.threads} host threads", "sort_passes": CPU_SORT_PASSES,
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cb.threads, "kind": "port",
                         "sample": f"{args.steps} full builds of the 65,536-triangle scene (C restatement of the "
                                   "reference CPU LBVH builder; Mojo is unavailable here)"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "closest_hit": {"value": round(mrays, 3), "unit": "MRays/s",
                        "sample": f"{nsample} of the 1024x1024 camera rays (every 16th), {cores} threads"},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- GPU arm
def run_bajo(args):
    import numpy as np
    import torch

    world, rank, local = dist_setup(args)
    from bajo_b200 import build as B
    if rank == 0 or world == 1:
        B.build()
    barrier(world)
    from bajo_b200 import _lib, bvh, camera, scenes

    L = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream

    verts_h = workload_triangles()
    verts = torch.from_numpy(verts_h).to(dev)
    ws = bvh.GpuBvhBuildWorkspace(N_TRIS, 1, device=dev)
    tree = bvh.build_triangle_bvh(verts, workspace=ws)
    # builds and traces go through the tree record as built (no staged top
    # levels: the tree was created without them, the reference's layout)
    c = tree.c_struct(stage_top=False)
    c_trace = tree.c_struct()
    cam = torch.from_numpy(camera.plain_lbvh_camera()).to(dev)
    n_rays = WIDTH * HEIGHT
    hits = torch.empty(8 * n_rays, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def stage_count():
        x = ctypes.c_int32(0)
        _lib.check(L.bajo_lbvh_stage_count(N_TRIS, 1, ctypes.byref(x)), "bajo_lbvh_stage_count")
        return x.value

    launches = ctypes.c_int32(0)
    _lib.check(L.bajo_lbvh_build_launches(N_TRIS, 1, ctypes.byref(launches)), "bajo_lbvh_build_launches")
    kernels_per_build = launches.value  # 1: the one-launch build
    n_ev = stage_count()                # 2: [start, build]

    def build_timed(events):
        arr = (ctypes.c_void_p * len(events))(*[e.cuda_event for e in events])
        _lib.check(L.bajo_lbvh_build_timed(verts.data_ptr(), ctypes.byref(c), ws.buffer.data_ptr(),
                                           ws.buffer.numel(), sh, arr, len(events)), "bajo_lbvh_build_timed")

    def build_plain():
        _lib.check(L.bajo_lbvh_build(verts.data_ptr(), ctypes.byref(c), ws.buffer.data_ptr(), ws.buffer.numel(), sh),
                   "bajo_lbvh_build")

    def new_events(k):
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        for e in evs:
            e.record(stream)  # materialise the handles
        return evs

    def trace(h=None):
        _lib.check(L.bajo_trace_camera(ctypes.byref(c_trace), cam.data_ptr(), n_rays, WIDTH, HEIGHT,
                                       _lib.TRI_WATERTIGHT, h.data_ptr(), None, None, None, sh), "bajo_trace_camera")

    # ---- warm-up
    evs = new_events(n_ev)
    for _ in range(args.warmup):
        build_plain()
        build_timed(evs)
        trace(hits)
    torch.cuda.synchronize()

    # ---- device-timed region: K builds through the public entry point with
    # events only around each build, K traces, then K builds with an event
    # between their kernels (the per-kernel split of the roofline entry)
    step_events = [new_events(2) for _ in range(args.steps)]
    stage_events = [new_events(n_ev) for _ in range(args.steps)]
    trace_events = [new_events(2) for _ in range(args.steps)]
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.zero_()
            step_events[k][0].record(stream)
            build_plain()
            step_events[k][1].record(stream)
            flush.zero_()
            trace_events[k][0].record(stream)
            trace(hits)
            trace_events[k][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        build_timed(stage_events[k])
    torch.cuda.synchronize()
    build_ms = [e[0].elapsed_time(e[1]) for e in step_events]
    trace_ms = [e[0].elapsed_time(e[1]) for e in trace_events]
    build_total = max_over_ranks(world, sum(build_ms) / 1e3)
    trace_total = max_over_ranks(world, sum(trace_ms) / 1e3)
    value = world * N_TRIS * args.steps / build_total / 1e6
    mrays = world * n_rays * args.steps / trace_total / 1e6

    # ---- the per-stage kernels of the same build (one scene takes them when
    # the one-launch build is switched off), with an event between every kernel
    _lib.check(L.bajo_lbvh_fused_max_set(0), "bajo_lbvh_fused_max_set")
    n_stage = stage_count()
    passes = n_stage - 5
    stage_ev = [new_events(n_stage) for _ in range(args.steps)]
    build_timed(stage_ev[0])
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        build_timed(stage_ev[k])
    torch.cuda.synchronize()
    _lib.check(L.bajo_lbvh_fused_max_set(_lib.FUSED_MAX_LEAVES), "bajo_lbvh_fused_max_set")
    pass_ms = [e[2 + p].elapsed_time(e[3 + p]) for e in stage_ev for p in range(passes)]
    stage = {
        "bounds": statistics.mean(e[0].elapsed_time(e[1]) for e in stage_ev),
        "morton": statistics.mean(e[1].elapsed_time(e[2]) for e in stage_ev),
        "sort": statistics.mean(e[2].elapsed_time(e[2 + passes]) for e in stage_ev),
        "hierarchy": statistics.mean(e[2 + passes].elapsed_time(e[4 + passes]) for e in stage_ev),
    }

    # ---- roofline: the build's dominant kernel (with the one-launch build its
    # only kernel; its events bracket that launch and a 4 KB memset)
    peak, peak_kind = measured_peaks()
    if n_ev == 2:
        kern_us = {"lbvh_fused_kernel": statistics.mean(e[0].elapsed_time(e[1]) for e in stage_events) * 1e3}
    else:  # the per-stage kernels
        kern_us = {"hierarchy_kernel": stage["hierarchy"] * 1e3}
    top = max(kern_us, key=kern_us.get)
    top_bytes = KERNEL_BYTES_PER_TRI[top] * N_TRIS
    achieved = top_bytes / (kern_us[top] / 1e6) / 1e9
    traffic = committed_traffic().get(f"{top}_65536")
    trace_dram = committed_traffic().get("trace_camera_65536")
    # the per-stage build's onesweep pass, for comparison
    pass_avg_s = statistics.mean(pass_ms) / 1e3
    pass_bytes = PASS_BYTES_PER_KEY * N_TRIS

    # ---- traversal instrumented bytes (per-ray node visits / triangle tests)
    stats = torch.empty(5 * n_rays, dtype=torch.int32, device=dev)
    _lib.check(L.bajo_trace_camera_stats(ctypes.byref(c_trace), cam.data_ptr(), n_rays, WIDTH, HEIGHT,
                                         _lib.TRI_WATERTIGHT, None, stats.data_ptr(), sh), "bajo_trace_camera_stats")
    torch.cuda.synchronize()
    st = stats.view(-1, 5).double()  # GpuTraversalStats: visits, child hits, leaf blocks, tri tests, max stack
    nodes_per_ray, tris_per_ray = float(st[:, 0].mean()), float(st[:, 3].mean())
    trace_bytes = n_rays * (nodes_per_ray * NODE_BYTES + tris_per_ray * TRI_BYTES + HIT_BYTES)
    trace_achieved = trace_bytes / (statistics.mean(trace_ms) / 1e3) / 1e9

    # ---- e2e through the public API: every step uploads its vertices from
    # pinned host memory, builds through bajo_lbvh_build and reads the root
    # child boxes back.  Pipelined as a host would drive the C ABI: the upload
    # of step k+1 runs on a copy stream into the other of two device vertex
    # buffers while step k builds, and each read-back runs on a third stream
    # after its build (on the build stream it queued behind the next upload).
    # The serialised form (one stream, step after step) is reported beside it.
    pinned_v = [torch.from_numpy(verts_h).pin_memory() for _ in range(2)]
    out_h = [torch.empty(12, dtype=torch.float32).pin_memory() for _ in range(2)]
    st_h = torch.empty(1, dtype=torch.int32).pin_memory()
    dev_v = [torch.empty_like(verts) for _ in range(2)]
    # two output trees, so a build never overwrites the tree whose root boxes
    # are still being read back (the C-ABI records a host makes, prepared once)
    trees = [tree, bvh.build_triangle_bvh(verts, workspace=ws)]
    c_e2e = [t_.c_struct(stage_top=False) for t_ in trees]
    root_box = [t_.node_bounds[:12] for t_ in trees]
    read_done = [torch.cuda.Event() for _ in range(2)]
    status_word = ws.buffer[:4].view(torch.int32)
    copy_stream = torch.cuda.Stream()
    read_stream = torch.cuda.Stream()
    uploaded = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]

    def e2e_build(k, read_on_side=False):
        b = k % 2
        if read_on_side:
            stream.wait_event(read_done[b])  # the read-back of step k - 2 is done with this tree
        _lib.check(L.bajo_lbvh_build(dev_v[b].data_ptr(), ctypes.byref(c_e2e[b]), ws.buffer.data_ptr(),
                                     ws.buffer.numel(), sh), "bajo_lbvh_build")
        if read_on_side:
            built = torch.cuda.Event()
            built.record(stream)
            with torch.cuda.stream(read_stream):
                read_stream.wait_event(built)
                out_h[b].copy_(root_box[b], non_blocking=True)
                read_done[b].record(read_stream)
        else:
            out_h[b].copy_(root_box[b], non_blocking=True)

    def e2e_pipelined(steps):
        for k in range(steps):
            b = k % 2
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(consumed[b])  # the build that read this buffer is done
                dev_v[b].copy_(pinned_v[b], non_blocking=True)
                uploaded[b].record(copy_stream)
            stream.wait_event(uploaded[b])
            e2e_build(k, read_on_side=True)
            consumed[b].record(stream)

    def e2e_serial(k):
        dev_v[0].copy_(pinned_v[0], non_blocking=True)
        e2e_build(0)

    for b in range(2):
        consumed[b].record(stream)
        read_done[b].record(stream)
    for _ in range(3):  # the pinned-upload path runs slower for its first few hundred copies
        e2e_pipelined(max(args.steps, 50))
    for k in range(2):
        e2e_serial(k)
    torch.cuda.synchronize()
    barrier(world)
    flush.zero_()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    copy_stream.wait_stream(stream)
    read_stream.wait_stream(stream)
    h0 = time.perf_counter()
    e2e_pipelined(args.steps)
    host_enqueue_us = (time.perf_counter() - h0) / args.steps * 1e6
    stream.wait_stream(read_stream)
    e_end.record(stream)
    e_end.synchronize()
    e2e_total = max_over_ranks(world, e_start.elapsed_time(e_end) / 1e3)
    # the upload alone, to show what bounds the pipeline
    h2d_ms = []
    for _ in range(args.steps):
        e_start.record(stream)
        dev_v[0].copy_(pinned_v[0], non_blocking=True)
        e_end.record(stream)
        e_end.synchronize()
        h2d_ms.append(e_start.elapsed_time(e_end))
    serial_ms = []
    for k in range(args.steps):
        flush.zero_()
        e_start.record(stream)
        e2e_serial(k)
        e_end.record(stream)
        e_end.synchronize()
        serial_ms.append(e_start.elapsed_time(e_end))
    # the device status word is sticky (every error sets a bit and nothing
    # clears it between builds), so one read after the timed steps checks them all
    st_h.copy_(status_word)
    if int(st_h.item()) != 0:
        raise RuntimeError(f"device status {int(st_h.item())}")
    e2e_value = world * N_TRIS * args.steps / e2e_total / 1e6
    serial_total = max_over_ranks(world, sum(serial_ms) / 1e3)
    e2e_serial_value = world * N_TRIS * args.steps / serial_total / 1e6

    # ---- sweep (sort and build at larger sizes), rank 0 only
    sweep = None
    if rank == 0 and world == 1 and not args.no_sweep:
        sweep = run_sweep(torch, bvh, _lib, L, dev, stream, peak)
        if not args.no_cpu_baseline:
            sweep["cpu_baseline"] = cpu_sort_baseline(torch, dev)

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras = run_extras(args, local)

    if rank != 0:
        barrier(world)
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(verts_h, args.cpu_seconds)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(build_total / args.steps * 1e3, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(), "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "sort": "bucket sort over the top 12 code bits (LSD passes when a bucket holds more than 256 keys)"
                if kernels_per_build == 1 else f"{passes} onesweep passes",
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(verts.numel() * 4),
                "d2h_bytes_per_step": 12 * 4,
                "what": "every step: pinned H2D of its vertices + bajo_lbvh_build + D2H of the root child boxes; "
                        "uploads on a copy stream into two device buffers overlap the previous step's build, "
                        "read-backs on a third stream; one event pair around all steps (device status read once "
                        "after them)",
                "serial_value": round(e2e_serial_value, 3),
                "serial_what": "the same steps on one stream, one after another, each timed alone",
                "h2d_us_median": round(statistics.median(h2d_ms) * 1e3, 1),
                "h2d_gb_s": round(verts.numel() * 4 / (statistics.median(h2d_ms) / 1e3) / 1e9, 2),
                "host_enqueue_us_per_step": round(host_enqueue_us, 1)},
        "roofline": {"kernel": top, "bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "algorithmic_bytes_per_launch": top_bytes,
                     "algorithmic_bytes_per_triangle": KERNEL_BYTES_PER_TRI[top],
                     "avg_launch_us": round(kern_us[top], 3), "peak_kind": peak_kind,
                     "build_kernels_us": {k: round(v, 3) for k, v in kern_us.items()}},
        "per_stage_build": {
            "what": "the same build through the per-stage kernels (bounds, Morton, onesweep passes, hierarchy; "
                    "bajo_lbvh_fused_max_set(0)), an event between every kernel",
            "stages_ms": {k: round(v, 5) for k, v in stage.items()},
            "onesweep_pass": {"achieved_gb_s": round(pass_bytes / pass_avg_s / 1e9, 2),
                              "frac": round(pass_bytes / pass_avg_s / 1e9 / peak, 4),
                              "avg_launch_us": round(pass_avg_s * 1e6, 3), "bytes_per_launch": pass_bytes,
                              "traffic": committed_traffic().get("onesweep_pass_65536")}},
        "closest_hit": {"value": round(mrays, 3), "unit": "MRays/s", "ms": round(statistics.mean(trace_ms), 4),
                        "nodes_per_ray": round(nodes_per_ray, 3), "tris_per_ray": round(tris_per_ray, 3),
                        "roofline": {"bound": "hbm (instrumented bytes: node + triangle loads, mostly L2)",
                                     "achieved": round(trace_achieved, 2), "peak": peak, "unit": "GB/s",
                                     "frac": round(trace_achieved / peak, 4),
                                     "dram_bytes_per_launch": trace_dram,
                                     "dram_frac": None if trace_dram is None else round(
                                         trace_dram / (statistics.mean(trace_ms) / 1e3) / 1e9 / peak, 4),
                                     "target_basis": "frac (instrumented node + triangle bytes served from "
                                                     "L1/L2/DRAM) is the figure compared with the 40% target; "
                                                     "dram_frac (ncu DRAM bytes of one launch) shows the tree "
                                                     "is cache resident"}},
        "gpu_launches": args.steps * (kernels_per_build + 1),
        "clocks": clocks.summary(),
    }
    if cpu:
        line["cpu_baseline"] = cpu
        try:
            mr, cores, ns = cpu_trace_sample(verts_h)
            line["closest_hit"]["cpu_baseline"] = {"value": round(mr, 3), "unit": "MRays/s", "cores": cores,
                                                   "kind": "port", "sample": f"{ns} rays (every 16th)"}
        except Exception as e:  # pragma: no cover
            line["closest_hit"]["cpu_baseline"] = {"error": str(e)}
    if sweep:
        line["sweep"] = sweep
    line.update(extras)
    print(json.dumps(line), flush=True)
    barrier(world)


# Radix sort sweep workload: N = 2^16 ... 2^28 in powers of 4; uniform u32
# keys (keys only, and with u32 payloads) and 63-bit Morton keys of points in
# 32 Gaussian clusters (sigma 0.02) with u32 payloads.  Algorithmic bytes per
# key (read + write of every live pass, plus one histogram read of the keys):
# u32 keys 4 x 8 + 4 = 36; u32 pairs 4 x 16 + 4 = 68; u64 keys + u32 payload
# over 63 live bits 8 x 24 + 8 = 200.
SWEEP_LOG2 = (16, 18, 20, 22, 24, 26, 28)
SWEEP_KINDS = {"sort_u32_keys": (36, False), "sort_u32_pairs": (68, True), "sort_u64_morton_pairs": (200, True)}
CPU_SORT_LOG2 = 22


def sweep_keys(torch, kind, n, seed, dev):
    """(keys, begin_bit, end_bit) of one sweep point, generated on the device."""
    from bajo_b200 import scenes
    if kind == "sort_u64_morton_pairs":
        p = scenes.clustered_points_torch(n, seed=seed, device=dev)
        k = scenes.morton63_torch(p)
        del p
        return k, 0, 63
    g = torch.Generator(device=dev).manual_seed(seed)
    return torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device=dev, generator=g), 0, 32


# CUB 12.9's radix sort (cub::DeviceRadixSort, the CUDA toolkit's library
# sort) timed on the same device buffers as the sweep: the library baseline
# the sweep is compared with.  Built on first use with the toolkit's nvcc.
CUB_BASELINE_SRC = r"""
#include <cub/cub.cuh>
#include <algorithm>
#include <vector>
#include <cstdint>
extern "C" int cub_sort_ms(int key_bytes, const void* keys, const uint32_t* vals, uint32_t n, int end_bit, int reps,
                           void* flush, size_t flush_bytes, float* median_ms) {
  void *kout = nullptr, *vout = nullptr, *tmp = nullptr;
  size_t tb = 0;
  cudaError_t e = cudaMalloc(&kout, (size_t)n * key_bytes);
  if (e == cudaSuccess && vals) e = cudaMalloc(&vout, (size_t)n * 4);
  auto run = [&](void* t, size_t& b) {
    if (key_bytes == 4 && vals)
      return cub::DeviceRadixSort::SortPairs(t, b, (const uint32_t*)keys, (uint32_t*)kout, vals, (uint32_t*)vout,
                                             (int)n, 0, end_bit);
    if (key_bytes == 4)
      return cub::DeviceRadixSort::SortKeys(t, b, (const uint32_t*)keys, (uint32_t*)kout, (int)n, 0, end_bit);
    if (vals)
      return cub::DeviceRadixSort::SortPairs(t, b, (const uint64_t*)keys, (uint64_t*)kout, vals, (uint32_t*)vout,
                                             (int)n, 0, end_bit);
    return cub::DeviceRadixSort::SortKeys(t, b, (const uint64_t*)keys, (uint64_t*)kout, (int)n, 0, end_bit);
  };
  if (e == cudaSuccess) e = run(nullptr, tb);
  if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  std::vector<float> ms;
  for (int r = 0; e == cudaSuccess && r <= reps; ++r) {
    cudaMemsetAsync(flush, r & 255, flush_bytes);
    cudaEventRecord(a);
    e = run(tmp, tb);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    if (r) ms.push_back(t);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(kout);
  cudaFree(vout);
  cudaFree(tmp);
  if (e != cudaSuccess || ms.empty()) return 1;
  std::sort(ms.begin(), ms.end());
  *median_ms = ms[ms.size() / 2];
  return 0;
}
"""


def cub_baseline_lib():
    """ctypes handle of the CUB timing library (built once into the package's
    build folder), or None when nvcc or the build is not available."""
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    out_dir = os.path.join(here, "bajo_b200", "_build", "cub_baseline")
    so = os.path.join(out_dir, "libcub_sort_baseline.so")
    src = os.path.join(out_dir, "cub_sort_baseline.cu")
    try:
        os.makedirs(out_dir, exist_ok=True)
        if not os.path.exists(so) or not os.path.exists(src) or open(src).read() != CUB_BASELINE_SRC:
            with open(src, "w") as f:
                f.write(CUB_BASELINE_SRC)
            nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
            subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared", "-Xcompiler",
                            "-fPIC", "-o", so, src], check=True, capture_output=True)
        lib = ctypes.CDLL(so)
        lib.cub_sort_ms.restype = ctypes.c_int
        lib.cub_sort_ms.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_float)]
        return lib
    except Exception:  # noqa: BLE001 - a missing toolkit only drops the comparison
        return None


CUB_SWEEP_LOG2 = (20, 24, 26, 28)


def run_sweep(torch, bvh, _lib, L, dev, stream, peak, reps=7):
    """Throughput of the sort sweep workload at every stated size and key
    kind, and of the LBVH build at larger sizes.  Each timed sample restores
    the unsorted keys and flushes L2 outside the event pair, so the events
    bracket the sort alone."""
    from bajo_b200 import sort
    out = {k: {} for k in SWEEP_KINDS}
    out["build"] = {}
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    cub = cub_baseline_lib()

    def timeit(prepare, fn):
        prepare()
        fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            prepare()
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.median(ms), min(ms)

    for lg in SWEEP_LOG2:
        n = 1 << lg
        for kind, (bytes_per_key, pairs) in SWEEP_KINDS.items():
            src_k, b, e = sweep_keys(torch, kind, n, seed=lg, dev=dev)
            keys = torch.empty_like(src_k)
            vals = torch.empty(n, dtype=torch.int32, device=dev) if pairs else None
            src_v = torch.arange(n, dtype=torch.int32, device=dev) if pairs else None
            ws = sort.RadixSortWorkspace(n, src_k.element_size(), pairs, b, e, device=dev)

            def prepare():
                keys.copy_(src_k)
                if pairs:
                    vals.copy_(src_v)

            if pairs:
                fn = lambda: sort.onesweep_radix_sort_pairs(keys, vals, workspace=ws, begin_bit=b, end_bit=e)  # noqa
            else:
                fn = lambda: sort.onesweep_radix_sort_keys(keys, workspace=ws, begin_bit=b, end_bit=e)  # noqa
            med, best = timeit(prepare, fn)
            uk = (keys.to(torch.int64) & 0xFFFFFFFF) if keys.dtype == torch.int32 else keys
            ok = bool((uk[1:] >= uk[:-1]).all())
            del uk
            if ws.status() != 0 or not ok:
                raise RuntimeError(f"sweep {kind} 2^{lg}: status {ws.status()}, sorted {ok}")
            point = {"gkeys_s": round(n / med / 1e6, 3), "ms": round(med, 5),
                     "hbm_frac": round(bytes_per_key * n / (med / 1e3) / 1e9 / peak, 4),
                     "best_gkeys_s": round(n / best / 1e6, 3)}
            if cub is not None and lg in CUB_SWEEP_LOG2:
                del ws
                ws = None
                torch.cuda.synchronize()
                cms = ctypes.c_float(0.0)
                if cub.cub_sort_ms(src_k.element_size(), src_k.data_ptr(), src_v.data_ptr() if pairs else None, n, e,
                                   reps, flush.data_ptr(), flush.numel(), ctypes.byref(cms)) == 0:
                    point["cub_gkeys_s"] = round(n / cms.value / 1e6, 3)
                    point["vs_cub"] = round(cms.value / med, 3)
            out[kind][f"2^{lg}"] = point
            del src_k, keys, vals, src_v, ws
    for lg in (20, 22, 24):
        n = 1 << lg
        g = torch.Generator(device=dev).manual_seed(0)
        c = torch.rand((n, 1, 3), generator=g, device=dev)
        off = (torch.rand((n, 3, 3), generator=g, device=dev) * 2 - 1) * 0.004
        v = (c + off).reshape(-1).contiguous()
        ws = bvh.GpuBvhBuildWorkspace(n, 1, device=dev)
        tree = bvh.build_triangle_bvh(v, workspace=ws)
        med, _ = timeit(lambda: None, lambda: bvh.build_triangle_bvh(v, workspace=ws, out=tree))
        # bytes per triangle: bounds 36+24, Morton 24+12, 4 passes x 24, topology ~24, refit 36+48+48
        out["build"][f"2^{lg}"] = {"mtri_s": round(n / med / 1e3, 1), "ms": round(med, 4),
                                   "hbm_frac": round(348 * n / (med / 1e3) / 1e9 / peak, 3)}
        del c, off, v, ws, tree
    out["bytes_per_key"] = {k: v[0] for k, v in SWEEP_KINDS.items()}
    out["timing"] = f"median of {reps} event-timed sorts; unsorted keys restored and L2 flushed before each"
    out["cub"] = ("cub::DeviceRadixSort of CUDA 12.9 (SortKeys / SortPairs, the same keys, bit range and L2 "
                  "flush, median of the same count), at 2^" + ", 2^".join(map(str, CUB_SWEEP_LOG2)) +
                  "; vs_cub = CUB time / this sort's time" if cub is not None else "nvcc unavailable: no CUB leg")
    return out


def cpu_sort_baseline(torch, dev, seconds=2.0):
    """The oracle's multithreaded stable LSD radix sort (the reference CPU
    builder's parallel pass) on every host thread: 2^22 keys of each sweep
    kind, repeated for about `seconds` each."""
    import numpy as np
    from oracle import oracle as O
    n = 1 << CPU_SORT_LOG2
    out = {}
    for kind, (_, pairs) in SWEEP_KINDS.items():
        k_dev, b, e = sweep_keys(torch, kind, n, seed=CPU_SORT_LOG2, dev=dev)
        src = k_dev.cpu().numpy().view(np.uint32 if k_dev.dtype == torch.int32 else np.uint64).copy()
        del k_dev
        cs = O.CpuSort(n, src.dtype.itemsize, pairs)
        keys = src.copy()
        vals = np.arange(n, dtype=np.uint32) if pairs else None
        times = []
        t_end = time.perf_counter() + seconds
        while time.perf_counter() < t_end or len(times) < 2:
            keys[:] = src
            if pairs:
                vals[:] = np.arange(n, dtype=np.uint32)
            t0 = time.perf_counter()
            cs.sort(keys, vals, b, e)
            times.append(time.perf_counter() - t0)
        t = statistics.median(times)
        out[kind] = {"value": round(n / t / 1e9, 4), "unit": "Gkeys/s", "cores": cs.threads, "kind": "port",
                     "sample": f"{len(times)} sorts of 2^{CPU_SORT_LOG2} keys (bits [{b}, {e})), median"}
    return out


def run_render(steps, warmup, spp=64, graph=True):
    """Path-tracing workload: 64 icospheres (subdivision 5) + box + quad
    light, 1280x720, `spp` samples per pixel, MIS, depth 8, FP32.  Device
    time of the render through render_gpu_triangles (median), and of the same
    render replayed as one CUDA graph through the handle API."""
    import torch
    from bajo_b200 import rt, scenes
    stream = torch.cuda.current_stream()
    sc = scenes.spheres_in_box()
    gsc = rt.GpuRtTriangleScene(sc)
    settings = rt.RenderSettings(1280, 720, spp, rng_seed=2026, max_depth=8)
    ws = rt.RenderWorkspace(settings, rt.MIS)
    for _ in range(max(1, warmup)):
        rt.render_gpu_triangles(settings, sc.camera, gsc, rt.MIS, workspace=ws)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        rt.render_gpu_triangles(settings, sc.camera, gsc, rt.MIS, workspace=ws)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    t = statistics.median(ms)
    rays, shadows = ws.ray_counts()
    paths = 1280 * 720 * spp
    out = {"workload": "64 icospheres (subdivision 5) + box + 0.25x0.25 light (emission 15), 1280x720, "
                       f"{spp} spp, MIS, depth 8", "bvh_policy": rt.DEFAULT_BVH_POLICY, "triangles": sc.n_tris,
           "ms": round(t, 3),
           "samples_s": round(paths / t * 1e3, 1), "mrays_s": round((rays + shadows) / t / 1e3, 2),
           "rays": rays, "shadow_rays": shadows, "status": ws.status()}
    if graph:
        renderer = rt.Renderer(settings, rt.MIS)
        side = torch.cuda.Stream()
        cam = torch.from_numpy(sc.camera.astype("float32")).cuda()
        px = torch.empty((720, 1280, 3), dtype=torch.float32, device="cuda")
        ms_graph = []
        with torch.cuda.stream(side):
            for _ in range(max(1, warmup)):
                renderer.enqueue(gsc, cam, px, stream=side)
            side.synchronize()
            for _ in range(steps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(side)
                renderer.enqueue(gsc, cam, px, stream=side)
                b.record(side)
                b.synchronize()
                ms_graph.append(a.elapsed_time(b))
        renderer.close()
        out["graph_ms"] = round(statistics.median(ms_graph), 3)
    # the same render under each acceleration-structure policy (the
    # reference's GPU_RT_BVH_* choices, bajo/rt/gpu/prepared_scene.mojo:29-33)
    by_policy = {}
    for policy in rt.BVH_POLICIES:
        g = gsc if policy == rt.DEFAULT_BVH_POLICY else rt.GpuRtTriangleScene(sc, bvh_policy=policy)
        rt.render_gpu_triangles(settings, sc.camera, g, rt.MIS, workspace=ws)
        pm = []
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            rt.render_gpu_triangles(settings, sc.camera, g, rt.MIS, workspace=ws)
            b.record(stream)
            b.synchronize()
            pm.append(a.elapsed_time(b))
        r2, s2 = ws.ray_counts()
        tp = statistics.median(pm)
        by_policy[policy] = {"ms": round(tp, 3), "samples_s": round(paths / tp * 1e3, 1),
                             "mrays_s": round((r2 + s2) / tp / 1e3, 2), "status": ws.status()}
        del g
    out["bvh_policies"] = by_policy
    out["_scene"] = sc
    return out


def cpu_render_sample(sc, seconds=10.0):
    """The oracle's restatement of the reference CPU path tracer (MIS, depth
    8) on every host thread over the path-tracing scene: 1280x720 at 1 sample
    per pixel, repeated for about `seconds`."""
    from oracle import oracle as O
    bvh = O.lbvh_build(sc.vertices)
    lights = O.rt_build_lights(sc)
    threads = O.n_threads()
    t_end = time.perf_counter() + seconds
    times = []
    while time.perf_counter() < t_end or not times:
        t0 = time.perf_counter()
        O.render(sc, sc.camera, 1280, 720, 1, max_depth=8, seed=2026 + len(times), algorithm=4, lights=lights,
                 bvh=bvh, threads=threads)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": round(1280 * 720 / t / 1e6, 3), "unit": "Msamples/s", "cores": threads, "kind": "port",
            "sample": f"{len(times)} renders of 1280x720 at 1 spp (MIS, depth 8), median"}


def cpu_batched_sample(verts, so, n_scenes=32, width=256, height=256):
    """CPU build + trace of the first `n_scenes` scenes of the batched
    workload: the restated reference CPU builder per scene and the oracle's
    primary + cosine-bounce trace of its 256x256 rays, on every host thread."""
    from oracle import oracle as O
    import numpy as np
    cam = workload_camera()
    tris = rays = 0
    t_build = t_trace = 0.0
    for s in range(n_scenes):
        sub = verts[9 * int(so[s]): 9 * int(so[s + 1])]
        cb = O.CpuLbvh(sub)
        t0 = time.perf_counter()
        cb.build()
        t_build += time.perf_counter() - t0
        o = O.lbvh_build(sub)
        t0 = time.perf_counter()
        _, p0, _, _ = O.trace_batch(o, cam, 0, width, height, seed=7, view_base=s)
        t_trace += time.perf_counter() - t0
        tris += int(so[s + 1] - so[s])
        rays += width * height + int(np.count_nonzero(p0 != O.EMPTY))
    t = t_build + t_trace
    return {"value": round(tris / t / 1e6, 3), "unit": "Mtri/s (build + trace)", "mrays_s": round(rays / t / 1e6, 3),
            "cores": O.n_threads(), "kind": "port",
            "sample": f"first {n_scenes} scenes ({tris} triangles, {rays} rays): CPU LBVH build + 256x256 primary "
                      "and bounce rays each"}


def run_batched(steps, warmup, n_scenes=4096):
    """Batched workload: 4,096 scenes (log-uniform 256..65,536 triangles),
    256x256 primary + one cosine bounce per pixel, build + trace replayed as
    one CUDA graph."""
    import torch
    from bajo_b200 import batch, camera, scenes
    verts, so = scenes.batched_scenes(n_scenes=n_scenes)
    v = torch.from_numpy(verts).cuda()
    g = batch.BatchedGraph(v, so, camera.plain_lbvh_camera(), 256, 256, seed=7)
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        g.replay()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        g.replay()
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    t = statistics.median(ms)
    p0 = g.result.p0
    bounce = int((p0 != -1).sum().item())
    rays = n_scenes * 256 * 256 + bounce
    return {"workload": f"{n_scenes} scenes, 256..65,536 triangles (log-uniform), 256x256 primary + one "
                        "cosine bounce per pixel, one CUDA-graph launch", "scenes": n_scenes,
            "triangles": int(so[-1]), "ms": round(t, 3),
            "build_trace_mtri_s": round(int(so[-1]) / t / 1e3, 1), "mrays_s": round(rays / t / 1e3, 1),
            "rays": rays, "status": g.status(), "_verts": verts, "_so": so}


def run_extras(args, local):
    """The other stated workloads, one GPU, each with its clock record and a
    CPU baseline: `render` (path tracing), `batched` (4,096 scenes) and
    `guided` (learned guiding vs plain MIS at equal time)."""
    out = {}
    with ClockSampler(local) as ck:
        r = run_render(3, 1, 64)
    sc = r.pop("_scene")
    r["clocks"] = ck.summary()
    if not args.no_cpu_baseline:
        r["cpu_baseline"] = cpu_render_sample(sc)
    out["render"] = r
    with ClockSampler(local) as ck:
        r = run_batched(5, 2)
    verts, so = r.pop("_verts"), r.pop("_so")
    r["clocks"] = ck.summary()
    if not args.no_cpu_baseline:
        r["cpu_baseline"] = cpu_batched_sample(verts, so)
    del verts, so
    out["batched"] = r
    gargs = parse_args([])
    with ClockSampler(local) as ck:
        r = run_guided(gargs)
    r["clocks"] = ck.summary()
    out["guided"] = r
    # the same comparison on the box lit only indirectly (its light faces the
    # ceiling), where the error is in the indirect light the guide learns
    gargs = parse_args(["--scene", "indirect"])
    with ClockSampler(local) as ck:
        r = run_guided(gargs)
    r["clocks"] = ck.summary()
    out["guided_indirect"] = r
    # and on the path-tracing workload's geometry with its light turned to
    # face the ceiling: 1.31M triangles, so a guided sample costs little
    # more than a plain one, and all light is indirect
    gargs = parse_args(["--scene", "spheres_up"])
    with ClockSampler(local) as ck:
        r = run_guided(gargs)
    r["clocks"] = ck.summary()
    out["guided_spheres_up"] = r
    return out


def guided_scene(name):
    from bajo_b200 import scenes
    if name == "indirect":
        return scenes.indirect_box_scene()
    if name == "door":
        return scenes.door_scene()
    return scenes.spheres_in_box(light_up=name == "spheres_up")


def run_guided(args):
    """Learned guiding against plain MIS at equal wall time.

    Scene: the path-tracing workload (64 icospheres in the lit box; or
    ``--scene indirect``, the box lit only by a panel facing the ceiling),
    1280x720, depth 8.  Error = MSE against a ``--ref-spp`` plain MIS render
    accumulated in FP64.  Plain: one 64-spp MIS render, device-timed.
    Guided: progressive passes of ``--spp-per-pass`` with the network trained
    after each of the first ``--train-passes`` passes (training time counted),
    then passes of ``--late-spp`` (larger passes keep the GPU busier in the
    later bounces); the first pass samples the BSDF only (``--first-guided``
    guides it too), since an untrained network only adds variance;
    after each pass the cumulative device time and the MSE (computed outside
    the timed region) are logged until the guided image is at least as good
    as the plain one or twice the plain time has passed.  The time to the
    plain MSE is the end of the first pass at or below it; the key
    ``guided_ms_to_plain_mse_interp`` also gives the crossing interpolated
    between that pass and the one before, with the error taken as
    proportional to 1 / time between them."""
    import torch
    from bajo_b200 import guide, rt, scenes
    stream = torch.cuda.current_stream()
    w, h = args.width, args.height
    sc = guided_scene(args.scene)
    gsc = rt.GpuRtTriangleScene(sc)

    def ev_time(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b), r

    chunk = 64
    st = rt.RenderSettings(w, h, chunk, max_depth=8)
    ws = rt.RenderWorkspace(st, rt.MIS)
    ref64 = torch.zeros((h, w, 3), dtype=torch.float64, device="cuda")
    t_ref = 0.0
    for k in range(args.ref_spp // chunk):
        st.rng_seed = 900001 + k
        t, _ = ev_time(lambda: rt.render_gpu_triangles(st, sc.camera, gsc, rt.MIS, workspace=ws, pixels64=ref64))
        t_ref += t
    ref = ref64 / (args.ref_spp // chunk * chunk)
    # plain MIS, 64 spp (first call warms up)
    st_plain = rt.RenderSettings(w, h, 64, rng_seed=2026, max_depth=8)
    rt.render_gpu_triangles(st_plain, sc.camera, gsc, rt.MIS, workspace=ws)
    t_plain, img = ev_time(lambda: rt.render_gpu_triangles(st_plain, sc.camera, gsc, rt.MIS, workspace=ws))
    mse_plain = float(((img.double() - ref) ** 2).mean())
    # guided, progressive
    gr = guide.GuidedRenderer(gsc, sc.camera, w, h, spp_per_pass=args.spp_per_pass, record_capacity=args.records,
                              batch=1 << 14, steps=args.train_steps, lr=1e-2)
    gr.render_pass(1, train=False)  # warm-up: kernel attributes, tuning table
    gr.prepare_pass(args.late_spp)  # the later passes' workspace, allocated before the clock starts
    torch.cuda.synchronize()
    gr.reset_image()
    gr.net = guide.GuideNetwork("cuda", seed=0)
    log, t_g, reached = [], 0.0, None
    k = 0
    while t_g < 2.0 * t_plain and k < 4096:
        train = k < args.train_passes
        frac = 0.0 if (k == 0 and not args.first_guided) else None  # the untrained network guides nothing
        spp_k = args.spp_per_pass if train else args.late_spp
        t, _ = ev_time(lambda: gr.render_pass(70001 + 7919 * k, train=train, guide_fraction=frac, spp=spp_k))
        t_g += t
        k += 1
        mse = float(((gr.image() - ref) ** 2).mean())
        log.append((round(t_g, 2), gr.samples, mse))
        if reached is None and mse <= mse_plain:
            reached = t_g
            break
    # crossing interpolated between the last pass above the plain MSE and the
    # first at or below it, with MSE ~ 1 / time between the two
    interp = None
    if reached is not None and len(log) >= 2:
        (t0, _, m0), (t1, _, m1) = log[-2], log[-1]
        if m0 > mse_plain >= m1 > 0.0 and t1 > t0:
            interp = t0 + (t1 - t0) * (1.0 / mse_plain - 1.0 / m0) / (1.0 / m1 - 1.0 / m0)
    # MSE at equal time: last logged point not past t_plain
    eq = [m for (t, _, m) in log if t <= t_plain]
    # guided throughput with a trained network and no training
    t_pass, _ = ev_time(lambda: gr.render_pass(5, train=False, spp=args.late_spp))
    samples = w * h * args.late_spp
    rays, shadows = gr.workspace.ray_counts()
    out = {"case": "guided", "scene": args.scene, "width": w, "height": h, "ref_spp": args.ref_spp,
           "ref_ms": round(t_ref, 1), "plain_ms": round(t_plain, 2), "plain_mse": mse_plain,
           "guided_ms_to_plain_mse": None if reached is None else round(reached, 2),
           "time_ratio": None if reached is None else round(reached / t_plain, 3),
           "guided_ms_to_plain_mse_interp": None if interp is None else round(interp, 2),
           "time_ratio_interp": None if interp is None else round(interp / t_plain, 3),
           "guided_mse_at_plain_time": eq[-1] if eq else None,
           "guided_spp_at_plain_time": max([s for (t, s, _) in log if t <= t_plain], default=0),
           "guided_samples_s": round(samples / t_pass * 1e3, 1),
           "plain_samples_s": round(w * h * 64 / t_plain * 1e3, 1),
           "guided_mrays_s": round((rays + shadows) / t_pass / 1e3, 1),
           "train_passes": args.train_passes, "spp_per_pass": args.spp_per_pass, "late_spp": args.late_spp,
           "train_steps": args.train_steps,
           "records_per_pass": args.records,
           "first_pass_guided": bool(args.first_guided),
           "log": log[:: max(1, len(log) // 40)], "status": gr.workspace.status()}
    return out


def run_guided_pass(args):
    """Throughput of guided passes with a network trained for
    --train-passes passes first (no training in the timed passes), next to
    plain MIS passes of the same size."""
    import torch
    from bajo_b200 import guide, rt, scenes
    stream = torch.cuda.current_stream()
    w, h, spp = args.width, args.height, args.spp_per_pass
    sc = guided_scene(args.scene)
    gsc = rt.GpuRtTriangleScene(sc)
    gr = guide.GuidedRenderer(gsc, sc.camera, w, h, spp_per_pass=spp, record_capacity=args.records, batch=1 << 14,
                              steps=args.train_steps)
    for k in range(args.train_passes):
        gr.render_pass(11 + k, train=True)
    st = rt.RenderSettings(w, h, spp, max_depth=8)
    ws = rt.RenderWorkspace(st, rt.MIS)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.median(ms)

    t_g = timed(lambda: gr.render_pass(5, train=False))
    g_rays = sum(gr.workspace.ray_counts())
    t_p = timed(lambda: rt.render_gpu_triangles(st, sc.camera, gsc, rt.MIS, workspace=ws))
    p_rays = sum(ws.ray_counts())
    n = w * h * spp
    return {"case": "guided_pass", "scene": args.scene, "width": w, "height": h, "spp": spp,
            "guided_ms": round(t_g, 3), "guided_samples_s": round(n / t_g * 1e3, 1),
            "guided_mrays_s": round(g_rays / t_g / 1e3, 1), "plain_ms": round(t_p, 3),
            "plain_samples_s": round(n / t_p * 1e3, 1), "plain_mrays_s": round(p_rays / t_p / 1e3, 1),
            "status": gr.workspace.status() | ws.status()}


def run_case(args):
    """One piece of the path alone, for ncu captures and tuning runs."""
    import torch
    from bajo_b200 import build as B
    B.build()
    from bajo_b200 import autotune, bvh, camera, sort
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    n = args.n
    out = {"case": args.case, "n": n}

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.median(ms)

    if args.case == "render":
        r = run_render(args.steps, args.warmup, args.spp)
        r.pop("_scene")
        out.update(r)
    elif args.case == "batched":
        r = run_batched(args.steps, args.warmup, args.scenes)
        r.pop("_verts"), r.pop("_so")
        out.update(r)
    elif args.case == "guided":
        out = run_guided(args)
    elif args.case == "guided_pass":
        out = run_guided_pass(args)
    elif args.case == "mlp_forward":
        # the guiding network's batched forward: mma.sync kernel and tcgen05 kernel
        from bajo_b200 import guide
        g = torch.Generator(device="cuda").manual_seed(0)
        pos = torch.rand((n, 3), generator=g, device="cuda")
        nrm = torch.nn.functional.normalize(torch.randn((n, 3), generator=g, device="cuda"), dim=1)
        box = torch.tensor([0, 0, 0, 1, 1, 1], dtype=torch.float32, device="cuda")
        net = guide.GuideNetwork("cuda", seed=0)
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        ms_mma = timed(lambda: net.forward(pos, nrm, box))
        ms_tc = timed(lambda: net.forward(pos, nrm, box, tensor_memory=True, status=status))
        flops = 2.0 * n * (3 * 64 * 64 + 32 * 64)  # the dense layers (output padded to 32)
        out.update({"ms_mma_sync": round(ms_mma, 5), "ms_tcgen05": round(ms_tc, 5),
                    "rows_s_mma_sync": round(n / ms_mma * 1e3, 1), "rows_s_tcgen05": round(n / ms_tc * 1e3, 1),
                    "tflops_tcgen05": round(flops / ms_tc / 1e9, 2), "status": int(status.item())})
    elif args.case == "mlp_train":
        # one training step of the guiding network on n records: gradient
        # (mma.sync kernel and tcgen05 kernel) and Adam
        from bajo_b200 import guide
        g = torch.Generator(device="cuda").manual_seed(0)
        pos = torch.rand((n, 3), generator=g, device="cuda")
        nrm = torch.nn.functional.normalize(torch.randn((n, 3), generator=g, device="cuda"), dim=1)
        dirs = torch.nn.functional.normalize(torch.randn((n, 3), generator=g, device="cuda"), dim=1)
        wts = torch.rand(n, generator=g, device="cuda")
        box = torch.tensor([0, 0, 0, 1, 1, 1], dtype=torch.float32, device="cuda")
        net = guide.GuideNetwork("cuda", seed=0)
        ms_mma = timed(lambda: net.gradient(pos, nrm, dirs, wts, box, tensor_memory=False))
        ms_tc = timed(lambda: net.gradient(pos, nrm, dirs, wts, box, tensor_memory=True))
        ms_adam = timed(lambda: net.adam(lr=0.0, grad_scale=0.0))
        # tensor-core work issued per row: forward (K = 80 with the bias
        # column), input gradients of layers 3..1, weight gradients (M = 64,
        # N = 80) of all four layers
        flops = 2.0 * n * ((3 * 64 * 80 + 32 * 80) + (2 * 64 * 64 + 64 * 32) + 4 * 64 * 80)
        out.update({"ms_grad_mma_sync": round(ms_mma, 5), "ms_grad_tcgen05": round(ms_tc, 5),
                    "ms_adam": round(ms_adam, 5), "rows_s_tcgen05": round(n / ms_tc * 1e3, 1),
                    "tflops_tcgen05": round(flops / ms_tc / 1e9, 2), "status": int(net.status.item())})
    elif args.case == "tune":
        out["results"] = autotune.tune_all(reps=args.steps, save_cache=False)
        out["device"] = autotune.device_key()
    elif args.case == "sort":
        kb = args.bits // 8
        g = torch.Generator(device="cuda").manual_seed(0)
        dt = torch.int32 if kb == 4 else torch.int64
        keys = torch.randint(-2**31, 2**31, (n,), dtype=dt, device="cuda", generator=g)
        vals = None if args.keys_only else torch.arange(n, dtype=torch.int32, device="cuda")
        end_bit = args.end_bit or args.bits
        ws = sort.RadixSortWorkspace(n, kb, vals is not None, 0, end_bit)
        if vals is None:
            ms = timed(lambda: sort.onesweep_radix_sort_keys(keys, workspace=ws, end_bit=end_bit))
        else:
            ms = timed(lambda: sort.onesweep_radix_sort_pairs(keys, vals, workspace=ws, end_bit=end_bit))
        v = ctypes.c_int32(0)
        from bajo_b200 import _lib
        _lib.load().bajo_sort_tuning_get(kb, int(vals is not None), n, ctypes.byref(v))
        out.update({"bits": args.bits, "end_bit": end_bit, "pairs": vals is not None, "ms": round(ms, 5),
                    "gkeys_s": round(n / ms / 1e6, 3), "variant": v.value, "status": ws.status()})
    elif args.case == "wide":
        from bajo_b200 import scenes, wide
        verts = torch.from_numpy(scenes.random_triangles(n, seed=0, spread=0.01 if n <= 65536 else 0.004)).cuda()
        tree = bvh.build_triangle_bvh(verts)
        w = wide.build_wide_bvh(tree, args.node_width, args.max_leaf)
        ms_build = timed(lambda: w.build(read_counts=False))
        cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
        hits = torch.empty(8 * WIDTH * HEIGHT, dtype=torch.float32, device="cuda")
        ms_wide = timed(lambda: w.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT))
        ms_bin = timed(lambda: tree.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT))
        stats = torch.zeros(5 * WIDTH * HEIGHT, dtype=torch.int32, device="cuda")
        w.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT, d_stats=stats)
        s = stats.view(-1, 5).double().mean(0)[[0, 3]].tolist()
        out.update({"node_width": args.node_width, "max_leaf": args.max_leaf, "wide_nodes": w.n_nodes, "leaf_blocks": w.n_leaf_blocks,
                    "collapse_ms": round(ms_build, 5), "collapse_mtri_s": round(n / ms_build / 1e3, 2),
                    "wide_trace_ms": round(ms_wide, 4), "wide_mrays_s": round(WIDTH * HEIGHT / ms_wide / 1e3, 2),
                    "binary_trace_ms": round(ms_bin, 4),
                    "binary_mrays_s": round(WIDTH * HEIGHT / ms_bin / 1e3, 2),
                    "wide_nodes_per_ray": round(s[0], 3), "tris_per_ray": round(s[1], 3), "status": w.status()})
    elif args.case == "cwbvh8":
        from bajo_b200 import scenes, wide
        verts = torch.from_numpy(scenes.random_triangles(n, seed=0, spread=0.01 if n <= 65536 else 0.004)).cuda()
        tree = bvh.build_triangle_bvh(verts, method=args.method)
        cw = wide.build_cwbvh8(tree)
        ms_build = timed(lambda: cw.build(read_count=False))
        cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
        hits = torch.empty(8 * WIDTH * HEIGHT, dtype=torch.float32, device="cuda")
        ms_cw = timed(lambda: cw.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT))
        ms_any = timed(lambda: cw.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT, any_hit=True))
        ms_bin = timed(lambda: tree.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT, tri_mode=0))
        nr = WIDTH * HEIGHT
        g = torch.Generator(device="cuda").manual_seed(1)
        rays = torch.empty(8, nr, dtype=torch.float32, device="cuda")
        rays[0:3].uniform_(0.0, 1.0, generator=g)
        rays[3].zero_()
        d = torch.randn(3, nr, device="cuda", generator=g)
        rays[4:7] = d / d.norm(dim=0, keepdim=True)
        rays[7].fill_(3.0e38)
        rays = rays.reshape(-1)
        ms_inc = timed(lambda: cw.launch_rays(rays, hits, nr))
        ms_inc_bin = timed(lambda: tree.launch_rays(rays, hits, nr, tri_mode=0))
        out.update({"method": args.method, "incoherent_mrays_s": round(nr / ms_inc / 1e3, 2),
                    "binary_mt_incoherent_mrays_s": round(nr / ms_inc_bin / 1e3, 2)})
        out.update({"cwbvh8_nodes": cw.n_nodes, "build_ms": round(ms_build, 5),
                    "build_mtri_s": round(n / ms_build / 1e3, 2),
                    "closest_ms": round(ms_cw, 4), "closest_mrays_s": round(WIDTH * HEIGHT / ms_cw / 1e3, 2),
                    "any_ms": round(ms_any, 4), "any_mrays_s": round(WIDTH * HEIGHT / ms_any / 1e3, 2),
                    "binary_mt_ms": round(ms_bin, 4), "binary_mt_mrays_s": round(WIDTH * HEIGHT / ms_bin / 1e3, 2),
                    "status": cw.status()})
    elif args.case == "hploc":
        # H-PLOC against LBVH on the same triangles: build time, then closest
        # hits of the camera and of incoherent rays through each tree
        from bajo_b200 import scenes
        verts = torch.from_numpy(scenes.random_triangles(n, seed=0, spread=0.01 if n <= 65536 else 0.004)).cuda()
        cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
        hits = torch.empty(8 * WIDTH * HEIGHT, dtype=torch.float32, device="cuda")
        nr = WIDTH * HEIGHT
        g = torch.Generator(device="cuda").manual_seed(1)
        rays = torch.empty(8, nr, dtype=torch.float32, device="cuda")
        rays[0:3].uniform_(0.0, 1.0, generator=g)
        rays[3].zero_()
        d = torch.randn(3, nr, device="cuda", generator=g)
        rays[4:7] = d / d.norm(dim=0, keepdim=True)
        rays[7].fill_(3.0e38)
        rays = rays.reshape(-1)
        for method in ("lbvh", "hploc"):
            ws = bvh.GpuBvhBuildWorkspace(n, 1, method=method)
            tree = bvh.build_triangle_bvh(verts, workspace=ws, method=method)
            ms_b = timed(lambda: bvh.build_triangle_bvh(verts, workspace=ws, out=tree, method=method))
            ms_c = timed(lambda: tree.launch_camera(cam, hits, nr, WIDTH, HEIGHT))
            ms_i = timed(lambda: tree.launch_rays(rays, hits, nr))
            out.update({f"{method}_build_ms": round(ms_b, 5), f"{method}_build_mtri_s": round(n / ms_b / 1e3, 2),
                        f"{method}_camera_mrays_s": round(nr / ms_c / 1e3, 2),
                        f"{method}_incoherent_mrays_s": round(nr / ms_i / 1e3, 2),
                        f"{method}_status": ws.status()})
    elif args.case == "tlas":
        # 8 BLASes of n / 8 triangles each, 512 randomly rotated, scaled and
        # placed instances (the shape of the reference's TLAS stress test,
        # test/bvh/gpu/test_blas_tlas.mojo:320); camera and incoherent rays
        import numpy as np
        from bajo_b200 import scenes, tlas
        rng = np.random.default_rng(0)
        per = max(n // 8, 1)
        verts = torch.from_numpy(np.concatenate(
            [scenes.random_triangles(per, seed=b, spread=0.02).reshape(-1) for b in range(8)])).cuda()
        seg = np.arange(9, dtype=np.int64) * per
        xf = []
        for _ in range(512):
            q = rng.normal(size=4)
            q /= np.linalg.norm(q)
            w, x, y, z = q
            rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                            [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                            [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
            xf.append(np.concatenate([rot * rng.uniform(0.5, 1.5), rng.uniform(-6, 6, (3, 1))], axis=1).reshape(-1))
        xf = np.array(xf, np.float32)
        bi = rng.integers(0, 8, 512).astype(np.uint32)
        blas_ws = bvh.GpuBvhBuildWorkspace(per * 8, 8)
        blas_set = bvh.build_triangle_bvh(verts, seg, workspace=blas_ws)
        t = tlas.build_triangle_tlas(blas_set, xf, bi)
        ms_blas = timed(lambda: bvh.build_triangle_bvh(verts, seg, workspace=blas_ws, out=blas_set))
        ms_tlas = timed(lambda: t.build())
        cam = torch.from_numpy(camera.camera([0.0, 2.0, -20.0], [0, 0, 0], [0, 1, 0], 0.5)).cuda()
        hits = torch.empty(8 * WIDTH * HEIGHT, dtype=torch.float32, device="cuda")
        nr = WIDTH * HEIGHT
        ms_cam = timed(lambda: t.launch_camera(cam, hits, nr, WIDTH, HEIGHT))
        ms_any = timed(lambda: t.launch_camera(cam, hits, nr, WIDTH, HEIGHT, any_hit=True))
        hit_frac = (hits.view(-1, 8)[:, 3].view(torch.int32) != -1).float().mean().item()
        g = torch.Generator(device="cuda").manual_seed(1)
        rays = torch.empty(8, nr, dtype=torch.float32, device="cuda")
        rays[0:3].uniform_(-6.0, 6.0, generator=g)
        rays[3].zero_()
        d = torch.randn(3, nr, device="cuda", generator=g)
        rays[4:7] = d / d.norm(dim=0, keepdim=True)
        rays[7].fill_(3.0e38)
        rays = rays.reshape(-1)
        ms_inc = timed(lambda: t.launch_rays(rays, hits, nr))
        out.update({"blas": 8, "instances": 512, "triangles_per_blas": per, "blas_build_ms": round(ms_blas, 5),
                    "tlas_build_ms": round(ms_tlas, 5), "camera_mrays_s": round(nr / ms_cam / 1e3, 2),
                    "camera_any_mrays_s": round(nr / ms_any / 1e3, 2), "camera_hit_fraction": round(hit_frac, 3),
                    "incoherent_mrays_s": round(nr / ms_inc / 1e3, 2), "status": int(t.status.item())})
    elif args.case in ("build", "trace"):
        from bajo_b200 import scenes
        verts = torch.from_numpy(scenes.random_triangles(n, seed=0, spread=0.01 if n <= 65536 else 0.004)).cuda()
        ws = bvh.GpuBvhBuildWorkspace(n, 1)
        tree = bvh.build_triangle_bvh(verts, workspace=ws)
        if args.case == "build":
            ms = timed(lambda: bvh.build_triangle_bvh(verts, workspace=ws, out=tree))
            staged = bvh.build_triangle_bvh(verts, stage_top=True)
            ms_stage = timed(lambda: staged.restage_top())
            out.update({"ms": round(ms, 5), "mtri_s": round(n / ms / 1e3, 2), "stage_top_ms": round(ms_stage, 5)})
        else:
            cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
            hits = torch.empty(8 * WIDTH * HEIGHT, dtype=torch.float32, device="cuda")
            ms = timed(lambda: tree.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT))
            staged = bvh.build_triangle_bvh(verts, stage_top=True)  # same tree plus the staged top levels
            ms_staged = timed(lambda: staged.launch_camera(cam, hits, WIDTH * HEIGHT, WIDTH, HEIGHT))
            # incoherent rays: origins uniform in the unit cube, directions uniform on the sphere
            nr = WIDTH * HEIGHT
            g = torch.Generator(device="cuda").manual_seed(1)
            rays = torch.empty(8, nr, dtype=torch.float32, device="cuda")
            rays[0:3].uniform_(0.0, 1.0, generator=g)
            rays[3].zero_()
            d = torch.randn(3, nr, device="cuda", generator=g)
            rays[4:7] = d / d.norm(dim=0, keepdim=True)
            rays[7].fill_(3.0e38)
            rays = rays.reshape(-1)
            ms_inc = timed(lambda: tree.launch_rays(rays, hits, nr))
            ms_inc_staged = timed(lambda: staged.launch_rays(rays, hits, nr))
            out.update({"ms": round(ms, 5), "mrays_s": round(WIDTH * HEIGHT / ms / 1e3, 2),
                        "staged_ms": round(ms_staged, 5),
                        "staged_mrays_s": round(WIDTH * HEIGHT / ms_staged / 1e3, 2),
                        "incoherent_mrays_s": round(nr / ms_inc / 1e3, 2),
                        "incoherent_staged_mrays_s": round(nr / ms_inc_staged / 1e3, 2)})
        out["status"] = ws.status()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.case:
        run_case(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    run_bajo(args)
    from bajo_b200 import dist
    dist.finish(int(os.environ.get("WORLD_SIZE", "1")))


if __name__ == "__main__":
    main()
