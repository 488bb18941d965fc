"""Project autotuner: sort tile shapes and digit widths, closest-hit block
sizes, and the size limit of the one-launch build.

- The sort kernels are compiled in several tile shapes (threads x keys per
  thread) and, for 64-bit keys, two digit widths (8 and 10 bits).  For each
  (key width, values, size bucket) the tuner times every shape the library
  allows on the current GPU with CUDA events and writes the fastest into the
  library's table (``bajo_sort_tuning_set``).
- The unstaged closest-hit kernels (camera and general rays) are compiled
  for blocks of 64, 128 and 256 threads and traversal stacks of 64, 24 and
  12 entries (a ray that needs more entries is traced again with 64); the
  tuner times each pair per ray-count bucket on a tree of the plain
  workload's kind, checks that the hits are identical, and installs the
  fastest (``bajo_trace_tuning_set``, ``bajo_trace_stack_tuning_set``).
- The one-launch build is timed against the per-stage kernels at every
  power of two up to its limit, and the largest size up to which it wins is
  installed (``bajo_lbvh_fused_max_set``).
- The wavefront tracer's bounce kernels (closest hit, shading, shadow rays)
  are compiled for blocks of 64, 128 and 256 threads; the tuner renders the
  path-tracing workload's scene (at a reduced resolution) with each block
  size of each kernel, checks that the images are identical, and installs
  the fastest (``bajo_render_tuning_set``).

Results are cached as JSON keyed by (kernel, size bucket, GPU name and SM
count) so a process can load them instead of re-measuring.
"""
from __future__ import annotations

import ctypes
import json
import os
import statistics

import torch

from . import _lib

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_cache.json")


def device_key() -> str:
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|{p.multi_processor_count}"


def _kernel_key(key_bytes: int, has_values: bool) -> str:
    return f"sort_u{8 * key_bytes}_{'pairs' if has_values else 'keys'}"


def _allowed(key_bytes, has_values, log2n, variant) -> bool:
    L = _lib.load()
    ok = L.bajo_sort_tuning_set(key_bytes, int(has_values), log2n, variant) == _lib.OK
    L.bajo_sort_tuning_set(key_bytes, int(has_values), log2n, -1)
    return ok


def time_sort(key_bytes: int, has_values: bool, n: int, end_bit: int | None = None, reps: int = 5) -> float:
    """Median milliseconds of one sort of n random keys with the current table."""
    from . import sort
    g = torch.Generator(device="cuda").manual_seed(n)
    if key_bytes == 4:
        src = torch.randint(-2**31, 2**31, (n,), dtype=torch.int32, device="cuda", generator=g)
    else:
        src = torch.randint(0, 2**62, (n,), dtype=torch.int64, device="cuda", generator=g)
    keys = src.clone()
    vals = torch.arange(n, dtype=torch.int32, device="cuda") if has_values else None
    end_bit = key_bytes * 8 if end_bit is None else end_bit
    ws = sort.RadixSortWorkspace(n, key_bytes, has_values, 0, end_bit)
    stream = torch.cuda.current_stream()
    ms = []
    for r in range(reps + 1):
        keys.copy_(src)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        if has_values:
            sort.onesweep_radix_sort_pairs(keys, vals, workspace=ws, end_bit=end_bit)
        else:
            sort.onesweep_radix_sort_keys(keys, workspace=ws, end_bit=end_bit)
        b.record(stream)
        b.synchronize()
        if r:
            ms.append(a.elapsed_time(b))
    return statistics.median(ms)


def tune_sort(key_bytes: int, has_values: bool, log2ns, end_bit: int | None = None, reps: int = 5) -> dict:
    """Time every allowed tile shape for each size 2^log2n and install the
    fastest in the tuning table.  Returns {log2n: {"best": v, "ms": [...]}}."""
    L = _lib.load()
    out = {}
    for lg in log2ns:
        n = 1 << lg
        times = {}
        for v in range(_lib.SORT_VARIANTS):
            if not _allowed(key_bytes, has_values, lg, v):
                continue
            L.bajo_sort_tuning_set(key_bytes, int(has_values), lg, v)
            times[v] = time_sort(key_bytes, has_values, n, end_bit, reps)
        best = min(times, key=times.get)
        L.bajo_sort_tuning_set(key_bytes, int(has_values), lg, best)
        out[lg] = {"best": best, "ms": {str(k): round(t, 5) for k, t in times.items()}}
    return out


TRACE_BLOCKS = (128, 64, 256)
TRACE_STACKS = (64, 24, 12)
_TRACE_KINDS = {"trace_camera": 0, "trace_rays": 1}


def _events_ms(fn, reps):
    stream = torch.cuda.current_stream()
    fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    return statistics.median(ms)


def tune_trace(kernel: str, log2rays, n_tris: int = 65536, reps: int = 5) -> dict:
    """Time every block size x traversal stack depth of one closest-hit
    kernel ("trace_camera" or "trace_rays") at 2^log2rays rays over n_tris
    random triangles, check that every choice gives the same hits bit for
    bit, and install the fastest pair.  Returns
    {log2rays: {"best": block, "stack": depth, "ms": {"block/depth": ...}}}."""
    from . import bvh, camera, scenes
    L = _lib.load()
    kind = _TRACE_KINDS[kernel]
    tree = bvh.build_triangle_bvh(torch.from_numpy(scenes.random_triangles(n_tris, seed=0)).cuda())
    cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
    out = {}
    for lg in log2rays:
        n = 1 << lg
        w = 1 << ((lg + 1) // 2)
        h = n // w
        hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
        if kind == 1:
            g = torch.Generator(device="cuda").manual_seed(lg)
            rays = torch.empty(8, n, dtype=torch.float32, device="cuda")
            rays[0:3].uniform_(0.0, 1.0, generator=g)
            rays[3].zero_()
            d = torch.randn(3, n, device="cuda", generator=g)
            rays[4:7] = d / d.norm(dim=0, keepdim=True)
            rays[7].fill_(3.0e38)
            rays = rays.reshape(-1)
            fn = lambda: tree.launch_rays(rays, hits, n)  # noqa: E731
        else:
            fn = lambda: tree.launch_camera(cam, hits, n, w, h)  # noqa: E731
        times, ref = {}, None
        for blk in TRACE_BLOCKS:
            for depth in TRACE_STACKS:
                _lib.check(L.bajo_trace_tuning_set(kind, lg, blk), "bajo_trace_tuning_set")
                _lib.check(L.bajo_trace_stack_tuning_set(kind, lg, depth), "bajo_trace_stack_tuning_set")
                times[(blk, depth)] = _events_ms(fn, reps)
                got = hits.clone()
                if ref is None:
                    ref = got
                elif not torch.equal(got.view(torch.int32), ref.view(torch.int32)):
                    raise RuntimeError(f"{kernel}: block {blk}, stack {depth} changed the hits")
        best_blk, best_depth = min(times, key=times.get)
        _lib.check(L.bajo_trace_tuning_set(kind, lg, best_blk), "bajo_trace_tuning_set")
        _lib.check(L.bajo_trace_stack_tuning_set(kind, lg, best_depth), "bajo_trace_stack_tuning_set")
        ms = {f"{b}/{d}": round(t, 5) for (b, d), t in times.items()}
        out[lg] = {"best": best_blk, "stack": best_depth, "ms": ms}
    return out


_RENDER_KINDS = {"render_trace": 0, "render_shade": 1, "render_shadow": 2}
RENDER_BLOCKS = (128, 64, 256)


def tune_render(width: int = 640, height: int = 360, spp: int = 8, reps: int = 5) -> dict:
    """Time every block size of each wavefront bounce kernel on the 64-sphere
    path-tracing scene (MIS, depth 8, the default tree) and install the
    fastest per kernel, the other kernels at their current choice; every
    block size must give the same image bit for bit.  Returns
    {kernel: {0: {"best": block, "ms": {...}}}}."""
    from . import rt, scenes
    L = _lib.load()
    sc = scenes.spheres_in_box()
    gsc = rt.GpuRtTriangleScene(sc)
    settings = rt.RenderSettings(width, height, spp, rng_seed=3, max_depth=8)
    ws = rt.RenderWorkspace(settings, rt.MIS)
    pixels = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
    cam = torch.from_numpy(sc.camera).cuda()
    fn = lambda: rt.render_gpu_triangles(settings, cam, gsc, rt.MIS, workspace=ws, pixels=pixels)  # noqa: E731
    out = {}
    for kernel, kind in _RENDER_KINDS.items():
        times, ref = {}, None
        for blk in RENDER_BLOCKS:
            _lib.check(L.bajo_render_tuning_set(kind, blk), "bajo_render_tuning_set")
            times[blk] = _events_ms(fn, reps)
            got = pixels.clone()
            if ref is None:
                ref = got
            elif not torch.equal(got.view(torch.int32), ref.view(torch.int32)):
                raise RuntimeError(f"{kernel}: block {blk} changed the image")
        best = min(times, key=times.get)
        _lib.check(L.bajo_render_tuning_set(kind, best), "bajo_render_tuning_set")
        out[kernel] = {0: {"best": best, "ms": {str(k): round(t, 4) for k, t in times.items()}}}
    return out


def tune_one_launch(log2tris=range(11, 18), reps: int = 7) -> dict:
    """Build time of one scene through the one-launch build and through the
    per-stage kernels at each size; installs the largest size up to which
    the one-launch build is faster.  Returns {log2n: {"best": limit, "ms": ...}}
    with the same limit in every entry."""
    from . import bvh, scenes
    L = _lib.load()
    out, limit = {}, 0
    for lg in log2tris:
        n = 1 << lg
        v = torch.from_numpy(scenes.random_triangles(n, seed=lg)).cuda()
        ws = bvh.GpuBvhBuildWorkspace(n, 1)
        tree = bvh.build_triangle_bvh(v, workspace=ws)
        t = {}
        for name, lim in (("one_launch", _lib.FUSED_MAX_LEAVES), ("per_stage", 0)):
            _lib.check(L.bajo_lbvh_fused_max_set(lim), "bajo_lbvh_fused_max_set")
            t[name] = _events_ms(lambda: bvh.build_triangle_bvh(v, workspace=ws, out=tree), reps)
        if t["one_launch"] < t["per_stage"] and limit == (n >> 1 if lg > min(log2tris) else 0):
            limit = n
        out[lg] = {"ms": {k: round(x, 5) for k, x in t.items()}}
    _lib.check(L.bajo_lbvh_fused_max_set(limit), "bajo_lbvh_fused_max_set")
    for lg in out:
        out[lg]["best"] = limit
    return out


def save(results: dict, path: str = CACHE) -> None:
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    dev = data.setdefault(device_key(), {})
    for kernel, table in results.items():
        dev.setdefault(kernel, {}).update({str(k): v["best"] for k, v in table.items()})
        stacks = {str(k): v["stack"] for k, v in table.items() if "stack" in v}
        if stacks:
            dev.setdefault(kernel + "_stack", {}).update(stacks)
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def load(path: str = CACHE) -> int:
    """Install cached choices for this GPU; returns how many entries were set."""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        data = json.load(f)
    table = data.get(device_key(), {})
    L = _lib.load()
    count = 0
    for kernel, entries in table.items():
        if kernel in _TRACE_KINDS:
            for lg, v in entries.items():
                count += L.bajo_trace_tuning_set(_TRACE_KINDS[kernel], int(lg), int(v)) == _lib.OK
            continue
        if kernel.endswith("_stack") and kernel[:-len("_stack")] in _TRACE_KINDS:
            for lg, v in entries.items():
                count += L.bajo_trace_stack_tuning_set(_TRACE_KINDS[kernel[:-len("_stack")]], int(lg),
                                                       int(v)) == _lib.OK
            continue
        if kernel in _RENDER_KINDS:
            for v in entries.values():
                count += L.bajo_render_tuning_set(_RENDER_KINDS[kernel], int(v)) == _lib.OK
            continue
        if kernel == "lbvh_one_launch":
            limits = set(entries.values())
            if len(limits) == 1:
                count += L.bajo_lbvh_fused_max_set(int(limits.pop())) == _lib.OK
            continue
        kb = 4 if "_u32_" in kernel else 8
        hv = kernel.endswith("pairs")
        for lg, v in entries.items():
            if L.bajo_sort_tuning_set(kb, int(hv), int(lg), int(v)) == _lib.OK:
                count += 1
    return count


PARTS = ("sort", "trace", "one_launch", "render")


def tune_all(reps: int = 5, save_cache: bool = True, parts=PARTS) -> dict:
    """The sort shapes the LBVH build and the sort sweep use, the closest-hit
    block sizes, the one-launch build's size limit and the wavefront bounce
    kernels' block sizes (``parts`` selects)."""
    res = {}
    if "sort" in parts:
        # 64-bit keys: up to 2^18 with the 30 live bits of single-scene LBVH
        # keys (where 10-bit digits compete), above with 44 bits (segmented)
        u64 = tune_sort(8, True, range(10, 19), end_bit=30, reps=reps)
        u64.update(tune_sort(8, True, range(19, 27), end_bit=44, reps=reps))
        res[_kernel_key(8, True)] = u64
        res[_kernel_key(4, True)] = tune_sort(4, True, range(10, 29), reps=reps)
        res[_kernel_key(4, False)] = tune_sort(4, False, range(10, 29), reps=reps)
    if "trace" in parts:
        res["trace_camera"] = tune_trace("trace_camera", range(16, 23, 2), reps=reps)
        res["trace_rays"] = tune_trace("trace_rays", range(16, 23, 2), reps=reps)
    if "one_launch" in parts:
        res["lbvh_one_launch"] = tune_one_launch(reps=reps)
    if "render" in parts:
        res.update(tune_render(reps=reps))
    if save_cache:
        save(res)
    return res


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="measure the tuned choices on this GPU and cache them")
    ap.add_argument("--parts", default=",".join(PARTS), help="comma-separated subset of " + ",".join(PARTS))
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    out = tune_all(reps=a.reps, parts=tuple(p for p in a.parts.split(",") if p))
    print(json.dumps({k: {str(lg): v["best"] for lg, v in t.items()} for k, t in out.items()}))
