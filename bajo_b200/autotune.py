"""Project autotuner for the sort tile shapes and digit widths.

The sort kernels are compiled in several tile shapes (threads x keys per
thread) and, for 64-bit keys, two digit widths (8 and 10 bits).  For each (key width, values, size bucket) the tuner times every
shape the library allows on the current GPU with CUDA events and writes the
fastest into the library's tuning table (``bajo_sort_tuning_set``).  Results
are cached as JSON keyed by (kernel, size bucket, GPU name and SM count) so a
process can load them instead of re-measuring.
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


def save(results: dict, path: str = CACHE) -> None:
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    dev = data.setdefault(device_key(), {})
    for kernel, table in results.items():
        dev.setdefault(kernel, {}).update({str(k): v["best"] for k, v in table.items()})
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
        kb = 4 if "_u32_" in kernel else 8
        hv = kernel.endswith("pairs")
        for lg, v in entries.items():
            if L.bajo_sort_tuning_set(kb, int(hv), int(lg), int(v)) == _lib.OK:
                count += 1
    return count


def tune_all(reps: int = 5, save_cache: bool = True) -> dict:
    """The shapes the LBVH build and the sort sweep use."""
    # 64-bit keys: up to 2^18 with the 30 live bits of single-scene LBVH keys
    # (where 10-bit digits compete), above with 44 bits (segmented builds)
    u64 = tune_sort(8, True, range(10, 19), end_bit=30, reps=reps)
    u64.update(tune_sort(8, True, range(19, 27), end_bit=44, reps=reps))
    res = {
        _kernel_key(8, True): u64,
        _kernel_key(4, True): tune_sort(4, True, range(10, 27), reps=reps),
    }
    if save_cache:
        save(res)
    return res
