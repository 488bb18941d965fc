"""Builds ``bajo_b200/libbajo_b200.so`` (the C-ABI CUDA library) for sm_100a.

The library is compiled in-tree with nvcc directly, so the shared object
travels with the source tree and is the only native code the package loads.

``-fmad=false``: no implicit multiply-add contraction.  The reference's float
formulas are restated with their own rounding (explicit fmaf() only where the
reference spells fma()), which is what makes results bit-identical to the CPU
oracle built with ``-ffp-contract=off``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbajo_b200.so")
SOURCES = ["sort.cu", "sort_static.cu", "lbvh.cu", "trace.cu", "camera.cu", "rt.cu", "render_handle.cu", "mlp.cu",
           "wide.cu", "cwbvh.cu", "hploc.cu", "tlas.cu"]
HEADERS = ["bajo_common.cuh", "onesweep.cuh", "traverse.cuh", "sampling.cuh", "mlp.cuh", "wide.cuh", "cwbvh.cuh"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
         "-I", os.path.join(ROOT, "include")]


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _inputs():
    return _sources() + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "bajo_b200.h"),
                                                                  __file__]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _inputs())


def _stale(obj: str, src: str) -> bool:
    """An object is rebuilt when it is missing or older than its source, any
    shared header, the C-ABI header or this script."""
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src, __file__, os.path.join(ROOT, "include", "bajo_b200.h")] + [os.path.join(CSRC, h) for h in HEADERS]
    return any(os.path.getmtime(p) > t for p in deps)


def build(verbose: bool = False, ptxas_verbose: bool = False, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    objs, jobs = [], []
    for src in _sources():
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or ptxas_verbose or _stale(obj, src):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj + ".tmp"]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append((cmd, obj))

    def compile_one(job):
        cmd, obj = job
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(obj + ".tmp", obj)

    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        list(ex.map(compile_one, jobs))
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv, force=True)
