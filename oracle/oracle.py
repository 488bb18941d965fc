"""ctypes wrapper around the C oracle (``oracle/libbajo_oracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is a CPU restatement of the reference's
LBVH build and closest-hit path (jgsimard/bajo, Mojo); see ``bajo_oracle.h``
for the per-function reference citations.  Only ``tests/``, the smoke check in
``__graft_entry__.py`` and the CPU-baseline leg of ``bench.py`` may import this
module.  The product library never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libbajo_oracle.so")

TRI_MT = 0
TRI_WATERTIGHT = 1
SENTINEL = 0xFFFFFFFF
LEAF_FLAG = 0x80000000
EMPTY = 0xFFFFFFFF


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_I = ctypes.c_int
_F = ctypes.c_float


class _BoLbvh(ctypes.Structure):
    _fields_ = [
        ("n_leaves", _U32), ("n_internal", _U32), ("n_segments", _U32),
        ("leaf_bounds", _P), ("seg_bounds", _P), ("sort_keys", _P), ("leaf_ids", _P),
        ("morton_codes", _P), ("node_meta", _P), ("node_bounds", _P),
        ("node_leaf_counts", _P), ("node_flags", _P), ("leaf_parent", _P), ("roots", _P),
        ("internal_offsets", _P), ("seg_offsets", _P),
    ]


def _declare(L: ctypes.CDLL) -> None:
    sig = {
        "bo_triangle_bounds": (None, [_P, _U32, _P]),
        "bo_segment_bounds": (None, [_P, _P, _U32, _P]),
        "bo_expand_bits_3d": (_U32, [_U32]),
        "bo_morton3": (_U32, [_F, _F, _F]),
        "bo_morton_common_prefix": (_I, [_U32, _U32, _U32, _U32]),
        "bo_morton_keys": (None, [_P, _P, _U32, _P, _U32, _P, _P]),
        "bo_sort_pairs_u64": (None, [_P, _P, _U32, _I, _I]),
        "bo_sort_pairs_u32": (None, [_P, _P, _U32, _I, _I]),
        "bo_sort_keys_u32": (None, [_P, _U32, _I, _I]),
        "bo_cpu_sort_scratch_bytes": (ctypes.c_size_t, [_U32, _U32, _I, _U32]),
        "bo_cpu_sort": (None, [_P, _P, _U32, _U32, _I, _I, _U32, _P]),
        "bo_morton63": (None, [_P, _U32, _P]),
        "bo_sort_keys_u64": (None, [_P, _U32, _I, _I]),
        "bo_internal_offsets": (None, [_P, _U32, _P]),
        "bo_lbvh_topology": (None, [_P, _P, _P, _U32, _P, _P, _P, _P, _P]),
        "bo_lbvh_topology_topdown": (None, [_P, _P, _P, _U32, _P, _P, _P, _P]),
        "bo_lbvh_refit": (None, [_P, _P, _P, _P, _U32, _U32, _P, _P]),
        "bo_lbvh_build": (None, [_P, _P, _U32, ctypes.POINTER(_BoLbvh)]),
        "bo_camera_from_vfov": (None, [_P, _P, _P, _F, _P]),
        "bo_camera_make": (None, [_P, _P, _P, _F, _P]),
        "bo_camera_rays": (None, [_P, _U32, _U32, _U32, _P]),
        "bo_trace_bvh2": (None, [ctypes.POINTER(_BoLbvh), _P, _P, _U32, _I, _P, _U32]),
        "bo_trace_brute": (None, [_P, _U32, _P, _U32, _I, _P, _U32]),
        "bo_trace_bvh2_stats": (None, [ctypes.POINTER(_BoLbvh), _P, _P, _U32, _I, _P]),
        "bo_cpu_build_lbvh": (_U32, [_P, _U32, _U32, _P, _P]),
        "bo_cpu_lbvh_scratch_bytes": (ctypes.c_size_t, [_U32, _U32]),
        "bo_cpu_build_lbvh_scratch": (_U32, [_P, _U32, _U32, _P, _P, _P]),
        "bo_cpu_trace": (None, [_P, _P, _P, _P, _U32, _I, _P, _U32]),
        "bo_rt_philox4x32_10": (None, [_P, _P, _P]),
        "bo_trace_batch": (None, [ctypes.POINTER(_BoLbvh), _P, _P, _U32, _U32, _U32, ctypes.c_uint64, _I, _P, _P, _P,
                                  _P, _U32]),
        "bo_trace_batch_views": (None, [ctypes.POINTER(_BoLbvh), _P, _P, _U32, _U32, _U32, ctypes.c_uint64, _I,
                                         _U32, _P, _P, _P, _P, _U32]),
        "bo_rt_uniform4": (None, [ctypes.c_uint64, _U32, _U32, _P]),
        "bo_rt_sincos_turns": (None, [_F, ctypes.POINTER(_F), ctypes.POINTER(_F)]),
        "bo_rt_build_lights": (_I, [_P, _P, _U32, _P, _P, _U32, ctypes.POINTER(_U32), ctypes.POINTER(_F)]),
        "bo_render": (None, [ctypes.POINTER(_BoLbvh), _P, _P, _P, _P, _P, _P, _P, _U32, _F, _P, _U32, _U32, _U32, _U32,
                             ctypes.c_uint64, _I, _P, _P, _U32]),
        "bo_render_cwbvh8": (None, [_P, _U32, _P, _U32, _P, _P, _P, _P, _P, _P, _P, _U32, _F, _P, _U32, _U32, _U32,
                                    _U32, ctypes.c_uint64, _I, _P, _P, _U32]),
        "bo_wide_build": (None, [ctypes.POINTER(_BoLbvh), _P, _U32, _U32, _P, _P, _P, _P, _P, _P]),
        "bo_cwbvh8_build": (None, [ctypes.POINTER(_BoLbvh), _P, _P, _P, _P, _P]),
        "bo_rt_series_pow": (ctypes.c_float, [ctypes.c_float, ctypes.c_float]),
        "bo_hploc_build": (ctypes.c_uint32, [ctypes.POINTER(_BoLbvh), ctypes.POINTER(_BoLbvh)]),
        "bo_tlas_instance_boxes": (None, [_P, _U32, _P, _P, _U32, _P]),
        "bo_trace_tlas": (None, [ctypes.POINTER(_BoLbvh), ctypes.POINTER(_BoLbvh), _P, _P, _P, _U32, _P, _U32,
                                 ctypes.c_int, ctypes.c_int, _P]),
        "bo_trace_cwbvh8": (None, [_P, _U32, _P, _U32, _P, _U32, ctypes.c_int, _P, _P, _U32]),
        "bo_mlp_param_count": (_U32, []),
        "bo_mlp_encode": (None, [_P, _P, _P, _P]),
        "bo_mlp_forward_f64": (None, [_P, _P, _P, _P, _U32, _P]),
        "bo_vmf_mixture_pdf": (ctypes.c_double, [_P, _P]),
        "bo_mlp_loss_f64": (ctypes.c_double, [_P, _P, _P, _P, _P, _U32, _P]),
        "bo_mlp_grad_f64": (ctypes.c_double, [_P, _P, _P, _P, _P, _U32, _P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def n_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


# ---------------------------------------------------------------- primitives
def expand_bits_3d(v: int) -> int:
    return lib().bo_expand_bits_3d(v)


def morton3(x: float, y: float, z: float) -> int:
    return lib().bo_morton3(x, y, z)


def morton_common_prefix(ca: int, ia: int, cb: int, ib: int) -> int:
    return lib().bo_morton_common_prefix(ca, ia, cb, ib)


def triangle_bounds(verts: np.ndarray) -> np.ndarray:
    v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1)
    n = v.size // 9
    out = np.empty(n * 6, np.float32)
    lib().bo_triangle_bounds(_ptr(v), n, _ptr(out))
    return out


def segment_bounds(bounds6: np.ndarray, seg_offsets: np.ndarray) -> np.ndarray:
    so = np.ascontiguousarray(seg_offsets, np.uint32)
    ns = so.size - 1
    out = np.empty(ns * 12, np.float32)
    lib().bo_segment_bounds(_ptr(bounds6), _ptr(so), ns, _ptr(out))
    return out


def morton_keys(bounds6, seg_offsets, seg_bounds12):
    so = np.ascontiguousarray(seg_offsets, np.uint32)
    n = bounds6.size // 6
    keys = np.empty(n, np.uint64)
    vals = np.empty(n, np.uint32)
    lib().bo_morton_keys(_ptr(bounds6), _ptr(so), so.size - 1, _ptr(seg_bounds12), n, _ptr(keys), _ptr(vals))
    return keys, vals


def sort_pairs(keys: np.ndarray, vals: np.ndarray, begin_bit=0, end_bit=None):
    k = np.array(keys, copy=True)
    v = np.array(vals, dtype=np.uint32, copy=True)
    if end_bit is None:
        end_bit = k.dtype.itemsize * 8
    if k.dtype == np.uint64:
        lib().bo_sort_pairs_u64(_ptr(k), _ptr(v), k.size, begin_bit, end_bit)
    elif k.dtype == np.uint32:
        lib().bo_sort_pairs_u32(_ptr(k), _ptr(v), k.size, begin_bit, end_bit)
    else:
        raise TypeError(k.dtype)
    return k, v


class CpuSort:
    """Multithreaded stable LSD radix sort (the CPU sort baseline), in place,
    with its scratch allocated once for up to ``n`` keys."""

    def __init__(self, n: int, key_bytes: int, has_values: bool, threads=None):
        self.n, self.key_bytes, self.has_values = n, key_bytes, has_values
        self.threads = threads or n_threads()
        self.scratch = np.zeros(max(int(lib().bo_cpu_sort_scratch_bytes(n, key_bytes, int(has_values),
                                                                       self.threads)), 1), np.uint8)

    def sort(self, keys: np.ndarray, vals=None, begin_bit=0, end_bit=None):
        assert keys.flags.c_contiguous and keys.dtype.itemsize == self.key_bytes and keys.size <= self.n
        assert (vals is not None) == self.has_values
        if end_bit is None:
            end_bit = self.key_bytes * 8
        lib().bo_cpu_sort(_ptr(keys), _ptr(vals) if vals is not None else None, keys.size, self.key_bytes,
                          begin_bit, end_bit, self.threads, _ptr(self.scratch))


def morton63(points: np.ndarray) -> np.ndarray:
    """63-bit Morton codes (21 bits per axis) of points in the unit cube."""
    p = np.ascontiguousarray(points, np.float32).reshape(-1)
    out = np.empty(p.size // 3, np.uint64)
    lib().bo_morton63(_ptr(p), out.size, _ptr(out))
    return out


def sort_keys(keys: np.ndarray, begin_bit=0, end_bit=None):
    k = np.array(keys, copy=True)
    if end_bit is None:
        end_bit = k.dtype.itemsize * 8
    if k.dtype == np.uint64:
        lib().bo_sort_keys_u64(_ptr(k), k.size, begin_bit, end_bit)
    elif k.dtype == np.uint32:
        lib().bo_sort_keys_u32(_ptr(k), k.size, begin_bit, end_bit)
    else:
        raise TypeError(k.dtype)
    return k


def internal_offsets(seg_offsets) -> np.ndarray:
    so = np.ascontiguousarray(seg_offsets, np.uint32)
    io = np.empty(so.size, np.uint32)
    lib().bo_internal_offsets(_ptr(so), so.size - 1, _ptr(io))
    return io


def topology(codes, seg_offsets, topdown=False):
    so = np.ascontiguousarray(seg_offsets, np.uint32)
    ns = so.size - 1
    io = internal_offsets(so)
    ni = int(io[-1])
    n = codes.size
    meta = np.zeros(max(ni, 1) * 4, np.uint32)
    lp = np.zeros(max(n, 1), np.uint32)
    lc = np.zeros(max(ni, 1), np.uint32)
    roots = np.zeros(max(ns, 1), np.uint32)
    codes = np.ascontiguousarray(codes, np.uint32)
    if topdown:
        lib().bo_lbvh_topology_topdown(_ptr(codes), _ptr(so), _ptr(io), ns, _ptr(meta), _ptr(lp), _ptr(lc), _ptr(roots))
    else:
        lib().bo_lbvh_topology(_ptr(codes), _ptr(so), _ptr(io), ns, _ptr(meta), _ptr(lp), _ptr(lc), _ptr(roots), None)
    return meta, lp, lc, roots


# ---------------------------------------------------------------- full build
@dataclass
class OracleLbvh:
    verts: np.ndarray
    seg_offsets: np.ndarray
    n_leaves: int
    n_internal: int
    leaf_bounds: np.ndarray
    seg_bounds: np.ndarray
    sort_keys: np.ndarray
    leaf_ids: np.ndarray
    morton_codes: np.ndarray
    node_meta: np.ndarray
    node_bounds: np.ndarray
    node_leaf_counts: np.ndarray
    node_flags: np.ndarray
    leaf_parent: np.ndarray
    roots: np.ndarray
    internal_offsets: np.ndarray
    _struct: _BoLbvh = None

    def struct(self) -> _BoLbvh:
        s = _BoLbvh()
        s.n_leaves, s.n_internal, s.n_segments = self.n_leaves, self.n_internal, self.seg_offsets.size - 1
        for name in ("leaf_bounds", "seg_bounds", "sort_keys", "leaf_ids", "morton_codes", "node_meta",
                     "node_bounds", "node_leaf_counts", "node_flags", "leaf_parent", "roots",
                     "internal_offsets", "seg_offsets"):
            setattr(s, name, _ptr(getattr(self, name)))
        return s


def lbvh_build(verts: np.ndarray, seg_offsets=None) -> OracleLbvh:
    v = np.ascontiguousarray(verts, np.float32).reshape(-1)
    n = v.size // 9
    so = np.array([0, n] if seg_offsets is None else seg_offsets, np.uint32)
    ns = so.size - 1
    io = np.zeros(ns + 1, np.uint32)
    lib().bo_internal_offsets(_ptr(so), ns, _ptr(io))
    ni = int(io[-1])
    m = max(ni, 1)
    o = OracleLbvh(
        verts=v, seg_offsets=so, n_leaves=n, n_internal=ni,
        leaf_bounds=np.zeros(max(n, 1) * 6, np.float32), seg_bounds=np.zeros(ns * 12, np.float32),
        sort_keys=np.zeros(max(n, 1), np.uint64), leaf_ids=np.zeros(max(n, 1), np.uint32),
        morton_codes=np.zeros(max(n, 1), np.uint32), node_meta=np.zeros(m * 4, np.uint32),
        node_bounds=np.zeros(m * 12, np.float32), node_leaf_counts=np.zeros(m, np.uint32),
        node_flags=np.zeros(m, np.uint32), leaf_parent=np.zeros(max(n, 1), np.uint32),
        roots=np.zeros(ns, np.uint32), internal_offsets=io,
    )
    s = o.struct()
    lib().bo_lbvh_build(_ptr(v), _ptr(so), ns, ctypes.byref(s))
    o._struct = s
    return o


def hploc_build(verts: np.ndarray, seg_offsets=None) -> OracleLbvh:
    """The H-PLOC tree over the same sorted leaves as lbvh_build (same leaf
    bounds, keys and ids; its own node arrays, ids in task post order)."""
    k = lbvh_build(verts, seg_offsets)
    m = max(k.n_internal, 1)
    o = OracleLbvh(
        verts=k.verts, seg_offsets=k.seg_offsets, n_leaves=k.n_leaves, n_internal=k.n_internal,
        leaf_bounds=k.leaf_bounds, seg_bounds=k.seg_bounds, sort_keys=k.sort_keys, leaf_ids=k.leaf_ids,
        morton_codes=k.morton_codes, node_meta=np.full(m * 4, SENTINEL, np.uint32),
        node_bounds=np.zeros(m * 12, np.float32), node_leaf_counts=np.zeros(m, np.uint32),
        node_flags=np.zeros(m, np.uint32), leaf_parent=np.full(max(k.n_leaves, 1), SENTINEL, np.uint32),
        roots=np.full(k.roots.size, SENTINEL, np.uint32), internal_offsets=k.internal_offsets,
    )
    ks, os_ = k.struct(), o.struct()
    err = lib().bo_hploc_build(ctypes.byref(ks), ctypes.byref(os_))
    if err:
        raise RuntimeError(f"oracle H-PLOC failed ({err})")
    o._struct = os_
    return o


def tlas_instance_boxes(blas: OracleLbvh, transforms: np.ndarray, blas_idx: np.ndarray) -> np.ndarray:
    """Each instance's world box as a [min, max, min] triangle record (n, 9)."""
    xf = np.ascontiguousarray(transforms, np.float32).reshape(-1)
    bi = np.ascontiguousarray(blas_idx, np.uint32)
    out = np.zeros(bi.size * 9, np.float32)
    lib().bo_tlas_instance_boxes(_ptr(blas.seg_bounds), blas.seg_offsets.size - 1, _ptr(xf), _ptr(bi), bi.size,
                                 _ptr(out))
    return out.reshape(-1, 9)


def trace_tlas(top: OracleLbvh, blas: OracleLbvh, inv_transforms: np.ndarray, blas_idx: np.ndarray,
               rays_soa: np.ndarray, any_hit: bool = False, tri_mode=TRI_WATERTIGHT) -> np.ndarray:
    """Closest or any hit of SoA rays through a top-level tree over instances
    of a segmented BLAS set; hits8 with the instance in word 3."""
    rays = np.ascontiguousarray(rays_soa, np.float32).reshape(-1)
    n = rays.size // 8
    inv = np.ascontiguousarray(inv_transforms, np.float32).reshape(-1)
    bi = np.ascontiguousarray(blas_idx, np.uint32)
    hits = np.zeros(n * 8, np.float32)
    ts, bs = top.struct(), blas.struct()
    lib().bo_trace_tlas(ctypes.byref(ts), ctypes.byref(bs), _ptr(blas.verts), _ptr(inv), _ptr(bi), bi.size,
                        _ptr(rays), n, int(any_hit), int(tri_mode), _ptr(hits))
    return hits


def canonical_tree(bvh, seg: int = 0) -> list:
    """Segment seg's tree as a list of words, independent of internal node
    ids: pre-order, one entry per node, leaf = ("L", sorted index), internal
    = ("N", leaf count, both child boxes as u32 bits)."""
    meta = np.asarray(bvh.node_meta).reshape(-1, 4)
    nb = np.asarray(bvh.node_bounds).view(np.uint32).reshape(-1, 12)
    lc = np.asarray(bvh.node_leaf_counts)
    out, stack = [], [int(np.asarray(bvh.roots)[seg])]
    while stack:
        r = stack.pop()
        if r == SENTINEL:
            out.append(("E",))
        elif r & LEAF_FLAG:
            out.append(("L", r & 0x7FFFFFFF))
        else:
            out.append(("N", int(lc[r]), tuple(int(x) for x in nb[r])))
            stack += [int(meta[r, 2]), int(meta[r, 1])]
    return out


# ---------------------------------------------------------------- camera/trace
def camera_from_vfov(origin, target, world_up, vfov_deg) -> np.ndarray:
    out = np.zeros(20, np.float32)
    a = [np.ascontiguousarray(x, np.float32) for x in (origin, target, world_up)]
    lib().bo_camera_from_vfov(_ptr(a[0]), _ptr(a[1]), _ptr(a[2]), float(vfov_deg), _ptr(out))
    return out


def camera_make(origin, target, world_up, fov_scale) -> np.ndarray:
    out = np.zeros(20, np.float32)
    a = [np.ascontiguousarray(x, np.float32) for x in (origin, target, world_up)]
    lib().bo_camera_make(_ptr(a[0]), _ptr(a[1]), _ptr(a[2]), float(fov_scale), _ptr(out))
    return out


def camera_rays(cameras20: np.ndarray, n_rays: int, width: int, height: int) -> np.ndarray:
    cams = np.ascontiguousarray(cameras20, np.float32)
    out = np.empty(8 * n_rays, np.float32)
    lib().bo_camera_rays(_ptr(cams), n_rays, width, height, _ptr(out))
    return out


def trace_bvh2(bvh: OracleLbvh, rays_soa: np.ndarray, tri_mode=TRI_WATERTIGHT, threads=None) -> np.ndarray:
    rays = np.ascontiguousarray(rays_soa, np.float32)
    n = rays.size // 8
    hits = np.empty(8 * n, np.float32)
    s = bvh.struct()
    lib().bo_trace_bvh2(ctypes.byref(s), _ptr(bvh.verts), _ptr(rays), n, tri_mode, _ptr(hits),
                        threads or n_threads())
    return hits


def trace_bvh2_stats(bvh: OracleLbvh, rays_soa: np.ndarray, tri_mode=TRI_WATERTIGHT) -> np.ndarray:
    rays = np.ascontiguousarray(rays_soa, np.float32)
    n = rays.size // 8
    stats = np.empty(5 * n, np.uint32)  # GpuTraversalStats per ray (trace.mojo:62-90)
    s = bvh.struct()
    lib().bo_trace_bvh2_stats(ctypes.byref(s), _ptr(bvh.verts), _ptr(rays), n, tri_mode, _ptr(stats))
    return stats


def trace_brute(verts: np.ndarray, rays_soa: np.ndarray, tri_mode=TRI_WATERTIGHT, threads=None) -> np.ndarray:
    v = np.ascontiguousarray(verts, np.float32).reshape(-1)
    rays = np.ascontiguousarray(rays_soa, np.float32)
    n = rays.size // 8
    hits = np.empty(8 * n, np.float32)
    lib().bo_trace_brute(_ptr(v), v.size // 9, _ptr(rays), n, tri_mode, _ptr(hits), threads or n_threads())
    return hits


# ---------------------------------------------------------------- CPU baseline
class CpuLbvh:
    """The reference's CPU LBVH (BVH2, leaf size 1) restated in C; the timed
    CPU baseline.  ``build`` returns the node count."""

    NODE_DTYPE = np.dtype([("bmin", np.float32, 3), ("bmax", np.float32, 3), ("left_or_first", np.uint32),
                           ("count", np.uint32)])

    def __init__(self, verts: np.ndarray, threads=None):
        self.verts = np.ascontiguousarray(verts, np.float32).reshape(-1)
        self.n = self.verts.size // 9
        self.threads = threads or n_threads()
        self.nodes = np.zeros(max(2 * self.n - 1, 1), self.NODE_DTYPE)
        self.items = np.zeros(max(self.n, 1), np.uint32)
        # the builder's buffers live as long as the builder (no allocation per build)
        self.scratch = np.zeros(max(int(lib().bo_cpu_lbvh_scratch_bytes(self.n, self.threads)), 1), np.uint8)
        self.node_count = 0

    def build(self) -> int:
        self.node_count = lib().bo_cpu_build_lbvh_scratch(_ptr(self.verts), self.n, self.threads, _ptr(self.nodes),
                                                          _ptr(self.items), _ptr(self.scratch))
        return self.node_count

    def trace(self, rays_soa: np.ndarray, tri_mode=TRI_WATERTIGHT, hits=None) -> np.ndarray:
        rays = np.ascontiguousarray(rays_soa, np.float32)
        n = rays.size // 8
        if hits is None:
            hits = np.empty(8 * n, np.float32)
        lib().bo_cpu_trace(_ptr(self.nodes), _ptr(self.items), _ptr(self.verts), _ptr(rays), n, tri_mode,
                           _ptr(hits), self.threads)
        return hits


def hits_prim(hits8: np.ndarray) -> np.ndarray:
    return hits8.reshape(-1, 8)[:, 2].view(np.uint32)


def hits_t(hits8: np.ndarray) -> np.ndarray:
    return hits8.reshape(-1, 8)[:, 7]


# ---------------------------------------------------------------- path tracer
def philox4x32_10(ctr, key) -> list:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().bo_rt_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return [int(x) for x in out]


def rt_uniform4(seed: int, path_id: int, stage: int) -> np.ndarray:
    out = np.zeros(4, np.float32)
    lib().bo_rt_uniform4(seed, path_id, stage, _ptr(out))
    return out


def rt_sincos_turns(u: float):
    s, c = ctypes.c_float(), ctypes.c_float()
    lib().bo_rt_sincos_turns(u, ctypes.byref(s), ctypes.byref(c))
    return s.value, c.value


def rt_build_lights(scene):
    n_em = int(np.count_nonzero((scene.surfaces >> 28) == 3))
    out = np.zeros(max(n_em, 1) * 16, np.float32)
    n = ctypes.c_uint32(0)
    w = ctypes.c_float(0.0)
    rc = lib().bo_rt_build_lights(_ptr(scene.vertices), _ptr(scene.surfaces), scene.n_tris, _ptr(scene.emissives),
                                  _ptr(out), max(n_em, 1), ctypes.byref(n), ctypes.byref(w))
    assert rc == 0
    return out, n.value, w.value


def render(scene, camera, width, height, spp, max_depth=8, seed=2026, algorithm=4, lights=None, bvh=None,
           threads=None, return_samples=False, cwbvh8=None):
    """CPU restatement of the wavefront tracer: (height, width, 3) pixels.
    ``cwbvh8`` (an OracleCwbvh8 of the scene's tree) traces through the
    compressed 8-wide tree instead of the binary LBVH."""
    if bvh is None and cwbvh8 is None:
        bvh = lbvh_build(scene.vertices)
    if lights is None:
        lights, n_lights, total = rt_build_lights(scene)
    else:
        lights, n_lights, total = lights
    cam = np.ascontiguousarray(camera, np.float32)
    pixels = np.zeros(3 * width * height, np.float32)
    samples = np.zeros(3 * width * height * spp, np.float32) if return_samples else None
    metals = getattr(scene, "metals", None)
    dielectrics = getattr(scene, "dielectrics", None)
    metals = None if metals is None else np.ascontiguousarray(metals, np.float32).reshape(-1)
    dielectrics = None if dielectrics is None else np.ascontiguousarray(dielectrics, np.float32).reshape(-1)
    tail = (_ptr(scene.surfaces), _ptr(scene.lambertians), _ptr(scene.emissives),
            None if metals is None else _ptr(metals), None if dielectrics is None else _ptr(dielectrics),
            _ptr(lights), n_lights, total, _ptr(cam), width, height, spp, max_depth, seed, algorithm, _ptr(pixels),
            None if samples is None else _ptr(samples), threads or n_threads())
    if cwbvh8 is not None:
        verts = np.ascontiguousarray(scene.vertices, np.float32).reshape(-1)
        n0 = int(cwbvh8.node_offsets[1]) - int(cwbvh8.node_offsets[0])
        lib().bo_render_cwbvh8(_ptr(cwbvh8.nodes), n0, _ptr(cwbvh8.triangles), cwbvh8.triangles.size // CW_TRI_WORDS,
                               _ptr(verts), *tail)
    else:
        s = bvh.struct()
        lib().bo_render(ctypes.byref(s), _ptr(bvh.verts), *tail)
    img = pixels.reshape(height, width, 3)
    return (img, samples.reshape(height, width, spp, 3)) if return_samples else img


def trace_batch(bvh: OracleLbvh, cams, cam_stride, width, height, seed=7, tri_mode=TRI_WATERTIGHT, threads=None,
                view_base=0):
    """Primary + cosine bounce rays of every segment; `view_base` > 0 treats
    segment k as view view_base + k of a larger batch (its random streams)."""
    n = (bvh.seg_offsets.size - 1) * width * height
    t0, t1 = np.zeros(n, np.float32), np.zeros(n, np.float32)
    p0, p1 = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    c = np.ascontiguousarray(cams, np.float32)
    s = bvh.struct()
    lib().bo_trace_batch_views(ctypes.byref(s), _ptr(bvh.verts), _ptr(c), cam_stride, width, height, seed, tri_mode,
                               view_base, _ptr(t0), _ptr(p0), _ptr(t1), _ptr(p1), threads or n_threads())
    return t0, p0, t1, p1


# ---- path-guiding network (FP64) -------------------------------------------
def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def mlp_param_count() -> int:
    return int(lib().bo_mlp_param_count())


def mlp_encode(p, n, box) -> np.ndarray:
    out = np.zeros(64, np.float32)
    p, n, box = _f32(p), _f32(n), _f32(box)
    lib().bo_mlp_encode(_ptr(p), _ptr(n), _ptr(box), _ptr(out))
    return out


def mlp_forward(params, pos, nrm, box) -> np.ndarray:
    params = np.ascontiguousarray(params, np.float64)
    pos, nrm, box = _f32(pos), _f32(nrm), _f32(box)
    n = pos.size // 3
    out = np.zeros((n, 20), np.float64)
    lib().bo_mlp_forward_f64(_ptr(params), _ptr(pos), _ptr(nrm), _ptr(box), n, _ptr(out))
    return out


def vmf_mixture_pdf(out20, d) -> float:
    o = np.ascontiguousarray(out20, np.float64)
    d = _f32(d)
    return float(lib().bo_vmf_mixture_pdf(_ptr(o), _ptr(d)))


def mlp_loss(params, pos, nrm, dirs, w, box) -> float:
    params = np.ascontiguousarray(params, np.float64)
    pos, nrm, dirs, w, box = _f32(pos), _f32(nrm), _f32(dirs), _f32(w), _f32(box)
    return float(lib().bo_mlp_loss_f64(_ptr(params), _ptr(pos), _ptr(nrm), _ptr(dirs), _ptr(w), w.size, _ptr(box)))


def mlp_grad(params, pos, nrm, dirs, w, box):
    """(gradient [n_params] f64, loss) of sum -w log pdf(dir)."""
    params = np.ascontiguousarray(params, np.float64)
    pos, nrm, dirs, w, box = _f32(pos), _f32(nrm), _f32(dirs), _f32(w), _f32(box)
    g = np.zeros(params.size, np.float64)
    loss = lib().bo_mlp_grad_f64(_ptr(params), _ptr(pos), _ptr(nrm), _ptr(dirs), _ptr(w), w.size, _ptr(box),
                                 _ptr(g))
    return g, float(loss)


# ---- wide BVH collapse ------------------------------------------------------
@dataclass
class OracleWide:
    width: int
    nodes: np.ndarray         # [n_nodes * 7 * W] f32 (meta as bits)
    leaf_indices: np.ndarray  # [n_blocks * W] u32
    leaf_tris: np.ndarray     # [n_blocks * 12 * W] f32
    leaf_sorted: np.ndarray   # [n_blocks * W] u32
    node_offsets: np.ndarray  # [S+1]
    leaf_offsets: np.ndarray  # [S+1]


def wide_build(bvh: OracleLbvh, width: int, max_leaf: int = 4) -> OracleWide:
    """Sequential BVH2 -> W-wide collapse with fat leaves; a node's internal
    children take consecutive ids, its leaf blocks consecutive blocks."""
    n = max(bvh.n_leaves, 1)
    S = bvh.seg_offsets.size - 1
    nodes = np.zeros(n * 7 * width, np.float32)
    li = np.zeros(n * width, np.uint32)
    lt = np.zeros(n * 12 * width, np.float32)
    ls = np.zeros(n * width, np.uint32)
    no = np.zeros(S + 1, np.uint32)
    lo = np.zeros(S + 1, np.uint32)
    s = bvh.struct()
    lib().bo_wide_build(ctypes.byref(s), _ptr(bvh.verts), width, max_leaf, _ptr(nodes), _ptr(li), _ptr(lt), _ptr(ls),
                        _ptr(no), _ptr(lo))
    nn, nb = int(no[-1]), int(lo[-1])
    return OracleWide(width, nodes[:nn * 7 * width], li[:nb * width], lt[:nb * 12 * width], ls[:nb * width], no, lo)


# ---- CWBVH8 -------------------------------------------------------------------
CW_NODE_WORDS = 20
CW_TRI_WORDS = 12


@dataclass
class OracleCwbvh8:
    wide_nodes: np.ndarray    # [n_nodes * 56] f32: the W = 8 octant-slot collapse (meta as bits)
    nodes: np.ndarray         # [n_nodes * 20] f32: 80-byte compressed nodes
    triangles: np.ndarray     # [n_tris * 12] f32: e1, 0, e2, 0, v0, prim bits
    node_offsets: np.ndarray  # [S+1]


def cwbvh8_build(bvh: OracleLbvh) -> OracleCwbvh8:
    """W = 8 collapse with octant slots and leaves of at most 3 triangles,
    encoded as CWBVH8 nodes and triangle records."""
    n = max(bvh.n_leaves, 1)
    S = bvh.seg_offsets.size - 1
    wide = np.zeros(n * 56, np.float32)
    nodes = np.zeros(n * CW_NODE_WORDS, np.float32)
    tris = np.zeros(n * CW_TRI_WORDS, np.float32)
    no = np.zeros(S + 1, np.uint32)
    s = bvh.struct()
    lib().bo_cwbvh8_build(ctypes.byref(s), _ptr(bvh.verts), _ptr(wide), _ptr(nodes), _ptr(tris), _ptr(no))
    nn = int(no[-1])
    return OracleCwbvh8(wide[:nn * 56], nodes[:nn * CW_NODE_WORDS], tris[:bvh.n_leaves * CW_TRI_WORDS], no)


def trace_cwbvh8(cw: OracleCwbvh8, rays: np.ndarray, any_hit: bool = False, threads: int = 0,
                 with_errors: bool = False):
    """Closest or any hit of SoA rays [8][n] over segment 0's CWBVH8 tree:
    hits8 [n * 8] f32 (u, v, prim bits, inst bits, normal, t)."""
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1)
    n = rays.size // 8
    hits = np.zeros(n * 8, np.float32)
    err = np.zeros(max(n, 1), np.uint32)
    n0 = int(cw.node_offsets[1]) - int(cw.node_offsets[0])
    nt = cw.triangles.size // CW_TRI_WORDS
    lib().bo_trace_cwbvh8(_ptr(cw.nodes), n0, _ptr(cw.triangles), nt, _ptr(rays), n, int(any_hit), _ptr(hits),
                          _ptr(err), threads or os.cpu_count() or 1)
    return (hits, err[:n]) if with_errors else hits


# ---- staged top levels --------------------------------------------------------
TOP_NODES = 256
TOP_FLAG = 0x40000000


def stage_top(bvh: OracleLbvh, k: int = TOP_NODES) -> np.ndarray:
    """The staged top levels of segment 0's tree as u32 words: header
    [count, root ref, 0, 0] then k records of 16 words [left AABB (6) |
    right AABB (6) | left ref, right ref, 0, 0].  Slots follow breadth-first
    order, left child before right; a staged child is referenced as
    TOP_FLAG | slot, every other child keeps its tagged global ref.  This
    layout is the library's own (the reference reads the whole tree from
    global memory), restated here to check it word for word."""
    out = np.zeros(4 + 16 * k, np.uint32)
    root = int(bvh.roots[0])
    out[1] = root
    if root == SENTINEL or root & LEAF_FLAG:
        return out
    meta = bvh.node_meta.reshape(-1, 4)
    nb = bvh.node_bounds.view(np.uint32).reshape(-1, 12)
    refs = [root]
    slot_of = {root: 0}
    i = 0
    while i < len(refs):  # breadth first: refs grows level by level
        m = meta[refs[i]]
        for c in (int(m[1]), int(m[2])):
            if not (c & LEAF_FLAG) and len(refs) < k:
                slot_of[c] = len(refs)
                refs.append(c)
        i += 1
    for s, r in enumerate(refs):
        rec = out[4 + 16 * s: 4 + 16 * (s + 1)]
        rec[0:12] = nb[r]
        m = meta[r]
        for j, c in enumerate((int(m[1]), int(m[2]))):
            rec[12 + j] = TOP_FLAG | slot_of[c] if c in slot_of else c
    out[0] = len(refs)
    return out
