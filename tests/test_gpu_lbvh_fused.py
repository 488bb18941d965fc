"""The one-launch LBVH build (bounds, Morton keys, sort and hierarchy in one
cooperative kernel for a single scene of up to 2^17 triangles) against the
per-stage kernels and the oracle, bit for bit, on sizes around its 512-leaf
tiles and on inputs that take the bucket sort (random triangles, a
degenerate axis) or its LSD fallback (duplicate centroids, one far outlier:
buckets past 256 keys)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402

from test_gpu_lbvh import assert_same_build, h  # noqa: E402

SIZES = [2, 3, 31, 100, 511, 512, 513, 2047, 2048, 2049, 6000, 65535, 65536, 65537, 100_003, 131071, 131072]


def _build(v, fused: bool):
    from bajo_b200 import _lib, bvh
    L = _lib.load()
    assert L.bajo_lbvh_fused_max_set(_lib.FUSED_MAX_LEAVES if fused else 0) == _lib.OK
    try:
        d = torch.from_numpy(np.ascontiguousarray(v, np.float32)).cuda()
        b = bvh.build_triangle_bvh(d)
        torch.cuda.synchronize()
        assert b.workspace.status() == 0
        return b
    finally:
        L.bajo_lbvh_fused_max_set(_lib.FUSED_MAX_LEAVES)


def _arrays(b, n):
    return [h(b.leaf_bounds, np.uint32)[: 6 * n], h(b.seg_bounds, np.uint32)[:12], h(b.sort_keys, np.uint64)[:n],
            h(b.leaf_ids, np.uint32)[:n], h(b.morton_codes, np.uint32)[:n], h(b.leaf_parent, np.uint32)[:n],
            h(b.node_meta, np.uint32)[: 4 * (n - 1)], h(b.node_bounds, np.uint32)[: 12 * (n - 1)],
            h(b.node_leaf_counts, np.uint32)[: n - 1], h(b.node_flags, np.uint32)[: n - 1],
            h(b.leaf_tris, np.uint32)[: 12 * n], h(b.roots, np.uint32)[:1], h(b.internal_offsets, np.uint32)[:2]]


def _scene(kind, n, seed):
    v = scenes.random_triangles(n, seed=seed).reshape(-1, 3, 3)
    if kind == "duplicates":  # many triangles share a centroid: equal codes
        v[: n // 2] = v[0]
    elif kind == "outlier":  # one far triangle squeezes the rest into few codes
        v[n // 3] += 1000.0
    elif kind == "flat":  # a degenerate axis
        v[:, :, 2] = 0.5
    return np.ascontiguousarray(v.reshape(-1))


@pytest.mark.parametrize("n", SIZES)
def test_fused_equals_oracle_and_stage_kernels(oracle, n):
    from bajo_b200 import _lib
    L = _lib.load()
    v = _scene("random", n, seed=n)
    launches = ctypes.c_int32(0)
    assert L.bajo_lbvh_build_launches(n, 1, ctypes.byref(launches)) == _lib.OK
    assert launches.value == 1
    f = _build(v, True)
    assert_same_build(f, oracle.lbvh_build(v))
    s = _build(v, False)
    for a, b in zip(_arrays(f, n), _arrays(s, n)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["duplicates", "outlier", "flat"])
@pytest.mark.parametrize("n", [5000, 65536, 131072])
def test_fused_hard_inputs(oracle, kind, n):
    v = _scene(kind, n, seed=7)
    f = _build(v, True)
    assert_same_build(f, oracle.lbvh_build(v))


@pytest.mark.parametrize("cap", [1, 2, 3, 64, 700])
@pytest.mark.parametrize("kind,n", [("random", 513), ("random", 2049), ("random", 65536), ("duplicates", 65536),
                                    ("outlier", 100_003), ("random", 131072)])
def test_fused_top_ranges(oracle, cap, kind, n):
    """The top of the tree over the tiles' largest subtrees, cut into ranges
    of at most `cap` subtrees per CTA: the splits between ranges meet in
    global memory, and the arrays stay identical to the per-stage build's."""
    from bajo_b200 import _lib
    L = _lib.load()
    v = _scene(kind, n, seed=n + cap)
    assert L.bajo_lbvh_fused_top_cap_set(cap) == _lib.OK
    try:
        f = _build(v, True)
    finally:
        assert L.bajo_lbvh_fused_top_cap_set(0) == _lib.OK
    s = _build(v, False)
    for a, b in zip(_arrays(f, n), _arrays(s, n)):
        assert np.array_equal(a, b)
    if n == 65536 and cap == 64:
        assert_same_build(f, oracle.lbvh_build(v))


def test_fused_top_cap_limits():
    from bajo_b200 import _lib
    L = _lib.load()
    assert L.bajo_lbvh_fused_top_cap_set(_lib.LBVH_TOP_CAP + 1) == _lib.ERR_TOO_LARGE
    assert L.bajo_lbvh_fused_top_cap_set(_lib.LBVH_TOP_CAP) == _lib.OK
    assert L.bajo_lbvh_fused_top_cap_set(0) == _lib.OK


@pytest.mark.parametrize("fn", ["bajo_lbvh_build", "bajo_hploc_build"])
@pytest.mark.parametrize("field", ["node_bounds", "node_meta", "leaf_tris"])
def test_build_rejects_unaligned_records(fn, field):
    """Node boxes and triangle records are read and written 16 bytes at a
    time: a record array that is not 16-byte aligned is refused up front."""
    from bajo_b200 import _lib, bvh
    L = _lib.load()
    n = 1000
    d = torch.from_numpy(scenes.random_triangles(n, seed=3)).cuda()
    ws = bvh.GpuBvhBuildWorkspace(n, 1)
    t = bvh.build_triangle_bvh(d, workspace=ws)
    c = t.c_struct(stage_top=False)
    setattr(c, field, getattr(t, field).data_ptr() + 4)
    s = torch.cuda.current_stream().cuda_stream
    assert getattr(L, fn)(d.data_ptr(), ctypes.byref(c), ws.buffer.data_ptr(), ws.buffer.numel(),
                          s) == _lib.ERR_INVALID_ARGUMENT
    torch.cuda.synchronize()


def test_fused_rebuilds_reuse_workspace(oracle):
    """Repeated builds through one workspace (the barrier counter and
    histograms are cleared per build) and interleaved sizes."""
    from bajo_b200 import bvh
    v1 = scenes.random_triangles(65536, seed=1)
    v2 = scenes.random_triangles(70000, seed=2)
    ws = bvh.GpuBvhBuildWorkspace(70000, 1)
    d1, d2 = torch.from_numpy(v1).cuda(), torch.from_numpy(v2).cuda()
    t1 = bvh.build_triangle_bvh(d1, workspace=ws)
    for _ in range(3):
        t1 = bvh.build_triangle_bvh(d1, workspace=ws, out=t1)
    t2 = bvh.build_triangle_bvh(d2, workspace=ws)
    torch.cuda.synchronize()
    assert ws.status() == 0
    assert_same_build(t1, oracle.lbvh_build(v1))
    assert_same_build(t2, oracle.lbvh_build(v2))


def test_fused_unaligned_vertices(oracle):
    """Vertex buffers that are not 16-byte aligned take the scalar loads."""
    from bajo_b200 import bvh
    n = 9000
    v = scenes.random_triangles(n, seed=4)
    big = torch.zeros(v.size + 1, dtype=torch.float32, device="cuda")
    big[1:] = torch.from_numpy(v).cuda()
    d = big[1:]
    assert d.data_ptr() % 16 != 0
    b = bvh.build_triangle_bvh(d)
    torch.cuda.synchronize()
    assert b.workspace.status() == 0
    assert_same_build(b, oracle.lbvh_build(v))


def test_fused_limits():
    from bajo_b200 import _lib
    L = _lib.load()
    assert L.bajo_lbvh_fused_max_set(_lib.FUSED_MAX_LEAVES + 1) == _lib.ERR_TOO_LARGE
    x = ctypes.c_int32(0)
    assert L.bajo_lbvh_build_launches(_lib.FUSED_MAX_LEAVES + 1, 1, ctypes.byref(x)) == _lib.OK and x.value > 1
    assert L.bajo_lbvh_build_launches(1000, 2, ctypes.byref(x)) == _lib.OK and x.value > 1  # segmented
    assert L.bajo_lbvh_build_launches(1, 1, ctypes.byref(x)) == _lib.OK and x.value > 1
    assert L.bajo_lbvh_stage_count(65536, 1, ctypes.byref(x)) == _lib.OK and x.value == 2


def test_fused_timed_build_events(oracle):
    """The stage-timed build takes the same path: two events."""
    from bajo_b200 import _lib, bvh
    L = _lib.load()
    n = 65536
    v = scenes.random_triangles(n, seed=12)
    d = torch.from_numpy(v).cuda()
    ws = bvh.GpuBvhBuildWorkspace(n, 1)
    t = bvh.build_triangle_bvh(d, workspace=ws)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for e in evs:
        e.record()
    arr = (ctypes.c_void_p * 2)(*[e.cuda_event for e in evs])
    c = t.c_struct(stage_top=False)
    s = torch.cuda.current_stream().cuda_stream
    assert L.bajo_lbvh_build_timed(d.data_ptr(), ctypes.byref(c), ws.buffer.data_ptr(), ws.buffer.numel(), s, arr,
                                   2) == _lib.OK
    torch.cuda.synchronize()
    assert evs[0].elapsed_time(evs[1]) > 0
    assert ws.status() == 0
    assert_same_build(t, oracle.lbvh_build(v))
