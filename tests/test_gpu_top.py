"""GPU parity of the staged top levels: the build writes the oracle's
breadth-first records word for word, and closest hits (rays, camera and the
instrumented camera counts) through the staged kernels equal the unstaged
kernels' and the oracle's bit for bit."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import _lib, bvh, camera, scenes  # noqa: E402

FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def staged_words(tree):
    return tree.top_nodes.view(torch.int32).cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_top_matches_oracle(oracle, golden_dir, name):
    verts = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))[name + "__verts"]
    tree = bvh.build_triangle_bvh(dev(verts.astype(np.float32)), stage_top=True)
    assert np.array_equal(staged_words(tree), oracle.stage_top(oracle.lbvh_build(verts)))


@pytest.mark.parametrize("n", [1, 2, 3, 200, 256, 257, 258, 513, 65536])
def test_random_top_matches_oracle(oracle, n):
    verts = scenes.random_triangles(n, seed=n)
    tree = bvh.build_triangle_bvh(dev(verts), stage_top=True)
    want = oracle.stage_top(oracle.lbvh_build(verts))
    assert np.array_equal(staged_words(tree), want)
    count, root = tree.top_header()
    assert count == min(_lib.TOP_NODES, max(n - 1, 0))
    assert root == int(tree.roots[0].item()) & 0xFFFFFFFF


def test_segmented_tree_stages_segment_zero(oracle):
    verts = scenes.random_triangles(3000, seed=8)
    seg = np.array([0, 700, 701, 3000], np.uint32)
    tree = bvh.build_triangle_bvh(dev(verts), seg, stage_top=True)
    assert np.array_equal(staged_words(tree), oracle.stage_top(oracle.lbvh_build(verts, seg)))


def test_restage_after_rebuild_of_other_geometry(oracle):
    a = scenes.random_triangles(5000, seed=1)
    b = scenes.random_triangles(5000, seed=2)
    tree = bvh.build_triangle_bvh(dev(a), stage_top=True)
    c = tree.c_struct(stage_top=False)  # a build that leaves top_nodes alone
    import ctypes
    _lib.check(_lib.load().bajo_lbvh_build(dev(b).data_ptr(), ctypes.byref(c), tree.workspace.buffer.data_ptr(),
                                           tree.workspace.buffer.numel(), None), "bajo_lbvh_build")
    torch.cuda.synchronize()
    assert np.array_equal(staged_words(tree), oracle.stage_top(oracle.lbvh_build(a)))  # stale
    tree.restage_top()
    assert np.array_equal(staged_words(tree), oracle.stage_top(oracle.lbvh_build(b)))


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.5, 1.5, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:64, 0] = 0.0
    d[64:128, 1:] = 0.0
    rays = np.zeros((8, n), np.float32)
    rays[0:3] = o.T
    rays[3] = rng.uniform(0.0, 0.1, n)
    rays[4:7] = d.T
    rays[7] = rng.uniform(0.5, 5.0, n)
    return rays.reshape(-1)


def _trace(tree, rays, mode, staged):
    import ctypes
    n = rays.size // 8
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    c = tree.c_struct(stage_top=staged)
    _lib.check(_lib.load().bajo_trace_rays(ctypes.byref(c), dev(rays).data_ptr(), n, mode, hits.data_ptr(), None,
                                           None, st.data_ptr(), None), "bajo_trace_rays")
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return hits.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 1])
def test_staged_hits_equal_unstaged_and_oracle(oracle, golden_dir, mode):
    g = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))
    tg = np.load(os.path.join(golden_dir, "trace_fixtures.npz"))
    for name in FIXTURES:
        verts, rays = g[name + "__verts"], tg[name + "__rays"]
        tree = bvh.build_triangle_bvh(dev(verts.astype(np.float32)), stage_top=True)
        a = _trace(tree, rays, mode, True)
        b = _trace(tree, rays, mode, False)
        ref = oracle.trace_bvh2(oracle.lbvh_build(verts), rays, mode)
        assert np.array_equal(a.view(np.uint32), ref.view(np.uint32)), name
        assert np.array_equal(b.view(np.uint32), ref.view(np.uint32)), name


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n_tris", [300, 30000])
def test_staged_random_rays(oracle, mode, n_tris):
    v = scenes.random_triangles(n_tris, seed=3, spread=0.03)
    tree = bvh.build_triangle_bvh(dev(v), stage_top=True)
    rays = _rays(300_000, 9)  # more rays than one pass of the persistent grid
    a = _trace(tree, rays, mode, True)
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), rays, mode)
    assert np.array_equal(a.view(np.uint32), ref.view(np.uint32))


def test_staged_camera_and_counts_equal_unstaged():
    import ctypes
    v = scenes.random_triangles(65536, seed=0)
    tree = bvh.build_triangle_bvh(dev(v), stage_top=True)
    cam = dev(camera.plain_lbvh_camera())
    n = 1024 * 1024
    out = {}
    for staged in (True, False):
        c = tree.c_struct(stage_top=staged)
        hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
        stats = torch.zeros(5 * n, dtype=torch.int32, device="cuda")
        _lib.check(_lib.load().bajo_trace_camera(ctypes.byref(c), cam.data_ptr(), n, 1024, 1024, 1, hits.data_ptr(),
                                                 None, None, None, None), "bajo_trace_camera")
        h2 = torch.empty_like(hits)
        _lib.check(_lib.load().bajo_trace_camera_stats(ctypes.byref(c), cam.data_ptr(), n, 1024, 1024, 1,
                                                       h2.data_ptr(), stats.data_ptr(), None),
                   "bajo_trace_camera_stats")
        torch.cuda.synchronize()
        assert torch.equal(hits.view(torch.int32), h2.view(torch.int32))
        out[staged] = (hits.view(torch.int32), stats)
    assert torch.equal(out[True][0], out[False][0])
    assert torch.equal(out[True][1], out[False][1])  # same nodes visited, in the same order


def test_unaligned_top_nodes_rejected():
    import ctypes
    v = scenes.random_triangles(100, seed=0)
    tree = bvh.build_triangle_bvh(dev(v), stage_top=True)
    c = tree.c_struct()
    c.top_nodes = tree.top_nodes.data_ptr() + 4
    assert _lib.load().bajo_lbvh_stage_top(ctypes.byref(c), None) == _lib.ERR_INVALID_ARGUMENT
    hits = torch.empty(8, dtype=torch.float32, device="cuda")
    rays = dev(_rays(1, 0))
    assert _lib.load().bajo_trace_rays(ctypes.byref(c), rays.data_ptr(), 1, 1, hits.data_ptr(), None, None, None,
                                       None) == _lib.ERR_INVALID_ARGUMENT
