"""GPU parity of the wide BVH: the collapsed layout equals the oracle's bit for
bit (nodes, leaf payloads, packed leaf triangles, offsets) for W = 4 and 8,
single and segmented trees; wide closest hits equal the oracle's binary-tree
hits bit for bit for both triangle tests."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import bvh, camera, scenes, wide  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_wide(verts, W, seg=None, max_leaf=4):
    tree = bvh.build_triangle_bvh(dev(np.asarray(verts, np.float32)), seg)
    w = wide.build_wide_bvh(tree, W, max_leaf)
    assert w.status() == 0
    return tree, w


def compare_layout(w, ow, W):
    nn, nb = int(ow.node_offsets[-1]), int(ow.leaf_offsets[-1])
    assert (w.n_nodes, w.n_leaf_blocks) == (nn, nb)
    S = ow.node_offsets.size
    assert np.array_equal(w.node_offsets[:S].cpu().numpy().view(np.uint32), ow.node_offsets)
    assert np.array_equal(w.leaf_offsets[:S].cpu().numpy().view(np.uint32), ow.leaf_offsets)
    assert np.array_equal(w.nodes[:nn * 7 * W].cpu().numpy().view(np.uint32), ow.nodes.view(np.uint32))
    assert np.array_equal(w.leaf_indices[:nb * W].cpu().numpy().view(np.uint32), ow.leaf_indices)
    assert np.array_equal(w.leaf_tris[:nb * 12 * W].cpu().numpy().view(np.uint32), ow.leaf_tris.view(np.uint32))
    assert np.array_equal(w.leaf_sorted[:nb * W].cpu().numpy().view(np.uint32), ow.leaf_sorted)


FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


@pytest.mark.parametrize("W", [4, 8])
@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_layouts_match_oracle(oracle, golden_dir, name, W):
    verts = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))[name + "__verts"]
    _, w = gpu_wide(verts, W)
    compare_layout(w, oracle.wide_build(oracle.lbvh_build(verts), W), W)


@pytest.mark.parametrize("W", [4, 8])
@pytest.mark.parametrize("n", [2, 3, 4, 5, 17, 4096, 65536])
def test_random_layouts_match_oracle(oracle, n, W):
    verts = scenes.random_triangles(n, seed=n)
    _, w = gpu_wide(verts, W)
    compare_layout(w, oracle.wide_build(oracle.lbvh_build(verts), W), W)


@pytest.mark.parametrize("W,max_leaf", [(4, 1), (4, 2), (8, 1)])
def test_small_leaf_layouts_match_oracle(oracle, W, max_leaf):
    for n in (1, 5, 3000):
        verts = scenes.random_triangles(n, seed=n + 11)
        _, w = gpu_wide(verts, W, max_leaf=max_leaf)
        compare_layout(w, oracle.wide_build(oracle.lbvh_build(verts), W, max_leaf), W)


@pytest.mark.parametrize("W", [4, 8])
def test_segmented_layout_matches_oracle(oracle, W):
    verts = scenes.random_triangles(5000, seed=3)
    seg = np.array([0, 1, 4, 4, 5, 37, 900, 4096, 5000], np.uint32)  # includes 1-, 3- and 0-triangle scenes
    _, w = gpu_wide(verts, W, seg)
    compare_layout(w, oracle.wide_build(oracle.lbvh_build(verts, seg), W), W)


def test_batched_layout_is_deterministic(oracle):
    verts, so = scenes.batched_scenes(n_scenes=64, lo=16, hi=20000, seed=2)
    tree, w = gpu_wide(verts, 4, so)
    used = {"nodes": w.n_nodes * 7 * 4, "leaf_tris": w.n_leaf_blocks * 12 * 4, "leaf_indices": w.n_leaf_blocks * 4}
    first = {a: getattr(w, a)[:k].clone().view(torch.int32) for a, k in used.items()}
    w.build()
    for a, k in used.items():  # bitwise over the written prefix (the tail is never written)
        assert torch.equal(first[a], getattr(w, a)[:k].view(torch.int32)), a
    compare_layout(w, oracle.wide_build(oracle.lbvh_build(verts, so), 4), 4)


def _trace(w, rays, mode):
    n = rays.size // 8
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    st = w.launch_rays(dev(rays), hits, n, tri_mode=mode)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return hits.cpu().numpy()


@pytest.mark.parametrize("W,max_leaf", [(4, 4), (8, 4), (4, 1)])
@pytest.mark.parametrize("mode", [0, 1])
def test_wide_hits_equal_binary_hits(oracle, golden_dir, mode, W, max_leaf):
    g = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))
    tg = np.load(os.path.join(golden_dir, "trace_fixtures.npz"))
    for name in FIXTURES:
        verts, rays = g[name + "__verts"], tg[name + "__rays"]
        _, w = gpu_wide(verts, W, max_leaf=max_leaf)
        got = _trace(w, rays, mode)
        ref = oracle.trace_bvh2(oracle.lbvh_build(verts), rays, mode)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), name


@pytest.mark.parametrize("W", [4, 8])
@pytest.mark.parametrize("mode", [0, 1])
def test_wide_random_rays(oracle, mode, W):
    v = scenes.random_triangles(30000, seed=2, spread=0.03)
    _, w = gpu_wide(v, W)
    rng = np.random.default_rng(5)
    n = 200_000
    o = rng.uniform(-0.5, 1.5, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:100, 0] = 0.0
    d[100:200, 1:] = 0.0
    rays = np.zeros((8, n), np.float32)
    rays[0:3] = o.T
    rays[3] = rng.uniform(0.0, 0.1, n)
    rays[4:7] = d.T
    rays[7] = rng.uniform(0.5, 5.0, n)
    rays = rays.reshape(-1)
    got = _trace(w, rays, mode)
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), rays, mode)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("W,max_leaf", [(4, 4), (8, 4), (4, 1)])
def test_wide_camera_plain_workload(oracle, W, max_leaf):
    """65,536 triangles, 1024x1024 camera rays: wide hits = binary hits, and
    the instrumented counts show fewer node visits than the binary tree."""
    v = scenes.random_triangles(65536, seed=0)
    tree, w = gpu_wide(v, W, max_leaf=max_leaf)
    cam = dev(camera.plain_lbvh_camera())
    n = 1024 * 1024
    hw = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    stats = torch.zeros(5 * n, dtype=torch.int32, device="cuda")
    st = w.launch_camera(cam, hw, n, 1024, 1024, d_stats=stats)
    hb = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    tree.launch_camera(cam, hb, n, 1024, 1024)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert torch.equal(hw.view(torch.int32), hb.view(torch.int32))  # misses carry prim 0xFFFFFFFF: compare bits
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), oracle.camera_rays(camera.plain_lbvh_camera(), n, 1024, 1024),
                            oracle.TRI_WATERTIGHT)
    assert np.array_equal(hw.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    s = stats.view(-1, 5).double().mean(0).cpu().numpy()
    print(f"W={W} max_leaf={max_leaf}: {s[0]:.2f} wide nodes, {s[3]:.2f} triangles per ray")
    assert s[0] < 24.0  # the binary tree visits ~24 nodes per ray here
    st = stats.view(-1, 5).cpu().numpy()
    assert np.all(st[:, 2] <= st[:, 3]) and np.all(st[:, 3] <= max_leaf * st[:, 2])  # blocks hold 1..max_leaf
