"""GPU parity of the H-PLOC build: every segment's tree equals the oracle's
node for node once internal ids are set aside (pre-order canonical form:
leaf positions, leaf counts, both child boxes as bits), parent links agree,
the status is clean, closest hits of rays and camera rays equal the oracle's
bit for bit, and the wide collapse and the CWBVH8 build take H-PLOC trees
unchanged."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import bvh, camera, scenes, wide  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(tree):
    u = lambda t: t.cpu().numpy().view(np.uint32)  # noqa: E731
    return SimpleNamespace(node_meta=u(tree.node_meta), node_bounds=tree.node_bounds.cpu().numpy(),
                           node_leaf_counts=u(tree.node_leaf_counts), roots=u(tree.roots),
                           leaf_parent=u(tree.leaf_parent))


def gpu_hploc(verts, seg=None):
    tree = bvh.build_triangle_bvh(dev(np.asarray(verts, np.float32).reshape(-1)), seg, method="hploc")
    assert tree.workspace.status() == 0
    return tree


def check_against_oracle(oracle, tree, verts, seg=None):
    ref = oracle.hploc_build(verts, seg)
    h = host(tree)
    S = ref.seg_offsets.size - 1
    for s in range(S):
        assert oracle.canonical_tree(h, s) == oracle.canonical_tree(ref, s), s
    meta = h.node_meta.reshape(-1, 4)
    for r in range(int(ref.n_internal)):  # every node's children point back at it
        for c in meta[r, 1:3]:
            c = int(c)
            parent = int(h.leaf_parent[c & 0x7FFFFFFF]) if c & oracle.LEAF_FLAG else int(meta[c, 0])
            assert parent == r
    return ref


FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_trees_match_oracle(oracle, golden_dir, name):
    verts = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))[name + "__verts"]
    check_against_oracle(oracle, gpu_hploc(verts), verts)


@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 33, 257, 4096, 65536, 1 << 20])
def test_random_trees_match_oracle(oracle, n):
    verts = scenes.random_triangles(n, seed=n, spread=0.02)
    check_against_oracle(oracle, gpu_hploc(verts), verts)


def test_segmented_trees_match_oracle(oracle):
    verts = scenes.random_triangles(5000, seed=3)
    seg = np.array([0, 0, 1, 4, 4, 5, 37, 900, 4096, 5000, 5000], np.uint32)
    check_against_oracle(oracle, gpu_hploc(verts, seg), verts, seg)
    d = np.tile(np.asarray(scenes.duplicate_centroid_scene(), np.float32).reshape(-1), 40)
    dup = np.concatenate([np.asarray(scenes.random_triangles(7, seed=1), np.float32).reshape(-1), d])
    seg2 = np.array([0, 7, dup.size // 9], np.uint32)
    check_against_oracle(oracle, gpu_hploc(dup, seg2), dup, seg2)


def test_batched_trees_match_oracle(oracle):
    verts, so = scenes.batched_scenes(n_scenes=48, lo=8, hi=20000, seed=4)
    check_against_oracle(oracle, gpu_hploc(verts, so), verts, so)


def test_rebuild_is_structurally_identical(oracle):
    verts = scenes.random_triangles(200_000, seed=7)
    a = oracle.canonical_tree(host(gpu_hploc(verts)))
    b = oracle.canonical_tree(host(gpu_hploc(verts)))
    assert a == b


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.5, 1.5, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:64, 0] = 0.0
    r = np.zeros((8, n), np.float32)
    r[0:3], r[3], r[4:7], r[7] = o.T, rng.uniform(0.0, 0.1, n), d.T, rng.uniform(0.5, 5.0, n)
    return r.reshape(-1)


@pytest.mark.parametrize("tri_mode", [0, 1])
def test_hits_match_oracle(oracle, tri_mode):
    v = scenes.random_triangles(30000, seed=3, spread=0.03)
    tree = gpu_hploc(v)
    rays = _rays(300_000, 9)
    hits = torch.empty(8 * 300_000, dtype=torch.float32, device="cuda")
    tree.launch_rays(dev(rays), hits, 300_000, tri_mode=tri_mode)
    torch.cuda.synchronize()
    ref = oracle.trace_bvh2(oracle.hploc_build(v), rays, tri_mode)
    assert np.array_equal(hits.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    # the order-free closest hit: the LBVH tree gives the same hits
    assert np.array_equal(ref.view(np.uint32), oracle.trace_bvh2(oracle.lbvh_build(v), rays, tri_mode).view(np.uint32))


def test_camera_hits_match_oracle(oracle):
    v = scenes.random_triangles(65536, seed=0)
    tree = gpu_hploc(v)
    cam = camera.plain_lbvh_camera()
    w = h = 512
    hits = torch.empty(8 * w * h, dtype=torch.float32, device="cuda")
    tree.launch_camera(dev(cam), hits, w * h, w, h)
    torch.cuda.synchronize()
    ref = oracle.trace_bvh2(oracle.hploc_build(v), oracle.camera_rays(cam, w * h, w, h))
    assert np.array_equal(hits.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_wide_and_cwbvh8_take_hploc_trees(oracle):
    v = scenes.random_triangles(20000, seed=11, spread=0.03)
    tree = gpu_hploc(v)
    rays = _rays(100_000, 3)
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), rays, 0)
    w8 = wide.build_wide_bvh(tree, 8, 4)
    assert w8.status() == 0
    hits = torch.empty(8 * 100_000, dtype=torch.float32, device="cuda")
    w8.launch_rays(dev(rays), hits, 100_000, tri_mode=0)
    torch.cuda.synchronize()
    assert np.array_equal(hits.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    cw = wide.build_cwbvh8(tree)
    assert cw.status() == 0
    st = cw.launch_rays(dev(rays), hits, 100_000)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    got = hits.cpu().numpy().reshape(-1, 8)
    same = got[:, 2].view(np.uint32) == ref.reshape(-1, 8)[:, 2].view(np.uint32)
    assert same.mean() > 0.999
