"""CPU tests of the oracle against the reference's known answers and the
independent golden fixtures (tests/golden/make_golden.py).  No GPU."""
import hashlib
import json
import os

import numpy as np
import pytest

from bajo_b200 import scenes


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ---------------------------------------------------------------- Morton KATs
def test_morton_kats(oracle, golden_dir):
    """test/core/test_morton.mojo:13-87."""
    k = json.load(open(os.path.join(golden_dir, "morton_kats.json")))
    for v, e in k["expand_bits_3d"]:
        assert oracle.expand_bits_3d(v) == e
    for x, y, z, e in k["morton3"]:
        assert oracle.morton3(x, y, z) == e
    for ca, ia, cb, ib, e in k["common_prefix"]:
        assert oracle.morton_common_prefix(ca, ia, cb, ib) == e


def test_morton_clamps_out_of_range(oracle):
    assert oracle.morton3(-0.5, 0.0, 0.0) == 0
    assert oracle.morton3(2.0, 2.0, 2.0) == (1 << 30) - 1
    assert oracle.morton3(1.0 - 1e-7, 0.0, 0.0) == oracle.expand_bits_3d(1023)


# ---------------------------------------------------------------- sort KATs
def test_sort_kat_histogram_and_perm(oracle, golden_dir):
    """test/sort/test_onesweep.mojo:18-71 keys; stable order vs Python sorted."""
    k = json.load(open(os.path.join(golden_dir, "sort_kats.json")))
    n = k["hist_u32"]["n"]
    i = np.arange(n, dtype=np.uint64)
    keys = (((i * 13) ^ (i << 16) ^ (i >> 3)) & 0xFFFFFFFF).astype(np.uint32)
    for b in range(4):
        h = np.bincount((keys >> (8 * b)) & 255, minlength=256)
        assert h.tolist() == k["hist_u32"]["hist"][b]
    sk, sv = oracle.sort_pairs(keys, np.arange(n, dtype=np.uint32))
    assert _sha(sv.astype("<u4")) == k["hist_u32"]["perm_sha256"]
    assert np.all(sk[1:] >= sk[:-1])


def test_sort_kat_single_pass(oracle, golden_dir):
    """test/sort/test_onesweep.mojo:105-207: one binning pass == stable counting sort."""
    k = json.load(open(os.path.join(golden_dir, "sort_kats.json")))["pass_u32"]
    n = k["n"]
    i = np.arange(n, dtype=np.uint64)
    keys = (((i * 17) ^ (i << 13) ^ (i >> 5)) & 0xFFFFFFFF).astype(np.uint32)
    _, v = oracle.sort_pairs(keys, np.arange(n, dtype=np.uint32), 0, 8)
    assert _sha(v.astype("<u4")) == k["perm_sha256"]
    _, v = oracle.sort_pairs(keys, np.arange(n, dtype=np.uint32))
    assert _sha(v.astype("<u4")) == k["full_perm_sha256"]


def composite_keys(n):
    i = np.arange(n, dtype=np.uint64)
    seg = (i * 7) % 19
    mort = ((i * 2654435761) & 0xFFFFFFFF) ^ ((i << 11) & 0xFFFFFFFF) ^ (i >> 3)
    return ((seg << 32) | (mort & 0xFFFFFFFF)).astype(np.uint64)


def test_sort_kat_composite_u64(oracle, golden_dir):
    """test/sort/test_radix_sort.mojo:316-344 (u64 composite keys, N=10,003)."""
    k = json.load(open(os.path.join(golden_dir, "sort_kats.json")))["composite_u64"]
    keys = composite_keys(k["n"])
    sk, sv = oracle.sort_pairs(keys, np.arange(k["n"], dtype=np.uint32))
    assert _sha(sv.astype("<u4")) == k["perm_sha256"]
    assert np.array_equal(sk, keys[sv])


@pytest.mark.parametrize("n", [0, 1, 2, 7, 1000, 4097])
def test_sort_matches_numpy_stable(oracle, n):
    rng = np.random.default_rng(n)
    for dt, bits in ((np.uint32, 32), (np.uint64, 64)):
        keys = rng.integers(0, 50, size=n).astype(dt) << dt(bits - 8)  # many equal keys
        k, v = oracle.sort_pairs(keys, np.arange(n, dtype=np.uint32))
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(v, order.astype(np.uint32))
        assert np.array_equal(oracle.sort_keys(keys), np.sort(keys))


# ---------------------------------------------------------------- LBVH fixtures
FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


@pytest.fixture(scope="module")
def lbvh_golden(golden_dir):
    return np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_lbvh_matches_golden(oracle, lbvh_golden, name):
    g = {k.split("__", 1)[1]: lbvh_golden[k] for k in lbvh_golden.files if k.startswith(name + "__")}
    b = oracle.lbvh_build(g["verts"])
    n = b.n_leaves
    ni = max(n - 1, 0)
    assert np.array_equal(b.leaf_bounds[: 6 * n].view(np.uint32), g["leaf_bounds"].view(np.uint32))
    assert np.array_equal(b.seg_bounds.view(np.uint32), g["seg_bounds"].view(np.uint32))
    assert np.array_equal(b.leaf_ids[:n], g["leaf_ids"])
    assert np.array_equal(b.morton_codes[:n], g["morton_codes"])
    assert np.array_equal(b.leaf_parent[:n], g["leaf_parent"])
    if ni:
        assert np.array_equal(b.node_meta[: 4 * ni], g["node_meta"][: 4 * ni])
        assert np.array_equal(b.node_leaf_counts[:ni], g["node_leaf_counts"][:ni])
        assert np.array_equal(b.node_bounds[: 12 * ni].view(np.uint32), g["node_bounds"][: 12 * ni].view(np.uint32))
        assert np.all(b.node_flags[:ni] == 2)


@pytest.mark.parametrize("n", [2, 3, 100, 65536])
def test_topology_bottom_up_equals_top_down(oracle, n):
    v = scenes.random_triangles(n, seed=n)
    b = oracle.lbvh_build(v)
    a = oracle.topology(b.morton_codes[:n], b.seg_offsets)
    c = oracle.topology(b.morton_codes[:n], b.seg_offsets, topdown=True)
    for x, y in zip(a, c):
        assert np.array_equal(x, y)


def test_validators_on_oracle_tree(oracle):
    from bajo_b200.bvh import validate_topology, validate_refit_bounds
    v = scenes.random_triangles(5000, seed=1)
    b = oracle.lbvh_build(v)
    t = validate_topology(b.node_meta, b.leaf_parent, b.n_leaves)
    assert t.ok and t.root_count == 1
    lo, hi = scenes.bounds_of(v)
    r = validate_refit_bounds(b.node_bounds, b.node_flags, b.node_meta, b.n_leaves, lo, hi)
    assert r.ok and r.diff == 0.0


def test_validators_catch_planted_errors(oracle):
    """A mistake planted in the oracle's output must be caught."""
    from bajo_b200.bvh import validate_topology, validate_refit_bounds
    v = scenes.random_triangles(300, seed=2)
    b = oracle.lbvh_build(v)
    meta = b.node_meta.copy()
    meta[4 * 5 + 1] = meta[4 * 6 + 1]  # duplicate a child link
    assert not validate_topology(meta, b.leaf_parent, b.n_leaves).ok
    flags = b.node_flags.copy()
    flags[3] = 1
    lo, hi = scenes.bounds_of(v)
    assert not validate_refit_bounds(b.node_bounds, flags, b.node_meta, b.n_leaves, lo, hi).ok


def test_segmented_build_equals_independent_builds(oracle):
    """Each segment of a batched build is the tree of that scene alone
    (segmented LBVH, bajo/bvh/gpu/builder/lbvh.mojo:30-62,235-329)."""
    parts = [scenes.random_triangles(n, seed=10 + n) for n in (5, 1, 0, 300, 2, 77)]
    counts = [p.size // 9 for p in parts]
    so = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    b = oracle.lbvh_build(np.concatenate(parts), so)
    for s, p in enumerate(parts):
        n = counts[s]
        lo, hi = so[s], so[s + 1]
        if n == 0:
            assert b.roots[s] == oracle.SENTINEL
            continue
        single = oracle.lbvh_build(p)
        assert np.array_equal(b.leaf_ids[lo:hi] - lo, single.leaf_ids[:n])
        assert np.array_equal(b.morton_codes[lo:hi], single.morton_codes[:n])
        if n == 1:
            assert b.roots[s] == (oracle.LEAF_FLAG | lo)
            continue
        ib = b.internal_offsets[s]
        m = b.node_meta.reshape(-1, 4)[ib: ib + n - 1].astype(np.int64)
        ms = single.node_meta.reshape(-1, 4)[: n - 1].astype(np.int64)
        for col in (1, 2):
            leaf = (m[:, col] & oracle.LEAF_FLAG) != 0
            rel = np.where(leaf, (m[:, col] & 0x7FFFFFFF) - lo + oracle.LEAF_FLAG, m[:, col] - ib)
            assert np.array_equal(rel, ms[:, col])
        assert np.array_equal(b.node_bounds.reshape(-1, 12)[ib: ib + n - 1].view(np.uint32),
                              single.node_bounds.reshape(-1, 12)[: n - 1].view(np.uint32))


# ---------------------------------------------------------------- traversal
@pytest.fixture(scope="module")
def trace_golden(golden_dir):
    return np.load(os.path.join(golden_dir, "trace_fixtures.npz"))


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_trace_matches_float64_bruteforce(oracle, lbvh_golden, trace_golden, name, mode):
    verts = lbvh_golden[name + "__verts"]
    rays = trace_golden[name + "__rays"]
    robust = trace_golden[name + "__robust"]
    b = oracle.lbvh_build(verts)
    h = oracle.trace_bvh2(b, rays, mode)
    prim = oracle.hits_prim(h)
    t = oracle.hits_t(h)
    gp, gt = trace_golden[name + "__prim"], trace_golden[name + "__t"]
    assert np.array_equal(prim[robust], gp[robust])
    hit = robust & (gp != oracle.EMPTY)
    assert np.all(np.abs(t[hit] - gt[hit]) <= 1e-6 * np.abs(gt[hit]) + 1e-7)


@pytest.mark.parametrize("mode", [0, 1])
def test_bvh_traversal_equals_bruteforce(oracle, mode):
    v = scenes.random_triangles(3000, seed=5, spread=0.05)
    b = oracle.lbvh_build(v)
    cam = oracle.camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, -0.5], [0, 1, 0], 60.0)
    rays = oracle.camera_rays(cam, 64 * 48, 64, 48)
    h1 = oracle.trace_bvh2(b, rays, mode)
    h2 = oracle.trace_brute(v, rays, mode)
    assert np.array_equal(h1.view(np.uint32), h2.view(np.uint32))


def test_watertight_closes_shared_edges(oracle):
    """Rays through the shared vertices / edges of a grid mesh always hit
    (watertight); ties go to the lowest primitive id."""
    v = scenes.grid_mesh(4, 4, z=0.5)
    xs = np.linspace(0.0, 1.0, 5, dtype=np.float32)
    pts = [(x, y) for x in xs[1:-1] for y in xs[1:-1]]  # interior vertices
    pts += [(x + 0.125, y) for x in xs[:-1] for y in xs[1:-1]]  # horizontal edges
    n = len(pts)
    rays = np.zeros((8, n), np.float32)
    for i, (x, y) in enumerate(pts):
        rays[:, i] = [x, y, -1.0, 0.0, 0.0, 0.0, 1.0, np.finfo(np.float32).max]
    rays = rays.reshape(-1)
    b = oracle.lbvh_build(v)
    h = oracle.trace_bvh2(b, rays, oracle.TRI_WATERTIGHT)
    prim = oracle.hits_prim(h)
    assert np.all(prim != oracle.EMPTY)
    assert np.allclose(oracle.hits_t(h), 1.5)
    brute = oracle.trace_brute(v, rays, oracle.TRI_WATERTIGHT)
    assert np.array_equal(oracle.hits_prim(brute), prim)


def test_cpu_baseline_builder_traces_like_oracle(oracle):
    v = scenes.random_triangles(20000, seed=9)
    cb = oracle.CpuLbvh(v, threads=4)
    assert cb.build() == 2 * 20000 - 1
    b = oracle.lbvh_build(v)
    cam = oracle.camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, -0.5], [0, 1, 0], 60.0)
    rays = oracle.camera_rays(cam, 128 * 128, 128, 128)
    for mode in (0, 1):
        a, c = oracle.trace_bvh2(b, rays, mode), cb.trace(rays, mode)
        assert np.array_equal(oracle.hits_prim(a), oracle.hits_prim(c))
        assert np.array_equal(oracle.hits_t(a).view(np.uint32), oracle.hits_t(c).view(np.uint32))


def test_cpu_baseline_builder_same_tree_on_any_thread_count(oracle):
    """The timed CPU builder's node ids come from per-task ranges assigned in
    frontier order, so the whole node array is the same at every thread count
    (and equal to the serial run of the reference's shared-counter order)."""
    v = scenes.random_triangles(50000, seed=3)
    ref = oracle.CpuLbvh(v, threads=1)
    ref.build()
    for threads in (2, 3, 8, 16):
        cb = oracle.CpuLbvh(v, threads=threads)
        for _ in range(3):  # repeated builds reuse the builder's scratch
            assert cb.build() == 2 * 50000 - 1
            assert cb.nodes.tobytes() == ref.nodes.tobytes()
            assert np.array_equal(cb.items, ref.items)


def test_inline_min_max_match_libm(oracle):
    """bo_fminf / bo_fmaxf (branch-free min / max used across the oracle)
    return libm's fminf / fmaxf bits on signed zeros, infinities, quiet NaNs,
    subnormals and random pairs."""
    import ctypes
    f = oracle.lib().bo_minmax_selftest
    f.restype, f.argtypes = ctypes.c_uint32, [ctypes.c_uint32, ctypes.c_uint64]
    assert f(1 << 20, 11) == 0
