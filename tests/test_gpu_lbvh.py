"""GPU parity of the LBVH build against the oracle: every output array is
bit-identical (bounds, keys, sorted ids, topology, refit boxes, flags)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402


def build_gpu(verts: np.ndarray, seg_offsets=None):
    from bajo_b200 import bvh
    v = torch.from_numpy(np.ascontiguousarray(verts, np.float32)).cuda()
    b = bvh.build_triangle_bvh(v, seg_offsets)
    torch.cuda.synchronize()
    assert b.workspace.status() == 0
    return b


def h(t, dtype):
    return t.cpu().numpy().view(dtype)


def assert_same_build(b, o):
    n = o.n_leaves
    ni = o.n_internal
    S = o.seg_offsets.size - 1
    assert np.array_equal(h(b.internal_offsets, np.uint32), o.internal_offsets)
    assert np.array_equal(h(b.leaf_bounds, np.uint32)[: 6 * n], o.leaf_bounds.view(np.uint32)[: 6 * n])
    assert np.array_equal(h(b.seg_bounds, np.uint32)[: 12 * S], o.seg_bounds.view(np.uint32))
    assert np.array_equal(h(b.sort_keys, np.uint64)[:n], o.sort_keys[:n])
    assert np.array_equal(h(b.leaf_ids, np.uint32)[:n], o.leaf_ids[:n])
    assert np.array_equal(h(b.morton_codes, np.uint32)[:n], o.morton_codes[:n])
    assert np.array_equal(h(b.roots, np.uint32)[:S], o.roots)
    assert np.array_equal(h(b.leaf_parent, np.uint32)[:n], o.leaf_parent[:n])
    if ni:
        assert np.array_equal(h(b.node_meta, np.uint32)[: 4 * ni], o.node_meta[: 4 * ni])
        assert np.array_equal(h(b.node_leaf_counts, np.uint32)[:ni], o.node_leaf_counts[:ni])
        assert np.array_equal(h(b.node_flags, np.uint32)[:ni], o.node_flags[:ni])
        assert np.array_equal(h(b.node_bounds, np.uint32)[: 12 * ni], o.node_bounds.view(np.uint32)[: 12 * ni])
    # packed triangle records: [v0, prim | v1, 0 | v2, 0] in sorted order
    tris = h(b.leaf_tris, np.float32)[: 12 * n].reshape(-1, 12)
    ids = o.leaf_ids[:n]
    v = o.verts.reshape(-1, 9)[ids]
    assert np.array_equal(tris[:, [0, 1, 2, 4, 5, 6, 8, 9, 10]].view(np.uint32), v.view(np.uint32))
    starts = o.seg_offsets[np.searchsorted(o.seg_offsets, np.arange(n), side="right") - 1]
    assert np.array_equal(tris[:, 3].view(np.uint32), ids - starts)


FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_scenes_match_oracle_and_golden(oracle, golden_dir, name):
    g = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))
    verts = g[name + "__verts"]
    b = build_gpu(verts)
    o = oracle.lbvh_build(verts)
    assert_same_build(b, o)
    n = o.n_leaves
    assert np.array_equal(h(b.leaf_ids, np.uint32)[:n], g[name + "__leaf_ids"])
    if n > 1:
        assert np.array_equal(h(b.node_meta, np.uint32)[: 4 * (n - 1)], g[name + "__node_meta"][: 4 * (n - 1)])


@pytest.mark.parametrize("n", [2, 3, 255, 256, 257, 5632, 65536, 1 << 17, (1 << 17) + 1, 1 << 20])
def test_random_scenes_match_oracle(oracle, n):
    v = scenes.random_triangles(n, seed=n)
    assert_same_build(build_gpu(v), oracle.lbvh_build(v))


def test_plain_lbvh_workload_validators(oracle):
    """65,536 triangles, seed 0: validators of bajo/bvh/gpu/validate.mojo."""
    from bajo_b200.bvh import validate_topology, validate_refit_bounds
    v = scenes.random_triangles(65536, seed=0)
    b = build_gpu(v)
    t = validate_topology(h(b.node_meta, np.uint32), h(b.leaf_parent, np.uint32), 65536)
    assert t.ok and t.root_count == 1 and t.root_idx == 0
    lo, hi = scenes.bounds_of(v)
    r = validate_refit_bounds(h(b.node_bounds, np.float32), h(b.node_flags, np.uint32), h(b.node_meta, np.uint32),
                              65536, lo, hi)
    assert r.ok and r.diff == 0.0


# totals below and above the bottom-up hierarchy size limit (2^17 triangles)
@pytest.mark.parametrize("counts", [[5, 1, 0, 300, 2, 77], [1000] * 7, [0, 0, 3], [1], [70000, 3, 9000],
                                    [70000, 1, 0, 70000, 513]])
def test_segmented_build_matches_oracle(oracle, counts):
    parts = [scenes.random_triangles(c, seed=100 + i) for i, c in enumerate(counts)]
    so = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    verts = np.concatenate(parts) if sum(counts) else np.zeros(0, np.float32)
    b = build_gpu(verts, so)
    assert_same_build(b, oracle.lbvh_build(verts, so))


def test_many_segments(oracle):
    rng = np.random.default_rng(4)
    counts = np.exp(rng.uniform(np.log(1), np.log(400), size=600)).astype(np.int64)
    parts = [scenes.random_triangles(int(c), seed=i) for i, c in enumerate(counts)]
    so = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    verts = np.concatenate(parts)
    assert_same_build(build_gpu(verts, so), oracle.lbvh_build(verts, so))


def test_rebuild_reuses_buffers(oracle):
    """A second build into the same buffers and workspace gives the same tree."""
    from bajo_b200 import bvh
    v = scenes.random_triangles(20000, seed=3)
    d = torch.from_numpy(v).cuda()
    b = bvh.build_triangle_bvh(d)
    b2 = bvh.build_triangle_bvh(d, workspace=b.workspace, out=b)
    torch.cuda.synchronize()
    assert b2 is b
    assert_same_build(b2, oracle.lbvh_build(v))
