"""CPU checks of the H-PLOC restatement (no GPU): every leaf sits in its
segment's tree exactly once, parents and children agree, each node's child
boxes are its children's boxes, leaf counts add up, closest hits equal the
LBVH tree's, and the clustered trees have no larger SAH than the LBVH's on
random scenes.  Duplicate Morton codes in segments that do not start at 0
exercise the (code, global position) key order of the climb."""
import numpy as np
import pytest

from bajo_b200 import scenes
from oracle import oracle

LEAF = oracle.LEAF_FLAG
SENT = oracle.SENTINEL


def _box(b, ref):
    if ref & LEAF:
        return b.leaf_bounds.reshape(-1, 6)[b.leaf_ids[ref & 0x7FFFFFFF]]
    nb = b.node_bounds.reshape(-1, 12)[ref]
    return np.concatenate([np.minimum(nb[0:3], nb[6:9]), np.maximum(nb[3:6], nb[9:12])])


def _check(b):
    meta = b.node_meta.reshape(-1, 4)
    nb = b.node_bounds.reshape(-1, 12)
    for s in range(b.seg_offsets.size - 1):
        lo, hi = int(b.seg_offsets[s]), int(b.seg_offsets[s + 1])
        r = int(b.roots[s])
        if hi == lo:
            assert r == SENT
            continue
        seen, stack, internal = [], [r], 0
        while stack:
            x = stack.pop()
            if x & LEAF:
                seen.append(x & 0x7FFFFFFF)
                continue
            internal += 1
            lc = 0
            for k, c in enumerate(meta[x, 1:3]):
                c = int(c)
                parent = int(b.leaf_parent[c & 0x7FFFFFFF]) if c & LEAF else int(meta[c, 0])
                assert parent == x
                assert np.array_equal(nb[x, 6 * k:6 * k + 6].view(np.uint32), _box(b, c).view(np.uint32))
                lc += 1 if c & LEAF else int(b.node_leaf_counts[c])
                stack.append(c)
            assert lc == int(b.node_leaf_counts[x])
        assert sorted(seen) == list(range(lo, hi))
        assert internal == hi - lo - 1
        assert (int(meta[r, 0]) == SENT) if not r & LEAF else (int(b.leaf_parent[r & 0x7FFFFFFF]) == SENT)


def _sah(b):
    r = int(b.roots[0])
    if r & LEAF:
        return 0.0
    def area(x):
        d = (x[3:6] - x[0:3]).astype(np.float64)
        return 2 * (d[0] * d[1] + d[0] * d[2] + d[1] * d[2])
    return sum(area(_box(b, i)) for i in range(b.n_internal)) / area(_box(b, r))


@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 33, 100, 5000])
def test_structure(n):
    _check(oracle.hploc_build(scenes.random_triangles(n, seed=n, spread=0.02)))


def test_segmented_and_duplicate_codes():
    v = scenes.random_triangles(700, seed=9)
    _check(oracle.hploc_build(v, np.array([0, 1, 4, 4, 37, 300, 700], np.uint32)))
    d = scenes.duplicate_centroid_scene()
    dd = np.concatenate([np.asarray(scenes.random_triangles(5, seed=1), np.float32).reshape(-1),
                         np.tile(np.asarray(d, np.float32).reshape(-1), 8)])
    n = dd.size // 9
    _check(oracle.hploc_build(dd, np.array([0, 5, n], np.uint32)))


def test_hits_equal_lbvh_tree():
    v = scenes.random_triangles(20000, seed=5, spread=0.03)
    rng = np.random.default_rng(2)
    m = 20000
    rays = np.zeros((8, m), np.float32)
    rays[0:3] = rng.uniform(-0.5, 1.5, (3, m))
    d = rng.normal(size=(3, m))
    rays[4:7] = d / np.linalg.norm(d, axis=0)
    rays[7] = 1e30
    a = oracle.trace_bvh2(oracle.lbvh_build(v), rays.reshape(-1))
    b = oracle.trace_bvh2(oracle.hploc_build(v), rays.reshape(-1))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("n", [1000, 30000])
def test_sah_no_worse_than_lbvh(n):
    v = scenes.random_triangles(n, seed=3, spread=0.05)
    assert _sah(oracle.hploc_build(v)) <= _sah(oracle.lbvh_build(v)) * 1.0001
