"""CPU checks of the wide-BVH oracle (no GPU): the collapsed tree covers every
triangle exactly once in blocks of at most max_leaf (1..4), lane boxes are the unions of
what they hold, a node's internal children are consecutive nodes after it and
its leaf blocks consecutive blocks (both in lane order), and leaf lanes pack
the reference's [v0][prim][e1][0][e2][0] record."""
import numpy as np
import pytest

from bajo_b200 import scenes
from oracle import oracle

EMPTY = 0xFFFFFFFF


def _scenes():
    yield "single", scenes.single_triangle_scene(), None
    yield "small", scenes.small_scene(), None
    yield "strip", scenes.strip_scene(5), None
    yield "two_depth", scenes.two_depth_scene(), None
    yield "duplicate", scenes.duplicate_centroid_scene(), None
    yield "degenerate", scenes.degenerate_axis_scene(), None
    yield "grid", scenes.grid_mesh(7, 5), None
    yield "random", scenes.random_triangles(3000, seed=4), None
    v = scenes.random_triangles(700, seed=9)
    yield "segmented", v, np.array([0, 1, 4, 4, 37, 300, 700], np.uint32)


def _check_segment(ow, bvh, verts, s, W, max_leaf=4):
    nb, ne = int(ow.node_offsets[s]), int(ow.node_offsets[s + 1])
    lb, le = int(ow.leaf_offsets[s]), int(ow.leaf_offsets[s + 1])
    i0, i1 = int(bvh.seg_offsets[s]), int(bvh.seg_offsets[s + 1])
    if i1 == i0:
        assert ne == nb and le == lb
        return
    nodes = ow.nodes.reshape(-1, 7, W)
    meta = nodes[:, 6, :].view(np.uint32)
    li = ow.leaf_indices.reshape(-1, W)
    lt = ow.leaf_tris.reshape(-1, 12, W)
    seen = np.zeros(i1 - i0, np.int32)
    v = verts.reshape(-1, 3, 3)
    referenced_nodes, referenced_blocks = [], []

    def lane_box(i, j):
        return nodes[i, 0:3, j], nodes[i, 3:6, j]

    for i in range(nb, ne):
        kids = [nb + (int(m) & 0x03FFFFFF) for m in meta[i] if int(m) != EMPTY and int(m) >> 26 == 0]
        blocks = [lb + (int(m) & 0x03FFFFFF) for m in meta[i] if int(m) != EMPTY and int(m) >> 26 != 0]
        assert kids == list(range(kids[0], kids[0] + len(kids))) if kids else True
        assert blocks == list(range(blocks[0], blocks[0] + len(blocks))) if blocks else True
        for j in range(W):
            m = int(meta[i, j])
            if m == EMPTY:
                assert np.all(nodes[i, 0:3, j] == np.float32(3.4028235e38))
                continue
            cnt, data = m >> 26, m & 0x03FFFFFF
            mn, mx = lane_box(i, j)
            if cnt == 0:
                c = nb + data
                assert nb < c < ne and c > i  # children after their parent
                referenced_nodes.append(c)
                cm = meta[c]
                ok = cm != EMPTY
                assert np.array_equal(mn, nodes[c, 0:3][:, ok].min(axis=1))
                assert np.array_equal(mx, nodes[c, 3:6][:, ok].max(axis=1))
            else:
                assert 1 <= cnt <= max_leaf
                blk = lb + data
                assert lb <= blk < le
                referenced_blocks.append(blk)
                items = li[blk]
                assert np.all(items[:cnt] != EMPTY) and np.all(items[cnt:] == EMPTY)
                tri = v[items[:cnt]]
                assert np.all(tri.min(axis=(1)).min(axis=0) >= mn) and np.all(tri.max(axis=1).max(axis=0) <= mx)
                for k, it in enumerate(items[:cnt]):
                    seen[it - i0] += 1
                    assert np.array_equal(lt[blk, 0:3, k], v[it, 0])
                    assert int(lt[blk, 3, k].view(np.uint32)) == it - i0
                    assert np.array_equal(lt[blk, 4:7, k], v[it, 1] - v[it, 0])
                    assert np.array_equal(lt[blk, 8:11, k], v[it, 2] - v[it, 0])
                    assert lt[blk, 7, k] == 0 and lt[blk, 11, k] == 0
                    assert int(bvh.leaf_ids[ow.leaf_sorted[blk * W + k]]) == it
    assert np.all(seen == 1)
    # every node but the root and every block is referenced exactly once
    assert sorted(referenced_nodes) == list(range(nb + 1, ne))
    assert sorted(referenced_blocks) == list(range(lb, le))
    assert ne - nb <= max(1, i1 - i0 - 1) and le - lb <= i1 - i0


@pytest.mark.parametrize("W,max_leaf", [(4, 4), (8, 4), (4, 1), (8, 2)])
def test_oracle_wide_structure(W, max_leaf):
    for name, verts, seg in _scenes():
        bvh = oracle.lbvh_build(verts, seg)
        ow = oracle.wide_build(bvh, W, max_leaf)
        for s in range(bvh.seg_offsets.size - 1):
            _check_segment(ow, bvh, np.asarray(verts, np.float32), s, W, max_leaf)


def test_wide_nodes_use_the_width():
    bvh = oracle.lbvh_build(scenes.random_triangles(20000, seed=1))
    n4 = int(oracle.wide_build(bvh, 4).node_offsets[-1])
    n8 = int(oracle.wide_build(bvh, 8).node_offsets[-1])
    blocks = int(oracle.wide_build(bvh, 4).leaf_offsets[-1])
    # fat leaves average more than one triangle; wider nodes mean fewer nodes
    assert blocks < 20000 / 1.5 and n8 < n4 < blocks
