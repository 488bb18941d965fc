"""CPU checks of the staged-top restatement (no GPU): slots are breadth first,
every staged node's parent is staged before it, staged children are tagged
with their slot and the rest keep their global refs, records carry the node's
own child boxes."""
import numpy as np
import pytest

from bajo_b200 import scenes
from oracle import oracle

FLAG = oracle.TOP_FLAG


@pytest.mark.parametrize("n", [1, 2, 5, 255, 256, 257, 600, 5000])
@pytest.mark.parametrize("k", [1, 7, 256])
def test_stage_top_structure(n, k):
    b = oracle.lbvh_build(scenes.random_triangles(n, seed=n))
    w = oracle.stage_top(b, k)
    count, root = int(w[0]), int(w[1])
    assert root == int(b.roots[0])
    assert count == min(k, max(n - 1, 0))
    rec = w[4:].reshape(k, 16)
    assert np.all(rec[count:] == 0)
    meta = b.node_meta.reshape(-1, 4)
    # walk the staged slots: recover each slot's global node and its depth
    node = {0: root} if count else {}
    depth = {0: 0}
    for s in range(count):
        r = node[s]
        assert np.array_equal(rec[s, :12], b.node_bounds.view(np.uint32).reshape(-1, 12)[r])
        assert rec[s, 14] == 0 and rec[s, 15] == 0
        for j in range(2):
            c, g = int(rec[s, 12 + j]), int(meta[r, 1 + j])
            if c & FLAG and not c & oracle.LEAF_FLAG:
                slot = c & (FLAG - 1)
                assert s < slot < count
                node[slot] = g
                depth[slot] = depth[s] + 1
            else:
                assert c == g
    assert sorted(node) == list(range(count))
    d = [depth[s] for s in range(count)]
    assert d == sorted(d)  # breadth first
    # the staged nodes are the first `count` internal nodes of a breadth-first walk
    order, q = [], [root] if count else []
    while q:
        r = q.pop(0)
        order.append(r)
        q += [int(c) for c in meta[r, 1:3] if not int(c) & oracle.LEAF_FLAG]
    assert [node[s] for s in range(count)] == order[:count]
