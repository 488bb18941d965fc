"""CPU checks of the CWBVH8 restatement (no GPU).

Known answers from the reference's own tests
(test/bvh/gpu/test_segmented_empty.mojo:30-47,149-177,238-255): a triangle at
z = 6 is hit at t = 6 by a ray along +z; empty segments take no nodes; two
segments of 5 and 17 triangles take exactly consecutive storage.  Structure:
every triangle is referenced exactly once with the reference's
[e1][0][e2][0][v0][prim] record, a node's internal children are consecutive
nodes after it, each lane's dequantized box contains the uncompressed lane
box and is at most one quantum larger per side, and the octant slots follow
the greedy rule.  Hits equal the binary tree's (golden-pinned) hits."""
import numpy as np
import pytest

from bajo_b200 import scenes
from oracle import oracle

EMPTY = 0xFFFFFFFF


def _tri_at(z, count=1):
    v = []
    for i in range(count):
        x = 3.0 * i
        v += [[x - 1.0, -1.0, z], [x + 1.0, -1.0, z], [x, 1.0, z]]
    return np.array(v, np.float32).reshape(-1, 9)


def _ray_soa(o, d, tmin=0.0, tmax=3.4028235e38):
    o = np.atleast_2d(np.asarray(o, np.float32))
    d = np.atleast_2d(np.asarray(d, np.float32))
    r = np.zeros((8, o.shape[0]), np.float32)
    r[0:3], r[3], r[4:7], r[7] = o.T, tmin, d.T, tmax
    return r.reshape(-1)


def decode(cw, s=0):
    """Per node of segment s: (p, scale, imask, child_base, tri_base, bytes[8],
    qlo[8][3], qhi[8][3])."""
    nb, ne = int(cw.node_offsets[s]), int(cw.node_offsets[s + 1])
    w = cw.nodes.view(np.uint32).reshape(-1, 20)
    f = cw.nodes.reshape(-1, 20)
    out = []
    for i in range(nb, ne):
        e = [(int(w[i, 3]) >> (8 * k)) & 0xFF for k in range(3)]
        scale = np.array([np.uint32(x << 23).view(np.float32) for x in e], np.float32)
        by = [(int(w[i, 6 + j // 4]) >> (8 * (j % 4))) & 0xFF for j in range(8)]
        q = np.array([[(int(w[i, 8 + 2 * pl + j // 4]) >> (8 * (j % 4))) & 0xFF for pl in range(6)]
                      for j in range(8)], np.float32)
        out.append((f[i, 0:3].copy(), scale, int(w[i, 3]) >> 24, int(w[i, 4]), int(w[i, 5]), by, q[:, 0:3],
                    q[:, 3:6]))
    return out


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


def _check_segment(cw, bvh, verts, s):
    nb, ne = int(cw.node_offsets[s]), int(cw.node_offsets[s + 1])
    i0, i1 = int(bvh.seg_offsets[s]), int(bvh.seg_offsets[s + 1])
    if i1 == i0:
        assert ne == nb
        return
    v = verts.reshape(-1, 3, 3)
    tris = cw.triangles.reshape(-1, 12)
    wide = cw.wide_nodes.reshape(-1, 7, 8)
    seen = np.zeros(i1 - i0, np.int32)
    children = []
    for k, (p, sc, imask, cb, tb, by, qlo, qhi) in enumerate(decode(cw, s)):
        i = nb + k
        meta = wide[i, 6].view(np.uint32)
        lo = p[None, :] + qlo * sc[None, :]
        hi = p[None, :] + qhi * sc[None, :]
        n_int, off = 0, 0
        for j in range(8):
            m = int(meta[j])
            if m == EMPTY:
                assert by[j] == 0
                continue
            # conservative and at most one quantum loose per side
            assert np.all(lo[j] <= wide[i, 0:3, j]) and np.all(hi[j] >= wide[i, 3:6, j])
            assert np.all(lo[j] + sc >= wide[i, 0:3, j]) or np.any(qlo[j] == 0)
            cnt = m >> 26
            if cnt == 0:
                assert imask >> j & 1 and by[j] == 0x20 | (24 + j)
                assert (m & 0x03FFFFFF) == cb + n_int
                children.append(nb + cb + n_int)
                assert cb + n_int > k
                n_int += 1
            else:
                assert not imask >> j & 1
                assert 1 <= cnt <= 3 and by[j] == (((1 << cnt) - 1) << 5 | off)
                for t in range(cnt):
                    rec = tris[i0 + tb + off + t]
                    prim = int(rec[11:12].view(np.uint32)[0])
                    it = i0 + prim
                    seen[prim] += 1
                    assert np.array_equal(rec[8:11], v[it, 0])
                    assert np.array_equal(rec[0:3], v[it, 1] - v[it, 0])
                    assert np.array_equal(rec[4:7], v[it, 2] - v[it, 0])
                    assert rec[3] == 0 and rec[7] == 0
                off += cnt
    assert np.all(seen == 1)
    assert sorted(children) == list(range(nb + 1, ne))


def test_structure():
    for name, verts, seg in _scenes():
        verts = np.asarray(verts, np.float32)
        bvh = oracle.lbvh_build(verts, seg)
        cw = oracle.cwbvh8_build(bvh)
        for s in range(bvh.seg_offsets.size - 1):
            _check_segment(cw, bvh, verts, s)


def _greedy_ok(p_box, boxes, lanes):
    """The (candidate, slot) pairs, replayed in increasing cost, are each the
    cheapest pair left at their turn."""
    pc = (p_box[0] + p_box[1]) * np.float32(0.5)
    sgn = np.array([[-1 if s & 4 else 1, -1 if s & 2 else 1, -1 if s & 1 else 1] for s in range(8)], np.float32)
    cc = (boxes[:, 0] + boxes[:, 1]) * np.float32(0.5) - pc
    cost = np.array([[np.float32(np.float32(c[0] * g[0] + c[1] * g[1]) + c[2] * g[2]) for g in sgn] for c in cc])
    pairs = sorted(zip(range(len(lanes)), lanes), key=lambda kv: cost[kv[0], kv[1]])
    free_c, free_s = set(range(len(lanes))), set(range(8))
    for c, s in pairs:
        best = min(cost[a, b] for a in free_c for b in free_s)
        if cost[c, s] > best:
            return False
        free_c.discard(c)
        free_s.discard(s)
    return True


@pytest.mark.parametrize("n", [50, 3000])
def test_octant_slots_are_greedy(n):
    bvh = oracle.lbvh_build(scenes.random_triangles(n, seed=n, spread=0.05))
    cw = oracle.cwbvh8_build(bvh)
    wide = cw.wide_nodes.reshape(-1, 7, 8)
    for i in range(int(cw.node_offsets[1])):
        meta = wide[i, 6].view(np.uint32)
        lanes = [j for j in range(8) if int(meta[j]) != EMPTY]
        if len(lanes) < 2:
            continue
        boxes = np.stack([np.stack([wide[i, 0:3, j], wide[i, 3:6, j]]) for j in lanes])
        p_box = np.stack([boxes[:, 0].min(axis=0), boxes[:, 1].max(axis=0)])
        assert _greedy_ok(p_box, boxes, lanes), i


def test_single_triangle_known_answer():
    # test_triangle_hploc_cwbvh8_empty_segments_trace: t = 6 along +z
    verts = _tri_at(6.0)
    cw = oracle.cwbvh8_build(oracle.lbvh_build(verts))
    h = oracle.trace_cwbvh8(cw, _ray_soa([0, 0, 0], [0, 0, 1])).reshape(-1, 8)
    assert abs(h[0, 7] - 6.0) < 1e-5 and int(h[0, 2:3].view(np.uint32)[0]) == 0
    occ = oracle.trace_cwbvh8(cw, _ray_soa([0, 0, 0], [0, 0, 1]), any_hit=True).reshape(-1, 8)
    assert occ[0, 7] == 0.0 and int(occ[0, 2:3].view(np.uint32)[0]) == EMPTY
    miss = oracle.trace_cwbvh8(cw, _ray_soa([0, 0, 0], [0, 0, -1])).reshape(-1, 8)
    assert int(miss[0, 2:3].view(np.uint32)[0]) == EMPTY and miss[0, 7] == np.float32(3.4028235e38)


def test_empty_and_consecutive_segments():
    # test_nonempty_segments_use_exact_consecutive_storage (5 and 17 triangles)
    # and empty segments around a single triangle
    verts = np.concatenate([_tri_at(4.0, 5), _tri_at(8.0, 17), _tri_at(6.0)])
    seg = np.array([0, 0, 5, 5, 22, 23, 23], np.uint32)
    bvh = oracle.lbvh_build(verts, seg)
    cw = oracle.cwbvh8_build(bvh)
    no = cw.node_offsets.astype(np.int64)
    assert no[1] == no[0] and no[3] == no[2] and no[6] == no[5]
    assert np.all(np.diff(no) >= 0) and cw.triangles.size == 23 * 12
    for s in range(6):
        _check_segment(cw, bvh, verts, s)
    # segment 4 (the triangle at z = 6), traced through its own nodes and records
    sub = oracle.OracleCwbvh8(cw.wide_nodes, cw.nodes[no[4] * 20:], cw.triangles[22 * 12:],
                              np.array([0, no[5] - no[4]], np.uint32))
    h = oracle.trace_cwbvh8(sub, _ray_soa([0, 0, 0], [0, 0, 1])).reshape(-1, 8)
    assert abs(h[0, 7] - 6.0) < 1e-5


def _rays(n, seed, lo=-0.5, hi=1.5):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:16, 0] = 0.0
    r = np.zeros((8, n), np.float32)
    r[0:3], r[3], r[4:7], r[7] = o.T, 1e-4, d.T, 1e30
    return r.reshape(-1)


@pytest.mark.parametrize("n_tris", [1, 9, 300, 20000])
def test_hits_equal_binary_tree(n_tris):
    v = scenes.random_triangles(n_tris, seed=n_tris, spread=0.05)
    bvh = oracle.lbvh_build(v)
    cw = oracle.cwbvh8_build(bvh)
    rays = _rays(20000, 3)
    h, err = oracle.trace_cwbvh8(cw, rays, with_errors=True)
    ref = oracle.trace_bvh2(bvh, rays, 0).reshape(-1, 8)
    h = h.reshape(-1, 8)
    assert not err.any()
    same = h[:, 2].view(np.uint32) == ref[:, 2].view(np.uint32)
    assert same.mean() >= 0.999
    hit = same & (ref[:, 2].view(np.uint32) != EMPTY)
    np.testing.assert_allclose(h[hit, 7], ref[hit, 7], rtol=1e-6)
    occ = oracle.trace_cwbvh8(cw, rays, any_hit=True).reshape(-1, 8)
    assert np.array_equal(occ[:, 7] == 0.0, h[:, 2].view(np.uint32) != EMPTY)
