"""GPU parity of the batched build + trace (one segmented LBVH over many
scenes, primary + cosine bounce per pixel) against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402


def test_batched_build_and_trace_match_oracle(oracle):
    from bajo_b200 import batch, camera
    verts, so = scenes.batched_scenes(n_scenes=48, lo=16, hi=3000, seed=3)
    res = batch.build_and_trace(torch.from_numpy(verts).cuda(), so, camera.plain_lbvh_camera(), 24, 16, seed=7)
    torch.cuda.synchronize()
    o = oracle.lbvh_build(verts, so)
    ref = oracle.trace_batch(o, camera.plain_lbvh_camera(), 0, 24, 16, seed=7)
    for got, want in zip(res.outputs(), ref):
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert (ref[1] != oracle.EMPTY).any()


def test_batched_graph_replay_matches_eager(oracle):
    """The CUDA-graph replay of build + trace gives the eager result."""
    from bajo_b200 import batch, camera
    verts, so = scenes.batched_scenes(n_scenes=64, lo=256, hi=4096, seed=5)
    v = torch.from_numpy(verts).cuda()
    eager = batch.build_and_trace(v, so, camera.plain_lbvh_camera(), 32, 32, seed=9)
    g = batch.BatchedGraph(v, so, camera.plain_lbvh_camera(), 32, 32, seed=9)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager.outputs(), g.result.outputs()):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert g.status() == 0


def _h(t, dt):
    return t.cpu().numpy().view(dt)


def test_full_batched_workload_sampled_scenes_match_oracle(oracle):
    """The batched workload at its stated size: 4,096 scenes of 256..65,536
    triangles (log-uniform), 256x256 primary rays plus one cosine bounce per
    pixel, built and traced by one CUDA-graph launch.  64 sampled scenes
    (the smallest and largest among them) have build arrays and hits equal to
    the oracle's build and trace of that scene alone, with the batch's global
    leaf / node numbering and ray indices mapped back; every scene satisfies
    the whole-batch invariants."""
    from bajo_b200 import batch, camera
    W = H = 256
    ppv = W * H
    verts, so = scenes.batched_scenes()  # 4,096 scenes, seed 0
    S = so.size - 1
    assert S == 4096
    cam = camera.plain_lbvh_camera()
    v = torch.from_numpy(verts).cuda()
    g = batch.BatchedGraph(v, so, cam, W, H, seed=7)
    g.replay()
    torch.cuda.synchronize()
    assert g.status() == 0
    t = g.tree
    res = g.result
    so64 = so.astype(np.int64)
    io = _h(t.internal_offsets, np.uint32).astype(np.int64)
    assert np.array_equal(io, np.concatenate([[0], np.cumsum(np.maximum(np.diff(so64) - 1, 0))]))

    # ---- whole-batch invariants (on the device)
    dev_so = torch.from_numpy(so64).cuda()
    seg_of_ray = torch.arange(S, device="cuda").repeat_interleave(ppv)
    size_of_ray = (dev_so[1:] - dev_so[:-1])[seg_of_ray]
    for p in (res.p0, res.p1):
        pl = p.to(torch.int64) & 0xFFFFFFFF  # segment-local triangle index, as the leaf records hold it
        hit = pl != 0xFFFFFFFF
        assert bool(((pl < size_of_ray) | ~hit).all())  # a scene's rays hit only its own triangles
    assert bool((res.p0 != -1).any()) and bool((res.p1 != -1).any())
    assert bool((res.t0[res.p0 != -1] > 0).all())
    assert bool((res.p1[res.p0 == -1] == -1).all())  # no bounce without a primary hit
    seg_of_leaf = torch.arange(S, device="cuda").repeat_interleave(dev_so[1:] - dev_so[:-1])
    ids = t.leaf_ids.to(torch.int64) & 0xFFFFFFFF
    ids = ids[: so64[-1]]
    assert bool(((ids >= dev_so[seg_of_leaf]) & (ids < dev_so[seg_of_leaf + 1])).all())
    assert bool((torch.sort(ids).values == torch.arange(so64[-1], device="cuda")).all())  # a permutation
    roots = _h(t.roots, np.uint32)[:S].astype(np.int64)
    assert np.array_equal(roots, io[:-1])
    counts = _h(t.node_leaf_counts, np.uint32)
    assert np.array_equal(counts[roots], np.diff(so64))  # every root covers its whole scene
    ni = int(io[-1])
    assert bool((t.node_flags[:ni] == 2).all())  # every internal node refit by both children

    # ---- 64 sampled scenes against the oracle, scene by scene
    rng = np.random.default_rng(11)
    sizes = np.diff(so64)
    sample = sorted(set(rng.choice(S, 62, replace=False).tolist()) | {int(sizes.argmin()), int(sizes.argmax())})
    t0, p0, t1, p1 = (x.view(-1) for x in (res.t0, res.p0, res.t1, res.p1))
    meta_all = t.node_meta.view(-1, 4)
    for s in sample:
        a, b = int(so64[s]), int(so64[s + 1])
        n = b - a
        i0, i1 = int(io[s]), int(io[s + 1])
        o = oracle.lbvh_build(verts[9 * a: 9 * b])
        assert np.array_equal(_h(t.leaf_ids[a:b], np.uint32) - a, o.leaf_ids[:n])
        assert np.array_equal(_h(t.morton_codes[a:b], np.uint32), o.morton_codes[:n])
        keys = _h(t.sort_keys[a:b], np.uint64)
        assert np.array_equal(keys & np.uint64(0xFFFFFFFF), o.sort_keys[:n] & np.uint64(0xFFFFFFFF))
        assert np.all((keys >> np.uint64(32)) == s)
        assert np.array_equal(_h(t.leaf_bounds[6 * a: 6 * b], np.uint32), o.leaf_bounds.view(np.uint32)[: 6 * n])
        assert np.array_equal(_h(t.seg_bounds[12 * s: 12 * s + 12], np.uint32), o.seg_bounds.view(np.uint32))
        assert np.array_equal(_h(t.leaf_parent[a:b], np.uint32).astype(np.int64) - i0, o.leaf_parent[:n])
        meta = _h(meta_all[i0:i1], np.uint32).astype(np.int64).copy()
        parent, kids, fence = meta[:, 0], meta[:, 1:3], meta[:, 3]
        parent[parent != 0xFFFFFFFF] -= i0
        leaf = (kids & 0x80000000) != 0
        kids[leaf] = ((kids[leaf] & 0x7FFFFFFF) - a) | 0x80000000
        kids[~leaf] -= i0
        fence -= a
        assert np.array_equal(meta, o.node_meta[: 4 * (n - 1)].reshape(-1, 4).astype(np.int64))
        assert np.array_equal(_h(t.node_bounds[12 * i0: 12 * i1], np.uint32), o.node_bounds.view(np.uint32)[: 12 * (n - 1)])
        assert np.array_equal(_h(t.node_leaf_counts[i0:i1], np.uint32), o.node_leaf_counts[: n - 1])
        rt0, rp0, rt1, rp1 = oracle.trace_batch(o, cam, 0, W, H, seed=7, view_base=s)
        sl = slice(s * ppv, (s + 1) * ppv)
        assert np.array_equal(_h(t0[sl], np.uint32), rt0.view(np.uint32))
        assert np.array_equal(_h(t1[sl], np.uint32), rt1.view(np.uint32))
        for got, want in ((p0, rp0), (p1, rp1)):
            assert np.array_equal(_h(got[sl], np.uint32), want)  # local ids on both sides
        assert (rp0 != oracle.EMPTY).any()
