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
