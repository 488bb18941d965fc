"""The path tracer through the compressed 8-wide tree (the reference's
default triangle policy, GPU_RT_BVH_CWBVH8_*, bajo/rt/gpu/prepared_scene.mojo:
29-33,52-53): images bit-identical to the oracle's renderer walking the same
CWBVH8 tree (its own Moller-Trumbore test and first-visited tie rule), for
PATH / NEE / MIS, metal and glass, and the 1.31M-triangle workload; and within
the plain renderer's noise of the binary-tree image."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402


def _oracle_cw(oracle, sc, policy):
    t = oracle.hploc_build(sc.vertices) if policy == "cwbvh8_hploc" else oracle.lbvh_build(sc.vertices)
    return oracle.cwbvh8_build(t)


@pytest.mark.parametrize("policy", ["cwbvh8", "cwbvh8_hploc"])
@pytest.mark.parametrize("algorithm", [0, 3, 4])
def test_cwbvh8_render_matches_oracle(oracle, policy, algorithm):
    from bajo_b200 import rt
    sc = scenes.small_rt_scene()
    gsc = rt.GpuRtTriangleScene(sc, bvh_policy=policy)
    w, h, spp = 48, 27, 4
    settings = rt.RenderSettings(w, h, spp, rng_seed=2026, max_depth=8)
    ws = rt.RenderWorkspace(settings, algorithm)
    img = rt.render_gpu_triangles(settings, sc.camera, gsc, algorithm, workspace=ws)
    torch.cuda.synchronize()
    assert ws.status() == 0 and gsc.cwbvh8.status() == 0
    ref = oracle.render(sc, sc.camera, w, h, spp, max_depth=8, seed=2026, algorithm=algorithm,
                        cwbvh8=_oracle_cw(oracle, sc, policy))
    got = img.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert got.mean() > 0.05


@pytest.mark.parametrize("algorithm", [0, 4])
def test_cwbvh8_materials_render_matches_oracle(oracle, algorithm):
    from bajo_b200 import rt
    sc = scenes.materials_in_box(n_spheres=8, subdivisions=2)
    gsc = rt.GpuRtTriangleScene(sc, bvh_policy="cwbvh8")
    w, h, spp = 40, 24, 8
    settings = rt.RenderSettings(w, h, spp, rng_seed=404, max_depth=12)
    img = rt.render_gpu_triangles(settings, sc.camera, gsc, algorithm)
    torch.cuda.synchronize()
    ref = oracle.render(sc, sc.camera, w, h, spp, max_depth=12, seed=404, algorithm=algorithm,
                        cwbvh8=_oracle_cw(oracle, sc, "cwbvh8"))
    assert np.array_equal(img.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_cwbvh8_large_scene_matches_oracle(oracle):
    from bajo_b200 import rt
    sc = scenes.spheres_in_box()
    gsc = rt.GpuRtTriangleScene(sc, bvh_policy="cwbvh8")
    w, h, spp = 32, 18, 2
    img = rt.render_gpu_triangles(rt.RenderSettings(w, h, spp), sc.camera, gsc, rt.MIS)
    torch.cuda.synchronize()
    ref = oracle.render(sc, sc.camera, w, h, spp, algorithm=4, cwbvh8=_oracle_cw(oracle, sc, "cwbvh8"))
    assert np.array_equal(img.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_cwbvh8_and_binary_images_agree_statistically():
    """Same scene and seed through both trees: the hit rules differ only on
    edges and ties, so the images differ by far less than their noise."""
    from bajo_b200 import rt
    sc = scenes.small_rt_scene()
    st = rt.RenderSettings(64, 36, 64, rng_seed=9, max_depth=8)
    a = rt.render_gpu_triangles(st, sc.camera, rt.GpuRtTriangleScene(sc, bvh_policy="lbvh"), rt.MIS).double()
    b = rt.render_gpu_triangles(st, sc.camera, rt.GpuRtTriangleScene(sc, bvh_policy="cwbvh8"), rt.MIS).double()
    torch.cuda.synchronize()
    assert float((a - b).abs().mean()) < 1e-3 * float(a.abs().mean()) + 1e-6


def test_guided_render_through_cwbvh8():
    """The guided tracer takes the same policy (its trace, material and
    shadow kernels have both trees)."""
    from bajo_b200 import guide, rt
    sc = scenes.small_rt_scene()
    gsc = rt.GpuRtTriangleScene(sc, bvh_policy="cwbvh8")
    gr = guide.GuidedRenderer(gsc, sc.camera, 48, 27, spp_per_pass=2, record_capacity=1 << 14, batch=1 << 12,
                              steps=2)
    gr.render_pass(3, train=True)
    gr.render_pass(4, train=False)
    torch.cuda.synchronize()
    assert gr.workspace.status() == 0
    img = gr.image()
    assert torch.isfinite(img).all() and float(img.mean()) > 0.01
