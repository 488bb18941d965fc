"""GPU parity of the wavefront path tracer against the oracle: bit-identical
pixels for PATH / NEE / MIS, chunk invariance, FP64 sums."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402


@pytest.fixture(scope="module")
def small():
    from bajo_b200 import rt
    sc = scenes.small_rt_scene()
    return sc, rt.GpuRtTriangleScene(sc, bvh_policy="lbvh")


@pytest.mark.parametrize("algorithm", [0, 3, 4])
def test_render_matches_oracle(oracle, small, algorithm):
    from bajo_b200 import rt
    sc, gsc = small
    w, h, spp = 48, 27, 4
    settings = rt.RenderSettings(w, h, spp, rng_seed=2026, max_depth=8)
    ws = rt.RenderWorkspace(settings, algorithm)
    img = rt.render_gpu_triangles(settings, sc.camera, gsc, algorithm, workspace=ws)
    torch.cuda.synchronize()
    assert ws.status() == 0
    ref = oracle.render(sc, sc.camera, w, h, spp, max_depth=8, seed=2026, algorithm=algorithm)
    got = img.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert got.mean() > 0.05


def test_chunking_does_not_change_the_image(small):
    """Chunked == full-capacity render (test/rt/test_gpu.mojo:446-478)."""
    from bajo_b200 import rt
    sc, gsc = small
    w, h, spp = 40, 30, 8
    full = rt.render_gpu_triangles(rt.RenderSettings(w, h, spp), sc.camera, gsc, rt.MIS)
    chunked = rt.render_gpu_triangles(rt.RenderSettings(w, h, spp, chunk_paths=spp * 37), sc.camera, gsc, rt.MIS)
    torch.cuda.synchronize()
    assert torch.equal(full, chunked)


def test_fp64_sums(oracle, small):
    from bajo_b200 import rt
    sc, gsc = small
    w, h, spp = 16, 9, 8
    acc = torch.zeros((h, w, 3), dtype=torch.float64, device="cuda")
    settings = rt.RenderSettings(w, h, spp, rng_seed=5)
    rt.render_gpu_triangles(settings, sc.camera, gsc, rt.MIS, pixels64=acc)
    rt.render_gpu_triangles(settings, sc.camera, gsc, rt.MIS, pixels64=acc)
    torch.cuda.synchronize()
    _, smp = oracle.render(sc, sc.camera, w, h, spp, seed=5, algorithm=4, return_samples=True)
    ref = np.zeros((h, w, 3))
    for s in range(spp):
        ref += smp[:, :, s, :].astype(np.float64)
    assert np.array_equal(acc.cpu().numpy(), 2 * ref)


def test_large_scene_render_matches_oracle(oracle):
    """The 64-icosphere workload (1.31M triangles) at a small resolution."""
    from bajo_b200 import rt
    sc = scenes.spheres_in_box()
    assert sc.n_tris == 12 + 2 + 64 * 20480
    gsc = rt.GpuRtTriangleScene(sc, bvh_policy="lbvh")
    w, h, spp = 32, 18, 2
    img = rt.render_gpu_triangles(rt.RenderSettings(w, h, spp), sc.camera, gsc, rt.MIS)
    torch.cuda.synchronize()
    ref = oracle.render(sc, sc.camera, w, h, spp, algorithm=4)
    assert np.array_equal(img.cpu().numpy().view(np.uint32), ref.view(np.uint32))


@pytest.fixture(scope="module")
def materials():
    from bajo_b200 import rt
    sc = scenes.materials_in_box(n_spheres=8, subdivisions=2)
    return sc, rt.GpuRtTriangleScene(sc, bvh_policy="lbvh")


@pytest.mark.parametrize("algorithm", [0, 3, 4])
def test_materials_render_matches_oracle(oracle, materials, algorithm):
    """Lambertian, mirror, glossy metal and glass spheres: the material pass
    and the delta flag give the oracle's image bit for bit."""
    from bajo_b200 import rt
    sc, gsc = materials
    w, h, spp = 40, 24, 8
    settings = rt.RenderSettings(w, h, spp, rng_seed=404, max_depth=12)
    ws = rt.RenderWorkspace(settings, algorithm)
    img = rt.render_gpu_triangles(settings, sc.camera, gsc, algorithm, workspace=ws)
    torch.cuda.synchronize()
    assert ws.status() == 0
    ref = oracle.render(sc, sc.camera, w, h, spp, max_depth=12, seed=404, algorithm=algorithm)
    got = img.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert got.mean() > 0.05


def test_guided_render_runs_with_materials(materials):
    from bajo_b200 import guide
    sc, gsc = materials
    gr = guide.GuidedRenderer(gsc, sc.camera, 32, 20, max_depth=8, record_capacity=1 << 14, steps=2, batch=1 << 10)
    img = gr.render(passes=3, train_passes=2).cpu().numpy()
    assert gr.workspace.status() == 0 and np.all(np.isfinite(img)) and img.mean() > 0.05


@pytest.mark.parametrize("spp,chunk_rows", [(1, 0), (2, 0), (4, 0), (8, 0), (2, 8), (4, 4)])
def test_tiled_primary_rays_match_oracle(oracle, small, spp, chunk_rows):
    """At 1, 2, 4 or 8 samples per pixel, with chunks of whole tile rows,
    the primary rays are queued by pixel tiles (a warp's samples cover a 2-D
    block of pixels); the image stays the oracle's bit for bit, also when
    the image is rendered in chunks of `chunk_rows` rows."""
    from bajo_b200 import rt
    sc, gsc = small
    w, h = 64, 32
    chunk = chunk_rows * w * spp
    settings = rt.RenderSettings(w, h, spp, rng_seed=77, max_depth=6, chunk_paths=chunk)
    ws = rt.RenderWorkspace(settings, rt.MIS)
    img = rt.render_gpu_triangles(settings, sc.camera, gsc, rt.MIS, workspace=ws)
    torch.cuda.synchronize()
    assert ws.status() == 0
    ref = oracle.render(sc, sc.camera, w, h, spp, max_depth=6, seed=77, algorithm=rt.MIS)
    assert np.array_equal(img.cpu().numpy().view(np.uint32), ref.view(np.uint32))
