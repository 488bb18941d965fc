"""Handle-based rendering (bajo_render_create / enqueue / download /
destroy): on a side stream the render is recorded into a CUDA graph once and
replayed; images, ray counts and status equal the direct bajo_render's bit
for bit, the graph follows new camera values in the same buffer, and a new
buffer or new settings records a new graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import rt, scenes  # noqa: E402


@pytest.fixture(scope="module")
def small():
    sc = scenes.small_rt_scene()
    return sc, rt.GpuRtTriangleScene(sc, bvh_policy="lbvh")


def _direct(sc, gsc, settings, cam, algorithm=rt.MIS):
    ws = rt.RenderWorkspace(settings, algorithm)
    img = rt.render_gpu_triangles(settings, cam, gsc, algorithm, workspace=ws)
    torch.cuda.synchronize()
    return img.cpu().numpy(), ws.ray_counts()


@pytest.mark.parametrize("algorithm", [rt.PATH, rt.NEE, rt.MIS])
def test_graph_replay_equals_direct_render(small, algorithm):
    sc, gsc = small
    settings = rt.RenderSettings(48, 27, 4, rng_seed=7, max_depth=8, chunk_paths=4 * 300)
    cam = torch.from_numpy(np.asarray(sc.camera, np.float32)).cuda()
    ref, (rays, shadows) = _direct(sc, gsc, settings, cam, algorithm)
    r = rt.Renderer(settings, algorithm)
    side = torch.cuda.Stream()
    px = torch.empty((27, 48, 3), dtype=torch.float32, device="cuda")
    with torch.cuda.stream(side):
        for k in range(3):
            px.fill_(-1.0)
            r.enqueue(gsc, cam, px, stream=side)
            img, a, b, status = r.download(px, stream=side)
            assert status == 0
            assert np.array_equal(img.view(np.uint32), ref.view(np.uint32)), k
            assert (a, b) == (rays, shadows)
    assert r.graph_launches() == 3
    r.close()


def test_default_stream_renders_directly(small):
    sc, gsc = small
    settings = rt.RenderSettings(32, 18, 2, rng_seed=3)
    cam = torch.from_numpy(np.asarray(sc.camera, np.float32)).cuda()
    ref, _ = _direct(sc, gsc, settings, cam)
    r = rt.Renderer(settings)
    px = torch.empty((18, 32, 3), dtype=torch.float32, device="cuda")
    r.enqueue(gsc, cam, px)
    img, _, _, status = r.download(px)
    assert status == 0 and np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    assert r.graph_launches() == 0  # the legacy default stream cannot be captured
    r.close()


def test_replay_reads_new_camera_values_and_new_buffers_rerecord(small):
    sc, gsc = small
    settings = rt.RenderSettings(40, 30, 2, rng_seed=11)
    cam = torch.from_numpy(np.asarray(sc.camera, np.float32)).cuda()
    moved = sc.camera.copy()
    moved[0] += 0.05  # camera origin x
    r = rt.Renderer(settings)
    side = torch.cuda.Stream()
    px = torch.empty((30, 40, 3), dtype=torch.float32, device="cuda")
    with torch.cuda.stream(side):
        r.enqueue(gsc, cam, px, stream=side)
        r.download(px, stream=side)
        cam.copy_(torch.from_numpy(moved))          # same buffer, new values: the graph replays
        r.enqueue(gsc, cam, px, stream=side)
        img, _, _, _ = r.download(px, stream=side)
        other = torch.empty_like(px)                  # a new output buffer records a new graph
        r.enqueue(gsc, cam, other, stream=side)
        img2, _, _, _ = r.download(other, stream=side)
    ref, _ = _direct(sc, gsc, settings, torch.from_numpy(moved).cuda())
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(img2.view(np.uint32), ref.view(np.uint32))
    assert r.graph_launches() == 3
    r.close()
