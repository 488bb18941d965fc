"""GPU tests of the guided wavefront tracer: with the network switched off it
is the MIS tracer bit for bit; with a trained network it stays unbiased
against a long MIS render; its training records are well formed; and the
trained network lowers the error at equal samples per pixel on a scene lit
only indirectly."""
import numpy as np
import pytest
import torch

from bajo_b200 import guide, rt, scenes

pytestmark = pytest.mark.gpu

W, H = 48, 36


@pytest.fixture(scope="module")
def indirect():
    s = scenes.indirect_box_scene()
    return s, rt.GpuRtTriangleScene(s, bvh_policy="lbvh")


def _mis(gs, cam, spp, seed, w=W, h=H):
    st = rt.RenderSettings(w, h, spp, rng_seed=seed)
    sum64 = torch.zeros((h, w, 3), dtype=torch.float64, device="cuda")
    img = rt.render_gpu_triangles(st, cam, gs, rt.MIS, pixels64=sum64)
    return img, sum64


def test_fraction_zero_is_the_mis_tracer(indirect):
    s, gs = indirect
    cam = s.camera
    for seed in (3, 4):
        mis, _ = _mis(gs, cam, 4, seed)
        gr = guide.GuidedRenderer(gs, cam, W, H, guide_fraction=0.0, spp_per_pass=4)
        gr.render_pass(seed, train=True, guide_fraction=0.0)  # records collected, image unaffected
        torch.cuda.synchronize()
        assert torch.equal(gr.pixels, mis)
        assert gr.workspace.status() == 0
        assert gr.records.count() > 0


def test_passes_of_different_sizes_accumulate_samples(indirect):
    """A 2-spp pass then a 4-spp pass (its own workspace) at guide fraction
    0: the FP64 sum is the two MIS renders' sample sums and the image their
    6-sample mean."""
    s, gs = indirect
    cam = s.camera
    _, sum2 = _mis(gs, cam, 2, 11)
    _, sum4 = _mis(gs, cam, 4, 12)
    gr = guide.GuidedRenderer(gs, cam, W, H, guide_fraction=0.0, spp_per_pass=2)
    gr.prepare_pass(4)
    gr.render_pass(11, train=False, guide_fraction=0.0)
    gr.render_pass(12, train=False, guide_fraction=0.0, spp=4)
    torch.cuda.synchronize()
    assert gr.samples == 6 and gr.workspace.status() == 0
    assert torch.equal(gr.sum64, sum2 + sum4)
    assert torch.equal(gr.image(), (sum2 + sum4) / 6)


def test_records_are_well_formed(indirect):
    s, gs = indirect
    gr = guide.GuidedRenderer(gs, s.camera, W, H, record_capacity=1 << 14, spp_per_pass=4)
    gr.render_pass(9, train=False)
    gr.records.reset()
    gr.render_pass(10, train=False)  # no collection when train=False
    assert gr.records.count() == 0
    gr.settings.rng_seed = 11
    g = gr.guide_c(0.5, True)
    import ctypes
    from bajo_b200 import _lib
    c = gr.settings.c(guide.GUIDED)
    sc = gs.c()
    _lib.check(_lib.load().bajo_render_guided(ctypes.byref(sc), gr.cam.data_ptr(), ctypes.byref(c), ctypes.byref(g),
                                              gr.pixels.data_ptr(), None, gr.workspace.buffer.data_ptr(),
                                              gr.workspace.buffer.numel(), _lib.stream_handle()),
               "bajo_render_guided")
    n = gr.records.count()
    assert 0 < n <= gr.records.capacity
    pos, nrm, d, wt = [a.cpu().numpy() for a in gr.records.arrays()]
    assert np.all(pos >= -1e-3) and np.all(pos <= 1 + 1e-3)  # on the box's surfaces
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1, atol=1e-4)
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-4)
    assert np.all(np.sum(nrm * d, axis=1) > -1e-6)  # continuations leave the surface
    assert np.all(np.isfinite(wt)) and np.all(wt >= 0) and np.count_nonzero(wt) > n // 20


@pytest.fixture(scope="module")
def trained(indirect):
    s, gs = indirect
    gr = guide.GuidedRenderer(gs, s.camera, W, H, record_capacity=1 << 15, spp_per_pass=8, batch=1 << 13,
                              steps=16)
    l0 = None
    for k in range(24):
        gr.render_pass(100 + k, train=True)
        if l0 is None:
            l0 = float(gr.net.loss_buf.item())
    gr.reset_image()
    return gr, l0


def test_training_runs_on_tracer_records(trained):
    gr, l0 = trained
    assert gr.net.step == 24 * 16
    assert np.isfinite(float(gr.net.loss_buf.item())) and np.isfinite(l0)
    p = gr.net.params32.cpu().numpy()
    assert np.all(np.isfinite(p)) and not np.allclose(p, guide.init_params(0))


def test_guided_is_unbiased(indirect, trained):
    s, gs = indirect
    gr, _ = trained
    img = gr.render(passes=64, train_passes=0, seed=5000).cpu().numpy()  # 512 spp
    assert gr.workspace.status() == 0
    _, ref64 = _mis(gs, s.camera, 2048, 77)
    ref = (ref64 / 2048).cpu().numpy()
    # whole-image and 6x6-pixel block means agree
    assert img.mean() == pytest.approx(ref.mean(), rel=1.5e-2)
    bi = img.reshape(H // 6, 6, W // 6, 6, 3).mean(axis=(1, 3))
    br = ref.reshape(H // 6, 6, W // 6, 6, 3).mean(axis=(1, 3))
    assert np.all(np.abs(bi - br) <= 0.06 * br + 0.02 * ref.mean()), np.abs(bi - br).max()


def test_trained_network_lowers_error_at_equal_spp(indirect, trained):
    """MSE against a 4096-spp MIS render: the trained guide at 16 spp beats
    plain MIS at 16 spp (averaged over 4 seeds)."""
    s, gs = indirect
    gr, _ = trained
    _, ref64 = _mis(gs, s.camera, 4096, 991)
    ref = ref64 / 4096
    mse_plain, mse_guided = [], []
    for k in range(4):
        img, _ = _mis(gs, s.camera, 16, 300 + k)
        mse_plain.append(float(((img.double() - ref) ** 2).mean()))
        gr.reset_image()
        gi = gr.render(passes=2, train_passes=0, seed=400 + 13 * k)
        mse_guided.append(float(((gi - ref) ** 2).mean()))
    ratio = np.mean(mse_guided) / np.mean(mse_plain)
    print("guided / plain MSE at 16 spp:", ratio)
    assert ratio < 0.85
