"""Every choice the autotuner can install gives the same results: the
closest-hit kernels' block sizes (64 / 128 / 256 threads) leave the hits
bit-identical, the wavefront bounce kernels' block sizes leave the images
bit-identical, and the one-launch build on or off leaves the tree
bit-identical (its own parity is in test_gpu_lbvh_fused.py)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402


def _rays(n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = torch.empty(8, n, dtype=torch.float32, device="cuda")
    r[0:3].uniform_(0.0, 1.0, generator=g)
    r[3].zero_()
    d = torch.randn(3, n, device="cuda", generator=g)
    r[4:7] = d / d.norm(dim=0, keepdim=True)
    r[7].fill_(3.0e38)
    return r.reshape(-1)


def _deep_stack_scene(p=(0.5, 0.5, 0.5)):
    """64 triangles whose box centres give the Morton codes 0, 1, 2, 4, ...,
    2^29 and all ones (two triangles each), every box containing `p`.  The
    Karras tree is then a spine of 31 levels whose right children are 2-leaf
    subtrees; a ray from `p` enters every box at t = 0, so it descends the
    spine (ties go left) and pushes every right child: 30 stack entries."""
    p = np.asarray(p, np.float64)
    centres = [np.zeros(3)]  # code 0 (also the centroid bounds' minimum)
    for k in range(30):  # code 1 << k: axis k % 3 (x least significant), quantised value 2^(k // 3)
        u = np.full(3, 0.25 / 1024)
        u[k % 3] = (2 ** (k // 3) + 0.5) / 1024
        centres.append(u)
    centres.append(np.ones(3))  # all ones (the maximum)
    tris = []
    for m in centres:
        h = np.abs(p - m) + 0.01
        for j in range(2):
            tris.append(np.stack([m - h, m + h, m + np.array([h[0], -h[1], 0.0]) * (0.5 + 0.25 * j)]))
    return np.array(tris, np.float32).reshape(-1)


@pytest.mark.parametrize("mode", [0, 1])
def test_trace_stack_depths_give_identical_hits(oracle, mode):
    """Every traversal stack depth (64, the reference's 24, 12) and block
    size of the closest-hit kernels gives the oracle's hits bit for bit, on
    a scene whose rays need 30 stack entries: with 24 or 12 every ray runs
    out and is traced again with 64."""
    from bajo_b200 import _lib, bvh, camera
    L = _lib.load()
    v = _deep_stack_scene()
    tree = bvh.build_triangle_bvh(torch.from_numpy(v).cuda())
    cam_np = camera.camera_from_vfov([0.5, 0.5, 0.5], [0.9, 0.7, 1.0], [0.0, 1.0, 0.0], 90.0)
    cam = torch.from_numpy(cam_np).cuda()
    w, h = 64, 48
    n = w * h
    m = 5000
    g = np.random.default_rng(2)
    r = np.zeros((8, m), np.float32)
    r[0:3] = 0.5
    d = g.normal(size=(3, m))
    r[4:7] = d / np.linalg.norm(d, axis=0)
    r[7] = 3.0e38
    r = r.reshape(-1)
    rays = torch.from_numpy(r).cuda()
    stats = torch.zeros(bvh.STATS_WORDS * n, dtype=torch.int32, device="cuda")
    tree.launch_camera_instrumented(cam, None, stats, n, w, h, tri_mode=mode)
    assert int(stats.view(n, bvh.STATS_WORDS)[:, 4].min().item()) > 24
    ob = oracle.lbvh_build(v)
    ref_cam = oracle.trace_bvh2(ob, oracle.camera_rays(cam_np, n, w, h), mode).view(np.uint32)
    ref_rays = oracle.trace_bvh2(ob, r, mode).view(np.uint32)
    try:
        for blk in (64, 128, 256):
            for depth in (64, 24, 12):
                for kind, cnt in ((0, n), (1, m)):
                    lg = int(np.ceil(np.log2(cnt)))
                    assert L.bajo_trace_tuning_set(kind, lg, blk) == _lib.OK
                    assert L.bajo_trace_stack_tuning_set(kind, lg, depth) == _lib.OK
                    got = ctypes.c_int32(0)
                    assert L.bajo_trace_stack_tuning_get(kind, cnt, ctypes.byref(got)) == _lib.OK
                    assert got.value == depth
                status = torch.zeros(1, dtype=torch.int32, device="cuda")
                hc = torch.empty(8 * n, dtype=torch.float32, device="cuda")
                tree.launch_camera(cam, hc, n, w, h, tri_mode=mode, d_status=status)
                hr = torch.empty(8 * m, dtype=torch.float32, device="cuda")
                tree.launch_rays(rays, hr, m, tri_mode=mode, d_status=status)
                torch.cuda.synchronize()
                assert int(status.item()) == 0, (blk, depth)
                assert np.array_equal(hc.cpu().numpy().view(np.uint32), ref_cam), (blk, depth)
                assert np.array_equal(hr.cpu().numpy().view(np.uint32), ref_rays), (blk, depth)
    finally:
        for kind in (0, 1):
            for lg in range(33):
                L.bajo_trace_tuning_set(kind, lg, 0)
                L.bajo_trace_stack_tuning_set(kind, lg, 0)


def test_trace_stack_tuning_limits():
    from bajo_b200 import _lib
    L = _lib.load()
    got = ctypes.c_int32(0)
    assert L.bajo_trace_stack_tuning_set(0, 20, 16) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_trace_stack_tuning_set(2, 20, 24) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_trace_stack_tuning_set(1, 33, 24) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_trace_stack_tuning_get(0, 100, None) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_trace_stack_tuning_set(1, 20, 0) == _lib.OK
    assert L.bajo_trace_stack_tuning_get(1, 1 << 20, ctypes.byref(got)) == _lib.OK and got.value == 64


@pytest.mark.parametrize("mode", [0, 1])
def test_trace_block_sizes_give_identical_hits(oracle, mode):
    from bajo_b200 import _lib, bvh, camera
    L = _lib.load()
    v = scenes.random_triangles(20000, seed=4)
    tree = bvh.build_triangle_bvh(torch.from_numpy(v).cuda())
    cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
    w, h = 96, 64
    n = w * h
    rays = _rays(5000, 3)
    ref_cam = oracle.trace_bvh2(oracle.lbvh_build(v), oracle.camera_rays(camera.plain_lbvh_camera(), n, w, h), mode)
    outs = {}
    try:
        for blk in (64, 128, 256):
            for kind in (0, 1):
                lg = int(np.ceil(np.log2(n if kind == 0 else 5000)))
                assert L.bajo_trace_tuning_set(kind, lg, blk) == _lib.OK
                got = ctypes.c_int32(0)
                assert L.bajo_trace_tuning_get(kind, n if kind == 0 else 5000, ctypes.byref(got)) == _lib.OK
                assert got.value == blk
            hc = torch.empty(8 * n, dtype=torch.float32, device="cuda")
            tree.launch_camera(cam, hc, n, w, h, tri_mode=mode)
            hr = torch.empty(8 * 5000, dtype=torch.float32, device="cuda")
            tree.launch_rays(rays, hr, 5000, tri_mode=mode)
            torch.cuda.synchronize()
            outs[blk] = (hc.cpu().numpy().view(np.uint32), hr.cpu().numpy().view(np.uint32))
    finally:
        for kind in (0, 1):
            for lg in range(33):
                L.bajo_trace_tuning_set(kind, lg, 0)
    for blk in (64, 256):
        assert np.array_equal(outs[blk][0], outs[128][0])
        assert np.array_equal(outs[blk][1], outs[128][1])
    assert np.array_equal(outs[128][0], ref_cam.view(np.uint32))


def test_trace_tuning_limits():
    from bajo_b200 import _lib
    L = _lib.load()
    assert L.bajo_trace_tuning_set(0, 20, 96) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_trace_tuning_set(2, 20, 64) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_trace_tuning_set(1, 33, 64) == _lib.ERR_INVALID_ARGUMENT
    got = ctypes.c_int32(0)
    assert L.bajo_trace_tuning_set(1, 20, 0) == _lib.OK
    assert L.bajo_trace_tuning_get(1, 1 << 20, ctypes.byref(got)) == _lib.OK and got.value == 128


def test_tuner_runs_and_keeps_results(oracle):
    """A short tuning run of the closest-hit blocks and the one-launch limit
    installs choices that reproduce the oracle's tree and hits."""
    from bajo_b200 import _lib, autotune, bvh, camera
    L = _lib.load()
    try:
        res = autotune.tune_trace("trace_camera", [16], reps=2)
        assert res[16]["best"] in (64, 128, 256) and res[16]["stack"] in (64, 24, 12)
        fe = autotune.tune_one_launch(range(15, 17), reps=2)
        assert set(v["best"] for v in fe.values()) <= {0, 1 << 15, 1 << 16}
        v = scenes.random_triangles(1 << 16, seed=9)
        t = bvh.build_triangle_bvh(torch.from_numpy(v).cuda())
        torch.cuda.synchronize()
        o = oracle.lbvh_build(v)
        assert np.array_equal(t.node_meta.cpu().numpy().view(np.uint32)[: 4 * ((1 << 16) - 1)],
                              o.node_meta[: 4 * ((1 << 16) - 1)])
        cam = torch.from_numpy(camera.plain_lbvh_camera()).cuda()
        hits = torch.empty(8 * 65536, dtype=torch.float32, device="cuda")
        t.launch_camera(cam, hits, 65536, 256, 256)
        torch.cuda.synchronize()
        ref = oracle.trace_bvh2(o, oracle.camera_rays(camera.plain_lbvh_camera(), 65536, 256, 256))
        assert np.array_equal(hits.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    finally:
        for lg in range(33):
            L.bajo_trace_tuning_set(0, lg, 0)
            L.bajo_trace_stack_tuning_set(0, lg, 0)
        L.bajo_lbvh_fused_max_set(_lib.FUSED_MAX_LEAVES)


@pytest.mark.parametrize("policy", ["lbvh", "cwbvh8"])
def test_render_block_sizes_give_identical_images(policy):
    """Every block size of the wavefront bounce kernels (closest hit,
    shading, shadow rays) renders the same image bit for bit, for the plain
    algorithms and the guided one, with materials and without."""
    from bajo_b200 import _lib, guide, rt
    L = _lib.load()
    mats = scenes.materials_in_box(n_spheres=6, subdivisions=2)
    lit = scenes.small_rt_scene()
    w, h = 40, 24
    images = {}
    try:
        for blocks in ((128, 128, 128), (64, 64, 64), (256, 256, 256), (64, 256, 128)):
            for kind, blk in enumerate(blocks):
                assert L.bajo_render_tuning_set(kind, blk) == _lib.OK
                got = ctypes.c_int32(0)
                assert L.bajo_render_tuning_get(kind, ctypes.byref(got)) == _lib.OK and got.value == blk
            out = []
            for sc in (lit, mats):
                gsc = rt.GpuRtTriangleScene(sc, bvh_policy=policy)
                for algorithm in (rt.PATH, rt.NEE, rt.MIS):
                    settings = rt.RenderSettings(w, h, 4, rng_seed=7, max_depth=6)
                    img = rt.render_gpu_triangles(settings, sc.camera, gsc, algorithm)
                    out.append(img.cpu().numpy().view(np.uint32).copy())
                gr = guide.GuidedRenderer(gsc, sc.camera, w, h, max_depth=6, record_capacity=1 << 12, steps=2,
                                          batch=1 << 10, spp_per_pass=2)
                # no training: its gradient atomics sum in any order
                out.append(gr.render(passes=2, train_passes=0, seed=11).cpu().numpy().view(np.uint64).copy())
                assert gr.workspace.status() == 0
            torch.cuda.synchronize()
            images[blocks] = out
    finally:
        for kind in range(3):
            L.bajo_render_tuning_set(kind, 0)
    ref = images[(128, 128, 128)]
    for blocks, out in images.items():
        for a, b in zip(out, ref):
            assert np.array_equal(a, b), blocks


def test_render_tuning_limits():
    from bajo_b200 import _lib
    L = _lib.load()
    got = ctypes.c_int32(0)
    assert L.bajo_render_tuning_set(0, 96) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_render_tuning_set(3, 64) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_render_tuning_set(-1, 64) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_render_tuning_get(0, None) == _lib.ERR_INVALID_ARGUMENT
    assert L.bajo_render_tuning_set(2, 0) == _lib.OK
    assert L.bajo_render_tuning_get(2, ctypes.byref(got)) == _lib.OK and got.value == 128
