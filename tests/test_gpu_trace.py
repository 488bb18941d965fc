"""GPU parity of closest-hit traversal against the oracle: bit-identical 8-word
hits (prim ids, t, barycentrics, normals) for both triangle tests."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import scenes  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def build(verts):
    from bajo_b200 import bvh
    b = bvh.build_triangle_bvh(dev(verts.astype(np.float32)))
    return b


def trace_rays(b, rays, mode):
    n = rays.size // 8
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    b.launch_rays(dev(rays), hits, n, tri_mode=mode, d_t=t, d_prim=p, d_status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    hh = hits.cpu().numpy()
    assert np.array_equal(hh.reshape(-1, 8)[:, 7].view(np.uint32), t.cpu().numpy().view(np.uint32))
    assert np.array_equal(hh.reshape(-1, 8)[:, 2].view(np.uint32), p.cpu().numpy().view(np.uint32))
    return hh


@pytest.mark.parametrize("mode", [0, 1])
def test_plain_lbvh_camera_matches_oracle(oracle, mode):
    """65,536 triangles, 1024x1024 pinhole rays from (0.5, 0.5, -1.5), +z, 60 deg."""
    from bajo_b200 import camera
    v = scenes.random_triangles(65536, seed=0)
    b = build(v)
    cam = camera.plain_lbvh_camera()
    n = 1024 * 1024
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    b.launch_camera(dev(cam), hits, n, 1024, 1024, tri_mode=mode)
    torch.cuda.synchronize()
    o = oracle.lbvh_build(v)
    rays = oracle.camera_rays(cam, n, 1024, 1024)
    ref = oracle.trace_bvh2(o, rays, mode)
    got = hits.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert (oracle.hits_prim(got) != oracle.EMPTY).mean() > 0.1


@pytest.mark.parametrize("mode", [0, 1])
def test_random_rays_match_oracle(oracle, mode):
    v = scenes.random_triangles(30000, seed=2, spread=0.03)
    b = build(v)
    rng = np.random.default_rng(5)
    n = 200_000
    o = rng.uniform(-0.5, 1.5, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:100, 0] = 0.0  # axis-parallel components
    d[100:200, 1:] = 0.0
    rays = np.zeros((8, n), np.float32)
    rays[0:3] = o.T
    rays[3] = rng.uniform(0.0, 0.1, n)
    rays[4:7] = d.T
    rays[7] = rng.uniform(0.5, 5.0, n)
    rays = rays.reshape(-1)
    got = trace_rays(b, rays, mode)
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), rays, mode)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("mode", [0, 1])
def test_fixture_scenes(oracle, golden_dir, name, mode):
    g = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))
    tg = np.load(os.path.join(golden_dir, "trace_fixtures.npz"))
    verts = g[name + "__verts"]
    rays = tg[name + "__rays"]
    got = trace_rays(build(verts), rays, mode)
    ref = oracle.trace_bvh2(oracle.lbvh_build(verts), rays, mode)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    brute = oracle.trace_brute(verts, rays, mode)
    assert np.array_equal(got.view(np.uint32), brute.view(np.uint32))
    robust = tg[name + "__robust"]
    assert np.array_equal(oracle.hits_prim(got)[robust], tg[name + "__prim"][robust])


def test_shared_edges_lowest_prim(oracle):
    v = scenes.grid_mesh(16, 16, z=0.5)
    xs = np.linspace(0.0, 1.0, 17, dtype=np.float32)
    pts = [(x, y) for x in xs[1:-1] for y in xs[1:-1]] + [(x + 1 / 32, y) for x in xs[:-1] for y in xs[1:-1]]
    n = len(pts)
    rays = np.zeros((8, n), np.float32)
    for i, (x, y) in enumerate(pts):
        rays[:, i] = [x, y, -1.0, 0.0, 0.0, 0.0, 1.0, np.finfo(np.float32).max]
    rays = rays.reshape(-1)
    got = trace_rays(build(v), rays, oracle.TRI_WATERTIGHT)
    assert np.all(oracle.hits_prim(got) != oracle.EMPTY)
    brute = oracle.trace_brute(v, rays, oracle.TRI_WATERTIGHT)
    assert np.array_equal(got.view(np.uint32), brute.view(np.uint32))


def test_large_scene_camera_property(oracle):
    """2^20 triangles: GPU hits equal the oracle on a 256x256 camera."""
    from bajo_b200 import camera
    v = scenes.random_triangles(1 << 20, seed=1, spread=0.004)
    b = build(v)
    cam = camera.plain_lbvh_camera()
    n = 256 * 256
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    b.launch_camera(dev(cam), hits, n, 256, 256)
    torch.cuda.synchronize()
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), oracle.camera_rays(cam, n, 256, 256), oracle.TRI_WATERTIGHT)
    assert np.array_equal(hits.cpu().numpy().view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n_tris", [1, 2, 1000, 65536])
def test_instrumented_counts_match_oracle(oracle, mode, n_tris):
    """bajo_trace_camera_stats writes the reference's five GpuTraversalStats
    counters per ray (node visits, internal child hits, leaf blocks, triangle
    tests, deepest stack); the walk is the oracle's, so every counter of
    every ray is equal."""
    from bajo_b200 import camera
    v = scenes.random_triangles(n_tris, seed=n_tris)
    b = build(v)
    cam = camera.plain_lbvh_camera()
    w = h = 256
    n = w * h
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    stats = torch.zeros(5 * n, dtype=torch.int32, device="cuda")
    b.launch_camera_instrumented(dev(cam), hits, stats, n, w, h, tri_mode=mode)
    torch.cuda.synchronize()
    o = oracle.lbvh_build(v)
    rays = oracle.camera_rays(cam, n, w, h)
    want = oracle.trace_bvh2_stats(o, rays, mode)
    got = stats.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, want)
    s = got.reshape(-1, 5)
    assert np.array_equal(s[:, 2], s[:, 3])  # one triangle per binary leaf
    if n_tris > 2:
        assert s[:, 4].max() > 0


@pytest.mark.parametrize("mode", [0, 1])
def test_three_camera_views_match_oracle(oracle, mode):
    """One launch over three 64x48 views (camera record of view i at 20 * i,
    camera_launch.mojo:34-55), as the reference's camera fixtures do
    (test/bvh/fixtures.mojo:141): hits equal the oracle's per ray."""
    from bajo_b200 import camera
    v = scenes.random_triangles(5000, seed=21, spread=0.03)
    b = build(v)
    cams = np.concatenate([
        camera.camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, 0.5], [0.0, 1.0, 0.0], 60.0),
        camera.camera_from_vfov([2.0, 0.7, 0.5], [0.5, 0.5, 0.5], [0.0, 1.0, 0.0], 45.0),
        camera.camera_from_vfov([0.4, 2.5, 0.6], [0.5, 0.5, 0.5], [0.0, 0.0, 1.0], 75.0),
    ]).astype(np.float32)
    w, h = 64, 48
    n = 3 * w * h
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    b.launch_camera(dev(cams), hits, n, w, h, tri_mode=mode)
    torch.cuda.synchronize()
    ref = oracle.trace_bvh2(oracle.lbvh_build(v), oracle.camera_rays(cams, n, w, h), mode)
    got = hits.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    per_view = (oracle.hits_prim(got).reshape(3, -1) != oracle.EMPTY).mean(axis=1)
    assert np.all(per_view > 0.02)  # every view sees geometry


@pytest.mark.parametrize("w,h,short", [(37, 23, 5), (9, 4, 0), (1, 1, 0), (8, 5, 3), (129, 2, 77)])
def test_camera_tiles_at_image_edges(oracle, w, h, short):
    """The camera kernels give each warp an 8 x 4 pixel tile; images that are
    not whole tiles, a 1 x 1 image and a last view cut short (n three views
    minus `short` rays) still trace exactly ray i = pixel i, with hits and
    traversal counters equal to the oracle's."""
    from bajo_b200 import bvh as _bvh, camera
    v = scenes.random_triangles(3000, seed=31, spread=0.04)
    b = build(v)
    cams = np.concatenate([
        camera.camera_from_vfov([0.5, 0.5, -1.5], [0.5, 0.5, 0.5], [0.0, 1.0, 0.0], 60.0),
        camera.camera_from_vfov([2.0, 0.7, 0.5], [0.5, 0.5, 0.5], [0.0, 1.0, 0.0], 45.0),
        camera.camera_from_vfov([0.4, 2.5, 0.6], [0.5, 0.5, 0.5], [0.0, 0.0, 1.0], 75.0),
    ]).astype(np.float32)
    n = 3 * w * h - short
    hits = torch.full((8 * n + 8,), -7.0, dtype=torch.float32, device="cuda")  # one guard record past n
    b.launch_camera(dev(cams), hits, n, w, h)
    stats = torch.zeros(_bvh.STATS_WORDS * n, dtype=torch.int32, device="cuda")
    b.launch_camera_instrumented(dev(cams), None, stats, n, w, h)
    torch.cuda.synchronize()
    ob = oracle.lbvh_build(v)
    rays = oracle.camera_rays(cams, n, w, h)
    got = hits.cpu().numpy()
    assert np.array_equal(got[:8 * n].view(np.uint32), oracle.trace_bvh2(ob, rays).view(np.uint32))
    assert np.all(got[8 * n:] == -7.0)  # nothing written past ray n - 1
    assert np.array_equal(stats.cpu().numpy().view(np.uint32), oracle.trace_bvh2_stats(ob, rays))
