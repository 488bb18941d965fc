"""GPU parity of the CWBVH8 build and traversal: compressed nodes, triangle
records and segment offsets equal the oracle's word for word (fixtures,
random sizes, segmented trees with empty segments); closest and any hits of
ray buffers and camera rays equal the oracle's bit for bit; known answers of
the reference's tests; host-injected corruption ends with a status, not a
fault."""
import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import _lib, bvh, camera, scenes, wide  # noqa: E402

EMPTY = 0xFFFFFFFF


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_cw(verts, seg=None):
    tree = bvh.build_triangle_bvh(dev(np.asarray(verts, np.float32)), seg)
    cw = wide.build_cwbvh8(tree)
    assert cw.status() == 0
    return tree, cw


def compare(cw, ocw):
    nn = int(ocw.node_offsets[-1])
    assert cw.n_nodes == nn
    S = ocw.node_offsets.size
    assert np.array_equal(cw.node_offsets[:S].cpu().numpy().view(np.uint32), ocw.node_offsets)
    assert np.array_equal(cw.nodes[:nn * 20].cpu().numpy().view(np.uint32), ocw.nodes.view(np.uint32))
    nt = ocw.triangles.size
    assert np.array_equal(cw.triangles[:nt].cpu().numpy().view(np.uint32), ocw.triangles.view(np.uint32))


FIXTURES = ["small", "single", "duplicate_centroid", "strip16", "two_depth", "degenerate_axis", "grid8",
            "random1000"]


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_encoding_matches_oracle(oracle, golden_dir, name):
    verts = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))[name + "__verts"]
    _, cw = gpu_cw(verts)
    compare(cw, oracle.cwbvh8_build(oracle.lbvh_build(verts)))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 17, 257, 4096, 65536, 1 << 18])
def test_random_encoding_matches_oracle(oracle, n):
    verts = scenes.random_triangles(n, seed=n)
    _, cw = gpu_cw(verts)
    compare(cw, oracle.cwbvh8_build(oracle.lbvh_build(verts)))


def test_segmented_encoding_matches_oracle(oracle):
    verts = scenes.random_triangles(5000, seed=3)
    seg = np.array([0, 0, 1, 4, 4, 5, 37, 900, 4096, 5000, 5000], np.uint32)
    _, cw = gpu_cw(verts, seg)
    compare(cw, oracle.cwbvh8_build(oracle.lbvh_build(verts, seg)))


def test_batched_encoding_matches_oracle(oracle):
    verts, so = scenes.batched_scenes(n_scenes=32, lo=16, hi=20000, seed=5)
    _, cw = gpu_cw(verts, so)
    compare(cw, oracle.cwbvh8_build(oracle.lbvh_build(verts, so)))


def _rays(n, seed, lo=-0.5, hi=1.5):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:64, 0] = 0.0
    d[64:128, 1:] = 0.0
    r = np.zeros((8, n), np.float32)
    r[0:3], r[3], r[4:7], r[7] = o.T, rng.uniform(0.0, 0.1, n), d.T, rng.uniform(0.5, 5.0, n)
    return r.reshape(-1)


def _trace(cw, rays, any_hit):
    n = rays.size // 8
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    st = cw.launch_rays(dev(rays), hits, n, any_hit, d_t=t, d_prim=prim)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    h = hits.cpu().numpy()
    assert np.array_equal(t.cpu().numpy().view(np.uint32), h.reshape(-1, 8)[:, 7].view(np.uint32))
    assert np.array_equal(prim.cpu().numpy().view(np.uint32), h.reshape(-1, 8)[:, 2].view(np.uint32))
    return h


@pytest.mark.parametrize("any_hit", [False, True])
def test_fixture_hits_match_oracle(oracle, golden_dir, any_hit):
    g = np.load(os.path.join(golden_dir, "lbvh_fixtures.npz"))
    tg = np.load(os.path.join(golden_dir, "trace_fixtures.npz"))
    for name in FIXTURES:
        verts, rays = g[name + "__verts"], tg[name + "__rays"]
        _, cw = gpu_cw(verts)
        ref = oracle.trace_cwbvh8(oracle.cwbvh8_build(oracle.lbvh_build(verts)), rays, any_hit)
        assert np.array_equal(_trace(cw, rays, any_hit).view(np.uint32), ref.view(np.uint32)), name


@pytest.mark.parametrize("any_hit", [False, True])
@pytest.mark.parametrize("n_tris", [300, 30000, 1 << 18])
def test_random_hits_match_oracle(oracle, n_tris, any_hit):
    v = scenes.random_triangles(n_tris, seed=3, spread=0.03)
    _, cw = gpu_cw(v)
    rays = _rays(300_000, 9)
    ref = oracle.trace_cwbvh8(oracle.cwbvh8_build(oracle.lbvh_build(v)), rays, any_hit)
    assert np.array_equal(_trace(cw, rays, any_hit).view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("any_hit", [False, True])
def test_camera_hits_match_oracle(oracle, any_hit):
    v = scenes.random_triangles(65536, seed=0)
    _, cw = gpu_cw(v)
    cams = np.stack([camera.plain_lbvh_camera(),
                     camera.camera([1.6, 0.4, -1.2], [0.5, 0.5, 0.5], [0, 1, 0], 0.8)]).astype(np.float32)
    w, h = 512, 384
    n = 2 * w * h
    hits = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    st = cw.launch_camera(dev(cams.reshape(-1)), hits, n, w, h, any_hit)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    rays = oracle.camera_rays(cams.reshape(-1), n, w, h)
    ref = oracle.trace_cwbvh8(oracle.cwbvh8_build(oracle.lbvh_build(v)), rays, any_hit)
    assert np.array_equal(hits.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_hits_agree_with_binary_tree():
    v = scenes.random_triangles(65536, seed=0)
    tree, cw = gpu_cw(v)
    cam = dev(camera.plain_lbvh_camera())
    n = 1024 * 1024
    a = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    b = torch.empty(8 * n, dtype=torch.float32, device="cuda")
    cw.launch_camera(cam, a, n, 1024, 1024)
    c = tree.c_struct()
    _lib.check(_lib.load().bajo_trace_camera(ctypes.byref(c), cam.data_ptr(), n, 1024, 1024, _lib.TRI_MT,
                                             b.data_ptr(), None, None, None, None), "bajo_trace_camera")
    torch.cuda.synchronize()
    pa, pb = a.view(-1, 8)[:, 2].view(torch.int32), b.view(-1, 8)[:, 2].view(torch.int32)
    assert (pa == pb).float().mean().item() >= 0.9999


def _tri_at(z, count=1):
    v = []
    for i in range(count):
        x = 3.0 * i
        v += [[x - 1.0, -1.0, z], [x + 1.0, -1.0, z], [x, 1.0, z]]
    return np.array(v, np.float32).reshape(-1, 9)


def test_known_answers_and_segment_views(oracle):
    # test_segmented_empty.mojo: a triangle at z = 6 is hit at t = 6 along
    # +z; empty segments take no nodes; 5 + 17 triangles take exactly
    # consecutive storage
    verts = np.concatenate([_tri_at(4.0, 5), _tri_at(8.0, 17), _tri_at(6.0)])
    seg = np.array([0, 0, 5, 5, 22, 23, 23], np.uint32)
    _, cw = gpu_cw(verts, seg)
    compare(cw, oracle.cwbvh8_build(oracle.lbvh_build(verts, seg)))
    no = cw.node_offsets[:7].cpu().numpy()
    assert no[1] == no[0] and no[3] == no[2] and no[6] == no[5]
    cam = dev(camera.camera([0, 0, 0], [0, 0, 1], [0, 1, 0], 0.75))
    for s, first_tri, z in ((1, 0, 4.0), (3, 5, 8.0), (4, 22, 6.0)):
        view = wide.BajoCwbvh8C()
        view.n_segments = 1
        view.n_tris = int(seg[s + 1] - seg[s])
        view.node_offsets = cw.node_offsets.data_ptr()
        view.nodes = cw.nodes.data_ptr() + int(no[s]) * 80
        view.triangles = cw.triangles.data_ptr() + first_tri * 48
        hits = torch.empty(8, dtype=torch.float32, device="cuda")
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.check(_lib.load().bajo_trace_cwbvh8_camera(ctypes.byref(view), int(no[s + 1] - no[s]), cam.data_ptr(),
                                                        1, 1, 1, 0, hits.data_ptr(), None, None, st.data_ptr(), None),
                   "bajo_trace_cwbvh8_camera")
        torch.cuda.synchronize()
        h = hits.cpu().numpy()
        assert int(st.item()) == 0 and abs(h[7] - z) < 1e-5 and int(h[2:3].view(np.uint32)[0]) == 0, s


def test_corrupt_child_and_triangle_refs_report_status():
    v = scenes.random_triangles(4096, seed=1)
    _, cw = gpu_cw(v)
    rays = dev(_rays(4096, 2))
    hits = torch.empty(8 * 4096, dtype=torch.float32, device="cuda")
    words = cw.nodes.view(torch.int32)
    good = words[:cw.n_nodes * 20].clone()
    words[4] = 0x7FFFFF00  # root's first internal child out of range
    st = cw.launch_rays(rays, hits, 4096)
    torch.cuda.synchronize()
    assert int(st.item()) & _lib.STATUS_BAD_TOPOLOGY
    words[:cw.n_nodes * 20] = good
    words[20 * (cw.n_nodes - 1) + 5] = 0x7FFFFF00  # a node's triangles out of range
    st = cw.launch_rays(dev(_rays(300_000, 4)), torch.empty(8 * 300_000, device="cuda"), 300_000)
    torch.cuda.synchronize()
    assert int(st.item()) & _lib.STATUS_BAD_TOPOLOGY
    words[:cw.n_nodes * 20] = good
    st = cw.launch_rays(rays, hits, 4096)
    torch.cuda.synchronize()
    assert int(st.item()) == 0


def test_invalid_arguments():
    v = scenes.random_triangles(64, seed=1)
    tree, cw = gpu_cw(v)
    L = _lib.load()
    c = cw.c_struct()
    c.nodes = cw.nodes.data_ptr() + 4
    assert L.bajo_trace_cwbvh8_rays(ctypes.byref(c), cw.n_nodes, cw.nodes.data_ptr(), 1, 0, None, None, None,
                                    cw.workspace.data_ptr(), None) == _lib.ERR_INVALID_ARGUMENT
    c = cw.c_struct()
    assert L.bajo_trace_cwbvh8_rays(ctypes.byref(c), cw.n_nodes, cw.nodes.data_ptr(), 1, 2, None, None, None,
                                    cw.workspace.data_ptr(), None) == _lib.ERR_INVALID_ARGUMENT
    t = tree.c_struct()
    assert L.bajo_cwbvh8_build(ctypes.byref(t), ctypes.byref(c), cw.workspace.data_ptr(), 16, None) == \
        _lib.ERR_WORKSPACE_TOO_SMALL


@pytest.mark.parametrize("w,h,short", [(37, 23, 5), (1, 1, 0), (129, 2, 77)])
def test_camera_tiles_at_image_edges(oracle, w, h, short):
    """8 x 4 pixel tiles per warp at image sizes that are not whole tiles and
    with a last view cut short: the oracle's CWBVH8 walk, ray by ray."""
    v = scenes.random_triangles(3000, seed=32, spread=0.04)
    _, cw = gpu_cw(v)
    cams = np.stack([camera.plain_lbvh_camera(),
                     camera.camera([1.6, 0.4, -1.2], [0.5, 0.5, 0.5], [0, 1, 0], 0.8)]).astype(np.float32)
    n = 2 * w * h - short
    hits = torch.full((8 * n + 8,), -7.0, dtype=torch.float32, device="cuda")
    st = cw.launch_camera(dev(cams.reshape(-1)), hits, n, w, h, False)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    rays = oracle.camera_rays(cams.reshape(-1), n, w, h)
    ref = oracle.trace_cwbvh8(oracle.cwbvh8_build(oracle.lbvh_build(v)), rays, False)
    got = hits.cpu().numpy()
    assert np.array_equal(got[:8 * n].view(np.uint32), ref.view(np.uint32))
    assert np.all(got[8 * n:] == -7.0)
