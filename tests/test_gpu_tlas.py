"""GPU parity of the two-level trees: instance boxes equal the oracle's bit
for bit, closest and any hits of rays and camera rays through the top-level
tree equal the oracle's bit for bit (both triangle tests, LBVH and H-PLOC
BLAS sets, an empty BLAS), and the reference's TLAS known answers hold."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import _lib, bvh, camera, scenes, tlas  # noqa: E402
from bajo_b200.tlas import invert_affine  # noqa: E402


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def tri_at(z):
    return np.array([[-1, -1, z, 1, -1, z, 0, 1, z]], np.float32)


def translate(x, y, z):
    return np.array([1, 0, 0, x, 0, 1, 0, y, 0, 0, 1, z], np.float32)


def blas_set(meshes, method="lbvh"):
    verts = np.concatenate([m.reshape(-1) for m in meshes]).astype(np.float32)
    counts = [m.reshape(-1, 9).shape[0] for m in meshes]
    seg = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    return verts, seg, bvh.build_triangle_bvh(dev(verts), seg, method=method)


def random_instances(n_inst, n_blas, seed):
    rng = np.random.default_rng(seed)
    xf = []
    for _ in range(n_inst):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        m = rot * rng.uniform(0.5, 2.0)
        t = rng.uniform(-4, 4, 3)
        xf.append(np.concatenate([m, t[:, None]], axis=1).reshape(-1))
    return np.array(xf, np.float32), rng.integers(0, n_blas, n_inst).astype(np.uint32)


def one_hit(t, cam_o, cam_d):
    cam = dev(camera.camera(cam_o, np.add(cam_o, cam_d), [0, 1, 0], 0.75))
    hits = torch.empty(8, dtype=torch.float32, device="cuda")
    st = t.launch_camera(cam, hits, 1, 1, 1)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    h = hits.cpu().numpy()
    return float(h[7]), int(h[2:3].view(np.uint32)[0]), int(h[3:4].view(np.uint32)[0])


def test_known_answers():
    # test_gpu_triangle_tlas_uses_instance_blas_index
    _, _, bs = blas_set([tri_at(2.0), tri_at(6.0)])
    t = tlas.build_triangle_tlas(bs, [translate(-10, 0, 0), translate(10, 0, 0)], [0, 1])
    got = one_hit(t, [10, 0, 0], [0, 0, 1])
    assert abs(got[0] - 6.0) < 1e-5 and got[1:] == (0, 1)
    # test_gpu_triangle_tlas_closest_hit_across_different_blas
    _, _, bs = blas_set([tri_at(8.0), tri_at(3.0)])
    t = tlas.build_triangle_tlas(bs, [translate(0, 0, 0), translate(0, 0, 0)], [0, 1])
    got = one_hit(t, [0, 0, 0], [0, 0, 1])
    assert abs(got[0] - 3.0) < 1e-5 and got[1:] == (0, 1)


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros((8, n), np.float32)
    r[0:3] = rng.uniform(-6, 6, (3, n))
    d = rng.normal(size=(3, n))
    r[4:7] = d / np.linalg.norm(d, axis=0)
    r[4, :64] = 0.0
    r[3] = rng.uniform(0.0, 0.1, n)
    r[7] = rng.uniform(2.0, 30.0, n)
    return r.reshape(-1)


@pytest.mark.parametrize("method", ["lbvh", "hploc"])
@pytest.mark.parametrize("tri_mode", [0, 1])
@pytest.mark.parametrize("any_hit", [False, True])
def test_random_instances_match_oracle(oracle, method, tri_mode, any_hit):
    meshes = [scenes.random_triangles(n, seed=n, spread=0.1).reshape(-1, 9) for n in (2000, 500, 60, 7)]
    verts, seg, bs = blas_set(meshes, method)
    xf, bi = random_instances(300, 4, 5)
    t = tlas.build_triangle_tlas(bs, xf, bi)
    ob = oracle.lbvh_build(verts, seg)
    boxes = oracle.tlas_instance_boxes(ob, xf, bi)
    assert np.array_equal(t.boxes[:300 * 9].cpu().numpy().view(np.uint32), boxes.reshape(-1).view(np.uint32))
    top = oracle.lbvh_build(boxes)
    inv = t.inv_transforms.cpu().numpy()
    rays = _rays(200_000, 7)
    hits = torch.empty(8 * 200_000, dtype=torch.float32, device="cuda")
    st = t.launch_rays(dev(rays), hits, 200_000, any_hit, tri_mode)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = oracle.trace_tlas(top, ob, inv, bi, rays, any_hit, tri_mode)
    got = hits.cpu().numpy()
    assert (ref.reshape(-1, 8)[:, 3].view(np.uint32) != oracle.SENTINEL).mean() > 0.05
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_camera_and_empty_blas_match_oracle(oracle):
    meshes = [scenes.random_triangles(3000, seed=1, spread=0.05).reshape(-1, 9), np.zeros((0, 9), np.float32),
              scenes.random_triangles(40, seed=2, spread=0.2).reshape(-1, 9)]
    verts, seg, bs = blas_set(meshes)
    xf, bi = random_instances(64, 3, 9)
    t = tlas.build_triangle_tlas(bs, xf, bi)
    cam = camera.camera([0.0, 1.0, -14.0], [0, 0, 0], [0, 1, 0], 0.6)
    w, h = 256, 192
    hits = torch.empty(8 * w * h, dtype=torch.float32, device="cuda")
    st = t.launch_camera(dev(cam), hits, w * h, w, h)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ob = oracle.lbvh_build(verts, seg)
    top = oracle.lbvh_build(oracle.tlas_instance_boxes(ob, xf, bi))
    ref = oracle.trace_tlas(top, ob, t.inv_transforms.cpu().numpy(), bi, oracle.camera_rays(cam, w * h, w, h))
    got = hits.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    inst = got.reshape(-1, 8)[:, 3].view(np.uint32)
    hit_inst = inst[inst != 0xFFFFFFFF]
    assert hit_inst.size > 1000 and not np.any(bi[hit_inst] == 1)  # the empty BLAS is never hit


def test_bad_blas_index_reports_status():
    _, _, bs = blas_set([tri_at(2.0)])
    t = tlas.build_triangle_tlas(bs, [translate(0, 0, 0)], [0])
    t.blas_idx.fill_(5)
    hits = torch.empty(8, dtype=torch.float32, device="cuda")
    cam = dev(camera.camera([0, 0, 0], [0, 0, 1], [0, 1, 0], 0.75))
    st = t.launch_camera(cam, hits, 1, 1, 1)
    torch.cuda.synchronize()
    assert int(st.item()) & _lib.STATUS_BAD_TOPOLOGY
    b = bs.c_struct(False)
    assert _lib.load().bajo_tlas_instance_boxes(ctypes.byref(b), t.transforms.data_ptr() + 4, t.blas_idx.data_ptr(), 1,
                                                t.boxes.data_ptr(), None, None) == _lib.ERR_INVALID_ARGUMENT
