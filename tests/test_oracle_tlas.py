"""CPU checks of the two-level restatement (no GPU): the known answers of the
reference's TLAS tests (test/bvh/gpu/test_blas_tlas.mojo:128-237: the
instance's BLAS index is used; the closest hit wins across different BLASes),
instance boxes contain their transformed triangles, and instanced closest hits
agree with a brute force over the instanced triangles moved to world space."""
import numpy as np
import pytest

from bajo_b200 import scenes
from bajo_b200.tlas import invert_affine
from oracle import oracle


def tri_at(z):
    return np.array([[-1, -1, z, 1, -1, z, 0, 1, z]], np.float32)


def translate(x, y, z):
    return np.array([1, 0, 0, x, 0, 1, 0, y, 0, 0, 1, z], np.float32)


def ray(o, d):
    r = np.zeros((8, 1), np.float32)
    r[0:3, 0], r[4:7, 0], r[7, 0] = o, d, 3.4028235e38
    return r.reshape(-1)


def two_level(blas_meshes, transforms, blas_idx):
    verts = np.concatenate([m.reshape(-1) for m in blas_meshes])
    counts = [m.reshape(-1, 9).shape[0] for m in blas_meshes]
    seg = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    blas = oracle.lbvh_build(verts, seg)
    xf = np.asarray(transforms, np.float32).reshape(-1, 12)
    boxes = oracle.tlas_instance_boxes(blas, xf, blas_idx)
    top = oracle.lbvh_build(boxes)
    return blas, top, invert_affine(xf), boxes


def hit_of(h):
    h = h.reshape(-1, 8)[0]
    return float(h[7]), int(h[2:3].view(np.uint32)[0]), int(h[3:4].view(np.uint32)[0])


def test_instance_uses_its_blas_index():
    blas, top, inv, _ = two_level([tri_at(2.0), tri_at(6.0)], [translate(-10, 0, 0), translate(10, 0, 0)], [0, 1])
    t, prim, inst = hit_of(oracle.trace_tlas(top, blas, inv, [0, 1], ray([10, 0, 0], [0, 0, 1])))
    assert abs(t - 6.0) < 1e-5 and prim == 0 and inst == 1


def test_closest_hit_across_different_blas():
    blas, top, inv, _ = two_level([tri_at(8.0), tri_at(3.0)], [translate(0, 0, 0), translate(0, 0, 0)], [0, 1])
    r = ray([0, 0, 0], [0, 0, 1])
    t, prim, inst = hit_of(oracle.trace_tlas(top, blas, inv, [0, 1], r))
    assert abs(t - 3.0) < 1e-5 and prim == 0 and inst == 1
    occ = oracle.trace_tlas(top, blas, inv, [0, 1], r, any_hit=True).reshape(-1, 8)[0]
    assert occ[7] == 0.0 and int(occ[2:3].view(np.uint32)[0]) == oracle.SENTINEL
    assert int(occ[3:4].view(np.uint32)[0]) in (0, 1)


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


def test_boxes_contain_transformed_triangles():
    meshes = [scenes.random_triangles(n, seed=n).reshape(-1, 9) for n in (50, 300, 1)]
    xf, bi = random_instances(40, 3, 1)
    blas, top, inv, boxes = two_level(meshes, xf, bi)
    for i in range(40):
        v = meshes[bi[i]].reshape(-1, 3).astype(np.float64)
        m = xf[i].reshape(3, 4).astype(np.float64)
        w = v @ m[:, :3].T + m[:, 3]
        assert np.all(w >= boxes[i, 0:3] - 1e-4) and np.all(w <= boxes[i, 3:6] + 1e-4)


def test_hits_agree_with_world_space_brute_force():
    meshes = [scenes.random_triangles(n, seed=n, spread=0.1).reshape(-1, 9) for n in (200, 500, 60)]
    xf, bi = random_instances(30, 3, 2)
    blas, top, inv, _ = two_level(meshes, xf, bi)
    rng = np.random.default_rng(3)
    m = 4000
    rays = np.zeros((8, m), np.float32)
    rays[0:3] = rng.uniform(-6, 6, (3, m))
    d = rng.normal(size=(3, m))
    rays[4:7] = d / np.linalg.norm(d, axis=0)
    rays[7] = 1e30
    got = oracle.trace_tlas(top, blas, inv, bi, rays.reshape(-1), tri_mode=0).reshape(-1, 8)
    world, owner = [], []
    for i in range(len(bi)):
        v = meshes[bi[i]].reshape(-1, 3).astype(np.float64)
        mm = xf[i].reshape(3, 4).astype(np.float64)
        world.append((v @ mm[:, :3].T + mm[:, 3]).astype(np.float32).reshape(-1, 9))
        owner += [(i, p) for p in range(meshes[bi[i]].shape[0])]
    ref = oracle.trace_brute(np.concatenate(world), rays.reshape(-1), 0).reshape(-1, 8)
    ref_owner = [owner[int(p)] if int(p) != oracle.SENTINEL else None for p in ref[:, 2].view(np.uint32)]
    got_owner = [(int(i), int(p)) if int(p) != oracle.SENTINEL else None
                 for i, p in zip(got[:, 3].view(np.uint32), got[:, 2].view(np.uint32))]
    same = np.mean([a == b for a, b in zip(ref_owner, got_owner)])
    assert same > 0.995 and sum(r is not None for r in ref_owner) > 200
    hit = np.array([a is not None and a == b for a, b in zip(ref_owner, got_owner)])
    np.testing.assert_allclose(got[hit, 7], ref[hit, 7], rtol=2e-4)
