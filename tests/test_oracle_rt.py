"""CPU tests of the path-tracer pieces: Philox known answers, the shared
sin/cos polynomial, the light alias table (library host code vs oracle), and
unbiasedness of PATH / NEE / MIS on the oracle.  No GPU."""
import numpy as np
import pytest

from bajo_b200 import scenes


def test_philox_known_answers(oracle):
    """Philox-4x32-10 test vectors published with the Random123 library
    (Salmon et al., SC'11)."""
    kats = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in kats:
        assert oracle.philox4x32_10(ctr, key) == want


def test_stage_streams_are_distinct_and_deterministic(oracle):
    """Every (path, stage) owns its own stream (bajo/rt/wavefront_contract.mojo:107;
    test/rt/test_cpu.mojo:168-181)."""
    a = oracle.rt_uniform4(2026, 7, 1)
    assert np.array_equal(a, oracle.rt_uniform4(2026, 7, 1))
    others = [oracle.rt_uniform4(2026, 7, (1 << 30) | 1), oracle.rt_uniform4(2026, 8, 1),
              oracle.rt_uniform4(2027, 7, 1)]
    for o in others:
        assert not np.array_equal(a, o)
    u = np.concatenate([oracle.rt_uniform4(1, p, 3) for p in range(5000)])
    assert 0.0 <= u.min() and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01


def test_sincos_turns_accuracy(oracle):
    for u in np.linspace(0.0, 1.0, 2001, endpoint=False, dtype=np.float32):
        s, c = oracle.rt_sincos_turns(float(u))
        assert abs(s - np.sin(2 * np.pi * float(u))) < 3e-7
        assert abs(c - np.cos(2 * np.pi * float(u))) < 3e-7


def test_light_table_library_equals_oracle(lib, oracle):
    from bajo_b200 import rt
    sc = scenes.small_rt_scene()
    a = rt.build_lights(sc)
    b = oracle.rt_build_lights(sc)
    assert a[1] == b[1] == 2
    assert np.float32(a[2]) == np.float32(b[2])
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))


def test_alias_table_reconstructs_power(lib, oracle):
    """The alias table samples each light with probability weight / total
    (test/rt/test_cpu.mojo:138-166)."""
    from bajo_b200 import rt
    rng = np.random.default_rng(3)
    n = 9
    verts = rng.random((n, 9)).astype(np.float32)
    em = rng.uniform(0.5, 20.0, (n, 3)).astype(np.float32)
    surf = np.array([scenes.surface_id(scenes.MAT_EMISSIVE, i) for i in range(n)], np.uint32)
    sc = scenes.RtScene(verts, surf, np.zeros(3, np.float32), em)
    lights, count, total = rt.build_lights(sc)
    rec = lights.reshape(-1, 16)[:count]
    prob = rec[:, 12].astype(np.float64)
    alias = rec[:, 13].view(np.uint32)
    p = prob.copy()
    for j in range(count):
        if alias[j] != j:
            p[alias[j]] += 1.0 - prob[j]
    p /= count
    v = verts.reshape(n, 3, 3).astype(np.float64)
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    w = area * em.mean(axis=1)
    assert np.allclose(p, w / w.sum(), atol=1e-5)


@pytest.mark.parametrize("algorithm", [0, 3, 4])
def test_oracle_render_deterministic(oracle, algorithm):
    sc = scenes.small_rt_scene()
    a = oracle.render(sc, sc.camera, 16, 9, 2, algorithm=algorithm, threads=1)
    b = oracle.render(sc, sc.camera, 16, 9, 2, algorithm=algorithm, threads=4)
    assert np.array_equal(a, b)


def test_path_nee_mis_are_unbiased(oracle):
    """All three estimators converge to the same image: per-image mean within
    4 standard errors, and few pixels beyond 4 sigma."""
    sc = scenes.small_rt_scene()
    w, h, spp = 24, 14, 256
    res = {}
    for alg in (0, 3, 4):
        img, smp = oracle.render(sc, sc.camera, w, h, spp, algorithm=alg, return_samples=True, seed=11 + alg)
        m = smp.astype(np.float64).mean(axis=2)
        se = smp.astype(np.float64).std(axis=2, ddof=1) / np.sqrt(spp)
        res[alg] = (m, se)
    for a, b in ((0, 4), (3, 4), (0, 3)):
        ma, sa = res[a]
        mb, sb = res[b]
        diff = ma.mean() - mb.mean()
        se_img = np.sqrt(((sa ** 2) + (sb ** 2)).sum()) / sa.size
        assert abs(diff) < 4 * se_img + 1e-6, (a, b, diff, se_img)
    # per pixel only between the light-tailed estimators (PATH's rare direct
    # light hits make its per-pixel sample variance unreliable at this spp)
    (ma, sa), (mb, sb) = res[3], res[4]
    z = np.abs(ma - mb) / np.sqrt(sa ** 2 + sb ** 2 + 1e-12)
    assert (z > 4).mean() < 0.01


def test_guiding_scene_variants():
    """The indirectly lit scenes of the guiding comparisons: the sphere
    workload with its light turned to face the ceiling (same geometry), and
    the two-room door scene."""
    from bajo_b200 import scenes
    base = scenes.spheres_in_box()
    up = scenes.spheres_in_box(light_up=True)
    assert up.vertices.shape == base.vertices.shape
    tri = up.vertices.reshape(-1, 3, 3).astype(np.float64)
    light = tri[12:14]  # the light quad follows the 12 box triangles
    nrm = np.cross(light[:, 1] - light[:, 0], light[:, 2] - light[:, 0])
    assert np.all(nrm[:, 1] > 0) and np.allclose(light[:, :, 1], 0.85)
    assert float(up.emissives.ravel()[0]) == 4 * float(base.emissives.ravel()[0])
    door = scenes.door_scene()
    t = door.vertices.reshape(-1, 3, 3)
    assert np.all((t >= -1e-6) & (t <= 1 + 1e-6))
    wall = t[12:18]
    assert np.allclose(wall[:, :, 2], 0.5)
