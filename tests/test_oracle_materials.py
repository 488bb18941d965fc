"""CPU checks of the metal and dielectric shading restatement (no GPU): the
series power against numpy, a known answer (a horizontal view through glass
or at a mirror sees the horizon sky exactly: every path leaves horizontally,
straight on or reversed, and the sky depends only on the height of the
direction), and unbiasedness of PATH against MIS on mirror and glass
spheres."""
import numpy as np
import pytest

from bajo_b200 import scenes
from bajo_b200.camera import camera_from_vfov
from oracle import oracle


def test_series_pow_accuracy():
    lib = oracle.lib()
    xs = np.concatenate([np.linspace(1e-6, 1.0, 400), [0.5, 0.999999, 1.0]]).astype(np.float32)
    for y in (0.0, 0.01, 0.3, 1.0, 2.0, 7.5, 98.0, 798.0):
        for x in xs:
            got = lib.bo_rt_series_pow(float(x), float(y))
            want = float(np.float64(x) ** y)
            # the float rounding of z = y log2 x is amplified |z| times by 2^z
            z = abs(y * np.log2(np.float64(x))) if x > 0 else 0.0
            assert abs(got - want) <= (2e-6 + 1.2e-7 * z) * want + 1e-37, (x, y, got, want)
    assert lib.bo_rt_series_pow(0.0, 2.0) == 0.0 and lib.bo_rt_series_pow(0.0, 0.0) == 1.0


def _pane(kind_surface, z=0.5):
    # a 4 x 4 quad facing the camera at depth z, both windings (a slab of zero thickness for glass)
    v = np.array([[-2, -2, z], [2, -2, z], [2, 2, z], [-2, -2, z], [2, 2, z], [-2, 2, z]], np.float32)
    back = v[[0, 2, 1, 3, 5, 4]] + np.array([0, 0, 0.01], np.float32)
    tris = np.concatenate([v, back]).reshape(-1, 9)
    return tris, np.full(4, kind_surface, np.uint32)


@pytest.mark.parametrize("kind", ["glass", "mirror"])
def test_horizontal_view_sees_horizon_sky(kind):
    if kind == "glass":
        tris, surf = _pane(scenes.surface_id(scenes.MAT_DIELECTRIC, 0))
        extra = dict(dielectrics=np.array([1.5], np.float32))
    else:
        tris, surf = _pane(scenes.surface_id(scenes.MAT_METAL, 0))
        extra = dict(metals=np.array([[1.0, 1.0, 1.0, 0.0]], np.float32))
    sc = scenes.RtScene(tris, surf, np.zeros((1, 3), np.float32), np.zeros((1, 3), np.float32), **extra)
    cam = camera_from_vfov([0.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, 1.0, 0.0], 0.01)
    img = oracle.render(sc, cam, 8, 8, 4, max_depth=8, algorithm=0)
    horizon = np.array([0.75, 0.85, 1.0], np.float32)  # sky_color at direction height 0
    assert np.allclose(img, horizon, atol=2e-4), img.reshape(-1, 3)[:4]


def test_estimators_agree_on_mirror_and_glass():
    """PATH, NEE and MIS converge to the same image with mirror and glass
    spheres.  Depth 32: glass and mirrors lengthen paths, and at a shallow
    limit NEE / MIS keep the last vertex's light sample that PATH cannot
    reach (at depth 8 PATH is 3% darker here).  NEE and MIS, both
    light-sampled, must agree within 4 standard errors; PATH, heavy-tailed,
    within 4% of them -- a lost delta flag (no emission after glass or a
    mirror under NEE) costs far more."""
    sc = scenes.materials_in_box(n_spheres=6, subdivisions=2, kinds=(1, 3))
    w, h, spp = 10, 6, 1024
    res = {}
    for alg in (0, 3, 4):
        _, smp = oracle.render(sc, sc.camera, w, h, spp, max_depth=32, algorithm=alg, return_samples=True,
                               seed=31 + alg)
        s = smp.astype(np.float64)
        res[alg] = (s.mean(), np.sqrt((s.std(axis=2, ddof=1) ** 2 / spp).sum()) / (w * h * 3))
    (mn, sn), (mm, sm) = res[3], res[4]
    assert abs(mn - mm) < 4 * np.hypot(sn, sm)
    assert abs(res[0][0] - mm) < 0.04 * mm
