"""PBRT reader (bajo/parser/pbrt): the reference's own example scene gives
the counts its test expects (test/pbrt/test_pbrt.mojo:11-24), transforms,
scopes, materials, lights, includes and shapes give known answers, every
unsupported or malformed input raises, and a parsed scene renders through the
oracle with light reaching the camera."""
import math
import os

import numpy as np
import pytest

from bajo_b200 import pbrt, scenes

REFERENCE_ROOT = os.environ.get("BAJO_REFERENCE_ROOT", "/root/reference")
SHOWCASE = os.path.join(REFERENCE_ROOT, "examples", "scenes", "pbrt_showcase.pbrt")


@pytest.mark.skipif(not os.path.exists(SHOWCASE), reason="reference example scenes not present")
def test_reference_showcase_counts():
    s = pbrt.read_pbrt(SHOWCASE)
    assert (s.width, s.height, s.samples_per_pixel, s.max_depth) == (640, 480, 64, 10)
    assert s.integrator == "path"
    assert s.n_spheres == 3 and s.n_triangles == 10
    assert (len(s.lambertians), len(s.metals), len(s.dielectrics), len(s.emissives)) == (4, 1, 1, 1)
    from bajo_b200 import rt
    assert rt.build_lights(s.to_rt_scene(1))[1] == 2  # the light quad's two triangles


HEADER = """Film "rgb" "integer xresolution" [6] "integer yresolution" [5]   # a comment
ColorSpace "srgb"
PixelFilter "box" "float xradius" [0.5]
Accelerator "bvh" "integer maxnodeprims" [2]
Option "bool disablepixeljitter" true
"""


def test_defaults_and_header():
    s = pbrt.parse_pbrt(HEADER + 'WorldBegin\nShape "sphere"\n')
    assert (s.width, s.height, s.samples_per_pixel, s.max_depth, s.rng_seed) == (6, 5, 16, 8, 2026)
    np.testing.assert_array_equal(s.camera_origin, [0, 0, 5])
    np.testing.assert_array_equal(s.camera_target, [0, 0, 0])
    assert s.camera_fov == 45.0
    assert s.sphere_radii.tolist() == [1.0]
    assert s.sphere_surfaces.tolist() == [scenes.surface_id(scenes.MAT_LAMBERTIAN, 0)]
    np.testing.assert_array_equal(s.lambertians, [[0.5, 0.5, 0.5]])


def test_named_material_translate_scale():
    src = HEADER + """WorldBegin
MakeNamedMaterial "ochre" "string type" "diffuse" "rgb reflectance" [0.6 0.4 0.1]
AttributeBegin
  NamedMaterial "ochre"
  Translate -1 0.5 4
  Scale 3 3 3
  Shape "sphere" "float radius" [0.25]
AttributeEnd
Shape "sphere" "float radius" 2
WorldEnd
"""
    s = pbrt.parse_pbrt(src)
    np.testing.assert_allclose(s.sphere_centers, [[-1, 0.5, 4], [0, 0, 0]])
    np.testing.assert_allclose(s.sphere_radii, [0.75, 2.0])
    lam = scenes.surface_id(scenes.MAT_LAMBERTIAN, 1)
    assert s.sphere_surfaces.tolist() == [lam, scenes.surface_id(scenes.MAT_LAMBERTIAN, 0)]
    np.testing.assert_allclose(s.lambertians[1], [0.6, 0.4, 0.1])


def test_material_models():
    src = """WorldBegin
Material "coateddiffuse" "rgb reflectance" [0.3 0.2 0.1] "float roughness" [0.01]
Shape "sphere"
Material "matte"
Shape "sphere"
Material "conductor" "rgb reflectance" [0.8 0.7 0.6] "float roughness" [2.5]
Shape "sphere"
Material "metal"
Shape "sphere"
Material "glass" "float eta" [1.33]
Shape "sphere"
Material "dielectric"
Shape "sphere"
"""
    s = pbrt.parse_pbrt(src)
    kinds = [int(x) >> 28 for x in s.sphere_surfaces]
    assert kinds == [0, 0, 1, 1, 2, 2]
    np.testing.assert_allclose(s.lambertians[1:], [[0.3, 0.2, 0.1], [0.5, 0.5, 0.5]])
    np.testing.assert_allclose(s.metals, [[0.8, 0.7, 0.6, 1.0], [0.9, 0.9, 0.9, 0.05]])  # roughness clamps to 1
    np.testing.assert_allclose(s.dielectrics, [1.33, 1.5])


def test_area_lights_are_scoped_and_per_shape():
    src = """WorldBegin
AttributeBegin
AreaLightSource "diffuse" "rgb L" [2 4 6] "float scale" [0.5]
Shape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0]
Shape "sphere" "float radius" 0.1
AttributeEnd
Shape "trianglemesh" "point P" [0 0 1 1 0 1 0 1 1]
"""
    s = pbrt.parse_pbrt(src)
    np.testing.assert_allclose(s.emissives, [[1, 2, 3], [1, 2, 3]])
    assert [int(x) for x in s.triangle_surfaces] == [scenes.surface_id(3, 0), scenes.surface_id(0, 0)]
    assert s.sphere_surfaces.tolist() == [scenes.surface_id(3, 1)]


def test_rotate_and_matrices():
    s = pbrt.parse_pbrt("""WorldBegin
AttributeBegin
Rotate 90 0 0 2
Shape "trianglemesh" "point3 P" [1 0 0  0 1 0  0 0 1]
AttributeEnd
AttributeBegin
Transform [1 0 0 5  0 2 0 6  0 0 3 7  0 0 0 1]
ConcatTransform [1 0 0 1  0 1 0 1  0 0 1 1  0 0 0 1]
Shape "trianglemesh" "point3 P" [0 0 0  1 0 0  0 1 0]
AttributeEnd
TransformBegin
Translate 9 9 9
TransformEnd
Identity
Shape "trianglemesh" "point3 P" [0 0 0  1 0 0  0 1 0]
""")
    t = s.triangle_vertices
    np.testing.assert_allclose(t[0], [[0, 1, 0], [-1, 0, 0], [0, 0, 1]], atol=1e-6)
    np.testing.assert_allclose(t[1], [[6, 8, 10], [7, 8, 10], [6, 10, 10]])
    np.testing.assert_allclose(t[2], [[0, 0, 0], [1, 0, 0], [0, 1, 0]])
    # an arbitrary axis: the map is a rotation
    r = pbrt._rotation(37.0, 1.0, -2.0, 0.5)
    m = np.array(r.m, np.float64).reshape(3, 4)[:, :3]
    np.testing.assert_allclose(m @ m.T, np.eye(3), atol=2e-6)
    assert abs(np.linalg.det(m) - 1.0) < 2e-6
    assert abs(np.trace(m) - (1 + 2 * math.cos(math.radians(37.0)))) < 2e-6


def test_compose_is_float32_in_order():
    a = pbrt.Affine([0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.1, 1.2, 1.3])
    b = pbrt.Affine([1.7, -0.3, 0.25, 3.0, 0.1, 2.2, -1.5, 0.5, 0.3, 0.4, 0.9, -2.0])
    c = a.compose(b)
    am = np.array(a.m, np.float32).reshape(3, 4)
    bm = np.array(b.m, np.float32).reshape(3, 4)
    for r in range(3):
        for k in range(4):
            want = am[r, 0] * bm[0, k] + am[r, 1] * bm[1, k] + am[r, 2] * bm[2, k]
            if k == 3:
                want = want + am[r, 3]
            assert c.m[4 * r + k] == want and isinstance(c.m[4 * r + k], np.float32)


def test_reverse_orientation_and_unindexed_meshes():
    s = pbrt.parse_pbrt("""WorldBegin
AttributeBegin
ReverseOrientation
Shape "trianglemesh" "point3 P" [0 0 0  1 0 0  0 1 0  2 0 0  3 0 0  2 1 0]
AttributeEnd
Shape "loopsubdiv" "integer levels" [2] "point3 P" [0 0 0  1 0 0  0 1 0  1 1 0] "integer indices" [0 1 2  2 1 3]
""")
    t = s.triangle_vertices
    assert t.shape == (4, 3, 3)
    np.testing.assert_array_equal(t[0], [[0, 0, 0], [0, 1, 0], [1, 0, 0]])
    np.testing.assert_array_equal(t[1], [[2, 0, 0], [2, 1, 0], [3, 0, 0]])
    np.testing.assert_array_equal(t[3], [[0, 1, 0], [1, 0, 0], [1, 1, 0]])


def test_camera_sampler_integrator():
    s = pbrt.parse_pbrt("""LookAt 1 2 3  0 0 0  0 0 1
Camera "perspective" "float fov" 30
Sampler "halton" "integer pixelsamples" [4]
Integrator "path" "integer maxdepth" [5]
WorldBegin
Shape "sphere"
""")
    np.testing.assert_array_equal(s.camera_origin, [1, 2, 3])
    np.testing.assert_array_equal(s.camera_up, [0, 0, 1])
    assert (s.camera_fov, s.samples_per_pixel, s.max_depth) == (30.0, 4, 5)
    from bajo_b200 import camera
    np.testing.assert_array_equal(s.camera(), camera.camera_from_vfov([1, 2, 3], [0, 0, 0], [0, 0, 1], 30.0))


def test_include_resolves_against_including_file():
    loader = pbrt.MemoryPbrtTextLoader()
    loader.add_file("a/main.pbrt", 'WorldBegin\nInclude "sub/b.pbrt"\n')
    loader.add_file("a/sub/b.pbrt", 'Include "c.pbrt"\nShape "sphere" "float radius" 2\n')
    loader.add_file("a/sub/c.pbrt", 'Shape "sphere" "float radius" 1\n')
    s = pbrt.read_pbrt("a/main.pbrt", loader)
    assert s.sphere_radii.tolist() == [1.0, 2.0]


def test_include_from_disk(tmp_path):
    (tmp_path / "inc.pbrt").write_text('Material "conductor"\nShape "sphere"\n')
    (tmp_path / "main.pbrt").write_text('WorldBegin\nInclude "inc.pbrt"\n')
    s = pbrt.read_pbrt(str(tmp_path / "main.pbrt"))
    assert len(s.metals) == 1 and s.n_spheres == 1


@pytest.mark.parametrize("src", [
    'Integrator "bdpt"\nWorldBegin\nShape "sphere"',
    'WorldBegin\nShape "plymesh" "string filename" "x.ply"',
    'WorldBegin\nScale 1 2 1\nShape "sphere"',
    'WorldBegin\nShape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0] "integer indices" [0 1 3]',
    'WorldBegin\nShape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0] "integer indices" [0 1]',
    'WorldBegin\nShape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1]',
    'WorldBegin\nShape "trianglemesh" "point3 P" [0 0 0 1 0 0] ',
    'WorldBegin\nShape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0] "integer indices" [0 1 1.5]',
    'Camera "orthographic"\nWorldBegin\nShape "sphere"',
    'ColorSpace "aces2065-1"\nWorldBegin\nShape "sphere"',
    'WorldBegin\nMaterial "hair"\nShape "sphere"',
    'WorldBegin\nNamedMaterial "nope"\nShape "sphere"',
    'WorldBegin\nAreaLightSource "goniometric"\nShape "sphere"',
    'WorldBegin\nLightSource "point"\nShape "sphere"',
    'WorldBegin\nAttributeEnd\nShape "sphere"',
    'WorldBegin\nTransformEnd\nShape "sphere"',
    'WorldBegin\nAttributeBegin\nShape "sphere"',
    'WorldBegin\nTransformBegin\nShape "sphere"',
    'WorldBegin\n',
    'WorldBegin\nRotate 10 0 0 0\nShape "sphere"',
    'WorldBegin\nTransform [1 0 0 0 0 1 0 0 0 0 1 0 0 0 1 1]\nShape "sphere"',
    'WorldBegin\nTransform [1 0 0 0 0 1 0 0 0 0 1 0]\nShape "sphere"',
    'WorldBegin\nTransform 1 0 0 0\nShape "sphere"',
    'WorldBegin\nShape "sphere" "float radius" [abc]',
    'WorldBegin\nShape "sphere" "float radius" [1e]',
    'WorldBegin\nShape "sphere" "float radius" [0.5',
    'WorldBegin\nShape "sphere" "float radius"',
    'WorldBegin\nShape "sphere" "string name',
    'Film "rgb" "integer xresolution" [2.5]\nWorldBegin\nShape "sphere"',
    'WorldBegin\nMaterial "diffuse" "rgb reflectance" [0.1 0.2]\nShape "sphere"',
    '"WorldBegin"\nShape "sphere"',
    'WorldBegin\nTranslate 1 2',
    'WorldBegin\nInclude "missing.pbrt"\nShape "sphere"',
])
def test_rejects_unsupported_and_malformed(src):
    with pytest.raises(pbrt.PbrtParseError):
        pbrt.parse_pbrt(src)


def test_include_nesting_limit():
    loader = pbrt.MemoryPbrtTextLoader()
    loader.add_file("loop.pbrt", 'Include "loop.pbrt"\n')
    with pytest.raises(pbrt.PbrtParseError, match="nesting"):
        pbrt.read_pbrt("loop.pbrt", loader)


def test_error_names_the_line():
    with pytest.raises(pbrt.PbrtParseError, match="line 3"):
        pbrt.parse_pbrt('WorldBegin\nShape "sphere"\nMakeBelieve 1\n')


def test_tessellation_keeps_surfaces_and_radius():
    s = pbrt.parse_pbrt("""WorldBegin
Material "glass"
Translate 1 2 3
Shape "sphere" "float radius" 0.5
Identity
Material "diffuse" "rgb reflectance" [0.2 0.3 0.4]
Shape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0]
""")
    rs = s.to_rt_scene(2)
    assert rs.n_tris == 1 + 320
    assert int(rs.surfaces[0]) == scenes.surface_id(0, 1)
    assert set(int(x) for x in rs.surfaces[1:]) == {scenes.surface_id(scenes.MAT_DIELECTRIC, 0)}
    v = rs.vertices.reshape(-1, 3)[3:]
    np.testing.assert_allclose(np.linalg.norm(v - [1, 2, 3], axis=1), 0.5, rtol=1e-6)
    assert rs.metals is None and rs.dielectrics.tolist() == [1.5]


CORNELL = """LookAt 0 1 3.2  0 1 0  0 1 0
Camera "perspective" "float fov" [45]
Film "rgb" "integer xresolution" [12] "integer yresolution" [10]
Sampler "independent" "integer pixelsamples" [4]
Integrator "path" "integer maxdepth" [6]
WorldBegin
MakeNamedMaterial "wall" "string type" "diffuse" "rgb reflectance" [0.7 0.7 0.7]
MakeNamedMaterial "chrome" "string type" "conductor" "rgb reflectance" [0.9 0.9 0.8] "float roughness" [0.0]
AttributeBegin
NamedMaterial "wall"
Shape "trianglemesh" "point3 P" [-1 0 -1  1 0 -1  1 0 1  -1 0 1] "integer indices" [0 2 1  0 3 2]
Shape "trianglemesh" "point3 P" [-1 0 -1  -1 2 -1  1 2 -1  1 0 -1] "integer indices" [0 2 1  0 3 2]
AttributeEnd
AttributeBegin
AreaLightSource "diffuse" "rgb L" [6 6 6]
ReverseOrientation
Shape "trianglemesh" "point3 P" [-0.3 1.95 -0.3  0.3 1.95 -0.3  0.3 1.95 0.3  -0.3 1.95 0.3]
    "integer indices" [0 1 2  0 2 3]
AttributeEnd
AttributeBegin
NamedMaterial "chrome"
Translate -0.4 0.35 0
Shape "sphere" "float radius" [0.35]
AttributeEnd
AttributeBegin
Material "dielectric" "float eta" [1.5]
Translate 0.45 0.3 0.2
Shape "sphere" "float radius" [0.3]
AttributeEnd
WorldEnd
"""


def test_parsed_scene_renders_with_oracle(oracle):
    s = pbrt.parse_pbrt(CORNELL)
    rs = s.to_rt_scene(2)
    img = oracle.render(rs, rs.camera, s.width, s.height, s.samples_per_pixel, max_depth=s.max_depth,
                        seed=s.rng_seed, algorithm=4)
    assert img.shape == (10, 12, 3) and np.all(np.isfinite(img)) and img.sum() > 0.0


@pytest.mark.parametrize("text,value", [("1e-3", 0.001), ("+2", 2.0), (".5", 0.5), ("-0", 0.0), ("3.", 3.0),
                                        ("12.5E+1", 125.0), ("", 0.0)])
def test_number_tokens(text, value):
    assert pbrt.parse_f32(text) == np.float32(value)


@pytest.mark.parametrize("text", ["1.5x", "0x10", "nan", "inf", "1e", "--1", "1e400"])
def test_bad_number_tokens(text):
    with pytest.raises(pbrt.PbrtParseError):
        pbrt.parse_f32(text)


def test_integer_tokens():
    assert pbrt.parse_int("3.0") == 3 and pbrt.parse_int("-7") == -7
    with pytest.raises(pbrt.PbrtParseError):
        pbrt.parse_int("3.25")
