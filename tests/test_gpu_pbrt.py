"""GPU parity of a PBRT-described scene: the reader's scene, tessellated for
the triangle path tracer, renders on the GPU bit for bit like the oracle for
every integrator, with the file's camera, image size, samples, depth and
seed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import pbrt, rt  # noqa: E402

MAIN = """LookAt 0 1.1 3.4  0 0.9 0  0 1 0
Camera "perspective" "float fov" [42]
Film "rgb" "integer xresolution" [36] "integer yresolution" [24]
Sampler "independent" "integer pixelsamples" [6]
Integrator "path" "integer maxdepth" [10]
WorldBegin
MakeNamedMaterial "white" "string type" "diffuse" "rgb reflectance" [0.73 0.73 0.73]
MakeNamedMaterial "red" "string type" "matte" "rgb reflectance" [0.65 0.06 0.05]
MakeNamedMaterial "brushed" "string type" "conductor" "rgb reflectance" [0.95 0.64 0.54] "float roughness" [0.2]
AttributeBegin
NamedMaterial "white"
Shape "trianglemesh" "point3 P" [-1 0 -1  1 0 -1  1 0 1  -1 0 1] "integer indices" [0 2 1  0 3 2]
Shape "trianglemesh" "point3 P" [-1 0 -1  -1 2 -1  1 2 -1  1 0 -1] "integer indices" [0 2 1  0 3 2]
Shape "trianglemesh" "point3 P" [-1 2 -1  -1 2 1  1 2 1  1 2 -1] "integer indices" [0 2 1  0 3 2]
AttributeEnd
AttributeBegin
NamedMaterial "red"
Rotate 90 0 0 1
Translate 1 1 0
Shape "trianglemesh" "point3 P" [-1 0 -1  -1 0 1  1 0 1  1 0 -1] "integer indices" [0 2 1  0 3 2]
AttributeEnd
AttributeBegin
AreaLightSource "diffuse" "rgb L" [10 9 8] "float scale" [1.5]
Shape "trianglemesh" "point3 P" [-0.25 1.98 -0.25  0.25 1.98 -0.25  0.25 1.98 0.25  -0.25 1.98 0.25]
    "integer indices" [0 1 2  0 2 3]
AttributeEnd
Include "objects.pbrt"
WorldEnd
"""

OBJECTS = """AttributeBegin
NamedMaterial "brushed"
Translate -0.45 0.3 -0.2
Shape "sphere" "float radius" [0.3]
AttributeEnd
AttributeBegin
Material "glass" "float eta" [1.45]
Translate 0.4 0.35 0.3
Scale 0.5 0.5 0.5
Shape "sphere" "float radius" [0.7]
AttributeEnd
AttributeBegin
Material "metal" "rgb reflectance" [0.9 0.9 0.9] "float roughness" [0]
Translate 0.3 0.8 -0.6
Shape "sphere" "float radius" [0.2]
AttributeEnd
"""


@pytest.fixture(scope="module")
def scene():
    loader = pbrt.MemoryPbrtTextLoader()
    loader.add_file("box/main.pbrt", MAIN)
    loader.add_file("box/objects.pbrt", OBJECTS)
    s = pbrt.read_pbrt("box/main.pbrt", loader)
    rs = s.to_rt_scene(3)
    return s, rs, rt.GpuRtTriangleScene(rs, bvh_policy="lbvh")


@pytest.mark.parametrize("algorithm", [rt.PATH, rt.NEE, rt.MIS])
def test_pbrt_scene_renders_like_oracle(oracle, scene, algorithm):
    s, rs, gsc = scene
    settings = s.render_settings()
    ws = rt.RenderWorkspace(settings, algorithm)
    img = rt.render_gpu_triangles(settings, rs.camera, gsc, algorithm, workspace=ws)
    torch.cuda.synchronize()
    assert ws.status() == 0
    ref = oracle.render(rs, rs.camera, s.width, s.height, s.samples_per_pixel, max_depth=s.max_depth,
                        seed=s.rng_seed, algorithm=algorithm)
    got = img.cpu().numpy()
    assert got.shape == (24, 36, 3)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert got.mean() > 0.02
