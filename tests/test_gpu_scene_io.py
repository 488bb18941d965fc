"""GPU check of the OBJ path into the C ABI: a mesh written as OBJ text, read
and packed by scene_io, built by bajo_lbvh_build and traced from a camera,
gives the oracle's hits bit for bit; its shading image is written as PPM."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from bajo_b200 import bvh, camera, scene_io  # noqa: E402


def _terrain_obj(nx, ny):
    xs, ys = np.meshgrid(np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1))
    zs = 0.1 * np.sin(6 * xs) * np.cos(5 * ys)
    lines = [f"v {x:.6f} {y:.6f} {z:.6f}" for x, y, z in zip(xs.ravel(), ys.ravel(), zs.ravel())]
    for y in range(ny):
        for x in range(nx):
            a = y * (nx + 1) + x + 1
            lines.append(f"f {a} {a + 1} {a + nx + 2} {a + nx + 1}")
    return "\n".join(lines) + "\n"


def test_obj_mesh_builds_and_traces_like_the_oracle(oracle, tmp_path):
    path = tmp_path / "terrain.obj"
    path.write_text(_terrain_obj(120, 90))
    tris = scene_io.pack_obj_triangles(str(path))
    assert tris.shape == (2 * 120 * 90, 9)
    tree = bvh.build_triangle_bvh(torch.from_numpy(tris).cuda())
    cam = camera.camera([0.5, 0.5, -0.6], [0.5, 0.5, 0.0], [0, 1, 0], 0.9)
    w, h = 160, 120
    hits = torch.empty(8 * w * h, dtype=torch.float32, device="cuda")
    tree.launch_camera(torch.from_numpy(cam).cuda(), hits, w * h, w, h)
    torch.cuda.synchronize()
    got = hits.cpu().numpy()
    rays = oracle.camera_rays(cam, w * h, w, h)
    ref = oracle.trace_bvh2(oracle.lbvh_build(tris), rays)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert (got.reshape(-1, 8)[:, 2].view(np.uint32) != 0xFFFFFFFF).mean() > 0.5
    normals = np.abs(got.reshape(-1, 8)[:, 4:7])
    out = tmp_path / "normals.ppm"
    scene_io.write_ppm_from_colors(str(out), w, h, normals)
    img = scene_io.read_ppm(str(out))
    assert img.shape == (h, w, 3) and img.max() > 0
