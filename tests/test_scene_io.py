"""CPU tests of the OBJ/MTL reader and the image writers.

The OBJ cases are the reference's own (test/obj/test_obj.mojo:23-318), with
the same inputs and expected values; the PPM checks follow
write_ppm_from_colors (bajo/rt/cpu/depth_first.mojo:287-315).  A packed OBJ
mesh also goes through the oracle build and traversal."""
import numpy as np
import pytest

from bajo_b200.scene_io import (MemoryObjTextLoader, ObjParseError, color_to_bytes, pack_triangles, parse_obj,
                                read_obj, read_ppm, triangulated_indices, write_npy, write_ppm_from_colors)


def test_basic_triangle():
    mesh = parse_obj("v 0 0 0\nv 1 0 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 0 1\nvn 0 0 1\nf 1/1/1 2/2/1 3/3/1",
                     "triangle.obj")
    assert mesh.position_count(include_dummy=False) == 3
    assert mesh.texcoord_count(include_dummy=False) == 3
    assert mesh.normal_count(include_dummy=False) == 1
    assert mesh.face_count() == 1 and mesh.index_count() == 3
    assert (mesh.indices[0].p, mesh.indices[0].t, mesh.indices[0].n) == (1, 1, 1)
    assert (mesh.indices[2].p, mesh.indices[2].t, mesh.indices[2].n) == (3, 3, 1)


def test_negative_indices_and_triangulation():
    mesh = parse_obj("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf -4 -3 -2 -1", "quad.obj")
    tris = triangulated_indices(mesh)
    assert mesh.face_vertices[0] == 4
    assert mesh.indices[0].p == 1 and mesh.indices[3].p == 4
    assert [t.p for t in tris] == [1, 2, 3, 1, 3, 4]


@pytest.mark.parametrize("text", ["v 0 0 0\nf 2 1 1", "v 0 0 0\nf -2 -1 -1", "v 0 0 0\nvt 0 0\nf 1/2 1/1 1/1",
                                  "v 0 0 0\nvn 0 0 1\nf 1//2 1//1 1//1", "v 0 0 0\nf 999999999999999999999 1 1",
                                  "v 0 0 0\nvt 0 0\nvn 0 0 1\nf 1/1/1 1/1 1/1/1"])
def test_face_indices_are_range_validated(text):
    with pytest.raises(ObjParseError):
        parse_obj(text, "invalid.obj")


def test_decimal_exponent_work_is_bounded():
    mesh = parse_obj("v 1e3 1e-3 1e+2", "exponents.obj")
    assert mesh.positions[3:6] == pytest.approx([1000.0, 0.001, 100.0])
    for text in ("v 1e309 0 0", "v 1e-309 0 0", "v 1e999999999999999999999 0 0"):
        with pytest.raises(ObjParseError):
            parse_obj(text, "invalid.obj")


def test_vertex_colors_lazy_fill():
    mesh = parse_obj("v 0 0 0\nv 1 0 0 0.25 0.5 0.75\nv 2 0 0", "colors.obj")
    assert mesh.color_count() == 4
    assert mesh.colors == pytest.approx([1, 1, 1, 1, 1, 1, 0.25, 0.5, 0.75, 1, 1, 1])


def test_groups_objects_and_lines():
    mesh = parse_obj("o Cube\ng Front\nv 0 0 0\nv 1 0 0\nv 0 1 0\nl 1 2\nf 1 2 3", "groups.obj")
    tris = triangulated_indices(mesh)
    assert mesh.face_count() == 2 and mesh.face_lines == [1, 0] and len(tris) == 3
    assert mesh.object_count() == 1 and mesh.objects[0].name == "Cube" and mesh.objects[0].face_count == 2
    assert mesh.group_count() == 1 and mesh.groups[0].name == "Front" and mesh.groups[0].face_count == 2


def test_material_fallback_replacement_and_textures():
    loader = MemoryObjTextLoader()
    loader.add_file("assets/material_test.obj", "usemtl matA\nmtllib matA.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3")
    loader.add_file("assets/matA.mtl", "newmtl matA\nKa 0.01 0.02 0.03\nKd 0.1 0.2 0.3\nKs 0.4 0.5 0.6\n"
                                       "Ke 0.7 0.8 0.9\nNs 42\nNi 1.45\nd 0.5\nillum 2\nmap_Kd diffuse.png\n"
                                       "bump normal.png")
    mesh = read_obj("assets/material_test.obj", loader)
    mat = mesh.materials[mesh.face_materials[0]]
    assert mesh.material_count() == 1 and not mat.fallback
    assert mat.Kd == pytest.approx((0.1, 0.2, 0.3))
    assert mat.Ns == pytest.approx(42.0) and mat.Ni == pytest.approx(1.45) and mat.d == pytest.approx(0.5)
    assert mat.illum == 2
    assert mesh.texture_count() == 3 and mesh.texture_count(include_dummy=False) == 2
    assert mat.map_Kd == 1 and mesh.textures[1].name == "diffuse.png"
    assert mesh.textures[1].path == "assets/diffuse.png"
    assert mat.map_bump == 2 and mesh.textures[2].name == "normal.png"
    assert mesh.textures[2].path == "assets/normal.png"


def test_memory_loader_mtllib_with_spaces_and_texture_dedup():
    loader = MemoryObjTextLoader()
    loader.add_file("models/model.obj", "mtllib material library.mtl\nusemtl matB\nv 0 0 0\nv 1 0 0\nv 0 1 0\n"
                                        "f 1 2 3\n")
    loader.add_file("models/material library.mtl", "newmtl matB\nmap_Ka shared.png\nmap_Kd shared.png\n"
                                                   "map_bump -bm 0.5 shared.png\n")
    mesh = read_obj("models/model.obj", loader)
    mat = mesh.materials[mesh.face_materials[0]]
    assert mesh.face_count() == 1 and mesh.position_count(include_dummy=False) == 3
    assert mesh.material_count() == 1 and mat.name == "matB"
    assert mesh.texture_count() == 2 and mesh.texture_count(include_dummy=False) == 1
    assert mat.map_Ka == 1 and mat.map_Kd == 1 and mat.map_bump == 1
    assert mesh.textures[1].path == "models/shared.png"


def test_parse_obj_from_string():
    mesh = parse_obj("v 0 0 0 \nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    assert mesh.face_count() == 1 and mesh.index_count() == 3


def test_comments_blank_lines_and_crlf():
    mesh = parse_obj("# comment\r\n\r\nv 0 0 0 # inline comment\r\nv 1 0 0\r\nv 0 1 0\r\nf 1 2 3\r", "comments.obj")
    assert mesh.position_count(include_dummy=False) == 3
    assert mesh.face_count() == 1 and mesh.index_count() == 3


def test_missing_texcoord_face_form():
    mesh = parse_obj("v 0 0 0\nv 1 0 0\nv 0 1 0\nvn 0 0 1\nf 1//1 2//1 3//1", "missing_texcoord.obj")
    assert mesh.face_count() == 1
    assert (mesh.indices[0].p, mesh.indices[0].t, mesh.indices[0].n) == (1, 0, 1)
    assert (mesh.indices[2].p, mesh.indices[2].t, mesh.indices[2].n) == (3, 0, 1)


def test_multiple_groups_flush_offsets():
    mesh = parse_obj("g A\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3\ng B\nf 2 4 3", "groups2.obj")
    assert mesh.group_count() == 2
    a, b = mesh.groups
    assert (a.name, a.face_count, a.face_offset, a.index_offset) == ("A", 1, 0, 0)
    assert (b.name, b.face_count, b.face_offset, b.index_offset) == ("B", 1, 1, 3)


def test_tr_only_transparency():
    loader = MemoryObjTextLoader()
    loader.add_file("materials/glass.obj", "mtllib glass.mtl\nusemtl glass\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3")
    loader.add_file("materials/glass.mtl", "newmtl glass\nTr 0.25")
    mesh = read_obj("materials/glass.obj", loader)
    assert mesh.materials[mesh.face_materials[0]].d == pytest.approx(0.75)


def test_d_overrides_tr_order():
    loader = MemoryObjTextLoader()
    loader.add_file("materials/mat.obj", "mtllib mat.mtl\nusemtl mat\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3")
    loader.add_file("materials/mat.mtl", "newmtl mat\nd 0.4\nTr 0.9")
    mesh = read_obj("materials/mat.obj", loader)
    assert mesh.materials[mesh.face_materials[0]].d == pytest.approx(0.4)


def test_obj_file_round_trip_through_oracle(tmp_path):
    # a 6 x 4 quad grid written as OBJ, packed, built and traced by the oracle
    from oracle import oracle
    nx, ny = 6, 4
    lines = [f"v {x / nx} {y / ny} {0.1 * x * y}" for y in range(ny + 1) for x in range(nx + 1)]
    for y in range(ny):
        for x in range(nx):
            a = y * (nx + 1) + x + 1
            lines.append(f"f {a} {a + 1} {a + nx + 2} {a + nx + 1}")
    path = tmp_path / "grid.obj"
    path.write_text("\n".join(lines) + "\n")
    tris = pack_triangles(read_obj(str(path)))
    assert tris.shape == (2 * nx * ny, 9) and tris.dtype == np.float32
    rays = np.zeros((8, 64), np.float32)
    rng = np.random.default_rng(0)
    rays[0:2] = rng.uniform(0.05, 0.95, (2, 64))
    rays[2], rays[3], rays[6], rays[7] = -1.0, 0.0, 1.0, 1e30
    hits = oracle.trace_bvh2(oracle.lbvh_build(tris), rays.reshape(-1)).reshape(-1, 8)
    ref = oracle.trace_brute(tris, rays.reshape(-1)).reshape(-1, 8)
    assert np.all(hits[:, 2].view(np.uint32) != 0xFFFFFFFF)
    assert np.array_equal(hits.view(np.uint32), ref.view(np.uint32))


def test_color_to_bytes_matches_reference_formula():
    x = np.array([-1.0, 0.0, 0.25, 1.0, 4.0, 0.5, 1e-8], np.float32)
    want = [0, 0, 128, 255, 255, int(np.float32(256.0) * np.sqrt(np.float32(0.5))), 0]
    assert color_to_bytes(x).tolist() == want


def test_ppm_and_npy_writers(tmp_path):
    w, h = 5, 3
    px = np.random.default_rng(1).uniform(-0.2, 1.5, (h * w, 3)).astype(np.float32)
    p = tmp_path / "img.ppm"
    write_ppm_from_colors(str(p), w, h, px)
    data = p.read_bytes()
    assert data.startswith(b"P6\n5 3\n255\n") and len(data) == len(b"P6\n5 3\n255\n") + w * h * 3
    img = read_ppm(str(p))
    assert img.shape == (h, w, 3) and np.array_equal(img.reshape(-1, 3), color_to_bytes(px))
    q = tmp_path / "img.npy"
    write_npy(str(q), w, h, px)
    assert np.array_equal(np.load(q), px.reshape(h, w, 3))
    with pytest.raises(ValueError):
        write_ppm_from_colors(str(p), w + 1, h, px)
