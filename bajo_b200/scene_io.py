"""Scene input and image output: the reference's OBJ/MTL reader and its PPM
writer, for feeding meshes to the C ABI build and saving rendered images.

OBJ/MTL restates ``bajo/parser/obj`` (``ObjMesh`` types.mojo:84-271, line
parser obj.mojo:177-267, index cursor cursor.mojo:65-317, number parser
f32.mojo:14-107, MTL reader mtl.mojo:9-118, loaders loaders.mojo:1-27,
``triangulated_indices`` __init__.mojo:50-82, ``pack_obj_triangles``
pack.mojo:5-23):

- element arrays keep the OBJ dummy element at index 0 (position (0, 0, 0),
  texcoord (0, 0), normal (0, 0, 1), texture ("", "")), so face indices are
  1-based array indices; negative indices count back from the end;
- the first vertex of a face fixes its form (``p``, ``p/t``, ``p//n`` or
  ``p/t/n``) and the others must match; indices past the elements read so
  far, zero indices and stray characters raise ``ObjParseError``;
- numbers accumulate digits in double precision, scale by a binary power of
  ten whose exponent may not exceed 308, and round once to float32;
- ``#`` and a carriage return end a line; ``g`` / ``o`` open a group /
  object holding the faces that follow (empty ones are dropped); ``l``
  records a line, kept out of the triangles; faces of fewer than 3 vertices
  (lines of fewer than 2) are dropped;
- a vertex colour (``v x y z r g b``) makes every vertex coloured, 1.0 where
  none was given;
- ``usemtl`` before its ``mtllib`` creates a fallback material that the
  library's definition replaces; ``Tr`` sets ``d = 1 - Tr`` unless ``d``
  came first; texture maps are deduplicated by path and resolved against the
  MTL file's directory, option flags (``-bm 0.5``) skipped.

The PBRT reader (``bajo/parser/pbrt``) is restated in ``bajo_b200.pbrt``.

``write_ppm_from_colors`` restates bajo/rt/cpu/depth_first.mojo:287-315:
binary P6 with each channel stored as ``uint8(256 * clamp(sqrt(x), 0,
0.999))`` (0 for x <= 0), computed in float32.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

_MAX_DECIMAL_EXPONENT = 308


class ObjParseError(ValueError):
    """Malformed OBJ or MTL input (the reference raises a String error)."""


@dataclass
class ObjIndex:
    p: int
    t: int
    n: int


@dataclass
class ObjGroup:
    name: str
    face_count: int
    face_offset: int
    index_offset: int


@dataclass
class ObjTexture:
    name: str
    path: str


@dataclass
class ObjMaterial:
    name: str = ""
    fallback: bool = False
    Ka: tuple = (0.0, 0.0, 0.0)
    Kd: tuple = (1.0, 1.0, 1.0)
    Ks: tuple = (0.0, 0.0, 0.0)
    Ke: tuple = (0.0, 0.0, 0.0)
    Kt: tuple = (0.0, 0.0, 0.0)
    Ns: float = 1.0
    Ni: float = 1.0
    Tf: tuple = (1.0, 1.0, 1.0)
    d: float = 1.0
    illum: int = 1
    map_Ka: int = 0
    map_Kd: int = 0
    map_Ks: int = 0
    map_Ke: int = 0
    map_Kt: int = 0
    map_Ns: int = 0
    map_Ni: int = 0
    map_d: int = 0
    map_bump: int = 0


@dataclass
class ObjMesh:
    positions: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    texcoords: list = field(default_factory=lambda: [0.0, 0.0])
    normals: list = field(default_factory=lambda: [0.0, 0.0, 1.0])
    colors: list = field(default_factory=list)
    face_vertices: list = field(default_factory=list)
    face_materials: list = field(default_factory=list)
    face_lines: list = field(default_factory=list)
    indices: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    material_names: dict = field(default_factory=dict)
    textures: list = field(default_factory=lambda: [ObjTexture("", "")])
    texture_names: dict = field(default_factory=dict)
    objects: list = field(default_factory=list)
    groups: list = field(default_factory=list)
    _current_material: int = 0
    _current_object: ObjGroup = field(default_factory=lambda: ObjGroup("", 0, 0, 0))
    _current_group: ObjGroup = field(default_factory=lambda: ObjGroup("", 0, 0, 0))

    def position_count(self, include_dummy: bool = True) -> int:
        return len(self.positions) // 3 - (0 if include_dummy else 1)

    def texcoord_count(self, include_dummy: bool = True) -> int:
        return len(self.texcoords) // 2 - (0 if include_dummy else 1)

    def normal_count(self, include_dummy: bool = True) -> int:
        return len(self.normals) // 3 - (0 if include_dummy else 1)

    def color_count(self) -> int:
        return len(self.colors) // 3

    def face_count(self) -> int:
        return len(self.face_vertices)

    def index_count(self) -> int:
        return len(self.indices)

    def material_count(self) -> int:
        return len(self.materials)

    def texture_count(self, include_dummy: bool = True) -> int:
        return len(self.textures) - (0 if include_dummy else 1)

    def object_count(self) -> int:
        return len(self.objects)

    def group_count(self) -> int:
        return len(self.groups)

    # -- parser state (types.mojo:165-271) --
    def _flush_object(self):
        if self._current_object.face_count > 0:
            self.objects.append(self._current_object)
        self._current_object = ObjGroup("", 0, len(self.face_vertices), len(self.indices))

    def _flush_group(self):
        if self._current_group.face_count > 0:
            self.groups.append(self._current_group)
        self._current_group = ObjGroup("", 0, len(self.face_vertices), len(self.indices))

    def _begin_object(self, name: str):
        self._flush_object()
        self._current_object.name = name

    def _begin_group(self, name: str):
        self._flush_group()
        self._current_group.name = name

    def _finish(self):
        self._flush_group()
        self._flush_object()

    def _ensure_material(self, name: str, fallback: bool = True) -> int:
        if name in self.material_names:
            return self.material_names[name]
        idx = len(self.materials)
        self.materials.append(ObjMaterial(name, fallback=fallback))
        self.material_names[name] = idx
        return idx

    def _upsert_material(self, material: ObjMaterial) -> int:
        if material.name in self.material_names:
            idx = self.material_names[material.name]
            if self.materials[idx].fallback:
                self.materials[idx] = material
                return idx
        idx = len(self.materials)
        self.materials.append(material)
        self.material_names.setdefault(material.name, idx)
        return idx

    def _add_texture(self, name: str, base: str) -> int:
        path = os.path.join(base, name)
        if path in self.texture_names:
            return self.texture_names[path]
        idx = len(self.textures)
        self.textures.append(ObjTexture(name, path))
        self.texture_names[path] = idx
        return idx

    def _push_color(self, r: float, g: float, b: float):
        target = len(self.positions) - 3
        while len(self.colors) < target:
            self.colors.append(1.0)
        self.colors.extend([r, g, b])

    def _push_element_meta(self, n: int, is_line: bool):
        if n == 0 or (not is_line and n < 3) or (is_line and n < 2):
            return
        self.face_vertices.append(n)
        self.face_materials.append(self._current_material)
        if is_line or self.face_lines:
            while len(self.face_lines) < len(self.face_vertices) - 1:
                self.face_lines.append(0)
            self.face_lines.append(1 if is_line else 0)
        self._current_group.face_count += 1
        self._current_object.face_count += 1


class PathObjTextLoader:
    """Reads OBJ / MTL text from the file system."""

    def read_text(self, path: str) -> str:
        with open(path, "r", encoding="utf-8", newline="") as f:
            return f.read()


class MemoryObjTextLoader:
    """OBJ / MTL text held in memory, keyed by path."""

    def __init__(self):
        self.files: dict[str, str] = {}

    def add_file(self, path: str, text: str):
        self.files[path] = text

    def read_text(self, path: str) -> str:
        if path in self.files:
            return self.files[path]
        raise ObjParseError("MemoryObjTextLoader: file not found: " + path)


# -- line cursor (cursor.mojo, primitives.mojo) ------------------------------
def _is_ws(c: str) -> bool:
    return c in " \t\r"


def _is_line_cut(c: str) -> bool:
    return c in "\r#"


def _is_ws_or_line_cut(c: str) -> bool:
    return c in " \t\r#"


def _fix_index(raw: int, count_with_dummy: int) -> int:
    resolved = raw if raw > 0 else (count_with_dummy + raw if raw < 0 else 0)
    if resolved <= 0 or resolved >= count_with_dummy:
        raise ObjParseError(f"OBJ index {raw} is out of range for {count_with_dummy - 1} available elements")
    return resolved


class _Cursor:
    def __init__(self, line: str):
        self.s = line
        self.pos = 0

    def skip_ws(self):
        while self.pos < len(self.s):
            c = self.s[self.pos]
            if _is_line_cut(c):
                self.s = self.s[:self.pos]
                break
            if not _is_ws(c):
                break
            self.pos += 1

    def has_next(self) -> bool:
        self.skip_ws()
        return self.pos < len(self.s)

    def f32_at_pos(self) -> float:
        s, p, end = self.s, self.pos, len(self.s)
        if p >= end:
            return 0.0
        sign = 1.0
        if s[p] == "-":
            sign, p = -1.0, p + 1
        elif s[p] == "+":
            p += 1
        num = 0.0
        while p < end and s[p].isdigit() and s[p].isascii():
            num = num * 10.0 + float(ord(s[p]) - 48)
            p += 1
        if p < end and s[p] == ".":
            p += 1
            fra, div = 0.0, 1.0
            while p < end and s[p].isdigit() and s[p].isascii():
                fra = fra * 10.0 + float(ord(s[p]) - 48)
                div *= 10.0
                p += 1
            num += fra / div
        if p < end and s[p] in "eE":
            p += 1
            exp_sign = 1
            if p < end and s[p] == "-":
                exp_sign, p = -1, p + 1
            elif p < end and s[p] == "+":
                p += 1
            ev, has_digit = 0, False
            while p < end and s[p].isdigit() and s[p].isascii():
                has_digit = True
                digit = ord(s[p]) - 48
                if ev > (_MAX_DECIMAL_EXPONENT - digit) // 10:
                    raise ObjParseError(f"OBJ decimal exponent exceeds {_MAX_DECIMAL_EXPONENT}")
                ev = ev * 10 + digit
                p += 1
            if not has_digit:
                raise ObjParseError("missing OBJ decimal exponent digits")
            if ev > 0:
                power, base, rem = 1.0, 10.0, ev
                while rem > 0:
                    if rem & 1:
                        power *= base
                    rem //= 2
                    if rem > 0:
                        base *= base
                num = num * power if exp_sign == 1 else num / power
        self.pos = p
        return float(np.float32(sign * num))

    def next_f32(self) -> float:
        self.skip_ws()
        return self.f32_at_pos()

    def _signed_here(self) -> bool:
        return self.pos < len(self.s) and self.s[self.pos] in "+-"

    def _index_int(self, slash_terminates: bool, count_with_dummy: int) -> int:
        if self.pos >= len(self.s):
            raise ObjParseError("missing OBJ index")
        sign = 1
        if self.s[self.pos] == "-":
            sign = -1
            self.pos += 1
        elif self.s[self.pos] == "+":
            self.pos += 1
        out = 0
        while self.pos < len(self.s) and self.s[self.pos].isdigit() and self.s[self.pos].isascii():
            out = out * 10 + (ord(self.s[self.pos]) - 48)
            if out > count_with_dummy - 1:
                raise ObjParseError("OBJ index exceeds the available element count")
            self.pos += 1
        if out == 0:
            raise ObjParseError("missing or zero OBJ index")
        if self.pos < len(self.s):
            c = self.s[self.pos]
            if not ((slash_terminates and c == "/") or _is_ws_or_line_cut(c)):
                raise ObjParseError("invalid character in OBJ index")
        return sign * out

    def _slash(self) -> bool:
        if self.pos < len(self.s) and self.s[self.pos] == "/":
            self.pos += 1
            return True
        return False

    def face_index(self, shape: int | None, lim) -> tuple[ObjIndex, int]:
        """One face vertex; shape None = the first vertex, which fixes it."""
        lp, lt, ln = lim
        fix = self._signed_here()
        p = self._index_int(True if shape != 1 else False, lp) if shape is not None else self._index_int(True, lp)
        t = n = 0
        if shape is None:
            shape = 1
            if self._slash():
                if self._slash():
                    shape = 3
                    fix |= self._signed_here()
                    n = self._index_int(False, ln)
                else:
                    shape = 2
                    fix |= self._signed_here()
                    t = self._index_int(True, lt)
                    if self._slash():
                        shape = 4
                        fix |= self._signed_here()
                        n = self._index_int(False, ln)
        elif shape == 2:
            if self._slash():
                fix |= self._signed_here()
                t = self._index_int(False, lt)
            if t == 0:
                raise ObjParseError("missing OBJ texture index")
        elif shape == 3:
            if self._slash() and self._slash():
                fix |= self._signed_here()
                n = self._index_int(False, ln)
            if n == 0:
                raise ObjParseError("missing OBJ normal index")
        elif shape == 4:
            if self._slash():
                fix |= self._signed_here()
                t = self._index_int(True, lt)
                if self._slash():
                    fix |= self._signed_here()
                    n = self._index_int(False, ln)
            if t == 0 or n == 0:
                raise ObjParseError("missing OBJ texture or normal index")
        if fix:
            p = _fix_index(p, lp)
            t = _fix_index(t, lt) if t != 0 else 0
            n = _fix_index(n, ln) if n != 0 else 0
        return ObjIndex(p, t, n), shape

    def rest_of_line(self) -> str:
        self.skip_ws()
        if self.pos >= len(self.s):
            return ""
        start, end = self.pos, len(self.s)
        for q in range(start, end):
            if _is_line_cut(self.s[q]):
                end = q
                self.s = self.s[:end]
                break
        text = self.s[start:end]
        self.pos = len(self.s)
        return text.rstrip(" \t\r")

    def next_word(self) -> str:
        self.skip_ws()
        if self.pos >= len(self.s):
            return ""
        start = self.pos
        while self.pos < len(self.s):
            c = self.s[self.pos]
            if _is_ws_or_line_cut(c):
                if _is_line_cut(c):
                    self.s = self.s[:self.pos]
                break
            self.pos += 1
        return self.s[start:self.pos]


def _word_ends(s: str, p: int) -> bool:
    return p >= len(s) or _is_ws_or_line_cut(s[p])


def _parse_floats(mesh_list: list, cur: _Cursor, k: int) -> list | None:
    vals = []
    for _ in range(k):
        cur.skip_ws()
        if cur.pos >= len(cur.s):
            return None
        vals.append(cur.f32_at_pos())
    mesh_list.extend(vals)
    return vals


def _parse_face(mesh: ObjMesh, cur: _Cursor, is_line: bool):
    start = len(mesh.indices)
    lim = (mesh.position_count(), mesh.texcoord_count(), mesh.normal_count())
    count, shape = 0, None
    while True:
        cur.skip_ws()
        if cur.pos >= len(cur.s):
            break
        idx, shape = cur.face_index(shape, lim)
        mesh.indices.append(idx)
        count += 1
    if count >= (2 if is_line else 3):
        mesh._push_element_meta(count, is_line)
    else:
        del mesh.indices[start:]


def _read_mtl_text(mesh: ObjMesh, base: str, text: str):
    current, have, found_d = ObjMaterial(), False, False
    for line in text.split("\n"):
        cur = _Cursor(line)
        tag = cur.next_word()
        if not tag:
            continue
        if tag == "newmtl":
            if have:
                mesh._upsert_material(current)
            current, have, found_d = ObjMaterial(cur.rest_of_line(), fallback=False), True, False
        elif have:
            if tag in ("Ka", "Kd", "Ks", "Ke", "Kt", "Tf"):
                setattr(current, tag, (cur.next_f32(), cur.next_f32(), cur.next_f32()))
            elif tag in ("Ns", "Ni"):
                setattr(current, tag, cur.next_f32())
            elif tag == "illum":
                current.illum = int(cur.next_f32())
            elif tag == "d":
                current.d = cur.next_f32()
                found_d = True
            elif tag == "Tr":
                if not found_d:
                    current.d = float(np.float32(1.0) - np.float32(cur.next_f32()))
            elif tag[:4] == "map_" or tag == "bump":
                name = ""
                while cur.has_next():  # the last word that is not an option flag
                    word = cur.next_word()
                    if not word:
                        break
                    if word[0] != "-":
                        name = word
                if name:
                    val = mesh._add_texture(name, base)
                    key = "map_bump" if tag == "bump" else tag
                    if key in ("map_Ka", "map_Kd", "map_Ks", "map_Ke", "map_Kt", "map_Ns", "map_Ni", "map_d",
                               "map_bump"):
                        setattr(current, key, val)
    if have:
        mesh._upsert_material(current)


def parse_obj(text: str, path: str = "", loader=None) -> ObjMesh:
    """OBJ text to an ``ObjMesh``; ``mtllib`` files are read through
    ``loader`` relative to ``path`` (an empty in-memory loader when None, so
    an ``mtllib`` line then raises)."""
    loader = loader if loader is not None else MemoryObjTextLoader()
    mesh = ObjMesh()
    for line in text.split("\n"):
        cur = _Cursor(line)
        cur.skip_ws()
        if cur.pos >= len(cur.s):
            continue
        s, p = cur.s, cur.pos
        c0 = s[p]
        if c0 == "v" and _word_ends(s, p + 1):
            cur.pos = p + 1
            if _parse_floats(mesh.positions, cur, 3) is not None:
                cur.skip_ws()
                if cur.pos < len(cur.s):
                    rgb = []
                    for _ in range(3):
                        cur.skip_ws()
                        if cur.pos >= len(cur.s):
                            break
                        rgb.append(cur.f32_at_pos())
                    if len(rgb) == 3:
                        mesh._push_color(*rgb)
        elif c0 == "v" and p + 1 < len(s) and s[p + 1] == "t":
            if _word_ends(s, p + 2):
                cur.pos = p + 2
                _parse_floats(mesh.texcoords, cur, 2)
        elif c0 == "v" and p + 1 < len(s) and s[p + 1] == "n":
            if _word_ends(s, p + 2):
                cur.pos = p + 2
                _parse_floats(mesh.normals, cur, 3)
        elif c0 == "f" and _word_ends(s, p + 1):
            cur.pos = p + 1
            _parse_face(mesh, cur, False)
        elif c0 == "l" and _word_ends(s, p + 1):
            cur.pos = p + 1
            _parse_face(mesh, cur, True)
        elif c0 == "g" and _word_ends(s, p + 1):
            cur.pos = p + 1
            mesh._begin_group(cur.rest_of_line())
        elif c0 == "o" and _word_ends(s, p + 1):
            cur.pos = p + 1
            mesh._begin_object(cur.rest_of_line())
        else:
            tag = cur.next_word()
            if tag == "usemtl":
                name = cur.rest_of_line()
                if name:
                    mesh._current_material = mesh._ensure_material(name, fallback=True)
            elif tag == "mtllib":
                name = cur.rest_of_line()
                if name:
                    mtl_path = os.path.join(os.path.dirname(path), name)
                    _read_mtl_text(mesh, os.path.dirname(mtl_path), loader.read_text(mtl_path))
    if mesh.colors:
        while len(mesh.colors) < len(mesh.positions):
            mesh.colors.append(1.0)
    mesh._finish()
    return mesh


def read_obj(path: str, loader=None) -> ObjMesh:
    """Read and parse an OBJ file (and its MTL libraries) through ``loader``
    (the file system by default)."""
    loader = loader if loader is not None else PathObjTextLoader()
    return parse_obj(loader.read_text(path), path, loader)


def triangulated_indices(mesh: ObjMesh) -> list:
    """Fan triangulation of every polygon face (lines skipped): (first, i,
    i + 1) for i in 1..n-2."""
    out, offset = [], 0
    for f, n in enumerate(mesh.face_vertices):
        is_line = bool(mesh.face_lines[f]) if mesh.face_lines else False
        if not is_line and n >= 3:
            first = mesh.indices[offset]
            for i in range(1, n - 1):
                out += [first, mesh.indices[offset + i], mesh.indices[offset + i + 1]]
        offset += n
    return out


def pack_triangles(mesh: ObjMesh) -> np.ndarray:
    """The triangulated faces as a float32 (n_triangles, 9) array of vertex
    positions: the vertex layout bajo_lbvh_build takes."""
    idx = np.array([i.p for i in triangulated_indices(mesh)], np.int64)
    pos = np.asarray(mesh.positions, np.float32).reshape(-1, 3)
    return np.ascontiguousarray(pos[idx].reshape(-1, 9))


def pack_obj_triangles(path: str, loader=None) -> np.ndarray:
    """``read_obj`` then ``pack_triangles``."""
    return pack_triangles(read_obj(path, loader))


# -- images --------------------------------------------------------------------
def color_to_bytes(colors) -> np.ndarray:
    """uint8(256 * clamp(sqrt(x), 0, 0.999)), 0 for x <= 0, in float32."""
    c = np.asarray(colors, np.float32)
    g = np.where(c > np.float32(0.0), np.sqrt(np.maximum(c, np.float32(0.0))), np.float32(0.0)).astype(np.float32)
    g = np.clip(g, np.float32(0.0), np.float32(0.999))
    return (np.float32(256.0) * g).astype(np.uint8)


def write_ppm_from_colors(path: str, width: int, height: int, pixels) -> None:
    """Binary P6 image of width x height linear RGB pixels (row-major, top
    row first), gamma 2 as the reference's CPU renderer writes it."""
    px = np.asarray(pixels, np.float32).reshape(-1, 3)
    if px.shape[0] != width * height:
        raise ValueError(f"expected {width * height} pixels, got {px.shape[0]}")
    with open(path, "wb") as f:
        f.write(f"P6\n{width} {height}\n255\n".encode("ascii"))
        f.write(color_to_bytes(px).tobytes())


def read_ppm(path: str) -> np.ndarray:
    """A binary P6 file (as written above) as a (height, width, 3) uint8 array."""
    with open(path, "rb") as f:
        data = f.read()
    parts, pos = [], 0
    while len(parts) < 4:
        while data[pos:pos + 1].isspace():
            pos += 1
        start = pos
        while not data[pos:pos + 1].isspace():
            pos += 1
        parts.append(data[start:pos])
    if parts[0] != b"P6" or parts[3] != b"255":
        raise ValueError("not an 8-bit binary PPM")
    w, h = int(parts[1]), int(parts[2])
    return np.frombuffer(data[pos + 1:pos + 1 + w * h * 3], np.uint8).reshape(h, w, 3)


def write_npy(path: str, width: int, height: int, pixels) -> None:
    """The linear float32 pixels as a (height, width, 3) .npy array."""
    np.save(path, np.asarray(pixels, np.float32).reshape(height, width, 3))
