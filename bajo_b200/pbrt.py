"""PBRT-v4 text scene reader (``bajo/parser/pbrt``: lexer and directive
interpreter parser.mojo:32-747, loaders loaders.mojo:1-27, entry points
__init__.mojo:1-28).

The reader maps the subset the reference maps and rejects everything else
with ``PbrtParseError`` instead of dropping it:

- ``LookAt`` / ``Camera "perspective" "float fov"`` set a pinhole camera
  (``Camera.from_vfov``: fov is the vertical field of view); ``Film`` sets
  the image size, ``Sampler`` the samples per pixel, ``Integrator "path"``
  the maximum depth; ``PixelFilter``, ``Accelerator``, ``Option`` and
  ``ColorSpace "srgb"`` are consumed;
- ``WorldBegin`` resets the transform; ``AttributeBegin/End`` scope the
  graphics state (transform, material, area light, orientation),
  ``TransformBegin/End`` the transform alone; ``Identity``, ``Translate``,
  ``Scale``, ``Rotate``, ``Transform`` and ``ConcatTransform`` build affine
  float32 transforms (``Transform``'s 16 values are read row by row and the
  last row must be 0 0 0 1);
- materials: ``diffuse`` / ``matte`` / ``coateddiffuse`` (its substrate) are
  Lambertian with ``rgb reflectance`` (0.5); ``conductor`` / ``metal`` are
  metals with ``rgb reflectance`` (0.9) and fuzz = ``float roughness``
  (0.05) clamped to [0, 1]; ``dielectric`` / ``glass`` take ``float eta``
  (1.5).  ``MakeNamedMaterial`` (``string type``, default diffuse) and
  ``NamedMaterial`` name them;
- ``AreaLightSource "diffuse"`` makes every later shape of the scope an
  emitter of ``rgb L`` x ``float scale``, a new emissive entry per shape;
- shapes: ``sphere`` (``float radius``, uniform scale only: the axis
  lengths may differ by at most 1e-5), ``trianglemesh`` and ``loopsubdiv``
  (its control cage) with ``point3 P`` (or ``point P``) and optional
  ``integer indices``; ``ReverseOrientation`` swaps the last two vertices;
- ``Include`` reads a file relative to the including file, at most 32 deep.

Numbers use the OBJ reader's float parser and must fill their token;
integers must be integral.  A fresh scene holds one Lambertian (0.5) as the
default surface, 640 x 480 pixels, 16 samples, depth 8, seed 2026.

Spheres stay analytic in ``PbrtScene``; ``to_rt_scene`` tessellates them as
icospheres for the triangle path tracer.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import scenes
from .scene_io import ObjParseError, _Cursor

f32 = np.float32


class PbrtParseError(ValueError):
    """A PBRT input the reader does not map (parser.mojo raises ``Error``)."""


class PathPbrtTextLoader:
    """Reads files from the file system (loaders.mojo:11-14)."""

    def read_text(self, path: str) -> str:
        with open(path, "r", encoding="utf-8") as fh:
            return fh.read()


class MemoryPbrtTextLoader:
    """Serves files from a dict (loaders.mojo:17-27)."""

    def __init__(self):
        self.files: dict[str, str] = {}

    def add_file(self, path: str, text: str) -> None:
        self.files[path] = text

    def read_text(self, path: str) -> str:
        if path in self.files:
            return self.files[path]
        raise PbrtParseError("MemoryPbrtTextLoader: file not found: " + path)


# --- affine float32 transforms (parser.mojo:330-420) -------------------------
class Affine:
    """Row-major 3x4 float32 affine map: x' = M x + t."""

    __slots__ = ("m",)

    def __init__(self, m):
        self.m = [f32(v) for v in m]

    @staticmethod
    def identity() -> "Affine":
        return Affine([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0])

    def compose(self, b: "Affine") -> "Affine":
        """The map that applies b, then self (parser.mojo:330-346): every
        entry a sum of float32 products, added left to right."""
        a, b = self.m, b.m
        out = []
        for r in range(3):
            a0, a1, a2, at = a[4 * r], a[4 * r + 1], a[4 * r + 2], a[4 * r + 3]
            for c in range(4):
                v = a0 * b[c] + a1 * b[4 + c] + a2 * b[8 + c]
                out.append(v + at if c == 3 else v)
        return Affine(out)

    def point(self, p) -> np.ndarray:
        m = self.m
        x, y, z = f32(p[0]), f32(p[1]), f32(p[2])
        return np.array([m[4 * r] * x + m[4 * r + 1] * y + m[4 * r + 2] * z + m[4 * r + 3] for r in range(3)], f32)

    def vector(self, v) -> np.ndarray:
        m = self.m
        x, y, z = f32(v[0]), f32(v[1]), f32(v[2])
        return np.array([m[4 * r] * x + m[4 * r + 1] * y + m[4 * r + 2] * z for r in range(3)], f32)


def _translation(x, y, z) -> Affine:
    return Affine([1, 0, 0, x, 0, 1, 0, y, 0, 0, 1, z])


def _scale(x, y, z) -> Affine:
    return Affine([x, 0, 0, 0, 0, y, 0, 0, 0, 0, z, 0])


def _rotation(angle, x, y, z) -> Affine:
    """Rodrigues rotation by `angle` degrees about (x, y, z), in float32
    (parser.mojo:357-385)."""
    x, y, z = f32(x), f32(y), f32(z)
    length = f32(math.sqrt(f32(x * x + y * y + z * z)))
    if length == 0.0:
        raise PbrtParseError("PBRT Rotate axis must be non-zero")
    nx, ny, nz = x / length, y / length, z / length
    rad = f32(angle) * f32(math.pi / 180.0)
    c, s = f32(math.cos(rad)), f32(math.sin(rad))
    t = f32(1.0) - c
    return Affine([t * nx * nx + c, t * nx * ny - s * nz, t * nx * nz + s * ny, 0,
                   t * nx * ny + s * nz, t * ny * ny + c, t * ny * nz - s * nx, 0,
                   t * nx * nz - s * ny, t * ny * nz + s * nx, t * nz * nz + c, 0])


def _matrix(values) -> Affine:
    if len(values) != 16:
        raise PbrtParseError("PBRT transform matrix requires 16 values")
    m = [parse_f32(v) for v in values]
    if m[12] != 0.0 or m[13] != 0.0 or m[14] != 0.0 or m[15] != 1.0:
        raise PbrtParseError("projective PBRT transforms are not supported")
    return Affine(m[:12])


# --- lexer (parser.mojo:38-129) ----------------------------------------------
@dataclass
class Token:
    value: str
    quoted: bool
    line: int


_SPACE = " \t\r\n"


class Lexer:
    """Tokens: ``[``, ``]``, double-quoted strings (newlines allowed inside)
    and bare words ending at white space, ``#``, ``[`` or ``]``; ``#``
    comments run to the end of the line."""

    def __init__(self, text: str):
        self.s, self.pos, self.line = text, 0, 1

    def _skip_space(self) -> None:
        s, n = self.s, len(self.s)
        while self.pos < n:
            c = s[self.pos]
            if c == "#":
                nl = s.find("\n", self.pos)
                if nl < 0:
                    self.pos = n
                else:
                    self.pos, self.line = nl + 1, self.line + 1
            elif c == "\n":
                self.pos, self.line = self.pos + 1, self.line + 1
            elif c in " \t\r":
                self.pos += 1
            else:
                break

    def has_next(self) -> bool:
        self._skip_space()
        return self.pos < len(self.s)

    def next_is_quoted(self) -> bool:
        self._skip_space()
        return self.pos < len(self.s) and self.s[self.pos] == '"'

    def next(self) -> Token:
        self._skip_space()
        s, n = self.s, len(self.s)
        if self.pos >= n:
            raise PbrtParseError("unexpected end of PBRT input")
        line, c = self.line, s[self.pos]
        if c in "[]":
            self.pos += 1
            return Token(c, False, line)
        if c == '"':
            end = s.find('"', self.pos + 1)
            if end < 0:
                raise PbrtParseError(f"unterminated PBRT string at line {line}")
            value = s[self.pos + 1:end]
            self.line += value.count("\n")
            self.pos = end + 1
            return Token(value, True, line)
        start = self.pos
        while self.pos < n and s[self.pos] not in _SPACE and s[self.pos] not in "#[]":
            self.pos += 1
        return Token(s[start:self.pos], False, line)


def parse_f32(text: str) -> np.float32:
    """The OBJ reader's float parser over the whole token
    (parser.mojo:306-311)."""
    cur = _Cursor(text)
    try:
        v = cur.f32_at_pos()
    except ObjParseError as exc:
        raise PbrtParseError("invalid PBRT number: " + text) from exc
    if cur.pos != len(text):
        raise PbrtParseError("invalid PBRT number: " + text)
    return f32(v)


def parse_int(text: str) -> int:
    v = parse_f32(text)
    if not math.isfinite(float(v)) or int(v) != v:
        raise PbrtParseError("invalid PBRT integer: " + text)
    return int(v)


class Parameters:
    """Declarations in file order ("float radius" -> ["0.5"]); lookups take
    the first match (parser.mojo:132-190)."""

    def __init__(self):
        self.entries: list[tuple[str, list[str]]] = []

    def has(self, decl: str) -> bool:
        return any(d == decl for d, _ in self.entries)

    def values(self, decl: str) -> list[str]:
        for d, v in self.entries:
            if d == decl:
                return list(v)
        return []

    def _first(self, decl: str):
        for d, v in self.entries:
            if d == decl and v:
                return v[0]
        return None

    def string(self, decl: str, default: str) -> str:
        v = self._first(decl)
        return default if v is None else v

    def f32(self, decl: str, default: float) -> np.float32:
        v = self._first(decl)
        return f32(default) if v is None else parse_f32(v)

    def integer(self, decl: str, default: int) -> int:
        v = self._first(decl)
        return default if v is None else parse_int(v)

    def color(self, name: str, default) -> np.ndarray:
        for d, v in self.entries:
            if d in ("rgb " + name, "color " + name):
                if len(v) != 3:
                    raise PbrtParseError("PBRT color parameter requires three values")
                return np.array([parse_f32(x) for x in v], f32)
        return np.asarray(default, f32).reshape(3).copy()


def parse_params(lex: Lexer) -> Parameters:
    """Quoted declarations, each followed by one value or a [ ... ] list
    (parser.mojo:314-327)."""
    params = Parameters()
    while lex.next_is_quoted():
        decl = lex.next().value
        if not lex.has_next():
            raise PbrtParseError("missing value for PBRT parameter " + decl)
        first = lex.next()
        vals = []
        if first.value == "[":
            while True:
                if not lex.has_next():
                    raise PbrtParseError("unterminated PBRT parameter array")
                item = lex.next()
                if item.value == "]":
                    break
                vals.append(item.value)
        else:
            vals.append(first.value)
        params.entries.append((decl, vals))
    return params


# --- scene description (SceneDescription, bajo/rt/scene_description.mojo) ----
@dataclass
class PbrtScene:
    """What a PBRT file describes: analytic spheres, world-space triangles,
    per-shape surface ids, material tables, camera and render settings."""
    sphere_centers: np.ndarray
    sphere_radii: np.ndarray
    sphere_surfaces: np.ndarray
    triangle_vertices: np.ndarray      # (n_tris, 3, 3) float32
    triangle_surfaces: np.ndarray
    lambertians: np.ndarray            # (k, 3)
    metals: np.ndarray                 # (k, 4): albedo rgb, fuzz
    dielectrics: np.ndarray            # (k,)
    emissives: np.ndarray              # (k, 3)
    camera_origin: np.ndarray
    camera_target: np.ndarray
    camera_up: np.ndarray
    camera_fov: float
    width: int
    height: int
    samples_per_pixel: int
    max_depth: int
    rng_seed: int = 2026
    integrator: str = "path"

    @property
    def n_spheres(self) -> int:
        return int(self.sphere_radii.size)

    @property
    def n_triangles(self) -> int:
        return int(self.triangle_surfaces.size)

    def camera(self) -> np.ndarray:
        """The 20-float camera record (``Camera.from_vfov``)."""
        from .camera import camera_from_vfov
        return camera_from_vfov(self.camera_origin, self.camera_target, self.camera_up, float(self.camera_fov))

    def render_settings(self):
        from .rt import RenderSettings
        return RenderSettings(self.width, self.height, self.samples_per_pixel, rng_seed=self.rng_seed,
                              max_depth=self.max_depth)

    def to_rt_scene(self, sphere_subdivisions: int = 3) -> scenes.RtScene:
        """The triangle scene the path tracer takes: the triangles in file
        order, then every sphere as an outward icosphere of
        20 * 4^sphere_subdivisions triangles (float64 unit sphere scaled and
        moved, rounded once to float32) with the sphere's surface."""
        parts = [self.triangle_vertices.reshape(-1, 3, 3).astype(np.float64)]
        surf = [self.triangle_surfaces.astype(np.uint32)]
        if self.n_spheres:
            unit = scenes.icosphere(sphere_subdivisions)
            for c, r, s in zip(self.sphere_centers, self.sphere_radii, self.sphere_surfaces):
                parts.append(unit * float(r) + c.astype(np.float64))
                surf.append(np.full(unit.shape[0], s, np.uint32))
        lam = self.lambertians if self.lambertians.size else np.zeros((1, 3), f32)
        emi = self.emissives if self.emissives.size else np.zeros((1, 3), f32)
        return scenes.RtScene(np.concatenate(parts).astype(np.float32), np.concatenate(surf), lam, emi,
                              self.camera(), "PBRT scene",
                              metals=self.metals if self.metals.size else None,
                              dielectrics=self.dielectrics if self.dielectrics.size else None)


@dataclass
class _State:
    transform: Affine
    surface: int
    area_light: bool = False
    emission: np.ndarray = field(default_factory=lambda: np.zeros(3, f32))
    reverse_orientation: bool = False

    def copy(self) -> "_State":
        return _State(self.transform, self.surface, self.area_light, self.emission.copy(),
                      self.reverse_orientation)


class _Builder:
    """Graphics state and the scene under construction (parser.mojo:193-303)."""

    def __init__(self):
        self.centers, self.radii, self.sphere_surfaces = [], [], []
        self.tris, self.tri_surfaces = [], []
        self.lambertians, self.metals, self.dielectrics, self.emissives = [], [], [], []
        self.named: dict[str, int] = {}
        self.state = _State(Affine.identity(), self.add_lambertian(np.full(3, 0.5, f32)))
        self.attribute_stack: list[_State] = []
        self.transform_stack: list[Affine] = []
        self.origin = np.array([0, 0, 5], f32)
        self.target = np.zeros(3, f32)
        self.up = np.array([0, 1, 0], f32)
        self.fov = f32(45.0)
        self.width, self.height, self.spp, self.max_depth = 640, 480, 16, 8

    def add_lambertian(self, albedo) -> int:
        self.lambertians.append(np.asarray(albedo, f32))
        return scenes.surface_id(scenes.MAT_LAMBERTIAN, len(self.lambertians) - 1)

    def add_metal(self, albedo, fuzz) -> int:
        self.metals.append(np.array([albedo[0], albedo[1], albedo[2], fuzz], f32))
        return scenes.surface_id(scenes.MAT_METAL, len(self.metals) - 1)

    def add_dielectric(self, eta) -> int:
        self.dielectrics.append(f32(eta))
        return scenes.surface_id(scenes.MAT_DIELECTRIC, len(self.dielectrics) - 1)

    def add_emissive(self, radiance) -> int:
        self.emissives.append(np.asarray(radiance, f32).copy())
        return scenes.surface_id(scenes.MAT_EMISSIVE, len(self.emissives) - 1)

    def finish(self) -> PbrtScene:
        if self.attribute_stack or self.transform_stack:
            raise PbrtParseError("unclosed PBRT attribute or transform scope")
        if not self.radii and not self.tris:
            raise PbrtParseError("PBRT scene contains no supported shapes")
        arr = lambda rows, w: np.array(rows, f32).reshape(-1, w)  # noqa: E731
        return PbrtScene(arr(self.centers, 3), np.array(self.radii, f32), np.array(self.sphere_surfaces, np.uint32),
                         np.array(self.tris, f32).reshape(-1, 3, 3), np.array(self.tri_surfaces, np.uint32),
                         arr(self.lambertians, 3), arr(self.metals, 4), np.array(self.dielectrics, f32),
                         arr(self.emissives, 3), self.origin, self.target, self.up, float(self.fov), self.width,
                         self.height, self.spp, self.max_depth)


def _surface(b: _Builder, model: str, params: Parameters) -> int:
    """parser.mojo:423-441."""
    if model in ("diffuse", "matte", "coateddiffuse"):
        return b.add_lambertian(params.color("reflectance", (0.5, 0.5, 0.5)))
    if model in ("conductor", "metal"):
        rough = min(max(params.f32("float roughness", 0.05), f32(0.0)), f32(1.0))
        return b.add_metal(params.color("reflectance", (0.9, 0.9, 0.9)), rough)
    if model in ("dielectric", "glass"):
        return b.add_dielectric(params.f32("float eta", 1.5))
    raise PbrtParseError("unsupported PBRT material: " + model)


def _add_triangle(b: _Builder, p0, p1, p2, surface: int) -> None:
    if b.state.reverse_orientation:
        p1, p2 = p2, p1
    b.tris.append([p0, p1, p2])
    b.tri_surfaces.append(surface)


def _shape(b: _Builder, kind: str, params: Parameters) -> None:
    """parser.mojo:444-586."""
    surface = b.state.surface
    if b.state.area_light:
        surface = b.add_emissive(b.state.emission)
    xf = b.state.transform
    if kind == "sphere":
        center = xf.point((0, 0, 0))
        lengths = [f32(math.sqrt(f32(f32(a[0] * a[0] + a[1] * a[1]) + a[2] * a[2])))
                   for a in (xf.vector((1, 0, 0)), xf.vector((0, 1, 0)), xf.vector((0, 0, 1)))]
        sx, sy, sz = lengths
        if abs(sx - sy) > 1e-5 or abs(sx - sz) > 1e-5:
            raise PbrtParseError("non-uniformly transformed PBRT spheres are not supported")
        b.centers.append(center)
        b.radii.append(f32(params.f32("float radius", 1.0) * sx))
        b.sphere_surfaces.append(surface)
        return
    if kind in ("trianglemesh", "loopsubdiv"):
        pts = params.values("point3 P") or params.values("point P")
        if len(pts) % 3:
            raise PbrtParseError("PBRT trianglemesh P must contain xyz triples")
        idx = params.values("integer indices")
        if not idx:
            if len(pts) % 9:
                raise PbrtParseError("unindexed PBRT trianglemesh must contain triangles")
            for base in range(0, len(pts), 9):
                p = [xf.point([parse_f32(pts[base + 3 * k + j]) for j in range(3)]) for k in range(3)]
                _add_triangle(b, p[0], p[1], p[2], surface)
            return
        if len(idx) % 3:
            raise PbrtParseError("PBRT trianglemesh indices must contain triples")
        count = len(pts) // 3
        for base in range(0, len(idx), 3):
            ii = [parse_int(idx[base + k]) for k in range(3)]
            if any(i < 0 or i >= count for i in ii):
                raise PbrtParseError("PBRT trianglemesh index is out of range")
            p = [xf.point([parse_f32(pts[3 * i + j]) for j in range(3)]) for i in ii]
            _add_triangle(b, p[0], p[1], p[2], surface)
        return
    raise PbrtParseError("unsupported PBRT shape: " + kind)


def _fixed(lex: Lexer, count: int) -> list:
    return [parse_f32(lex.next().value) for _ in range(count)]


def _bracket_values(lex: Lexer) -> list:
    if lex.next().value != "[":
        raise PbrtParseError("expected '[' in PBRT transform")
    vals = []
    while True:
        t = lex.next()
        if t.value == "]":
            return vals
        vals.append(t.value)


def _parse_text(b: _Builder, text: str, path: str, loader, depth: int) -> None:
    """The directive loop (parser.mojo:604-739)."""
    if depth > 32:
        raise PbrtParseError("PBRT Include nesting exceeds 32 files")
    lex = Lexer(text)
    st = b
    while lex.has_next():
        tok = lex.next()
        if tok.quoted:
            raise PbrtParseError(f"expected PBRT directive at line {tok.line}")
        cmd = tok.value
        if cmd == "LookAt":
            v = _fixed(lex, 9)
            st.origin, st.target, st.up = (np.array(v[0:3], f32), np.array(v[3:6], f32), np.array(v[6:9], f32))
        elif cmd == "Camera":
            if lex.next().value != "perspective":
                raise PbrtParseError("only PBRT perspective cameras are supported")
            st.fov = parse_params(lex).f32("float fov", 45.0)
        elif cmd == "Film":
            lex.next()
            p = parse_params(lex)
            st.width, st.height = p.integer("integer xresolution", 640), p.integer("integer yresolution", 480)
        elif cmd == "Sampler":
            lex.next()
            st.spp = parse_params(lex).integer("integer pixelsamples", 16)
        elif cmd == "Integrator":
            if lex.next().value != "path":
                raise PbrtParseError("only the PBRT path integrator is supported")
            st.max_depth = parse_params(lex).integer("integer maxdepth", 8)
        elif cmd in ("PixelFilter", "Accelerator"):
            lex.next()
            parse_params(lex)
        elif cmd == "ColorSpace":
            if lex.next().value != "srgb":
                raise PbrtParseError("only the PBRT sRGB color space is supported")
        elif cmd == "Option":
            parse_params(lex)
        elif cmd == "WorldBegin":
            st.state.transform = Affine.identity()
        elif cmd == "AttributeBegin":
            st.attribute_stack.append(st.state.copy())
        elif cmd == "AttributeEnd":
            if not st.attribute_stack:
                raise PbrtParseError("PBRT AttributeEnd without AttributeBegin")
            st.state = st.attribute_stack.pop()
        elif cmd == "TransformBegin":
            st.transform_stack.append(st.state.transform)
        elif cmd == "TransformEnd":
            if not st.transform_stack:
                raise PbrtParseError("PBRT TransformEnd without TransformBegin")
            st.state.transform = st.transform_stack.pop()
        elif cmd == "Identity":
            st.state.transform = Affine.identity()
        elif cmd == "Translate":
            st.state.transform = st.state.transform.compose(_translation(*_fixed(lex, 3)))
        elif cmd == "Scale":
            st.state.transform = st.state.transform.compose(_scale(*_fixed(lex, 3)))
        elif cmd == "Rotate":
            st.state.transform = st.state.transform.compose(_rotation(*_fixed(lex, 4)))
        elif cmd == "Transform":
            st.state.transform = _matrix(_bracket_values(lex))
        elif cmd == "ConcatTransform":
            st.state.transform = st.state.transform.compose(_matrix(_bracket_values(lex)))
        elif cmd == "ReverseOrientation":
            st.state.reverse_orientation = not st.state.reverse_orientation
        elif cmd == "Material":
            model = lex.next().value
            st.state.surface = _surface(st, model, parse_params(lex))
        elif cmd == "MakeNamedMaterial":
            name = lex.next().value
            p = parse_params(lex)
            st.named[name] = _surface(st, p.string("string type", "diffuse"), p)
        elif cmd == "NamedMaterial":
            name = lex.next().value
            if name not in st.named:
                raise PbrtParseError("unknown PBRT named material: " + name)
            st.state.surface = st.named[name]
        elif cmd == "AreaLightSource":
            if lex.next().value != "diffuse":
                raise PbrtParseError("only diffuse PBRT area lights are supported")
            p = parse_params(lex)
            st.state.area_light = True
            st.state.emission = p.color("L", (1.0, 1.0, 1.0)) * p.f32("float scale", 1.0)
        elif cmd == "Shape":
            kind = lex.next().value
            _shape(st, kind, parse_params(lex))
        elif cmd == "Include":
            name = lex.next().value
            inc = os.path.join(os.path.dirname(path), name)
            _parse_text(st, loader.read_text(inc), inc, loader, depth + 1)
        elif cmd == "WorldEnd":
            pass
        else:
            raise PbrtParseError(f"unsupported PBRT directive '{cmd}' at line {tok.line}")


def read_pbrt(path: str, loader=None) -> PbrtScene:
    """Reads a PBRT file and its includes (__init__.mojo:15-23)."""
    loader = loader or PathPbrtTextLoader()
    b = _Builder()
    _parse_text(b, loader.read_text(path), path, loader, 0)
    return b.finish()


def parse_pbrt(text: str, path: str = "", loader=None) -> PbrtScene:
    """Parses PBRT text; includes resolve through `loader` (an in-memory
    loader by default, __init__.mojo:26-28)."""
    loader = loader or MemoryPbrtTextLoader()
    b = _Builder()
    _parse_text(b, text, path, loader, 0)
    return b.finish()
