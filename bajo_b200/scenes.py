"""Seeded synthetic scenes with the shapes of the reference's benchmark
fixtures (no assets are needed or shipped).

``random_triangles`` is the plain LBVH workload: every triangle is a centroid
uniform in [0,1]^3 plus three vertex offsets uniform in [-0.01, 0.01] per axis,
FP32, 9 floats per triangle (the vertex layout of
``bajo/bvh/gpu/triangle_bvh.mojo:617``, TRI_LEAF_VERTEX_STRIDE = 9).
"""
from __future__ import annotations

import numpy as np


def random_triangles(n: int, seed: int = 0, spread: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3), dtype=np.float32)
    off = rng.uniform(-spread, spread, size=(n, 3, 3)).astype(np.float32)
    return np.ascontiguousarray((c + off).reshape(n * 9), dtype=np.float32)


def clustered_points(n: int, seed: int = 0, clusters: int = 32, sigma: float = 0.02) -> np.ndarray:
    """Points in `clusters` Gaussian clusters (sigma) clipped to the unit cube."""
    rng = np.random.default_rng(seed)
    centers = rng.random((clusters, 3))
    which = rng.integers(0, clusters, size=n)
    p = centers[which] + rng.normal(0.0, sigma, size=(n, 3))
    return np.clip(p, 0.0, 1.0).astype(np.float32)


def clustered_points_torch(n: int, seed: int = 0, clusters: int = 32, sigma: float = 0.02, device="cuda"):
    """Points in `clusters` Gaussian clusters (sigma) clipped to the unit cube,
    generated on `device` with a seeded torch generator (the sort workload's
    points at up to 2^28 keys, too many for a host generator)."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    centers = torch.rand((clusters, 3), generator=g, device=device)
    which = torch.randint(0, clusters, (n,), generator=g, device=device)
    p = centers[which]
    del which
    p += torch.randn((n, 3), generator=g, device=device) * sigma
    return p.clamp_(0.0, 1.0)


def _expand_bits_21_torch(v):
    v = v & 0x1FFFFF
    v = (v | (v << 32)) & 0x001F00000000FFFF
    v = (v | (v << 16)) & 0x001F0000FF0000FF
    v = (v | (v << 8)) & 0x100F00F00F00F00F
    v = (v | (v << 4)) & 0x10C30C30C30C30C3
    v = (v | (v << 2)) & 0x1249249249249249
    return v


def morton63_torch(points):
    """63-bit Morton codes (21 bits per axis, e(z) << 2 | e(y) << 1 | e(x)) of
    points in the unit cube, as int64 holding the unsigned code: per axis
    u = clamp(trunc(c * 2^21), 0, 2^21 - 1)."""
    import torch
    code = None
    for axis, shift in ((2, 2), (1, 1), (0, 0)):
        q = (points[:, axis] * 2097152.0).clamp_(0.0, 2097151.0).to(torch.int64)
        e = _expand_bits_21_torch(q) << shift
        code = e if code is None else code.bitwise_or_(e)
        del q, e
    return code


def uniform_u32(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)


# --- reference test fixtures (test/bvh/fixtures.mojo) -------------------------
def _tri(cx, cy, z):
    # fixtures.mojo:21-26
    return [cx - 1.0, cy - 1.0, z, cx + 1.0, cy - 1.0, z, cx, cy + 1.0, z]


def strip_scene(count: int, z: float = 2.0) -> np.ndarray:
    # fixtures.mojo:29-38 (the two-argument _append_tri uses cy = 0, y = -1/+1)
    out = []
    for i in range(count):
        cx = float(i * 4 - count * 2)
        out += _tri(cx, 0.0, z)
    return np.array(out, np.float32)


def two_depth_scene() -> np.ndarray:
    # fixtures.mojo:41-45
    return np.array(_tri(0.0, 0.0, 2.0) + _tri(0.0, 0.0, 4.0), np.float32)


def small_scene() -> np.ndarray:
    # fixtures.mojo:48-58
    out = []
    for z in (2.0, 4.0):
        for cx, cy in ((-1.0, -1.0), (1.0, -1.0), (-1.0, 1.0), (1.0, 1.0)):
            out += _tri(cx, cy, z)
    return np.array(out, np.float32)


def single_triangle_scene() -> np.ndarray:
    # fixtures.mojo:61-64
    return np.array(_tri(0.0, 0.0, 2.0), np.float32)


def duplicate_centroid_scene() -> np.ndarray:
    # fixtures.mojo:67-73
    return np.array([-0.5, -0.5, 2.0, 0.5, -0.5, 2.0, 0.0, 0.5, 2.0] * 12, np.float32)


def degenerate_axis_scene(n: int = 64, seed: int = 3) -> np.ndarray:
    """All triangles in the plane z = 2 (zero centroid extent on one axis,
    the degenerate-axis case of test/bvh/gpu/test_bounds_bvh.mojo:550)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-4.0, 4.0, size=(n, 1, 3)).astype(np.float32)
    off = rng.uniform(-0.3, 0.3, size=(n, 3, 3)).astype(np.float32)
    v = c + off
    v[:, :, 2] = 2.0
    return np.ascontiguousarray(v.reshape(-1), np.float32)


def grid_mesh(nx: int, ny: int, z: float = 0.5) -> np.ndarray:
    """A watertight grid of 2*nx*ny triangles over [0,1]^2 at height z: every
    interior edge is shared by two triangles (tie and watertightness cases)."""
    xs = np.linspace(0.0, 1.0, nx + 1, dtype=np.float32)
    ys = np.linspace(0.0, 1.0, ny + 1, dtype=np.float32)
    out = []
    for j in range(ny):
        for i in range(nx):
            a = (xs[i], ys[j], z)
            b = (xs[i + 1], ys[j], z)
            c = (xs[i + 1], ys[j + 1], z)
            d = (xs[i], ys[j + 1], z)
            out += [*a, *b, *c, *a, *c, *d]
    return np.array(out, np.float32)


def bounds_of(verts: np.ndarray):
    v = verts.reshape(-1, 3)
    return v.min(axis=0), v.max(axis=0)


# --- path-tracing scenes ------------------------------------------------------
MAT_LAMBERTIAN = 0
MAT_METAL = 1
MAT_DIELECTRIC = 2
MAT_EMISSIVE = 3


def surface_id(kind: int, index: int) -> int:
    """SurfaceId: kind in the top 4 bits (bajo/rt/types.mojo:24-34)."""
    return (kind << 28) | (index & 0x0FFFFFFF)


def icosphere(subdivisions: int) -> np.ndarray:
    """Unit icosphere as (n_tris, 3, 3) float64, outward winding:
    20 * 4^subdivisions triangles."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    tris = verts[np.array(f)]
    for _ in range(subdivisions):
        a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        tris = np.stack([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1), np.stack([ca, bc, c], 1),
                         np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3, 3)
    return tris


def _quad(p0, p1, p2, p3):
    return [[p0, p1, p2], [p0, p2, p3]]


def unit_box_inward():
    """The 12 triangles of [0,1]^3 with normals pointing into the box."""
    q = []
    q += _quad((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0))  # floor, normal +y
    q += _quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1))  # ceiling, normal -y
    q += _quad((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1))  # back wall z=1, normal -z
    q += _quad((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0))  # front wall z=0, normal +z
    q += _quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1))  # left x=0, normal +x
    q += _quad((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0))  # right x=1, normal -x
    return np.array(q, np.float64)


def ceiling_light(size: float = 0.25, y: float = 0.999):
    """A size x size quad centred under the ceiling, facing down (-y)."""
    h = size / 2
    return np.array(_quad((0.5 - h, y, 0.5 - h), (0.5 + h, y, 0.5 - h), (0.5 + h, y, 0.5 + h),
                          (0.5 - h, y, 0.5 + h)), np.float64)


class RtScene:
    """Triangle scene for the path tracer: vertices (9 f32 per triangle),
    per-triangle surface ids and material tables (SceneData,
    bajo/rt/types.mojo:382)."""

    def __init__(self, vertices, surfaces, lambertians, emissives, camera=None, description="", metals=None,
                 dielectrics=None):
        self.vertices = np.ascontiguousarray(vertices, np.float32).reshape(-1)
        self.surfaces = np.ascontiguousarray(surfaces, np.uint32)
        self.lambertians = np.ascontiguousarray(lambertians, np.float32).reshape(-1)
        self.emissives = np.ascontiguousarray(emissives, np.float32).reshape(-1)
        # metals: 4 f32 each (albedo rgb, fuzz); dielectrics: 1 f32 each (refraction index)
        self.metals = None if metals is None else np.ascontiguousarray(metals, np.float32).reshape(-1)
        self.dielectrics = None if dielectrics is None else np.ascontiguousarray(dielectrics, np.float32).reshape(-1)
        self.camera = camera
        self.description = description

    @property
    def n_tris(self):
        return self.vertices.size // 9


def spheres_in_box(n_spheres: int = 64, subdivisions: int = 5, seed: int = 0, emission: float = 15.0,
                   rmin: float = 0.03, rmax: float = 0.1, light_up: bool = False) -> RtScene:
    """The procedural path-tracing workload: a 12-triangle unit box (albedo
    0.75) with a 0.25 x 0.25 emissive quad (emission 15) just below the
    ceiling, and n_spheres icospheres (radius uniform in [rmin, rmax], centres
    uniform inside the box and clear of the walls and of the camera) with
    Lambertian albedo uniform in [0.2, 0.8] per channel.  The camera sits just
    inside the front wall looking at the back wall, 60 degree vertical FOV.

    light_up: the same quad at height 0.85 facing the ceiling (emission 4x),
    so the spheres and walls see only light that bounced off the ceiling
    patch above it (the geometry is unchanged)."""
    rng = np.random.default_rng(seed)
    unit = icosphere(subdivisions)
    light = ceiling_light(0.25, 0.85)[:, ::-1] if light_up else ceiling_light()
    parts, surf = [unit_box_inward(), light], [[surface_id(MAT_LAMBERTIAN, 0)] * 12,
                                              [surface_id(MAT_EMISSIVE, 0)] * 2]
    if light_up:
        emission = 4.0 * emission
    albedo = [[0.75, 0.75, 0.75]]
    for s in range(n_spheres):
        r = rng.uniform(rmin, rmax)
        lo = np.array([r + 0.01, r + 0.01, r + 0.2])
        hi = np.array([1 - r - 0.01, 1 - r - 0.06, 1 - r - 0.01])
        c = lo + rng.random(3) * (hi - lo)
        parts.append(unit * r + c)
        albedo.append(list(rng.uniform(0.2, 0.8, 3)))
        surf.append([surface_id(MAT_LAMBERTIAN, s + 1)] * unit.shape[0])
    from .camera import camera_from_vfov
    cam = camera_from_vfov([0.5, 0.5, 0.02], [0.5, 0.5, 1.0], [0.0, 1.0, 0.0], 60.0)
    return RtScene(np.concatenate(parts).astype(np.float32), np.concatenate(surf).astype(np.uint32),
                   np.array(albedo, np.float32), np.array([[emission] * 3], np.float32), cam,
                   f"unit box + {n_spheres} icospheres (subdivision {subdivisions}) + "
                   + ("light facing the ceiling" if light_up else "ceiling light"))


def indirect_box_scene(emission: float = 40.0, size: float = 0.2, y: float = 0.85, n_spheres: int = 3,
                       seed: int = 5) -> RtScene:
    """The unit box lit only indirectly: its light is a size x size panel at
    height y facing the ceiling (the emissive side is its top), so apart from
    the ceiling patch above it every surface receives light that bounced off
    that patch -- light that next-event estimation cannot reach and cosine
    sampling finds rarely, the case path guiding exists for.  A few
    subdivision-2 icospheres sit on the floor half."""
    rng = np.random.default_rng(seed)
    panel = ceiling_light(size, y)[:, ::-1]  # reversed winding: normal +y
    parts = [unit_box_inward(), panel]
    surf = [[surface_id(MAT_LAMBERTIAN, 0)] * 12, [surface_id(MAT_EMISSIVE, 0)] * 2]
    albedo = [[0.75, 0.75, 0.75]]
    unit = icosphere(2)
    for s in range(n_spheres):
        r = rng.uniform(0.08, 0.15)
        c = np.array([rng.uniform(r + 0.05, 1 - r - 0.05), r, rng.uniform(0.4, 0.9)])
        parts.append(unit * r + c)
        albedo.append(list(rng.uniform(0.3, 0.8, 3)))
        surf.append([surface_id(MAT_LAMBERTIAN, s + 1)] * unit.shape[0])
    from .camera import camera_from_vfov
    cam = camera_from_vfov([0.5, 0.5, 0.02], [0.5, 0.4, 1.0], [0.0, 1.0, 0.0], 70.0)
    return RtScene(np.concatenate(parts).astype(np.float32), np.concatenate(surf).astype(np.uint32),
                   np.array(albedo, np.float32), np.array([[emission] * 3], np.float32), cam,
                   f"unit box lit by an upward-facing {size} x {size} panel + {n_spheres} icospheres")


def door_scene(n_spheres: int = 16, subdivisions: int = 4, emission: float = 60.0, door_w: float = 0.16,
               door_h: float = 0.3, seed: int = 11) -> RtScene:
    """The unit box split by a wall at z = 0.5 with a door_w x door_h opening
    at the floor: the 0.25 x 0.25 ceiling light hangs over the back half, the
    camera and n_spheres icospheres sit in the front half.  No point of the
    front half sees the light (the line to it passes the wall above the
    door), so its light has bounced in the back half and come through the
    door: next-event estimation finds nothing there and cosine sampling
    finds the door rarely, while the incident light is concentrated in the
    door's direction -- the case path guiding is for."""
    rng = np.random.default_rng(seed)
    x0, x1 = 0.5 - door_w / 2, 0.5 + door_w / 2
    wall = []
    wall += _quad((0, 0, 0.5), (x0, 0, 0.5), (x0, 1, 0.5), (0, 1, 0.5))
    wall += _quad((x1, 0, 0.5), (1, 0, 0.5), (1, 1, 0.5), (x1, 1, 0.5))
    wall += _quad((x0, door_h, 0.5), (x1, door_h, 0.5), (x1, 1, 0.5), (x0, 1, 0.5))
    h = 0.125
    light = np.array(_quad((0.5 - h, 0.999, 0.78 - h), (0.5 + h, 0.999, 0.78 - h), (0.5 + h, 0.999, 0.78 + h),
                           (0.5 - h, 0.999, 0.78 + h)), np.float64)
    parts = [unit_box_inward(), np.array(wall, np.float64), light]
    surf = [[surface_id(MAT_LAMBERTIAN, 0)] * 12, [surface_id(MAT_LAMBERTIAN, 0)] * len(wall),
            [surface_id(MAT_EMISSIVE, 0)] * 2]
    albedo = [[0.75, 0.75, 0.75]]
    unit = icosphere(subdivisions)
    for k in range(n_spheres):
        r = rng.uniform(0.03, 0.07)
        c = np.array([rng.uniform(r + 0.02, 1 - r - 0.02), rng.uniform(r + 0.01, 0.6), rng.uniform(0.15, 0.45 - r)])
        parts.append(unit * r + c)
        albedo.append(list(rng.uniform(0.3, 0.8, 3)))
        surf.append([surface_id(MAT_LAMBERTIAN, k + 1)] * unit.shape[0])
    from .camera import camera_from_vfov
    cam = camera_from_vfov([0.5, 0.5, 0.02], [0.5, 0.35, 1.0], [0.0, 1.0, 0.0], 70.0)
    return RtScene(np.concatenate(parts).astype(np.float32), np.concatenate(surf).astype(np.uint32),
                   np.array(albedo, np.float32), np.array([[emission] * 3], np.float32), cam,
                   f"unit box split by a wall with a {door_w} x {door_h} door; light behind the wall; "
                   f"{n_spheres} icospheres in front")


def materials_in_box(n_spheres: int = 12, subdivisions: int = 3, seed: int = 3, kinds=(0, 1, 2, 3)) -> RtScene:
    """The lit unit box with icospheres of every material the renderer
    shades, taking `kinds` in turn: 0 Lambertian, 1 mirror metal (fuzz 0),
    2 glossy metal (fuzz 0.05 to 0.4), 3 glass (refraction index 1.5)."""
    rng = np.random.default_rng(seed)
    unit = icosphere(subdivisions)
    parts, surf = [unit_box_inward(), ceiling_light()], [[surface_id(MAT_LAMBERTIAN, 0)] * 12,
                                                        [surface_id(MAT_EMISSIVE, 0)] * 2]
    albedo, metals, dielectrics = [[0.75, 0.75, 0.75]], [], []
    for s in range(n_spheres):
        r = rng.uniform(0.06, 0.12)
        lo = np.array([r + 0.01, r + 0.01, r + 0.25])
        hi = np.array([1 - r - 0.01, 1 - r - 0.06, 1 - r - 0.01])
        parts.append(unit * r + (lo + rng.random(3) * (hi - lo)))
        kind = kinds[s % len(kinds)]
        if kind == 0:
            surf.append([surface_id(MAT_LAMBERTIAN, len(albedo))] * unit.shape[0])
            albedo.append(list(rng.uniform(0.2, 0.8, 3)))
        elif kind in (1, 2):
            surf.append([surface_id(MAT_METAL, len(metals))] * unit.shape[0])
            metals.append(list(rng.uniform(0.5, 0.95, 3)) + [0.0 if kind == 1 else float(rng.uniform(0.05, 0.4))])
        else:
            surf.append([surface_id(MAT_DIELECTRIC, len(dielectrics))] * unit.shape[0])
            dielectrics.append(1.5)
    from .camera import camera_from_vfov
    cam = camera_from_vfov([0.5, 0.5, 0.02], [0.5, 0.5, 1.0], [0.0, 1.0, 0.0], 60.0)
    return RtScene(np.concatenate(parts).astype(np.float32), np.concatenate(surf).astype(np.uint32),
                   np.array(albedo, np.float32), np.array([[15.0] * 3], np.float32), cam,
                   f"unit box + {n_spheres} icospheres: Lambertian, mirror, glossy metal, glass",
                   metals=np.array(metals, np.float32), dielectrics=np.array(dielectrics, np.float32))


def small_rt_scene(seed: int = 1) -> RtScene:
    """A small scene for parity tests: the box, the light and 4 icospheres of
    subdivision 2 (1,294 triangles)."""
    return spheres_in_box(n_spheres=4, subdivisions=2, seed=seed, rmin=0.1, rmax=0.2)


def batched_scenes(n_scenes: int = 4096, lo: int = 256, hi: int = 65536, seed: int = 0):
    """The batched workload: n_scenes independent scenes whose triangle counts
    are log-uniform in [lo, hi], each generated like the plain LBVH workload
    with its own seed.  Returns (vertices, segment offsets)."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_scenes)).astype(np.int64)
    counts = np.clip(counts, lo, hi)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    verts = np.empty(int(offsets[-1]) * 9, np.float32)
    for s, c in enumerate(counts):
        verts[offsets[s] * 9: offsets[s + 1] * 9] = random_triangles(int(c), seed=seed * 100003 + s + 1)
    return verts, offsets.astype(np.uint32)
