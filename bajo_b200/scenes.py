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
