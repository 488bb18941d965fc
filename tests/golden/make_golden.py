"""Generate the golden fixtures that pin the C oracle.

Run from the repository root:  python tests/golden/make_golden.py

Everything here is computed WITHOUT the C oracle, from an independent
pure-Python / numpy restatement of the reference, so that the oracle is
checked against something it did not produce:

* ``morton_kats.json`` -- the known-answer tests of the reference's Morton
  module (test/core/test_morton.mojo:13-87), written out as data;
* ``sort_kats.json`` -- the reference's sort test keys
  (test/sort/test_onesweep.mojo:42, :138; test/sort/test_radix_sort.mojo:316)
  with per-byte histograms and a SHA-256 of the stable-sorted permutation
  (Python's ``sorted`` is stable);
* ``lbvh_fixtures.npz`` -- the fixture scenes of test/bvh/fixtures.mojo plus a
  few edge cases, with bounds, Morton keys, sorted ids, the Karras topology
  (bajo/bvh/gpu/builder/lbvh.mojo:164-329) and refit boxes computed in
  Python with numpy float32 arithmetic;
* ``trace_fixtures.npz`` -- camera rays over those scenes and a float64
  brute-force closest hit (prim id, t) with a mask of rays whose answer is
  robust (no near-tie, not grazing an edge), as in the reference's
  brute-force check (test/bvh/fixtures.mojo:179-210).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from bajo_b200 import scenes  # noqa: E402  (pure numpy generators)

F = np.float32
SENT = 0xFFFFFFFF
LEAF = 0x80000000


# ---------------------------------------------------------------- Morton KATs
def morton_kats():
    step = float(F(1.0) / F(1024.0))
    return {
        "source": "test/core/test_morton.mojo:13-87",
        "expand_bits_3d": [[1, 1], [2, 8], [4, 64]],
        "morton3": [[0.0, 0.0, 0.0, 0], [step, 0.0, 0.0, 1], [0.0, step, 0.0, 2], [0.0, 0.0, step, 4],
                    [step, step, step, 7], [1.0, 1.0, 1.0, (1 << 30) - 1]],
        "common_prefix": [[0, 0, 0, 0, 64], [0, 0, 0, 1, 63], [0, 0, 1, 0, 31]],
    }


# ---------------------------------------------------------------- sort KATs
def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def sort_kats():
    out = {"source": ["test/sort/test_onesweep.mojo:42", "test/sort/test_onesweep.mojo:138",
                      "test/sort/test_radix_sort.mojo:316-344"]}
    # global histogram keys, N = 100,000: (i*13) ^ (i<<16) ^ (i>>3), low 32 bits
    n = 100_000
    keys = [((i * 13) ^ (i << 16) ^ (i >> 3)) & 0xFFFFFFFF for i in range(n)]
    hist = [[0] * 256 for _ in range(4)]
    for k in keys:
        for b in range(4):
            hist[b][(k >> (8 * b)) & 255] += 1
    perm = sorted(range(n), key=lambda i: keys[i])
    out["hist_u32"] = {"n": n, "formula": "(i*13)^(i<<16)^(i>>3)", "hist": hist,
                       "perm_sha256": _sha(np.array(perm, "<u4"))}
    # one binning pass, N = 20,000: (i*17) ^ (i<<13) ^ (i>>5), digit = low byte
    n = 20_000
    keys = [((i * 17) ^ (i << 13) ^ (i >> 5)) & 0xFFFFFFFF for i in range(n)]
    perm = sorted(range(n), key=lambda i: keys[i] & 255)
    out["pass_u32"] = {"n": n, "formula": "(i*17)^(i<<13)^(i>>5)", "perm_sha256": _sha(np.array(perm, "<u4")),
                       "full_perm_sha256": _sha(np.array(sorted(range(n), key=lambda i: keys[i]), "<u4"))}
    # composite u64 keys, N = 10,003 (test_radix_sort.mojo:316-326)
    n = 10_003

    def comp(i):
        seg = (i * 7) % 19
        mort = ((i * 2654435761) & 0xFFFFFFFF) ^ ((i << 11) & 0xFFFFFFFF) ^ (i >> 3)
        return (seg << 32) | (mort & 0xFFFFFFFF)

    keys = [comp(i) for i in range(n)]
    perm = sorted(range(n), key=lambda i: keys[i])
    out["composite_u64"] = {"n": n, "perm_sha256": _sha(np.array(perm, "<u4"))}
    return out


# ---------------------------------------------------------------- LBVH in Python
def expand_bits(v: int) -> int:
    v = (v ^ (v << 16)) & 0xFF0000FF
    v = (v ^ (v << 8)) & 0x0300F00F
    v = (v ^ (v << 4)) & 0x030C30C3
    v = (v ^ (v << 2)) & 0x09249249
    return v


def quant(c: np.float32) -> int:
    s = F(c) * F(1024.0)
    u = 0 if not s > 0 else int(s)
    return min(u, 1023)


def morton(x, y, z) -> int:
    return (expand_bits(quant(z)) << 2) | (expand_bits(quant(y)) << 1) | expand_bits(quant(x))


def clz64(x: int) -> int:
    return 64 - x.bit_length()


def py_lbvh(verts: np.ndarray):
    v = verts.reshape(-1, 3, 3).astype(F)
    n = v.shape[0]
    mn = np.minimum(np.minimum(v[:, 0], v[:, 1]), v[:, 2])
    mx = np.maximum(np.maximum(v[:, 0], v[:, 1]), v[:, 2])
    cen = (mn + mx) * F(0.5)
    cmin, cmax = cen.min(axis=0), cen.max(axis=0)
    ext = cmax - cmin
    inv = np.where(np.abs(ext) > F(1e-20), F(1.0) / np.where(np.abs(ext) > F(1e-20), ext, F(1.0)), F(0.0)).astype(F)
    codes = []
    for i in range(n):
        d = (cen[i] - cmin).astype(F)
        u = (d * inv).astype(F)
        codes.append(morton(u[0], u[1], u[2]))
    order = sorted(range(n), key=lambda i: codes[i])
    sc = [codes[i] for i in order]

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        return clz64(((sc[i] << 32) | i) ^ ((sc[j] << 32) | j))

    ni = max(n - 1, 0)
    meta = np.zeros((max(ni, 1), 4), np.uint32)
    lp = np.zeros(n, np.uint32)
    lc = np.zeros(max(ni, 1), np.uint32)
    if n == 1:
        lp[0] = SENT
    for i in range(ni):
        d = -1 if delta(i, i + 1) < delta(i, i - 1) else 1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax <<= 1
            if lmax > n * 2:
                break
        l, t = 0, lmax >> 1
        while t > 0:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t >>= 1
        j = i + l * d
        first, last = min(i, j), max(i, j)
        lc[i] = last - first + 1
        if first == 0 and last == n - 1:
            meta[i, 0] = SENT
        pref = delta(first, last)
        split, step = first, last - first
        while step > 1:
            step = (step + 1) >> 1
            ns = split + step
            if ns < last and delta(first, ns) > pref:
                split = ns
        if split == first:
            left = LEAF | split
            lp[split] = i
        else:
            left = split
            meta[split, 0] = i
        if split + 1 == last:
            right = LEAF | (split + 1)
            lp[split + 1] = i
        else:
            right = split + 1
            meta[split + 1, 0] = i
        meta[i, 1], meta[i, 2], meta[i, 3] = left, right, last
    # refit, children first
    nb = np.zeros((max(ni, 1), 12), F)
    done = {}

    def box(ref):
        if ref & LEAF:
            it = order[ref & 0x7FFFFFFF]
            return mn[it], mx[it]
        if ref not in done:
            lmin, lmax_ = box(int(meta[ref, 1]))
            rmin, rmax = box(int(meta[ref, 2]))
            nb[ref, 0:3], nb[ref, 3:6], nb[ref, 6:9], nb[ref, 9:12] = lmin, lmax_, rmin, rmax
            done[ref] = (np.minimum(lmin, rmin), np.maximum(lmax_, rmax))
        return done[ref]

    if ni:
        sys.setrecursionlimit(10000)
        box(int(np.nonzero(meta[:ni, 0] == SENT)[0][0]))
    seg_bounds = np.concatenate([mn.min(axis=0), mx.max(axis=0), cmin, cmax]).astype(F)
    return {
        "leaf_bounds": np.concatenate([mn, mx], axis=1).astype(F).reshape(-1),
        "seg_bounds": seg_bounds,
        "morton_unsorted": np.array(codes, np.uint32),
        "leaf_ids": np.array(order, np.uint32),
        "morton_codes": np.array(sc, np.uint32),
        "node_meta": meta.reshape(-1),
        "leaf_parent": lp,
        "node_leaf_counts": lc,
        "node_bounds": nb.reshape(-1),
    }


FIXTURES = {
    "small": lambda: scenes.small_scene(),
    "single": lambda: scenes.single_triangle_scene(),
    "duplicate_centroid": lambda: scenes.duplicate_centroid_scene(),
    "strip16": lambda: scenes.strip_scene(16),
    "two_depth": lambda: scenes.two_depth_scene(),
    "degenerate_axis": lambda: scenes.degenerate_axis_scene(64, 3),
    "grid8": lambda: scenes.grid_mesh(8, 8),
    "random1000": lambda: scenes.random_triangles(1000, 7, 0.05),
}


# ---------------------------------------------------------------- rays + brute force (float64)
def fixture_rays(verts: np.ndarray, w=24, h=18, seed=11):
    """Rays at pixel centres of a camera placed like _make_camera_rays_and_params
    (test/bvh/fixtures.mojo:141-176), plus a few random rays."""
    p = verts.reshape(-1, 3).astype(np.float64)
    lo, hi = p.min(axis=0), p.max(axis=0)
    center = (lo + hi) * 0.5
    scene_w = max(float((hi - lo).max()), 1.0)
    eye = center + np.array([0.1 * scene_w, (hi - lo)[1] * 0.2, -2.5 * scene_w])
    fwd = center - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    rays = []
    for py in range(h):
        for px in range(w):
            sx = ((px + 0.5) / w) * 2 - 1
            sy = 1 - ((py + 0.5) / h) * 2
            d = fwd + right * (sx * (w / h) * 0.75) + up * (sy * 0.75)
            rays.append((eye, d / np.linalg.norm(d)))
    rng = np.random.default_rng(seed)
    for _ in range(64):
        o = center + rng.normal(0, scene_w, 3)
        tgt = lo + rng.random(3) * (hi - lo)
        d = tgt - o
        rays.append((o, d / np.linalg.norm(d)))
    n = len(rays)
    soa = np.zeros((8, n), F)
    for i, (o, d) in enumerate(rays):
        soa[0:3, i] = o
        soa[3, i] = 0.0
        soa[4:7, i] = d
        soa[7, i] = np.finfo(F).max
    return soa.reshape(-1)


def brute64(verts: np.ndarray, rays_soa: np.ndarray):
    v = verts.reshape(-1, 3, 3).astype(np.float64)
    r = rays_soa.reshape(8, -1).astype(np.float64)
    n = r.shape[1]
    prim = np.full(n, SENT, np.uint32)
    t_out = r[7].astype(F).copy()
    robust = np.ones(n, bool)
    for i in range(n):
        o, d = r[0:3, i], r[4:7, i]
        e1, e2 = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
        pv = np.cross(d, e2)
        det = np.einsum("ij,ij->i", e1, pv)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / det
            tv = o - v[:, 0]
            u = np.einsum("ij,ij->i", tv, pv) * inv
            q = np.cross(tv, e1)
            vv = (q @ d) * inv
            t = np.einsum("ij,ij->i", e2, q) * inv
        ok = (np.abs(det) > 1e-12) & (u >= 0) & (u <= 1) & (vv >= 0) & (u + vv <= 1) & (t > 0)
        if not ok.any():
            # robust miss unless some triangle is grazed
            edge = (np.abs(det) > 1e-12) & (u > -1e-5) & (vv > -1e-5) & (u + vv < 1 + 1e-5) & (t > 0)
            robust[i] = not edge.any()
            continue
        ts = np.where(ok, t, np.inf)
        best = int(np.argmin(ts))
        prim[i] = best
        t_out[i] = F(ts[best])
        others = np.sort(ts)[1] if ok.sum() > 1 else np.inf
        margin = min(u[best], vv[best], 1 - u[best] - vv[best])
        near_edge = (np.abs(det) > 1e-12) & (u > -1e-5) & (vv > -1e-5) & (u + vv < 1 + 1e-5) & (t > 0) & ~ok
        close_other = near_edge & (t < ts[best] * (1 + 1e-4))
        robust[i] = (others > ts[best] * (1 + 1e-5)) and margin > 1e-5 and not close_other.any()
    return prim, t_out, robust


def main():
    with open(os.path.join(HERE, "morton_kats.json"), "w") as f:
        json.dump(morton_kats(), f, indent=1)
    with open(os.path.join(HERE, "sort_kats.json"), "w") as f:
        json.dump(sort_kats(), f, indent=1)
    lb, tr = {}, {}
    for name, make in FIXTURES.items():
        verts = make()
        lb[f"{name}__verts"] = verts
        for k, a in py_lbvh(verts).items():
            lb[f"{name}__{k}"] = a
        rays = fixture_rays(verts)
        prim, t, robust = brute64(verts, rays)
        tr[f"{name}__rays"] = rays
        tr[f"{name}__prim"] = prim
        tr[f"{name}__t"] = t
        tr[f"{name}__robust"] = robust
    np.savez_compressed(os.path.join(HERE, "lbvh_fixtures.npz"), **lb)
    np.savez_compressed(os.path.join(HERE, "trace_fixtures.npz"), **tr)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
