// traverse.cuh -- closest-hit / any-hit traversal of the binary LBVH.
//
// Restates the reference's two-child near-first loop
// (bajo/bvh/gpu/trace.mojo:340-428) over the binary node layout the build
// emits: node_bounds holds both child boxes of a node (48 B) and node_meta its
// tagged child refs (16 B), so one node costs four 16-byte loads; leaves are
// the sorted 48-byte triangle records.  Leaf children are intersected at once,
// the nearer internal child is taken, the other is pushed while it is still
// within reach.
//
// Differences from the reference, shared with the oracle:
//  - ties in t go to the lowest primitive id (the reference keeps the first
//    candidate visited);
//  - child boxes are entered while t_near <= t_far * (1 + 2^-20), which makes
//    the result independent of the visiting order;
//  - ray axes with |d| <= 1e-9 are tested by containment;
//  - BAJO_TRI_WATERTIGHT selects the watertight test of Woop, Benthin and
//    Wald (JCGT 2013); BAJO_TRI_MT is the reference's Moller-Trumbore
//    (bajo/core/intersect.mojo:415-459).
//
// With TOP, the first BAJO_TOP_NODES nodes of the tree (breadth first, built
// by the LBVH build into BajoLbvh::top_nodes) are read from shared memory:
// each block copies them once with a bulk asynchronous copy (TMA) completing
// on an mbarrier.  Refs tagged BAJO_TOP_FLAG name a staged slot; the boxes and
// child order are the same, so the hits are the same.
#pragma once

#include "bajo_common.cuh"

namespace bajo {
namespace trav {

constexpr int kTraceBlock = 128;
constexpr int kStack = 64;  // Karras trees over 64-bit keys are at most 64 levels deep

struct Ray {
  f3 o, d, rcp;
  float tmin, tmax;
  int kx, ky, kz;
  float sx, sy, sz;
  bool px, py, pz;  // |d| <= 1e-9 on this axis
};

// ray.mojo:86-111 rcp_direction (|d| > 1e-9 ? 1/d : +-1e9)
__device__ __forceinline__ float rcp1(float d) {
  const float eps = 1.0e-9f;
  const float large = 1.0f / eps;
  return fabsf(d) > eps ? 1.0f / d : (d < 0.0f ? -large : large);
}

__device__ __forceinline__ Ray make_ray(f3 o, f3 d, float tmin, float tmax) {
  Ray r;
  r.o = o;
  r.d = d;
  r.tmin = tmin;
  r.tmax = tmax;
  r.rcp = mk(rcp1(d.x), rcp1(d.y), rcp1(d.z));
  r.px = !(fabsf(d.x) > 1.0e-9f);
  r.py = !(fabsf(d.y) > 1.0e-9f);
  r.pz = !(fabsf(d.z) > 1.0e-9f);
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  r.kx = r.kz == 2 ? 0 : r.kz + 1;
  r.ky = r.kx == 2 ? 0 : r.kx + 1;
  float dz = comp(d, r.kz);
  if (dz < 0.0f) {
    int t = r.kx;
    r.kx = r.ky;
    r.ky = t;
  }
  r.sx = comp(d, r.kx) / dz;
  r.sy = comp(d, r.ky) / dz;
  r.sz = 1.0f / dz;
  return r;
}

struct Hit {
  float t, u, v;
  uint32_t prim, leaf;
};

// Per-ray traversal counters, in the order of the reference's
// GpuTraversalStats (bajo/bvh/gpu/trace.mojo:62-90): internal nodes visited,
// internal children whose box was hit, leaf blocks entered, triangles
// tested, deepest stack.
constexpr int kStatNodeVisits = 0, kStatChildHits = 1, kStatLeafBlocks = 2, kStatPrimTests = 3, kStatMaxStack = 4;
constexpr int kStatWords = BAJO_TRACE_STATS_WORDS;

__device__ __forceinline__ bool better(float t, uint32_t prim, const Hit& h) {
  return t < h.t || (t == h.t && prim < h.prim);
}

// One slab: (b - o) * rcp, except on axes the ray is parallel to
// (|d| <= 1e-9), which are tested by containment ([-inf, inf] when the origin
// lies in [bmin, bmax], empty otherwise).  With the reference's +-1e9
// reciprocal (ray.mojo:86-111) a ray running exactly along a box face gets an
// empty slab; containment keeps such rays inside the closed box.
// PAR = false compiles the slab for rays with no parallel axis (the common
// case: no selects); the result is the same as with PAR = true for them.
template <bool PAR>
__device__ __forceinline__ void slab(float bmin, float bmax, float o, float rcp, bool par, float& t0, float& t1) {
  const float a = (bmin - o) * rcp, b = (bmax - o) * rcp;
  if constexpr (PAR) {
    t0 = par ? (bmin <= o ? -INFINITY : INFINITY) : a;
    t1 = par ? (bmax >= o ? INFINITY : -INFINITY) : b;
  } else {
    t0 = a;
    t1 = b;
  }
}

__device__ __forceinline__ bool has_parallel_axis(const Ray& r) { return r.px || r.py || r.pz; }

// intersect.mojo:193-215, far bound scaled by kSlack
template <bool PAR = true>
__device__ __forceinline__ bool box_hit(const Ray& r, float4 a, float2 b, float tlimit, float& tnear) {
  // a = (min x, min y, min z, max x), b = (max y, max z)
  float t0x, t1x, t0y, t1y, t0z, t1z;
  slab<PAR>(a.x, a.w, r.o.x, r.rcp.x, r.px, t0x, t1x);
  slab<PAR>(a.y, b.x, r.o.y, r.rcp.y, r.py, t0y, t1y);
  slab<PAR>(a.z, b.y, r.o.z, r.rcp.z, r.pz, t0z, t1z);
  float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
  float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), tlimit));
  tnear = tn;
  return tn <= tf * kSlack;
}

// intersect.mojo:415-459
__device__ __forceinline__ bool tri_mt(const Ray& r, f3 v0, f3 e1, f3 e2, float& t, float& u, float& v) {
  f3 p = cross(r.d, e2);
  float det = dot(e1, p);
  bool det_ok = det > 1e-8f || det < -1e-8f;
  float inv_det = 1.0f / det;
  f3 tv = r.o - v0;
  float uu = dot(tv, p) * inv_det;
  f3 q = cross(tv, e1);
  float vv = dot(r.d, q) * inv_det;
  float tt = dot(e2, q) * inv_det;
  t = tt;
  u = uu;
  v = vv;
  return det_ok && uu >= 0.0f && uu <= 1.0f && vv >= 0.0f && (uu + vv) <= 1.0f && tt > r.tmin;
}

// Woop, Benthin, Wald, "Watertight Ray/Triangle Intersection", JCGT 2(1)
// 2013: shear into ray space, edge functions without contraction (built with
// -fmad=false), double-precision re-evaluation of exactly-zero edges.
__device__ __forceinline__ bool tri_wt(const Ray& r, f3 v0, f3 v1, f3 v2, float& t, float& u, float& v) {
  f3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
  float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
  float Ax = comp(A, r.kx) - r.sx * Akz, Ay = comp(A, r.ky) - r.sy * Akz;
  float Bx = comp(B, r.kx) - r.sx * Bkz, By = comp(B, r.ky) - r.sy * Bkz;
  float Cx = comp(C, r.kx) - r.sx * Ckz, Cy = comp(C, r.ky) - r.sy * Ckz;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = U + V + W;
  if (det == 0.0f) return false;
  float Az = r.sz * Akz, Bz = r.sz * Bkz, Cz = r.sz * Ckz;
  float T = U * Az + V * Bz + W * Cz;
  float tt = T / det;
  t = tt;
  u = V / det;
  v = W / det;
  return tt > r.tmin;
}

template <int MODE>
__device__ __forceinline__ void test_tri(const Ray& r, const float4* __restrict__ tris, uint32_t leaf, Hit& h) {
  const float4 a = __ldg(tris + (size_t)leaf * 3 + 0);
  const float4 b = __ldg(tris + (size_t)leaf * 3 + 1);
  const float4 c = __ldg(tris + (size_t)leaf * 3 + 2);
  const uint32_t prim = __float_as_uint(a.w);
  f3 v0 = mk(a.x, a.y, a.z), v1 = mk(b.x, b.y, b.z), v2 = mk(c.x, c.y, c.z);
  float t, u, v;
  bool ok;
  if constexpr (MODE == BAJO_TRI_MT) ok = tri_mt(r, v0, v1 - v0, v2 - v0, t, u, v);
  else ok = tri_wt(r, v0, v1, v2, t, u, v);
  if (ok && t < r.tmax && better(t, prim, h)) {
    h.t = t;
    h.u = u;
    h.v = v;
    h.prim = prim;
    h.leaf = leaf;
  }
}

// ---- staged top levels -----------------------------------------------------
constexpr uint32_t kTopMask = BAJO_TOP_FLAG - 1u;
constexpr uint32_t kTopFloat4 = 1u + 4u * BAJO_TOP_NODES;  // header + records
constexpr uint64_t kStageWaitNs = 200000000ull;            // 200 ms

struct TopSmem {
  float4 rec[kTopFloat4];
  unsigned long long bar;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_timer_ns() - t0 > kStageWaitNs) return false;
  return true;
}

// Copies the staged top levels (g, BAJO_TOP_BYTES, 16-byte aligned) into
// shared memory: thread 0 arms the mbarrier with the byte count and issues
// one cp.async.bulk (no multicast); every thread waits, at most 200 ms.
// Returns the records when the copy arrived and belongs to `root`, else
// nullptr (the caller traverses from global memory; a timeout also raises
// BAJO_STATUS_STAGE_TIMEOUT).  Must be called by every thread of the block.
__device__ __forceinline__ const float4* stage_top(TopSmem& sm, const float4* __restrict__ g, uint32_t root,
                                                   uint32_t* status) {
  const uint32_t bar = smem_addr(&sm.bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(BAJO_TOP_BYTES)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(sm.rec)),
                 "l"(g), "r"(BAJO_TOP_BYTES), "r"(bar)
                 : "memory");
  }
  if (!mbar_wait_bounded(bar, 0)) {
    raise_status(status, BAJO_STATUS_STAGE_TIMEOUT);
    return nullptr;
  }
  const float4 h = sm.rec[0];
  const uint32_t count = __float_as_uint(h.x);
  if (count == 0 || count > BAJO_TOP_NODES || __float_as_uint(h.y) != root) return nullptr;
  return sm.rec + 1;
}

// A block that gave up waiting must not leave while the copy may still land
// in its shared memory: wait once more (bounded) before returning.
__device__ __forceinline__ void stage_top_drain(TopSmem& sm, const float4* staged) {
  if (staged == nullptr && threadIdx.x == 0) mbar_wait_bounded(smem_addr(&sm.bar), 0);
}

// Camera launches give each warp an 8 x 4 tile of pixels (tiles in rows,
// views one after another), so that a warp's rays leave the camera side by
// side instead of along one image row (1024^2 camera rays over the 65,536
// triangle workload: 0.316 against 0.349 ms).  Ray i is still pixel i of the
// row-major image, so the results do not depend on it.  tile_ray maps the
// launch's thread g to its ray i; false for lanes past the image or past n.
// A launch needs camera_threads(...) threads (whole warps of every view).
constexpr uint32_t kTileW = 8, kTileH = 4;
__host__ __device__ __forceinline__ uint64_t camera_tiles(uint32_t width, uint32_t height) {
  return (uint64_t)((width + kTileW - 1) / kTileW) * ((height + kTileH - 1) / kTileH);
}
__device__ __forceinline__ bool tile_ray(uint64_t g, uint32_t n, uint32_t width, uint32_t height, uint32_t& i) {
  const uint32_t tiles_x = (width + kTileW - 1) / kTileW;
  const uint64_t per_view = camera_tiles(width, height);
  const uint64_t warp = g >> 5, view = warp / per_view, tv = warp - view * per_view;
  const uint32_t lane = (uint32_t)(g & 31u);
  const uint32_t px = (uint32_t)(tv % tiles_x) * kTileW + lane % kTileW;
  const uint32_t py = (uint32_t)(tv / tiles_x) * kTileH + lane / kTileW;
  if (px >= width || py >= height) return false;
  const uint64_t at = view * ((uint64_t)width * height) + (uint64_t)py * width + px;
  if (at >= n) return false;
  i = (uint32_t)at;
  return true;
}
__host__ __device__ __forceinline__ uint64_t camera_threads(uint32_t n, uint32_t width, uint32_t height) {
  const uint64_t ppv = (uint64_t)width * height;
  return ppv ? (n + ppv - 1) / ppv * camera_tiles(width, height) * 32u : 0u;
}

// A traversal with a stack shallower than kStack that runs out of entries
// returns this in Hit::leaf; trace_bvh2 then traces the ray again with the
// full stack, so every stack depth gives the same hit.
constexpr uint32_t kRetrace = 0xFFFFFFFEu;

// max_nodes: node visits allowed (the node count): a tree is never visited
// twice per node, so more visits means a corrupt tree.  With TOP, `top` holds
// the staged records and refs tagged BAJO_TOP_FLAG are read from it.  STACK
// entries of traversal stack (kStack holds the deepest Karras tree).
template <int MODE, bool STATS, bool ANY, bool PAR, bool TOP = false, int STACK = kStack>
__device__ __forceinline__ Hit trace_bvh2_impl(const Ray& r, uint32_t root, const float4* __restrict__ nb,
                                               const uint4* __restrict__ meta, const float4* __restrict__ tris,
                                               uint32_t max_nodes, uint32_t* status, uint32_t* stats,
                                               const float4* top = nullptr) {
  Hit h;
  h.t = r.tmax;
  h.u = h.v = 0.0f;
  h.prim = kEmpty;
  h.leaf = kEmpty;
  if (root == kSentinel) return h;
  if (root & kLeafFlag) {
    test_tri<MODE>(r, tris, root & kIndexMask, h);
    if constexpr (STATS) {
      ++stats[kStatLeafBlocks];
      ++stats[kStatPrimTests];
    }
    return h;
  }
  // any-hit queries stop at the first accepted triangle; boxes are culled
  // against the ray's own t_max (bajo/bvh/gpu/trace.mojo:458-499)
  static_assert(STACK >= 1 && STACK <= kStack, "traversal stack depth");
  uint32_t stack[STACK];
  int sp = 0;
  uint32_t cur = root;
  // a corrupt tree or a full stack ends the walk; the status bit is raised
  // after the loop, which keeps the atomic out of the loop's code
  uint32_t fail = 0;
  for (uint32_t visits = 0;; ++visits) {
    const bool staged = TOP && (cur & BAJO_TOP_FLAG);
    if (visits >= max_nodes || (staged ? (cur & kTopMask) >= BAJO_TOP_NODES : cur >= max_nodes)) {
      fail = BAJO_STATUS_BAD_TOPOLOGY;
      break;
    }
    if constexpr (STATS) ++stats[kStatNodeVisits];
    float4 b0, b1, b2;  // b0 L: min xyz, max x | b1 L: max yz, R: min xy | b2 R: min z, max xyz
    uint2 m;            // left, right child refs
    if (staged) {
      const float4* p = top + (size_t)(cur & kTopMask) * 4;
      b0 = p[0];
      b1 = p[1];
      b2 = p[2];
      const float4 c = p[3];
      m = make_uint2(__float_as_uint(c.x), __float_as_uint(c.y));
    } else {
      b0 = __ldg(nb + (size_t)cur * 3 + 0);
      b1 = __ldg(nb + (size_t)cur * 3 + 1);
      b2 = __ldg(nb + (size_t)cur * 3 + 2);
      const uint4 g = __ldg(meta + cur);
      m = make_uint2(g.y, g.z);
    }
    float tl, tr;
    const float limit0 = ANY ? r.tmax : h.t;
    const bool hl = box_hit<PAR>(r, b0, make_float2(b1.x, b1.y), limit0, tl);
    const bool hr = box_hit<PAR>(r, make_float4(b1.z, b1.w, b2.x, b2.y), make_float2(b2.z, b2.w), limit0, tr);
    bool vl = false, vr = false;
    if (hl) {
      if (m.x & kLeafFlag) {
        test_tri<MODE>(r, tris, m.x & kIndexMask, h);
        if constexpr (STATS) {
          ++stats[kStatLeafBlocks];
          ++stats[kStatPrimTests];
        }
        if (ANY && h.leaf != kEmpty) return h;
      } else vl = true;
    }
    if (hr) {
      if (m.y & kLeafFlag) {
        test_tri<MODE>(r, tris, m.y & kIndexMask, h);
        if constexpr (STATS) {
          ++stats[kStatLeafBlocks];
          ++stats[kStatPrimTests];
        }
        if (ANY && h.leaf != kEmpty) return h;
      } else vr = true;
    }
    if constexpr (STATS) stats[kStatChildHits] += (uint32_t)vl + (uint32_t)vr;
    int near = -1;
    if (vl) near = 0;
    if (vr && (near == -1 || tr < tl)) near = 1;
    if (near >= 0) {
      const float limit = (ANY ? r.tmax : h.t) * kSlack;
      const bool far_valid = near == 0 ? vr : vl;
      const float far_t = near == 0 ? tr : tl;
      const float near_t = near == 0 ? tl : tr;
      if (far_valid && far_t <= limit) {
        if (sp < STACK) {
          stack[sp++] = near == 0 ? m.y : m.x;
        } else if constexpr (STACK < kStack) {
          h.leaf = kRetrace;  // the caller traces this ray again with kStack entries
          return h;
        } else {  // deeper than any Karras tree over 64-bit keys: a corrupt tree
          fail = BAJO_STATUS_STACK_OVERFLOW;
          break;
        }
        if constexpr (STATS) stats[kStatMaxStack] = max(stats[kStatMaxStack], (uint32_t)sp);
      }
      if (near_t <= limit) {
        cur = near == 0 ? m.x : m.y;
        continue;
      }
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
  if (fail) raise_status(status, fail);
  return h;
}

// Rays with an axis parallel to the boxes (|d| <= 1e-9) take the containment
// slab; every other ray takes the select-free one.  With STACK < kStack a ray
// whose traversal needs more entries is traced again with kStack (counted
// twice by STATS, which the instrumented kernels therefore never combine
// with a short stack).
template <int MODE, bool STATS = false, bool ANY = false, int STACK = kStack>
__device__ __forceinline__ Hit trace_bvh2(const Ray& r, uint32_t root, const float4* __restrict__ nb,
                                          const uint4* __restrict__ meta, const float4* __restrict__ tris,
                                          uint32_t max_nodes, uint32_t* status, uint32_t* stats = nullptr) {
  static_assert(STACK == kStack || !STATS, "instrumented traversals use the full stack");
  if (has_parallel_axis(r)) {
    const Hit h = trace_bvh2_impl<MODE, STATS, ANY, true, false, STACK>(r, root, nb, meta, tris, max_nodes, status,
                                                                         stats);
    if (STACK == kStack || h.leaf != kRetrace) return h;
    return trace_bvh2_impl<MODE, STATS, ANY, true>(r, root, nb, meta, tris, max_nodes, status, stats);
  }
  const Hit h = trace_bvh2_impl<MODE, STATS, ANY, false, false, STACK>(r, root, nb, meta, tris, max_nodes, status,
                                                                        stats);
  if (STACK == kStack || h.leaf != kRetrace) return h;
  return trace_bvh2_impl<MODE, STATS, ANY, false>(r, root, nb, meta, tris, max_nodes, status, stats);
}

// Same, starting from the staged top (slot 0 is `root`) when `top` is set.
// Trees of 2^30 or more nodes are never staged (the build leaves the count 0).
template <int MODE, bool STATS = false, bool ANY = false>
__device__ __forceinline__ Hit trace_bvh2_top(const Ray& r, uint32_t root, const float4* __restrict__ nb,
                                              const uint4* __restrict__ meta, const float4* __restrict__ tris,
                                              uint32_t max_nodes, uint32_t* status, const float4* top,
                                              uint32_t* stats = nullptr) {
  // without staged records no ref carries BAJO_TOP_FLAG (node indices stay
  // below 2^30), so the same loop runs from the global root
  const uint32_t start = top ? BAJO_TOP_FLAG : root;
  if (has_parallel_axis(r))
    return trace_bvh2_impl<MODE, STATS, ANY, true, true>(r, start, nb, meta, tris, max_nodes, status, stats, top);
  return trace_bvh2_impl<MODE, STATS, ANY, false, true>(r, start, nb, meta, tris, max_nodes, status, stats, top);
}

}  // namespace trav
}  // namespace bajo
