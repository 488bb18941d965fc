// wide.cuh -- the W-wide BVH (W = 4 or 8) collapsed from the binary LBVH:
// node and leaf layouts, the child-opening rule, and closest-hit traversal.
//
// Layouts are the reference's (bajo/bvh/constants.mojo:26,47-55,
// bajo/bvh/wide_meta.mojo:7-47):
//  - node i: 7 fields x W lanes of f32, field-major: [min x][min y][min z]
//    [max x][max y][max z][meta] (meta as u32 bits); an empty lane has an
//    invalid box (min = FLT_MAX, max = -FLT_MAX) and meta 0xFFFFFFFF;
//  - meta = count << 26 | index: count 0 = internal child (index = wide node),
//    count k in 1..4 = leaf block of k triangles (index = leaf block); indices
//    are local to the segment;
//  - leaf block b: W payloads (item ids, 0xFFFFFFFF padding) and W packed
//    triangles, AoSoA [v0 x, y, z][prim][e1 x, y, z][0][e2 x, y, z][0] x W
//    (pack_segmented_triangle_leaf_lanes_kernel, triangle_bvh.mojo:81-148),
//    prim = segment-local id, e1 = v1 - v0, e2 = v2 - v0.
// This library adds leaf_sorted[b][lane] = the binary tree's sorted leaf of
// each lane, which the watertight test uses to read the original vertices.
#pragma once

#include "traverse.cuh"

namespace bajo {
namespace wide {

constexpr int kFields = 7;
constexpr uint32_t kFatLeaf = 4;  // HIPRT fat leaves: binary subtrees of <= 4 triangles (the largest leaf)
constexpr uint32_t kCountShift = 26, kDataMask = 0x03FFFFFFu;
constexpr int kLeafStride = 12;   // TRI_LEAF_PACKED_STRIDE

__host__ __device__ __forceinline__ uint32_t pack_meta(uint32_t data, uint32_t count) {
  return (count << kCountShift) | (data & kDataMask);
}

struct Box {
  f3 mn, mx;
};

__device__ __forceinline__ float area(const Box& b) {
  const f3 d = b.mx - b.mn;
  return 2.0f * ((d.x * d.y + d.x * d.z) + d.y * d.z);
}

// bounds of a binary ref: a leaf's AABB (item order) or the union of an
// internal node's two child boxes (_encoded_bounds, binary_layout.mojo:65-80)
__device__ __forceinline__ Box ref_bounds(uint32_t ref, const float* __restrict__ leaf_bounds,
                                          const uint32_t* __restrict__ leaf_ids,
                                          const float* __restrict__ node_bounds) {
  Box b;
  if (ref & kLeafFlag) {
    const float* p = leaf_bounds + (size_t)__ldg(leaf_ids + (ref & kIndexMask)) * 6;
    b.mn = mk(__ldg(p + 0), __ldg(p + 1), __ldg(p + 2));
    b.mx = mk(__ldg(p + 3), __ldg(p + 4), __ldg(p + 5));
  } else {
    const float* p = node_bounds + (size_t)(ref & kIndexMask) * 12;
    b.mn = vmin(mk(__ldg(p + 0), __ldg(p + 1), __ldg(p + 2)), mk(__ldg(p + 6), __ldg(p + 7), __ldg(p + 8)));
    b.mx = vmax(mk(__ldg(p + 3), __ldg(p + 4), __ldg(p + 5)), mk(__ldg(p + 9), __ldg(p + 10), __ldg(p + 11)));
  }
  return b;
}

__device__ __forceinline__ uint32_t ref_count(uint32_t ref, const uint32_t* __restrict__ node_leaf_counts) {
  return (ref & kLeafFlag) ? 1u : __ldg(node_leaf_counts + (ref & kIndexMask));
}

// max_leaf: triangles a leaf block may hold (1 = every triangle its own
// leaf, the reference's fat_leaves = false; 4 = HIPRT fat leaves)
__device__ __forceinline__ bool terminal(uint32_t ref, uint32_t count, uint32_t max_leaf) {
  return (ref & kLeafFlag) || count <= max_leaf;
}

// Children of the wide node rooted at binary internal node x
// (hploc_literature_to_wide_kernel, wide_collapse.mojo:318-444): start from
// x's two children; first open the internal candidate of largest surface
// area among those with more than max_leaf triangles until W candidates or
// none is left, then open the largest remaining internal candidates until
// full.  An opened candidate is replaced by its left child and its right child
// is appended.  Ties keep the first candidate.  Only internal candidates are
// ever opened, so only their areas are read: `area` holds each internal
// node's box area (area(), computed once per node by the bottom-up pass; L2
// loads, as the values were written by other threads during that pass).
// Returns the candidate count.
template <int W>
__device__ __forceinline__ int open_children(uint32_t x, const uint32_t* __restrict__ node_meta,
                                             const uint32_t* __restrict__ node_leaf_counts,
                                             const float* area, uint32_t max_leaf, uint32_t cand[W],
                                             uint32_t cnt[W]) {
  float ar[W];
  cand[0] = __ldg(node_meta + (size_t)x * 4 + 1);
  cand[1] = __ldg(node_meta + (size_t)x * 4 + 2);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    cnt[k] = ref_count(cand[k], node_leaf_counts);
    ar[k] = (cand[k] & kLeafFlag) ? 0.0f : __ldcg(area + (cand[k] & kIndexMask));
  }
  int n = 2;
  for (int phase = 0; phase < 2; ++phase) {
    while (n < W) {
      int pos = -1;
      float best = -1.0f;
      for (int k = 0; k < n; ++k) {
        if (cand[k] & kLeafFlag) continue;
        if (phase == 0 && cnt[k] <= max_leaf) continue;
        if (ar[k] > best) {
          best = ar[k];
          pos = k;
        }
      }
      if (pos < 0) break;
      const uint32_t y = cand[pos] & kIndexMask;
      cand[pos] = __ldg(node_meta + (size_t)y * 4 + 1);
      cand[n] = __ldg(node_meta + (size_t)y * 4 + 2);
      cnt[pos] = ref_count(cand[pos], node_leaf_counts);
      cnt[n] = ref_count(cand[n], node_leaf_counts);
      ar[pos] = (cand[pos] & kLeafFlag) ? 0.0f : __ldcg(area + (cand[pos] & kIndexMask));
      ar[n] = (cand[n] & kLeafFlag) ? 0.0f : __ldcg(area + (cand[n] & kIndexMask));
      ++n;
    }
  }
  return n;
}

// ---------------------------------------------------------------------------
// traversal
// ---------------------------------------------------------------------------
struct View {
  const float* nodes;          // the segment's first node
  const float* leaf_tris;      // the segment's first leaf block (AoSoA)
  const uint32_t* leaf_sorted; // the segment's first leaf block
  const float4* bvh2_tris;     // binary tree's sorted triangle records
  uint32_t n_nodes;            // visit bound
  uint32_t n_blocks;           // leaf blocks of the segment
};

// Closest hit (or any hit) over the wide tree.  Leaf lanes are tested when
// their box is hit; the nearest hit internal child is visited next and the
// others are pushed farthest first with their entry distance, and skipped on
// pop once the hit is nearer.  The same order-independent rules as the
// binary traversal (lowest prim on ties, conservative slabs) make the result
// equal to the binary tree's bit for bit.
template <int W, int MODE, bool STATS, bool ANY, bool PAR>
__device__ __forceinline__ trav::Hit trace_wide_impl(const trav::Ray& r, const View& v, uint32_t* status,
                                                     uint32_t* stats) {
  trav::Hit h;
  h.t = r.tmax;
  h.u = h.v = 0.0f;
  h.prim = kEmpty;
  h.leaf = kEmpty;
  if (v.n_nodes == 0) return h;
  uint2 stack[trav::kStack];
  int sp = 0;
  uint32_t cur = 0;
  uint32_t fail = 0;  // status bits, raised after the loop (no atomic in the loop's code)
  for (uint32_t visits = 0;; ++visits) {
    if (visits >= v.n_nodes || cur >= v.n_nodes) {
      fail |= BAJO_STATUS_BAD_TOPOLOGY;
      break;
    }
    if constexpr (STATS) ++stats[trav::kStatNodeVisits];
    const float4* node = reinterpret_cast<const float4*>(v.nodes + (size_t)cur * kFields * W);
    float f[kFields][W];
#pragma unroll
    for (int q = 0; q < kFields * W / 4; ++q) {
      const float4 x = __ldg(node + q);
      f[(4 * q) / W][(4 * q) % W] = x.x;
      f[(4 * q + 1) / W][(4 * q + 1) % W] = x.y;
      f[(4 * q + 2) / W][(4 * q + 2) % W] = x.z;
      f[(4 * q + 3) / W][(4 * q + 3) % W] = x.w;
    }
    uint32_t ci[W];
    float ct[W];
    int nc = 0;
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const uint32_t meta = __float_as_uint(f[6][j]);
      if (meta == kEmpty) continue;
      float tn;
      const float limit = ANY ? r.tmax : h.t;
      if (!trav::box_hit<PAR>(r, make_float4(f[0][j], f[1][j], f[2][j], f[3][j]), make_float2(f[4][j], f[5][j]),
                         limit, tn))
        continue;
      const uint32_t count = meta >> kCountShift, data = meta & kDataMask;
      if (count == 0) {
        if constexpr (STATS) ++stats[trav::kStatChildHits];
        ci[nc] = data;
        ct[nc] = tn;
        ++nc;
        continue;
      }
      if (data >= v.n_blocks) {
        fail |= BAJO_STATUS_BAD_TOPOLOGY;
        continue;
      }
      if constexpr (STATS) ++stats[trav::kStatLeafBlocks];
      const size_t base = (size_t)data * kLeafStride * W;
      for (uint32_t k = 0; k < count; ++k) {
        if constexpr (STATS) ++stats[trav::kStatPrimTests];
        float t, u, vv;
        bool ok;
        uint32_t prim;
        if constexpr (MODE == BAJO_TRI_MT) {
          const float* L = v.leaf_tris + base + k;
          const f3 v0 = mk(__ldg(L + 0 * W), __ldg(L + 1 * W), __ldg(L + 2 * W));
          prim = __float_as_uint(__ldg(L + 3 * W));
          const f3 e1 = mk(__ldg(L + 4 * W), __ldg(L + 5 * W), __ldg(L + 6 * W));
          const f3 e2 = mk(__ldg(L + 8 * W), __ldg(L + 9 * W), __ldg(L + 10 * W));
          ok = trav::tri_mt(r, v0, e1, e2, t, u, vv);
        } else {
          const uint32_t sl = __ldg(v.leaf_sorted + (size_t)data * W + k);
          const float4 a = __ldg(v.bvh2_tris + (size_t)sl * 3 + 0);
          const float4 b = __ldg(v.bvh2_tris + (size_t)sl * 3 + 1);
          const float4 c = __ldg(v.bvh2_tris + (size_t)sl * 3 + 2);
          prim = __float_as_uint(a.w);
          ok = trav::tri_wt(r, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), mk(c.x, c.y, c.z), t, u, vv);
        }
        if (ok && t < r.tmax && trav::better(t, prim, h)) {
          h.t = t;
          h.u = u;
          h.v = vv;
          h.prim = prim;
          h.leaf = __ldg(v.leaf_sorted + (size_t)data * W + k);
          if (ANY) {
            if (fail) raise_status(status, fail);
            return h;
          }
        }
      }
    }
    // order the hit internal children by entry distance, nearest first
#pragma unroll
    for (int a = 1; a < W; ++a) {
      if (a >= nc) break;
      const float tk = ct[a];
      const uint32_t ik = ci[a];
      int b = a - 1;
      while (b >= 0 && ct[b] > tk) {
        ct[b + 1] = ct[b];
        ci[b + 1] = ci[b];
        --b;
      }
      ct[b + 1] = tk;
      ci[b + 1] = ik;
    }
    const float limit = (ANY ? r.tmax : h.t) * kSlack;
    for (int k = nc - 1; k >= 1; --k) {
      if (ct[k] > limit) continue;
      if (sp < trav::kStack) stack[sp++] = make_uint2(ci[k], __float_as_uint(ct[k]));
      else fail |= BAJO_STATUS_STACK_OVERFLOW;
      if constexpr (STATS) stats[trav::kStatMaxStack] = max(stats[trav::kStatMaxStack], (uint32_t)sp);
    }
    if (nc > 0 && ct[0] <= limit) {
      cur = ci[0];
      continue;
    }
    bool found = false;
    while (sp > 0) {
      const uint2 e = stack[--sp];
      if (__uint_as_float(e.y) <= (ANY ? r.tmax : h.t) * kSlack) {
        cur = e.x;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  if (fail) raise_status(status, fail);
  return h;
}

template <int W, int MODE, bool STATS = false, bool ANY = false>
__device__ __forceinline__ trav::Hit trace_wide(const trav::Ray& r, const View& v, uint32_t* status,
                                                uint32_t* stats = nullptr) {
  if (trav::has_parallel_axis(r)) return trace_wide_impl<W, MODE, STATS, ANY, true>(r, v, status, stats);
  return trace_wide_impl<W, MODE, STATS, ANY, false>(r, v, status, stats);
}

}  // namespace wide
}  // namespace bajo
