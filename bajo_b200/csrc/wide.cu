// wide.cu -- deterministic BVH2 -> W-wide collapse (W = 4, 8) of a built
// binary LBVH, and closest-hit traversal of the wide tree.
//
// Reference: hploc_literature_to_wide_kernel (bajo/bvh/gpu/builder/
// wide_collapse.mojo:148-644; H-PLOC paper section 3.4, HIPRT fat leaves) and
// pack_segmented_triangle_leaf_lanes_kernel (bajo/bvh/gpu/triangle_bvh.mojo:
// 81-148), driven by enqueue_segmented_wide_build (segmented_build.mojo:89)
// with max_leaf_size = leaf width and fat leaves on.  The reference hands out
// node and leaf ids with atomics while its work queue runs -- a node takes its
// internal children's ids as one contiguous range and its leaf blocks as
// another (wide_collapse.mojo:551-559) -- so its layout differs from run to
// run; here ids have the same shape and are fixed:
//   1. count_kernel climbs the binary tree bottom-up (refit-style arrival
//      flags) and, at every internal node x, applies the opening rule to
//      find the children the wide node rooted at x would have, and the
//      number of wide nodes NW(x) and leaf blocks NL(x) of that collapsed
//      subtree;
//   2. offsets_kernel turns the roots' counts into per-segment node and leaf
//      offsets and publishes each root's task;
//   3. assign_kernel processes the wide nodes through a FIFO queue: a node's
//      task (binary node, first descendant id D, first leaf block, first
//      triangle) is written by its parent, which then appends the node's id
//      to the queue; every thread takes queue slots in turn and waits (with a
//      bound) until its slot is filled.  The set of processed nodes is closed
//      under children, so while a slot is empty some resident thread holds an
//      earlier slot and will fill it: a resident grid always progresses.
//      Node I gives its internal children the ids D, D + 1, ... in lane
//      order, hands child c the descendant range after its siblings' (D +
//      internal children + the NW - 1 of the children before it) with the
//      matching leaf base, publishes the children's tasks, and only then
//      writes its own lane boxes and leaf blocks.  Ids depend only on the
//      tree, never on the processing order.
//
// The CWBVH8 build (W = 8, leaves of at most 3 triangles) runs the same three
// kernels with octant slots (spatial_slots, wide_collapse.mojo:457-521: the
// candidates go to the eight lanes by a greedy centroid-octant assignment) and
// encodes each node straight from its lane boxes into the 80-byte compressed
// node of _encode_cwbvh8_node (compressed_bounds_bvh.mojo:84-325), packing its
// triangles as 48-byte records (pack_segmented_cwbvh_triangles_kernel,
// :372-404).  The reference reserves a node's triangle range with an atomic
// counter; here node I's range starts at the first triangle of I's subtree in
// depth-first lane order (own leaf lanes, then each internal child's subtree),
// one of the orders that atomic can produce.
#include <algorithm>

#include "wide.cuh"

namespace bajo {
int sm_count();

namespace wide {

constexpr int kBlock = 128;
constexpr uint64_t kWaitNs = 200000000ull;  // 200 ms bound on one task wait

struct Work {
  uint32_t* flags;      // [internal] arrival counters
  uint32_t* cands;      // [internal][W] children of the wide node rooted there
  uint32_t* cinfo;      // [internal] candidate count | terminal mask << 8
  uint32_t* nw;         // [internal] wide nodes of the collapsed subtree
  uint32_t* nl;         // [internal] leaf blocks of the collapsed subtree
  uint32_t* task_ref;   // [wide node] binary ref
  uint32_t* task_leaf;  // [wide node] first leaf block (global)
  uint32_t* task_seg;   // [wide node] segment
  uint32_t* task_desc;  // [wide node] id of its first internal child (global)
  uint32_t* task_tri;   // [wide node] first triangle of its subtree (global; CWBVH8)
  float* area;          // [internal] box area of each binary node
  uint32_t* queue;      // [slot] 1 + id of a wide node whose task is published (0 = not yet)
  uint32_t* head;       // next queue slot to take
  uint32_t* tail;       // next queue slot to fill
  uint32_t* status;
};

template <int W>
__global__ void __launch_bounds__(kBlock) count_kernel(uint32_t n, const uint32_t* __restrict__ node_meta,
                                                       const uint32_t* __restrict__ leaf_parent,
                                                       const uint32_t* __restrict__ node_leaf_counts,
                                                       const float* __restrict__ leaf_bounds,
                                                       const uint32_t* __restrict__ leaf_ids,
                                                       const float* __restrict__ node_bounds, uint32_t max_leaf,
                                                       Work wk) {
  const uint32_t s = blockIdx.x * kBlock + threadIdx.x;
  if (s >= n) return;
  uint32_t parent = leaf_parent[s];
  for (int depth = 0; parent != kSentinel; ++depth) {
    if (depth > 128 || parent >= n) {
      raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
      return;
    }
    // the second arrival sees every result of the subtree (acq_rel chain)
    if (atomic_add_acq_rel_gpu(&wk.flags[parent], 1u) == 0) return;
    const uint32_t x = parent;
    wk.area[x] = area(ref_bounds(x, leaf_bounds, leaf_ids, node_bounds));
    uint32_t cand[W], cnt[W];
    const int nc = open_children<W>(x, node_meta, node_leaf_counts, wk.area, max_leaf, cand, cnt);
    uint32_t nodes = 1, leaves = 0, mask = 0;
    for (int k = 0; k < nc; ++k) {
      if (terminal(cand[k], cnt[k], max_leaf)) {
        ++leaves;
        mask |= 1u << k;
      } else {
        const uint32_t c = cand[k] & kIndexMask;
        nodes += __ldcg(wk.nw + c);
        leaves += __ldcg(wk.nl + c);
      }
    }
    for (int k = 0; k < W; ++k) wk.cands[(size_t)x * W + k] = k < nc ? cand[k] : kEmpty;
    wk.cinfo[x] = (uint32_t)nc | (mask << 8);
    wk.nw[x] = nodes;
    wk.nl[x] = leaves;
    parent = __ldg(node_meta + (size_t)x * 4 + 0);
  }
}

// node / leaf-block counts of a segment's root
__device__ __forceinline__ void root_counts(uint32_t s, const uint32_t* __restrict__ seg_offsets,
                                            const uint32_t* __restrict__ roots,
                                            const uint32_t* __restrict__ node_leaf_counts, uint32_t max_leaf,
                                            const Work& wk, uint32_t& nodes, uint32_t& leaves) {
  nodes = leaves = 0;
  if (seg_offsets[s + 1] == seg_offsets[s]) return;
  const uint32_t r = roots[s];
  if (terminal(r, ref_count(r, node_leaf_counts), max_leaf)) {
    nodes = leaves = 1;
  } else {
    nodes = wk.nw[r & kIndexMask];
    leaves = wk.nl[r & kIndexMask];
  }
}

// one block: exclusive scans of the per-segment counts, then the roots' tasks
__global__ void __launch_bounds__(1024) offsets_kernel(uint32_t n_seg, const uint32_t* __restrict__ seg_offsets,
                                                       const uint32_t* __restrict__ roots,
                                                       const uint32_t* __restrict__ node_leaf_counts,
                                                       uint32_t max_leaf, Work wk, uint32_t cap,
                                                       uint32_t* __restrict__ node_offsets,
                                                       uint32_t* __restrict__ leaf_offsets) {
  __shared__ uint32_t sn[1024], sl[1024];
  const uint32_t t = threadIdx.x;
  const uint32_t per = (n_seg + 1023) / 1024;
  const uint32_t b = t * per, e = min(n_seg, b + per);
  uint32_t an = 0, al = 0;
  for (uint32_t s = b; s < e; ++s) {
    uint32_t cn, cl;
    root_counts(s, seg_offsets, roots, node_leaf_counts, max_leaf, wk, cn, cl);
    an += cn;
    al += cl;
  }
  sn[t] = an;
  sl[t] = al;
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) {  // inclusive Hillis-Steele scan
    const uint32_t vn = t >= off ? sn[t - off] : 0, vl = t >= off ? sl[t - off] : 0;
    __syncthreads();
    sn[t] += vn;
    sl[t] += vl;
    __syncthreads();
  }
  uint32_t pn = sn[t] - an, pl = sl[t] - al;
  for (uint32_t s = b; s < e; ++s) {
    uint32_t cn, cl;
    root_counts(s, seg_offsets, roots, node_leaf_counts, max_leaf, wk, cn, cl);
    node_offsets[s] = pn;
    leaf_offsets[s] = pl;
    if (cn && pn < cap) {
      wk.task_ref[pn] = roots[s];
      wk.task_leaf[pn] = pl;
      wk.task_seg[pn] = s;
      wk.task_desc[pn] = pn + 1u;
      wk.task_tri[pn] = seg_offsets[s];
      wk.queue[atomicAdd(wk.tail, 1u)] = pn + 1u;
    }
    pn += cn;
    pl += cl;
  }
  if (t == 1023) {
    node_offsets[n_seg] = sn[1023];
    leaf_offsets[n_seg] = sl[1023];
  }
}

struct Out {
  float* nodes;
  uint32_t* leaf_indices;
  float* leaf_tris;
  uint32_t* leaf_sorted;
  float4* cw_nodes;  // CWBVH8: [node][5] (80 B)
  float4* cw_tris;   // CWBVH8: [triangle][3] (48 B)
};

// leaf block `blk` (global) from the binary subtree `ref` (<= 4 leaves),
// left to right (_write_hploc_terminal_leaf_block, wide_collapse.mojo:67-104)
template <int W>
__device__ void write_leaf_block(uint32_t ref, uint32_t blk, const uint32_t* __restrict__ node_meta,
                                 const uint32_t* __restrict__ leaf_ids, const float4* __restrict__ tris,
                                 const Out& o, uint32_t* status) {
  uint32_t stack[kFatLeaf + 1];
  int sp = 0, lane = 0;
  stack[sp++] = ref;
  float* L = o.leaf_tris + (size_t)blk * kLeafStride * W;
  while (sp > 0) {
    const uint32_t cur = stack[--sp];
    if (cur & kLeafFlag) {
      if (lane >= W) {
        raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        return;
      }
      const uint32_t sl = cur & kIndexMask;
      const float4 a = __ldg(tris + (size_t)sl * 3 + 0);
      const float4 b = __ldg(tris + (size_t)sl * 3 + 1);
      const float4 c = __ldg(tris + (size_t)sl * 3 + 2);
      const f3 v0 = mk(a.x, a.y, a.z);
      const f3 e1 = mk(b.x, b.y, b.z) - v0, e2 = mk(c.x, c.y, c.z) - v0;
      o.leaf_indices[(size_t)blk * W + lane] = __ldg(leaf_ids + sl);
      o.leaf_sorted[(size_t)blk * W + lane] = sl;
      L[0 * W + lane] = v0.x; L[1 * W + lane] = v0.y; L[2 * W + lane] = v0.z; L[3 * W + lane] = a.w;
      L[4 * W + lane] = e1.x; L[5 * W + lane] = e1.y; L[6 * W + lane] = e1.z; L[7 * W + lane] = 0.0f;
      L[8 * W + lane] = e2.x; L[9 * W + lane] = e2.y; L[10 * W + lane] = e2.z; L[11 * W + lane] = 0.0f;
      ++lane;
    } else {
      if (sp + 2 > (int)kFatLeaf + 1) {
        raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        return;
      }
      const uint32_t y = cur & kIndexMask;
      stack[sp++] = __ldg(node_meta + (size_t)y * 4 + 2);  // right first: lanes run left to right
      stack[sp++] = __ldg(node_meta + (size_t)y * 4 + 1);
    }
  }
  for (; lane < W; ++lane) {
    o.leaf_indices[(size_t)blk * W + lane] = kEmpty;
    o.leaf_sorted[(size_t)blk * W + lane] = kEmpty;
    for (int fld = 0; fld < kLeafStride; ++fld) L[fld * W + lane] = fld == 3 ? __uint_as_float(kEmpty) : 0.0f;
  }
}

// CWBVH8 triangle records of the binary subtree `ref` (<= 3 leaves), left to
// right, from global position `pos` (pack_segmented_cwbvh_triangles_kernel,
// compressed_bounds_bvh.mojo:372-404): [e1][0][e2][0][v0][segment-local prim].
// Returns the position after the last record.
__device__ uint32_t write_cw_tris(uint32_t ref, uint32_t pos, uint32_t cap, const uint32_t* __restrict__ node_meta,
                                  const float4* __restrict__ tris, const Out& o, uint32_t* status) {
  uint32_t stack[kFatLeaf + 1];
  int sp = 0;
  stack[sp++] = ref;
  while (sp > 0) {
    const uint32_t cur = stack[--sp];
    if (cur & kLeafFlag) {
      if (pos >= cap) {
        raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        return pos;
      }
      const uint32_t sl = cur & kIndexMask;
      const float4 a = __ldg(tris + (size_t)sl * 3 + 0);
      const float4 b = __ldg(tris + (size_t)sl * 3 + 1);
      const float4 c = __ldg(tris + (size_t)sl * 3 + 2);
      float4* r = o.cw_tris + (size_t)pos * 3;
      r[0] = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, 0.0f);
      r[1] = make_float4(c.x - a.x, c.y - a.y, c.z - a.z, 0.0f);
      r[2] = a;  // v0 and the prim bits
      ++pos;
    } else {
      if (sp + 2 > (int)kFatLeaf + 1) {
        raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        return pos;
      }
      const uint32_t y = cur & kIndexMask;
      stack[sp++] = __ldg(node_meta + (size_t)y * 4 + 2);
      stack[sp++] = __ldg(node_meta + (size_t)y * 4 + 1);
    }
  }
  return pos;
}

// _power_of_two_scale_exponent (compressed_bounds_bvh.mojo:43-53): the
// smallest 2^(e - 127) with 255 * 2^(e - 127) >= extent, e in [1, 254]
__device__ __forceinline__ uint32_t cw_exponent(float extent) {
  if (extent <= 0.0f) return 127u;
  const uint32_t bits = __float_as_uint(extent / 255.0f);
  uint32_t e = (bits >> 23) & 0xFFu;
  if (bits & 0x007FFFFFu) e += 1u;
  return e < 1u ? 1u : (e > 254u ? 254u : e);
}

__device__ __forceinline__ int cw_clamp255(float f) { return f >= 0.0f ? (f <= 255.0f ? (int)f : 255) : 0; }

// _quantize_lower / _quantize_upper (:61-76).  (value - start) / scale is
// computed as (value - start) * 2^(127 - e): the reciprocal of a power of two
// is exact (2^-127 as a subnormal for e = 254), so both round the same exact
// value once.
__device__ __forceinline__ float cw_inv_scale(uint32_t e) {
  return e < 254u ? __uint_as_float((254u - e) << 23) : __uint_as_float(0x00400000u);
}

__device__ __forceinline__ uint32_t cw_qlo(float value, float start, float scale, float inv) {
  int q = cw_clamp255(floorf((value - start) * inv));
  if (__fmaf_rn((float)q, scale, start) > value && q > 0) q -= 1;
  return (uint32_t)q;
}

__device__ __forceinline__ uint32_t cw_qhi(float value, float start, float scale, float inv) {
  int q = cw_clamp255(ceilf((value - start) * inv));
  if (__fmaf_rn((float)q, scale, start) < value && q < 255) q += 1;
  return (uint32_t)q;
}

// _encode_cwbvh8_node (:84-325) from the eight lanes' boxes and metas
// (internal data = segment-local child id, leaf count 1..3): node bounds are
// the lanes' minimum / maximum in lane order (fmin / fmax as a < b ? a : b),
// then p, per-axis exponents | imask << 24, child base, triangle base, the
// lane bytes (internal: 001 | slot + 24; leaf: unary count | triangle offset;
// empty: 0) and the 8-bit planes of every lane.
__device__ void write_cw_node(float4* __restrict__ out, const Box (&bx)[8], const uint32_t (&meta)[8],
                              uint32_t tri_base) {
  float lx = FLT_MAX, ly = FLT_MAX, lz = FLT_MAX, hx = -FLT_MAX, hy = -FLT_MAX, hz = -FLT_MAX;
  uint32_t child_base = 0, n_int = 0, imask = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if (meta[j] == kEmpty) continue;
    lx = lx < bx[j].mn.x ? lx : bx[j].mn.x;
    ly = ly < bx[j].mn.y ? ly : bx[j].mn.y;
    lz = lz < bx[j].mn.z ? lz : bx[j].mn.z;
    hx = hx > bx[j].mx.x ? hx : bx[j].mx.x;
    hy = hy > bx[j].mx.y ? hy : bx[j].mx.y;
    hz = hz > bx[j].mx.z ? hz : bx[j].mx.z;
    if ((meta[j] >> kCountShift) == 0) {
      if (n_int == 0) child_base = meta[j] & kDataMask;
      ++n_int;
      imask |= 1u << j;
    }
  }
  uint32_t ex = cw_exponent(hx - lx), ey = cw_exponent(hy - ly), ez = cw_exponent(hz - lz);
  if (__fmaf_rn(255.0f, __uint_as_float(ex << 23), lx) < hx && ex < 254u) ++ex;
  if (__fmaf_rn(255.0f, __uint_as_float(ey << 23), ly) < hy && ey < 254u) ++ey;
  if (__fmaf_rn(255.0f, __uint_as_float(ez << 23), lz) < hz && ez < 254u) ++ez;
  const float sx = __uint_as_float(ex << 23), sy = __uint_as_float(ey << 23), sz = __uint_as_float(ez << 23);
  const float ix = cw_inv_scale(ex), iy = cw_inv_scale(ey), iz = cw_inv_scale(ez);
  uint32_t m[2] = {0u, 0u}, q[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) q[k] = 0u;
  uint32_t leaf_off = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int g = j >> 2, sh = (j & 3) * 8;
    if (meta[j] == kEmpty) continue;
    const uint32_t count = meta[j] >> kCountShift;
    uint32_t byte;
    if (count == 0) {
      byte = 0x20u | (24u + (uint32_t)j);
    } else {
      byte = (((1u << count) - 1u) << 5) | leaf_off;
      leaf_off += count;
    }
    m[g] |= byte << sh;
    q[0 + g] |= cw_qlo(bx[j].mn.x, lx, sx, ix) << sh;
    q[2 + g] |= cw_qlo(bx[j].mn.y, ly, sy, iy) << sh;
    q[4 + g] |= cw_qlo(bx[j].mn.z, lz, sz, iz) << sh;
    q[6 + g] |= cw_qhi(bx[j].mx.x, lx, sx, ix) << sh;
    q[8 + g] |= cw_qhi(bx[j].mx.y, ly, sy, iy) << sh;
    q[10 + g] |= cw_qhi(bx[j].mx.z, lz, sz, iz) << sh;
  }
  out[0] = make_float4(lx, ly, lz, __uint_as_float(ex | (ey << 8) | (ez << 16) | (imask << 24)));
  out[1] = make_float4(__uint_as_float(child_base), __uint_as_float(tri_base), __uint_as_float(m[0]),
                       __uint_as_float(m[1]));
  out[2] = make_float4(__uint_as_float(q[0]), __uint_as_float(q[1]), __uint_as_float(q[2]), __uint_as_float(q[3]));
  out[3] = make_float4(__uint_as_float(q[4]), __uint_as_float(q[5]), __uint_as_float(q[6]), __uint_as_float(q[7]));
  out[4] = make_float4(__uint_as_float(q[8]), __uint_as_float(q[9]), __uint_as_float(q[10]), __uint_as_float(q[11]));
}

// octant slots (spatial_slots, wide_collapse.mojo:457-521): perm[slot] =
// candidate placed in that lane (-1 = empty).  Repeatedly the unassigned
// candidate and free slot of lowest cost (centroid(candidate) -
// centroid(parent)) . s(slot), s(slot) = (bit 2 ? -1 : 1, bit 1 ? -1 : 1,
// bit 0 ? -1 : 1), are paired; candidates, then slots, are scanned in
// ascending order and the first minimum below FLT_MAX is kept; with none
// (NaN boxes) the first unassigned candidate takes the first free slot.
__device__ void octant_slots(const Box& parent, const uint32_t* __restrict__ cands, int nc,
                             const float* __restrict__ leaf_bounds, const uint32_t* __restrict__ leaf_ids,
                             const float* __restrict__ node_bounds, int (&perm)[8]) {
  const f3 pc = (parent.mn + parent.mx) * 0.5f;
  f3 d[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    perm[k] = -1;
    if (k < nc) {
      const Box b = ref_bounds(cands[k], leaf_bounds, leaf_ids, node_bounds);
      d[k] = (b.mn + b.mx) * 0.5f - pc;
    }
  }
  // Each candidate's cheapest free slot (lowest slot on ties; -1 when no
  // cost is below FLT_MAX).  The cheapest candidate (lowest index on ties)
  // then takes its slot, and only the candidates that wanted that slot look
  // again -- the same pairs, in the same order, as a full rescan.
  auto cost = [&](int k, int sl) {
    return (((sl & 4) ? -d[k].x : d[k].x) + ((sl & 2) ? -d[k].y : d[k].y)) + ((sl & 1) ? -d[k].z : d[k].z);
  };
  float bc_cost[8];
  int bc_slot[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    bc_cost[k] = FLT_MAX;
    bc_slot[k] = -1;
    if (k < nc) {
#pragma unroll
      for (int sl = 0; sl < 8; ++sl) {
        const float c = cost(k, sl);
        if (c < bc_cost[k]) {
          bc_cost[k] = c;
          bc_slot[k] = sl;
        }
      }
    }
  }
  uint32_t assigned = 0, occupied = 0;
  for (int it = 0; it < nc; ++it) {
    float best = FLT_MAX;
    int bc = -1, bs = -1;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < nc && !(assigned >> k & 1u) && bc_slot[k] >= 0 && bc_cost[k] < best) {
        best = bc_cost[k];
        bc = k;
        bs = bc_slot[k];
      }
    }
    if (bc < 0) {
      bc = __ffs(~assigned) - 1;
      bs = __ffs(~occupied) - 1;
    }
    assigned |= 1u << bc;
    occupied |= 1u << bs;
#pragma unroll
    for (int sl = 0; sl < 8; ++sl)
      if (sl == bs) perm[sl] = bc;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k < nc && !(assigned >> k & 1u) && bc_slot[k] == bs) {
        bc_cost[k] = FLT_MAX;
        bc_slot[k] = -1;
#pragma unroll
        for (int sl = 0; sl < 8; ++sl) {
          if (occupied >> sl & 1u) continue;
          const float c = cost(k, sl);
          if (c < bc_cost[k]) {
            bc_cost[k] = c;
            bc_slot[k] = sl;
          }
        }
      }
    }
  }
}

template <int W>
__device__ __forceinline__ void store_lane(float* node, int lane, const Box& b, uint32_t meta) {
  node[0 * W + lane] = b.mn.x;
  node[1 * W + lane] = b.mn.y;
  node[2 * W + lane] = b.mn.z;
  node[3 * W + lane] = b.mx.x;
  node[4 * W + lane] = b.mx.y;
  node[5 * W + lane] = b.mx.z;
  node[6 * W + lane] = __uint_as_float(meta);
}

__device__ __forceinline__ Box empty_box() {
  Box b;
  b.mn = mk(FLT_MAX, FLT_MAX, FLT_MAX);
  b.mx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  return b;
}

// CW = the CWBVH8 build (W = 8, octant slots, compressed nodes and triangle
// records instead of wide nodes and leaf blocks)
template <int W, bool CW>
__global__ void __launch_bounds__(kBlock) assign_kernel(uint32_t n_seg, const uint32_t* __restrict__ node_meta,
                                                        const uint32_t* __restrict__ node_leaf_counts,
                                                        const float* __restrict__ leaf_bounds,
                                                        const uint32_t* __restrict__ leaf_ids,
                                                        const float* __restrict__ node_bounds,
                                                        const float4* __restrict__ tris,
                                                        const uint32_t* __restrict__ seg_offsets,
                                                        const uint32_t* __restrict__ node_offsets,
                                                        const uint32_t* __restrict__ leaf_offsets, uint32_t cap,
                                                        uint32_t max_leaf, Work wk, Out o) {
  static_assert(!CW || W == 8, "CWBVH8 nodes are 8 wide");
  // node and leaf-block totals never exceed the triangle count; more means
  // the binary tree is corrupt
  uint32_t total = node_offsets[n_seg];
  if (total > cap || leaf_offsets[n_seg] > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
    return;
  }
  for (;;) {
    // take the next queue slots, one atomic per converged group of lanes
    const unsigned active = __activemask();
    const int lane = (int)(threadIdx.x & 31u), leader = __ffs(active) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(wk.head, (uint32_t)__popc(active));
    base = __shfl_sync(active, base, leader);
    const uint32_t slot = base + (uint32_t)__popc(active & ((1u << lane) - 1u));
    if (slot >= total) break;
    uint32_t qv = ld_acquire_gpu(wk.queue + slot);
    if (qv == 0) {
      const uint64_t t0 = global_timer_ns();
      while ((qv = ld_acquire_gpu(wk.queue + slot)) == 0) {
        if (global_timer_ns() - t0 > kWaitNs) {
          raise_status(wk.status, BAJO_STATUS_WIDE_TIMEOUT);
          return;
        }
      }
    }
    const uint32_t I = qv - 1u;
    if (I >= total) {
      raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
      continue;
    }
    const uint32_t x = wk.task_ref[I], B = wk.task_leaf[I], s = wk.task_seg[I], D = wk.task_desc[I];
    const uint32_t T = CW ? wk.task_tri[I] : 0u;
    const uint32_t nb = node_offsets[s], lb = leaf_offsets[s];
    const uint32_t t_seg = CW ? seg_offsets[s] : 0u;
    float* node = CW ? nullptr : o.nodes + (size_t)I * kFields * W;
    Box lane_box[W];
    uint32_t lane_meta[W];
    const uint32_t xc = ref_count(x, node_leaf_counts);
    if (terminal(x, xc, max_leaf)) {  // a segment of at most max_leaf triangles: one node, one leaf block
      if (B >= cap) {
        raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
        continue;
      }
      if constexpr (CW) write_cw_tris(x, T, cap, node_meta, tris, o, wk.status);
      else write_leaf_block<W>(x, B, node_meta, leaf_ids, tris, o, wk.status);
#pragma unroll
      for (int j = 0; j < W; ++j) {
        lane_box[j] = j == 0 ? ref_bounds(x, leaf_bounds, leaf_ids, node_bounds) : empty_box();
        lane_meta[j] = j == 0 ? pack_meta(B - lb, xc) : kEmpty;
      }
    } else {
      const uint32_t xi = x & kIndexMask;
      const uint32_t info = wk.cinfo[xi];
      const int nc = (int)(info & 0xFF);
      const uint32_t mask = info >> 8;
      const uint32_t* cands = wk.cands + (size_t)xi * W;
      int perm[W];
      if constexpr (CW) {
        octant_slots(ref_bounds(x, leaf_bounds, leaf_ids, node_bounds), cands, nc, leaf_bounds, leaf_ids,
                     node_bounds, reinterpret_cast<int(&)[8]>(perm));
      } else {
#pragma unroll
        for (int j = 0; j < W; ++j) perm[j] = j < nc ? j : -1;
      }
      const uint32_t n_leaf = __popc(mask & ((1u << nc) - 1u)), n_int = (uint32_t)nc - n_leaf;
      uint32_t own_tris = 0;
      if constexpr (CW) {
        for (int k = 0; k < nc; ++k)
          if (mask & (1u << k)) own_tris += ref_count(cands[k], node_leaf_counts);
      }
      // first the children's tasks, so the next level starts while this
      // node writes its leaf payloads
      uint32_t own = B, child = D, desc = D + n_int, child_leaf = B + n_leaf, child_t = T + own_tris;
      uint32_t qs = n_int ? atomicAdd(wk.tail, n_int) : 0u;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const int k = perm[j];
        if (k < 0) {
          lane_meta[j] = kEmpty;
          continue;
        }
        const uint32_t c = cands[k];
        const uint32_t cnt = ref_count(c, node_leaf_counts);
        if (mask & (1u << k)) {
          lane_meta[j] = pack_meta(own - lb, cnt);
          ++own;
        } else {
          const uint32_t ci = c & kIndexMask;
          lane_meta[j] = pack_meta(child - nb, 0);
          if (child < total && desc <= total && qs < total) {
            wk.task_ref[child] = c;
            wk.task_leaf[child] = child_leaf;
            wk.task_seg[child] = s;
            wk.task_desc[child] = desc;
            if constexpr (CW) wk.task_tri[child] = child_t;
            st_release_gpu(wk.queue + qs, child + 1u);
            ++qs;
          } else {
            raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
          }
          ++child;
          desc += wk.nw[ci] - 1u;
          child_leaf += wk.nl[ci];
          child_t += cnt;
        }
      }
      // then the lane boxes and the leaf payloads
      uint32_t own_t = T;
      own = B;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const int k = perm[j];
        if (k < 0) {
          lane_box[j] = empty_box();
          continue;
        }
        const uint32_t c = cands[k];
        lane_box[j] = ref_bounds(c, leaf_bounds, leaf_ids, node_bounds);
        if (!(mask & (1u << k))) continue;
        if (own >= cap) {
          raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
          lane_meta[j] = kEmpty;
          continue;
        }
        if constexpr (CW) own_t = write_cw_tris(c, own_t, cap, node_meta, tris, o, wk.status);
        else write_leaf_block<W>(c, own, node_meta, leaf_ids, tris, o, wk.status);
        ++own;
      }
    }
    if constexpr (CW) {
      if constexpr (W == 8) write_cw_node(o.cw_nodes + (size_t)I * 5, lane_box, lane_meta, T - t_seg);
    } else {
#pragma unroll
      for (int j = 0; j < W; ++j) store_lane<W>(node, j, lane_box[j], lane_meta[j]);
    }
  }
}

// ---------------------------------------------------------------------------
// traversal kernels (single tree: segment 0)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_hit(const trav::Hit& h, const float4* __restrict__ tris, uint32_t i,
                                          float* __restrict__ hits8, float* __restrict__ out_t,
                                          uint32_t* __restrict__ out_prim) {
  if (hits8) {
    f3 n = mk(0.0f, 0.0f, 0.0f);
    if (h.leaf != kEmpty) {
      const float4 a = __ldg(tris + (size_t)h.leaf * 3 + 0);
      const float4 b = __ldg(tris + (size_t)h.leaf * 3 + 1);
      const float4 c = __ldg(tris + (size_t)h.leaf * 3 + 2);
      const f3 v0 = mk(a.x, a.y, a.z);
      n = normalize(cross(mk(b.x, b.y, b.z) - v0, mk(c.x, c.y, c.z) - v0));
    }
    float4* o = reinterpret_cast<float4*>(hits8 + (size_t)i * 8);
    o[0] = make_float4(h.u, h.v, __uint_as_float(h.prim), __uint_as_float(kEmpty));
    o[1] = make_float4(n.x, n.y, n.z, h.t);
  }
  if (out_t) out_t[i] = h.t;
  if (out_prim) out_prim[i] = h.prim;
}

template <int W, int MODE>
__global__ void __launch_bounds__(trav::kTraceBlock) wide_rays_kernel(const float* __restrict__ rays, uint32_t n,
                                                                      View v, float* __restrict__ hits8,
                                                                      float* __restrict__ out_t,
                                                                      uint32_t* __restrict__ out_prim,
                                                                      uint32_t* __restrict__ status) {
  const uint32_t i = blockIdx.x * trav::kTraceBlock + threadIdx.x;
  if (i >= n) return;
  const f3 o = mk(rays[i], rays[(size_t)n + i], rays[2 * (size_t)n + i]);
  const float tmin = rays[3 * (size_t)n + i];
  const f3 d = mk(rays[4 * (size_t)n + i], rays[5 * (size_t)n + i], rays[6 * (size_t)n + i]);
  const float tmax = rays[7 * (size_t)n + i];
  const trav::Hit h = trace_wide<W, MODE>(trav::make_ray(o, d, tmin, tmax), v, status);
  store_hit(h, v.bvh2_tris, i, hits8, out_t, out_prim);
}

template <int W, int MODE, bool STATS>
__global__ void __launch_bounds__(trav::kTraceBlock) wide_camera_kernel(
    const float* __restrict__ cams, uint32_t n, uint32_t width, uint32_t height, float inv_h, View v,
    float* __restrict__ hits8, float* __restrict__ out_t, uint32_t* __restrict__ out_prim,
    uint32_t* __restrict__ status, uint32_t* __restrict__ stats) {
  uint32_t i;  // every warp an 8 x 4 pixel tile (trav::tile_ray)
  if (!trav::tile_ray((uint64_t)blockIdx.x * trav::kTraceBlock + threadIdx.x, n, width, height, i)) return;
  const uint32_t ppv = width * height;
  const uint32_t view = i / ppv, local = i - view * ppv;
  const float* c = cams + (size_t)view * 20;
  const uint32_t px = local % width, py = local / width;
  const float sx = (2.0f * ((float)px + 0.5f) - (float)width) * inv_h;
  const float sy = 1.0f - 2.0f * ((float)py + 0.5f) * inv_h;
  const float fs = __ldg(c + 12);
  const f3 fwd = mk(__ldg(c + 3), __ldg(c + 4), __ldg(c + 5));
  const f3 right = mk(__ldg(c + 6), __ldg(c + 7), __ldg(c + 8));
  const f3 up = mk(__ldg(c + 9), __ldg(c + 10), __ldg(c + 11));
  const f3 dir = normalize((fwd + right * (sx * fs)) + up * (sy * fs));
  uint32_t st[trav::kStatWords] = {0, 0, 0, 0, 0};
  const trav::Hit h =
      trace_wide<W, MODE, STATS>(trav::make_ray(mk(__ldg(c + 0), __ldg(c + 1), __ldg(c + 2)), dir, 0.0f, FLT_MAX),
                                 v, status, st);
  store_hit(h, v.bvh2_tris, i, hits8, out_t, out_prim);
  if constexpr (STATS) {
#pragma unroll
    for (int k = 0; k < trav::kStatWords; ++k) stats[(size_t)i * trav::kStatWords + k] = st[k];
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Plan {
  size_t flags, queue, cands, cinfo, nw, nl, task_ref, task_leaf, task_seg, task_desc, task_tri, area,
      leaf_offsets, zero_bytes, total;
};

// cw_segments > 0: the CWBVH8 build, which also keeps the per-segment leaf
// offsets ([S+1]) in the workspace
inline Plan make_plan(uint32_t n, uint32_t width, uint32_t cw_segments = 0) {
  Plan p;
  const size_t cap = std::max<uint32_t>(n, 1);
  size_t o = 256;  // status word
  p.flags = o;
  o = a256(o + cap * 4);
  p.queue = o;
  o = a256(o + cap * 4);
  p.zero_bytes = o;  // status, queue counters, flags and queue are cleared per build
  p.cands = o;
  o = a256(o + cap * width * 4);
  p.cinfo = o;
  o = a256(o + cap * 4);
  p.nw = o;
  o = a256(o + cap * 4);
  p.nl = o;
  o = a256(o + cap * 4);
  p.task_ref = o;
  o = a256(o + cap * 4);
  p.task_leaf = o;
  o = a256(o + cap * 4);
  p.task_seg = o;
  o = a256(o + cap * 4);
  p.task_desc = o;
  o = a256(o + cap * 4);
  p.task_tri = o;
  if (cw_segments) o = a256(o + cap * 4);
  p.area = o;
  o = a256(o + cap * 4);
  p.leaf_offsets = o;
  if (cw_segments) o = a256(o + ((size_t)cw_segments + 1) * 4);
  p.total = o;
  return p;
}

template <int W, bool CW>
cudaError_t build(const BajoLbvh* b, uint32_t* node_offsets, uint32_t* leaf_offsets, const Out& o,
                  unsigned char* ws, const Plan& p, uint32_t max_leaf, cudaStream_t st) {
  Work wk;
  wk.status = (uint32_t*)ws;
  wk.flags = (uint32_t*)(ws + p.flags);
  wk.queue = (uint32_t*)(ws + p.queue);
  wk.head = wk.status + 1;
  wk.tail = wk.status + 2;
  wk.cands = (uint32_t*)(ws + p.cands);
  wk.cinfo = (uint32_t*)(ws + p.cinfo);
  wk.nw = (uint32_t*)(ws + p.nw);
  wk.nl = (uint32_t*)(ws + p.nl);
  wk.task_ref = (uint32_t*)(ws + p.task_ref);
  wk.task_leaf = (uint32_t*)(ws + p.task_leaf);
  wk.task_seg = (uint32_t*)(ws + p.task_seg);
  wk.task_desc = (uint32_t*)(ws + p.task_desc);
  wk.task_tri = (uint32_t*)(ws + p.task_tri);
  wk.area = (float*)(ws + p.area);
  cudaError_t e = cudaMemsetAsync(ws, 0, p.zero_bytes, st);
  if (e != cudaSuccess) return e;
  const uint32_t n = b->n_leaves;
  if (n > 0) {
    count_kernel<W><<<(n + kBlock - 1) / kBlock, kBlock, 0, st>>>(n, b->node_meta, b->leaf_parent,
                                                                 b->node_leaf_counts, b->leaf_bounds, b->leaf_ids,
                                                                 b->node_bounds, max_leaf, wk);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  offsets_kernel<<<1, 1024, 0, st>>>(b->n_segments, b->seg_offsets, b->roots, b->node_leaf_counts, max_leaf, wk,
                                     std::max<uint32_t>(n, 1), node_offsets, leaf_offsets);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  // every block resident, so a task's producer always runs
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, assign_kernel<W, CW>, kBlock, 0)) != cudaSuccess)
    return e;
  uint32_t grid = (uint32_t)std::max(1, per_sm) * (uint32_t)sm_count();
  const uint32_t need = (n + kBlock - 1) / kBlock;
  if (grid > need) grid = need;
  assign_kernel<W, CW><<<grid, kBlock, 0, st>>>(b->n_segments, b->node_meta, b->node_leaf_counts, b->leaf_bounds,
                                               b->leaf_ids, b->node_bounds,
                                               reinterpret_cast<const float4*>(b->leaf_tris), b->seg_offsets,
                                               node_offsets, leaf_offsets, std::max<uint32_t>(n, 1), max_leaf, wk, o);
  return cudaGetLastError();
}

template <int W, int MODE>
cudaError_t launch_rays(const View& v, const float* rays, uint32_t n, float* hits8, float* t, uint32_t* prim,
                        uint32_t* status, cudaStream_t st) {
  wide_rays_kernel<W, MODE><<<(n + trav::kTraceBlock - 1) / trav::kTraceBlock, trav::kTraceBlock, 0, st>>>(
      rays, n, v, hits8, t, prim, status);
  return cudaGetLastError();
}

template <int W, int MODE, bool STATS>
cudaError_t launch_camera(const View& v, const float* cams, uint32_t n, uint32_t w, uint32_t h, float* hits8,
                          float* t, uint32_t* prim, uint32_t* status, uint32_t* stats, cudaStream_t st) {
  const uint32_t grid = (uint32_t)((trav::camera_threads(n, w, h) + trav::kTraceBlock - 1) / trav::kTraceBlock);
  wide_camera_kernel<W, MODE, STATS><<<grid, trav::kTraceBlock, 0, st>>>(cams, n, w, h, 1.0f / (float)h, v, hits8, t,
                                                                        prim, status, stats);
  return cudaGetLastError();
}

// the tree of segment 0; n_nodes from the host-side count
bool make_view(const BajoWideBvh* w, uint32_t n_nodes, uint32_t n_blocks, View& v) {
  if (!w || !w->nodes || !w->leaf_tris || !w->leaf_sorted || !w->bvh2_leaf_tris) return false;
  v.nodes = w->nodes;
  v.leaf_tris = w->leaf_tris;
  v.leaf_sorted = w->leaf_sorted;
  v.bvh2_tris = reinterpret_cast<const float4*>(w->bvh2_leaf_tris);
  v.n_nodes = n_nodes;
  v.n_blocks = n_blocks;
  return true;
}

}  // namespace wide
}  // namespace bajo

extern "C" {

int32_t bajo_wide_sizes(uint32_t n_tris, uint32_t n_segments, uint32_t width, BajoWideSizes* s) {
  if (!s || n_segments == 0 || (width != 4 && width != 8)) return BAJO_ERR_INVALID_ARGUMENT;
  const size_t cap = std::max<uint32_t>(n_tris, 1);
  s->node_offsets = (size_t)(n_segments + 1) * 4;
  s->leaf_offsets = (size_t)(n_segments + 1) * 4;
  s->nodes = cap * bajo::wide::kFields * width * 4;
  s->leaf_indices = cap * width * 4;
  s->leaf_tris = cap * bajo::wide::kLeafStride * width * 4;
  s->leaf_sorted = cap * width * 4;
  s->workspace = bajo::wide::make_plan(n_tris, width).total;
  return BAJO_OK;
}

int32_t bajo_wide_build(const BajoLbvh* b, BajoWideBvh* out, void* ws, size_t ws_bytes, void* stream) {
  using namespace bajo::wide;
  if (!b || !out || !ws || (out->width != 4 && out->width != 8) || b->n_segments == 0) return BAJO_ERR_INVALID_ARGUMENT;
  if (!out->node_offsets || !out->leaf_offsets || !out->nodes || !out->leaf_indices || !out->leaf_tris ||
      !out->leaf_sorted || !b->seg_offsets || !b->roots || !b->node_meta || !b->node_leaf_counts || !b->leaf_parent ||
      !b->leaf_bounds || !b->leaf_ids || !b->node_bounds || !b->leaf_tris)
    return BAJO_ERR_INVALID_ARGUMENT;
  const Plan p = make_plan(b->n_leaves, out->width);
  if (ws_bytes < p.total) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  out->n_segments = b->n_segments;
  out->bvh2_leaf_tris = b->leaf_tris;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t max_leaf = out->max_leaf ? out->max_leaf : kFatLeaf;
  if (max_leaf > kFatLeaf) return BAJO_ERR_INVALID_ARGUMENT;
  const Out o{out->nodes, out->leaf_indices, out->leaf_tris, out->leaf_sorted, nullptr, nullptr};
  unsigned char* w = (unsigned char*)ws;
  const cudaError_t e = out->width == 4
                            ? build<4, false>(b, out->node_offsets, out->leaf_offsets, o, w, p, max_leaf, st)
                            : build<8, false>(b, out->node_offsets, out->leaf_offsets, o, w, p, max_leaf, st);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_cwbvh8_sizes(uint32_t n_tris, uint32_t n_segments, BajoCwbvh8Sizes* s) {
  if (!s || n_segments == 0) return BAJO_ERR_INVALID_ARGUMENT;
  const size_t cap = std::max<uint32_t>(n_tris, 1);
  s->node_offsets = (size_t)(n_segments + 1) * 4;
  s->nodes = cap * BAJO_CWBVH8_NODE_WORDS * 4;
  s->triangles = cap * BAJO_CWBVH8_TRI_WORDS * 4;
  s->workspace = bajo::wide::make_plan(n_tris, 8, n_segments).total;
  return BAJO_OK;
}

int32_t bajo_cwbvh8_build(const BajoLbvh* b, BajoCwbvh8* out, void* ws, size_t ws_bytes, void* stream) {
  using namespace bajo::wide;
  if (!b || !out || !ws || b->n_segments == 0 || !out->node_offsets || !out->nodes || !out->triangles ||
      !b->seg_offsets || !b->roots || !b->node_meta || !b->node_leaf_counts || !b->leaf_parent || !b->leaf_bounds ||
      !b->leaf_ids || !b->node_bounds || !b->leaf_tris)
    return BAJO_ERR_INVALID_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(out->nodes) | reinterpret_cast<uintptr_t>(out->triangles)) & 15u)
    return BAJO_ERR_INVALID_ARGUMENT;
  const Plan p = make_plan(b->n_leaves, 8, b->n_segments);
  if (ws_bytes < p.total) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  out->n_segments = b->n_segments;
  out->n_tris = b->n_leaves;
  unsigned char* w = (unsigned char*)ws;
  const Out o{nullptr, nullptr, nullptr, nullptr, reinterpret_cast<float4*>(out->nodes),
              reinterpret_cast<float4*>(out->triangles)};
  const cudaError_t e = build<8, true>(b, out->node_offsets, (uint32_t*)(w + p.leaf_offsets), o, w, p,
                                       BAJO_CWBVH8_MAX_LEAF, (cudaStream_t)stream);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_cwbvh8_count(const BajoCwbvh8* c, void* stream, uint32_t* n_nodes) {
  if (!c || !c->node_offsets || !n_nodes || c->n_segments == 0) return BAJO_ERR_INVALID_ARGUMENT;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return BAJO_ERR_CUDA;
  if (cudaMemcpy(n_nodes, c->node_offsets + c->n_segments, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return BAJO_ERR_CUDA;
  return BAJO_OK;
}

int32_t bajo_wide_counts(const BajoWideBvh* w, void* stream, uint32_t* n_nodes, uint32_t* n_leaf_blocks) {
  if (!w || !w->node_offsets || !w->leaf_offsets || !n_nodes || !n_leaf_blocks || w->n_segments == 0)
    return BAJO_ERR_INVALID_ARGUMENT;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return BAJO_ERR_CUDA;
  if (cudaMemcpy(n_nodes, w->node_offsets + w->n_segments, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(n_leaf_blocks, w->leaf_offsets + w->n_segments, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return BAJO_ERR_CUDA;
  return BAJO_OK;
}

int32_t bajo_trace_wide_rays(const BajoWideBvh* w, uint32_t n_nodes, uint32_t n_leaf_blocks, const float* d_rays,
                             uint32_t n,
                             int32_t tri_mode, float* d_hits8, float* d_t, uint32_t* d_prim, uint32_t* d_status,
                             void* stream) {
  using namespace bajo::wide;
  View v;
  if (!make_view(w, n_nodes, n_leaf_blocks, v) || (n && !d_rays) || (tri_mode != BAJO_TRI_MT && tri_mode != BAJO_TRI_WATERTIGHT) ||
      !d_status)
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (w->width == 4)
    e = tri_mode == BAJO_TRI_MT ? launch_rays<4, BAJO_TRI_MT>(v, d_rays, n, d_hits8, d_t, d_prim, d_status, st)
                                : launch_rays<4, BAJO_TRI_WATERTIGHT>(v, d_rays, n, d_hits8, d_t, d_prim, d_status, st);
  else
    e = tri_mode == BAJO_TRI_MT ? launch_rays<8, BAJO_TRI_MT>(v, d_rays, n, d_hits8, d_t, d_prim, d_status, st)
                                : launch_rays<8, BAJO_TRI_WATERTIGHT>(v, d_rays, n, d_hits8, d_t, d_prim, d_status, st);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_wide_camera(const BajoWideBvh* w, uint32_t n_nodes, uint32_t n_leaf_blocks,
                               const float* d_cameras, uint32_t n,
                               uint32_t width, uint32_t height, int32_t tri_mode, float* d_hits8, float* d_t,
                               uint32_t* d_prim, uint32_t* d_status, uint32_t* d_stats, void* stream) {
  using namespace bajo::wide;
  View v;
  if (!make_view(w, n_nodes, n_leaf_blocks, v) || !d_cameras || width == 0 || height == 0 ||
      (tri_mode != BAJO_TRI_MT && tri_mode != BAJO_TRI_WATERTIGHT) || !d_status)
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  const bool mt = tri_mode == BAJO_TRI_MT;
#define BAJO_WIDE_CAM(WW, MM, SS) launch_camera<WW, MM, SS>(v, d_cameras, n, width, height, d_hits8, d_t, d_prim, d_status, d_stats, st)
  if (w->width == 4) {
    if (d_stats) e = mt ? BAJO_WIDE_CAM(4, BAJO_TRI_MT, true) : BAJO_WIDE_CAM(4, BAJO_TRI_WATERTIGHT, true);
    else e = mt ? BAJO_WIDE_CAM(4, BAJO_TRI_MT, false) : BAJO_WIDE_CAM(4, BAJO_TRI_WATERTIGHT, false);
  } else {
    if (d_stats) e = mt ? BAJO_WIDE_CAM(8, BAJO_TRI_MT, true) : BAJO_WIDE_CAM(8, BAJO_TRI_WATERTIGHT, true);
    else e = mt ? BAJO_WIDE_CAM(8, BAJO_TRI_MT, false) : BAJO_WIDE_CAM(8, BAJO_TRI_WATERTIGHT, false);
  }
#undef BAJO_WIDE_CAM
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

}  // extern "C"
