// lbvh.cu -- sm_100a LBVH build: triangle bounds, per-segment bounds, Morton
// keys, onesweep sort, Karras topology, atomic-flag refit.  Restates
// bajo/bvh/gpu/builder/lbvh.mojo (GPU driver) and binary_layout.mojo with the
// reference's buffer layouts; see include/bajo_b200.h for the boundary.
#include <atomic>
#include <chrono>
#include <mutex>

#include "onesweep.cuh"

namespace bajo {

int sm_count();

namespace {

constexpr int kBlock = 256;
// hierarchy CTA: sorted leaves per CTA (also the unit that decides which
// splits meet in global memory, section 3).  512 measured faster than 1,024:
// the local climbs spread over twice the SMs for one more global level.
constexpr int kRefitBlock = 512;
// Builds of up to this many triangles emit the hierarchy bottom-up in the
// refit pass (section 3); larger ones run the top-down topology kernel and
// the refit separately (section 4), which keeps more warps resident per SM.
// Measured crossover on B200: 2^17 triangles (101 vs 108 us; 2^18: 144 vs
// 141 us).
constexpr uint32_t kMergedMaxLeaves = 1u << 17;

// Per segment, 12 ordered words: [min bounds xyz, max bounds xyz,
// min centroid xyz, max centroid xyz].  Minima are stored complemented so
// that every slot is an atomicMax that starts from 0.
__device__ __forceinline__ uint32_t enc_min(float f) { return ~float_to_ordered(f); }
__device__ __forceinline__ uint32_t enc_max(float f) { return float_to_ordered(f); }
__device__ __forceinline__ float dec_min(uint32_t u) { return u == 0 ? FLT_MAX : ordered_to_float(~u); }
__device__ __forceinline__ float dec_max(uint32_t u) { return u == 0 ? -FLT_MAX : ordered_to_float(u); }

// ---------------------------------------------------------------------------
// 1. triangle bounds + per-segment root / centroid bounds
//    (compute_triangle_bounds_kernel, triangle_bvh.mojo:680;
//     compute/reduce_segment_bounds_partials, binary_layout.mojo:128-205)
//    One pass: coalesced vertex loads staged in shared memory, warp max
//    reductions on order-preserving integer images, one set of atomics per
//    block.  Block 0 also writes the internal-node offsets
//    (_internal_segment_offsets, binary_layout.mojo:219).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) bounds_kernel(const float* __restrict__ verts, uint32_t n,
                                                        const uint32_t* __restrict__ seg_offsets, uint32_t n_seg,
                                                        uint32_t* __restrict__ internal_offsets,
                                                        float* __restrict__ leaf_bounds,
                                                        uint32_t* __restrict__ seg_ord) {
  __shared__ float s_v[kBlock * 9];
  __shared__ uint32_t s_red[kBlock / 32][12];
  __shared__ uint32_t s_scan[8];
  const uint32_t tid = threadIdx.x;

  if (blockIdx.x == 0) {
    // internal offsets: exclusive scan of max(count - 1, 0)
    uint32_t carry = 0;
    for (uint32_t base = 0; base < n_seg; base += kBlock) {
      uint32_t s = base + tid, c = 0;
      if (s < n_seg) {
        uint32_t cnt = seg_offsets[s + 1] - seg_offsets[s];
        c = cnt > 0 ? cnt - 1 : 0;
      }
      uint32_t ex = onesweep::scan256_exclusive<kBlock>(c, s_scan);
      if (s < n_seg) internal_offsets[s] = carry + ex;
      if (tid == kBlock - 1) s_scan[0] = ex + c;  // chunk total
      __syncthreads();
      carry += s_scan[0];
      __syncthreads();
    }
    if (tid == 0) internal_offsets[n_seg] = carry;
  }

  const uint32_t base = blockIdx.x * kBlock;
  if (base >= n) return;
  const uint32_t cnt = min((uint32_t)kBlock, n - base);
  const float* src = verts + (size_t)base * 9;
  for (uint32_t k = tid; k < cnt * 9; k += kBlock) s_v[k] = src[k];
  __syncthreads();

  const bool live = tid < cnt;
  f3 mn = mk(FLT_MAX, FLT_MAX, FLT_MAX), mx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  if (live) {
    const float* v = s_v + tid * 9;
    f3 a = mk(v[0], v[1], v[2]), b = mk(v[3], v[4], v[5]), c = mk(v[6], v[7], v[8]);
    mn = vmin(vmin(a, b), c);
    mx = vmax(vmax(a, b), c);
  }
  __syncthreads();
  // stage the 6-float bounds and write them coalesced
  if (live) {
    float* o = s_v + tid * 6;
    o[0] = mn.x; o[1] = mn.y; o[2] = mn.z; o[3] = mx.x; o[4] = mx.y; o[5] = mx.z;
  }
  __syncthreads();
  float* dst = leaf_bounds + (size_t)base * 6;
  for (uint32_t k = tid; k < cnt * 6; k += kBlock) dst[k] = s_v[k];

  // centroid = (min + max) * 0.5   (core/aabb.mojo:53)
  f3 c = (mn + mx) * 0.5f;
  uint32_t w[12] = {0};
  if (live) {
    w[0] = enc_min(mn.x); w[1] = enc_min(mn.y); w[2] = enc_min(mn.z);
    w[3] = enc_max(mx.x); w[4] = enc_max(mx.y); w[5] = enc_max(mx.z);
    w[6] = enc_min(c.x); w[7] = enc_min(c.y); w[8] = enc_min(c.z);
    w[9] = enc_max(c.x); w[10] = enc_max(c.y); w[11] = enc_max(c.z);
  }
  uint32_t seg_first = 0, seg_last = 0, seg = 0;
  if (n_seg > 1) {
    seg_first = segment_for_item(seg_offsets, n_seg + 1, base);
    seg_last = segment_for_item(seg_offsets, n_seg + 1, base + cnt - 1);
    seg = live ? segment_for_item(seg_offsets, n_seg + 1, base + tid) : seg_last;
  }
  if (seg_first == seg_last) {
    const uint32_t warp = tid >> 5, lane = tid & 31;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      uint32_t r = __reduce_max_sync(0xFFFFFFFFu, w[k]);
      if (lane == 0) s_red[warp][k] = r;
    }
    __syncthreads();
    if (tid < 12) {
      uint32_t r = 0;
#pragma unroll
      for (int q = 0; q < kBlock / 32; ++q) r = max(r, s_red[q][tid]);
      if (r) atomicMax(&seg_ord[(size_t)seg_first * 12 + tid], r);
    }
  } else if (live) {
#pragma unroll
    for (int k = 0; k < 12; ++k) atomicMax(&seg_ord[(size_t)seg * 12 + k], w[k]);
  }
}

// shared histogram copies per pass of the Morton kernel
__host__ __device__ constexpr uint32_t morton_hist_copies(uint32_t passes, uint32_t digit_bits) {
  return digit_bits > 8 ? 2u : (passes <= 4 ? 8u : 4u);
}

// ---------------------------------------------------------------------------
// 2. Morton keys + every live digit histogram of the sort
//    (compute_bounds_morton_codes_kernel, lbvh.mojo:30-62, fused with
//     global_histogram, onesweep.mojo:31).  Grid-strided so that each block
//    flushes its shared histograms once.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) morton_kernel(const float* __restrict__ leaf_bounds, uint32_t n,
                                                        const uint32_t* __restrict__ seg_offsets, uint32_t n_seg,
                                                        const uint32_t* __restrict__ seg_ord,
                                                        float* __restrict__ seg_bounds_out,
                                                        uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                                        uint32_t passes, uint32_t end_bit, uint32_t digit_bits,
                                                        uint32_t* __restrict__ ghist,
                                                        uint32_t* __restrict__ node_flags) {
  extern __shared__ uint32_t s_hist[];  // passes * copies * radix
  const uint32_t radix = 1u << digit_bits, copies = morton_hist_copies(passes, digit_bits);
  const uint32_t words = passes * copies * radix;
  for (uint32_t i = threadIdx.x; i < words; i += kBlock) s_hist[i] = 0;
  if (blockIdx.x == 0) {
    for (uint32_t k = threadIdx.x; k < n_seg * 12; k += kBlock) {
      uint32_t u = seg_ord[k];
      uint32_t f = k % 12;
      bool is_min = (f < 3) || (f >= 6 && f < 9);
      seg_bounds_out[k] = is_min ? dec_min(u) : dec_max(u);
    }
  }
  __syncthreads();
  const uint32_t copy = (threadIdx.x >> 5) % copies;
  // single-segment fast path keeps the centroid frame in registers
  uint32_t cur_seg = 0xFFFFFFFFu;
  f3 cmin = mk(0, 0, 0), inv = mk(0, 0, 0);
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    uint32_t seg = n_seg > 1 ? segment_for_item(seg_offsets, n_seg + 1, i) : 0;
    if (seg != cur_seg) {
      const uint32_t* o = seg_ord + (size_t)seg * 12;
      cmin = mk(dec_min(__ldg(o + 6)), dec_min(__ldg(o + 7)), dec_min(__ldg(o + 8)));
      f3 cmax = mk(dec_max(__ldg(o + 9)), dec_max(__ldg(o + 10)), dec_max(__ldg(o + 11)));
      f3 ext = cmax - cmin;
      inv = mk(safe_inv1(ext.x), safe_inv1(ext.y), safe_inv1(ext.z));
      cur_seg = seg;
    }
    const float2* b = reinterpret_cast<const float2*>(leaf_bounds + (size_t)i * 6);
    float2 b0 = b[0], b1 = b[1], b2 = b[2];
    f3 mn = mk(b0.x, b0.y, b1.x), mx = mk(b1.y, b2.x, b2.y);
    f3 c = (mn + mx) * 0.5f;
    f3 d = c - cmin;
    uint32_t code = morton3(d.x * inv.x, d.y * inv.y, d.z * inv.z);
    uint64_t key = ((uint64_t)seg << 32) | code;
    keys[i] = key;
    vals[i] = i;
    node_flags[i] = 0;  // arrival counters of the hierarchy kernel
    for (uint32_t p = 0; p < passes; ++p) {
      uint32_t sh = digit_bits * p;
      uint32_t bits = min(digit_bits, end_bit - sh);
      uint32_t dg = (uint32_t)(key >> sh) & ((1u << bits) - 1u);
      atomicAdd(&s_hist[(p * copies + copy) * radix + dg], 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < passes * radix; i += kBlock) {
    uint32_t p = i >> digit_bits, dg = i & (radix - 1u), s = 0;
    for (uint32_t c = 0; c < copies; ++c) s += s_hist[(p * copies + c) * radix + dg];
    if (s) atomicAdd(&ghist[i], s);
  }
}

// ---------------------------------------------------------------------------
// 3. Karras hierarchy, refit and sorted triangle records in one bottom-up pass
//    (builds of up to kMergedMaxLeaves triangles)
//    (init_segmented_lbvh_roots_kernel, lbvh.mojo:235;
//     build_lbvh_topology_kernel, lbvh.mojo:257-329;
//     refit_lbvh_bounds_from_leaves_kernel, lbvh.mojo:116-161;
//     pack_segmented_triangle_leaf_lanes_kernel, triangle_bvh.mojo:81).
//
//    The reference finds every internal node's range and split top-down
//    (one thread per node, two binary searches over the codes), then refits
//    the boxes bottom-up.  Here one thread per sorted leaf climbs and builds
//    the same binary radix tree bottom-up (Apetrei, "Fast and simple
//    agglomerative LBVH construction", 2014): a node [f, l] is the left child
//    of its parent iff delta(l, l+1) > delta(f-1, f), so its parent splits at
//    l (left child) or f-1 (right child).  The two children of a split meet
//    there; the second to arrive knows the parent's whole range and continues
//    upwards with the union of the two boxes.  Karras numbering: a
//    non-root internal node is indexed by its last position when it is a left
//    child and by its first when it is a right child; the root is 0.  The
//    arrays are bit-identical to the top-down construction (same ranges,
//    splits, numbering, boxes).
//
//    A CTA owns kRefitBlock consecutive sorted leaves.  Splits whose
//    sibling starts inside the CTA meet in shared memory (arrival counter,
//    child boxes, far range ends and their deltas in shared slots); a climb
//    step there touches shared memory only, and once every climb of the CTA
//    has ended, one pass writes the records of all parents built in it (a
//    slot holds everything its parent's record needs).  A split
//    whose sibling lies (partly) outside meets in global memory after the
//    CTA's local climbs are done: node_flags of the split counts the
//    arrivals (acquire), the first arrival publishes its subtree (already
//    written to the node arrays) with a release flag bit, and passes its far
//    end's delta in the counter word; the second reads the sibling's box
//    from its node record or triangle record.  node_flags ends at 2 for
//    every internal node.  (An acq_rel arrival add, which would spare the
//    flag bit, was measured slower on B200: its release makes the second
//    arrival, the one that climbs on, wait for its own stores first.)
// ---------------------------------------------------------------------------
constexpr uint32_t kArrive = 1u;
constexpr uint32_t kLeafArrive = 0x10u;   // the arrival is a leaf
constexpr uint32_t kBoxReady = 0x100u;    // first arrival published
constexpr uint64_t kRefitWaitNs = 200000000ull;

// lbvh.mojo:221-232 + core/morton.mojo:22: clz64 of the (code, local index)
// keys of two positions of one segment.
__device__ __forceinline__ int delta_codes(uint32_t ci, uint32_t li, uint32_t cj, uint32_t lj) {
  const uint64_t x = (((uint64_t)ci << 32) | li) ^ (((uint64_t)cj << 32) | lj);
  return x ? __clzll((long long)x) : 64;
}

struct SegInfo {
  uint32_t lb, len, ib;
};

// Writes internal node k = the parent [F, L] (global positions) split at
// gamma, and its children's parent links.
__device__ __forceinline__ void write_parent(const SegInfo& g, uint32_t k, uint32_t F, uint32_t L, uint32_t gamma,
                                             f3 lmn, f3 lmx, f3 rmn, f3 rmx, uint32_t* __restrict__ node_meta,
                                             uint32_t* __restrict__ node_leaf_counts,
                                             uint32_t* __restrict__ leaf_parent, float* __restrict__ node_bounds) {
  const uint32_t lg = gamma - g.lb;
  const bool left_leaf = gamma == F, right_leaf = gamma + 1 == L;
  const uint32_t left = left_leaf ? (kLeafFlag | gamma) : g.ib + lg;
  const uint32_t right = right_leaf ? (kLeafFlag | (gamma + 1)) : g.ib + lg + 1;
  uint32_t* m = node_meta + (size_t)k * 4;
  if (F == g.lb && L == g.lb + g.len - 1) m[0] = kSentinel;  // the root
  m[1] = left;
  *reinterpret_cast<uint2*>(m + 2) = make_uint2(right, L);  // right child, fence = leaf_begin + last
  node_leaf_counts[k] = L - F + 1;
  float4* b = reinterpret_cast<float4*>(node_bounds + (size_t)k * 12);  // 16-byte aligned (checked by the build)
  b[0] = make_float4(lmn.x, lmn.y, lmn.z, lmx.x);
  b[1] = make_float4(lmx.y, lmx.z, rmn.x, rmn.y);
  b[2] = make_float4(rmn.z, rmx.x, rmx.y, rmx.z);
  if (left_leaf) leaf_parent[gamma] = k;
  else node_meta[(size_t)(g.ib + lg) * 4] = k;
  if (right_leaf) leaf_parent[gamma + 1] = k;
  else node_meta[(size_t)(g.ib + lg + 1) * 4] = k;
}

// Writes the parent split at gamma whose children [F, gamma] and [gamma + 1,
// L] met in a shared-memory slot: dL, dR are the deltas at F and after L,
// lb / rb the children's boxes (min xyz, max xyz).  node_flags may be null.
__device__ __forceinline__ void write_slot_parent(const SegInfo& g, uint32_t gamma, uint32_t F, uint32_t L, int dL,
                                                  int dR, const float* lb, const float* rb,
                                                  uint32_t* __restrict__ node_meta,
                                                  uint32_t* __restrict__ node_leaf_counts,
                                                  uint32_t* __restrict__ leaf_parent, float* __restrict__ node_bounds,
                                                  uint32_t* __restrict__ node_flags) {
  const bool root = F == g.lb && L == g.lb + g.len - 1;
  const uint32_t k = g.ib + (root ? 0u : (dR > dL ? L - g.lb : F - g.lb));
  write_parent(g, k, F, L, gamma, mk(lb[0], lb[1], lb[2]), mk(lb[3], lb[4], lb[5]), mk(rb[0], rb[1], rb[2]),
               mk(rb[3], rb[4], rb[5]), node_meta, node_leaf_counts, leaf_parent, node_bounds);
  if (node_flags) node_flags[g.ib + (gamma - g.lb)] = 2u;  // (the one-launch build sets them all up front)
}

__device__ __forceinline__ void tri_box(const float4* __restrict__ rec, f3& mn, f3& mx) {
  const float4 a = __ldcg(rec + 0), b = __ldcg(rec + 1), c = __ldcg(rec + 2);
  const f3 va = mk(a.x, a.y, a.z), vb = mk(b.x, b.y, b.z), vc = mk(c.x, c.y, c.z);
  mn = vmin(vmin(va, vb), vc);
  mx = vmax(vmax(va, vb), vc);
}

// A subtree on its way up: sorted leaves [f, l] (global positions), the
// deltas at its two ends (-1 at a segment end), its box, and whether it is a
// single leaf.
struct Climb {
  uint32_t f, l;
  int dl, dr;
  f3 mn, mx;
  bool leaf;
};

// The shared-memory phase of one CTA's share: sorted leaves [blockIdx.x *
// kRefitBlock, +kRefitBlock) with kRefitBlock threads and kRefitBlock * 72 + 8
// bytes of shared memory.  Returns true for a thread whose subtree c still
// has to meet its sibling outside the CTA.  The subtrees returned by all
// threads of a CTA are the largest ones inside its tile, so they cover the
// tile's leaves once each, in disjoint ranges.
__device__ __forceinline__ bool hierarchy_local(
    const float* __restrict__ verts, const uint32_t* __restrict__ leaf_ids, const uint32_t* __restrict__ codes,
    uint32_t n, const uint32_t* __restrict__ seg_offsets, uint32_t n_seg, const uint32_t* __restrict__ internal_offsets,
    uint32_t* __restrict__ node_meta, uint32_t* __restrict__ node_leaf_counts, uint32_t* __restrict__ leaf_parent,
    float* __restrict__ node_bounds, uint32_t* __restrict__ node_flags, float* __restrict__ leaf_tris,
    uint32_t* __restrict__ roots, uint32_t* __restrict__ status, unsigned char* __restrict__ hier_smem,
    const uint32_t* bound2, SegInfo& g, Climb& out) {
  float(*s_box)[2][6] = reinterpret_cast<float(*)[2][6]>(hier_smem);                      // [B][side]
  uint32_t(*s_far)[2] = reinterpret_cast<uint32_t(*)[2]>(hier_smem + kRefitBlock * 48);   // far end
  int(*s_dfar)[2] = reinterpret_cast<int(*)[2]>(hier_smem + kRefitBlock * 56);            // its delta
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(hier_smem + kRefitBlock * 64);            // arrivals
  uint32_t* s_code = reinterpret_cast<uint32_t*>(hier_smem + kRefitBlock * 68);           // [B + 2]
  const uint32_t tid = threadIdx.x;
  const uint32_t c0 = blockIdx.x * kRefitBlock;  // first sorted leaf of this CTA
  const uint32_t s = c0 + tid;

  // roots (init_segmented_lbvh_roots_kernel)
  for (uint32_t i = blockIdx.x * kRefitBlock + tid; i < n_seg; i += gridDim.x * kRefitBlock) {
    const uint32_t lb = seg_offsets[i], le = seg_offsets[i + 1];
    if (le == lb) roots[i] = kSentinel;
    else if (le - lb == 1) {
      roots[i] = kLeafFlag | lb;
      leaf_parent[lb] = kSentinel;
    } else roots[i] = internal_offsets[i];
  }

  s_cnt[tid] = 0;
  s_code[tid + 1] = s < n ? codes[s] : 0u;
  // the sorted codes just outside the tile (bound2: given by the caller)
  if (tid == 0) s_code[0] = (c0 > 0 && c0 - 1 < n) ? (bound2 ? bound2[0] : codes[c0 - 1]) : 0u;
  if (tid == kRefitBlock - 1) s_code[kRefitBlock + 1] = (s + 1 < n) ? (bound2 ? bound2[1] : codes[s + 1]) : 0u;

  g = SegInfo{0, 0, 0};
  bool active = s < n;
  f3 mn, mx;
  if (active) {
    const uint32_t seg = n_seg > 1 ? segment_for_item(seg_offsets, n_seg + 1, s) : 0;
    g.lb = seg_offsets[seg];
    g.len = seg_offsets[seg + 1] - g.lb;
    g.ib = internal_offsets[seg];
    const uint32_t item = leaf_ids[s];
    if (item >= n) {  // only after a failed sort
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      active = false;
    } else {
      const float* v = verts + (size_t)item * 9;
      const f3 a = mk(__ldg(v + 0), __ldg(v + 1), __ldg(v + 2));
      const f3 b = mk(__ldg(v + 3), __ldg(v + 4), __ldg(v + 5));
      const f3 c = mk(__ldg(v + 6), __ldg(v + 7), __ldg(v + 8));
      float4* rec = reinterpret_cast<float4*>(leaf_tris + (size_t)s * 12);
      rec[0] = make_float4(a.x, a.y, a.z, __uint_as_float(item - g.lb));
      rec[1] = make_float4(b.x, b.y, b.z, 0.0f);
      rec[2] = make_float4(c.x, c.y, c.z, 0.0f);
      mn = vmin(vmin(a, b), c);
      mx = vmax(vmax(a, b), c);
      if (g.len < 2) active = false;  // a one-leaf segment: the leaf is the root
    }
  }
  __syncthreads();  // codes staged

  // the climbing subtree [f, l] and the deltas at its two ends
  uint32_t f = s, l = s;
  bool leaf = true;
  int dl = -1, dr = -1;
  if (active) {
    const uint32_t li = s - g.lb;
    if (li > 0) dl = delta_codes(s_code[tid], li - 1, s_code[tid + 1], li);
    if (li + 1 < g.len) dr = delta_codes(s_code[tid + 1], li, s_code[tid + 2], li + 1);
  }
  // phase 1: splits whose sibling starts inside this CTA, in shared memory
  bool global = false;
  int pending = -1;  // shared slot where this subtree arrived first
  for (int depth = 0; active; ++depth) {
    if (depth > 128) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      active = false;
      break;
    }
    const bool is_left = dr > dl;
    const uint32_t gamma = is_left ? l : f - 1;
    if (is_left ? (l + 1 >= c0 + kRefitBlock) : (f < c0 + 1)) {
      global = true;
      break;
    }
    const uint32_t slot = gamma - c0, side = is_left ? 0 : 1;
    float* mine = s_box[slot][side];
    mine[0] = mn.x; mine[1] = mn.y; mine[2] = mn.z; mine[3] = mx.x; mine[4] = mx.y; mine[5] = mx.z;
    s_far[slot][side] = is_left ? f : l;
    s_dfar[slot][side] = is_left ? dl : dr;
    fence_acq_rel_cta();
    if (atomicAdd(&s_cnt[slot], 1u) == 0) {
      pending = (int)slot;
      break;
    }
    fence_acq_rel_cta();
    const float* sib = s_box[slot][side ^ 1];
    const f3 smn = mk(sib[0], sib[1], sib[2]), smx = mk(sib[3], sib[4], sib[5]);
    const uint32_t sfar = s_far[slot][side ^ 1];
    const int sd = s_dfar[slot][side ^ 1];
    // the parent [F, L] is complete in the slot (both children's boxes, far
    // ends and deltas); its record is written after the climbs
    const uint32_t F = is_left ? f : sfar, L = is_left ? sfar : l;
    mn = vmin(mn, smn);
    mx = vmax(mx, smx);
    f = F;
    l = L;
    dl = is_left ? dl : sd;
    dr = is_left ? sd : dr;
    leaf = false;
    if (F == g.lb && L == g.lb + g.len - 1) active = false;  // the root
  }
  __syncthreads();  // every local climb of this CTA has ended
  // the records of the parents built here: slot tid is the split at this
  // thread's leaf s, inside its segment g
  if (tid + 1 < kRefitBlock && s_cnt[tid] == 2u)
    write_slot_parent(g, s, s_far[tid][0], s_far[tid][1], s_dfar[tid][0], s_dfar[tid][1], s_box[tid][0],
                      s_box[tid][1], node_meta, node_leaf_counts, leaf_parent, node_bounds, node_flags);
  if (pending >= 0 && s_cnt[pending] == 1) global = true;  // the sibling comes from outside
  out = Climb{f, l, dl, dr, mn, mx, leaf};
  __syncthreads();  // the records are written (a climber that goes on fences before its release)
  return global;
}

// The climb of subtree c through the splits whose children were built by
// different CTAs, in global memory (the protocol described above), up to the
// segment's root or to the first split where c arrives first.  flags: the
// arrival counters, zero before the build (node_flags, or a scratch array).
__device__ __forceinline__ void climb_global(const SegInfo& g, Climb c, uint32_t* __restrict__ node_meta,
                                             uint32_t* __restrict__ node_leaf_counts,
                                             uint32_t* __restrict__ leaf_parent, float* __restrict__ node_bounds,
                                             uint32_t* __restrict__ flags, const float* __restrict__ leaf_tris,
                                             uint32_t* __restrict__ status) {
  uint32_t f = c.f, l = c.l;
  int dl = c.dl, dr = c.dr;
  f3 mn = c.mn, mx = c.mx;
  bool leaf = c.leaf;
  for (int depth = 0;; ++depth) {
    if (depth > 128) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      return;
    }
    const bool is_left = dr > dl;
    const uint32_t gamma = is_left ? l : f - 1;
    const uint32_t lg = gamma - g.lb;
    uint32_t* flag = flags + g.ib + lg;
    const int dfar = is_left ? dl : dr;
    const uint32_t inc = kArrive | (leaf ? kLeafArrive : 0u) | ((uint32_t)(dfar + 1) << 16);
    const uint32_t old = atomic_add_acquire_gpu(flag, inc);
    if ((old & 0xFu) == 0) {  // first: publish the subtree written above
      red_add_release_gpu(flag, kBoxReady);
      return;
    }
    // the first arrival's release may still be in flight
    if (!(old & kBoxReady) && !wait_bits_acquire(flag, kBoxReady, kRefitWaitNs)) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      return;
    }
    const bool sib_leaf = (old & kLeafArrive) != 0;
    const int sd = (int)((old >> 16) & 0x7Fu) - 1;
    f3 smn, smx;
    uint32_t sfar;
    if (is_left) {  // sibling = right child, starts at gamma + 1
      if (sib_leaf) {
        sfar = gamma + 1;
        tri_box(reinterpret_cast<const float4*>(leaf_tris) + (size_t)(gamma + 1) * 3, smn, smx);
      } else {
        const uint32_t ks = g.ib + lg + 1;
        sfar = __ldcg(node_meta + (size_t)ks * 4 + 3);
        const float4* nb = reinterpret_cast<const float4*>(node_bounds) + (size_t)ks * 3;
        const float4 b0 = __ldcg(nb + 0), b1 = __ldcg(nb + 1), b2 = __ldcg(nb + 2);
        smn = vmin(mk(b0.x, b0.y, b0.z), mk(b1.z, b1.w, b2.x));
        smx = vmax(mk(b0.w, b1.x, b1.y), mk(b2.y, b2.z, b2.w));
      }
    } else {  // sibling = left child, ends at gamma
      if (sib_leaf) {
        sfar = gamma;
        tri_box(reinterpret_cast<const float4*>(leaf_tris) + (size_t)gamma * 3, smn, smx);
      } else {
        const uint32_t ks = g.ib + lg;
        sfar = gamma + 1 - __ldcg(node_leaf_counts + ks);
        const float4* nb = reinterpret_cast<const float4*>(node_bounds) + (size_t)ks * 3;
        const float4 b0 = __ldcg(nb + 0), b1 = __ldcg(nb + 1), b2 = __ldcg(nb + 2);
        smn = vmin(mk(b0.x, b0.y, b0.z), mk(b1.z, b1.w, b2.x));
        smx = vmax(mk(b0.w, b1.x, b1.y), mk(b2.y, b2.z, b2.w));
      }
    }
    *flag = 2u;
    const uint32_t F = is_left ? f : sfar, L = is_left ? sfar : l;
    if (F > L || L >= g.lb + g.len || F < g.lb) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      return;
    }
    const int dL = is_left ? dl : sd, dR = is_left ? sd : dr;
    const bool root = F == g.lb && L == g.lb + g.len - 1;
    const uint32_t k = g.ib + (root ? 0u : (dR > dL ? L - g.lb : F - g.lb));
    if (is_left) write_parent(g, k, F, L, gamma, mn, mx, smn, smx, node_meta, node_leaf_counts, leaf_parent, node_bounds);
    else write_parent(g, k, F, L, gamma, smn, smx, mn, mx, node_meta, node_leaf_counts, leaf_parent, node_bounds);
    if (root) return;
    mn = vmin(mn, smn);
    mx = vmax(mx, smx);
    f = F;
    l = L;
    dl = dL;
    dr = dR;
    leaf = false;
  }
}

// One CTA's share of the hierarchy, both phases.
__device__ __forceinline__ void hierarchy_tile(
    const float* __restrict__ verts, const uint32_t* __restrict__ leaf_ids, const uint32_t* __restrict__ codes,
    uint32_t n, const uint32_t* __restrict__ seg_offsets, uint32_t n_seg, const uint32_t* __restrict__ internal_offsets,
    uint32_t* __restrict__ node_meta, uint32_t* __restrict__ node_leaf_counts, uint32_t* __restrict__ leaf_parent,
    float* __restrict__ node_bounds, uint32_t* __restrict__ node_flags, float* __restrict__ leaf_tris,
    uint32_t* __restrict__ roots, uint32_t* __restrict__ status, unsigned char* __restrict__ hier_smem) {
  SegInfo g;
  Climb c;
  if (hierarchy_local(verts, leaf_ids, codes, n, seg_offsets, n_seg, internal_offsets, node_meta, node_leaf_counts,
                      leaf_parent, node_bounds, node_flags, leaf_tris, roots, status, hier_smem, nullptr, g, c)) {
    __threadfence();  // the records the CTA wrote, before the release that publishes the subtree
    climb_global(g, c, node_meta, node_leaf_counts, leaf_parent, node_bounds, node_flags, leaf_tris, status);
  }
}

__global__ void __launch_bounds__(kRefitBlock) hierarchy_kernel(
    const float* __restrict__ verts, const uint32_t* __restrict__ leaf_ids, const uint32_t* __restrict__ codes,
    uint32_t n, const uint32_t* __restrict__ seg_offsets, uint32_t n_seg, const uint32_t* __restrict__ internal_offsets,
    uint32_t* __restrict__ node_meta, uint32_t* __restrict__ node_leaf_counts, uint32_t* __restrict__ leaf_parent,
    float* __restrict__ node_bounds, uint32_t* __restrict__ node_flags, float* __restrict__ leaf_tris,
    uint32_t* __restrict__ roots, uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char hier_smem[];
  hierarchy_tile(verts, leaf_ids, codes, n, seg_offsets, n_seg, internal_offsets, node_meta, node_leaf_counts,
                 leaf_parent, node_bounds, node_flags, leaf_tris, roots, status, hier_smem);
}

// ---------------------------------------------------------------------------
// 4. Large builds: Karras topology top-down, then the refit
//    (init_segmented_lbvh_roots_kernel, lbvh.mojo:235;
//    build_lbvh_topology_kernel, lbvh.mojo:257-329).
// ---------------------------------------------------------------------------
// lbvh.mojo:221-232 + core/morton.mojo:22: clz64 of the (code, local index)
// keys, -1 outside the segment.
__device__ __forceinline__ int delta(const uint32_t* __restrict__ codes, int64_t len, int64_t i, int64_t j) {
  if (j < 0 || j >= len) return -1;
  uint64_t a = ((uint64_t)__ldg(codes + i) << 32) | (uint32_t)i;
  uint64_t b = ((uint64_t)__ldg(codes + j) << 32) | (uint32_t)j;
  uint64_t x = a ^ b;
  return x ? __clzll((long long)x) : 64;
}

__global__ void __launch_bounds__(kBlock) topology_kernel(const uint32_t* __restrict__ codes_all,
                                                          const uint32_t* __restrict__ seg_offsets, uint32_t n_seg,
                                                          const uint32_t* __restrict__ internal_offsets,
                                                          uint32_t n, uint32_t* __restrict__ node_meta,
                                                          uint32_t* __restrict__ leaf_parent,
                                                          uint32_t* __restrict__ node_leaf_counts,
                                                          uint32_t* __restrict__ node_flags,
                                                          float* __restrict__ node_bounds,
                                                          uint32_t* __restrict__ roots) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n_seg) {
    uint32_t lb = seg_offsets[i], le = seg_offsets[i + 1];
    if (le == lb) roots[i] = kSentinel;
    else if (le - lb == 1) {
      roots[i] = kLeafFlag | lb;
      leaf_parent[lb] = kSentinel;
    } else roots[i] = internal_offsets[i];
  }
  const uint32_t total = internal_offsets[n_seg];
  if (i >= total) return;
  const uint32_t seg = n_seg > 1 ? segment_for_item(internal_offsets, n_seg + 1, i) : 0;
  const uint32_t ib = internal_offsets[seg], lb = seg_offsets[seg];
  const int64_t len = (int64_t)seg_offsets[seg + 1] - lb;
  const uint32_t* codes = codes_all + lb;
  const int64_t li = (int64_t)i - ib;

  // _lbvh_find_range, lbvh.mojo:164-191
  int d_next = delta(codes, len, li, li + 1);
  int d_prev = delta(codes, len, li, li - 1);
  int64_t d = (d_next < d_prev) ? -1 : 1;
  int delta_min = delta(codes, len, li, li - d);
  int64_t lmax = 2;
  while (delta(codes, len, li, li + lmax * d) > delta_min) {
    lmax <<= 1;
    if (lmax > len * 2) break;
  }
  int64_t l = 0;
  for (int64_t t = lmax >> 1; t > 0; t >>= 1)
    if (delta(codes, len, li, li + (l + t) * d) > delta_min) l += t;
  int64_t j = li + l * d;
  int64_t first = li < j ? li : j, last = li < j ? j : li;

  // _lbvh_find_split, lbvh.mojo:194-218
  int node_prefix = delta(codes, len, first, last);
  int64_t split = first, step = last - first;
  while (step > 1) {
    step = (step + 1) >> 1;
    int64_t ns = split + step;
    if (ns < last && delta(codes, len, first, ns) > node_prefix) split = ns;
  }

  node_leaf_counts[i] = (uint32_t)(last - first + 1);
  node_flags[i] = 0;
  // nodes whose children meet in global memory during the refit start from
  // the invalid box (AABB.invalid, bajo/core/aabb.mojo:28), which lets the
  // refit read a sibling's slot before its arrival atomic returns
  if ((lb + (uint32_t)first) / kRefitBlock != (lb + (uint32_t)last) / kRefitBlock) {
    float4* nb4 = reinterpret_cast<float4*>(node_bounds + (size_t)i * 12);
    const float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX);
    const float4 mid = make_float4(-FLT_MAX, -FLT_MAX, FLT_MAX, FLT_MAX);
    const float4 hi = make_float4(FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX);
    nb4[0] = lo;
    nb4[1] = mid;
    nb4[2] = hi;
  }
  if (first == 0 && last == len - 1) node_meta[(size_t)i * 4 + 0] = kSentinel;
  uint32_t left = ib + (uint32_t)split, right = ib + (uint32_t)split + 1;
  if (split == first) {
    left = kLeafFlag | (lb + (uint32_t)split);
    leaf_parent[lb + split] = i;
  } else {
    node_meta[(size_t)(ib + split) * 4 + 0] = i;
  }
  if (split + 1 == last) {
    right = kLeafFlag | (lb + (uint32_t)split + 1);
    leaf_parent[lb + split + 1] = i;
  } else {
    node_meta[(size_t)(ib + split + 1) * 4 + 0] = i;
  }
  node_meta[(size_t)i * 4 + 1] = left;
  node_meta[(size_t)i * 4 + 2] = right;
  node_meta[(size_t)i * 4 + 3] = lb + (uint32_t)last;
}

// ---------------------------------------------------------------------------
// 4b. refit + sorted triangle records
//    (refit_lbvh_bounds_from_leaves_kernel, lbvh.mojo:116-161;
//     pack_segmented_triangle_leaf_lanes_kernel, triangle_bvh.mojo:81).
//    One thread per sorted leaf climbs towards the root; the first arrival at
//    a node stops, the second merges both child boxes and continues.
//    A CTA owns kRefitBlock consecutive sorted leaves.  Nodes whose leaf
//    range lies inside the CTA's leaves (almost all of them: a Karras node's
//    range is contiguous) meet in shared memory: arrival counter and the
//    first arrival's box in shared slots, no L2 round trip.  Only the nodes
//    whose range crosses a CTA boundary meet in global memory, with the
//    arrival counted first (acquire) and the first arrival then publishing
//    its box with a release flag bit (kBoxReady), so the arrival that
//    continues does not wait for its own box stores.  The continuing arrival
//    reads the sibling's slot while its atomic is in flight (the slot starts
//    invalid, so a complete box is a final one): one L2 round trip per level
//    instead of two in the common case.  node_flags ends at 2 for every
//    internal node either way.  512 leaves per CTA measured faster than
//    1,024 (16M-triangle build 15% faster): more CTAs resident per SM.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kRefitBlock) refit_kernel(const float* __restrict__ verts,
                                                            const uint32_t* __restrict__ leaf_ids, uint32_t n,
                                                            const uint32_t* __restrict__ seg_offsets, uint32_t n_seg,
                                                            const uint32_t* __restrict__ internal_offsets,
                                                            const uint32_t* __restrict__ node_meta,
                                                            const uint32_t* __restrict__ node_leaf_counts,
                                                            const uint32_t* __restrict__ leaf_parent,
                                                            float* __restrict__ node_bounds,
                                                            uint32_t* __restrict__ node_flags,
                                                            float* __restrict__ leaf_tris, uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char refit_smem[];
  uint4* s_meta = reinterpret_cast<uint4*>(refit_smem);                             // [kRefitBlock]
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(refit_smem + kRefitBlock * 16);     // [kRefitBlock]
  uint32_t* s_flag = reinterpret_cast<uint32_t*>(refit_smem + kRefitBlock * 20);    // [kRefitBlock]
  float(*s_box)[2][6] = reinterpret_cast<float(*)[2][6]>(refit_smem + kRefitBlock * 24);
  s_flag[threadIdx.x] = 0;
  const uint32_t c0 = blockIdx.x * kRefitBlock;  // first sorted leaf of this CTA
  const uint32_t s = c0 + threadIdx.x;
  uint32_t seg = 0, lb = 0, ib = 0;
  if (s < n) {
    if (n_seg > 1) seg = segment_for_item(seg_offsets, n_seg + 1, s);
    lb = seg_offsets[seg];
    ib = internal_offsets[seg];
    // the internal node whose own index sits at this leaf position (one end
    // of every Karras node's range is its index): its record is read from
    // shared memory while the climb stays inside this CTA's leaves
    const uint32_t li = s - lb, len = seg_offsets[seg + 1] - lb;
    if (li + 1 < len) {
      s_meta[threadIdx.x] = *reinterpret_cast<const uint4*>(node_meta + (size_t)(ib + li) * 4);
      s_cnt[threadIdx.x] = node_leaf_counts[ib + li];
    }
  }
  __syncthreads();
  if (s >= n) return;
  const uint32_t item = leaf_ids[s];
  if (item >= n) {  // only after a failed sort
    raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
    return;
  }
  const float* v = verts + (size_t)item * 9;
  f3 a = mk(__ldg(v + 0), __ldg(v + 1), __ldg(v + 2));
  f3 b = mk(__ldg(v + 3), __ldg(v + 4), __ldg(v + 5));
  f3 c = mk(__ldg(v + 6), __ldg(v + 7), __ldg(v + 8));
  const uint32_t prim = item - lb;
  float4* rec = reinterpret_cast<float4*>(leaf_tris + (size_t)s * 12);
  rec[0] = make_float4(a.x, a.y, a.z, __uint_as_float(prim));
  rec[1] = make_float4(b.x, b.y, b.z, 0.0f);
  rec[2] = make_float4(c.x, c.y, c.z, 0.0f);

  f3 mn = vmin(vmin(a, b), c), mx = vmax(vmax(a, b), c);
  uint32_t cur = kLeafFlag | s;
  uint32_t parent = leaf_parent[s];
  // A Karras tree over 64-bit keys is at most 64 levels deep; a longer climb
  // or an out-of-range parent means the topology is corrupt.
  for (int depth = 0; parent != kSentinel; ++depth) {
    if (depth > 128 || parent >= n) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      return;
    }
    const uint32_t pos = lb + (parent - ib);  // leaf position of the parent's own index
    uint4 m;
    uint32_t cnt;
    if (pos >= c0 && pos < c0 + kRefitBlock) {
      m = s_meta[pos - c0];
      cnt = s_cnt[pos - c0];
    } else {
      m = *reinterpret_cast<const uint4*>(node_meta + (size_t)parent * 4);
      cnt = __ldg(node_leaf_counts + parent);
    }
    const bool is_left = m.y == cur;
    if (!is_left && m.z != cur) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      return;
    }
    const uint32_t last = m.w, first = last + 1 - cnt;
    const bool local = first >= c0 && last < c0 + kRefitBlock;
    float* slot = node_bounds + (size_t)parent * 12 + (is_left ? 0 : 6);
    if (local) {
      float2* s2 = reinterpret_cast<float2*>(slot);
      s2[0] = make_float2(mn.x, mn.y);
      s2[1] = make_float2(mn.z, mx.x);
      s2[2] = make_float2(mx.y, mx.z);
    } else {  // read early by the sibling's arrival (below): strong stores
      st_relaxed_gpu_f2(slot + 0, mn.x, mn.y);
      st_relaxed_gpu_f2(slot + 2, mn.z, mx.x);
      st_relaxed_gpu_f2(slot + 4, mx.y, mx.z);
    }
    f3 smn, smx;
    if (local) {
      // both children live in this CTA; one end of a Karras node's range is
      // its own local index, so lb + (parent - ib) - c0 is a unique slot
      const uint32_t k = lb + (parent - ib) - c0;
      float* mine = s_box[k][is_left ? 0 : 1];
      mine[0] = mn.x; mine[1] = mn.y; mine[2] = mn.z; mine[3] = mx.x; mine[4] = mx.y; mine[5] = mx.z;
      fence_acq_rel_cta();
      if (atomicAdd(&s_flag[k], 1u) == 0) return;
      fence_acq_rel_cta();
      const float* sib = s_box[k][is_left ? 1 : 0];
      smn = mk(sib[0], sib[1], sib[2]);
      smx = mk(sib[3], sib[4], sib[5]);
      node_flags[parent] = 2u;
    } else {
      // The sibling's slot is read before the arrival atomic returns, so the
      // continuing arrival usually pays one L2 round trip per level.  The
      // slot is written once per build and starts invalid (topology_kernel),
      // so six values that all differ from the invalid box are final; any
      // invalid value is read again after the handshake.
      const float* sib = node_bounds + (size_t)parent * 12 + (is_left ? 6 : 0);
      const float2 q0 = ld_relaxed_gpu_f2(sib), q1 = ld_relaxed_gpu_f2(sib + 2), q2 = ld_relaxed_gpu_f2(sib + 4);
      const uint32_t old = atomic_add_acquire_gpu(&node_flags[parent], 1u);
      if ((old & 0xFFu) == 0) {  // first: publish the box stored above
        red_add_release_gpu(&node_flags[parent], kBoxReady);
        return;
      }
      smn = mk(q0.x, q0.y, q1.x);
      smx = mk(q1.y, q2.x, q2.y);
      const bool ready = smn.x != FLT_MAX && smn.y != FLT_MAX && smn.z != FLT_MAX && smx.x != -FLT_MAX &&
                         smx.y != -FLT_MAX && smx.z != -FLT_MAX;
      if (ready && !(old & kBoxReady)) {
        // the first arrival's kBoxReady add may still be in flight: cancel
        // it arithmetically so the counter ends at 2 in either order
        atomicSub(&node_flags[parent], kBoxReady);
      } else {
        if (!ready) {
          if (!(old & kBoxReady) && !wait_bits_acquire(&node_flags[parent], kBoxReady, kRefitWaitNs)) {
            raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
            return;
          }
          smn = mk(__ldcg(sib + 0), __ldcg(sib + 1), __ldcg(sib + 2));
          smx = mk(__ldcg(sib + 3), __ldcg(sib + 4), __ldcg(sib + 5));
        }
        node_flags[parent] = 2u;
      }
    }
    mn = vmin(mn, smn);
    mx = vmax(mx, smx);
    cur = parent;
    parent = m.x;
  }
}

// ---------------------------------------------------------------------------
// 5. One-launch build of one scene of up to fused::kMaxLeaves triangles:
//    bounds, Morton keys, the sort and the hierarchy in one cooperative
//    launch.
//
//    At 65,536 triangles every kernel of the per-stage build is latency
//    bound, and its sort is four onesweep passes of about 10 us each.  Here
//    one CTA per kTile keys (= hierarchy_kernel's kRefitBlock sorted leaves)
//    runs the phases, which meet at grid-wide barriers (bounded waits,
//    BAJO_STATUS_GRID_TIMEOUT):
//      A  triangle bounds, root and centroid bounds              -> barrier 1
//      B  Morton codes (kept in registers) and the histogram of the top
//         kBucketBits code bits                                   -> barrier 2
//    Sort, fast path (every bucket holds at most kBucketMax keys, which
//    every CTA reads off the same histogram):
//      S1 each key goes to its bucket's range of a scratch buffer (slot from
//         a per-bucket atomic counter, so the order inside a bucket is
//         arbitrary)                                              -> barrier 3
//      S2 each CTA loads the buckets that cover its tile (and the positions
//         just before and after it) into shared memory and ranks every key
//         inside its bucket by (code, item id).  Item ids are unique, so this
//         is exactly the order of a stable sort by code: the multi-pass LSD
//         sort's output.  No barrier: the CTA goes on with its own tile.
//    Sort, otherwise: every pass's digit histogram                -> barrier 3
//    and LSD radix passes over the 30-bit code (8-bit digits): each tile
//    ranks its keys (stable, in position order) and scatters them to
//    base(digit) + counts of the digit in earlier tiles + rank, counting the
//    next pass's digits per destination tile as it scatters, so a pass needs
//    one barrier                                                  -> barriers 4-7
//      H  hierarchy_local (section 3) over the CTA's sorted leaves; the
//         largest subtrees inside the tile go to the tile's list  -> one barrier
//      T  build_top: the splits between those subtrees, in shared memory of
//         one CTA per kTopCap of them (global memory only between CTAs).
//    Every output array is bit-identical to the per-stage build's.
// ---------------------------------------------------------------------------
namespace fused {
constexpr int kThreads = kRefitBlock;                // the hierarchy phase's CTA
constexpr int kKpt = 1;                              // keys per thread
constexpr uint32_t kTile = kThreads * kKpt;          // keys (and sorted leaves) per CTA
constexpr uint32_t kMaxLeaves = 1u << 17;
constexpr uint32_t kMaxTiles = kMaxLeaves / kTile;  // 256
constexpr int kPasses = 4;                           // LSD digits [0,8) [8,16) [16,24) [24,30)
constexpr int kWarps = kThreads / 32;
constexpr int kBucketBits = 12;                      // buckets: the top 12 of the 30 code bits
constexpr uint32_t kBuckets = 1u << kBucketBits;
constexpr uint32_t kBucketShift = 30 - kBucketBits;
constexpr uint32_t kBucketMax = 256;                 // fast path: no bucket larger than this
constexpr uint32_t kLoadMax = kTile + 2 + 2 * kBucketMax;  // keys a CTA ranks on the fast path, at most
constexpr uint64_t kWaitNs = 200ull * 1000ull * 1000ull;

// Top of the hierarchy: every CTA lists the largest subtrees inside its tile
// (at most kTileTops: a subtree hangs off one of the two paths from the tile's
// end leaves up to their common ancestor, and every node on such a path has a
// longer common key prefix than its parent, at most 64 bits), and one CTA
// per kTopCap of them, in position order, builds the splits between them in
// shared memory.
constexpr uint32_t kTileTops = 136;
constexpr uint32_t kTopCap = 1536;

// Workspace (bytes from the start of the build workspace; word 0 is the
// status word): the launch's epoch flag, the barrier counter and the
// ordered root and centroid bounds (CTA 0 clears the last two, then stores
// the epoch, which every CTA waits for before it first touches them, so no
// clearing launch precedes the build); the LSD digit histograms, bucket
// histogram and fill counters (zeroed by phase A); per-(pass, tile) digit
// counts; two key / item buffers; the tiles' subtree lists (first leaf |
// (delta at it + 1) << 24, and box) and counts; arrival counters of the
// splits between two CTAs' ranges of the top (zeroed by phase A).
struct Layout {
  size_t off_epoch, off_bar, off_seg_ord, off_ghist, off_bhist, off_bfill, off_counts, off_ka, off_va, off_kb, off_vb,
      off_top_fd, off_top_box, off_top_cnt, off_top_flags, total;
};
__host__ __device__ constexpr size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
__host__ __device__ constexpr Layout layout(uint32_t n) {
  Layout l{};
  l.off_epoch = 256;
  l.off_bar = 384;
  l.off_seg_ord = 512;
  l.off_ghist = 768;
  l.off_bhist = a256(l.off_ghist + (size_t)kPasses * 256 * 4);
  l.off_bfill = l.off_bhist + (size_t)kBuckets * 4;
  l.off_counts = a256(l.off_bfill + (size_t)kBuckets * 4);
  l.off_ka = a256(l.off_counts + (size_t)kPasses * kMaxTiles * 256 * 4);
  l.off_va = a256(l.off_ka + (size_t)n * 4);
  l.off_kb = a256(l.off_va + (size_t)n * 4);
  l.off_vb = a256(l.off_kb + (size_t)n * 4);
  const size_t tiles = (n + kTile - 1) / kTile;
  l.off_top_fd = a256(l.off_vb + (size_t)n * 4);
  l.off_top_box = a256(l.off_top_fd + tiles * kTileTops * 4);
  l.off_top_cnt = a256(l.off_top_box + tiles * kTileTops * 24);
  l.off_top_flags = a256(l.off_top_cnt + tiles * 4);
  l.total = a256(l.off_top_flags + (size_t)n * 4);
  return l;
}

// Shared memory, one buffer reused by the phases.
constexpr size_t kSmemVerts = (size_t)kTile * 9 * 4;                                 // phase A
constexpr size_t kSmemFast = (size_t)kBuckets * 4 + 80 * 4 + (size_t)kLoadMax * 8;  // fast sort
constexpr size_t kSmemLsd = (size_t)kWarps * 256 * 4 + 256 * 4 * 5 + (size_t)kPasses * 256 * 4 + 64;
constexpr size_t kSmemHier = (size_t)kRefitBlock * 72 + 8 + 64;                     // phase H + tile marks
// phase T (top of the hierarchy): tile starts, then per subtree its first
// leaf, delta and arrival counter, per split two far ends, deltas and boxes
struct TopSmem {
  size_t tstart, first, delta, cnt, far, dfar, box, edge, total;
};
__host__ __device__ constexpr TopSmem top_smem() {
  TopSmem t{};
  t.tstart = 0;
  t.first = t.tstart + (kMaxTiles + 1) * 4 + 12;
  t.delta = t.first + (kTopCap + 1) * 4;
  t.cnt = (t.delta + kTopCap + 1 + 15) & ~(size_t)15;
  t.far = t.cnt + kTopCap * 4;
  t.dfar = t.far + kTopCap * 4;
  t.box = (t.dfar + kTopCap * 2 + 15) & ~(size_t)15;
  t.edge = t.box + kTopCap * 48;
  t.total = t.edge + 2 * 48;
  return t;
}
constexpr size_t kSmemTop = top_smem().total;
constexpr size_t kSmemMax2 = kSmemFast > kSmemLsd ? kSmemFast : kSmemLsd;
constexpr size_t kSmemMax3 = kSmemHier > kSmemMax2 ? kSmemHier : kSmemMax2;
constexpr size_t kSmemMax4 = kSmemTop > kSmemMax3 ? kSmemTop : kSmemMax3;
constexpr size_t kSmem = ((kSmemVerts > kSmemMax4 ? kSmemVerts : kSmemMax4) + 15) & ~(size_t)15;
static_assert(kSmem <= 100 * 1024, "two CTAs per SM");
static_assert(kTopCap == BAJO_LBVH_TOP_CAP, "header and kernel agree");

// Grid-wide barrier number k (1, 2, ...) of a cooperative launch: every CTA
// adds one to *bar (released) and waits until all of them have, for at most
// kWaitNs.  Returns false when the wait ran out (status bit raised); the CTA
// then leaves the kernel, and the others run out at their next barrier.
__device__ __forceinline__ bool grid_sync(uint32_t* bar, uint32_t k, uint32_t* status, uint32_t* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    red_add_release_gpu(bar, 1u);
    const uint32_t target = k * gridDim.x;
    uint32_t ok = 1;
    if (ld_acquire_gpu(bar) < target) {
      const uint64_t t0 = global_timer_ns();
      while (ld_acquire_gpu(bar) < target) {
        if (global_timer_ns() - t0 > kWaitNs) {
          raise_status(status, BAJO_STATUS_GRID_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    *s_flag = ok;
  }
  __syncthreads();
  return *s_flag != 0;
}

// Waits (one thread, at most kWaitNs) until CTA 0 has published this
// launch's epoch; false, with the status bit raised, when it never came.
__device__ __forceinline__ bool wait_epoch(const uint32_t* flag, uint32_t epoch, uint32_t* status) {
  if (ld_acquire_gpu(flag) == epoch) return true;
  const uint64_t t0 = global_timer_ns();
  while (ld_acquire_gpu(flag) != epoch) {
    if (global_timer_ns() - t0 > kWaitNs) {
      raise_status(status, BAJO_STATUS_GRID_TIMEOUT);
      return false;
    }
  }
  return true;
}

// Exclusive scan over kBuckets entries in shared memory (in place), kThreads
// threads with kBuckets / kThreads consecutive entries each; returns the total
// and the largest entry through *s_res (res[0] total, res[1] max).
__device__ __forceinline__ void scan_buckets(uint32_t* s_b, uint32_t* s_tmp, uint32_t* s_res) {
  constexpr uint32_t kPer = kBuckets / kThreads;
  static_assert(kBuckets % kThreads == 0, "whole runs per thread");
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t v[kPer], sum = 0, mx = 0;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    v[k] = s_b[tid * kPer + k];
    sum += v[k];
    mx = max(mx, v[k]);
  }
  uint32_t inc = onesweep::warp_inclusive_scan(sum);
  mx = __reduce_max_sync(0xFFFFFFFFu, mx);
  if (lane == 31) s_tmp[warp] = inc;
  if (lane == 0) s_tmp[32 + warp] = mx;
  __syncthreads();
  uint32_t before = 0, total = 0, gmax = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    before += (w < (int)warp) ? s_tmp[w] : 0u;
    total += s_tmp[w];
    gmax = max(gmax, s_tmp[32 + w]);
  }
  uint32_t run = before + inc - sum;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    s_b[tid * kPer + k] = run;
    run += v[k];
  }
  if (tid == 0) {
    s_res[0] = total;
    s_res[1] = gmax;
  }
  __syncthreads();
}

// A subtree whose next split lies outside this CTA's range of the list.
struct TopEdge {
  uint32_t a, b;  // list positions (of this CTA's range)
  int dl, dr;
  float box[6];
  uint32_t valid, pad;
};
static_assert(sizeof(TopEdge) == 48, "two edges in the shared layout");

// Phase T: the splits between the tiles' largest subtrees, as a bottom-up
// climb over them with the rules used inside a tile: the split between list
// positions i and i + 1 lies at the last leaf of subtree i, its delta is the
// one at subtree i + 1's first leaf, and slot i of shared memory is where the
// two meet.  A climb step touches shared memory only; the parents' records
// are written after the climbs, in one pass.
//
// When the list holds at most cap subtrees (the usual case: about 9 per
// tile of random triangles), EVERY CTA climbs the whole list in its own
// shared memory (the same tree each time) and writes its share of the
// records, so no CTA waits on another and the writes are spread over all
// SMs.  Otherwise the list is cut into ceil(total / cap) equal ranges, one
// per CTA (at most one per CTA: a cap below kTile is only for tests), and
// the splits between ranges meet in global memory (climb_global, arrival
// counters in top_flags).
__device__ __forceinline__ void build_top(uint32_t n, const BajoLbvh& t, const uint32_t* __restrict__ top_fd,
                                          const float2* __restrict__ top_box, const uint32_t* __restrict__ top_cnt,
                                          uint32_t* __restrict__ top_flags, uint32_t cap,
                                          unsigned char* __restrict__ smem, uint32_t* __restrict__ status) {
  constexpr TopSmem ly = top_smem();
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  uint32_t* s_ts = reinterpret_cast<uint32_t*>(smem + ly.tstart);  // [tiles + 1] list start of every tile
  uint32_t* s_first = reinterpret_cast<uint32_t*>(smem + ly.first);  // [m + 1] first leaf
  int8_t* s_delta = reinterpret_cast<int8_t*>(smem + ly.delta);      // [m + 1] delta at the first leaf
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + ly.cnt);      // [m - 1] arrivals + (first side << 8)
  uint16_t(*s_far)[2] = reinterpret_cast<uint16_t(*)[2]>(smem + ly.far);   // [m - 1] far ends (list positions)
  int8_t(*s_dfar)[2] = reinterpret_cast<int8_t(*)[2]>(smem + ly.dfar);     // [m - 1] deltas at them
  float(*s_box)[2][6] = reinterpret_cast<float(*)[2][6]>(smem + ly.box);  // [m - 1] children's boxes
  TopEdge* s_edge = reinterpret_cast<TopEdge*>(smem + ly.edge);            // [0] left end, [1] right end
  const uint32_t tid = threadIdx.x, nt = gridDim.x;
  const SegInfo g{0, n, 0};

  const uint32_t v = tid < nt ? __ldcg(top_cnt + tid) : 0u;
  const uint32_t ex = onesweep::scan256_exclusive<kThreads>(v, s_cnt);
  if (tid < nt) s_ts[tid] = ex;
  if (tid + 1 == nt) s_ts[nt] = ex + v;
  if (tid < 2) s_edge[tid].valid = 0u;
  __syncthreads();
  const uint32_t total = s_ts[nt];
  if (total < 2) return;  // the whole tree is inside one tile
  const uint32_t nr = min((total + cap - 1) / cap, nt);  // ranges (cap >= kTile never needs the clamp)
  if (nr > 1 && blockIdx.x >= nr) return;
  const uint32_t j0 = nr == 1 ? 0u : (uint32_t)((uint64_t)blockIdx.x * total / nr);
  const uint32_t m = (nr == 1 ? total : (uint32_t)((uint64_t)(blockIdx.x + 1) * total / nr)) - j0;
  auto entry = [&](uint32_t j) {  // list position -> slot of its tile's list
    uint32_t a = 0, z = nt + 1;   // first tile q with s_ts[q] > j
    while (a < z) {
      const uint32_t mid = (a + z) >> 1;
      if (s_ts[mid] > j) z = mid;
      else a = mid + 1;
    }
    return (a - 1u) * kTileTops + (j - s_ts[a - 1u]);
  };

  // every subtree of the range: its first leaf, the delta there and its box
  // (kTopCap <= 3 * kThreads: three per thread, every load in flight at once)
  static_assert(kTopCap <= 3 * kThreads, "three subtrees per thread");
  uint32_t fd[3];
  float2 bx[3][3];
  const bool has_after = j0 + m < total;  // the subtree after the range
  const uint32_t fd_after = (tid == 0 && has_after) ? __ldcg(top_fd + entry(j0 + m)) : 0u;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const uint32_t i = tid + r * kThreads;
    fd[r] = 0u;
    bx[r][0] = bx[r][1] = bx[r][2] = make_float2(0.0f, 0.0f);
    if (i < m) {
      const uint32_t at = entry(j0 + i);
      fd[r] = __ldcg(top_fd + at);
      bx[r][0] = __ldcg(top_box + (size_t)at * 3 + 0);
      bx[r][1] = __ldcg(top_box + (size_t)at * 3 + 1);
      bx[r][2] = __ldcg(top_box + (size_t)at * 3 + 2);
    }
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const uint32_t i = tid + r * kThreads;
    if (i < m) {
      s_first[i] = fd[r] & 0xFFFFFFu;
      s_delta[i] = (int8_t)((int)(fd[r] >> 24) - 1);
      s_cnt[i] = 0u;
    }
  }
  if (tid == 0) {
    s_first[m] = has_after ? (fd_after & 0xFFFFFFu) : n;
    s_delta[m] = has_after ? (int8_t)((int)(fd_after >> 24) - 1) : (int8_t)-1;
  }
  __syncthreads();
  // each box, far end and far delta into the split where the subtree
  // arrives (or into an edge slot); then the arrival itself
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const uint32_t i = tid + r * kThreads;
    if (i < m) {
      const int dl = s_delta[i], dr = s_delta[i + 1];
      const bool is_left = dr > dl;
      float* dst;
      if (is_left ? i + 1 >= m : i == 0) {
        TopEdge& e = s_edge[is_left ? 1 : 0];
        e.a = i;
        e.b = i;
        e.dl = dl;
        e.dr = dr;
        e.valid = 1u;
        dst = e.box;
      } else {
        const uint32_t slot = is_left ? i : i - 1, side = is_left ? 0u : 1u;
        s_far[slot][side] = (uint16_t)i;
        s_dfar[slot][side] = (int8_t)(is_left ? dl : dr);
        dst = s_box[slot][side];
      }
      dst[0] = bx[r][0].x;
      dst[1] = bx[r][0].y;
      dst[2] = bx[r][1].x;
      dst[3] = bx[r][1].y;
      dst[4] = bx[r][2].x;
      dst[5] = bx[r][2].y;
    }
  }
  __syncthreads();
  uint32_t cur[3];  // per subtree of this thread: the split where it arrived second, or kNone
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const uint32_t i = tid + r * kThreads;
    cur[r] = kNone;
    if (i < m) {
      const bool is_left = s_delta[i + 1] > s_delta[i];
      if (!(is_left ? i + 1 >= m : i == 0)) {
        const uint32_t slot = is_left ? i : i - 1;
        if (atomicAdd(&s_cnt[slot], 1u + ((is_left ? 0u : 1u) << 8)) != 0u) cur[r] = slot;
      }
    }
  }
  // One step: the second arrival at split q has both children in the slot;
  // their union climbs to the next split (or ends at the root or an edge).
  auto step = [&](uint32_t q) -> uint32_t {
    fence_acq_rel_cta();  // after the arrival: the first one's writes
    const uint32_t fa = *reinterpret_cast<const uint32_t*>(s_far[q]);
    const uint32_t a = fa & 0xFFFFu, b = fa >> 16;
    const int dl = s_dfar[q][0], dr = s_dfar[q][1];
    if (nr == 1 && a == 0u && b + 1 == m) return kNone;  // the root
    const float4* bq = reinterpret_cast<const float4*>(s_box[q]);
    const float4 x0 = bq[0], x1 = bq[1], x2 = bq[2];
    const f3 mn = vmin(mk(x0.x, x0.y, x0.z), mk(x1.z, x1.w, x2.x));
    const f3 mx = vmax(mk(x0.w, x1.x, x1.y), mk(x2.y, x2.z, x2.w));
    const bool is_left = dr > dl;
    float* dst;
    if (is_left ? b + 1 >= m : a == 0u) {  // the next split is outside this range
      TopEdge& e = s_edge[is_left ? 1 : 0];
      e.a = a;
      e.b = b;
      e.dl = dl;
      e.dr = dr;
      e.valid = 1u;
      dst = e.box;
    } else {
      const uint32_t q2 = is_left ? b : a - 1u, side = is_left ? 0u : 1u;
      dst = s_box[q2][side];
      s_far[q2][side] = (uint16_t)(is_left ? a : b);
      s_dfar[q2][side] = (int8_t)(is_left ? dl : dr);
      float2* d2 = reinterpret_cast<float2*>(dst);
      d2[0] = make_float2(mn.x, mn.y);
      d2[1] = make_float2(mn.z, mx.x);
      d2[2] = make_float2(mx.y, mx.z);
      fence_acq_rel_cta();
      return atomicAdd(&s_cnt[q2], 1u + (side << 8)) != 0u ? q2 : kNone;
    }
    dst[0] = mn.x; dst[1] = mn.y; dst[2] = mn.z; dst[3] = mx.x; dst[4] = mx.y; dst[5] = mx.z;
    return kNone;
  };
  // the climbs: one step per round for every thread (its first climb still
  // going), so the lanes of a warp take their steps together
  for (int round = 0;; ++round) {
    const uint32_t q = cur[0] != kNone ? cur[0] : (cur[1] != kNone ? cur[1] : cur[2]);
    if (q == kNone) break;
    if (round > 3 * 160) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
      break;
    }
    const uint32_t nq = step(q);
    if (cur[0] != kNone) cur[0] = nq;
    else if (cur[1] != kNone) cur[1] = nq;
    else cur[2] = nq;
  }
  __syncthreads();

  // the records of the parents built here; with one range, every CTA writes
  // its share of them
  const uint32_t ns = m - 1;
  const uint32_t q0 = nr == 1 ? (uint32_t)((uint64_t)blockIdx.x * ns / nt) : 0u;
  const uint32_t q1 = nr == 1 ? (uint32_t)((uint64_t)(blockIdx.x + 1) * ns / nt) : ns;
  for (uint32_t q = q0 + tid; q < q1; q += kThreads)
    if ((s_cnt[q] & 0xFFu) == 2u)
      write_slot_parent(g, s_first[q + 1] - 1u, s_first[s_far[q][0]], s_first[s_far[q][1] + 1] - 1u, s_dfar[q][0],
                        s_dfar[q][1], s_box[q][0], s_box[q][1], t.node_meta, t.node_leaf_counts, t.leaf_parent,
                        t.node_bounds, nullptr);
  if (nr == 1) return;  // the root is built
  __syncthreads();
  __threadfence();  // the records this CTA wrote, before any release below

  // the subtrees whose sibling lies (partly) in another range climb on in
  // global memory: first arrivals whose split saw no second one, and the edges
  for (uint32_t q = tid; q < m + 1; q += kThreads) {
    Climb c;
    const float* o;
    uint32_t a, b;
    if (q + 1 < m) {
      const uint32_t cv = s_cnt[q];
      if ((cv & 0xFFu) != 1u) continue;
      const uint32_t side = cv >> 8;
      o = s_box[q][side];
      if (side == 0u) {
        a = s_far[q][0];
        b = q;
        c.dl = s_dfar[q][0];
        c.dr = s_delta[q + 1];
      } else {
        a = q + 1;
        b = s_far[q][1];
        c.dl = s_delta[q + 1];
        c.dr = s_dfar[q][1];
      }
    } else {
      const TopEdge& e = s_edge[q + 1 - m];
      if (!e.valid) continue;
      o = e.box;
      a = e.a;
      b = e.b;
      c.dl = e.dl;
      c.dr = e.dr;
    }
    c.f = s_first[a];
    c.l = s_first[b + 1] - 1u;
    c.mn = mk(o[0], o[1], o[2]);
    c.mx = mk(o[3], o[4], o[5]);
    c.leaf = c.f == c.l;
    climb_global(g, c, t.node_meta, t.node_leaf_counts, t.leaf_parent, t.node_bounds, top_flags, t.leaf_tris,
                 status);
  }
}

template <bool VEC>
__global__ void __launch_bounds__(kThreads, 2) lbvh_fused_kernel(const float* __restrict__ verts, uint32_t n,
                                                                 BajoLbvh t, unsigned char* __restrict__ ws,
                                                                 uint32_t top_cap, uint32_t epoch,
                                                                 uint32_t* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t s_red[kWarps][12];
  __shared__ uint32_t s_flag;
  __shared__ uint32_t s_bound[2];  // sorted codes at positions base - 1 and base + kTile
  constexpr Layout kL0 = layout(0);
  const Layout L = layout(n);
  uint32_t* epoch_flag = reinterpret_cast<uint32_t*>(ws + kL0.off_epoch);
  uint32_t* bar = reinterpret_cast<uint32_t*>(ws + kL0.off_bar);
  uint32_t* seg_ord = reinterpret_cast<uint32_t*>(ws + kL0.off_seg_ord);
  uint32_t* ghist = reinterpret_cast<uint32_t*>(ws + kL0.off_ghist);
  uint32_t* counts = reinterpret_cast<uint32_t*>(ws + kL0.off_counts);  // [pass][tile][digit]
  uint32_t* bhist = reinterpret_cast<uint32_t*>(ws + kL0.off_bhist);    // [bucket] keys
  uint32_t* bfill = reinterpret_cast<uint32_t*>(ws + kL0.off_bfill);    // [bucket] slots handed out
  uint32_t* const ka = reinterpret_cast<uint32_t*>(ws + L.off_ka);
  uint32_t* const va = reinterpret_cast<uint32_t*>(ws + L.off_va);
  uint32_t* const kb = reinterpret_cast<uint32_t*>(ws + L.off_kb);
  uint32_t* const vb = reinterpret_cast<uint32_t*>(ws + L.off_vb);

  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t c = blockIdx.x;
  const uint32_t base = c * kTile;
  const uint32_t cnt = min(kTile, n - base);
  // key k of this thread sits at tile position warp*32*kKpt + 32*k + lane,
  // so (warp, k, lane) order is position order
  const uint32_t pos0 = warp * 32 * kKpt + lane;

  // ---------------- phase A: triangle bounds, root and centroid bounds
  {
    float* s_v = reinterpret_cast<float*>(smem);
    const float* src = verts + (size_t)base * 9;
    const uint32_t nf = cnt * 9;
    if (VEC) {
      const float4* s4 = reinterpret_cast<const float4*>(src);
      float4* d4 = reinterpret_cast<float4*>(s_v);
      for (uint32_t q = tid; q < nf / 4; q += kThreads) d4[q] = __ldg(s4 + q);
      for (uint32_t q = (nf & ~3u) + tid; q < nf; q += kThreads) s_v[q] = __ldg(src + q);
    } else {
      for (uint32_t q = tid; q < nf; q += kThreads) s_v[q] = __ldg(src + q);
    }
    // node_flags end at 2 for every internal node (the per-stage build's
    // arrival counters); the top's arrival counters start at zero; the next
    // passes' digit counts of this tile are accumulated by atomics
    uint32_t* top_flags = reinterpret_cast<uint32_t*>(ws + L.off_top_flags);
    for (uint32_t q = base + tid; q < min(base + kTile, n - 1); q += kThreads) {
      t.node_flags[q] = 2u;
      top_flags[q] = 0u;
    }
    for (uint32_t q = tid; q < (kPasses - 1) * 256; q += kThreads)
      counts[((q >> 8) + 1) * kMaxTiles * 256 + c * 256 + (q & 255)] = 0u;
    for (uint32_t q = c * kThreads + tid; q < 2 * kBuckets; q += gridDim.x * kThreads) bhist[q] = 0u;  // + bfill
    for (uint32_t q = c * kThreads + tid; q < kPasses * 256; q += gridDim.x * kThreads) ghist[q] = 0u;
    if (c == 0 && tid == 0) {
      t.internal_offsets[0] = 0;
      t.internal_offsets[1] = n - 1;
    }
    if (c == 0 && tid < 13) (tid == 0 ? bar : seg_ord + tid - 1)[0] = 0u;  // the counter, the 12 bounds
    if (tid == 0) s_flag = 1u;
    __syncthreads();
    if (c == 0 && tid == 0) {  // the counter and the bounds are clear: this launch's epoch
      __threadfence();
      st_relaxed_gpu(epoch_flag, epoch);
    }
  }
  float cx[kKpt], cy[kKpt], cz[kKpt];
  {
    const float* s_v = reinterpret_cast<const float*>(smem);
    uint32_t w[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) w[q] = 0;
#pragma unroll
    for (int k = 0; k < kKpt; ++k) {
      const uint32_t p = pos0 + 32 * k;
      cx[k] = cy[k] = cz[k] = 0.0f;
      if (p < cnt) {
        const float* v = s_v + p * 9;
        const f3 a = mk(v[0], v[1], v[2]), b = mk(v[3], v[4], v[5]), cc = mk(v[6], v[7], v[8]);
        const f3 mn = vmin(vmin(a, b), cc), mx = vmax(vmax(a, b), cc);
        float2* o = reinterpret_cast<float2*>(t.leaf_bounds + (size_t)(base + p) * 6);
        o[0] = make_float2(mn.x, mn.y);
        o[1] = make_float2(mn.z, mx.x);
        o[2] = make_float2(mx.y, mx.z);
        const f3 ce = (mn + mx) * 0.5f;  // core/aabb.mojo:53
        cx[k] = ce.x;
        cy[k] = ce.y;
        cz[k] = ce.z;
        w[0] = max(w[0], enc_min(mn.x)); w[1] = max(w[1], enc_min(mn.y)); w[2] = max(w[2], enc_min(mn.z));
        w[3] = max(w[3], enc_max(mx.x)); w[4] = max(w[4], enc_max(mx.y)); w[5] = max(w[5], enc_max(mx.z));
        w[6] = max(w[6], enc_min(ce.x)); w[7] = max(w[7], enc_min(ce.y)); w[8] = max(w[8], enc_min(ce.z));
        w[9] = max(w[9], enc_max(ce.x)); w[10] = max(w[10], enc_max(ce.y)); w[11] = max(w[11], enc_max(ce.z));
      }
    }
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      const uint32_t r = __reduce_max_sync(0xFFFFFFFFu, w[q]);
      if (lane == 0) s_red[warp][q] = r;
    }
    __syncthreads();
    if (tid == 0 && !wait_epoch(epoch_flag, epoch, status)) s_flag = 0u;
    __syncthreads();  // the counter and the bounds are cleared for this launch
    if (s_flag == 0u) return;  // (waited in vain: the status says so)
    if (tid < 12) {
      uint32_t r = 0;
#pragma unroll
      for (int q = 0; q < kWarps; ++q) r = max(r, s_red[q][tid]);
      if (r) atomicMax(&seg_ord[tid], r);
    }
  }
  if (!grid_sync(bar, 1, status, &s_flag)) return;

  // ---------------- phase B: Morton codes and the bucket histogram
  uint32_t key[kKpt], val[kKpt];
  uint32_t nbar = 1;  // grid barriers passed
  {
    const f3 cmin = mk(dec_min(__ldcg(seg_ord + 6)), dec_min(__ldcg(seg_ord + 7)), dec_min(__ldcg(seg_ord + 8)));
    const f3 cmax = mk(dec_max(__ldcg(seg_ord + 9)), dec_max(__ldcg(seg_ord + 10)), dec_max(__ldcg(seg_ord + 11)));
    const f3 ext = cmax - cmin;
    const f3 inv = mk(safe_inv1(ext.x), safe_inv1(ext.y), safe_inv1(ext.z));
    if (c == 0 && tid < 12) {
      const uint32_t u = __ldcg(seg_ord + tid);
      const bool is_min = tid < 3 || (tid >= 6 && tid < 9);
      t.seg_bounds[tid] = is_min ? dec_min(u) : dec_max(u);
    }
#pragma unroll
    for (int k = 0; k < kKpt; ++k) {
      const uint32_t p = pos0 + 32 * k;
      if (p < cnt) {
        const f3 d = mk(cx[k], cy[k], cz[k]) - cmin;
        key[k] = morton3(d.x * inv.x, d.y * inv.y, d.z * inv.z);
        val[k] = base + p;
        atomicAdd(&bhist[key[k] >> kBucketShift], 1u);
      } else {
        key[k] = 0xFFFFFFFFu;  // padding: the top digit in every pass, after every real key
        val[k] = 0;
      }
    }
  }
  if (!grid_sync(bar, ++nbar, status, &s_flag)) return;

  // ---------------- sort, fast path: buckets of the top code bits.  It ends
  // with this CTA's tile of sorted keys written and the codes just before
  // and after the tile in s_bound, so the hierarchy needs no more barriers.
  bool sorted = false;
  {
    uint32_t* s_b = reinterpret_cast<uint32_t*>(smem);  // [kBuckets] bucket starts
    uint32_t* s_tmp = s_b + kBuckets;                    // scan scratch [64] + results [2]
    for (uint32_t q = tid; q < kBuckets; q += kThreads) s_b[q] = __ldcg(bhist + q);
    __syncthreads();
    scan_buckets(s_b, s_tmp, s_tmp + 64);
    const bool fast = s_tmp[65] <= kBucketMax;  // every CTA reads the same histogram
    if (fast) {
      // S1: every key to a slot of its bucket's range
#pragma unroll
      for (int k = 0; k < kKpt; ++k) {
        if (pos0 + 32 * k < cnt) {
          const uint32_t b = key[k] >> kBucketShift;
          const uint32_t slot = s_b[b] + atomicAdd(&bfill[b], 1u);
          if (slot < n) {
            ka[slot] = key[k];
            va[slot] = val[k];
          }
        }
      }
      if (!grid_sync(bar, ++nbar, status, &s_flag)) return;
      // S2: the buckets that hold the sorted positions base - 1 .. base +
      // kTile, ranked in shared memory by (code, item); a bucket that also
      // reaches into a neighbouring tile is ranked by both CTAs
      uint2* s_kv = reinterpret_cast<uint2*>(s_tmp + 64 + 16);  // [kLoadMax] (code, item)
      auto bucket_at = [&](uint32_t p) {  // the (non-empty) bucket holding sorted position p
        uint32_t a = 0, z = kBuckets;     // first b with s_b[b] > p
        while (a < z) {
          const uint32_t m = (a + z) >> 1;
          if (s_b[m] > p) z = m;
          else a = m + 1;
        }
        return a - 1u;  // s_b[0] = 0 <= p
      };
      const uint32_t p0 = base > 0 ? base - 1 : 0u, p1 = min(base + kTile, n - 1);
      const uint32_t b1 = bucket_at(p1);
      const uint32_t lo = s_b[bucket_at(p0)], hi = b1 + 1 < kBuckets ? s_b[b1 + 1] : n;
      const uint32_t m = hi > lo ? hi - lo : 0u;
      if (m > kLoadMax) {  // cannot happen when every bucket fits kBucketMax
        if (tid == 0) raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        return;
      }
      for (uint32_t q = tid; q < m; q += kThreads) s_kv[q] = make_uint2(__ldcg(ka + lo + q), __ldcg(va + lo + q));
      __syncthreads();
      for (uint32_t q = tid; q < m; q += kThreads) {
        const uint2 me = s_kv[q];
        const uint32_t b = me.x >> kBucketShift;
        const uint32_t bs = s_b[b];
        const uint32_t be = b + 1 < kBuckets ? s_b[b + 1] : n;
        const uint64_t mine = ((uint64_t)me.x << 32) | me.y;
        uint32_t rank = 0;
        for (uint32_t j = bs - lo; j < be - lo; ++j) {
          const uint2 o = s_kv[j];
          rank += (((uint64_t)o.x << 32) | o.y) < mine ? 1u : 0u;
        }
        const uint32_t dst = bs + rank;
        if (dst >= base && dst < base + cnt) {
          t.morton_codes[dst] = me.x;
          t.leaf_ids[dst] = me.y;
          t.sort_keys[dst] = (uint64_t)me.x;
        } else if (dst + 1 == base) {
          s_bound[0] = me.x;
        } else if (dst == base + kTile) {
          s_bound[1] = me.x;
        }
      }
    }
    __syncthreads();  // the bucket starts are no longer read: the passes reuse the buffer
    sorted = fast;
  }

  // ---------------- sort, otherwise: LSD radix passes
  if (!sorted) {
    uint32_t* s_wh = reinterpret_cast<uint32_t*>(smem);           // [kWarps][256]: counts, then starts
    uint32_t* s_off = s_wh + kWarps * 256;                         // [256] global position - tile position
    uint32_t* s_pre = s_off + 256;                                 // [2][256] counts of the earlier tiles
    uint32_t* s_tmp = s_pre + 512;                                 // scan scratch
    const uint32_t d_own = tid & 255u, half = tid >> 8;
    {
      // every pass's digit histogram (ghist was zeroed by phase A)
      // and this tile's digit counts of pass 0
      uint32_t* s_hist = s_wh;  // [kPasses][256]
      for (uint32_t q = tid; q < kPasses * 256; q += kThreads) s_hist[q] = 0;
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kKpt; ++k)
        if (pos0 + 32 * k < cnt)
#pragma unroll
          for (int ps = 0; ps < kPasses; ++ps) atomicAdd(&s_hist[ps * 256 + ((key[k] >> (8 * ps)) & 255u)], 1u);
      __syncthreads();
      for (uint32_t q = tid; q < kPasses * 256; q += kThreads) {
        const uint32_t h = s_hist[q];
        if (h) atomicAdd(&ghist[q], h);
        if (q < 256) counts[c * 256 + q] = h;
      }
      if (!grid_sync(bar, ++nbar, status, &s_flag)) return;
    }
    for (int ps = 0; ps < kPasses; ++ps) {
      const uint32_t sh = 8u * ps;
      // counts of this pass's digit d_own in the earlier tiles (half of them per thread)
      uint32_t pre = 0;
      const uint32_t* cp = counts + (size_t)ps * kMaxTiles * 256 + d_own;
      for (uint32_t q = half; q < c; q += 2) pre += __ldcg(cp + q * 256);
      const uint32_t gcount = __ldcg(ghist + ps * 256 + d_own);
      if (ps > 0) {
        const uint32_t* ks = (ps & 1) ? ka : kb;  // written by the previous pass
        const uint32_t* vs = (ps & 1) ? va : vb;
#pragma unroll
        for (int k = 0; k < kKpt; ++k) {
          const uint32_t p = pos0 + 32 * k;
          key[k] = p < cnt ? __ldcg(ks + base + p) : 0xFFFFFFFFu;
          val[k] = p < cnt ? __ldcg(vs + base + p) : 0u;
        }
      }
      for (uint32_t q = tid; q < kWarps * 256; q += kThreads) s_wh[q] = 0;
      s_pre[half * 256 + d_own] = pre;
      __syncthreads();
      // rank among equal digits of the warp, in position order
      uint32_t* wh = s_wh + warp * 256;
      const uint32_t lt = lanemask_lt();
      uint32_t rank[kKpt];
#pragma unroll
      for (int k = 0; k < kKpt; ++k) {
        const uint32_t d = (key[k] >> sh) & 255u;
        const uint32_t peers = onesweep::match_label<8>(d);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t before = 0;
        if (lane == leader) before = atomicAdd(&wh[d], (uint32_t)__popc(peers));
        before = __shfl_sync(0xFFFFFFFFu, before, leader);
        rank[k] = before + __popc(peers & lt);
      }
      __syncthreads();
      uint32_t total = 0;
      if (tid < 256) {
#pragma unroll
        for (int w = 0; w < kWarps; ++w) total += s_wh[w * 256 + tid];
      }
      const uint32_t tstart = onesweep::scan256_exclusive<kThreads>(total, s_tmp);
      const uint32_t gbase = onesweep::scan256_exclusive<kThreads>(tid < 256 ? gcount : 0u, s_tmp);
      if (tid < 256) {
        uint32_t run = tstart;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
          const uint32_t cw = s_wh[w * 256 + tid];
          s_wh[w * 256 + tid] = run;
          run += cw;
        }
        s_off[tid] = gbase + s_pre[tid] + s_pre[256 + tid] - tstart;
      }
      __syncthreads();
      const bool last = ps == kPasses - 1;
      uint32_t* kd = (ps & 1) ? kb : ka;
      uint32_t* vd = (ps & 1) ? vb : va;
      uint32_t* next_counts = counts + (size_t)(ps + 1) * kMaxTiles * 256;
#pragma unroll
      for (int k = 0; k < kKpt; ++k) {
        const uint32_t p = pos0 + 32 * k;
        const bool ok = p < cnt;
        const uint32_t d = (key[k] >> sh) & 255u;
        const uint32_t dst = s_off[d] + rank[k] + s_wh[warp * 256 + d];
        if (last) {
          if (ok && dst < n) {
            t.morton_codes[dst] = key[k];
            t.leaf_ids[dst] = val[k];
            t.sort_keys[dst] = (uint64_t)key[k];
          }
        } else {
          if (ok && dst < n) {
            kd[dst] = key[k];
            vd[dst] = val[k];
          }
          // the next pass's digit counts of the destination tile, one atomic
          // per (tile, digit) run of the warp
          const uint32_t tag = ok ? (((dst / kTile) << 8) | ((key[k] >> (sh + 8)) & 255u)) : 0xFFFFFFFFu;
          const uint32_t same = __match_any_sync(0xFFFFFFFFu, tag);
          if (ok && lane == (uint32_t)(__ffs(same) - 1) && dst < n)
            atomicAdd(next_counts + tag, (uint32_t)__popc(same));
        }
      }
      if (!grid_sync(bar, ++nbar, status, &s_flag)) return;
    }
  }

  // ---------------- phase H: the bottom-up hierarchy, refit and triangle
  // records over this CTA's kTile sorted leaves (section 3).  After the fast
  // path the tile's sorted keys are this CTA's own writes and the two
  // boundary codes are in s_bound; after the passes a barrier has ended them.
  uint32_t* s_mark = reinterpret_cast<uint32_t*>(smem + (size_t)kRefitBlock * 72 + 8);  // starts of the tops
  if (tid < kWarps) s_mark[tid] = 0u;
  __syncthreads();
  SegInfo g;
  Climb top;
  const bool is_top =
      hierarchy_local(verts, t.leaf_ids, t.morton_codes, n, t.seg_offsets, 1, t.internal_offsets, t.node_meta,
                      t.node_leaf_counts, t.leaf_parent, t.node_bounds, nullptr, t.leaf_tris, t.roots, status,
                      smem, sorted ? s_bound : nullptr, g, top);
  // this tile's largest subtrees go to its list, in position order
  uint32_t* top_fd = reinterpret_cast<uint32_t*>(ws + L.off_top_fd);
  float2* top_box = reinterpret_cast<float2*>(ws + L.off_top_box);
  uint32_t* top_cnt = reinterpret_cast<uint32_t*>(ws + L.off_top_cnt);
  if (is_top) atomicOr(&s_mark[(top.f - base) >> 5], 1u << ((top.f - base) & 31));
  __syncthreads();
  if (is_top) {
    const uint32_t p = top.f - base, w = p >> 5;
    uint32_t e = __popc(s_mark[w] & ((1u << (p & 31)) - 1u));
    for (uint32_t q = 0; q < w; ++q) e += __popc(s_mark[q]);
    if (e < kTileTops) {
      const size_t at = (size_t)c * kTileTops + e;
      top_fd[at] = top.f | ((uint32_t)(top.dl + 1) << 24);
      top_box[at * 3 + 0] = make_float2(top.mn.x, top.mn.y);
      top_box[at * 3 + 1] = make_float2(top.mn.z, top.mx.x);
      top_box[at * 3 + 2] = make_float2(top.mx.y, top.mx.z);
    } else {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
    }
  }
  if (tid == 0) {
    uint32_t e = 0;
    for (int q = 0; q < kWarps; ++q) e += __popc(s_mark[q]);
    top_cnt[c] = min(e, kTileTops);
  }
  if (!grid_sync(bar, ++nbar, status, &s_flag)) return;
  build_top(n, t, top_fd, top_box, top_cnt, reinterpret_cast<uint32_t*>(ws + L.off_top_flags), top_cap, smem,
            status);
}


// Launch state per device: the kernel attributes are set and the co-resident
// CTA count is known.
struct DeviceState {
  bool ready = false;
  int max_ctas = 0;
};
DeviceState g_fused_state[64];
std::atomic<uint32_t> g_fused_max_leaves{kMaxLeaves};
std::atomic<uint32_t> g_top_cap{kTopCap};

// Launch epochs: unique per launch in this process, never 0, and started at
// a value drawn from the clock so that a workspace left by another process
// is unlikely to hold the epochs this one uses.
std::atomic<uint32_t> g_epoch{0};
std::once_flag g_epoch_once;
uint32_t next_epoch() {
  std::call_once(g_epoch_once, [] {
    const uint64_t t = (uint64_t)std::chrono::steady_clock::now().time_since_epoch().count();
    g_epoch.store((uint32_t)(t ^ (t >> 32)) | 1u);
  });
  uint32_t e = g_epoch.fetch_add(1u, std::memory_order_relaxed);
  if (e == 0u) e = g_epoch.fetch_add(1u, std::memory_order_relaxed);
  return e;
}

bool can_run(uint32_t n, uint32_t n_seg) {
  return n_seg == 1 && n >= 2 && n <= g_fused_max_leaves.load(std::memory_order_relaxed) && n <= kMaxLeaves;
}

// Enqueues the build (one cooperative launch); *launched = false when the
// grid cannot be co-resident on this device (the caller then runs the
// per-stage kernels).
cudaError_t launch(const float* d_verts, const BajoLbvh* bvh, unsigned char* ws, uint32_t* status, cudaStream_t st,
                   bool* launched) {
  *launched = false;
  const uint32_t n = bvh->n_leaves;
  const uint32_t G = (n + kTile - 1) / kTile;
  const bool vec = ((uintptr_t)d_verts & 15) == 0;
  auto kern = vec ? lbvh_fused_kernel<true> : lbvh_fused_kernel<false>;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaSuccess;
  DeviceState& ds = g_fused_state[dev];
  if (!ds.ready) {
    int per_sm_t = 0, per_sm_f = 0;
    if ((e = cudaFuncSetAttribute(lbvh_fused_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSmem)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(lbvh_fused_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSmem)) != cudaSuccess)
      return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_t, lbvh_fused_kernel<true>, kThreads, kSmem)) !=
            cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, lbvh_fused_kernel<false>, kThreads, kSmem)) !=
            cudaSuccess)
      return e;
    ds.max_ctas = min(per_sm_t, per_sm_f) * sm_count();
    ds.ready = true;
  }
  if ((int)G > ds.max_ctas) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kSmem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BajoLbvh tcopy = *bvh;
  const uint32_t cap = g_top_cap.load(std::memory_order_relaxed);
  const uint32_t epoch = next_epoch();
  e = cudaLaunchKernelEx(&cfg, kern, d_verts, n, tcopy, ws, cap, epoch, status);
  if (e == cudaSuccess) *launched = true;
  return e;
}
}  // namespace fused

// ---------------------------------------------------------------------------
// staged top levels
// ---------------------------------------------------------------------------
// The first BAJO_TOP_NODES internal nodes of segment 0's tree in breadth-first
// order (left before right), one level per round: every frontier node counts
// its internal children, a block scan gives them consecutive slots, and the
// children that fit become the next frontier.  Nodes whose children fall past
// the last slot keep their global refs, so any prefix of levels is a valid
// tree top.  Output layout: header [count, root ref, 0, 0] then 64-byte
// records [left AABB | right AABB | left ref, right ref, 0, 0].
constexpr uint32_t kTop = BAJO_TOP_NODES;
static_assert(kTop % 32 == 0 && kTop <= 1024, "one thread per slot");

__global__ void __launch_bounds__(kTop) stage_top_kernel(const uint32_t* __restrict__ roots,
                                                         const uint4* __restrict__ meta,
                                                         const float4* __restrict__ nb, uint32_t n_leaves,
                                                         float4* __restrict__ out) {
  __shared__ uint32_t s_ref[kTop];
  __shared__ uint2 s_child[kTop];
  __shared__ uint32_t s_warp[kTop / 32];
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t root = __ldg(roots);
  const bool stage = root != kSentinel && !(root & kLeafFlag) && n_leaves < BAJO_TOP_FLAG;
  if (t == 0) s_ref[0] = root;
  __syncthreads();
  uint32_t lo = 0, hi = stage ? 1u : 0u;
  while (lo < hi) {  // block-uniform
    const bool mine = t >= lo && t < hi;
    uint32_t cl = 0, cr = 0, cnt = 0;
    if (mine) {
      const uint4 m = __ldg(meta + s_ref[t]);
      cl = m.y;
      cr = m.z;
      cnt = (uint32_t)!(cl & kLeafFlag) + (uint32_t)!(cr & kLeafFlag);
    }
    // exclusive block scan of cnt
    uint32_t incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if ((int)lane >= d) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (uint32_t w = 0; w < kTop / 32; ++w) {
      const uint32_t c = s_warp[w];
      before += w < warp ? c : 0u;
      total += c;
    }
    if (mine) {
      uint32_t k = hi + before + incl - cnt;
      uint32_t rl = cl, rr = cr;
      if (!(cl & kLeafFlag)) {
        if (k < kTop) {
          s_ref[k] = cl;
          rl = BAJO_TOP_FLAG | k;
        }
        ++k;
      }
      if (!(cr & kLeafFlag)) {
        if (k < kTop) {
          s_ref[k] = cr;
          rr = BAJO_TOP_FLAG | k;
        }
      }
      s_child[t] = make_uint2(rl, rr);
    }
    __syncthreads();
    lo = hi;
    hi = min(kTop, hi + total);
  }
  const uint32_t n_staged = hi;
  float4* rec = out + 1 + (size_t)t * 4;
  if (t < n_staged) {
    const uint32_t r = s_ref[t];
    rec[0] = __ldg(nb + (size_t)r * 3 + 0);
    rec[1] = __ldg(nb + (size_t)r * 3 + 1);
    rec[2] = __ldg(nb + (size_t)r * 3 + 2);
    const uint2 c = s_child[t];
    rec[3] = make_float4(__uint_as_float(c.x), __uint_as_float(c.y), 0.0f, 0.0f);
  } else {
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    rec[0] = z;
    rec[1] = z;
    rec[2] = z;
    rec[3] = z;
  }
  if (t == 0) out[0] = make_float4(__uint_as_float(n_staged), __uint_as_float(root), 0.0f, 0.0f);
}

cudaError_t launch_stage_top(const BajoLbvh* bvh, cudaStream_t st) {
  stage_top_kernel<<<1, kTop, 0, st>>>(bvh->roots, reinterpret_cast<const uint4*>(bvh->node_meta),
                                       reinterpret_cast<const float4*>(bvh->node_bounds), bvh->n_leaves,
                                       reinterpret_cast<float4*>(bvh->top_nodes));
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// host plan
// ---------------------------------------------------------------------------
// Build workspace: the sort plan of the u64 keys, with the per-segment
// ordered bounds as the extra zeroed region.
// The keys' live bits: the 30 Morton bits, and above bit 32 the segment
// index when there are several segments.  variant / passes / digit_bits:
// the sort's tile shape and digit width from the tuning table; the
// workspace fits every variant the size allows.
struct BuildPlan {
  onesweep::Plan sort;
  int end_bit;
  int variant;
  uint32_t passes, digit_bits;
  size_t off_seg_ord, off_keys_alt, off_vals_alt, total;
};

BuildPlan make_build_plan(uint32_t n, uint32_t n_seg) {
  BuildPlan b{};
  int seg_bits = 0;
  while (seg_bits < 32 && ((n_seg - 1) >> seg_bits)) ++seg_bits;
  b.end_bit = n_seg > 1 ? 32 + seg_bits : 30;
  b.variant = onesweep::choose_variant<uint64_t, true>(n, sm_count());
  b.digit_bits = onesweep::variant_bits<uint64_t>(b.variant);
  b.passes = onesweep::passes_for(0, b.end_bit, b.digit_bits);
  b.sort = onesweep::make_plan<uint64_t>(n, true, onesweep::num_passes(0, b.end_bit), (size_t)n_seg * 12 * 4);
  b.off_seg_ord = b.sort.off_extra;
  b.off_keys_alt = b.sort.off_keys_alt;
  b.off_vals_alt = b.sort.off_vals_alt;
  b.total = b.sort.total;
  // room for the one-launch build as well (section 5)
  if (n_seg == 1 && n <= fused::kMaxLeaves && fused::layout(n).total > b.total) b.total = fused::layout(n).total;
  return b;
}

}  // namespace

size_t hploc_workspace_bytes(uint32_t n, uint32_t n_seg);  // hploc.cu
cudaError_t launch_hploc(const float* d_verts, BajoLbvh* bvh, unsigned char* extra, uint32_t* status,
                         cudaStream_t st);
}  // namespace bajo

extern "C" {

int32_t bajo_lbvh_sizes(uint32_t n, uint32_t n_seg, BajoLbvhSizes* s) {
  if (!s || n_seg == 0) return BAJO_ERR_INVALID_ARGUMENT;
  if (n > BAJO_SORT_MAX_KEYS) return BAJO_ERR_TOO_LARGE;
  const size_t N = n ? n : 1, M = N;
  s->internal_offsets = (size_t)(n_seg + 1) * 4;
  s->leaf_bounds = N * 24;
  s->seg_bounds = (size_t)n_seg * 48;
  s->sort_keys = N * 8;
  s->leaf_ids = N * 4;
  s->morton_codes = N * 4;
  s->node_meta = M * 16;
  s->node_bounds = M * 48;
  s->node_leaf_counts = M * 4;
  s->node_flags = M * 4;
  s->leaf_parent = N * 4;
  s->roots = (size_t)n_seg * 4;
  s->leaf_tris = N * 48;
  s->workspace = bajo::make_build_plan(n, n_seg).total;
  s->top_nodes = BAJO_TOP_BYTES;
  return BAJO_OK;
}

// hploc: the tree comes from H-PLOC (hploc.cu) instead of the LBVH topology
// and refit; its workspace is the LBVH build's plus hploc_workspace_bytes
static size_t hploc_extra_offset(uint32_t n, uint32_t n_seg) {
  return (bajo::make_build_plan(n, n_seg).total + 255) & ~(size_t)255;
}

// The bottom-up hierarchy + refit of builds of up to kMergedMaxLeaves
// triangles (section 3); node_flags must be zero and the sorted leaves ready.
static cudaError_t launch_hierarchy(const float* d_verts, BajoLbvh* bvh, uint32_t* status, cudaStream_t st) {
  using namespace bajo;
  const uint32_t n = bvh->n_leaves, S = bvh->n_segments;
  constexpr size_t hier_smem = (size_t)kRefitBlock * 72 + 8;
  cudaError_t e = cudaFuncSetAttribute(hierarchy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hier_smem);
  if (e != cudaSuccess) return e;
  const uint32_t grid = (max(max(n, S), 1u) + kRefitBlock - 1) / kRefitBlock;
  hierarchy_kernel<<<grid, kRefitBlock, hier_smem, st>>>(
      d_verts, bvh->leaf_ids, bvh->morton_codes, n, bvh->seg_offsets, S, bvh->internal_offsets, bvh->node_meta,
      bvh->node_leaf_counts, bvh->leaf_parent, bvh->node_bounds, bvh->node_flags, bvh->leaf_tris, bvh->roots, status);
  return cudaGetLastError();
}

static int32_t lbvh_build_impl(const float* d_verts, BajoLbvh* bvh, void* ws_, size_t ws_bytes, void* stream_,
                               cudaEvent_t* ev, int32_t n_ev, bool hploc = false) {
  using namespace bajo;
  if (!bvh || !ws_ || bvh->n_segments == 0 || !bvh->seg_offsets) return BAJO_ERR_INVALID_ARGUMENT;
  const uint32_t n = bvh->n_leaves, S = bvh->n_segments;
  if (n > BAJO_SORT_MAX_KEYS) return BAJO_ERR_TOO_LARGE;
  if (n > 0 && (!d_verts || !bvh->internal_offsets || !bvh->leaf_bounds || !bvh->seg_bounds || !bvh->sort_keys ||
                !bvh->leaf_ids || !bvh->morton_codes || !bvh->node_meta || !bvh->node_bounds ||
                !bvh->node_leaf_counts || !bvh->node_flags || !bvh->leaf_parent || !bvh->roots || !bvh->leaf_tris))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (bvh->top_nodes && ((uintptr_t)bvh->top_nodes & 15)) return BAJO_ERR_INVALID_ARGUMENT;
  if (n > 0 && (((uintptr_t)bvh->node_bounds & 15) || ((uintptr_t)bvh->node_meta & 15) ||
                ((uintptr_t)bvh->leaf_tris & 15)))
    return BAJO_ERR_INVALID_ARGUMENT;  // their records are read and written 16 bytes at a time
  BuildPlan plan = make_build_plan(n, S);
  const size_t need = hploc ? hploc_extra_offset(n, S) + hploc_workspace_bytes(n, S) : plan.total;
  if (ws_bytes < need) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  cudaStream_t st = (cudaStream_t)stream_;
  unsigned char* ws = (unsigned char*)ws_;
  uint32_t* status = (uint32_t*)ws;
  // one scene of up to fused::kMaxLeaves triangles: the one-launch build;
  // its stage events are [start, build]
  // (the one-launch build keeps 8- and 16-byte records in the workspace)
  if (!hploc && fused::can_run(n, S) && ((uintptr_t)ws & 15) == 0 && (!ev || n_ev == 2)) {
    if (ev && cudaEventRecord(ev[0], st) != cudaSuccess) return BAJO_ERR_CUDA;
    bool launched = false;
    if (fused::launch(d_verts, bvh, ws, status, st, &launched) != cudaSuccess) return BAJO_ERR_CUDA;
    if (launched) {
      if (ev && cudaEventRecord(ev[1], st) != cudaSuccess) return BAJO_ERR_CUDA;
      if (bvh->top_nodes && launch_stage_top(bvh, st) != cudaSuccess) return BAJO_ERR_CUDA;
      return BAJO_OK;
    }
    if (ev) return BAJO_ERR_INVALID_ARGUMENT;  // the per-stage kernels need their own events
  }
  if (ev && n_ev < (int32_t)(5 + plan.passes)) return BAJO_ERR_INVALID_ARGUMENT;
  // stage events: [start, bounds, morton, pass 0..P-1, topology, refit]
  auto mark = [&](int i) { return !ev || cudaEventRecord(ev[i], st) == cudaSuccess; };
  if (!mark(0)) return BAJO_ERR_CUDA;
  if (cudaMemsetAsync(ws + plan.sort.off_zero, 0, plan.sort.zero_bytes, st) != cudaSuccess) return BAJO_ERR_CUDA;
  uint32_t* seg_ord = (uint32_t*)(ws + plan.off_seg_ord);
  const uint32_t blocks = (n + kBlock - 1) / kBlock;

  bounds_kernel<<<blocks ? blocks : 1, kBlock, 0, st>>>(d_verts, n, bvh->seg_offsets, S, bvh->internal_offsets,
                                                        bvh->leaf_bounds, seg_ord);
  if (cudaGetLastError() != cudaSuccess || !mark(1)) return BAJO_ERR_CUDA;

  // sort buffers: the Morton kernel writes where an even/odd pass count lands
  // the result in bvh->sort_keys / bvh->leaf_ids
  const uint32_t passes = plan.passes;
  uint64_t* kalt = (uint64_t*)(ws + plan.off_keys_alt);
  uint32_t* valt = (uint32_t*)(ws + plan.off_vals_alt);
  // (with n <= 1 nothing is sorted and the keys stay where they are written)
  const bool even = (passes % 2) == 0 || n <= 1;
  uint64_t* k0 = even ? bvh->sort_keys : kalt;
  uint32_t* v0 = even ? bvh->leaf_ids : valt;
  uint64_t* k1 = even ? kalt : bvh->sort_keys;
  uint32_t* v1 = even ? valt : bvh->leaf_ids;
  uint32_t* ghist = (uint32_t*)(ws + plan.sort.off_ghist);
  {
    const size_t smem = (size_t)passes * morton_hist_copies(passes, plan.digit_bits) * (4u << plan.digit_bits);
    uint32_t grid = blocks;
    const uint32_t cap = (uint32_t)sm_count() * 8;
    if (grid > cap) grid = cap;
    if (grid == 0) grid = 1;
    if (smem > 48 * 1024) {
      if (cudaFuncSetAttribute(morton_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
        return BAJO_ERR_CUDA;
    }
    morton_kernel<<<grid, kBlock, smem, st>>>(bvh->leaf_bounds, n, bvh->seg_offsets, S, seg_ord, bvh->seg_bounds, k0,
                                              v0, passes, (uint32_t)plan.end_bit, plan.digit_bits, ghist,
                                              bvh->node_flags);
    if (cudaGetLastError() != cudaSuccess || !mark(2)) return BAJO_ERR_CUDA;
  }
  if (n > 1) {
    bool in_first = true;
    if (onesweep::run_passes<uint64_t, true>(k0, v0, k1, v1, bvh->morton_codes, plan.sort, ws, 0, plan.end_bit, st,
                                             &in_first, plan.variant, ev ? ev + 3 : nullptr) != cudaSuccess)
      return BAJO_ERR_CUDA;
  } else {
    // nothing to sort; keep the low word in step with the key
    if (n == 1 &&
        cudaMemcpyAsync(bvh->morton_codes, bvh->sort_keys, 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return BAJO_ERR_CUDA;
    for (uint32_t p = 0; p < passes; ++p)
      if (!mark(3 + p)) return BAJO_ERR_CUDA;
  }
  if (hploc) {
    if (!mark(3 + passes)) return BAJO_ERR_CUDA;
    if (launch_hploc(d_verts, bvh, ws + hploc_extra_offset(n, S), status, st) != cudaSuccess) return BAJO_ERR_CUDA;
  } else if (n <= kMergedMaxLeaves) {
    // one bottom-up pass builds the hierarchy and refits it: the topology
    // stage event is recorded right before it
    if (!mark(3 + passes)) return BAJO_ERR_CUDA;
    if (launch_hierarchy(d_verts, bvh, status, st) != cudaSuccess) return BAJO_ERR_CUDA;
  } else {
    topology_kernel<<<(max(n, S) + kBlock - 1) / kBlock, kBlock, 0, st>>>(
        bvh->morton_codes, bvh->seg_offsets, S, bvh->internal_offsets, n, bvh->node_meta, bvh->leaf_parent,
        bvh->node_leaf_counts, bvh->node_flags, bvh->node_bounds, bvh->roots);
    if (cudaGetLastError() != cudaSuccess || !mark(3 + passes)) return BAJO_ERR_CUDA;
    constexpr size_t refit_smem = kRefitBlock * (16 + 4 + 4 + 2 * 6 * 4);
    if (cudaFuncSetAttribute(refit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)refit_smem) !=
        cudaSuccess)
      return BAJO_ERR_CUDA;
    refit_kernel<<<(n + kRefitBlock - 1) / kRefitBlock, kRefitBlock, refit_smem, st>>>(
        d_verts, bvh->leaf_ids, n, bvh->seg_offsets, S, bvh->internal_offsets, bvh->node_meta, bvh->node_leaf_counts,
        bvh->leaf_parent, bvh->node_bounds, bvh->node_flags, bvh->leaf_tris, status);
    if (cudaGetLastError() != cudaSuccess) return BAJO_ERR_CUDA;
  }
  if (!mark(4 + passes)) return BAJO_ERR_CUDA;
  if (bvh->top_nodes && launch_stage_top(bvh, st) != cudaSuccess) return BAJO_ERR_CUDA;
  return BAJO_OK;
}

int32_t bajo_lbvh_build(const float* d_verts, BajoLbvh* bvh, void* ws, size_t ws_bytes, void* stream) {
  return lbvh_build_impl(d_verts, bvh, ws, ws_bytes, stream, nullptr, 0);
}

int32_t bajo_hploc_workspace_size(uint32_t n, uint32_t n_seg, size_t* bytes) {
  if (!bytes || n_seg == 0) return BAJO_ERR_INVALID_ARGUMENT;
  if (n > BAJO_SORT_MAX_KEYS) return BAJO_ERR_TOO_LARGE;
  *bytes = hploc_extra_offset(n, n_seg) + bajo::hploc_workspace_bytes(n, n_seg);
  return BAJO_OK;
}

int32_t bajo_hploc_build(const float* d_verts, BajoLbvh* bvh, void* ws, size_t ws_bytes, void* stream) {
  return lbvh_build_impl(d_verts, bvh, ws, ws_bytes, stream, nullptr, 0, true);
}

int32_t bajo_lbvh_build_timed(const float* d_verts, BajoLbvh* bvh, void* ws, size_t ws_bytes, void* stream,
                              void* const* events, int32_t n_events) {
  if (!events) return BAJO_ERR_INVALID_ARGUMENT;
  return lbvh_build_impl(d_verts, bvh, ws, ws_bytes, stream, (cudaEvent_t*)events, n_events);
}

int32_t bajo_lbvh_stage_top(const BajoLbvh* bvh, void* stream) {
  if (!bvh || !bvh->top_nodes || !bvh->roots || !bvh->node_meta || !bvh->node_bounds ||
      ((uintptr_t)bvh->top_nodes & 15))
    return BAJO_ERR_INVALID_ARGUMENT;
  return bajo::launch_stage_top(bvh, (cudaStream_t)stream) == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_lbvh_fused_max_set(uint32_t max_leaves) {
  if (max_leaves > bajo::fused::kMaxLeaves) return BAJO_ERR_TOO_LARGE;
  bajo::fused::g_fused_max_leaves.store(max_leaves, std::memory_order_relaxed);
  return BAJO_OK;
}

int32_t bajo_lbvh_fused_top_cap_set(uint32_t cap) {
  if (cap > bajo::fused::kTopCap) return BAJO_ERR_TOO_LARGE;
  bajo::fused::g_top_cap.store(cap ? cap : bajo::fused::kTopCap, std::memory_order_relaxed);
  return BAJO_OK;
}

int32_t bajo_lbvh_build_launches(uint32_t n_tris, uint32_t n_segments, int32_t* launches) {
  using namespace bajo;
  if (!launches || n_segments == 0) return BAJO_ERR_INVALID_ARGUMENT;
  if (n_tris > BAJO_SORT_MAX_KEYS) return BAJO_ERR_TOO_LARGE;
  if (fused::can_run(n_tris, n_segments)) {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
      const fused::DeviceState& ds = fused::g_fused_state[dev];
      if (!ds.ready || (int)((n_tris + fused::kTile - 1) / fused::kTile) <= ds.max_ctas) {
        *launches = 1;  // the one-launch build
        return BAJO_OK;
      }
    }
  }
  const BuildPlan plan = make_build_plan(n_tris, n_segments);
  *launches = (int32_t)(2 + (n_tris > 1 ? plan.passes : 0) + (n_tris <= kMergedMaxLeaves ? 1 : 2));
  return BAJO_OK;
}

int32_t bajo_lbvh_stage_count(uint32_t n_tris, uint32_t n_segments, int32_t* n_events) {
  if (!n_events || n_segments == 0) return BAJO_ERR_INVALID_ARGUMENT;
  int32_t launches = 0;
  if (bajo_lbvh_build_launches(n_tris, n_segments, &launches) == BAJO_OK && launches == 1 &&
      bajo::fused::can_run(n_tris, n_segments)) {
    *n_events = 2;  // [start, build]
    return BAJO_OK;
  }
  *n_events = (int32_t)(5 + bajo::make_build_plan(n_tris, n_segments).passes);
  return BAJO_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// bounded-wait self-test
// ---------------------------------------------------------------------------
namespace bajo {
namespace {
__global__ void wait_selftest_kernel(const uint32_t* flag, uint32_t bits, uint64_t limit_ns, uint32_t* status) {
  if (!wait_bits_acquire(flag, bits, limit_ns)) raise_status(status, BAJO_STATUS_WAIT_TIMEOUT);
}
}  // namespace
}  // namespace bajo

extern "C" int32_t bajo_wait_selftest(const uint32_t* d_flag, uint32_t bits, uint32_t limit_us, uint32_t* d_status,
                                      void* stream) {
  if (!d_flag || !d_status || bits == 0 || limit_us == 0 || limit_us > 1000000u) return BAJO_ERR_INVALID_ARGUMENT;
  bajo::wait_selftest_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(d_flag, bits, (uint64_t)limit_us * 1000ull,
                                                                d_status);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}
