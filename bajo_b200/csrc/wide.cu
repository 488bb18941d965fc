// wide.cu -- deterministic BVH2 -> W-wide collapse (W = 4, 8) of a built
// binary LBVH, and closest-hit traversal of the wide tree.
//
// Reference: hploc_literature_to_wide_kernel (bajo/bvh/gpu/builder/
// wide_collapse.mojo:148-644; H-PLOC paper section 3.4, HIPRT fat leaves) and
// pack_segmented_triangle_leaf_lanes_kernel (bajo/bvh/gpu/triangle_bvh.mojo:
// 81-148), driven by enqueue_segmented_wide_build (segmented_build.mojo:89)
// with max_leaf_size = leaf width and fat leaves on.  The reference hands out
// node and leaf ids with atomics while its work queue runs, so its layout
// differs from run to run; here ids are pre-order and fixed:
//   1. count_kernel climbs the binary tree bottom-up (refit-style arrival
//      flags) and, at every internal node x, applies the opening rule to
//      find the children the wide node rooted at x would have, and the
//      number of wide nodes NW(x) and leaf blocks NL(x) of that collapsed
//      subtree;
//   2. offsets_kernel turns the roots' counts into per-segment node and leaf
//      offsets and publishes each root's task;
//   3. assign_kernel walks wide node ids in increasing order: node I's task
//      (binary node, first leaf block) is published by its parent, which has
//      a smaller id, so every wait points backwards and a resident grid
//      always makes progress.  Node I writes its own leaf blocks first, then
//      gives child c the id I + 1 + (wide nodes of the children before it)
//      and the matching leaf base, and publishes c's task.
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
  uint32_t* ready;      // [wide node] task published
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
    uint32_t cand[W], cnt[W];
    const int nc =
        open_children<W>(x, node_meta, node_leaf_counts, leaf_bounds, leaf_ids, node_bounds, max_leaf, cand, cnt);
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
      wk.ready[pn] = 1u;
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

template <int W>
__device__ __forceinline__ void store_empty(float* node, int lane) {
  Box b;
  b.mn = mk(FLT_MAX, FLT_MAX, FLT_MAX);
  b.mx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  store_lane<W>(node, lane, b, kEmpty);
}

template <int W>
__global__ void __launch_bounds__(kBlock) assign_kernel(uint32_t n_seg, const uint32_t* __restrict__ node_meta,
                                                        const uint32_t* __restrict__ node_leaf_counts,
                                                        const float* __restrict__ leaf_bounds,
                                                        const uint32_t* __restrict__ leaf_ids,
                                                        const float* __restrict__ node_bounds,
                                                        const float4* __restrict__ tris,
                                                        const uint32_t* __restrict__ node_offsets,
                                                        const uint32_t* __restrict__ leaf_offsets, uint32_t cap,
                                                        uint32_t max_leaf, Work wk, Out o) {
  // node and leaf-block totals never exceed the triangle count; more means
  // the binary tree is corrupt
  uint32_t total = node_offsets[n_seg];
  if (total > cap || leaf_offsets[n_seg] > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
    return;
  }
  const uint32_t stride = gridDim.x * kBlock;
  for (uint32_t I = blockIdx.x * kBlock + threadIdx.x; I < total; I += stride) {
    const uint64_t t0 = global_timer_ns();
    while (ld_acquire_gpu(wk.ready + I) == 0) {
      if (global_timer_ns() - t0 > kWaitNs) {
        raise_status(wk.status, BAJO_STATUS_WIDE_TIMEOUT);
        return;
      }
    }
    const uint32_t x = wk.task_ref[I], B = wk.task_leaf[I], s = wk.task_seg[I];
    const uint32_t nb = node_offsets[s], lb = leaf_offsets[s];
    float* node = o.nodes + (size_t)I * kFields * W;
    const uint32_t xc = ref_count(x, node_leaf_counts);
    if (terminal(x, xc, max_leaf)) {  // a segment of at most max_leaf triangles: one node, one leaf block
      if (B >= cap) {
        raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
        continue;
      }
      write_leaf_block<W>(x, B, node_meta, leaf_ids, tris, o, wk.status);
      store_lane<W>(node, 0, ref_bounds(x, leaf_bounds, leaf_ids, node_bounds), pack_meta(B - lb, xc));
      for (int j = 1; j < W; ++j) store_empty<W>(node, j);
      continue;
    }
    const uint32_t xi = x & kIndexMask;
    const uint32_t info = wk.cinfo[xi];
    const int nc = (int)(info & 0xFF);
    const uint32_t mask = info >> 8;
    uint32_t leaf_next = B;
    for (int k = 0; k < nc; ++k) {
      if (!(mask & (1u << k))) continue;
      if (leaf_next >= cap) {
        raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
        break;
      }
      write_leaf_block<W>(wk.cands[(size_t)xi * W + k], leaf_next, node_meta, leaf_ids, tris, o, wk.status);
      ++leaf_next;
    }
    uint32_t own = B, child = I + 1, child_leaf = leaf_next;
    for (int k = 0; k < W; ++k) {
      if (k >= nc) {
        store_empty<W>(node, k);
        continue;
      }
      const uint32_t c = wk.cands[(size_t)xi * W + k];
      const Box bx = ref_bounds(c, leaf_bounds, leaf_ids, node_bounds);
      if (mask & (1u << k)) {
        store_lane<W>(node, k, bx, pack_meta(own - lb, ref_count(c, node_leaf_counts)));
        ++own;
      } else {
        const uint32_t ci = c & kIndexMask;
        store_lane<W>(node, k, bx, pack_meta(child - nb, 0));
        if (child < total) {
          wk.task_ref[child] = c;
          wk.task_leaf[child] = child_leaf;
          wk.task_seg[child] = s;
          st_release_gpu(wk.ready + child, 1u);
        } else {
          raise_status(wk.status, BAJO_STATUS_BAD_TOPOLOGY);
        }
        child += wk.nw[ci];
        child_leaf += wk.nl[ci];
      }
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
  const uint32_t i = blockIdx.x * trav::kTraceBlock + threadIdx.x;
  if (i >= n) return;
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
  size_t flags, ready, cands, cinfo, nw, nl, task_ref, task_leaf, task_seg, zero_bytes, total;
};

inline Plan make_plan(uint32_t n, uint32_t width) {
  Plan p;
  const size_t cap = std::max<uint32_t>(n, 1);
  size_t o = 256;  // status word
  p.flags = o;
  o = a256(o + cap * 4);
  p.ready = o;
  o = a256(o + cap * 4);
  p.zero_bytes = o;  // status, flags and ready are cleared per build
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
  p.total = o;
  return p;
}

template <int W>
cudaError_t build(const BajoLbvh* b, BajoWideBvh* out, unsigned char* ws, const Plan& p, uint32_t max_leaf,
                  cudaStream_t st) {
  Work wk;
  wk.status = (uint32_t*)ws;
  wk.flags = (uint32_t*)(ws + p.flags);
  wk.ready = (uint32_t*)(ws + p.ready);
  wk.cands = (uint32_t*)(ws + p.cands);
  wk.cinfo = (uint32_t*)(ws + p.cinfo);
  wk.nw = (uint32_t*)(ws + p.nw);
  wk.nl = (uint32_t*)(ws + p.nl);
  wk.task_ref = (uint32_t*)(ws + p.task_ref);
  wk.task_leaf = (uint32_t*)(ws + p.task_leaf);
  wk.task_seg = (uint32_t*)(ws + p.task_seg);
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
                                     std::max<uint32_t>(n, 1), out->node_offsets, out->leaf_offsets);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  // every block resident, so a task's producer always runs
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, assign_kernel<W>, kBlock, 0)) != cudaSuccess)
    return e;
  uint32_t grid = (uint32_t)std::max(1, per_sm) * (uint32_t)sm_count();
  const uint32_t need = (n + kBlock - 1) / kBlock;
  if (grid > need) grid = need;
  Out o{out->nodes, out->leaf_indices, out->leaf_tris, out->leaf_sorted};
  assign_kernel<W><<<grid, kBlock, 0, st>>>(b->n_segments, b->node_meta, b->node_leaf_counts, b->leaf_bounds,
                                           b->leaf_ids, b->node_bounds,
                                           reinterpret_cast<const float4*>(b->leaf_tris), out->node_offsets,
                                           out->leaf_offsets, std::max<uint32_t>(n, 1), max_leaf, wk, o);
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
  wide_camera_kernel<W, MODE, STATS><<<(n + trav::kTraceBlock - 1) / trav::kTraceBlock, trav::kTraceBlock, 0, st>>>(
      cams, n, w, h, 1.0f / (float)h, v, hits8, t, prim, status, stats);
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
  const cudaError_t e = out->width == 4 ? build<4>(b, out, (unsigned char*)ws, p, max_leaf, st)
                                        : build<8>(b, out, (unsigned char*)ws, p, max_leaf, st);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
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
