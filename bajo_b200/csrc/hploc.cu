// hploc.cu -- H-PLOC (Benthin, Meister, Barczak, Mehalwal, Tsakok, Kensler,
// HPG 2024): the binary tree of bajo_hploc_build, from the sorted Morton keys
// the LBVH front end produces.
//
// Restates init_hploc_multi_wave_kernel / build_hploc_multi_wave_kernel /
// finalize_hploc_multi_wave_kernel (bajo/bvh/gpu/builder/
// hploc_multi_wave.mojo:157-572):
//  - one thread per sorted leaf climbs the binary radix tree of the keys
//    (Apetrei's rule over XOR deltas of (code, global position) keys,
//    _hploc_find_parent_id :126-140); an atomic exchange on the split's slot
//    tells the first thread to stop and the second the sibling's range end;
//  - once a range holds more than 16 leaves (HPLOC_MERGING_THRESHOLD), or is
//    the whole segment, the warp takes it as a task: the two children's
//    cluster lists (packed at the range starts, at most 16 each) fill the
//    lanes, and PLOC rounds run until at most 16 clusters remain (1 for the
//    segment): every lane offers the merged-box area of each of the next 8
//    clusters (HPLOC_SEARCH_RADIUS) to both ends as a 64-bit key (area bits
//    << 32 | offset code) through a shared-memory atomicMin, mutual nearest
//    neighbours merge (the lower lane keeps the node), survivors compact in
//    order;
//  - a round's new nodes take consecutive ids from the segment's counter
//    (one atomic per round), so ids vary from run to run as in the reference;
//    children, boxes and leaf counts do not.
// No thread waits for another: the second arrival reads the sibling's
// results, which the first published before its exchange (fence).
#include "bajo_common.cuh"

namespace bajo {
namespace hploc {

constexpr int kBlock = 256;
constexpr int kThreshold = 16;  // HPLOC_MERGING_THRESHOLD = WARP_SIZE / 2
constexpr int kRadius = 8;      // HPLOC_SEARCH_RADIUS
constexpr unsigned kFull = 0xFFFFFFFFu;

struct Ws {
  uint32_t* slots;     // [N] parent slots (the sibling's far range end)
  uint32_t* clusters;  // [N] cluster lists, packed at each range start
  float* boxes;        // [M][6] box of every new node
  uint32_t* counters;  // [S] nodes made per segment
};

__device__ __forceinline__ uint64_t hdelta(const uint32_t* __restrict__ codes, uint32_t a, uint32_t b) {
  return ((((uint64_t)__ldg(codes + a)) << 32) | a) ^ ((((uint64_t)__ldg(codes + b)) << 32) | b);
}

__device__ __forceinline__ uint32_t enc_off(int i, int j) {
  const int s = j - i, d = (s < 0 ? -s : s) - 1;
  return (uint32_t)(d * 2 + (s < 0 ? 1 : 0));
}

__device__ __forceinline__ int dec_off(int i, uint32_t e) {
  const int d = (int)(e >> 1) + 1;
  return (e & 1u) ? i - d : i + d;
}

// bajo/core/aabb.mojo:47
__device__ __forceinline__ float area6(const float* b) {
  const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  return 2.0f * ((dx * dy + dx * dz) + dy * dz);
}

// leaves, parent slots, clusters and sorted triangle records; empty or
// single-leaf roots (init_hploc_multi_wave_kernel, :157-184)
__global__ void __launch_bounds__(kBlock) init_kernel(uint32_t n, const uint32_t* __restrict__ seg_offsets,
                                                      uint32_t n_seg, const uint32_t* __restrict__ leaf_ids,
                                                      const float* __restrict__ verts, Ws w,
                                                      uint32_t* __restrict__ leaf_parent, uint32_t* __restrict__ roots,
                                                      float* __restrict__ leaf_tris, uint32_t* __restrict__ status) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n) {
    w.slots[i] = kSentinel;
    leaf_parent[i] = kSentinel;
    w.clusters[i] = kLeafFlag | i;
    const uint32_t seg = n_seg > 1 ? segment_for_item(seg_offsets, n_seg + 1, i) : 0;
    const uint32_t item = leaf_ids[i];
    if (item >= n) {
      raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
    } else {
      const float* v = verts + (size_t)item * 9;
      float4* rec = reinterpret_cast<float4*>(leaf_tris + (size_t)i * 12);
      rec[0] = make_float4(__ldg(v + 0), __ldg(v + 1), __ldg(v + 2), __uint_as_float(item - seg_offsets[seg]));
      rec[1] = make_float4(__ldg(v + 3), __ldg(v + 4), __ldg(v + 5), 0.0f);
      rec[2] = make_float4(__ldg(v + 6), __ldg(v + 7), __ldg(v + 8), 0.0f);
    }
  }
  if (i < n_seg) {
    const uint32_t b = seg_offsets[i], e = seg_offsets[i + 1];
    w.counters[i] = 0;
    roots[i] = e - b == 1 ? (kLeafFlag | b) : kSentinel;
  }
}

__global__ void __launch_bounds__(kBlock) build_kernel(uint32_t n, const uint32_t* __restrict__ codes,
                                                       const uint32_t* __restrict__ seg_offsets, uint32_t n_seg,
                                                       const uint32_t* __restrict__ internal_offsets,
                                                       const float* __restrict__ leaf_bounds,
                                                       const uint32_t* __restrict__ leaf_ids, Ws w,
                                                       uint32_t* __restrict__ node_meta, float* __restrict__ node_bounds,
                                                       uint32_t* __restrict__ node_flags,
                                                       uint32_t* __restrict__ node_leaf_counts,
                                                       uint32_t* __restrict__ leaf_parent, uint32_t* __restrict__ roots,
                                                       uint32_t* __restrict__ status) {
  __shared__ float s_box[6][kBlock];
  __shared__ unsigned long long s_key[kBlock];
  __shared__ uint32_t s_ref[kBlock];
  if (n <= 1) return;
  const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
  const int lane = (int)(threadIdx.x & 31u), me = (int)threadIdx.x, wbase = me - lane;
  uint32_t left = idx, right = idx, split = 0;
  bool active = idx < n;
  uint32_t seg = 0, sb = 0, se = 0;
  if (active) {
    seg = n_seg > 1 ? segment_for_item(seg_offsets, n_seg + 1, idx) : 0;
    sb = seg_offsets[seg];
    se = seg_offsets[seg + 1];
  }
  auto cluster_box = [&](uint32_t ref, float* out) {
    const float* p = (ref & kLeafFlag) ? leaf_bounds + (size_t)__ldg(leaf_ids + (ref & kIndexMask)) * 6
                                       : w.boxes + (size_t)(ref & kIndexMask) * 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = __ldcg(p + k);
  };
  while (__ballot_sync(kFull, active)) {
    if (active) {
      uint32_t prev;
      const bool go_right = left == sb || (right + 1 != se && hdelta(codes, right, right + 1) <
                                                                hdelta(codes, left - 1, left));
      if (go_right) {
        prev = atomicExch(w.slots + right, left);
        if (prev != kSentinel) {
          split = right + 1;
          right = prev;
        }
      } else {
        prev = atomicExch(w.slots + left - 1, right);
        if (prev != kSentinel) {
          split = left;
          left = prev;
        }
      }
      if (prev == kSentinel) active = false;
      else __threadfence();  // the sibling's clusters and boxes, published before its exchange
    }
    const bool fin = active && right - left + 1 == se - sb;
    uint32_t tasks = __ballot_sync(kFull, active && (right - left + 1 > (uint32_t)kThreshold || fin));
    while (tasks) {
      const int tl = __ffs(tasks) - 1;
      const uint32_t t_left = __shfl_sync(kFull, left, tl), t_right = __shfl_sync(kFull, right, tl);
      const uint32_t t_split = __shfl_sync(kFull, split, tl), t_seg = __shfl_sync(kFull, seg, tl);
      const bool t_fin = __shfl_sync(kFull, (int)fin, tl) != 0;
      // the children's lists, left then right, packed into the lanes
      uint32_t ref = kSentinel;
      const int left_span = min((int)(t_split - t_left), kThreshold);
      const bool load_left = lane < left_span;
      if (load_left) ref = __ldcg(w.clusters + t_left + lane);
      const int num_left = __popc(__ballot_sync(kFull, load_left && ref != kSentinel));
      const int ri = lane - num_left;
      const int right_span = min((int)(t_right + 1 - t_split), kThreshold);
      const bool load_right = ri >= 0 && ri < right_span;
      if (load_right) ref = __ldcg(w.clusters + t_split + ri);
      else if (lane >= num_left) ref = kSentinel;
      const int num_right = __popc(__ballot_sync(kFull, load_right && ref != kSentinel));
      int count = num_left + num_right;
      const int before = count;
      const int threshold = t_fin ? 1 : kThreshold;
      float bx[6];
      if (lane < count) {
        cluster_box(ref, bx);
      } else {
        bx[0] = bx[1] = bx[2] = FLT_MAX;
        bx[3] = bx[4] = bx[5] = -FLT_MAX;
      }
      s_ref[me] = lane < count ? ref : kSentinel;
#pragma unroll
      for (int k = 0; k < 6; ++k) s_box[k][me] = bx[k];
      __syncwarp();
      bool failed = false;
      while (count > threshold) {
        const bool act = lane < count;
        if (act) {
          ref = s_ref[me];
#pragma unroll
          for (int k = 0; k < 6; ++k) bx[k] = s_box[k][me];
        }
        s_key[me] = ~0ull;
        __syncwarp();
        if (act) {
          unsigned long long own = ~0ull;
          const int last = min(lane + kRadius, count - 1);
          for (int j = lane + 1; j <= last; ++j) {
            float m[6];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              m[k] = fminf(bx[k], s_box[k][wbase + j]);
              m[3 + k] = fmaxf(bx[3 + k], s_box[3 + k][wbase + j]);
            }
            const unsigned long long bits = (unsigned long long)__float_as_uint(area6(m)) << 32;
            own = min(own, bits | enc_off(lane, j));
            atomicMin(s_key + wbase + j, bits | enc_off(j, lane));
          }
          atomicMin(s_key + me, own);
        }
        __syncwarp();
        int nearest = 32;
        bool mutual = false;
        if (act) {
          nearest = dec_off(lane, (uint32_t)s_key[me]);
          mutual = dec_off(nearest, (uint32_t)s_key[wbase + nearest]) == lane;
        }
        const bool merge = mutual && lane < nearest;
        const uint32_t mmask = __ballot_sync(kFull, merge);
        if (mmask == 0) {
          if (lane == 0) raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
          failed = true;
          break;
        }
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(w.counters + t_seg, (uint32_t)__popc(mmask));
        base = __shfl_sync(kFull, base, 0);
        uint32_t out = kSentinel;
        float obx[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) obx[k] = bx[k];
        if (merge) {
          const uint32_t nref = s_ref[wbase + nearest];
          float nbx[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) nbx[k] = s_box[k][wbase + nearest];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            obx[k] = fminf(bx[k], nbx[k]);
            obx[3 + k] = fmaxf(bx[3 + k], nbx[3 + k]);
          }
          const uint32_t node = internal_offsets[t_seg] + base + (uint32_t)__popc(mmask & ((1u << lane) - 1u));
          if (node < internal_offsets[t_seg + 1]) {
            float* nb = node_bounds + (size_t)node * 12;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
              nb[k] = bx[k];
              nb[6 + k] = nbx[k];
              w.boxes[(size_t)node * 6 + k] = obx[k];
            }
            *reinterpret_cast<uint4*>(node_meta + (size_t)node * 4) = make_uint4(kSentinel, ref, nref, kSentinel);
            node_flags[node] = 2u;
            const uint32_t lc = ((ref & kLeafFlag) ? 1u : __ldcg(node_leaf_counts + (ref & kIndexMask))) +
                                ((nref & kLeafFlag) ? 1u : __ldcg(node_leaf_counts + (nref & kIndexMask)));
            node_leaf_counts[node] = lc;
            if (ref & kLeafFlag) leaf_parent[ref & kIndexMask] = node;
            else node_meta[(size_t)(ref & kIndexMask) * 4] = node;
            if (nref & kLeafFlag) leaf_parent[nref & kIndexMask] = node;
            else node_meta[(size_t)(nref & kIndexMask) * 4] = node;
            out = node;
          } else {
            raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
          }
        } else if (act && !mutual) {
          out = ref;
        }
        const bool keep = out != kSentinel;
        const uint32_t kmask = __ballot_sync(kFull, keep);
        const int slot = wbase + __popc(kmask & ((1u << lane) - 1u));
        __syncwarp();
        if (keep) {
          s_ref[slot] = out;
#pragma unroll
          for (int k = 0; k < 6; ++k) s_box[k][slot] = obx[k];
        }
        __syncwarp();
        count = __popc(kmask);
        ref = lane < count ? s_ref[me] : kSentinel;
      }
      if (failed) {
        active = false;
        tasks = 0;
        break;
      }
      if (lane < before) w.clusters[t_left + lane] = ref;
      __threadfence();  // before the task's owner advertises the range at its next split
      if (t_fin && lane == 0) roots[t_seg] = ref;
      tasks &= tasks - 1;
    }
  }
}

// finalize_hploc_multi_wave_kernel (:548-572): every segment made exactly its
// internal-node count and has a root
__global__ void finalize_kernel(uint32_t n_seg, const uint32_t* __restrict__ seg_offsets,
                                const uint32_t* __restrict__ internal_offsets, Ws w,
                                const uint32_t* __restrict__ roots, uint32_t* __restrict__ status) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_seg) return;
  const uint32_t leaves = seg_offsets[s + 1] - seg_offsets[s];
  const uint32_t internal = internal_offsets[s + 1] - internal_offsets[s];
  if (leaves == 0) return;
  if (__ldcg(w.counters + s) != internal || roots[s] == kSentinel) raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
}

}  // namespace hploc

size_t hploc_workspace_bytes(uint32_t n, uint32_t n_seg) {
  const size_t N = n ? n : 1;
  auto a = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return a(N * 4) + a(N * 4) + a(N * 24) + a((size_t)n_seg * 4);
}

// the H-PLOC back end of bajo_hploc_build, after the sort: `extra` holds
// hploc_workspace_bytes(n, S)
cudaError_t launch_hploc(const float* d_verts, BajoLbvh* bvh, unsigned char* extra, uint32_t* status,
                         cudaStream_t st) {
  using namespace hploc;
  const uint32_t n = bvh->n_leaves, S = bvh->n_segments;
  const size_t N = n ? n : 1;
  auto a = [](size_t x) { return (x + 255) & ~(size_t)255; };
  Ws w;
  w.slots = (uint32_t*)extra;
  w.clusters = (uint32_t*)(extra + a(N * 4));
  w.boxes = (float*)(extra + a(N * 4) * 2);
  w.counters = (uint32_t*)(extra + a(N * 4) * 2 + a(N * 24));
  const uint32_t items = n > S ? n : S;
  init_kernel<<<(items + kBlock - 1) / kBlock, kBlock, 0, st>>>(n, bvh->seg_offsets, S, bvh->leaf_ids, d_verts, w,
                                                               bvh->leaf_parent, bvh->roots, bvh->leaf_tris, status);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (n > 1) {
    build_kernel<<<(n + kBlock - 1) / kBlock, kBlock, 0, st>>>(
        n, bvh->morton_codes, bvh->seg_offsets, S, bvh->internal_offsets, bvh->leaf_bounds, bvh->leaf_ids, w,
        bvh->node_meta, bvh->node_bounds, bvh->node_flags, bvh->node_leaf_counts, bvh->leaf_parent, bvh->roots,
        status);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  finalize_kernel<<<(S + 255) / 256, 256, 0, st>>>(S, bvh->seg_offsets, bvh->internal_offsets, w, bvh->roots, status);
  return cudaGetLastError();
}

}  // namespace bajo
