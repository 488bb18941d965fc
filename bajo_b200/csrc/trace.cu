// trace.cu -- closest-hit traversal entry points (GpuTriangleBvh.launch_rays /
// launch_camera, bajo/bvh/gpu/triangle_bvh.mojo:520-614).  The traversal
// itself is in traverse.cuh.
#include <atomic>
#include <mutex>

#include "sampling.cuh"
#include "traverse.cuh"

namespace bajo {
int sm_count();
namespace {

using namespace trav;

__device__ __forceinline__ void store_hit(const Hit& h, const float4* __restrict__ tris, uint32_t i,
                                          float* __restrict__ hits8, float* __restrict__ out_t,
                                          uint32_t* __restrict__ out_prim) {
  if (hits8) {
    f3 n = mk(0.0f, 0.0f, 0.0f);
    if (h.leaf != kEmpty) {
      const float4 a = __ldg(tris + (size_t)h.leaf * 3 + 0);
      const float4 b = __ldg(tris + (size_t)h.leaf * 3 + 1);
      const float4 c = __ldg(tris + (size_t)h.leaf * 3 + 2);
      f3 v0 = mk(a.x, a.y, a.z);
      n = normalize(cross(mk(b.x, b.y, b.z) - v0, mk(c.x, c.y, c.z) - v0));
    }
    float4* o = reinterpret_cast<float4*>(hits8 + (size_t)i * 8);
    o[0] = make_float4(h.u, h.v, __uint_as_float(h.prim), __uint_as_float(kEmpty));
    o[1] = make_float4(n.x, n.y, n.z, h.t);
  }
  if (out_t) out_t[i] = h.t;
  if (out_prim) out_prim[i] = h.prim;
}

// Kernels with TOP read the staged top levels from shared memory; they run
// one persistent block per resident slot (kTopBlock threads, grid-stride over
// the rays) so that each block copies the records once.
constexpr int kTopBlock = 512;
constexpr int kTopMinBlocks = 2;  // 64 registers: as many warps per SM as the 128-thread kernels

template <bool TOP>
struct StageSmem {
  using type = char;
};
template <>
struct StageSmem<true> {
  using type = TopSmem;
};

template <int MODE, bool TOP, int STACK = kStack>
__device__ __forceinline__ void ray_query(uint32_t i, const float* __restrict__ rays, uint32_t n, uint32_t n_nodes,
                                          uint32_t root, const float4* __restrict__ nb,
                                          const uint4* __restrict__ meta, const float4* __restrict__ tris,
                                          const float4* top, float* __restrict__ hits8, float* __restrict__ out_t,
                                          uint32_t* __restrict__ out_prim, uint32_t* __restrict__ status) {
  // field-major ray planes (ray_launch.mojo:95-112)
  f3 o = mk(rays[i], rays[(size_t)n + i], rays[2 * (size_t)n + i]);
  float tmin = rays[3 * (size_t)n + i];
  f3 d = mk(rays[4 * (size_t)n + i], rays[5 * (size_t)n + i], rays[6 * (size_t)n + i]);
  float tmax = rays[7 * (size_t)n + i];
  Ray r = make_ray(o, d, tmin, tmax);
  Hit h;
  if constexpr (TOP) h = trace_bvh2_top<MODE>(r, root, nb, meta, tris, n_nodes, status, top);
  else h = trace_bvh2<MODE, false, false, STACK>(r, root, nb, meta, tris, n_nodes, status);
  store_hit(h, tris, i, hits8, out_t, out_prim);
}

// Unstaged: 10 blocks of 128 per SM (48 registers): general rays are mostly
// incoherent and latency bound, and the extra warps outweigh the spills
// (+5% to +8% on random rays against 64 registers).
template <int MODE, bool TOP, int BLK = kTraceBlock, int STACK = kStack>
__global__ void __launch_bounds__(TOP ? kTopBlock : BLK, TOP ? kTopMinBlocks : 1280 / BLK)
    trace_rays_kernel(const float* __restrict__ rays, uint32_t n, uint32_t n_nodes, const uint32_t* __restrict__ roots,
                      const float4* __restrict__ nb, const uint4* __restrict__ meta, const float4* __restrict__ tris,
                      const float4* __restrict__ top_g, float* __restrict__ hits8, float* __restrict__ out_t,
                      uint32_t* __restrict__ out_prim, uint32_t* __restrict__ status) {
  __shared__ typename StageSmem<TOP>::type sm;
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (TOP) {
    const uint32_t root = __ldg(roots);
    const float4* top = stage_top(sm, top_g, root, status);
    for (uint32_t i = i0; i < n; i += gridDim.x * blockDim.x)
      ray_query<MODE, TOP>(i, rays, n, n_nodes, root, nb, meta, tris, top, hits8, out_t, out_prim, status);
    stage_top_drain(sm, top);
  } else if (i0 < n) {
    ray_query<MODE, TOP, STACK>(i0, rays, n, n_nodes, __ldg(roots), nb, meta, tris, nullptr, hits8, out_t, out_prim,
                                status);
  }
}

// camera.mojo:137-154 make_ray_raster; camera_launch.mojo:34-55.  With STATS
// it also writes per-ray [node visits, triangle tests] like the reference's
// instrumented kernel (triangle_bvh.mojo:813, GpuTraversalStats trace.mojo:62).
template <int MODE, bool STATS, bool TOP, int STACK = kStack>
__device__ __forceinline__ void camera_ray(uint32_t i, const float* __restrict__ cams, uint32_t n_nodes,
                                           uint32_t width, uint32_t height, float inv_h, uint32_t root,
                                           const float4* __restrict__ nb, const uint4* __restrict__ meta,
                                           const float4* __restrict__ tris, const float4* top,
                                           float* __restrict__ hits8, float* __restrict__ out_t,
                                           uint32_t* __restrict__ out_prim, uint32_t* __restrict__ status,
                                           uint32_t* __restrict__ stats) {
  const uint32_t ppv = width * height;
  const uint32_t view = i / ppv, local = i - view * ppv;
  const float* c = cams + (size_t)view * 20;
  const uint32_t px = local % width, py = local / width;
  const float sx = (2.0f * ((float)px + 0.5f) - (float)width) * inv_h;
  const float sy = 1.0f - 2.0f * ((float)py + 0.5f) * inv_h;
  const float fs = __ldg(c + 12);
  f3 fwd = mk(__ldg(c + 3), __ldg(c + 4), __ldg(c + 5));
  f3 right = mk(__ldg(c + 6), __ldg(c + 7), __ldg(c + 8));
  f3 up = mk(__ldg(c + 9), __ldg(c + 10), __ldg(c + 11));
  f3 dir = normalize((fwd + right * (sx * fs)) + up * (sy * fs));
  Ray r = make_ray(mk(__ldg(c + 0), __ldg(c + 1), __ldg(c + 2)), dir, 0.0f, FLT_MAX);
  uint32_t st[kStatWords] = {0, 0, 0, 0, 0};
  Hit h;
  if constexpr (TOP) h = trace_bvh2_top<MODE, STATS>(r, root, nb, meta, tris, n_nodes, status, top, st);
  else h = trace_bvh2<MODE, STATS, false, STACK>(r, root, nb, meta, tris, n_nodes, status, st);
  store_hit(h, tris, i, hits8, out_t, out_prim);
  if constexpr (STATS) {
#pragma unroll
    for (int k = 0; k < kStatWords; ++k) stats[(size_t)i * kStatWords + k] = st[k];
  }
}

template <int MODE, bool STATS, bool TOP, int BLK = kTraceBlock, int STACK = kStack>
__global__ void __launch_bounds__(TOP ? kTopBlock : BLK, TOP ? kTopMinBlocks : 0)
    trace_camera_kernel(const float* __restrict__ cams, uint32_t n, uint32_t n_nodes, uint32_t width, uint32_t height,
                        float inv_h, const uint32_t* __restrict__ roots, const float4* __restrict__ nb,
                        const uint4* __restrict__ meta, const float4* __restrict__ tris,
                        const float4* __restrict__ top_g, float* __restrict__ hits8, float* __restrict__ out_t,
                        uint32_t* __restrict__ out_prim, uint32_t* __restrict__ status,
                        uint32_t* __restrict__ stats) {
  __shared__ typename StageSmem<TOP>::type sm;
  const uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (TOP) {
    const uint32_t root = __ldg(roots);
    const float4* top = stage_top(sm, top_g, root, status);
    for (uint32_t i = i0; i < n; i += gridDim.x * blockDim.x)
      camera_ray<MODE, STATS, TOP>(i, cams, n_nodes, width, height, inv_h, root, nb, meta, tris, top, hits8, out_t,
                                   out_prim, status, stats);
    stage_top_drain(sm, top);
  } else {
    uint32_t i;
    if (tile_ray((uint64_t)blockIdx.x * blockDim.x + threadIdx.x, n, width, height, i))
      camera_ray<MODE, STATS, TOP, STACK>(i, cams, n_nodes, width, height, inv_h, __ldg(roots), nb, meta, tris,
                                          nullptr, hits8, out_t, out_prim, status, stats);
  }
}

// Batched closest hits over a segmented LBVH: ray i belongs to scene
// i / (width * height), starts at that scene's camera (cam_stride floats
// apart; 0 = one shared camera) and is traced against that scene's root.  A
// primary hit spawns one cosine-weighted bounce ray about the geometric normal
// oriented against the ray (the Lambertian sample of bajo/rt/shading.mojo:92,
// Philox stream (ray, stage 1)).  Misses report t = FLT_MAX / prim = EMPTY.
template <int MODE>
__global__ void __launch_bounds__(kTraceBlock) batch_trace_kernel(
    const float* __restrict__ cams, uint32_t cam_stride, uint32_t n, uint32_t n_nodes, uint32_t width,
    uint32_t height, float inv_h, const uint32_t* __restrict__ roots, const float4* __restrict__ nb,
    const uint4* __restrict__ meta, const float4* __restrict__ tris, uint64_t seed, float* __restrict__ t0,
    uint32_t* __restrict__ p0, float* __restrict__ t1, uint32_t* __restrict__ p1, uint32_t* __restrict__ status) {
  const uint32_t ppv = width * height;
  // every warp an 8 x 4 pixel tile of one scene's image (tile_ray)
  const uint64_t threads = camera_threads(n, width, height);
  for (uint64_t g = (uint64_t)blockIdx.x * kTraceBlock + threadIdx.x; g < threads;
       g += (uint64_t)gridDim.x * kTraceBlock) {
    uint32_t i;
    if (!tile_ray(g, n, width, height, i)) continue;
    const uint32_t view = i / ppv, local = i - view * ppv;
    const float* c = cams + (size_t)view * cam_stride;
    const uint32_t px = local % width, py = local / width;
    const float sx = (2.0f * ((float)px + 0.5f) - (float)width) * inv_h;
    const float sy = 1.0f - 2.0f * ((float)py + 0.5f) * inv_h;
    const float fs = __ldg(c + 12);
    const f3 fwd = mk(__ldg(c + 3), __ldg(c + 4), __ldg(c + 5));
    const f3 right = mk(__ldg(c + 6), __ldg(c + 7), __ldg(c + 8));
    const f3 up = mk(__ldg(c + 9), __ldg(c + 10), __ldg(c + 11));
    const f3 d = normalize((fwd + right * (sx * fs)) + up * (sy * fs));
    const f3 o = mk(__ldg(c + 0), __ldg(c + 1), __ldg(c + 2));
    const uint32_t root = __ldg(roots + view);
    const Hit h = trace_bvh2<MODE>(make_ray(o, d, 0.0f, FLT_MAX), root, nb, meta, tris, n_nodes, status);
    t0[i] = h.t;
    p0[i] = h.prim;
    float bt = FLT_MAX;
    uint32_t bp = kEmpty;
    if (h.leaf != kEmpty) {
      const float4 a = __ldg(tris + (size_t)h.leaf * 3 + 0);
      const float4 b = __ldg(tris + (size_t)h.leaf * 3 + 1);
      const float4 e = __ldg(tris + (size_t)h.leaf * 3 + 2);
      const f3 v0 = mk(a.x, a.y, a.z);
      const f3 outward = normalize(cross(mk(b.x, b.y, b.z) - v0, mk(e.x, e.y, e.z) - v0));
      const f3 normal = dot(d, outward) < 0.0f ? outward : mk(-outward.x, -outward.y, -outward.z);
      const float4 u = smp::uniform4(seed, i, smp::stage_bsdf(0));
      const f3 dir = smp::lambertian_dir(normal, u.x, u.y);
      const f3 p = mk(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
      const Hit h2 = trace_bvh2<MODE>(make_ray(p, dir, 0.001f, FLT_MAX), root, nb, meta, tris, n_nodes, status);
      bt = h2.t;
      bp = h2.prim;
    }
    t1[i] = bt;
    p1[i] = bp;
  }
}

bool bvh_ok(const BajoLbvh* b) {
  return b && b->roots && b->node_bounds && b->node_meta && b->leaf_tris && b->n_segments >= 1 &&
         !((uintptr_t)b->top_nodes & 15) && !((uintptr_t)b->node_bounds & 15) && !((uintptr_t)b->node_meta & 15) &&
         !((uintptr_t)b->leaf_tris & 15);  // records read 16 bytes at a time
}

// Grid of a TOP kernel: every resident block slot once, at most one ray per
// thread.
template <typename Kernel>
uint32_t top_grid(Kernel kernel, uint32_t n) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTopBlock, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const uint32_t cap = (uint32_t)per_sm * (uint32_t)sm_count();
  const uint32_t need = (n + kTopBlock - 1) / kTopBlock;
  return need < cap ? need : cap;
}

// Block sizes of the unstaged closest-hit kernels, chosen per call from a
// process-wide table indexed by (kind: 0 camera rays, 1 general rays,
// ceil(log2 n)) that the autotuner fills (bajo_trace_tuning_set); -1 means
// the built-in 128.  The block size changes only the launch shape: every
// variant gives the same hits.
constexpr int kTraceVariants = 3;
constexpr int kTraceBlocks[kTraceVariants] = {128, 64, 256};
std::atomic<int8_t> g_trace_tuning[2][33];
std::once_flag g_trace_tuning_once;

int trace_variant(int kind, uint32_t n) {
  std::call_once(g_trace_tuning_once, [] {
    for (auto& row : g_trace_tuning)
      for (auto& v : row) v.store(-1);
  });
  uint32_t lg = 0;
  while (lg < 32 && (1ull << lg) < n) ++lg;
  const int v = g_trace_tuning[kind][lg].load(std::memory_order_relaxed);
  return v >= 0 && v < kTraceVariants ? v : 0;
}

// Traversal stack depths of the same kernels, from a second table of the
// same shape (bajo_trace_stack_tuning_set); -1 means kStack (64).  A
// shallower stack keeps the traversal's local-memory footprint small; a ray
// that needs more entries is traced again with kStack, so every depth gives
// the same hits.  24 is the reference's GPU_STACK_SIZE
// (bajo/bvh/constants.mojo:16).
constexpr int kStackVariants = 3;
constexpr int kTraceStacks[kStackVariants] = {kStack, 24, 12};
std::atomic<int8_t> g_stack_tuning[2][33];
std::once_flag g_stack_tuning_once;

int stack_variant(int kind, uint32_t n) {
  std::call_once(g_stack_tuning_once, [] {
    for (auto& row : g_stack_tuning)
      for (auto& v : row) v.store(-1);
  });
  uint32_t lg = 0;
  while (lg < 32 && (1ull << lg) < n) ++lg;
  const int v = g_stack_tuning[kind][lg].load(std::memory_order_relaxed);
  return v >= 0 && v < kStackVariants ? v : 0;
}

template <int MODE, bool TOP, int BLK, int STACK = kStack>
void launch_rays_blk(const BajoLbvh* b, const float* rays, uint32_t n, float* hits8, float* t, uint32_t* prim,
                     uint32_t* status, cudaStream_t st) {
  const float4* nb = reinterpret_cast<const float4*>(b->node_bounds);
  const uint4* meta = reinterpret_cast<const uint4*>(b->node_meta);
  const float4* tris = reinterpret_cast<const float4*>(b->leaf_tris);
  const float4* top = reinterpret_cast<const float4*>(b->top_nodes);
  const uint32_t grid = TOP ? top_grid(trace_rays_kernel<MODE, TOP>, n) : (n + BLK - 1) / BLK;
  trace_rays_kernel<MODE, TOP, BLK, STACK><<<grid, TOP ? kTopBlock : BLK, 0, st>>>(
      rays, n, b->n_leaves, b->roots, nb, meta, tris, top, hits8, t, prim, status);
}

template <int MODE, int BLK>
void launch_rays_stack(const BajoLbvh* b, const float* rays, uint32_t n, float* hits8, float* t, uint32_t* prim,
                       uint32_t* status, cudaStream_t st) {
  switch (stack_variant(1, n)) {
    case 1: return launch_rays_blk<MODE, false, BLK, 24>(b, rays, n, hits8, t, prim, status, st);
    case 2: return launch_rays_blk<MODE, false, BLK, 12>(b, rays, n, hits8, t, prim, status, st);
    default: return launch_rays_blk<MODE, false, BLK, kStack>(b, rays, n, hits8, t, prim, status, st);
  }
}

template <int MODE, bool TOP>
void launch_rays(const BajoLbvh* b, const float* rays, uint32_t n, float* hits8, float* t, uint32_t* prim,
                 uint32_t* status, cudaStream_t st) {
  if constexpr (TOP) {
    launch_rays_blk<MODE, TOP, kTraceBlock>(b, rays, n, hits8, t, prim, status, st);
  } else {
    switch (trace_variant(1, n)) {
      case 1: return launch_rays_stack<MODE, 64>(b, rays, n, hits8, t, prim, status, st);
      case 2: return launch_rays_stack<MODE, 256>(b, rays, n, hits8, t, prim, status, st);
      default: return launch_rays_stack<MODE, 128>(b, rays, n, hits8, t, prim, status, st);
    }
  }
}

template <int MODE, bool STATS, bool TOP, int BLK, int STACK = kStack>
void launch_camera_blk(const BajoLbvh* b, const float* cams, uint32_t n, uint32_t width, uint32_t height,
                       float* hits8, float* t, uint32_t* prim, uint32_t* status, uint32_t* stats, cudaStream_t st) {
  const float4* nb = reinterpret_cast<const float4*>(b->node_bounds);
  const uint4* meta = reinterpret_cast<const uint4*>(b->node_meta);
  const float4* tris = reinterpret_cast<const float4*>(b->leaf_tris);
  const float4* top = reinterpret_cast<const float4*>(b->top_nodes);
  const float inv_h = 1.0f / (float)height;
  // unstaged: 32 threads per 8 x 4 tile of every view
  const uint64_t threads = camera_threads(n, width, height);
  const uint32_t grid = TOP ? top_grid(trace_camera_kernel<MODE, STATS, TOP>, n) : (uint32_t)((threads + BLK - 1) / BLK);
  trace_camera_kernel<MODE, STATS, TOP, BLK, STACK><<<grid, TOP ? kTopBlock : BLK, 0, st>>>(
      cams, n, b->n_leaves, width, height, inv_h, b->roots, nb, meta, tris, top, hits8, t, prim, status, stats);
}

template <int MODE, int BLK>
void launch_camera_stack(const BajoLbvh* b, const float* cams, uint32_t n, uint32_t width, uint32_t height,
                         float* hits8, float* t, uint32_t* prim, uint32_t* status, cudaStream_t st) {
  switch (stack_variant(0, n)) {
    case 1:
      return launch_camera_blk<MODE, false, false, BLK, 24>(b, cams, n, width, height, hits8, t, prim, status,
                                                            nullptr, st);
    case 2:
      return launch_camera_blk<MODE, false, false, BLK, 12>(b, cams, n, width, height, hits8, t, prim, status,
                                                            nullptr, st);
    default:
      return launch_camera_blk<MODE, false, false, BLK, kStack>(b, cams, n, width, height, hits8, t, prim, status,
                                                                nullptr, st);
  }
}

template <int MODE, bool STATS, bool TOP>
void launch_camera(const BajoLbvh* b, const float* cams, uint32_t n, uint32_t width, uint32_t height, float* hits8,
                   float* t, uint32_t* prim, uint32_t* status, uint32_t* stats, cudaStream_t st) {
  if constexpr (TOP || STATS) {
    launch_camera_blk<MODE, STATS, TOP, kTraceBlock>(b, cams, n, width, height, hits8, t, prim, status, stats, st);
  } else {
    switch (trace_variant(0, n)) {
      case 1: return launch_camera_stack<MODE, 64>(b, cams, n, width, height, hits8, t, prim, status, st);
      case 2: return launch_camera_stack<MODE, 256>(b, cams, n, width, height, hits8, t, prim, status, st);
      default: return launch_camera_stack<MODE, 128>(b, cams, n, width, height, hits8, t, prim, status, st);
    }
  }
}

template <bool STATS>
void launch_camera_any(const BajoLbvh* b, int32_t mode, const float* cams, uint32_t n, uint32_t width,
                       uint32_t height, float* hits8, float* t, uint32_t* prim, uint32_t* status, uint32_t* stats,
                       cudaStream_t st) {
  const bool top = b->top_nodes != nullptr;
  if (mode == BAJO_TRI_MT) {
    if (top) launch_camera<BAJO_TRI_MT, STATS, true>(b, cams, n, width, height, hits8, t, prim, status, stats, st);
    else launch_camera<BAJO_TRI_MT, STATS, false>(b, cams, n, width, height, hits8, t, prim, status, stats, st);
  } else {
    if (top)
      launch_camera<BAJO_TRI_WATERTIGHT, STATS, true>(b, cams, n, width, height, hits8, t, prim, status, stats, st);
    else
      launch_camera<BAJO_TRI_WATERTIGHT, STATS, false>(b, cams, n, width, height, hits8, t, prim, status, stats, st);
  }
}

}  // namespace
}  // namespace bajo

extern "C" {

int32_t bajo_trace_rays(const BajoLbvh* bvh, const float* d_rays, uint32_t n, int32_t mode, float* d_hits8,
                        float* d_t, uint32_t* d_prim, uint32_t* d_status, void* stream) {
  using namespace bajo;
  if (!bvh_ok(bvh) || (n && !d_rays) || (mode != BAJO_TRI_MT && mode != BAJO_TRI_WATERTIGHT))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const bool top = bvh->top_nodes != nullptr;
  if (mode == BAJO_TRI_MT) {
    if (top) launch_rays<BAJO_TRI_MT, true>(bvh, d_rays, n, d_hits8, d_t, d_prim, d_status, st);
    else launch_rays<BAJO_TRI_MT, false>(bvh, d_rays, n, d_hits8, d_t, d_prim, d_status, st);
  } else {
    if (top) launch_rays<BAJO_TRI_WATERTIGHT, true>(bvh, d_rays, n, d_hits8, d_t, d_prim, d_status, st);
    else launch_rays<BAJO_TRI_WATERTIGHT, false>(bvh, d_rays, n, d_hits8, d_t, d_prim, d_status, st);
  }
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_tuning_set(int32_t kind, uint32_t log2n, int32_t block) {
  using namespace bajo;
  if ((kind != 0 && kind != 1) || log2n > 32) return BAJO_ERR_INVALID_ARGUMENT;
  int v = -1;
  for (int k = 0; k < kTraceVariants; ++k)
    if (kTraceBlocks[k] == block) v = k;
  if (block != 0 && v < 0) return BAJO_ERR_INVALID_ARGUMENT;
  trace_variant(0, 1);  // initialise the table
  g_trace_tuning[kind][log2n].store((int8_t)v);
  return BAJO_OK;
}

int32_t bajo_trace_tuning_get(int32_t kind, uint32_t n, int32_t* block) {
  using namespace bajo;
  if ((kind != 0 && kind != 1) || !block) return BAJO_ERR_INVALID_ARGUMENT;
  *block = kTraceBlocks[trace_variant(kind, n)];
  return BAJO_OK;
}

int32_t bajo_trace_stack_tuning_set(int32_t kind, uint32_t log2n, int32_t depth) {
  using namespace bajo;
  if ((kind != 0 && kind != 1) || log2n > 32) return BAJO_ERR_INVALID_ARGUMENT;
  int v = -1;
  for (int k = 0; k < kStackVariants; ++k)
    if (kTraceStacks[k] == depth) v = k;
  if (depth != 0 && v < 0) return BAJO_ERR_INVALID_ARGUMENT;
  stack_variant(0, 1);  // initialise the table
  g_stack_tuning[kind][log2n].store((int8_t)v);
  return BAJO_OK;
}

int32_t bajo_trace_stack_tuning_get(int32_t kind, uint32_t n, int32_t* depth) {
  using namespace bajo;
  if ((kind != 0 && kind != 1) || !depth) return BAJO_ERR_INVALID_ARGUMENT;
  *depth = kTraceStacks[stack_variant(kind, n)];
  return BAJO_OK;
}

int32_t bajo_trace_camera(const BajoLbvh* bvh, const float* d_cams, uint32_t n, uint32_t width, uint32_t height,
                          int32_t mode, float* d_hits8, float* d_t, uint32_t* d_prim, uint32_t* d_status,
                          void* stream) {
  using namespace bajo;
  if (!bvh_ok(bvh) || (n && !d_cams) || width == 0 || height == 0 ||
      (mode != BAJO_TRI_MT && mode != BAJO_TRI_WATERTIGHT))
    return BAJO_ERR_INVALID_ARGUMENT;
  if ((uint64_t)width * height > 0xFFFFFFFFull) return BAJO_ERR_TOO_LARGE;
  if (n == 0) return BAJO_OK;
  launch_camera_any<false>(bvh, mode, d_cams, n, width, height, d_hits8, d_t, d_prim, d_status, nullptr,
                           (cudaStream_t)stream);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_batch(const BajoLbvh* bvh, const float* d_cams, uint32_t cam_stride, uint32_t width,
                         uint32_t height, uint64_t seed, int32_t mode, float* d_t0, uint32_t* d_prim0, float* d_t1,
                         uint32_t* d_prim1, uint32_t* d_status, void* stream) {
  using namespace bajo;
  if (!bvh_ok(bvh) || !d_cams || !d_t0 || !d_prim0 || !d_t1 || !d_prim1 || width == 0 || height == 0 ||
      (cam_stride != 0 && cam_stride < 20) || (mode != BAJO_TRI_MT && mode != BAJO_TRI_WATERTIGHT))
    return BAJO_ERR_INVALID_ARGUMENT;
  const uint64_t n64 = (uint64_t)bvh->n_segments * width * height;
  if (n64 > 0xFFFFFFFFull) return BAJO_ERR_TOO_LARGE;
  const uint32_t n = (uint32_t)n64;
  if (n == 0) return BAJO_OK;
  const uint64_t threads = camera_threads(n, width, height);
  uint64_t grid64 = (threads + kTraceBlock - 1) / kTraceBlock;
  const uint64_t cap = (uint64_t)sm_count() * 32;
  const uint32_t grid = (uint32_t)(grid64 > cap ? cap : grid64);
  const float inv_h = 1.0f / (float)height;
  const float4* nb = reinterpret_cast<const float4*>(bvh->node_bounds);
  const uint4* meta = reinterpret_cast<const uint4*>(bvh->node_meta);
  const float4* tris = reinterpret_cast<const float4*>(bvh->leaf_tris);
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == BAJO_TRI_MT)
    batch_trace_kernel<BAJO_TRI_MT><<<grid, kTraceBlock, 0, st>>>(d_cams, cam_stride, n, bvh->n_leaves, width, height,
                                                                  inv_h, bvh->roots, nb, meta, tris, seed, d_t0,
                                                                  d_prim0, d_t1, d_prim1, d_status);
  else
    batch_trace_kernel<BAJO_TRI_WATERTIGHT><<<grid, kTraceBlock, 0, st>>>(
        d_cams, cam_stride, n, bvh->n_leaves, width, height, inv_h, bvh->roots, nb, meta, tris, seed, d_t0, d_prim0,
        d_t1, d_prim1, d_status);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_camera_stats(const BajoLbvh* bvh, const float* d_cams, uint32_t n, uint32_t width,
                                uint32_t height, int32_t mode, float* d_hits8, uint32_t* d_stats, void* stream) {
  using namespace bajo;
  if (!bvh_ok(bvh) || (n && (!d_cams || !d_stats)) || width == 0 || height == 0 ||
      (mode != BAJO_TRI_MT && mode != BAJO_TRI_WATERTIGHT))
    return BAJO_ERR_INVALID_ARGUMENT;
  if ((uint64_t)width * height > 0xFFFFFFFFull) return BAJO_ERR_TOO_LARGE;
  if (n == 0) return BAJO_OK;
  launch_camera_any<true>(bvh, mode, d_cams, n, width, height, d_hits8, nullptr, nullptr, nullptr, d_stats,
                          (cudaStream_t)stream);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

}  // extern "C"
