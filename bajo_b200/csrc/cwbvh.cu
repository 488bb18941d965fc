// cwbvh.cu -- closest-hit / any-hit traversal of the compressed 8-wide BVH
// (CWBVH8; Ylitie, Karras, Laine, HPG 2017) that bajo_cwbvh8_build encodes.
//
// Restates trace_cwbvh8_triangles (bajo/bvh/gpu/triangle_bvh.mojo:1010-1104)
// with the node decode of _intersect_cwbvh8_node_tasks
// (bajo/bvh/gpu/compressed_bounds_bvh.mojo:469-576) and the record test of
// _intersect_cwbvh_triangle (triangle_bvh.mojo:962-1007):
//  - a node group is (base, mask): bits 24..31 of the mask are the hit
//    internal children (slot + 24, the slot XOR the inverted ray octant) and
//    bits 0..7 the node's imask, from which a child's rank among the node's
//    consecutive internal children is a popcount; a triangle group holds the
//    hit triangles in bits 0..23 relative to the node's first triangle;
//  - both are consumed highest bit first; a node group with children left is
//    pushed before its next child is opened, and the triangles of a node are
//    tested as soon as the node is decoded;
//  - a lane's box is p + q * 2^(e - 127) per axis, tested with fma against
//    the ray's reciprocal (rcp_direction: +-1e9 where |d| <= 1e-9) over
//    [max(t near, 0), min(t far, t)]; max / min are fmaxf / fminf, which
//    agree with the reference's select form (bajo/core/utils.mojo:60-70)
//    unless an operand is NaN;
//  - the lane bytes are split four at a time into bit positions and child
//    bits (the node's hit mask is the reference's, bit for bit);
//  - triangles use the determinant-scaled Moller-Trumbore test
//    (intersect_ray_tri_edges_scaled, bajo/core/intersect.mojo:462-505) with
//    the current hit distance as t_max, so the first of equal-distance
//    candidates in visiting order is kept, as in the reference.
// Every node costs five 16-byte loads, every triangle three; the quantized
// planes are turned into floats exactly (2^23 + q - 2^23).
#include "cwbvh.cuh"

namespace bajo {
namespace cw {

__device__ __forceinline__ void store(const Hit& h, const Tree& tr, uint32_t i, float* __restrict__ hits8,
                                      float* __restrict__ out_t, uint32_t* __restrict__ out_prim) {
  if (hits8) {
    f3 n = mk(0.0f, 0.0f, 0.0f);
    if (h.tri != kEmpty) {
      const float4 a = __ldg(tr.tris + (size_t)h.tri * 3 + 0), b = __ldg(tr.tris + (size_t)h.tri * 3 + 1);
      n = normalize(cross(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z)));
    }
    float4* w = reinterpret_cast<float4*>(hits8 + (size_t)i * 8);
    w[0] = make_float4(h.u, h.v, __uint_as_float(h.prim), __uint_as_float(kEmpty));
    w[1] = make_float4(n.x, n.y, n.z, h.t);
  }
  if (out_t) out_t[i] = h.t;
  if (out_prim) out_prim[i] = h.prim;
}

template <bool ANY>
__global__ void __launch_bounds__(kBlock) rays_kernel(const float* __restrict__ rays, uint32_t n, Tree tr,
                                                      float* __restrict__ hits8, float* __restrict__ out_t,
                                                      uint32_t* __restrict__ out_prim, uint32_t* __restrict__ status) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const f3 o = mk(rays[i], rays[(size_t)n + i], rays[2 * (size_t)n + i]);
  const f3 d = mk(rays[4 * (size_t)n + i], rays[5 * (size_t)n + i], rays[6 * (size_t)n + i]);
  const Hit h = trace<ANY>(o, d, rays[3 * (size_t)n + i], rays[7 * (size_t)n + i], tr, status);
  store(h, tr, i, hits8, out_t, out_prim);
}

// camera rays as the other trace kernels (_camera_ray, camera_launch.mojo:34;
// make_ray_raster, bajo/bvh/camera.mojo:137), t in [0, FLT_MAX]
template <bool ANY>
__global__ void __launch_bounds__(kBlock) camera_kernel(const float* __restrict__ cams, uint32_t n, uint32_t width,
                                                        uint32_t height, float inv_h, Tree tr,
                                                        float* __restrict__ hits8, float* __restrict__ out_t,
                                                        uint32_t* __restrict__ out_prim,
                                                        uint32_t* __restrict__ status) {
  uint32_t i;  // every warp an 8 x 4 pixel tile (trav::tile_ray)
  if (!trav::tile_ray((uint64_t)blockIdx.x * kBlock + threadIdx.x, n, width, height, i)) return;
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
  const Hit h = trace<ANY>(mk(__ldg(c + 0), __ldg(c + 1), __ldg(c + 2)), dir, 0.0f, FLT_MAX, tr, status);
  store(h, tr, i, hits8, out_t, out_prim);
}

bool make_tree(const BajoCwbvh8* c, uint32_t n_nodes, Tree& tr) {
  if (!c || !c->nodes || !c->triangles) return false;
  if ((reinterpret_cast<uintptr_t>(c->nodes) | reinterpret_cast<uintptr_t>(c->triangles)) & 15u) return false;
  tr.nodes = reinterpret_cast<const float4*>(c->nodes);
  tr.tris = reinterpret_cast<const float4*>(c->triangles);
  tr.n_nodes = n_nodes;
  tr.n_tris = c->n_tris;
  return true;
}

}  // namespace cw
}  // namespace bajo

extern "C" {

int32_t bajo_trace_cwbvh8_rays(const BajoCwbvh8* c, uint32_t n_nodes, const float* d_rays, uint32_t n,
                               int32_t any_hit, float* d_hits8, float* d_t, uint32_t* d_prim, uint32_t* d_status,
                               void* stream) {
  using namespace bajo::cw;
  Tree tr;
  if (!make_tree(c, n_nodes, tr) || (n && !d_rays) || (any_hit != 0 && any_hit != 1) || !d_status)
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t grid = (n + kBlock - 1) / kBlock;
  if (any_hit) rays_kernel<true><<<grid, kBlock, 0, st>>>(d_rays, n, tr, d_hits8, d_t, d_prim, d_status);
  else rays_kernel<false><<<grid, kBlock, 0, st>>>(d_rays, n, tr, d_hits8, d_t, d_prim, d_status);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_cwbvh8_camera(const BajoCwbvh8* c, uint32_t n_nodes, const float* d_cameras, uint32_t n,
                                 uint32_t width, uint32_t height, int32_t any_hit, float* d_hits8, float* d_t,
                                 uint32_t* d_prim, uint32_t* d_status, void* stream) {
  using namespace bajo::cw;
  Tree tr;
  if (!make_tree(c, n_nodes, tr) || !d_cameras || width == 0 || height == 0 || (any_hit != 0 && any_hit != 1) ||
      !d_status)
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t grid = (uint32_t)((bajo::trav::camera_threads(n, width, height) + kBlock - 1) / kBlock);
  const float inv_h = 1.0f / (float)height;
  if (any_hit)
    camera_kernel<true><<<grid, kBlock, 0, st>>>(d_cameras, n, width, height, inv_h, tr, d_hits8, d_t, d_prim,
                                                 d_status);
  else
    camera_kernel<false><<<grid, kBlock, 0, st>>>(d_cameras, n, width, height, inv_h, tr, d_hits8, d_t, d_prim,
                                                  d_status);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

}  // extern "C"
