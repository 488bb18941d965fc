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
#include "traverse.cuh"

namespace bajo {
namespace cw {

constexpr int kBlock = 128;
constexpr int kStack = 64;  // node groups; one per level of the wide tree at most

struct Tree {
  const float4* nodes;
  const float4* tris;
  uint32_t n_nodes;  // bound on node references and visits
  uint32_t n_tris;   // bound on triangle references
};

struct Hit {
  float t, u, v;
  uint32_t prim, tri;
};

// byte b of w as an exact float: 2^23 + q (one byte permute) minus 2^23
__device__ __forceinline__ float qbyte(uint32_t w, int b) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + b)) - 8388608.0f;
}

template <bool ANY>
__device__ __forceinline__ Hit trace(f3 o, f3 d, float tmin, float tmax, const Tree& tr, uint32_t* status) {
  Hit h;
  h.t = tmax;
  h.u = h.v = 0.0f;
  h.prim = kEmpty;
  h.tri = kEmpty;
  if (tr.n_nodes == 0) return h;
  const f3 rcp = mk(trav::rcp1(d.x), trav::rcp1(d.y), trav::rcp1(d.z));
  const bool negx = d.x < 0.0f, negy = d.y < 0.0f, negz = d.z < 0.0f;
  const uint32_t oi = 7u - ((negx ? 4u : 0u) | (negy ? 2u : 0u) | (negz ? 1u : 0u));
  uint2 stack[kStack];
  int sp = 0;
  uint32_t nbase = 0, nmask = 0x80000000u, tbase = 0, tmask = 0, visits = 0;
  for (;;) {
    if (nmask > 0x00FFFFFFu) {
      const uint32_t gm = nmask;
      const int bit = 31 - __clz(nmask);
      nmask &= ~(1u << bit);
      if (nmask > 0x00FFFFFFu) {
        if (sp >= kStack) {
          raise_status(status, BAJO_STATUS_STACK_OVERFLOW);
          break;
        }
        stack[sp++] = make_uint2(nbase, nmask);
      }
      const uint32_t slot = ((uint32_t)bit - 24u) ^ oi;
      const uint32_t ni = nbase + (uint32_t)__popc(gm & ((1u << slot) - 1u));
      if (ni >= tr.n_nodes || ++visits > tr.n_nodes) {
        raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        break;
      }
      const float4* nd = tr.nodes + (size_t)ni * 5;
      const float4 n0 = __ldg(nd + 0), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3),
                   n4 = __ldg(nd + 4);
      const uint32_t ei = __float_as_uint(n0.w);
      const float idx = __uint_as_float((ei & 0xFFu) << 23) * rcp.x;
      const float idy = __uint_as_float(((ei >> 8) & 0xFFu) << 23) * rcp.y;
      const float idz = __uint_as_float(((ei >> 16) & 0xFFu) << 23) * rcp.z;
      const float ox = (n0.x - o.x) * rcp.x, oy = (n0.y - o.y) * rcp.y, oz = (n0.z - o.z) * rcp.z;
      const uint32_t imask = ei >> 24;
      const float tlim = ANY ? tmax : h.t;
      // near / far planes per axis, by the ray's direction sign
      const uint32_t q[12] = {__float_as_uint(n2.x), __float_as_uint(n2.y), __float_as_uint(n2.z),
                              __float_as_uint(n2.w), __float_as_uint(n3.x), __float_as_uint(n3.y),
                              __float_as_uint(n3.z), __float_as_uint(n3.w), __float_as_uint(n4.x),
                              __float_as_uint(n4.y), __float_as_uint(n4.z), __float_as_uint(n4.w)};
      const uint32_t meta[2] = {__float_as_uint(n1.z), __float_as_uint(n1.w)};
      uint32_t hm = 0;
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        // four lanes at once: bit position (low 5 bits, XOR the inverted
        // octant on internal lanes) and child bits (top 3 bits) of each byte
        const uint32_t inner = ((((imask >> (4 * g)) & 0xFu) * 0x00204081u) & 0x01010101u) * oi;
        const uint32_t bit4 = (meta[g] ^ inner) & 0x1F1F1F1Fu, kids4 = (meta[g] >> 5) & 0x07070707u;
        const uint32_t nxw = negx ? q[6 + g] : q[0 + g], fxw = negx ? q[0 + g] : q[6 + g];
        const uint32_t nyw = negy ? q[8 + g] : q[2 + g], fyw = negy ? q[2 + g] : q[8 + g];
        const uint32_t nzw = negz ? q[10 + g] : q[4 + g], fzw = negz ? q[4 + g] : q[10 + g];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const float tnx = __fmaf_rn(qbyte(nxw, b), idx, ox), tfx = __fmaf_rn(qbyte(fxw, b), idx, ox);
          const float tny = __fmaf_rn(qbyte(nyw, b), idy, oy), tfy = __fmaf_rn(qbyte(fyw, b), idy, oy);
          const float tnz = __fmaf_rn(qbyte(nzw, b), idz, oz), tfz = __fmaf_rn(qbyte(fzw, b), idz, oz);
          const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
          const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tlim));
          if (tn <= tf) hm |= __byte_perm(kids4, 0u, 0x4440u + b) << __byte_perm(bit4, 0u, 0x4440u + b);
        }
      }
      nbase = __float_as_uint(n1.x);
      nmask = (hm & 0xFF000000u) | imask;
      tbase = __float_as_uint(n1.y);
      tmask = hm & 0x00FFFFFFu;
    } else {
      tbase = nbase;
      tmask = nmask;
      nmask = 0;
    }
    while (tmask != 0u) {
      const int bit = 31 - __clz(tmask);
      tmask &= ~(1u << bit);
      const uint32_t ti = tbase + (uint32_t)bit;
      if (ti >= tr.n_tris) {
        raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
        return h;
      }
      const float4* rec = tr.tris + (size_t)ti * 3;
      const float4 a = __ldg(rec + 0), b = __ldg(rec + 1), c = __ldg(rec + 2);
      const f3 e1 = mk(a.x, a.y, a.z), e2 = mk(b.x, b.y, b.z);
      const f3 p = cross(d, e2);
      const float det = dot(e1, p);
      const bool pos = det >= 0.0f;
      const float ad = pos ? det : -det;
      const f3 tv = o - mk(c.x, c.y, c.z);
      const float un = dot(tv, p);
      const f3 qv = cross(tv, e1);
      const float vn = dot(d, qv), tn = dot(e2, qv);
      const float us = pos ? un : -un, vs = pos ? vn : -vn, ts = pos ? tn : -tn;
      if (!(ad > 1e-8f && us >= 0.0f && us <= ad && vs >= 0.0f && (us + vs) <= ad && ts > tmin * ad &&
            ts < h.t * ad))
        continue;
      if (ANY) {
        h.t = 0.0f;
        return h;
      }
      const float inv = 1.0f / ad;
      h.t = ts * inv;
      h.u = us * inv;
      h.v = vs * inv;
      h.prim = __float_as_uint(c.w);
      h.tri = ti;
    }
    if (nmask <= 0x00FFFFFFu) {
      if (sp == 0) break;
      --sp;
      nbase = stack[sp].x;
      nmask = stack[sp].y;
    }
  }
  return h;
}

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
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
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
  const uint32_t grid = (n + kBlock - 1) / kBlock;
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
