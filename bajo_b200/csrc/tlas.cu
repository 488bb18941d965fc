// tlas.cu -- two-level traversal: a top-level tree over instances of the
// BLASes of a segmented triangle build (segment b = BLAS b).
//
// Restates the reference's TLAS path (bajo/bvh/gpu/tlas.mojo:54-235;
// Instance, bajo/bvh/types.mojo:153-190; tlas_common.mojo):
//  - an instance is a BLAS index and an affine transform (Affine3, 12 f32
//    row-major [m00 m01 m02 tx | m10 m11 m12 ty | m20 m21 m22 tz],
//    bajo/core/transform.mojo:22-47) with its inverse; its world box is the
//    BLAS root box under AABB.apply_transform (bajo/core/aabb.mojo:101-139);
//  - bajo_tlas_instance_boxes writes each instance's box as a three-vertex
//    record [min, max, min] whose triangle bounds are exactly that box, so the
//    top-level tree is an ordinary bajo_lbvh_build over those records (one
//    segment, one leaf per instance);
//  - the top-level walk is the binary near-first loop of traverse.cuh with
//    instances as leaves: the world ray goes to BLAS space through the inverse
//    transform (Affine3.ray: origin by point(), direction by vector(), same
//    t_min, t_max = the current hit distance) and the BLAS is traversed from
//    its segment's root; a BLAS hit is closer by construction (the BLAS test
//    keeps t < t_max), so it replaces the world hit with its instance id
//    (promote_tlas_local_hit, tlas_common.mojo:7-27);
//  - only the winning hit's normal is taken to world space, through the
//    inverse's transpose and normalised (finalize_tlas_hit_normal,
//    normal_from_inverse, transform.mojo:224-257);
//  - any hit returns t = 0, prim 0xFFFFFFFF and the occluding instance
//    (Hit.shadow_hit with inst set, tlas.mojo:118-122).
// Ties between instances at the same distance keep the first visited, as in
// the reference; the oracle walks in the same order.
#include "traverse.cuh"

namespace bajo {
namespace tlas {

constexpr int kBlock = 128;

struct Blas {
  const float4* nb;
  const uint4* meta;
  const float4* tris;
  const uint32_t* roots;
  uint32_t n_blas;
  uint32_t max_nodes;
};

struct Top {
  const float4* nb;
  const uint4* meta;
  const uint32_t* leaf_ids;  // sorted leaf -> instance
  const uint32_t* roots;     // the top-level root ref (device)
  uint32_t max_nodes;
  uint32_t n_inst;
  const float4* inv;         // [instance][3] rows of the world -> BLAS transform
  const uint32_t* blas;      // [instance] BLAS index
};

struct Hit {
  float t, u, v;
  uint32_t prim, inst, leaf;
};

// Affine3.point / Affine3.vector (transform.mojo:155-173)
__device__ __forceinline__ f3 xf_point(const float4& r0, const float4& r1, const float4& r2, f3 p) {
  return mk(__fmaf_rn(r0.x, p.x, __fmaf_rn(r0.y, p.y, __fmaf_rn(r0.z, p.z, r0.w))),
            __fmaf_rn(r1.x, p.x, __fmaf_rn(r1.y, p.y, __fmaf_rn(r1.z, p.z, r1.w))),
            __fmaf_rn(r2.x, p.x, __fmaf_rn(r2.y, p.y, __fmaf_rn(r2.z, p.z, r2.w))));
}

__device__ __forceinline__ f3 xf_vector(const float4& r0, const float4& r1, const float4& r2, f3 v) {
  return mk(__fmaf_rn(r0.x, v.x, __fmaf_rn(r0.y, v.y, r0.z * v.z)),
            __fmaf_rn(r1.x, v.x, __fmaf_rn(r1.y, v.y, r1.z * v.z)),
            __fmaf_rn(r2.x, v.x, __fmaf_rn(r2.y, v.y, r2.z * v.z)));
}

// one instance leaf: the BLAS walk in BLAS space, promoted on a hit
template <int MODE, bool ANY>
__device__ __forceinline__ bool test_instance(const trav::Ray& r, uint32_t sorted, const Top& top, const Blas& bl,
                                              Hit& h, uint32_t* status) {
  const uint32_t inst = __ldg(top.leaf_ids + sorted);
  if (inst >= top.n_inst) {
    raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
    return false;
  }
  const uint32_t b = __ldg(top.blas + inst);
  if (b >= bl.n_blas) {
    raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
    return false;
  }
  const float4 r0 = __ldg(top.inv + (size_t)inst * 3 + 0), r1 = __ldg(top.inv + (size_t)inst * 3 + 1),
               r2 = __ldg(top.inv + (size_t)inst * 3 + 2);
  const trav::Ray lr =
      trav::make_ray(xf_point(r0, r1, r2, r.o), xf_vector(r0, r1, r2, r.d), r.tmin, ANY ? r.tmax : h.t);
  const trav::Hit lh =
      trav::trace_bvh2<MODE, false, ANY>(lr, __ldg(bl.roots + b), bl.nb, bl.meta, bl.tris, bl.max_nodes, status);
  if (lh.leaf == kEmpty) return false;
  h.t = lh.t;
  h.u = lh.u;
  h.v = lh.v;
  h.prim = lh.prim;
  h.inst = inst;
  h.leaf = lh.leaf;
  return true;
}

// the binary near-first loop of trav::trace_bvh2_impl over the top-level tree
template <int MODE, bool ANY, bool PAR>
__device__ Hit trace_impl(const trav::Ray& r, const Top& top, const Blas& bl, uint32_t* status) {
  Hit h;
  h.t = r.tmax;
  h.u = h.v = 0.0f;
  h.prim = h.inst = h.leaf = kEmpty;
  const uint32_t root = __ldg(top.roots);
  if (root == kSentinel) return h;
  if (root & kLeafFlag) {
    test_instance<MODE, ANY>(r, root & kIndexMask, top, bl, h, status);
    return h;
  }
  uint32_t stack[trav::kStack];
  int sp = 0;
  uint32_t cur = root;
  uint32_t fail = 0;  // status bits, raised after the loop (no atomic in the loop's code)
  for (uint32_t visits = 0;; ++visits) {
    if (visits >= top.max_nodes || cur >= top.max_nodes) {
      fail |= BAJO_STATUS_BAD_TOPOLOGY;
      break;
    }
    const float4 b0 = __ldg(top.nb + (size_t)cur * 3 + 0), b1 = __ldg(top.nb + (size_t)cur * 3 + 1),
                 b2 = __ldg(top.nb + (size_t)cur * 3 + 2);
    const uint4 g = __ldg(top.meta + cur);
    const uint2 m = make_uint2(g.y, g.z);
    float tl, tr;
    const float limit0 = ANY ? r.tmax : h.t;
    const bool hl = trav::box_hit<PAR>(r, b0, make_float2(b1.x, b1.y), limit0, tl);
    const bool hr = trav::box_hit<PAR>(r, make_float4(b1.z, b1.w, b2.x, b2.y), make_float2(b2.z, b2.w), limit0, tr);
    bool vl = false, vr = false;
    if (hl) {
      if (m.x & kLeafFlag) {
        if (test_instance<MODE, ANY>(r, m.x & kIndexMask, top, bl, h, status) && ANY) {
          if (fail) raise_status(status, fail);
          return h;
        }
      } else vl = true;
    }
    if (hr) {
      if (m.y & kLeafFlag) {
        if (test_instance<MODE, ANY>(r, m.y & kIndexMask, top, bl, h, status) && ANY) {
          if (fail) raise_status(status, fail);
          return h;
        }
      } else vr = true;
    }
    int near = -1;
    if (vl) near = 0;
    if (vr && (near == -1 || tr < tl)) near = 1;
    if (near >= 0) {
      const float limit = (ANY ? r.tmax : h.t) * kSlack;
      const bool far_valid = near == 0 ? vr : vl;
      const float far_t = near == 0 ? tr : tl;
      const float near_t = near == 0 ? tl : tr;
      if (far_valid && far_t <= limit) {
        if (sp < trav::kStack) stack[sp++] = near == 0 ? m.y : m.x;
        else fail |= BAJO_STATUS_STACK_OVERFLOW;
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

template <int MODE, bool ANY>
__device__ __forceinline__ Hit trace(const trav::Ray& r, const Top& top, const Blas& bl, uint32_t* status) {
  if (trav::has_parallel_axis(r)) return trace_impl<MODE, ANY, true>(r, top, bl, status);
  return trace_impl<MODE, ANY, false>(r, top, bl, status);
}

template <bool ANY>
__device__ __forceinline__ void store(const Hit& h, const Top& top, const Blas& bl, uint32_t i,
                                      float* __restrict__ hits8) {
  f3 n = mk(0.0f, 0.0f, 0.0f);
  float t = h.t;
  uint32_t prim = h.prim;
  if (ANY) {
    if (h.leaf != kEmpty) {
      t = 0.0f;
      prim = kEmpty;
    }
  } else if (h.leaf != kEmpty) {
    const float4 a = __ldg(bl.tris + (size_t)h.leaf * 3 + 0), b = __ldg(bl.tris + (size_t)h.leaf * 3 + 1),
                 c = __ldg(bl.tris + (size_t)h.leaf * 3 + 2);
    const f3 v0 = mk(a.x, a.y, a.z);
    const f3 ln = normalize(cross(mk(b.x, b.y, b.z) - v0, mk(c.x, c.y, c.z) - v0));
    const float4 r0 = __ldg(top.inv + (size_t)h.inst * 3 + 0), r1 = __ldg(top.inv + (size_t)h.inst * 3 + 1),
                 r2 = __ldg(top.inv + (size_t)h.inst * 3 + 2);
    n = normalize(mk(__fmaf_rn(r0.x, ln.x, __fmaf_rn(r1.x, ln.y, r2.x * ln.z)),
                     __fmaf_rn(r0.y, ln.x, __fmaf_rn(r1.y, ln.y, r2.y * ln.z)),
                     __fmaf_rn(r0.z, ln.x, __fmaf_rn(r1.z, ln.y, r2.z * ln.z))));
  }
  float4* o = reinterpret_cast<float4*>(hits8 + (size_t)i * 8);
  o[0] = make_float4(ANY ? 0.0f : h.u, ANY ? 0.0f : h.v, __uint_as_float(prim), __uint_as_float(h.inst));
  o[1] = make_float4(n.x, n.y, n.z, t);
}

template <int MODE, bool ANY>
__global__ void __launch_bounds__(kBlock) rays_kernel(const float* __restrict__ rays, uint32_t n, Top top, Blas bl,
                                                      float* __restrict__ hits8, uint32_t* __restrict__ status) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const f3 o = mk(rays[i], rays[(size_t)n + i], rays[2 * (size_t)n + i]);
  const f3 d = mk(rays[4 * (size_t)n + i], rays[5 * (size_t)n + i], rays[6 * (size_t)n + i]);
  const Hit h = trace<MODE, ANY>(trav::make_ray(o, d, rays[3 * (size_t)n + i], rays[7 * (size_t)n + i]), top, bl,
                                 status);
  store<ANY>(h, top, bl, i, hits8);
}

template <int MODE, bool ANY>
__global__ void __launch_bounds__(kBlock) camera_kernel(const float* __restrict__ cams, uint32_t n, uint32_t width,
                                                        uint32_t height, float inv_h, Top top, Blas bl,
                                                        float* __restrict__ hits8, uint32_t* __restrict__ status) {
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
  const Hit h =
      trace<MODE, ANY>(trav::make_ray(mk(__ldg(c + 0), __ldg(c + 1), __ldg(c + 2)), dir, 0.0f, FLT_MAX), top, bl,
                       status);
  store<ANY>(h, top, bl, i, hits8);
}

// AABB.apply_transform of each instance's BLAS root box, as the three-vertex
// record [min, max, min] the top-level build takes
__global__ void __launch_bounds__(256) boxes_kernel(const float* __restrict__ seg_bounds, uint32_t n_blas,
                                                    const float4* __restrict__ xf, const uint32_t* __restrict__ blas,
                                                    uint32_t n, float* __restrict__ out9,
                                                    uint32_t* __restrict__ status) {
  const uint32_t i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const uint32_t b = blas[i];
  float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (b >= n_blas) {
    if (status) raise_status(status, BAJO_STATUS_BAD_TOPOLOGY);
  } else {
    const float* lb = seg_bounds + (size_t)b * 12;
    if (lb[0] <= lb[3]) {  // an empty BLAS keeps the empty box
      const float4 r[3] = {xf[(size_t)i * 3 + 0], xf[(size_t)i * 3 + 1], xf[(size_t)i * 3 + 2]};
      for (int k = 0; k < 3; ++k) mn[k] = mx[k] = r[k].w;  // the translation
      for (int col = 0; col < 3; ++col) {  // x, y, z columns of the linear part
        for (int k = 0; k < 3; ++k) {
          const float m = col == 0 ? r[k].x : (col == 1 ? r[k].y : r[k].z);
          const float a = m * lb[col], c = m * lb[3 + col];
          mn[k] = mn[k] + fminf(a, c);
          mx[k] = mx[k] + fmaxf(a, c);
        }
      }
    }
  }
  float* o = out9 + (size_t)i * 9;
  o[0] = mn[0]; o[1] = mn[1]; o[2] = mn[2];
  o[3] = mx[0]; o[4] = mx[1]; o[5] = mx[2];
  o[6] = mn[0]; o[7] = mn[1]; o[8] = mn[2];
}

bool make(const BajoLbvh* tl, const BajoLbvh* bs, const float* inv, const uint32_t* blas, uint32_t n_inst,
          Top& top, Blas& bl) {
  if (!tl || !bs || !inv || !blas || tl->n_segments != 1 || tl->n_leaves != n_inst || !tl->node_meta ||
      !tl->node_bounds || !tl->leaf_ids || !tl->roots || !bs->node_meta || !bs->node_bounds || !bs->leaf_tris ||
      !bs->roots || bs->n_segments == 0)
    return false;
  if (((uintptr_t)inv | (uintptr_t)tl->node_bounds | (uintptr_t)bs->node_bounds | (uintptr_t)bs->leaf_tris) & 15)
    return false;
  top.nb = reinterpret_cast<const float4*>(tl->node_bounds);
  top.meta = reinterpret_cast<const uint4*>(tl->node_meta);
  top.leaf_ids = tl->leaf_ids;
  top.roots = tl->roots;
  top.max_nodes = n_inst > 1 ? n_inst - 1 : 1;
  top.n_inst = n_inst;
  top.inv = reinterpret_cast<const float4*>(inv);
  top.blas = blas;
  bl.nb = reinterpret_cast<const float4*>(bs->node_bounds);
  bl.meta = reinterpret_cast<const uint4*>(bs->node_meta);
  bl.tris = reinterpret_cast<const float4*>(bs->leaf_tris);
  bl.roots = bs->roots;
  bl.n_blas = bs->n_segments;
  bl.max_nodes = bs->n_leaves > 1 ? bs->n_leaves - 1 : 1;
  return true;
}

}  // namespace tlas
}  // namespace bajo

extern "C" {

int32_t bajo_tlas_instance_boxes(const BajoLbvh* blas_set, const float* d_transforms, const uint32_t* d_blas,
                                 uint32_t n_instances, float* d_boxes9, uint32_t* d_status, void* stream) {
  if (!blas_set || !blas_set->seg_bounds || blas_set->n_segments == 0 || (n_instances && (!d_transforms ||
      !d_blas || !d_boxes9)) || ((uintptr_t)d_transforms & 15))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n_instances == 0) return BAJO_OK;
  bajo::tlas::boxes_kernel<<<(n_instances + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      blas_set->seg_bounds, blas_set->n_segments, reinterpret_cast<const float4*>(d_transforms), d_blas, n_instances,
      d_boxes9, d_status);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_tlas_rays(const BajoLbvh* tlas, const BajoLbvh* blas_set, const float* d_inv_transforms,
                             const uint32_t* d_blas, uint32_t n_instances, const float* d_rays, uint32_t n_rays,
                             int32_t any_hit, int32_t tri_mode, float* d_hits8, uint32_t* d_status, void* stream) {
  using namespace bajo::tlas;
  Top top;
  Blas bl;
  if (!make(tlas, blas_set, d_inv_transforms, d_blas, n_instances, top, bl) || (n_rays && (!d_rays || !d_hits8)) ||
      !d_status || (any_hit != 0 && any_hit != 1) || (tri_mode != BAJO_TRI_MT && tri_mode != BAJO_TRI_WATERTIGHT))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n_rays == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t grid = (n_rays + kBlock - 1) / kBlock;
  const bool mt = tri_mode == BAJO_TRI_MT;
#define BAJO_TLAS_RAYS(MM, AA) rays_kernel<MM, AA><<<grid, kBlock, 0, st>>>(d_rays, n_rays, top, bl, d_hits8, d_status)
  if (any_hit) {
    if (mt) BAJO_TLAS_RAYS(BAJO_TRI_MT, true);
    else BAJO_TLAS_RAYS(BAJO_TRI_WATERTIGHT, true);
  } else {
    if (mt) BAJO_TLAS_RAYS(BAJO_TRI_MT, false);
    else BAJO_TLAS_RAYS(BAJO_TRI_WATERTIGHT, false);
  }
#undef BAJO_TLAS_RAYS
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_trace_tlas_camera(const BajoLbvh* tlas, const BajoLbvh* blas_set, const float* d_inv_transforms,
                               const uint32_t* d_blas, uint32_t n_instances, const float* d_cameras, uint32_t n_rays,
                               uint32_t width, uint32_t height, int32_t any_hit, int32_t tri_mode, float* d_hits8,
                               uint32_t* d_status, void* stream) {
  using namespace bajo::tlas;
  Top top;
  Blas bl;
  if (!make(tlas, blas_set, d_inv_transforms, d_blas, n_instances, top, bl) || !d_cameras || width == 0 ||
      height == 0 || (n_rays && !d_hits8) || !d_status || (any_hit != 0 && any_hit != 1) ||
      (tri_mode != BAJO_TRI_MT && tri_mode != BAJO_TRI_WATERTIGHT))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (n_rays == 0) return BAJO_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t grid = (uint32_t)((bajo::trav::camera_threads(n_rays, width, height) + kBlock - 1) / kBlock);
  const float inv_h = 1.0f / (float)height;
  const bool mt = tri_mode == BAJO_TRI_MT;
#define BAJO_TLAS_CAM(MM, AA) \
  camera_kernel<MM, AA><<<grid, kBlock, 0, st>>>(d_cameras, n_rays, width, height, inv_h, top, bl, d_hits8, d_status)
  if (any_hit) {
    if (mt) BAJO_TLAS_CAM(BAJO_TRI_MT, true);
    else BAJO_TLAS_CAM(BAJO_TRI_WATERTIGHT, true);
  } else {
    if (mt) BAJO_TLAS_CAM(BAJO_TRI_MT, false);
    else BAJO_TLAS_CAM(BAJO_TRI_WATERTIGHT, false);
  }
#undef BAJO_TLAS_CAM
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

}  // extern "C"
