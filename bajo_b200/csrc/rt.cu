// rt.cu -- wavefront path tracing (PATH / NEE / MIS, and GUIDED with the
// learned proposal of mlp.cuh) of Lambertian, emissive, metal and dielectric
// triangle scenes over the binary LBVH, on sm_100a.
//
// Restates the reference's GPU wavefront renderer for triangle scenes:
//  - primary rays: gpu_rt_primary_kernel (bajo/rt/gpu/common_kernels.mojo:22),
//    Camera.make_ray_sampled (bajo/bvh/camera.mojo:156-209);
//  - closest hit + shading: gpu_rt_scene_trace_kernel
//    (bajo/rt/gpu/scene_trace.mojo:41-369): sky on miss (bajo/rt/common.mojo:24),
//    oriented normal (bajo/rt/geometry.mojo:20), next-event estimation with
//    the alias-table light sample (bajo/rt/gpu/path_shading.mojo:261-413),
//    MIS-weighted emission (:543-573), inline Lambertian sampling
//    (bajo/rt/shading.mojo:92-118) and Russian roulette (bajo/rt/common.mojo:43),
//    here split into a traversal kernel and a shading kernel joined by a
//    vertex queue;
//  - any-hit shadow rays (scene_trace.mojo:586);
//  - per-pixel resolve (common_kernels.mojo:97).
// Queues keep the reference's field-major ABI (bajo/rt/wavefront_contract.mojo:
// 41-96): path id (delta flag in bit 31) + 12 f32 planes, shadow id + 11
// planes, 3 planes of per-sample radiance.  Appends are warp-aggregated (one
// atomic per warp instead of one per thread, wavefront_contract.mojo:460).
//
// Random streams and direction sampling: sampling.cuh.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "mlp.cuh"
#include "cwbvh.cuh"
#include "sampling.cuh"
#include "traverse.cuh"

namespace bajo {
int sm_count();

namespace rt {

using trav::Ray;
using trav::Hit;
using smp::uniform4;
using smp::sincos_turns;
using smp::stage_bsdf;
using smp::stage_roulette;
using smp::stage_light;

constexpr uint32_t kDeltaBit = 0x80000000u;    // WAVE_PATH_DELTA_BIT, wavefront_contract.mojo:60
constexpr uint32_t kIdMask = 0x7FFFFFFFu;
constexpr int kPathPlanes = 12;                 // WavePathFloatAbi.PLANES
constexpr int kShadowPlanes = 11;               // WaveShadowFloatAbi.PLANES
constexpr uint32_t kIndexMask28 = 0x0FFFFFFFu;  // SURFACE_INDEX_MASK
constexpr float kInvPi = 0.3183098861837907f;   // BSDF_INV_PI, bajo/rt/shading.mojo:9
constexpr int kBlock = 128;
constexpr uint32_t kNoRecord = 0xFFFFFFFFu;

__device__ __forceinline__ float length2(f3 v) { return dot(v, v); }
__device__ __forceinline__ f3 neg(f3 v) { return mk(-v.x, -v.y, -v.z); }
__device__ __forceinline__ f3 mul(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ f3 divs(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }

// power_heuristic, bajo/rt/lighting.mojo:7-19
__device__ __forceinline__ float power_heuristic(float a, float b) {
  const float a2 = a * a, b2 = b * b, den = a2 + b2;
  return den > 0.0f ? a2 / den : 0.0f;
}

// sky_color, bajo/rt/common.mojo:24-33
__device__ __forceinline__ f3 sky(f3 d) {
  const f3 u = normalize(d);
  const float a = 0.5f * (u.y + 1.0f);
  return mk((1.0f - a) * 1.0f + a * 0.5f, (1.0f - a) * 1.0f + a * 0.7f, (1.0f - a) * 1.0f + a * 1.0f);
}

struct Queues {
  uint32_t* ids[2];
  float* fields[2];
  uint32_t* shadow_ids;
  float* shadow_fields;
  float* radiance;
  uint32_t* counters;  // [2b] = paths active at bounce b, [2b+1] = shadow rays of bounce b
  uint32_t* status;
  uint32_t capacity;
  uint32_t* rec[2];    // guided only: training-record index per path-queue slot (else null)
};

struct SceneView {
  const uint32_t* roots;
  const float4* nb;
  const uint4* meta;
  const float4* tris;
  uint32_t n_nodes;
  const uint32_t* surfaces;
  const float* lambertians;
  const float* emissives;
  const float* lights;
  uint32_t n_lights;
  float total_light_weight;
  const float* metals;       // 4 per metal: albedo rgb, fuzz
  const float* dielectrics;  // 1 per dielectric: refraction index
  bool has_materials;
  bool use_cw;  // trace through the compressed 8-wide tree (BajoRtScene::cwbvh8)
  cw::Tree cw;
};

// The hit triangle's first vertex, outward normal and item index from its
// record: a sorted BVH2 leaf record [v0, prim | v1, 0 | v2, 0] (the normal
// from v1 - v0 and v2 - v0), or a CWBVH8 record [e1, 0 | e2, 0 | v0, prim]
// whose edges were computed the same way at its build.  Both give the same
// bits for the same triangle.
struct TriFrame {
  f3 v0, outward;
  uint32_t prim;
};
template <bool CW>
__device__ __forceinline__ TriFrame tri_frame(const SceneView& sc, uint32_t rec) {
  TriFrame fr;
  if constexpr (CW) {
    const float4 a = __ldg(sc.cw.tris + (size_t)rec * 3 + 0);
    const float4 b = __ldg(sc.cw.tris + (size_t)rec * 3 + 1);
    const float4 cc = __ldg(sc.cw.tris + (size_t)rec * 3 + 2);
    fr.v0 = mk(cc.x, cc.y, cc.z);
    fr.outward = normalize(cross(mk(a.x, a.y, a.z), mk(b.x, b.y, b.z)));
    fr.prim = __float_as_uint(cc.w);
  } else {
    const float4 a = __ldg(sc.tris + (size_t)rec * 3 + 0);
    const float4 b = __ldg(sc.tris + (size_t)rec * 3 + 1);
    const float4 cc = __ldg(sc.tris + (size_t)rec * 3 + 2);
    fr.v0 = mk(a.x, a.y, a.z);
    fr.outward = normalize(cross(mk(b.x, b.y, b.z) - fr.v0, mk(cc.x, cc.y, cc.z) - fr.v0));
    fr.prim = __float_as_uint(a.w);
  }
  return fr;
}

// Closest hit of one path ray: (distance, record, item); record = kEmpty on
// a miss.  BVH2: the watertight test, ties to the lowest item id; CWBVH8:
// the reference's own walk and Moller-Trumbore test, first of equal-distance
// hits in visiting order.
struct PathHit {
  float t;
  uint32_t rec, prim;
};
template <bool CW>
__device__ __forceinline__ PathHit trace_path(const SceneView& sc, f3 o, f3 d, float tmin, float tmax,
                                              uint32_t* status) {
  PathHit ph;
  if constexpr (CW) {
    const cw::Hit h = cw::trace<false>(o, d, tmin, tmax, sc.cw, status);
    ph.t = h.t;
    ph.rec = h.tri;
    ph.prim = h.prim;
  } else {
    const Ray r = trav::make_ray(o, d, tmin, tmax);
    const Hit h = trav::trace_bvh2<BAJO_TRI_WATERTIGHT>(r, __ldg(sc.roots), sc.nb, sc.meta, sc.tris, sc.n_nodes,
                                                        status);
    ph.t = h.t;
    ph.rec = h.leaf;
    ph.prim = h.prim;
  }
  return ph;
}

// warp-aggregated queue append: one atomic per warp; every lane of the warp
// must call it (want = false for lanes with nothing to append)
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
  const uint32_t mask = __ballot_sync(0xFFFFFFFFu, want);
  if (!mask) return 0;
  const uint32_t lane = lane_id();
  const uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  return base + __popc(mask & lanemask_lt());
}

// ---------------------------------------------------------------------------
// primary rays (gpu_rt_primary_kernel, common_kernels.mojo:22-93;
// Camera.make_ray_sampled, camera.mojo:156-209; random_in_unit_disk,
// bajo/core/random.mojo:56)
// ---------------------------------------------------------------------------
// With tile_w > 0 (a chunk of whole rows of tile_w x tile_h tiles, spp
// dividing 32), queue slot idx holds the samples of an 8 x 4, 4 x 4, 4 x 2 or
// 2 x 2 pixel tile per warp instead of 32 consecutive samples of one row, so
// that a warp's rays leave the camera side by side.  A path's id, and with it
// its random numbers and radiance slot, stays its sample index: the image
// does not depend on the order.
__global__ void __launch_bounds__(kBlock) primary_kernel(const float* __restrict__ cam, Queues q, uint32_t count,
                                                         uint32_t sample_base, uint32_t width, uint32_t height,
                                                         uint32_t spp, uint64_t seed, uint32_t tile_w,
                                                         uint32_t tile_h) {
  const uint32_t idx = blockIdx.x * kBlock + threadIdx.x;
  if (idx == 0) q.counters[0] = count;
  if (idx >= count) return;
  const uint32_t cap = q.capacity;
  uint32_t local = idx;  // sample index within the chunk
  if (tile_w) {
    const uint32_t warp = idx >> 5, lane = idx & 31u, p = lane / spp, smp_k = lane - p * spp;
    const uint32_t tiles_x = width / tile_w;
    const uint32_t px = (warp % tiles_x) * tile_w + p % tile_w, py = (warp / tiles_x) * tile_h + p / tile_w;
    local = (py * width + px) * spp + smp_k;
  }
  const uint32_t path_id = sample_base + local;
  const uint32_t pixel = path_id / spp;
  const uint32_t px = pixel % width, py = pixel / width;
  const float4 r = uniform4(seed, path_id, 0);
  float st, ct;
  sincos_turns(r.x, st, ct);
  const float lr = sqrtf(r.y);
  const float lens_u = lr * ct, lens_v = lr * st;
  const float w = (float)width, h = (float)height;
  const float aspect = w / h;
  const float sx = (((float)px + r.z) / w) * 2.0f - 1.0f;
  const float sy = 1.0f - (((float)py + r.w) / h) * 2.0f;
  const f3 origin = mk(cam[0], cam[1], cam[2]);
  const f3 fwd = mk(cam[3], cam[4], cam[5]), right = mk(cam[6], cam[7], cam[8]), up = mk(cam[9], cam[10], cam[11]);
  const float fs = cam[12], focus = cam[13];
  const f3 du = mk(cam[14], cam[15], cam[16]), dv = mk(cam[17], cam[18], cam[19]);
  const f3 inner = (fwd + right * ((sx * aspect) * fs)) + up * (sy * fs);
  const f3 focal = origin + mk(focus * inner.x, focus * inner.y, focus * inner.z);
  const f3 ro = (origin + mk(lens_u * du.x, lens_u * du.y, lens_u * du.z)) + mk(lens_v * dv.x, lens_v * dv.y, lens_v * dv.z);
  const f3 d = normalize(focal - ro);
  q.ids[0][idx] = path_id | kDeltaBit;
  float* f = q.fields[0];
  f[0 * cap + idx] = ro.x; f[1 * cap + idx] = ro.y; f[2 * cap + idx] = ro.z; f[3 * cap + idx] = 0.001f;
  f[4 * cap + idx] = d.x; f[5 * cap + idx] = d.y; f[6 * cap + idx] = d.z; f[7 * cap + idx] = FLT_MAX;
  f[8 * cap + idx] = 1.0f; f[9 * cap + idx] = 1.0f; f[10 * cap + idx] = 1.0f; f[11 * cap + idx] = 0.0f;
  q.radiance[0 * cap + local] = 0.0f;
  q.radiance[1 * cap + local] = 0.0f;
  q.radiance[2 * cap + local] = 0.0f;
  if (q.rec[0]) q.rec[0][idx] = kNoRecord;
}

__device__ __forceinline__ void accumulate(const Queues& q, uint32_t sidx, f3 v) {
  q.radiance[0 * q.capacity + sidx] += v.x;
  q.radiance[1 * q.capacity + sidx] += v.y;
  q.radiance[2 * q.capacity + sidx] += v.z;
}

// ---------------------------------------------------------------------------
// Bounce kernels.  Every bounce runs three launches over the queues:
//  - trace_kernel<ALGO>: closest hit of every active path; sky on a miss,
//    (MIS-weighted) emission on an emitter (_route_surface_hit,
//    path_shading.mojo:543-573), Lambertian hits appended to a vertex queue;
//  - shade_kernel<ALGO> (guided_shade_kernel for BAJO_RENDER_GUIDED): per
//    vertex, next-event estimation (_sample_direct_light_candidate,
//    path_shading.mojo:261-413) and the continuation (_sample_lambertian,
//    bajo/rt/shading.mojo:92-118; russian_roulette, bajo/rt/common.mojo:43-67),
//    appending shadow rays and next-bounce paths;
//  - shadow_kernel: any-hit visibility of the light samples.
// The reference fuses the first two in gpu_rt_scene_trace_kernel
// (scene_trace.mojo:41-369).  Split, the traversal kernel keeps a smaller
// register footprint and no shading divergence, and the guided tracer runs
// its network between the two.  The arithmetic is the fused kernel's, so
// images are unchanged bit for bit.
// Guided tracing (BAJO_RENDER_GUIDED) draws the continuation by one-sample
// MIS between the cosine BSDF and the network's vMF mixture and weighs every
// MIS decision against that combined pdf.
// ---------------------------------------------------------------------------
constexpr int kVtxPlanes = 12;  // p xyz, oriented normal xyz, albedo rgb, throughput rgb
constexpr int kShadeThreads = 256;

struct ShadeCtx {
  uint32_t* vtx_ids;
  float* vtx;
  uint32_t* vcount;     // [b] = Lambertian vertices of bounce b (from the front of the vertex queue)
  uint32_t* mcount;     // [b] = metal / dielectric hits of bounce b (from the back)
  // guided tracing only
  const __half* params16;
  const float* box;
  float frac;           // probability of sampling the mixture
  float rec_frac;       // probability a continued vertex becomes a training record
  uint32_t rec_cap;
  uint32_t* rec_hdr;    // [0] = records appended, [1] = first record of the chunk
  float* rec_pos;
  float* rec_nrm;
  float* rec_dir;
  float* rec_weight;
  uint32_t* rec_sidx;
  float* rec_tn;
  float* rec_snap;
  float* rec_wpre;
};

// integer hash "lowbias32" (C. Wellons, hash-prospector): record selection
__device__ __forceinline__ uint32_t lowbias32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// vMF direction around unit mean mu (Jakob, "Numerically stable sampling of
// the von Mises-Fisher distribution on S^2", 2012): cos theta = 1 +
// log(u + (1 - u) e^-2kappa) / kappa, azimuth 2 pi v, in the orthonormal
// basis of Duff et al. (JCGT 2017).
__device__ __forceinline__ f3 vmf_sample(const float* mu, float kappa, float u, float v) {
  float w = 1.0f + logf(u + (1.0f - u) * expf(-2.0f * kappa)) / kappa;
  w = fminf(fmaxf(w, -1.0f), 1.0f);
  const float st = sqrtf(fmaxf(0.0f, 1.0f - w * w));
  float sp, cp;
  sincos_turns(v, sp, cp);
  const float x = mu[0], y = mu[1], z = mu[2];
  const float sgn = z >= 0.0f ? 1.0f : -1.0f;
  const float a = -1.0f / (sgn + z);
  const float b = x * y * a;
  const f3 t1 = mk(1.0f + sgn * x * x * a, sgn * b, -sgn * x);
  const f3 t2 = mk(b, sgn + y * y * a, -y);
  const f3 d = (t1 * (st * cp) + t2 * (st * sp)) + mk(x, y, z) * w;
  return normalize(d);
}

// 1,024 resident threads per SM whatever the block size BLK (64 registers, a
// few bytes spilled): the traversal is latency bound and 32 resident warps
// hide more of it than 24 unspilled ones (C2 render 142 ms against 159 ms at
// 80 registers).
template <int ALGO, bool CW, int BLK>
__global__ void __launch_bounds__(BLK, 1024 / BLK) trace_kernel(SceneView sc, Queues q, ShadeCtx c, uint32_t bounce,
                                                             uint32_t sample_base) {
  constexpr bool kMisWeights = ALGO == BAJO_RENDER_MIS || ALGO == BAJO_RENDER_GUIDED;
  const uint32_t count = q.counters[2 * bounce];
  const uint32_t cap = q.capacity;
  const uint32_t* src_ids = q.ids[bounce & 1];
  const float* src = q.fields[bounce & 1];
  const uint32_t* src_rec = q.rec[bounce & 1];
  const uint32_t stride = gridDim.x * BLK;
  for (uint32_t base = blockIdx.x * BLK; base < count; base += stride) {
    const uint32_t idx = base + threadIdx.x;
    bool want_vtx = false, want_mat = false;
    uint32_t path_id = 0, mat_leaf = 0;
    float mat_t = 0.0f;
    f3 vp, vn, va, vt;
    if (idx < count) {
      const uint32_t idw = src_ids[idx];
      path_id = idw & kIdMask;
      const bool delta = (idw & kDeltaBit) != 0;
      const f3 o = mk(src[0 * cap + idx], src[1 * cap + idx], src[2 * cap + idx]);
      const float tmin = src[3 * cap + idx];
      const f3 d = mk(src[4 * cap + idx], src[5 * cap + idx], src[6 * cap + idx]);
      const float tmax = src[7 * cap + idx];
      const f3 T = mk(src[8 * cap + idx], src[9 * cap + idx], src[10 * cap + idx]);
      const float prev_pdf = src[11 * cap + idx];
      const uint32_t sidx = path_id - sample_base;
      if (ALGO == BAJO_RENDER_GUIDED) {
        const uint32_t rec = src_rec[idx];
        if (rec != kNoRecord) {  // radiance gathered before this ray: the record's baseline
          c.rec_snap[3 * (size_t)rec + 0] = q.radiance[0 * cap + sidx];
          c.rec_snap[3 * (size_t)rec + 1] = q.radiance[1 * cap + sidx];
          c.rec_snap[3 * (size_t)rec + 2] = q.radiance[2 * cap + sidx];
        }
      }
      const PathHit h = trace_path<CW>(sc, o, d, tmin, tmax, q.status);
      if (h.rec == kEmpty) {
        accumulate(q, sidx, mul(T, sky(d)));
      } else {
        const float t = h.t;
        const f3 outward = tri_frame<CW>(sc, h.rec).outward;
        const bool front = dot(d, outward) < 0.0f;
        const f3 normal = front ? outward : neg(outward);
        const uint32_t surface = __ldg(sc.surfaces + h.prim);
        const uint32_t kind = surface >> 28, midx = surface & kIndexMask28;
        const f3 p = mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
        if (kind == BAJO_MAT_EMISSIVE) {
          if (front) {
            const f3 L = mk(sc.emissives[3 * midx], sc.emissives[3 * midx + 1], sc.emissives[3 * midx + 2]);
            float wgt = 1.0f;
            if (ALGO == BAJO_RENDER_NEE && bounce > 0 && !delta) wgt = 0.0f;
            if (kMisWeights && bounce > 0 && !delta) {
              const float lc = fmaxf(dot(normal, neg(normalize(d))), 0.0f);
              float lpdf = 0.0f;
              if (lc > 0.0f && sc.total_light_weight > 0.0f) {
                const float d2 = (t * t) * length2(d);
                lpdf = (d2 * ((L.x + L.y) + L.z)) / ((3.0f * lc) * sc.total_light_weight);
              }
              wgt = power_heuristic(prev_pdf, lpdf);
            }
            const f3 TL = mul(T, L);
            accumulate(q, sidx, mk(TL.x * wgt, TL.y * wgt, TL.z * wgt));
          }
        } else if (kind == BAJO_MAT_LAMBERTIAN) {
          want_vtx = true;
          vp = p;
          vn = normal;
          va = mk(sc.lambertians[3 * midx], sc.lambertians[3 * midx + 1], sc.lambertians[3 * midx + 2]);
          vt = T;
        } else if (kind == BAJO_MAT_METAL || kind == BAJO_MAT_DIELECTRIC) {
          want_mat = true;
          mat_leaf = h.rec;
          mat_t = t;
        }
      }
    }
    if (sc.has_materials) {
      // metal / dielectric hits go to the back of the vertex queue: the
      // source slot, the hit's sorted leaf and distance (material_kernel
      // recomputes the rest exactly as above)
      const uint32_t k = warp_append(&c.mcount[bounce], want_mat);
      if (want_mat) {
        // every path yields at most one vertex, so the two ends never meet
        const uint32_t slot = cap - 1u - k;
        if (k < cap) {
          c.vtx_ids[slot] = idx;
          c.vtx[0 * cap + slot] = __uint_as_float(mat_leaf);
          c.vtx[1 * cap + slot] = mat_t;
        } else {
          raise_status(q.status, BAJO_WAVE_PATH_OVERFLOW);
        }
      }
    }
    const uint32_t slot = warp_append(&c.vcount[bounce], want_vtx);
    if (want_vtx) {
      if (slot < cap) {
        c.vtx_ids[slot] = path_id;
        float* f = c.vtx;
        f[0 * cap + slot] = vp.x; f[1 * cap + slot] = vp.y; f[2 * cap + slot] = vp.z;
        f[3 * cap + slot] = vn.x; f[4 * cap + slot] = vn.y; f[5 * cap + slot] = vn.z;
        f[6 * cap + slot] = va.x; f[7 * cap + slot] = va.y; f[8 * cap + slot] = va.z;
        f[9 * cap + slot] = vt.x; f[10 * cap + slot] = vt.y; f[11 * cap + slot] = vt.z;
      } else {
        raise_status(q.status, BAJO_WAVE_PATH_OVERFLOW);
      }
    }
  }
}

struct ShadeOut {
  bool want_shadow = false, want_next = false, want_rec = false;
  f3 sh_o, sh_d, sh_c, nx_o, nx_d, nx_t, normal;
  float sh_tmax = 0.0f, nx_pdf = 0.0f, wpre = 0.0f;
  uint32_t path_id = 0;
};

// Next-event estimation and continuation of vertex i of bounce `bounce`.
template <int ALGO>
__device__ __forceinline__ void shade_vertex(const SceneView& sc, const ShadeCtx& c, uint32_t cap, uint32_t i,
                                             uint32_t bounce, uint32_t max_depth, uint64_t seed,
                                             const mlp::Mixture& mix, ShadeOut& o) {
  constexpr bool kGuided = ALGO == BAJO_RENDER_GUIDED;
  const float g = kGuided ? c.frac : 0.0f;
  const uint32_t path_id = c.vtx_ids[i];
  o.path_id = path_id;
  const f3 p = mk(c.vtx[0 * cap + i], c.vtx[1 * cap + i], c.vtx[2 * cap + i]);
  const f3 normal = mk(c.vtx[3 * cap + i], c.vtx[4 * cap + i], c.vtx[5 * cap + i]);
  o.normal = normal;
  const f3 albedo = mk(c.vtx[6 * cap + i], c.vtx[7 * cap + i], c.vtx[8 * cap + i]);
  const f3 T = mk(c.vtx[9 * cap + i], c.vtx[10 * cap + i], c.vtx[11 * cap + i]);
  if ((ALGO == BAJO_RENDER_NEE || ALGO == BAJO_RENDER_MIS || kGuided) && sc.n_lights > 0 &&
      sc.total_light_weight > 0.0f) {
    // _sample_direct_light_candidate, path_shading.mojo:261-413
    const float4 u = uniform4(seed, path_id, stage_light(bounce));
    const float as = u.x * (float)sc.n_lights;
    uint32_t li = (uint32_t)as;
    const float frac = as - (float)li;
    const float* lrec = sc.lights + (size_t)li * BAJO_LIGHT_STRIDE;
    if (frac > lrec[12]) li = __float_as_uint(lrec[13]);
    lrec = sc.lights + (size_t)li * BAJO_LIGHT_STRIDE;
    const f3 p0 = mk(lrec[0], lrec[1], lrec[2]), p1 = mk(lrec[3], lrec[4], lrec[5]),
             p2 = mk(lrec[6], lrec[7], lrec[8]);
    const f3 e1 = p1 - p0, e2 = p2 - p0;
    const f3 av = cross(e1, e2);
    const float tas = length2(av);
    if (tas > 0.0f) {
      const f3 ln = divs(av, sqrtf(tas));
      const float ru = sqrtf(u.y);
      const float b1 = ru * (1.0f - u.z);
      const float b2 = ru - b1;
      const f3 lp = (p0 + e1 * b1) + e2 * b2;
      const f3 tl = lp - p;
      const float d2 = length2(tl);
      if (d2 > 1.0e-8f) {
        const float dist = sqrtf(d2);
        const f3 dir = divs(tl, dist);
        const float scos = fmaxf(dot(normal, dir), 0.0f);
        const float lcos = fmaxf(dot(ln, neg(dir)), 0.0f);
        const float smax = dist - 0.002f;
        if (scos > 0.0f && lcos > 0.0f && smax > 0.001f) {
          const f3 E = mk(lrec[9], lrec[10], lrec[11]);
          const float lpdf = (d2 * ((E.x + E.y) + E.z)) / ((3.0f * lcos) * sc.total_light_weight);
          const float bpdf = fmaxf(dot(normal, normalize(dir)), 0.0f) * kInvPi;
          if (lpdf > 0.0f && bpdf > 0.0f) {
            float wgt = 1.0f;
            if (ALGO == BAJO_RENDER_MIS) wgt = power_heuristic(lpdf, bpdf);
            if (kGuided) {
              const float dd[3] = {dir.x, dir.y, dir.z};
              const float qpdf = (1.0f - g) * bpdf + (g > 0.0f ? g * mlp::mixture_pdf(mix, dd) : 0.0f);
              wgt = power_heuristic(lpdf, qpdf);
            }
            const float scale = (scos * wgt) / lpdf;
            if (scale > 0.0f) {
              const f3 value = albedo * kInvPi;
              const f3 tv = mul(mul(T, value), E);
              o.want_shadow = true;
              o.sh_o = p;
              o.sh_d = dir;
              o.sh_tmax = smax;
              o.sh_c = tv * scale;
            }
          }
        }
      }
    }
  }
  if (bounce + 1 < max_depth) {
    const float4 u = uniform4(seed, path_id, stage_bsdf(bounce));
    f3 dir;
    if (kGuided && u.w < g) {
      int k = 0;
      float acc = mix.pi[0];
      while (k < mlp::kLobes - 1 && u.z >= acc) acc += mix.pi[++k];
      dir = vmf_sample(mix.mu[k], mix.kap[k], u.x, u.y);
    } else {
      dir = smp::lambertian_dir(normal, u.x, u.y);
    }
    const float cosv = fmaxf(dot(normal, normalize(dir)), 0.0f);
    const float bp = cosv * kInvPi;
    if (!kGuided || bp > 0.0f) {
      float qpdf = bp;
      f3 Tn = mul(T, albedo);
      if (kGuided) {
        const float dd[3] = {dir.x, dir.y, dir.z};
        qpdf = (1.0f - g) * bp + (g > 0.0f ? g * mlp::mixture_pdf(mix, dd) : 0.0f);
        const float factor = bp / qpdf;
        if (factor != 1.0f) Tn = Tn * factor;
      }
      bool alive = !kGuided || qpdf > 0.0f;
      if (alive && bounce + 1 >= 5u) {
        const float m = fmaxf(Tn.x, fmaxf(Tn.y, Tn.z));
        if (m <= 0.0f) alive = false;
        else {
          const float survival = fminf(fmaxf(m, 0.05f), 0.95f);
          const float4 rr = uniform4(seed, path_id, stage_roulette(bounce));
          if (rr.x >= survival) alive = false;
          else Tn = divs(Tn, survival);
        }
      }
      if (alive) {
        o.want_next = true;
        o.nx_o = p;
        o.nx_d = dir;
        o.nx_t = Tn;
        o.nx_pdf = qpdf;
        if (kGuided) {
          o.wpre = cosv / qpdf;
          const uint32_t h = lowbias32(path_id ^ lowbias32(bounce * 0x9E3779B9u + (uint32_t)seed));
          o.want_rec = c.rec_cap > 0 && (float)(h >> 8) * (1.0f / 16777216.0f) < c.rec_frac;
        }
      }
    }
  }
}

// Queue appends of one shaded vertex; every lane of the warp calls this.
template <int ALGO>
__device__ __forceinline__ void emit(const Queues& q, const ShadeCtx& c, uint32_t bounce, uint32_t sample_base,
                                     const ShadeOut& o) {
  const uint32_t cap = q.capacity;
  if (ALGO != BAJO_RENDER_PATH) {
    const uint32_t sslot = warp_append(&q.counters[2 * bounce + 1], o.want_shadow);
    if (o.want_shadow) {
      if (sslot < cap) {
        q.shadow_ids[sslot] = o.path_id;
        float* f = q.shadow_fields;
        f[0 * cap + sslot] = o.sh_o.x; f[1 * cap + sslot] = o.sh_o.y; f[2 * cap + sslot] = o.sh_o.z;
        f[3 * cap + sslot] = 0.001f;
        f[4 * cap + sslot] = o.sh_d.x; f[5 * cap + sslot] = o.sh_d.y; f[6 * cap + sslot] = o.sh_d.z;
        f[7 * cap + sslot] = o.sh_tmax;
        f[8 * cap + sslot] = o.sh_c.x; f[9 * cap + sslot] = o.sh_c.y; f[10 * cap + sslot] = o.sh_c.z;
      } else {
        raise_status(q.status, BAJO_WAVE_SHADOW_OVERFLOW);
      }
    }
  }
  const uint32_t slot = warp_append(&q.counters[2 * (bounce + 1)], o.want_next);
  uint32_t rslot = kNoRecord;
  if (ALGO == BAJO_RENDER_GUIDED) rslot = warp_append(&c.rec_hdr[0], o.want_rec);
  if (o.want_next) {
    if (slot < cap) {
      uint32_t* dst_ids = q.ids[(bounce + 1) & 1];
      float* dst = q.fields[(bounce + 1) & 1];
      if (ALGO == BAJO_RENDER_GUIDED) {
        const uint32_t sidx = o.path_id - sample_base;
        uint32_t rec = kNoRecord;
        if (o.want_rec && rslot < c.rec_cap) {
          rec = rslot;
          const size_t r3 = 3 * (size_t)rslot;
          c.rec_pos[r3] = o.nx_o.x; c.rec_pos[r3 + 1] = o.nx_o.y; c.rec_pos[r3 + 2] = o.nx_o.z;
          c.rec_nrm[r3] = o.normal.x; c.rec_nrm[r3 + 1] = o.normal.y; c.rec_nrm[r3 + 2] = o.normal.z;
          c.rec_dir[r3] = o.nx_d.x; c.rec_dir[r3 + 1] = o.nx_d.y; c.rec_dir[r3 + 2] = o.nx_d.z;
          c.rec_tn[r3] = o.nx_t.x; c.rec_tn[r3 + 1] = o.nx_t.y; c.rec_tn[r3 + 2] = o.nx_t.z;
          c.rec_snap[r3] = q.radiance[0 * cap + sidx];
          c.rec_snap[r3 + 1] = q.radiance[1 * cap + sidx];
          c.rec_snap[r3 + 2] = q.radiance[2 * cap + sidx];
          c.rec_sidx[rslot] = sidx;
          c.rec_wpre[rslot] = o.wpre;
          c.rec_weight[rslot] = 0.0f;
        }
        q.rec[(bounce + 1) & 1][slot] = rec;
      }
      dst_ids[slot] = o.path_id;  // delta = false after a Lambertian bounce
      dst[0 * cap + slot] = o.nx_o.x; dst[1 * cap + slot] = o.nx_o.y; dst[2 * cap + slot] = o.nx_o.z;
      dst[3 * cap + slot] = 0.001f;
      dst[4 * cap + slot] = o.nx_d.x; dst[5 * cap + slot] = o.nx_d.y; dst[6 * cap + slot] = o.nx_d.z;
      dst[7 * cap + slot] = FLT_MAX;
      dst[8 * cap + slot] = o.nx_t.x; dst[9 * cap + slot] = o.nx_t.y; dst[10 * cap + slot] = o.nx_t.z;
      dst[11 * cap + slot] = o.nx_pdf;
    } else {
      raise_status(q.status, BAJO_WAVE_PATH_OVERFLOW);
    }
  }
}

template <int ALGO, int BLK>
__global__ void __launch_bounds__(BLK) shade_kernel(SceneView sc, Queues q, ShadeCtx c, uint32_t bounce,
                                                    uint32_t max_depth, uint32_t sample_base, uint64_t seed) {
  const uint32_t cap = q.capacity;
  const uint32_t count = min(c.vcount[bounce], cap);
  const mlp::Mixture none{};
  for (uint32_t base = blockIdx.x * BLK; base < count; base += gridDim.x * BLK) {
    const uint32_t i = base + threadIdx.x;
    ShadeOut o;
    if (i < count) shade_vertex<ALGO>(sc, c, cap, i, bounce, max_depth, seed, none, o);
    emit<ALGO>(q, c, bounce, sample_base, o);
  }
}

// Metal and dielectric hits of bounce `bounce` (gpu_rt_shade_dispatch_kernel
// and _gpu_rt_shade_one, bajo/rt/gpu/path_shading.mojo:690-786): the hit is
// rebuilt from the source path and triangle as trace_kernel built it, the
// material sample (smp::sample_metal / sample_dielectric) draws u, v from the
// bounce's BSDF stream, and the continued path (Russian roulette as for
// Lambertian bounces) carries the sample's pdf and delta flag.  No light
// sample is taken at these vertices, as in the reference.
template <int ALGO, bool CW>
__global__ void __launch_bounds__(kBlock) material_kernel(SceneView sc, Queues q, ShadeCtx c, uint32_t bounce,
                                                          uint32_t max_depth, uint64_t seed) {
  const uint32_t cap = q.capacity;
  const uint32_t count = min(c.mcount[bounce], cap);
  const uint32_t* src_ids = q.ids[bounce & 1];
  const float* src = q.fields[bounce & 1];
  for (uint32_t base = blockIdx.x * kBlock; base < count; base += gridDim.x * kBlock) {
    const uint32_t k = base + threadIdx.x;
    bool want = false;
    uint32_t path_id = 0;
    f3 p, dir, Tn;
    float pdf = 0.0f;
    bool delta = false;
    if (k < count && bounce + 1 < max_depth) {
      const uint32_t slot = cap - 1u - k;
      const uint32_t idx = c.vtx_ids[slot];
      const uint32_t leaf = __float_as_uint(c.vtx[0 * cap + slot]);
      const float t = c.vtx[1 * cap + slot];
      path_id = src_ids[idx] & kIdMask;
      const f3 o = mk(src[0 * cap + idx], src[1 * cap + idx], src[2 * cap + idx]);
      const f3 d = mk(src[4 * cap + idx], src[5 * cap + idx], src[6 * cap + idx]);
      const f3 T = mk(src[8 * cap + idx], src[9 * cap + idx], src[10 * cap + idx]);
      const TriFrame fr = tri_frame<CW>(sc, leaf);
      const f3 outward = fr.outward;
      const bool front = dot(d, outward) < 0.0f;
      const f3 normal = front ? outward : neg(outward);
      const uint32_t surface = __ldg(sc.surfaces + fr.prim);
      const uint32_t midx = surface & kIndexMask28;
      p = mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
      const float4 u = uniform4(seed, path_id, stage_bsdf(bounce));
      smp::BsdfSample smpl;
      if ((surface >> 28) == BAJO_MAT_METAL) {
        const float* m = sc.metals + 4 * (size_t)midx;
        smpl = smp::sample_metal(d, normal, mk(m[0], m[1], m[2]), m[3], u.x, u.y);
      } else {
        smpl = smp::sample_dielectric(d, normal, sc.dielectrics[midx], front, u.x);
      }
      if (smpl.ok) {
        Tn = mul(T, smpl.weight);
        bool alive = true;
        if (bounce + 1 >= 5u) {
          const float mx = fmaxf(Tn.x, fmaxf(Tn.y, Tn.z));
          if (mx <= 0.0f) alive = false;
          else {
            const float survival = fminf(fmaxf(mx, 0.05f), 0.95f);
            const float4 rr = uniform4(seed, path_id, stage_roulette(bounce));
            if (rr.x >= survival) alive = false;
            else Tn = divs(Tn, survival);
          }
        }
        want = alive;
        dir = smpl.dir;
        pdf = smpl.pdf;
        delta = smpl.delta;
      }
    }
    const uint32_t slot = warp_append(&q.counters[2 * (bounce + 1)], want);
    if (want) {
      if (slot < cap) {
        uint32_t* dst_ids = q.ids[(bounce + 1) & 1];
        float* dst = q.fields[(bounce + 1) & 1];
        if (ALGO == BAJO_RENDER_GUIDED) q.rec[(bounce + 1) & 1][slot] = kNoRecord;
        dst_ids[slot] = path_id | (delta ? kDeltaBit : 0u);
        dst[0 * cap + slot] = p.x; dst[1 * cap + slot] = p.y; dst[2 * cap + slot] = p.z;
        dst[3 * cap + slot] = 0.001f;
        dst[4 * cap + slot] = dir.x; dst[5 * cap + slot] = dir.y; dst[6 * cap + slot] = dir.z;
        dst[7 * cap + slot] = FLT_MAX;
        dst[8 * cap + slot] = Tn.x; dst[9 * cap + slot] = Tn.y; dst[10 * cap + slot] = Tn.z;
        dst[11 * cap + slot] = pdf;
      } else {
        raise_status(q.status, BAJO_WAVE_PATH_OVERFLOW);
      }
    }
  }
}

struct __align__(128) ShadeSmem {
  mlp::tc::Weights w;
  __half act[2 * mlp::tc::kRows * mlp::tc::kK];  // two 128-vertex tiles in core layout
  unsigned long long bar;
  uint32_t tmem;
};

// Guided shading.  Every CTA takes 256 vertices per step: each thread encodes
// one, the network runs on the two 128-row tiles on the 5th-generation
// tensor cores (mlp::tc::forward: tcgen05.mma into tensor memory), and each
// thread then shades its own vertex from its row's 20 outputs.
__global__ void __launch_bounds__(kShadeThreads, 2) guided_shade_kernel(SceneView sc, Queues q, ShadeCtx c,
                                                                        uint32_t bounce, uint32_t max_depth,
                                                                        uint32_t sample_base, uint64_t seed) {
  static_assert(kShadeThreads == 2 * mlp::tc::kRows, "two network tiles per step");
  extern __shared__ __align__(128) unsigned char raw[];
  ShadeSmem& s = *reinterpret_cast<ShadeSmem*>(raw);
  mlp::tc::load_weights<kShadeThreads>(s.w, c.params16);
  const uint32_t bar = mlp::tc::saddr(&s.bar);
  const uint32_t tmem = mlp::tc::setup<2>(bar, &s.tmem);
  uint32_t phase = 0;
  const uint32_t cap = q.capacity;
  const uint32_t count = min(c.vcount[bounce], cap);
  const int tid = threadIdx.x;
  unsigned char* const act = reinterpret_cast<unsigned char*>(s.act);
  unsigned char* const mine = act + (size_t)(tid / mlp::tc::kRows) * mlp::tc::kTileBytes;
  for (uint32_t base = blockIdx.x * kShadeThreads; base < count; base += gridDim.x * kShadeThreads) {
    const uint32_t i = base + tid;
    {
      uint32_t f[32];
      if (i < count) {
        const float p[3] = {c.vtx[0 * cap + i], c.vtx[1 * cap + i], c.vtx[2 * cap + i]};
        const float n[3] = {c.vtx[3 * cap + i], c.vtx[4 * cap + i], c.vtx[5 * cap + i]};
        mlp::tc::encode_pairs(p, n, c.box, f);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) f[j] = 0u;
      }
      mlp::tc::store_features(mine, tid % mlp::tc::kRows, f);
    }
    float out[mlp::kOut];
    if (!mlp::tc::forward<2>(s.w, act, tmem, bar, phase, out, q.status)) break;
    ShadeOut o;
    if (i < count) {
      mlp::Mixture mix;
      mlp::mixture_from_outputs(out, mix);
      shade_vertex<BAJO_RENDER_GUIDED>(sc, c, cap, i, bounce, max_depth, seed, mix, o);
    }
    emit<BAJO_RENDER_GUIDED>(q, c, bounce, sample_base, o);
  }
  mlp::tc::teardown<2>(tmem);
}

// ---------------------------------------------------------------------------
// any-hit shadow rays (gpu_rt_shadow_kernel, scene_trace.mojo:586)
// ---------------------------------------------------------------------------
template <bool CW, int BLK>
__global__ void __launch_bounds__(BLK) shadow_kernel(SceneView sc, Queues q, uint32_t bounce, uint32_t sample_base) {
  const uint32_t count = q.counters[2 * bounce + 1];
  const uint32_t cap = q.capacity;
  const float* f = q.shadow_fields;
  for (uint32_t i = blockIdx.x * BLK + threadIdx.x; i < count; i += gridDim.x * BLK) {
    const f3 o = mk(f[0 * cap + i], f[1 * cap + i], f[2 * cap + i]);
    const f3 d = mk(f[4 * cap + i], f[5 * cap + i], f[6 * cap + i]);
    bool open;
    if constexpr (CW) {
      open = cw::trace<true>(o, d, f[3 * cap + i], f[7 * cap + i], sc.cw, q.status).t != 0.0f;  // t = 0: occluded
    } else {
      const Ray r = trav::make_ray(o, d, f[3 * cap + i], f[7 * cap + i]);
      open = trav::trace_bvh2<BAJO_TRI_WATERTIGHT, false, true>(r, __ldg(sc.roots), sc.nb, sc.meta, sc.tris,
                                                                sc.n_nodes, q.status)
                 .leaf == kEmpty;
    }
    if (open) {
      const uint32_t sidx = q.shadow_ids[i] - sample_base;
      accumulate(q, sidx, mk(f[8 * cap + i], f[9 * cap + i], f[10 * cap + i]));
    }
  }
}

// ---------------------------------------------------------------------------
// per-pixel resolve (gpu_rt_resolve_kernel, common_kernels.mojo:97-136)
// ---------------------------------------------------------------------------
// Thread 0 also adds this chunk's traced rays (closest-hit and shadow, one
// per queue entry of every bounce) to the 64-bit totals.
__global__ void __launch_bounds__(kBlock) resolve_kernel(const float* __restrict__ radiance, uint32_t cap,
                                                         uint32_t pixel_base, uint32_t pixel_count, uint32_t spp,
                                                         float* __restrict__ pixels, double* __restrict__ pixels64,
                                                         const uint32_t* __restrict__ counters, uint32_t max_depth,
                                                         unsigned long long* __restrict__ totals) {
  const uint32_t p = blockIdx.x * kBlock + threadIdx.x;
  if (p == 0) {
    unsigned long long rays = 0, shadows = 0;
    for (uint32_t b = 0; b < max_depth; ++b) {
      rays += counters[2 * b];
      shadows += counters[2 * b + 1];
    }
    totals[0] += rays;
    totals[1] += shadows;
  }
  if (p >= pixel_count) return;
  float r = 0.0f, g = 0.0f, b = 0.0f;
  double r64 = 0.0, g64 = 0.0, b64 = 0.0;
  const uint32_t s0 = p * spp;
  for (uint32_t s = s0; s < s0 + spp; ++s) {
    const float x = radiance[s], y = radiance[cap + s], z = radiance[2 * cap + s];
    r += x;
    g += y;
    b += z;
    if (pixels64) {
      r64 += (double)x;
      g64 += (double)y;
      b64 += (double)z;
    }
  }
  const float scale = 1.0f / (float)spp;
  const size_t o = 3 * (size_t)(pixel_base + p);
  pixels[o + 0] = r * scale;
  pixels[o + 1] = g * scale;
  pixels[o + 2] = b * scale;
  if (pixels64) {
    pixels64[o + 0] += r64;
    pixels64[o + 1] += g64;
    pixels64[o + 2] += b64;
  }
}

// first record of the chunk = records appended so far (capped)
__global__ void records_begin_chunk_kernel(uint32_t* hdr, uint32_t cap) { hdr[1] = min(hdr[0], cap); }

// Records of the chunk: weight = mean_rgb((R_end - R_before) / T_after) *
// cos / pdf, the radiance gathered after the vertex per unit throughput.
__global__ void __launch_bounds__(kBlock) records_finish_chunk_kernel(ShadeCtx gc, const float* __restrict__ radiance,
                                                                      uint32_t cap) {
  const uint32_t start = gc.rec_hdr[1], end = min(gc.rec_hdr[0], gc.rec_cap);
  for (uint32_t i = start + blockIdx.x * kBlock + threadIdx.x; i < end; i += gridDim.x * kBlock) {
    const uint32_t sidx = gc.rec_sidx[i];
    float L = 0.0f;
    for (int c = 0; c < 3; ++c) {
      const float tn = gc.rec_tn[3 * (size_t)i + c];
      const float gathered = radiance[c * (size_t)cap + sidx] - gc.rec_snap[3 * (size_t)i + c];
      if (tn > 0.0f) L += gathered / tn;
    }
    float w = (L * (1.0f / 3.0f)) * gc.rec_wpre[i];
    if (!(w > 0.0f) || !isfinite(w)) w = 0.0f;
    gc.rec_weight[i] = w;
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
constexpr uint32_t kDefaultChunk = 1u << 22;

struct Layout {
  uint32_t cap, pixels_per_chunk, n_counters;
  size_t off_counters, off_ids[2], off_fields[2], off_shadow_ids, off_shadow_fields, off_radiance;
  size_t off_vtx_ids, off_vtx;  // vertex queue between the trace and shade kernels
  size_t off_rec[2];            // guided tracing only
  size_t total;
};

inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

bool make_layout(const BajoRenderSettings* s, Layout* L) {
  if (!s || s->width == 0 || s->height == 0 || s->spp == 0 || s->max_depth == 0 || s->max_depth > 1024) return false;
  uint32_t want = s->chunk_paths ? s->chunk_paths : kDefaultChunk;
  const uint64_t total_paths = (uint64_t)s->width * s->height * s->spp;
  if (total_paths > 0x7FFFFFFFull) return false;  // path ids carry the delta flag in bit 31
  if (want < s->spp) want = s->spp;
  uint32_t ppc = want / s->spp;
  const uint64_t npix = (uint64_t)s->width * s->height;
  if (ppc > npix) ppc = (uint32_t)npix;
  const bool guided = s->algorithm == BAJO_RENDER_GUIDED;
  L->pixels_per_chunk = ppc;
  L->cap = ppc * s->spp;
  // [2b] paths of bounce b, [2b+1] its shadow rays, then [2 max_depth + 2 +
  // b] the Lambertian vertices of bounce b
  L->n_counters = 4 * s->max_depth + 2;
  const size_t cap = L->cap;
  size_t o = 256;  // status word, then two 64-bit ray totals at offset 8
  L->off_counters = o;
  o = a256(o + (size_t)L->n_counters * 4);
  for (int k = 0; k < 2; ++k) {
    L->off_ids[k] = o;
    o = a256(o + cap * 4);
    L->off_fields[k] = o;
    o = a256(o + cap * 4 * kPathPlanes);
  }
  L->off_shadow_ids = o;
  o = a256(o + cap * 4);
  L->off_shadow_fields = o;
  o = a256(o + cap * 4 * kShadowPlanes);
  L->off_radiance = o;
  o = a256(o + cap * 4 * 3);
  L->off_vtx_ids = o;
  o = a256(o + cap * 4);
  L->off_vtx = o;
  o = a256(o + cap * 4 * kVtxPlanes);
  L->off_rec[0] = L->off_rec[1] = 0;
  if (guided) {
    for (int k = 0; k < 2; ++k) {
      L->off_rec[k] = o;
      o = a256(o + cap * 4);
    }
  }
  L->total = o;
  return true;
}

// scene and queue views over the caller's buffers; false on a missing array
bool make_views(const BajoRtScene* scene, unsigned char* w, const Layout& L, SceneView& sc, Queues& q) {
  const BajoLbvh* b = scene->bvh;
  if (!b->roots || !b->node_bounds || !b->node_meta || !b->leaf_tris || !scene->surfaces || !scene->lambertians ||
      !scene->emissives || (scene->n_lights && !scene->lights))
    return false;
  sc.roots = b->roots;
  sc.nb = reinterpret_cast<const float4*>(b->node_bounds);
  sc.meta = reinterpret_cast<const uint4*>(b->node_meta);
  sc.tris = reinterpret_cast<const float4*>(b->leaf_tris);
  sc.n_nodes = b->n_leaves;
  sc.surfaces = scene->surfaces;
  sc.lambertians = scene->lambertians;
  sc.emissives = scene->emissives;
  sc.lights = scene->lights;
  sc.n_lights = scene->n_lights;
  sc.total_light_weight = scene->total_light_weight;
  sc.metals = scene->metals;
  sc.dielectrics = scene->dielectrics;
  sc.has_materials = scene->metals || scene->dielectrics;
  // the compressed 8-wide tree, when the scene names one: a single-segment
  // build over the same triangles (bajo_cwbvh8_build of scene->bvh)
  sc.use_cw = scene->cwbvh8 != nullptr;
  sc.cw = cw::Tree{};
  if (sc.use_cw) {
    const BajoCwbvh8* c = scene->cwbvh8;
    if (c->n_segments != 1 || !c->nodes || !c->triangles || scene->cwbvh8_nodes == 0 ||
        ((uintptr_t)c->nodes & 15) || ((uintptr_t)c->triangles & 15))
      return false;
    sc.cw.nodes = reinterpret_cast<const float4*>(c->nodes);
    sc.cw.tris = reinterpret_cast<const float4*>(c->triangles);
    sc.cw.n_nodes = scene->cwbvh8_nodes;
    sc.cw.n_tris = c->n_tris;
  }
  for (int k = 0; k < 2; ++k) {
    q.ids[k] = (uint32_t*)(w + L.off_ids[k]);
    q.fields[k] = (float*)(w + L.off_fields[k]);
    q.rec[k] = L.off_rec[k] ? (uint32_t*)(w + L.off_rec[k]) : nullptr;
  }
  q.shadow_ids = (uint32_t*)(w + L.off_shadow_ids);
  q.shadow_fields = (float*)(w + L.off_shadow_fields);
  q.radiance = (float*)(w + L.off_radiance);
  q.counters = (uint32_t*)(w + L.off_counters);
  q.status = (uint32_t*)w;
  q.capacity = L.cap;
  return true;
}

ShadeCtx shade_ctx(unsigned char* w, const Layout& L, const Queues& q, uint32_t max_depth) {
  ShadeCtx c{};
  c.vtx_ids = (uint32_t*)(w + L.off_vtx_ids);
  c.vtx = (float*)(w + L.off_vtx);
  c.vcount = q.counters + 2 * max_depth + 2;
  c.mcount = c.vcount + max_depth;
  return c;
}

// Block sizes of the bounce kernels, chosen per launch from a process-wide
// table the autotuner fills (bajo_render_tuning_set): kind 0 = closest hit
// (trace_kernel), 1 = shading (shade_kernel), 2 = shadow rays
// (shadow_kernel); -1 = the built-in 128.  The reference fixes 64
// (GPU_RT_BLOCK_SIZE, bajo/rt/gpu/common_kernels.mojo:18).  The block size
// changes only the launch shape: every path's work and random numbers depend
// on its id, not on its queue slot, so every choice renders the same image.
constexpr int kRenderKinds = 3, kRenderVariants = 3;
constexpr int kRenderBlocks[kRenderVariants] = {128, 64, 256};
std::atomic<int8_t> g_render_tuning[kRenderKinds] = {{-1}, {-1}, {-1}};

int render_variant(int kind) {
  const int v = g_render_tuning[kind].load(std::memory_order_relaxed);
  return v >= 0 && v < kRenderVariants ? v : 0;
}

// grid of a grid-stride bounce kernel: one thread per queue slot, at most
// 2,048 threads per SM
uint32_t bounce_grid(uint32_t cap, int blk) {
  uint32_t grid = (cap + blk - 1) / blk;
  const uint32_t max_grid = (uint32_t)sm_count() * (2048u / (uint32_t)blk);
  return grid > max_grid ? max_grid : grid;
}

template <int ALGO, bool CW>
cudaError_t launch_trace(const SceneView& sc, const Queues& q, const ShadeCtx& c, uint32_t b, uint32_t sample_base,
                         cudaStream_t st) {
  const uint32_t cap = q.capacity;
  switch (render_variant(0)) {
    case 1: trace_kernel<ALGO, CW, 64><<<bounce_grid(cap, 64), 64, 0, st>>>(sc, q, c, b, sample_base); break;
    case 2: trace_kernel<ALGO, CW, 256><<<bounce_grid(cap, 256), 256, 0, st>>>(sc, q, c, b, sample_base); break;
    default: trace_kernel<ALGO, CW, 128><<<bounce_grid(cap, 128), 128, 0, st>>>(sc, q, c, b, sample_base);
  }
  return cudaGetLastError();
}

template <int ALGO>
cudaError_t launch_shade(const SceneView& sc, const Queues& q, const ShadeCtx& c, uint32_t b, uint32_t max_depth,
                         uint32_t sample_base, uint64_t seed, cudaStream_t st) {
  const uint32_t cap = q.capacity;
  switch (render_variant(1)) {
    case 1:
      shade_kernel<ALGO, 64><<<bounce_grid(cap, 64), 64, 0, st>>>(sc, q, c, b, max_depth, sample_base, seed);
      break;
    case 2:
      shade_kernel<ALGO, 256><<<bounce_grid(cap, 256), 256, 0, st>>>(sc, q, c, b, max_depth, sample_base, seed);
      break;
    default:
      shade_kernel<ALGO, 128><<<bounce_grid(cap, 128), 128, 0, st>>>(sc, q, c, b, max_depth, sample_base, seed);
  }
  return cudaGetLastError();
}

template <bool CW>
cudaError_t launch_shadow(const SceneView& sc, const Queues& q, uint32_t b, uint32_t sample_base, cudaStream_t st) {
  const uint32_t cap = q.capacity;
  switch (render_variant(2)) {
    case 1: shadow_kernel<CW, 64><<<bounce_grid(cap, 64), 64, 0, st>>>(sc, q, b, sample_base); break;
    case 2: shadow_kernel<CW, 256><<<bounce_grid(cap, 256), 256, 0, st>>>(sc, q, b, sample_base); break;
    default: shadow_kernel<CW, 128><<<bounce_grid(cap, 128), 128, 0, st>>>(sc, q, b, sample_base);
  }
  return cudaGetLastError();
}

template <int ALGO, bool CW>
cudaError_t launch_bounce_tree(const SceneView& sc, const Queues& q, const ShadeCtx& c, uint32_t grid, uint32_t b,
                               uint32_t max_depth, uint32_t sample_base, uint64_t seed, cudaStream_t st) {
  cudaError_t e = launch_trace<ALGO, CW>(sc, q, c, b, sample_base, st);
  if (e != cudaSuccess) return e;
  if ((e = launch_shade<ALGO>(sc, q, c, b, max_depth, sample_base, seed, st)) != cudaSuccess) return e;
  if (sc.has_materials) {
    material_kernel<ALGO, CW><<<grid, kBlock, 0, st>>>(sc, q, c, b, max_depth, seed);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (ALGO != BAJO_RENDER_PATH) e = launch_shadow<CW>(sc, q, b, sample_base, st);
  return e;
}

template <int ALGO>
cudaError_t launch_bounce(const SceneView& sc, const Queues& q, const ShadeCtx& c, uint32_t grid, uint32_t b,
                          uint32_t max_depth, uint32_t sample_base, uint64_t seed, cudaStream_t st) {
  return sc.use_cw ? launch_bounce_tree<ALGO, true>(sc, q, c, grid, b, max_depth, sample_base, seed, st)
                   : launch_bounce_tree<ALGO, false>(sc, q, c, grid, b, max_depth, sample_base, seed, st);
}

// Chunks of whole pixels: primary rays, `bounce(chunk, b)` per bounce, an
// optional per-chunk hook, the per-pixel resolve.
template <class Bounce, class Before, class After>
cudaError_t render_chunks(const BajoRenderSettings* s, const Layout& L, const Queues& q, const float* d_camera,
                          float* d_pixels, double* d_pixels64, unsigned long long* totals, cudaStream_t st,
                          Bounce bounce, Before before, After after) {
  const uint32_t n_pixels = s->width * s->height;
  cudaError_t e = cudaMemsetAsync(totals, 0, 16, st);
  if (e != cudaSuccess) return e;
  for (uint32_t pb = 0; pb < n_pixels; pb += L.pixels_per_chunk) {
    const uint32_t pc = std::min(L.pixels_per_chunk, n_pixels - pb);
    const uint32_t count = pc * s->spp;
    const uint32_t sample_base = pb * s->spp;
    if ((e = cudaMemsetAsync(q.counters, 0, (size_t)L.n_counters * 4, st)) != cudaSuccess) return e;
    if ((e = before()) != cudaSuccess) return e;
    // tiles when spp divides 32 (8 or fewer) and the chunk is whole rows of whole tiles
    uint32_t tw = 0, th = 0;
    switch (s->spp) {
      case 1: tw = 8; th = 4; break;
      case 2: tw = 4; th = 4; break;
      case 4: tw = 4; th = 2; break;
      case 8: tw = 2; th = 2; break;
      default: break;
    }
    if (tw && (pb % s->width != 0 || pc % s->width != 0 || s->width % tw != 0 || (pc / s->width) % th != 0))
      tw = th = 0;
    primary_kernel<<<(count + kBlock - 1) / kBlock, kBlock, 0, st>>>(d_camera, q, count, sample_base, s->width,
                                                                    s->height, s->spp, s->seed, tw, th);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    for (uint32_t bnc = 0; bnc < s->max_depth; ++bnc)
      if ((e = bounce(bnc, sample_base)) != cudaSuccess) return e;
    if ((e = after()) != cudaSuccess) return e;
    resolve_kernel<<<(pc + kBlock - 1) / kBlock, kBlock, 0, st>>>(q.radiance, L.cap, pb, pc, s->spp, d_pixels,
                                                                  d_pixels64, q.counters, s->max_depth, totals);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}


}  // namespace rt
}  // namespace bajo

extern "C" {

int32_t bajo_render_workspace_size(const BajoRenderSettings* settings, size_t* bytes) {
  bajo::rt::Layout L;
  if (!bytes || !bajo::rt::make_layout(settings, &L)) return BAJO_ERR_INVALID_ARGUMENT;
  *bytes = L.total;
  return BAJO_OK;
}

int32_t bajo_render(const BajoRtScene* scene, const float* d_camera, const BajoRenderSettings* s, float* d_pixels,
                    double* d_pixels64, void* d_ws, size_t ws_bytes, void* stream) {
  using namespace bajo;
  using namespace bajo::rt;
  Layout L;
  if (!scene || !scene->bvh || !d_camera || !d_pixels || !d_ws || !make_layout(s, &L)) return BAJO_ERR_INVALID_ARGUMENT;
  if (s->algorithm != BAJO_RENDER_PATH && s->algorithm != BAJO_RENDER_NEE && s->algorithm != BAJO_RENDER_MIS)
    return BAJO_ERR_INVALID_ARGUMENT;
  if (ws_bytes < L.total) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  SceneView sc;
  Queues q;
  unsigned char* w = (unsigned char*)d_ws;
  if (!make_views(scene, w, L, sc, q)) return BAJO_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t grid = bounce_grid(L.cap, kBlock);
  const int algo = s->algorithm;
  const ShadeCtx c = shade_ctx(w, L, q, s->max_depth);
  auto bounce = [&](uint32_t b, uint32_t sample_base) {
    if (algo == BAJO_RENDER_PATH)
      return launch_bounce<BAJO_RENDER_PATH>(sc, q, c, grid, b, s->max_depth, sample_base, s->seed, st);
    if (algo == BAJO_RENDER_NEE)
      return launch_bounce<BAJO_RENDER_NEE>(sc, q, c, grid, b, s->max_depth, sample_base, s->seed, st);
    return launch_bounce<BAJO_RENDER_MIS>(sc, q, c, grid, b, s->max_depth, sample_base, s->seed, st);
  };
  auto none = []() { return cudaSuccess; };
  const cudaError_t e = render_chunks(s, L, q, d_camera, d_pixels, d_pixels64, (unsigned long long*)(w + 8), st,
                                      bounce, none, none);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_render_guided(const BajoRtScene* scene, const float* d_camera, const BajoRenderSettings* s,
                           const BajoGuide* guide, float* d_pixels, double* d_pixels64, void* d_ws, size_t ws_bytes,
                           void* stream) {
  using namespace bajo;
  using namespace bajo::rt;
  Layout L;
  if (!scene || !scene->bvh || !d_camera || !d_pixels || !d_ws || !guide || !make_layout(s, &L))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (s->algorithm != BAJO_RENDER_GUIDED || !guide->params16 || !guide->box6 || !(guide->guide_fraction >= 0.0f) ||
      !(guide->guide_fraction <= 1.0f) || (guide->record_capacity && !guide->records))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (ws_bytes < L.total) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  SceneView sc;
  Queues q;
  unsigned char* w = (unsigned char*)d_ws;
  if (!make_views(scene, w, L, sc, q)) return BAJO_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  ShadeCtx gc = shade_ctx(w, L, q, s->max_depth);
  gc.params16 = (const __half*)guide->params16;
  gc.box = guide->box6;
  gc.frac = guide->guide_fraction;
  gc.rec_frac = guide->record_fraction;
  gc.rec_cap = guide->record_capacity;
  // without a record buffer the record counter lives in the workspace header
  // (bytes 24..31, after the status word and the two ray totals)
  unsigned char* rb = (unsigned char*)guide->records;
  const mlp::RecordLayout RL = mlp::record_layout(guide->record_capacity);
  gc.rec_hdr = rb ? (uint32_t*)rb : (uint32_t*)(w + 24);
  gc.rec_pos = rb ? (float*)(rb + RL.pos) : nullptr;
  gc.rec_nrm = rb ? (float*)(rb + RL.nrm) : nullptr;
  gc.rec_dir = rb ? (float*)(rb + RL.dir) : nullptr;
  gc.rec_weight = rb ? (float*)(rb + RL.weight) : nullptr;
  gc.rec_sidx = rb ? (uint32_t*)(rb + RL.sidx) : nullptr;
  gc.rec_tn = rb ? (float*)(rb + RL.tn) : nullptr;
  gc.rec_snap = rb ? (float*)(rb + RL.snap) : nullptr;
  gc.rec_wpre = rb ? (float*)(rb + RL.wpre) : nullptr;
  if (!rb) gc.rec_cap = 0;
  const size_t smem = sizeof(ShadeSmem);
  if (cudaFuncSetAttribute(guided_shade_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return BAJO_ERR_CUDA;
  // resident CTAs per SM: shared memory bounds them, and so does tensor
  // memory (128 of an SM's 512 columns per CTA)
  int per_sm = 0, sm_bytes = 0, dev = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, guided_shade_kernel, kShadeThreads, smem) !=
          cudaSuccess ||
      cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
    return BAJO_ERR_CUDA;
  per_sm = max(1, min(4, sm_bytes / (int)(smem + 1024)));
  uint32_t shade_grid = (L.cap + kShadeThreads - 1) / kShadeThreads;
  const uint32_t shade_max = (uint32_t)(sm_count() * per_sm);
  if (shade_grid > shade_max) shade_grid = shade_max;
  const uint32_t grid = bounce_grid(L.cap, kBlock);
  if (!rb && cudaMemsetAsync(gc.rec_hdr, 0, 8, st) != cudaSuccess) return BAJO_ERR_CUDA;
  auto bounce = [&](uint32_t b, uint32_t sample_base) {
    cudaError_t e = sc.use_cw ? launch_trace<BAJO_RENDER_GUIDED, true>(sc, q, gc, b, sample_base, st)
                              : launch_trace<BAJO_RENDER_GUIDED, false>(sc, q, gc, b, sample_base, st);
    if (e != cudaSuccess) return e;
    guided_shade_kernel<<<shade_grid, kShadeThreads, smem, st>>>(sc, q, gc, b, s->max_depth, sample_base, s->seed);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (sc.has_materials) {
      if (sc.use_cw)
        material_kernel<BAJO_RENDER_GUIDED, true><<<grid, kBlock, 0, st>>>(sc, q, gc, b, s->max_depth, s->seed);
      else
        material_kernel<BAJO_RENDER_GUIDED, false><<<grid, kBlock, 0, st>>>(sc, q, gc, b, s->max_depth, s->seed);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return sc.use_cw ? launch_shadow<true>(sc, q, b, sample_base, st) : launch_shadow<false>(sc, q, b, sample_base, st);
  };
  auto before = [&]() {
    if (gc.rec_cap == 0) return cudaSuccess;
    records_begin_chunk_kernel<<<1, 1, 0, st>>>(gc.rec_hdr, gc.rec_cap);
    return cudaGetLastError();
  };
  auto after = [&]() {
    if (gc.rec_cap == 0) return cudaSuccess;
    records_finish_chunk_kernel<<<grid, kBlock, 0, st>>>(gc, q.radiance, L.cap);
    return cudaGetLastError();
  };
  const cudaError_t e = render_chunks(s, L, q, d_camera, d_pixels, d_pixels64, (unsigned long long*)(w + 8), st,
                                      bounce, before, after);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_render_tuning_set(int32_t kernel, int32_t block) {
  using namespace bajo::rt;
  if (kernel < 0 || kernel >= kRenderKinds) return BAJO_ERR_INVALID_ARGUMENT;
  int v = -1;
  for (int k = 0; k < kRenderVariants; ++k)
    if (kRenderBlocks[k] == block) v = k;
  if (block != 0 && v < 0) return BAJO_ERR_INVALID_ARGUMENT;
  g_render_tuning[kernel].store((int8_t)v);
  return BAJO_OK;
}

int32_t bajo_render_tuning_get(int32_t kernel, int32_t* block) {
  using namespace bajo::rt;
  if (kernel < 0 || kernel >= kRenderKinds || !block) return BAJO_ERR_INVALID_ARGUMENT;
  *block = kRenderBlocks[render_variant(kernel)];
  return BAJO_OK;
}

int32_t bajo_render_stats(const void* d_ws, void* stream, uint64_t* rays, uint64_t* shadow_rays) {
  if (!d_ws || !rays || !shadow_rays) return BAJO_ERR_INVALID_ARGUMENT;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return BAJO_ERR_CUDA;
  unsigned long long t[2];
  if (cudaMemcpy(t, (const unsigned char*)d_ws + 8, 16, cudaMemcpyDeviceToHost) != cudaSuccess) return BAJO_ERR_CUDA;
  *rays = t[0];
  *shadow_rays = t[1];
  return BAJO_OK;
}

// LightStore._build_light_store + build_alias_table (bajo/rt/types.mojo:
// 190-247, 490-525): one record per emissive triangle with positive power
// area * mean(radiance); Walker-Vose alias table with the reference's
// small / large stacks.
int32_t bajo_rt_build_lights(const float* v, const uint32_t* surf, uint32_t n, const float* em, uint32_t n_em,
                             float* out, uint32_t max_lights, uint32_t* n_lights, float* total_weight) {
  if (!v || !surf || !n_lights || !total_weight || (max_lights && !out)) return BAJO_ERR_INVALID_ARGUMENT;
  struct Rec {
    uint32_t tri;
    float w;
  };
  std::vector<Rec> recs;
  float total = 0.0f;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t s = surf[i];
    if ((s >> 28) != BAJO_MAT_EMISSIVE) continue;
    const uint32_t m = s & 0x0FFFFFFFu;
    if (m >= n_em || !em) return BAJO_ERR_INVALID_ARGUMENT;
    const float* p = v + (size_t)9 * i;
    const float e1x = p[3] - p[0], e1y = p[4] - p[1], e1z = p[5] - p[2];
    const float e2x = p[6] - p[0], e2y = p[7] - p[1], e2z = p[8] - p[2];
    const float cx = std::fmaf(e1y, e2z, -(e1z * e2y));
    const float cy = std::fmaf(e1z, e2x, -(e1x * e2z));
    const float cz = std::fmaf(e1x, e2y, -(e1y * e2x));
    const float len2 = std::fmaf(cx, cx, std::fmaf(cy, cy, cz * cz));
    const float area = 0.5f * std::sqrt(len2);
    const float* L = em + 3 * (size_t)m;
    const float imp = std::max(((L[0] + L[1]) + L[2]) / 3.0f, 0.0f);
    const float w = area * imp;
    if (w > 0.0f) {
      total += w;
      recs.push_back({i, w});
    }
  }
  const uint32_t count = (uint32_t)recs.size();
  if (count > max_lights) return BAJO_ERR_TOO_LARGE;
  std::vector<float> prob(count, 1.0f), scaled(count, 0.0f);
  std::vector<uint32_t> alias(count, 0);
  if (count > 0 && total > 0.0f) {
    std::vector<uint32_t> small, large;
    for (uint32_t i = 0; i < count; ++i) {
      alias[i] = i;
      scaled[i] = recs[i].w * (float)count / total;
      if (scaled[i] < 1.0f) small.push_back(i);
      else large.push_back(i);
    }
    while (!small.empty() && !large.empty()) {
      const uint32_t si = small.back();
      small.pop_back();
      const uint32_t li = large.back();
      large.pop_back();
      prob[si] = scaled[si];
      alias[si] = li;
      scaled[li] = scaled[li] + scaled[si] - 1.0f;
      if (scaled[li] < 1.0f) small.push_back(li);
      else large.push_back(li);
    }
    for (uint32_t i : small) {
      prob[i] = 1.0f;
      alias[i] = i;
    }
    for (uint32_t i : large) {
      prob[i] = 1.0f;
      alias[i] = i;
    }
  }
  for (uint32_t k = 0; k < count; ++k) {
    float* r = out + (size_t)k * BAJO_LIGHT_STRIDE;
    const float* p = v + (size_t)9 * recs[k].tri;
    for (int j = 0; j < 9; ++j) r[j] = p[j];
    const float* L = em + 3 * (size_t)(surf[recs[k].tri] & 0x0FFFFFFFu);
    r[9] = L[0];
    r[10] = L[1];
    r[11] = L[2];
    r[12] = prob[k];
    std::memcpy(&r[13], &alias[k], 4);
    r[14] = 0.0f;
    r[15] = 0.0f;
  }
  *n_lights = count;
  *total_weight = total;
  return BAJO_OK;
}

}  // extern "C"
