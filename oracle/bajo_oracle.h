/*
 * bajo_oracle.h -- CPU oracle for the LBVH build + closest-hit path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * (jgsimard/bajo, pure Mojo) algorithms on the GPU LBVH / traversal path.  It
 * exists to check the CUDA library bit-for-bit and to provide the timed CPU
 * baseline.  Nothing in the product library links, loads or calls it; only the
 * tests, the smoke check and the benchmark's CPU-baseline leg do.
 *
 * Every function cites the reference file:line it follows.  Where this oracle
 * deliberately differs from the reference it says so (tie rule, conservative
 * box test, watertight triangle test).
 *
 * Floating point: compiled with -ffp-contract=off so that every product and
 * sum is rounded exactly as written; fused multiply-adds appear only where the
 * reference spells fma() itself (bajo/core/vec.mojo:440, :523-525).
 */
#ifndef BAJO_ORACLE_H
#define BAJO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Inline min / max.  bo_fminf / bo_fmaxf give C99 fminf / fmaxf results for
 * every quiet operand: the smaller (larger) of two numbers as `a < b ? a : b`
 * (`a > b ? a : b`), which is the reference's fmin / fmax
 * (bajo/core/utils.mojo:60-70), and the other operand when one is NaN.  On
 * x86-64 they are branch free (SSE minss / maxss, whose unordered and equal
 * cases return the second operand, plus a NaN mask on b); without
 * -ffast-math the compiler would otherwise call libm or branch per compare,
 * which cost the CPU builder most of its time. */
#if defined(__x86_64__) || defined(__SSE2__)
#include <emmintrin.h>
static inline float bo_fminf(float a, float b) {
  const __m128 va = _mm_set_ss(a), vb = _mm_set_ss(b);
  const __m128 nan_b = _mm_cmpunord_ss(vb, vb);
  return _mm_cvtss_f32(_mm_or_ps(_mm_and_ps(nan_b, va), _mm_andnot_ps(nan_b, _mm_min_ss(va, vb))));
}
static inline float bo_fmaxf(float a, float b) {
  const __m128 va = _mm_set_ss(a), vb = _mm_set_ss(b);
  const __m128 nan_b = _mm_cmpunord_ss(vb, vb);
  return _mm_cvtss_f32(_mm_or_ps(_mm_and_ps(nan_b, va), _mm_andnot_ps(nan_b, _mm_max_ss(va, vb))));
}
#else
static inline float bo_fminf(float a, float b) { return b != b ? a : (a < b ? a : b); }
static inline float bo_fmaxf(float a, float b) { return b != b ? a : (a > b ? a : b); }
#endif
/* Number of (a, b) pairs over special and random values (signalling NaNs
 * excluded: libm quiets them) where bo_fminf / bo_fmaxf differ from libm's
 * fminf / fmaxf bit for bit (0 = identical). */
uint32_t bo_minmax_selftest(uint32_t n_random, uint64_t seed);

#define BO_SENTINEL 0xFFFFFFFFu   /* LBVH_SENTINEL, bajo/bvh/constants.mojo:6 */
#define BO_LEAF_FLAG 0x80000000u  /* _BVH_LEAF_FLAG, bajo/bvh/tagged_ref.mojo:3 */
#define BO_EMPTY 0xFFFFFFFFu      /* EMPTY_LANE / MISS_PRIM, constants.mojo:19-20 */

/* triangle test selector */
#define BO_TRI_MT 0          /* Moller-Trumbore, bajo/core/intersect.mojo:415 */
#define BO_TRI_WATERTIGHT 1  /* Woop/Benthin/Wald 2013 watertight test */

/* ---- a1: per-triangle AABB (bajo/bvh/gpu/triangle_bvh.mojo:680) ---------- */
void bo_triangle_bounds(const float* verts, uint32_t n, float* bounds6);

/* ---- a2: per-segment root + centroid bounds, 12 floats per segment
 *      (bajo/bvh/gpu/builder/binary_layout.mojo:128-205) -------------------- */
void bo_segment_bounds(const float* bounds6, const uint32_t* seg_offsets,
                       uint32_t n_segments, float* seg_bounds12);

/* ---- a3: Morton composite keys (bajo/bvh/gpu/builder/lbvh.mojo:30) -------- */
uint32_t bo_expand_bits_3d(uint32_t v);                  /* core/morton.mojo:48 */
uint32_t bo_morton3(float x, float y, float z);          /* core/morton.mojo:61 */
int bo_morton_common_prefix(uint32_t ca, uint32_t ia,
                            uint32_t cb, uint32_t ib);   /* core/morton.mojo:22 */
void bo_morton_keys(const float* bounds6, const uint32_t* seg_offsets,
                    uint32_t n_segments, const float* seg_bounds12,
                    uint32_t n, uint64_t* keys, uint32_t* values);

/* ---- a4/a5: stable LSD radix sort, 8-bit digits --------------------------- */
void bo_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint32_t n,
                       int begin_bit, int end_bit);
void bo_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t n,
                       int begin_bit, int end_bit);
void bo_sort_keys_u32(uint32_t* keys, uint32_t n, int begin_bit, int end_bit);
/* Multithreaded stable LSD radix sort (the CPU sort baseline; the reference
 * CPU builder's parallel pass, bajo/bvh/cpu/builder/lbvh.mojo:65-110), keys
 * of key_bytes (4 or 8) with optional u32 values (vals may be NULL), into
 * caller-owned scratch of bo_cpu_sort_scratch_bytes bytes. */
size_t bo_cpu_sort_scratch_bytes(uint32_t n, uint32_t key_bytes, int has_values, uint32_t n_threads);
void bo_cpu_sort(void* keys, uint32_t* vals, uint32_t n, uint32_t key_bytes, int begin_bit, int end_bit,
                 uint32_t n_threads, void* scratch);
/* 63-bit Morton codes of points (3 floats each) in the unit cube, 21 bits per
 * axis: the sort workload's 64-bit keys. */
void bo_morton63(const float* xyz, uint32_t n, uint64_t* out);
void bo_sort_keys_u64(uint64_t* keys, uint32_t n, int begin_bit, int end_bit);

/* ---- a8: internal segment offsets (binary_layout.mojo:219) --------------- */
void bo_internal_offsets(const uint32_t* seg_offsets, uint32_t n_segments,
                         uint32_t* internal_offsets);

/* ---- a7/a8: Karras topology, bottom-up per node, GPU node numbering
 *      (lbvh.mojo:164-330).  node_meta is 4 u32 per internal node
 *      [parent, left, right, fence]; node_bounds (12 f32) initialised invalid.
 * ------------------------------------------------------------------------- */
void bo_lbvh_topology(const uint32_t* sorted_codes, const uint32_t* seg_offsets,
                      const uint32_t* internal_offsets, uint32_t n_segments,
                      uint32_t* node_meta, uint32_t* leaf_parent,
                      uint32_t* node_leaf_counts, uint32_t* roots,
                      float* node_bounds);
/* Top-down cross-check (bajo/bvh/cpu/builder/lbvh.mojo:144,270): same tree,
 * numbered with the Karras rule (root 0, children `split` / `split+1`). */
void bo_lbvh_topology_topdown(const uint32_t* sorted_codes,
                              const uint32_t* seg_offsets,
                              const uint32_t* internal_offsets,
                              uint32_t n_segments, uint32_t* node_meta,
                              uint32_t* leaf_parent, uint32_t* node_leaf_counts,
                              uint32_t* roots);

/* ---- a9: refit (lbvh.mojo:116) -> node_bounds, node_flags (==2) ----------- */
void bo_lbvh_refit(const float* leaf_bounds6, const uint32_t* leaf_ids,
                   const uint32_t* node_meta, const uint32_t* leaf_parent,
                   uint32_t n_leaves, uint32_t n_internal, float* node_bounds,
                   uint32_t* node_flags);

/* ---- full single-call build (Morton -> sort -> topology -> refit) --------- */
typedef struct BoLbvh {
  uint32_t n_leaves, n_internal, n_segments;
  float* leaf_bounds;        /* 6 * n_leaves                */
  float* seg_bounds;         /* 12 * n_segments             */
  uint64_t* sort_keys;       /* n_leaves, sorted            */
  uint32_t* leaf_ids;        /* n_leaves, sorted item ids   */
  uint32_t* morton_codes;    /* n_leaves, sorted low words  */
  uint32_t* node_meta;       /* 4 * max(n_internal,1)       */
  float* node_bounds;        /* 12 * max(n_internal,1)      */
  uint32_t* node_leaf_counts;/* max(n_internal,1)           */
  uint32_t* node_flags;      /* max(n_internal,1)           */
  uint32_t* leaf_parent;     /* n_leaves                    */
  uint32_t* roots;           /* n_segments                  */
  uint32_t* internal_offsets;/* n_segments + 1              */
  const uint32_t* seg_offsets; /* n_segments + 1, set by bo_lbvh_build */
} BoLbvh;
void bo_lbvh_build(const float* verts, const uint32_t* seg_offsets,
                   uint32_t n_segments, BoLbvh* out);

/* ---- a12: camera (bajo/bvh/camera.mojo:19-154) ----------------------------- */
/* 20-float camera record from origin/target/world_up and a vertical FOV in
 * degrees (Camera.from_vfov, camera.mojo:100). */
void bo_camera_from_vfov(const float origin[3], const float target[3],
                         const float world_up[3], float vfov_deg,
                         float out20[20]);
/* Camera.__init__ with an explicit fov_scale (camera.mojo:77). */
void bo_camera_make(const float origin[3], const float target[3],
                    const float world_up[3], float fov_scale, float out20[20]);
/* make_ray_raster (camera.mojo:137) via _camera_ray (camera_launch.mojo:34):
 * writes rays SoA, 8 planes x n ([ox,oy,oz,tmin,dx,dy,dz,tmax]). */
void bo_camera_rays(const float* cameras20, uint32_t n_rays, uint32_t width,
                    uint32_t height, float* rays_soa);

/* ---- a11: closest hit ------------------------------------------------------ */
/* Hit AoS, 8 words per ray: [u, v, prim, inst, nx, ny, nz, t]
 * (bajo/bvh/types.mojo:16-27).  Triangle records are read straight from the
 * 9-float vertex buffer through leaf_ids. */
void bo_trace_bvh2(const BoLbvh* bvh, const float* verts, const float* rays_soa,
                   uint32_t n_rays, int tri_mode, float* hits8,
                   uint32_t n_threads);
/* All triangles, no BVH: the order-free reference answer. */
void bo_trace_brute(const float* verts, uint32_t n_tris, const float* rays_soa,
                    uint32_t n_rays, int tri_mode, float* hits8,
                    uint32_t n_threads);
/* per-ray traversal counters on the BVH2 in the layout of GpuTraversalStats
 * (bajo/bvh/gpu/trace.mojo:62-90): stats[5*i + 0..4] = internal nodes
 * visited, internal children hit, leaf blocks entered, triangles tested,
 * deepest stack */
void bo_trace_bvh2_stats(const BoLbvh* bvh, const float* verts,
                         const float* rays_soa, uint32_t n_rays, int tri_mode,
                         uint32_t* stats);

/* ---- reference CPU builder, timed CPU baseline ---------------------------- */
/* bajo/bvh/cpu/builder/lbvh.mojo:166-359 restated with pthreads: parallel
 * Morton, parallel stable LSD radix sort, top-down parallel frontier build
 * (depth 3) with recursive AABB merge.  Returns the node count. */
typedef struct BoCpuNode {
  float bmin[3], bmax[3];
  uint32_t left_or_first; /* internal: left child index; leaf: first item */
  uint32_t count;         /* 0 = internal, else leaf item count          */
} BoCpuNode;
uint32_t bo_cpu_build_lbvh(const float* verts, uint32_t n, uint32_t n_threads,
                           BoCpuNode* nodes /* 2n-1 */,
                           uint32_t* item_indices /* n */);
/* The same build into caller-owned scratch of bo_cpu_lbvh_scratch_bytes(n,
 * n_threads) bytes (no allocation inside the build, as the reference keeps
 * its builder's buffers across rebuilds). */
size_t bo_cpu_lbvh_scratch_bytes(uint32_t n, uint32_t n_threads);
uint32_t bo_cpu_build_lbvh_scratch(const float* verts, uint32_t n, uint32_t n_threads,
                                   BoCpuNode* nodes, uint32_t* item_indices, void* scratch);
void bo_cpu_trace(const BoCpuNode* nodes, const uint32_t* item_indices,
                  const float* verts, const float* rays_soa, uint32_t n_rays,
                  int tri_mode, float* hits8, uint32_t n_threads);

/* ---- wavefront path tracer (PATH=0 / NEE=3 / MIS=4) ---------------------- */
/* Philox-4x32-10 block (Salmon et al., SC'11) */
void bo_rt_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void bo_rt_uniform4(uint64_t seed, uint32_t path_id, uint32_t stage, float out[4]);
void bo_rt_sincos_turns(float u, float* s, float* c);
int bo_rt_build_lights(const float* verts, const uint32_t* surfaces, uint32_t n_tris, const float* emissives,
                       float* out_lights, uint32_t max_lights, uint32_t* n_lights, float* total_weight);
/* x^y by the series the metal lobe uses (see sampling.cuh) */
float bo_rt_series_pow(float x, float y);
void bo_render(const BoLbvh* bvh, const float* verts, const uint32_t* surfaces, const float* lambertians,
               const float* emissives, const float* metals, const float* dielectrics, const float* lights,
               uint32_t n_lights, float total_weight,
               const float* camera20, uint32_t width, uint32_t height, uint32_t spp, uint32_t max_depth,
               uint64_t seed, int algorithm, float* pixels, float* sample_radiance, uint32_t n_threads);
/* bo_render through a compressed 8-wide tree (from bo_cwbvh8_build of the
 * scene's single-segment tree) instead of the binary LBVH. */
void bo_render_cwbvh8(const float* cw_nodes, uint32_t cw_n_nodes, const float* cw_tris, uint32_t cw_n_tris,
                      const float* verts, const uint32_t* surfaces, const float* lambertians, const float* emissives,
                      const float* metals, const float* dielectrics, const float* lights, uint32_t n_lights,
                      float total_weight, const float* cam, uint32_t width, uint32_t height, uint32_t spp,
                      uint32_t max_depth, uint64_t seed, int algorithm, float* pixels, float* sample_radiance,
                      uint32_t n_threads);

/* batched primary + one cosine bounce per pixel, segmented LBVH */
void bo_trace_batch(const BoLbvh* bvh, const float* verts, const float* cams, uint32_t cam_stride, uint32_t width,
                    uint32_t height, uint64_t seed, int mode, float* t0, uint32_t* p0, float* t1, uint32_t* p1,
                    uint32_t n_threads);
/* The same over the segments of `bvh` taken as views view_base, view_base+1,
 * ... of a larger batch: the bounce rays draw the random streams of their
 * index in that batch, so a scene built alone reproduces its rays there. */
void bo_trace_batch_views(const BoLbvh* bvh, const float* verts, const float* cams, uint32_t cam_stride,
                          uint32_t width, uint32_t height, uint64_t seed, int mode, uint32_t view_base, float* t0,
                          uint32_t* p0, float* t1, uint32_t* p1, uint32_t n_threads);

/* ---- a10: BVH2 -> W-wide collapse (bajo_oracle_wide.c) ------------------- */
/* Outputs sized for n_leaves nodes and leaf blocks; offsets [S+1];
 * max_leaf = triangles per leaf block (1..4, 0 = 4). */
void bo_wide_build(const BoLbvh* b, const float* verts, uint32_t width, uint32_t max_leaf, float* nodes,
                   uint32_t* leaf_indices, float* leaf_tris, uint32_t* leaf_sorted, uint32_t* node_offsets,
                   uint32_t* leaf_offsets);

/* ---- two-level trees (bajo_oracle.c) ------------------------------------- */
/* instance boxes as [min, max, min] records (see bajo_tlas_instance_boxes) */
void bo_tlas_instance_boxes(const float* seg_bounds, uint32_t n_blas, const float* transforms12,
                            const uint32_t* blas, uint32_t n, float* out9);
/* closest (any = 0) or any hit of SoA rays through `top` (an LBVH over the
 * instance boxes) and the segmented BLAS set `blas` (vertices blas_verts);
 * inv = world -> BLAS transforms (12 f32 each); hits8 with inst set */
void bo_trace_tlas(const BoLbvh* top, const BoLbvh* blas, const float* blas_verts, const float* inv,
                   const uint32_t* blas_idx, uint32_t n_inst, const float* rays, uint32_t n, int any, int mode,
                   float* hits8);

/* ---- H-PLOC (bajo_oracle_hploc.c) ---------------------------------------- */
/* The H-PLOC tree of the sorted leaves of `karras` (an LBVH built by
 * bo_lbvh_build: its leaf bounds, sorted ids, codes and offsets), written to
 * out's node_meta / node_bounds / node_leaf_counts / node_flags /
 * leaf_parent / roots (arrays distinct from karras's).  Returns 0, or bit 0 =
 * a PLOC round found no mutual pair, bit 1 = a segment's node count is off. */
uint32_t bo_hploc_build(const BoLbvh* karras, BoLbvh* out);

/* ---- CWBVH8 (bajo_oracle_wide.c, bajo_oracle.c) -------------------------- */
/* W = 8 collapse with octant slots and leaves of <= 3 triangles, encoded as
 * 80-byte nodes (20 words, `cw_nodes` sized for n_leaves nodes) and 48-byte
 * triangle records (12 words, n_leaves records); `wide_nodes` (n_leaves x 56
 * words) receives the uncompressed wide nodes; node_offsets [S+1]. */
void bo_cwbvh8_build(const BoLbvh* b, const float* verts, float* wide_nodes, float* cw_nodes, float* cw_tris,
                     uint32_t* node_offsets);
/* closest (any_hit = 0) or any hit of SoA rays over one CWBVH8 tree rooted at
 * node 0; hits8 as bo_trace_bvh2; err (may be NULL) per ray: bit 0 = node or
 * triangle out of range / too many visits, bit 1 = stack overflow */
void bo_trace_cwbvh8(const float* nodes, uint32_t n_nodes, const float* tris, uint32_t n_tris, const float* rays,
                     uint32_t n, int any_hit, float* hits8, uint32_t* err, uint32_t n_threads);

/* ---- path-guiding network (bajo_oracle_mlp.c), FP64 ---------------------- */
/* Parameters as doubles in the library's layout: W1[64x64] b1[64] W2 b2 W3 b3
 * W4[32x64] b4[32] (rows 20..31 of the output layer unused). */
uint32_t bo_mlp_param_count(void);
void bo_mlp_encode(const float* p, const float* n, const float* box6, float* feat64);
void bo_mlp_forward_f64(const double* params, const float* pos, const float* nrm, const float* box6, uint32_t n,
                        double* out20);
double bo_vmf_mixture_pdf(const double* out20, const float* dir);
double bo_mlp_loss_f64(const double* params, const float* pos, const float* nrm, const float* dir, const float* w,
                       uint32_t n, const float* box6);
double bo_mlp_grad_f64(const double* params, const float* pos, const float* nrm, const float* dir, const float* w,
                       uint32_t n, const float* box6, double* grad);

#ifdef __cplusplus
}
#endif
#endif
