/*
 * bajo_b200.h -- C ABI of the sm_100a LBVH build + closest-hit library.
 *
 * Drop-in boundary for the GPU path of jgsimard/bajo (Mojo).  The reference
 * exposes this path as Mojo generics over a DeviceContext; a Mojo host binds
 * these symbols with `external_call` / `DLHandle` instead.
 *
 * Conventions
 *  - Every pointer named d_* is DEVICE memory allocated by the caller.  The
 *    library never allocates: size queries (bajo_*_size) tell the caller how
 *    much workspace to provide.
 *  - `stream` is a cudaStream_t passed as void* (0 = legacy default stream).
 *    Calls only enqueue work; nothing synchronises unless the name says so.
 *  - Every function returns an int32 status (BAJO_OK = 0).  Errors found on
 *    the device (look-back timeout, traversal stack overflow) are OR-ed into a
 *    status word at the start of the workspace; read it with
 *    bajo_workspace_status after the stream has run.
 *  - Buffer layouts are the reference's (cited per field).
 */
#ifndef BAJO_B200_H
#define BAJO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (mirrors the reference's raise sites and device status
 *      words: bajo/rt/wavefront_contract.mojo:25-29,
 *      bajo/bvh/gpu/builder/wide_collapse.mojo:34-38) ----------------------- */
#define BAJO_OK 0
#define BAJO_ERR_INVALID_ARGUMENT 1
#define BAJO_ERR_WORKSPACE_TOO_SMALL 2
#define BAJO_ERR_TOO_LARGE 3
#define BAJO_ERR_CUDA 4
#define BAJO_ERR_DEVICE 5 /* a device status bit is set */

/* device status word bits */
#define BAJO_STATUS_LOOKBACK_TIMEOUT 0x1u /* sort look-back gave up waiting    */
#define BAJO_STATUS_STACK_OVERFLOW 0x2u   /* traversal stack would overflow    */
#define BAJO_STATUS_BAD_TOPOLOGY 0x4u     /* refit met an inconsistent parent  */
#define BAJO_STATUS_WIDE_TIMEOUT 0x40u    /* wide collapse gave up on a task   */
#define BAJO_STATUS_STAGE_TIMEOUT 0x80u   /* staged top levels did not arrive  */
#define BAJO_STATUS_WAIT_TIMEOUT 0x100u   /* bajo_wait_selftest gave up        */
#define BAJO_STATUS_GRID_TIMEOUT 0x200u   /* one-launch build: a grid barrier  */
                                          /* wait gave up                      */

/* triangle tests */
#define BAJO_TRI_MT 0         /* Moller-Trumbore, bajo/core/intersect.mojo:415 */
#define BAJO_TRI_WATERTIGHT 1 /* Woop/Benthin/Wald 2013 watertight test        */

/* Largest key count one sort call accepts (30-bit look-back counters). */
#define BAJO_SORT_MAX_KEYS ((1u << 30) - 1u)

/* ======================================================================== */
/* Workspace status                                                          */
/* ======================================================================== */
/* Synchronises `stream`, then copies the device status word that starts every
 * workspace into *status (0 = no device error). */
int32_t bajo_workspace_status(const void* d_workspace, void* stream, uint32_t* status);
/* Enqueues a reset of the status word to 0. */
int32_t bajo_workspace_status_clear(void* d_workspace, void* stream);

/* ======================================================================== */
/* Onesweep radix sort (stable, LSD, 8-bit digits, decoupled look-back)       */
/* ======================================================================== */
/* Replaces bajo/sort/gpu/onesweep.mojo:362 onesweep_radix_sort_keys,
 * :454 onesweep_radix_sort_pairs and bajo/sort/gpu/radix_sort.mojo:510
 * device_radix_sort_pairs (the sort the LBVH calls, lbvh.mojo:101).
 * Sorts bits [begin_bit, end_bit) in place: the result lands in d_keys /
 * d_vals, as the reference's DoubleBuffer does after an even pass count
 * (bajo/sort/gpu/utils.mojo:8-37).  Workspace holds the alternate buffers,
 * the digit histograms and the look-back flags.  n <= BAJO_SORT_MAX_KEYS. */
int32_t bajo_sort_workspace_size(uint32_t n, uint32_t key_bytes, int32_t has_values, int32_t begin_bit,
                                 int32_t end_bit, size_t* bytes);
int32_t bajo_sort_keys_u32(uint32_t* d_keys, uint32_t n, int32_t begin_bit, int32_t end_bit, void* d_workspace,
                           size_t workspace_bytes, void* stream);
int32_t bajo_sort_pairs_u32(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, int32_t begin_bit, int32_t end_bit,
                            void* d_workspace, size_t workspace_bytes, void* stream);
int32_t bajo_sort_keys_u64(uint64_t* d_keys, uint32_t n, int32_t begin_bit, int32_t end_bit, void* d_workspace,
                           size_t workspace_bytes, void* stream);
int32_t bajo_sort_pairs_u64(uint64_t* d_keys, uint32_t* d_vals, uint32_t n, int32_t begin_bit, int32_t end_bit,
                            void* d_workspace, size_t workspace_bytes, void* stream);

/* Autotuner hooks.  The sort kernels come in compiled variants (tile shape:
 * threads x keys per thread, digit width, pass kernel): BAJO_SORT_VARIANTS_U32
 * for 32-bit keys and BAJO_SORT_VARIANTS_U64 for 64-bit keys; the library
 * picks one per call from a process-wide table indexed by (key bytes, values,
 * ceil(log2 n)), filled by the project's autotuner (bajo_b200/autotune.py) or
 * left at -1 for the built-in choice.  Set entries before sorting, not
 * concurrently with sorts.  bajo_sort_tuning_get reports the variant a call
 * of size n would use. */
#define BAJO_SORT_VARIANTS_U32 7
#define BAJO_SORT_VARIANTS_U64 7
#define BAJO_SORT_VARIANTS 7 /* the larger of the two */
int32_t bajo_sort_tuning_set(uint32_t key_bytes, int32_t has_values, uint32_t log2n, int32_t variant);
int32_t bajo_sort_tuning_get(uint32_t key_bytes, int32_t has_values, uint32_t n, int32_t* variant);

/* Sort without any allocation by the library or the caller, for callers that
 * cannot call cudaMalloc or provide a workspace: hosts that own all device
 * memory and pass only the buffers they compute on, or frame loops where an
 * allocation would stall the device.  No counterpart in the reference.  Same
 * result as bajo_sort_pairs_u32 (stable, in place).  Its scratch is one fixed
 * device array inside the library (BAJO_SORT_NOALLOC_SCRATCH_BYTES, about
 * 10.5 MB, held on every GPU that loads the library until exit), so
 * n <= BAJO_SORT_NOALLOC_MAX_KEYS; larger n returns BAJO_ERR_TOO_LARGE.  All
 * calls on a device share that array: calls whose device work overlaps race
 * and must be serialised by the caller.  The first call on a device looks up
 * the array's address; make it before any stream capture.  Every call made
 * outside a capture looks the address up again, so after a device reset the
 * next uncaptured call uses the reloaded array.  d_status (may be NULL)
 * receives the BAJO_STATUS_* bits of this call. */
#define BAJO_SORT_NOALLOC_MAX_KEYS (1u << 20)
#define BAJO_SORT_NOALLOC_SCRATCH_BYTES 10490368u
int32_t bajo_sort_pairs_u32_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, int32_t begin_bit,
                                    int32_t end_bit, uint32_t* d_status, void* stream);

/* ======================================================================== */
/* LBVH build                                                                */
/* ======================================================================== */
/* Device buffers of one (optionally segmented) binary LBVH.  Field layouts
 * follow GpuBinaryBoundsBvh (bajo/bvh/gpu/builder/binary_layout.mojo:303-329)
 * and GpuBinaryTopologyWorkspace (:226-249).  N = n_leaves (triangles),
 * S = n_segments, M = max(N, 1) (upper bound on internal nodes). */
typedef struct BajoLbvh {
  uint32_t n_leaves;           /* N                                                      */
  uint32_t n_segments;         /* S >= 1                                                 */
  const uint32_t* seg_offsets; /* S+1 item offsets, [0] = 0, [S] = N (input)             */
  uint32_t* internal_offsets;  /* S+1 internal-node offsets, max(count-1,0) per segment  */
  float* leaf_bounds;          /* 6*N   per-item AABB [min xyz, max xyz]  (item order)    */
  float* seg_bounds;           /* 12*S  root AABB then centroid AABB per segment          */
  uint64_t* sort_keys;         /* N     sorted (segment << 32) | morton                   */
  uint32_t* leaf_ids;          /* N     sorted item ids (sort payload)                    */
  uint32_t* morton_codes;      /* N     low 32 bits of sort_keys                          */
  uint32_t* node_meta;         /* 4*M   [parent, left, right, fence], tagged child refs   */
  float* node_bounds;          /* 12*M  left-child AABB then right-child AABB             */
                               /* node_meta, node_bounds and leaf_tris are read and       */
                               /* written 16 bytes at a time: 16-byte aligned (the build  */
                               /* and the traversals refuse others)                       */
  uint32_t* node_leaf_counts;  /* M     leaves under each internal node                   */
  uint32_t* node_flags;        /* M     refit arrival counters (2 after a build)          */
  uint32_t* leaf_parent;       /* N     parent internal node of each sorted leaf          */
  uint32_t* roots;             /* S     tagged root ref per segment (SENTINEL if empty)   */
  float* leaf_tris;            /* 12*N  sorted triangle records [v0,prim | v1,0 | v2,0]   */
  float* top_nodes;            /* optional (NULL = none): BAJO_TOP_BYTES, the top levels  */
                               /* of segment 0's tree for the traversal (see below)       */
} BajoLbvh;

/* Staged top levels.  When bvh->top_nodes is set (16-byte aligned), the build
 * also writes the first BAJO_TOP_NODES internal nodes of segment 0's tree in
 * breadth-first order (left before right): a 16-byte header [staged count,
 * root ref, 0, 0] then one 64-byte record per slot [left-child AABB |
 * right-child AABB | left ref, right ref, 0, 0], where a child that is itself
 * staged is referenced as BAJO_TOP_FLAG | slot.  The closest-hit kernels copy
 * the records into shared memory once per block with one bulk asynchronous
 * copy and read the top of the tree from there; the hits do not change. */
#define BAJO_TOP_NODES 256u
#define BAJO_TOP_FLAG 0x40000000u
#define BAJO_TOP_BYTES (16u + 64u * BAJO_TOP_NODES)

/* Byte size of every BajoLbvh array for N triangles in S segments (in field
 * order: internal_offsets, leaf_bounds, seg_bounds, sort_keys, leaf_ids,
 * morton_codes, node_meta, node_bounds, node_leaf_counts, node_flags,
 * leaf_parent, roots, leaf_tris) and of the build workspace. */
typedef struct BajoLbvhSizes {
  size_t internal_offsets, leaf_bounds, seg_bounds, sort_keys, leaf_ids, morton_codes, node_meta, node_bounds,
      node_leaf_counts, node_flags, leaf_parent, roots, leaf_tris;
  size_t workspace;
  size_t top_nodes; /* BAJO_TOP_BYTES */
} BajoLbvhSizes;
int32_t bajo_lbvh_sizes(uint32_t n_tris, uint32_t n_segments, BajoLbvhSizes* sizes);

/* Replaces build_triangle_bvh (bajo/bvh/gpu/triangle_bvh.mojo:617) and the
 * segmented driver enqueue_segmented_wide_build
 * (bajo/bvh/gpu/builder/segmented_build.mojo:89) up to the binary LBVH
 * (build_binary_bvh_with_lbvh, bajo/bvh/gpu/builder/lbvh.mojo:332):
 * triangle bounds, per-segment bounds, Morton keys, onesweep sort of the live
 * key bits, Karras topology, atomic-flag refit, sorted triangle packing.
 * d_verts: 9 floats per triangle [v0 xyz, v1 xyz, v2 xyz].  bvh->seg_offsets
 * and every output array must be set by the caller.
 * One scene (S = 1) of 2 .. 2^17 triangles is built by one cooperative
 * kernel launch (grid barriers between the phases; a barrier wait that runs
 * out sets BAJO_STATUS_GRID_TIMEOUT); other builds launch one kernel per
 * stage.  Both give the same arrays bit for bit. */
int32_t bajo_lbvh_build(const float* d_verts, BajoLbvh* bvh, void* d_workspace, size_t workspace_bytes,
                        void* stream);

/* Largest scene (triangles) the one-launch build takes, at most 2^17 (the
 * default); 0 sends every build through the per-stage kernels.  Process wide,
 * like the sort tuning table: set it before building, not concurrently. */
int32_t bajo_lbvh_fused_max_set(uint32_t max_leaves);
/* The one-launch build ends with the splits between the tiles' largest
 * subtrees, built in shared memory by one CTA per `cap` of those subtrees
 * (default and maximum BAJO_LBVH_TOP_CAP = 1536; 0 restores it); splits
 * between two CTAs' ranges meet in global memory.  A smaller cap only moves
 * work into global memory (the tree is the same): tests use it to exercise
 * those splits.  Process wide; set it before building. */
#define BAJO_LBVH_TOP_CAP 1536u
int32_t bajo_lbvh_fused_top_cap_set(uint32_t cap);
/* Kernel launches bajo_lbvh_build makes for n_tris triangles in n_segments
 * segments on the current device (1 for the one-launch build). */
int32_t bajo_lbvh_build_launches(uint32_t n_tris, uint32_t n_segments, int32_t* launches);

/* H-PLOC build (GpuBvhBuildMethod.HPLOC, the reference's default builder,
 * triangle_bvh.mojo:472; build_hploc_multi_wave_kernel,
 * bajo/bvh/gpu/builder/hploc_multi_wave.mojo:187-545): the same bounds,
 * Morton keys and sort as bajo_lbvh_build, then Hierarchical PLOC
 * clustering (Benthin et al., HPG 2024) instead of the Karras topology and
 * refit.  Fills the same BajoLbvh arrays (node layout, sorted leaves and
 * triangle records, roots), so every traversal, the wide collapse and the
 * CWBVH8 build take its tree unchanged.  Internal node ids come from atomic
 * counters and vary from run to run, as in the reference; children, boxes
 * and leaf counts do not.  The workspace is larger than the LBVH build's
 * (bajo_hploc_workspace_size); the build status (bajo_workspace_status) gets
 * BAJO_STATUS_BAD_TOPOLOGY if a segment's node count or root is off. */
int32_t bajo_hploc_workspace_size(uint32_t n_tris, uint32_t n_segments, size_t* bytes);
int32_t bajo_hploc_build(const float* d_verts, BajoLbvh* bvh, void* d_workspace, size_t workspace_bytes,
                         void* stream);

/* Stage-timed build, the sync-free counterpart of the reference's
 * measure_stages / GpuBuildTimings (bajo/bvh/gpu/builder/lbvh.mojo:347-422):
 * `events` holds n_events cudaEvent_t handles created by the caller; the
 * build records them on `stream` at [start, bounds, morton, sort pass 0..P-1,
 * topology, refit]: bajo_lbvh_stage_count gives n_events = P + 5.  A build
 * that takes the one-launch build has two events instead, [start, build]
 * (bajo_lbvh_stage_count gives 2); with bajo_lbvh_fused_max_set(0) first, it
 * times the per-stage kernels. */
int32_t bajo_lbvh_build_timed(const float* d_verts, BajoLbvh* bvh, void* d_workspace, size_t workspace_bytes,
                              void* stream, void* const* events, int32_t n_events);
int32_t bajo_lbvh_stage_count(uint32_t n_tris, uint32_t n_segments, int32_t* n_events);

/* Rewrites bvh->top_nodes from the tree's current nodes (the build does this
 * itself when top_nodes is set).  Needed after a build through a record whose
 * top_nodes was NULL: the staged copy is not checked against the tree beyond
 * its root ref. */
int32_t bajo_lbvh_stage_top(const BajoLbvh* bvh, void* stream);

/* Diagnostic for the library's failure detection (the reference spins
 * without a bound, onesweep.mojo:246-270; its wide collapse bounds its spin
 * and reports a timeout, wide_collapse.mojo:236-253): one device thread waits
 * through the same bounded-wait helper the kernels use until any of `bits`
 * is set in *d_flag, for at most limit_us microseconds (1..1,000,000), and
 * on timeout ORs BAJO_STATUS_WAIT_TIMEOUT into *d_status and returns.  A
 * flag that nothing sets shows the wait ending with a status instead of
 * hanging the GPU. */
int32_t bajo_wait_selftest(const uint32_t* d_flag, uint32_t bits, uint32_t limit_us, uint32_t* d_status,
                           void* stream);

/* ======================================================================== */
/* Closest-hit traversal                                                     */
/* ======================================================================== */
/* Replaces GpuTriangleBvh.launch_rays[CLOSEST_HIT]
 * (bajo/bvh/gpu/triangle_bvh.mojo:587).  d_rays: SoA, 8 planes of n floats
 * [ox, oy, oz, tmin, dx, dy, dz, tmax] (bajo/bvh/gpu/ray_launch.mojo:95).
 * Outputs (either may be NULL): d_hits8, 8 words per ray
 * [u, v, prim, inst, nx, ny, nz, t] (bajo/bvh/types.mojo:16-27); d_t / d_prim,
 * compact SoA closest distance and primitive id.  Misses report t = tmax and
 * prim = 0xFFFFFFFF.  Ties in t go to the lowest primitive id.  Segment 0's
 * root is traced.  d_status (may be NULL) receives BAJO_STATUS_* bits. */
int32_t bajo_trace_rays(const BajoLbvh* bvh, const float* d_rays, uint32_t n_rays, int32_t tri_mode,
                        float* d_hits8, float* d_t, uint32_t* d_prim, uint32_t* d_status, void* stream);

/* Autotuner hook of the closest-hit kernels: block size (64, 128 or 256
 * threads; 0 = the built-in 128) of the unstaged camera (kind 0) and general
 * ray (kind 1) kernels per ceil(log2 n), process wide like the sort table.
 * The hits do not depend on it.  bajo_trace_tuning_get reports the block size
 * a call of n rays would use. */
int32_t bajo_trace_tuning_set(int32_t kind, uint32_t log2n, int32_t block);
int32_t bajo_trace_tuning_get(int32_t kind, uint32_t n, int32_t* block);
/* The same kernels' traversal stack depth: 64, 24 (the reference's
 * GPU_STACK_SIZE, bajo/bvh/constants.mojo:16) or 12 entries (0 = 64), per
 * kind and ceil(log2 n).  A ray whose traversal needs more entries than the
 * chosen depth is traced again with 64, so the hits do not depend on it
 * either.  New on this path. */
int32_t bajo_trace_stack_tuning_set(int32_t kind, uint32_t log2n, int32_t depth);
int32_t bajo_trace_stack_tuning_get(int32_t kind, uint32_t n, int32_t* depth);

/* Replaces GpuTriangleBvh.launch_camera (bajo/bvh/gpu/triangle_bvh.mojo:520):
 * primary rays generated in-kernel from 20-float camera records
 * (bajo/bvh/camera.mojo:19-37, make_ray_raster :137), one camera per
 * width*height rays (camera_launch.mojo:34). */
int32_t bajo_trace_camera(const BajoLbvh* bvh, const float* d_cameras, uint32_t n_rays, uint32_t width,
                          uint32_t height, int32_t tri_mode, float* d_hits8, float* d_t, uint32_t* d_prim,
                          uint32_t* d_status, void* stream);

/* Batched build + trace workload over a segmented LBVH (one scene per
 * segment; enqueue_segmented_wide_build + the BLAS-set trace,
 * bajo/bvh/gpu/builder/segmented_build.mojo:89, bajo/bvh/gpu/triangle_bvh.mojo:
 * 469): ray i belongs to scene i / (width*height), starts at that scene's
 * camera (cam_stride floats apart, 0 = one shared camera) and is traced
 * against that scene's root; a primary hit spawns one cosine-weighted bounce
 * ray about the oriented geometric normal (Philox stream (ray, stage 1)).
 * Outputs, n_segments*width*height each: primary t / prim, bounce t / prim
 * (segment-local prim ids; misses: t = FLT_MAX, prim = 0xFFFFFFFF). */
int32_t bajo_trace_batch(const BajoLbvh* bvh, const float* d_cameras, uint32_t cam_stride, uint32_t width,
                         uint32_t height, uint64_t seed, int32_t tri_mode, float* d_t0, uint32_t* d_prim0,
                         float* d_t1, uint32_t* d_prim1, uint32_t* d_status, void* stream);

/* Instrumented camera trace (trace_triangle_bvh_camera_instrumented_kernel,
 * bajo/bvh/gpu/triangle_bvh.mojo:813): same hits as bajo_trace_camera plus,
 * per ray, BAJO_TRACE_STATS_WORDS counters in the layout of
 * GpuTraversalStats (bajo/bvh/gpu/trace.mojo:62-90): d_stats[5i + 0]
 * internal nodes visited, + 1 internal children whose box was hit, + 2 leaf
 * blocks entered, + 3 triangles tested, + 4 deepest traversal stack. */
#define BAJO_TRACE_STATS_WORDS 5
int32_t bajo_trace_camera_stats(const BajoLbvh* bvh, const float* d_cameras, uint32_t n_rays, uint32_t width,
                                uint32_t height, int32_t tri_mode, float* d_hits8, uint32_t* d_stats,
                                void* stream);

/* ======================================================================== */
/* Wide BVH (W = 4 or 8) collapsed from the binary LBVH                      */
/* ======================================================================== */
/* Layouts of the reference (bajo/bvh/constants.mojo:26,47-55,
 * bajo/bvh/wide_meta.mojo:7-47): node i = 7 x W f32 field-major
 * [min x][min y][min z][max x][max y][max z][meta] (meta as u32 bits:
 * count << 26 | segment-local index; count 0 = internal child, 1..4 = leaf
 * block of that many triangles; 0xFFFFFFFF = empty lane with an invalid
 * box); leaf block b = W payloads (item ids) and W packed triangles
 * [v0 xyz][prim][e1 xyz][0][e2 xyz][0] x W (triangle_bvh.mojo:81-148).
 * leaf_sorted (this library's addition) holds each lane's sorted binary leaf,
 * which the watertight test uses to read the original vertices.  Node and
 * leaf ids are pre-order and deterministic (the reference allocates them with
 * atomics, wide_collapse.mojo:551-559). */
typedef struct BajoWideBvh {
  uint32_t width;              /* 4 or 8 (leaf blocks hold `width` lanes)          */
  uint32_t max_leaf;           /* triangles per leaf block, 1..4; 0 = 4 (the
                                  reference's fat leaves for triangles; 1 is its
                                  fat_leaves = false)                              */
  uint32_t n_segments;         /* set by bajo_wide_build                           */
  uint32_t* node_offsets;      /* [S+1] first wide node of each segment            */
  uint32_t* leaf_offsets;      /* [S+1] first leaf block of each segment           */
  float* nodes;                /* [node][7][W]                                     */
  uint32_t* leaf_indices;      /* [block][W], 0xFFFFFFFF padding                   */
  float* leaf_tris;            /* [block][12][W]                                   */
  uint32_t* leaf_sorted;       /* [block][W], 0xFFFFFFFF padding                   */
  const float* bvh2_leaf_tris; /* set by bajo_wide_build: the binary tree's records */
} BajoWideBvh;

typedef struct BajoWideSizes {
  size_t node_offsets, leaf_offsets, nodes, leaf_indices, leaf_tris, leaf_sorted, workspace;
} BajoWideSizes;

int32_t bajo_wide_sizes(uint32_t n_tris, uint32_t n_segments, uint32_t width, BajoWideSizes* sizes);

/* Replaces the collapse step of enqueue_segmented_wide_build
 * (bajo/bvh/gpu/builder/segmented_build.mojo:89; hploc_literature_to_wide_kernel,
 * wide_collapse.mojo:148) and the leaf packing
 * (pack_segmented_triangle_leaf_lanes_kernel, triangle_bvh.mojo:81) with fat
 * leaves of up to 4 triangles, for every segment of a built binary tree. */
int32_t bajo_wide_build(const BajoLbvh* bvh, BajoWideBvh* out, void* d_workspace, size_t workspace_bytes,
                        void* stream);

/* Synchronises `stream` and reads the total wide nodes and leaf blocks. */
int32_t bajo_wide_counts(const BajoWideBvh* wide, void* stream, uint32_t* n_nodes, uint32_t* n_leaf_blocks);

/* Closest hits over segment 0's wide tree (GpuTriangleBvh.launch_rays /
 * launch_camera on the wide layout, triangle_bvh.mojo:520-614; loop
 * trace_bounds_bvh_state, bajo/bvh/gpu/trace.mojo:431-552).  Same
 * arguments and outputs as bajo_trace_rays / bajo_trace_camera plus segment
 * 0's node and leaf-block counts (bajo_wide_counts; the node count bounds the
 * visits, the block count the leaf references); d_stats (may be NULL)
 * receives BAJO_TRACE_STATS_WORDS counters per ray, as
 * bajo_trace_camera_stats.  Hits equal the binary tree's bit for bit. */
int32_t bajo_trace_wide_rays(const BajoWideBvh* wide, uint32_t n_nodes, uint32_t n_leaf_blocks, const float* d_rays,
                             uint32_t n_rays,
                             int32_t tri_mode, float* d_hits8, float* d_t, uint32_t* d_prim, uint32_t* d_status,
                             void* stream);
int32_t bajo_trace_wide_camera(const BajoWideBvh* wide, uint32_t n_nodes, uint32_t n_leaf_blocks,
                               const float* d_cameras, uint32_t n_rays,
                               uint32_t width, uint32_t height, int32_t tri_mode, float* d_hits8, float* d_t,
                               uint32_t* d_prim, uint32_t* d_status, uint32_t* d_stats, void* stream);

/* ======================================================================== */
/* CWBVH8: compressed 8-wide BVH (Ylitie, Karras, Laine, HPG 2017)           */
/* ======================================================================== */
/* Layouts of the reference (bajo/bvh/gpu/compressed_bounds_bvh.mojo:25-39):
 * node = 20 words (80 B): [0..2] p = the node's minimum corner (f32),
 * [3] exponents x | y << 8 | z << 16 | imask << 24 (a lane's box is
 * p + q * 2^(e - 127)), [4] first internal child and [5] first triangle
 * (segment-local), [6..7] one byte per lane (internal child: 001 | slot + 24,
 * leaf: unary triangle count << 5 | triangle offset, empty: 0), [8 + 2 * plane
 * + group] the lanes' 8-bit planes (plane lo x, lo y, lo z, hi x, hi y, hi z;
 * group = lanes 0..3 / 4..7).  A node's internal children are consecutive
 * nodes in lane order.  Triangle = 12 words (48 B): e1 xyz, 0, e2 xyz, 0,
 * v0 xyz, segment-local prim (u32 bits); segment s's triangles start at the
 * binary tree's seg_offsets[s]. */
#define BAJO_CWBVH8_NODE_WORDS 20
#define BAJO_CWBVH8_TRI_WORDS 12
#define BAJO_CWBVH8_MAX_LEAF 3u /* triangles per leaf lane (CWBVH_MAX_LEAF_SIZE) */

typedef struct BajoCwbvh8 {
  uint32_t n_segments;    /* set by bajo_cwbvh8_build                      */
  uint32_t n_tris;        /* set by bajo_cwbvh8_build: triangle records   */
  uint32_t* node_offsets; /* [S+1] first node of each segment              */
  float* nodes;           /* [node][20], 16-byte aligned                   */
  float* triangles;       /* [triangle][12], 16-byte aligned               */
} BajoCwbvh8;

typedef struct BajoCwbvh8Sizes {
  size_t node_offsets, nodes, triangles, workspace;
} BajoCwbvh8Sizes;

int32_t bajo_cwbvh8_sizes(uint32_t n_tris, uint32_t n_segments, BajoCwbvh8Sizes* sizes);

/* Replaces build_triangle_blas_set[8, 4, layout = CWBVH8]
 * (bajo/bvh/gpu/triangle_bvh.mojo:366-485): the W = 8 collapse with leaves of
 * at most three triangles and octant slots (enqueue_segmented_wide_build with
 * fat_leaves and spatial_slots, segmented_build.mojo:89;
 * wide_collapse.mojo:457-521), encoded (encode_segmented_cwbvh8_nodes_kernel,
 * compressed_bounds_bvh.mojo:328) and packed
 * (pack_segmented_cwbvh_triangles_kernel, :372) for every segment of a built
 * binary tree, in one pass over the wide nodes.  Node ids and triangle ranges
 * are deterministic (the reference takes both from atomic counters).  The
 * build status (bajo_workspace_status) is BAJO_STATUS_BAD_TOPOLOGY for a
 * corrupt binary tree and BAJO_STATUS_WIDE_TIMEOUT for a task wait that gave
 * up. */
int32_t bajo_cwbvh8_build(const BajoLbvh* bvh, BajoCwbvh8* out, void* d_workspace, size_t workspace_bytes,
                          void* stream);

/* Synchronises `stream` and reads the total compressed nodes. */
int32_t bajo_cwbvh8_count(const BajoCwbvh8* cwbvh, void* stream, uint32_t* n_nodes);

/* Closest hits (any_hit = 0) or occlusion (any_hit = 1) over segment 0's tree
 * (trace_cwbvh8_triangles, triangle_bvh.mojo:1010-1104; node decode
 * _intersect_cwbvh8_node_tasks, compressed_bounds_bvh.mojo:469-576; record
 * test _intersect_cwbvh_triangle, triangle_bvh.mojo:962-1007, the
 * determinant-scaled Moller-Trumbore of intersect.mojo:462-505).  Rays and
 * outputs as bajo_trace_rays / bajo_trace_camera; an occluded ray reports
 * t = 0 and prim 0xFFFFFFFF (Hit.shadow_hit, bajo/bvh/types.mojo:46).
 * n_nodes (bajo_cwbvh8_count) bounds node references and visits;
 * *d_status gets BAJO_STATUS_BAD_TOPOLOGY for an out-of-range node or
 * triangle and BAJO_STATUS_STACK_OVERFLOW past 64 stacked node groups. */
int32_t bajo_trace_cwbvh8_rays(const BajoCwbvh8* cwbvh, uint32_t n_nodes, const float* d_rays, uint32_t n_rays,
                               int32_t any_hit, float* d_hits8, float* d_t, uint32_t* d_prim, uint32_t* d_status,
                               void* stream);
int32_t bajo_trace_cwbvh8_camera(const BajoCwbvh8* cwbvh, uint32_t n_nodes, const float* d_cameras,
                                 uint32_t n_rays, uint32_t width, uint32_t height, int32_t any_hit, float* d_hits8,
                                 float* d_t, uint32_t* d_prim, uint32_t* d_status, void* stream);

/* ======================================================================== */
/* Two-level trees: instances of the BLASes of a segmented build             */
/* ======================================================================== */
/* A BLAS set is a segmented BajoLbvh (bajo_lbvh_build or bajo_hploc_build),
 * segment b = BLAS b (build_triangle_blas_set, triangle_bvh.mojo:466).  An
 * instance i is d_blas[i] and an affine transform from BLAS space to world
 * space, 12 f32 row-major [m00 m01 m02 tx | m10 m11 m12 ty | m20 m21 m22 tz]
 * (Affine3, bajo/core/transform.mojo:22-47; Instance, bajo/bvh/types.mojo:
 * 153-190), 16-byte aligned; the traversal takes the inverse transforms
 * (world to BLAS space) in the same layout.
 *
 * bajo_tlas_instance_boxes writes, per instance, its BLAS root box under the
 * transform (AABB.apply_transform, bajo/core/aabb.mojo:101-139) as 9 floats
 * [min xyz, max xyz, min xyz]: a triangle record whose bounds are the box.
 * bajo_lbvh_build over those records (one segment, n_instances leaves) is
 * the top-level tree (build_triangle_tlas, bajo/bvh/gpu/tlas.mojo:618).
 * d_status (may be NULL) gets BAJO_STATUS_BAD_TOPOLOGY for a BLAS index out
 * of range. */
int32_t bajo_tlas_instance_boxes(const BajoLbvh* blas_set, const float* d_transforms, const uint32_t* d_blas,
                                 uint32_t n_instances, float* d_boxes9, uint32_t* d_status, void* stream);

/* Closest hits (any_hit = 0) or occlusion (any_hit = 1) through the
 * top-level tree (_trace_tlas_ray, bajo/bvh/gpu/tlas.mojo:176-232;
 * trace_triangle_tlas_camera_kernel :235): each instance leaf takes the ray
 * to BLAS space (Affine3.ray), traverses its BLAS with the current hit
 * distance as t_max and keeps a closer hit with its instance id; the winning
 * normal goes to world space through the inverse's transpose.  Rays, cameras
 * and hits as bajo_trace_rays / bajo_trace_camera; the hit's inst word is
 * the instance (0xFFFFFFFF on a miss), prim is BLAS-local.  An occluded ray
 * reports t = 0, prim 0xFFFFFFFF and the occluding instance. */
int32_t bajo_trace_tlas_rays(const BajoLbvh* tlas, const BajoLbvh* blas_set, const float* d_inv_transforms,
                             const uint32_t* d_blas, uint32_t n_instances, const float* d_rays, uint32_t n_rays,
                             int32_t any_hit, int32_t tri_mode, float* d_hits8, uint32_t* d_status, void* stream);
int32_t bajo_trace_tlas_camera(const BajoLbvh* tlas, const BajoLbvh* blas_set, const float* d_inv_transforms,
                               const uint32_t* d_blas, uint32_t n_instances, const float* d_cameras, uint32_t n_rays,
                               uint32_t width, uint32_t height, int32_t any_hit, int32_t tri_mode, float* d_hits8,
                               uint32_t* d_status, void* stream);

/* ======================================================================== */
/* Wavefront path tracing over one triangle LBVH                             */
/* ======================================================================== */
/* Render algorithms (RENDER, bajo/rt/types.mojo:53-59). */
#define BAJO_RENDER_PATH 0
#define BAJO_RENDER_NEE 3
#define BAJO_RENDER_MIS 4

/* Surface ids: kind in the top 4 bits, table index below
 * (SurfaceId, bajo/rt/types.mojo:24-34). */
#define BAJO_MAT_LAMBERTIAN 0u
#define BAJO_MAT_METAL 1u
#define BAJO_MAT_DIELECTRIC 2u
#define BAJO_MAT_EMISSIVE 3u
#define BAJO_SURFACE(kind, index) (((uint32_t)(kind) << 28) | ((uint32_t)(index) & 0x0FFFFFFFu))

/* Light records, 16 floats: [p0 xyz, p1 xyz, p2 xyz, emission rgb,
 * alias probability, alias index (u32 bits), pad, pad]
 * (GpuRtLights, bajo/rt/gpu/path_shading.mojo:60-74,146). */
#define BAJO_LIGHT_STRIDE 16

/* Queue status words (WAVE_STATUS, bajo/rt/wavefront_contract.mojo:25-29). */
#define BAJO_WAVE_PATH_OVERFLOW 0x10u
#define BAJO_WAVE_SHADOW_OVERFLOW 0x20u

typedef struct BajoRtScene {
  const BajoLbvh* bvh;       /* single-segment tree over the scene triangles       */
  const uint32_t* surfaces;  /* per triangle, item order: BAJO_SURFACE(kind, idx)  */
  const float* lambertians;  /* 3 f32 albedo per Lambertian material               */
  const float* emissives;    /* 3 f32 radiance per emissive material               */
  const float* lights;       /* BAJO_LIGHT_STRIDE f32 per emissive triangle        */
  uint32_t n_lights;
  float total_light_weight;  /* sum of area * mean(radiance) over the lights        */
  const float* metals;       /* 4 f32 per metal: albedo rgb, fuzz (NULL: none)     */
  const float* dielectrics;  /* 1 f32 refraction index per dielectric (NULL: none) */
  /* Acceleration structure of the closest-hit and shadow rays: NULL traces
   * bvh (the binary LBVH: watertight test, ties to the lowest triangle id);
   * else this compressed 8-wide tree built from bvh by bajo_cwbvh8_build,
   * with cwbvh8_nodes its node count (bajo_cwbvh8_count).  The CWBVH8 walk is
   * the reference's default triangle path (GPU_RT_BVH_CWBVH8_*,
   * bajo/rt/gpu/prepared_scene.mojo:29-33,52-53) with its own rules:
   * Moller-Trumbore, first of equal-distance hits in visiting order. */
  const struct BajoCwbvh8* cwbvh8;
  uint32_t cwbvh8_nodes;
} BajoRtScene;
/* Metal and dielectric surfaces (_sample_metal / _sample_dielectric,
 * bajo/rt/shading.mojo:122-198; gpu_rt_shade_dispatch_kernel,
 * bajo/rt/gpu/path_shading.mojo:786): mirror (fuzz <= 1e-4) or glossy
 * reflection, and Schlick-weighted reflection / refraction.  They take no
 * light sample; the continued path carries the sample's pdf and the delta
 * flag (mirror and dielectric).  With both tables NULL the renderer runs no
 * material pass. */

typedef struct BajoRenderSettings {
  uint32_t width, height, spp, max_depth;
  uint64_t seed;
  int32_t algorithm;     /* BAJO_RENDER_*                                         */
  uint32_t chunk_paths;  /* queue capacity in paths (0 = default); whole pixels   */
} BajoRenderSettings;

/* Host: emissive-triangle light records with a Walker-Vose alias table over
 * their power (LightStore, bajo/rt/types.mojo:190-247,490-525).  h_* are HOST
 * arrays; out_lights holds max_lights * BAJO_LIGHT_STRIDE floats. */
int32_t bajo_rt_build_lights(const float* h_verts, const uint32_t* h_surfaces, uint32_t n_tris,
                             const float* h_emissives, uint32_t n_emissives, float* out_lights, uint32_t max_lights,
                             uint32_t* n_lights, float* total_weight);

/* Workspace: two path queues (id + 12 f32 planes), a shadow queue (id + 11
 * planes), per-sample radiance (3 planes), per-bounce counters
 * (GpuRtRenderTarget, bajo/rt/gpu/resources.mojo:38). */
int32_t bajo_render_workspace_size(const BajoRenderSettings* settings, size_t* bytes);

/* Replaces render_gpu_triangles / enqueue_render_gpu_triangles
 * (bajo/rt/gpu/triangle_path.mojo:143,172) for Lambertian + emissive
 * triangle scenes: per chunk of whole pixels, primary rays
 * (gpu_rt_primary_kernel, bajo/rt/gpu/common_kernels.mojo:22), then per
 * bounce one closest-hit + shading kernel (gpu_rt_scene_trace_kernel,
 * bajo/rt/gpu/scene_trace.mojo:369) and one any-hit shadow kernel
 * (:586), then the per-pixel resolve (common_kernels.mojo:97).
 * d_pixels: 3 f32 per pixel (mean radiance).  d_pixels64 (may be NULL): 3 f64
 * per pixel to which the SUM of every sample is added (long reference
 * renders accumulate across calls). */
int32_t bajo_render(const BajoRtScene* scene, const float* d_camera, const BajoRenderSettings* settings,
                    float* d_pixels, double* d_pixels64, void* d_workspace, size_t workspace_bytes, void* stream);

/* Synchronises `stream` and reads the closest-hit and shadow rays traced by
 * the last bajo_render call on this workspace. */
int32_t bajo_render_stats(const void* d_workspace, void* stream, uint64_t* rays, uint64_t* shadow_rays);

/* Block sizes of the wavefront bounce kernels: 64, 128 or 256 threads (0
 * restores the built-in 128), process-wide, per kernel: the path rays'
 * closest hit, the shading of plain (non-guided) renders, the shadow rays.
 * The reference fixes 64 (GPU_RT_BLOCK_SIZE,
 * bajo/rt/gpu/common_kernels.mojo:18).  Every choice renders the same image
 * bit for bit; the autotuner times them and installs the fastest.  Read when
 * a render is launched (or recorded into a graph).  New on this path. */
#define BAJO_RENDER_KERNEL_TRACE 0
#define BAJO_RENDER_KERNEL_SHADE 1
#define BAJO_RENDER_KERNEL_SHADOW 2
int32_t bajo_render_tuning_set(int32_t kernel, int32_t block);
int32_t bajo_render_tuning_get(int32_t kernel, int32_t* block);


/* ======================================================================== */
/* Path guiding: a small MLP proposal trained online (new on this path; the  */
/* reference has no guiding)                                                 */
/* ======================================================================== */
/* Network: one-blob(position in box6, 3 x 16 bins) ++ one-blob(octahedral
 * normal, 2 x 8 bins) = 64 features -> 3 x (64, ReLU) -> 20 outputs =
 * 4 vMF lobes x (mean xyz, log kappa, weight logit).  FP16 weights and
 * activations, FP32 accumulation on the tensor cores.  Parameter layout
 * (bajo_mlp_param_count elements): W1[64x64] b1[64] W2 b2 W3 b3 W4[32x64]
 * b4[32], weights row-major [out][in]; rows 20..31 of W4/b4 are kept zero.
 * Mixture: mean = m / sqrt(|m|^2 + 1e-12), kappa = exp(clamp(s, -2, 8)), weights =
 * softmax(logits), lobe pdf kappa / (2 pi (1 - e^-2kappa)) e^(kappa (mu.w-1)). */
#define BAJO_MLP_OUTPUTS 20
int32_t bajo_mlp_param_count(uint32_t* count);

/* d_out20[20 i + c] = raw outputs for sample i (positions and normals are
 * 3 f32 each, box6 = [min xyz, max xyz]). */
int32_t bajo_mlp_forward(const void* d_params16, const float* d_pos, const float* d_nrm, uint32_t n,
                         const float* d_box6, float* d_out20, void* stream);
/* The same outputs from the 5th-generation tensor cores: 128-sample tiles per
 * CTA, each layer four tcgen05.mma (FP16 in, FP32 accumulator in tensor
 * memory) issued by one thread, read back with tcgen05.ld for the bias and
 * ReLU.  Agrees with bajo_mlp_forward to FP32 accumulation order.  d_status
 * (may be NULL) gets BAJO_STATUS_WAIT_TIMEOUT if the tensor cores never
 * signal completion (the launch then stops after freeing its tensor memory).
 * New on this path (no counterpart in the reference). */
int32_t bajo_mlp_forward_tc(const void* d_params16, const float* d_pos, const float* d_nrm, uint32_t n,
                            const float* d_box6, float* d_out20, uint32_t* d_status, void* stream);

/* d_grad32 = gradient of sum_i -w_i log pdf_i(dir_i) w.r.t. the parameters
 * (overwritten); *d_loss (may be NULL) = that sum. */
int32_t bajo_mlp_grad(const void* d_params16, const float* d_pos, const float* d_nrm, const float* d_dir,
                      const float* d_weight, uint32_t n, const float* d_box6, float* d_grad32, float* d_loss,
                      void* stream);

/* The same gradient from the 5th-generation tensor cores: per 128-sample
 * tile the forward keeps every layer's activations in shared memory, then
 * per layer one tcgen05.mma chain for the weight gradient (M = 64 outputs,
 * N = 80: inputs and the bias column, K = 128 samples, accumulated in tensor
 * memory over the CTA's tiles) and one for the input gradient (M = 128
 * samples, N = 64).  Agrees with bajo_mlp_grad to FP32 accumulation order.
 * d_grad32 must be 16-byte aligned (the gradients are added with 16-byte
 * atomics; else BAJO_ERR_INVALID_ARGUMENT), as must BajoGuideNet::grad.
 * d_status (may be NULL) gets BAJO_STATUS_WAIT_TIMEOUT if the tensor cores
 * never signal completion.  New on this path (no counterpart in the
 * reference). */
int32_t bajo_mlp_grad_tc(const void* d_params16, const float* d_pos, const float* d_nrm, const float* d_dir,
                         const float* d_weight, uint32_t n, const float* d_box6, float* d_grad32, float* d_loss,
                         uint32_t* d_status, void* stream);

/* One Adam step (Kingma & Ba) on FP32 master weights with gradient
 * grad_scale * d_grad32; refreshes the FP16 copy.  step counts from 1. */
int32_t bajo_mlp_adam(float* d_params32, void* d_params16, const float* d_grad32, float* d_m, float* d_v,
                      uint32_t step, float lr, float beta1, float beta2, float eps, float grad_scale, void* stream);

/* Guided wavefront rendering: BAJO_RENDER_MIS with the continuation drawn by
 * one-sample MIS from (1 - f) * cosine BSDF + f * network mixture and every
 * MIS weight (emission hits, light samples) taken against that combined
 * pdf, so the estimator stays unbiased for any network.  Per bounce: closest
 * hit + emission, then one fused kernel that runs the network over the
 * bounce's Lambertian vertices on the tensor cores and does next-event
 * estimation and the continuation sample, then the shadow rays.
 * Training records: a fraction of the continued vertices (chosen by a hash
 * of path and bounce) is kept, up to record_capacity per call; at the end of
 * each chunk a record holds position, normal, sampled direction and weight
 * mean_rgb(L_i(dir)) * cos / pdf, L_i being the radiance the path gathered
 * after the vertex divided by its throughput.
 * Record buffer (bajo_guide_records_size bytes): u32 count at byte 0 (zero
 * it to start collecting), then, each array starting on a 256-byte boundary
 * after a 256-byte header: pos f32[3 cap], nrm f32[3 cap], dir f32[3 cap],
 * weight f32[cap], then internal scratch. */
#define BAJO_RENDER_GUIDED 5
typedef struct BajoGuide {
  const void* params16;     /* network parameters (FP16)                         */
  const float* box6;        /* device: scene box for the position encoding       */
  float guide_fraction;     /* probability of sampling the network (0.5)         */
  float record_fraction;    /* probability a continued vertex becomes a record   */
  uint32_t record_capacity; /* records kept per call (0 = none)                  */
  void* records;            /* device buffer, bajo_guide_records_size bytes      */
} BajoGuide;

int32_t bajo_guide_records_size(uint32_t capacity, size_t* bytes);

/* settings->algorithm must be BAJO_RENDER_GUIDED; workspace from
 * bajo_render_workspace_size with the same settings. */
int32_t bajo_render_guided(const BajoRtScene* scene, const float* d_camera, const BajoRenderSettings* settings,
                           const BajoGuide* guide, float* d_pixels, double* d_pixels64, void* d_workspace,
                           size_t workspace_bytes, void* stream);

/* Handle-based rendering (render_gpu_triangles / enqueue_render_gpu_triangles,
 * bajo/rt/gpu/triangle_path.mojo:143,172; GpuRtRenderTarget download,
 * bajo/rt/gpu/resources.mojo:275).  The caller owns the workspace (at least
 * bajo_render_workspace_size bytes), the scene and the pixel buffers; the
 * handle is host memory holding the settings and a CUDA graph of the last
 * enqueued render.  bajo_render_enqueue renders like bajo_render (guide =
 * NULL) or bajo_render_guided (settings->algorithm BAJO_RENDER_GUIDED).  On a
 * stream other than the legacy default stream the first enqueue records the
 * render into a graph and launches it; later enqueues with the same
 * pointers, scene, guide and settings replay the graph with one launch (it
 * reads buffer contents at replay, so new camera or scene data in the same
 * buffers is picked up).  Inside a capture the caller started, the render is
 * recorded into that capture.  bajo_render_download synchronises `stream`,
 * copies the pixels (3 f32 each) to host memory when h_pixels is set and
 * reads the status word and the ray totals. */
typedef struct BajoRenderer BajoRenderer;
int32_t bajo_render_create(const BajoRenderSettings* settings, void* d_workspace, size_t workspace_bytes,
                           BajoRenderer** renderer);
int32_t bajo_render_enqueue(BajoRenderer* renderer, const BajoRtScene* scene, const float* d_camera,
                            const BajoGuide* guide, float* d_pixels, double* d_pixels64, void* stream);
int32_t bajo_render_download(BajoRenderer* renderer, const float* d_pixels, float* h_pixels, uint64_t* rays,
                             uint64_t* shadow_rays, uint32_t* status, void* stream);
int32_t bajo_render_graph_launches(const BajoRenderer* renderer, uint32_t* launches);
int32_t bajo_render_destroy(BajoRenderer* renderer);

/* Online training state (device arrays of bajo_mlp_param_count elements). */
typedef struct BajoGuideNet {
  float* params32;
  void* params16;
  float* adam_m;
  float* adam_v;
  float* grad;
  float* loss;      /* 1 f32: summed loss of the last step */
  uint32_t step;    /* Adam steps taken so far (advanced by bajo_guide_train) */
  uint32_t* status; /* device u32 (may be NULL): BAJO_STATUS_WAIT_TIMEOUT from the gradient kernel */
} BajoGuideNet;

/* `steps` Adam steps (beta 0.9 / 0.999, eps 1e-8, learning rate lr), each
 * on `batch` records taken cyclically from the buffer (count read on the
 * device, so no host synchronisation); the gradients come from the
 * tensor-memory kernel of bajo_mlp_grad_tc. */
int32_t bajo_guide_train(BajoGuideNet* net, const void* d_records, uint32_t record_capacity, const float* d_box6,
                         uint32_t batch, uint32_t steps, float lr, void* stream);

/* Host-side camera records (no device work).  Camera.__init__ and
 * Camera.from_vfov (bajo/bvh/camera.mojo:77-116): out20 receives
 * [origin, forward, right, up, fov_scale, focus_dist, disk_u, disk_v]
 * with a zero defocus angle. */
int32_t bajo_camera_make(const float* origin, const float* target, const float* world_up, float fov_scale,
                         float* out20);
int32_t bajo_camera_from_vfov(const float* origin, const float* target, const float* world_up, float vfov_deg,
                              float* out20);

/* Library version string. */
const char* bajo_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BAJO_B200_H */
