/* bajo_oracle_hploc.c -- TEST INFRASTRUCTURE ONLY: sequential restatement of
 * the H-PLOC builder (Benthin, Meister, Barczak, Mehalwal, Tsakok, Kensler,
 * HPG 2024) as the reference implements it in build_hploc_multi_wave_kernel
 * (bajo/bvh/gpu/builder/hploc_multi_wave.mojo:187-545).
 *
 * The reference's threads climb the binary radix tree of the sorted Morton
 * keys (_hploc_find_parent_id, :126-140; Apetrei's bottom-up rule over XOR
 * deltas of (code, global position) keys); the second thread to reach a node
 * owns the merged leaf range.  Here the leaves' climbs run one after another
 * in sorted order, one of the interleavings the GPU's threads can take (the
 * tree and the merges do not depend on which).  Whenever that range holds more than 16
 * leaves (HPLOC_MERGING_THRESHOLD, hploc_layout.mojo:5), or is the whole
 * segment, its two children's cluster lists (at most 16 each; a smaller range
 * contributes its leaves in sorted order) are concatenated and merged by PLOC
 * until at most 16 clusters remain (1 for the whole segment):
 *   - each cluster i looks at clusters i+1..i+8 (HPLOC_SEARCH_RADIUS) and
 *     every pair's merged-box surface area is offered to both ends as the
 *     64-bit key (area bits << 32 | offset code), offset code = 2 * (|j - i|
 *     - 1) + (j < i) (_hploc_encode_offset, :48-54); each cluster keeps the
 *     smallest key;
 *   - mutual nearest neighbours merge, the lower lane keeps the new node
 *     (left = its cluster, right = the neighbour's) and the higher lane's
 *     cluster leaves the list; non-mutual clusters stay, in order;
 *   - the new nodes of one round take consecutive ids in lane order.
 * Here ids come from one counter per segment, in the order the tasks run; the reference takes them from an atomic counter, so its ids
 * differ from run to run and only the tree itself (children, boxes, counts)
 * is compared. */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bajo_oracle.h"

#define LEAF 0x80000000u
#define IDX 0x7FFFFFFFu
#define SENT 0xFFFFFFFFu
#define THRESH 16
#define RADIUS 8

typedef struct {
  const BoLbvh* k;   /* sorted leaves: bounds, ids, codes, offsets */
  BoLbvh* o;         /* the H-PLOC tree being written */
  float* box;        /* [internal][6] each new node's own box */
  uint32_t counter;  /* nodes made in the current segment */
  uint32_t base;     /* first internal id of the current segment */
  uint32_t err;
} hctx;

static void cluster_box(const hctx* c, uint32_t ref, float out[6]) {
  if (ref & LEAF) memcpy(out, c->k->leaf_bounds + (size_t)c->k->leaf_ids[ref & IDX] * 6, 6 * sizeof(float));
  else memcpy(out, c->box + (size_t)(ref & IDX) * 6, 6 * sizeof(float));
}

static uint32_t cluster_leaves(const hctx* c, uint32_t ref) {
  return (ref & LEAF) ? 1u : c->o->node_leaf_counts[ref & IDX];
}

static void unite(const float a[6], const float b[6], float out[6]) {
  for (int k = 0; k < 3; ++k) {
    out[k] = bo_fminf(a[k], b[k]);
    out[3 + k] = bo_fmaxf(a[3 + k], b[3 + k]);
  }
}

/* surface area, bajo/core/aabb.mojo:47 */
static float area6(const float b[6]) {
  float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  return 2.0f * ((dx * dy + dx * dz) + dy * dz);
}

static uint32_t enc_off(int i, int j) {
  int s = j - i, d = (s < 0 ? -s : s) - 1;
  return (uint32_t)(d * 2 + (s < 0 ? 1 : 0));
}

static int dec_off(int i, uint32_t e) {
  int d = (int)(e >> 1) + 1;
  return (e & 1u) ? i - d : i + d;
}

static void set_parent(hctx* c, uint32_t ref, uint32_t parent) {
  if (ref & LEAF) c->o->leaf_parent[ref & IDX] = parent;
  else c->o->node_meta[(size_t)(ref & IDX) * 4 + 0] = parent;
}

/* PLOC rounds on list[0..n) until at most `threshold` clusters remain */
static int ploc(hctx* c, uint32_t* list, int n, int threshold) {
  float bx[32][6];
  for (int i = 0; i < n; ++i) cluster_box(c, list[i], bx[i]);
  while (n > threshold) {
    uint64_t d[32];
    for (int i = 0; i < n; ++i) d[i] = UINT64_MAX;
    for (int i = 0; i < n; ++i) {
      int last = i + RADIUS < n - 1 ? i + RADIUS : n - 1;
      for (int j = i + 1; j <= last; ++j) {
        float m[6];
        unite(bx[i], bx[j], m);
        float a = area6(m);
        uint32_t bits;
        memcpy(&bits, &a, 4);
        uint64_t ki = ((uint64_t)bits << 32) | enc_off(i, j), kj = ((uint64_t)bits << 32) | enc_off(j, i);
        if (ki < d[i]) d[i] = ki;
        if (kj < d[j]) d[j] = kj;
      }
    }
    int nearest[32], merge[32], mutual[32], merges = 0;
    for (int i = 0; i < n; ++i) {
      nearest[i] = dec_off(i, (uint32_t)d[i]);
      int nn = dec_off(nearest[i], (uint32_t)d[nearest[i]]);
      mutual[i] = (i == nn);
      merge[i] = mutual[i] && i < nearest[i];
      merges += merge[i];
    }
    if (merges == 0) {
      c->err |= 1u;
      return n;
    }
    uint32_t out[32];
    float obx[32][6];
    int m = 0;
    for (int i = 0; i < n; ++i) {
      if (merge[i]) {
        int j = nearest[i];
        uint32_t node = c->base + c->counter++;
        uint32_t* meta = c->o->node_meta + (size_t)node * 4;
        meta[0] = SENT;
        meta[1] = list[i];
        meta[2] = list[j];
        meta[3] = SENT;
        float* nb = c->o->node_bounds + (size_t)node * 12;
        memcpy(nb, bx[i], 6 * sizeof(float));
        memcpy(nb + 6, bx[j], 6 * sizeof(float));
        c->o->node_flags[node] = 2u;
        c->o->node_leaf_counts[node] = cluster_leaves(c, list[i]) + cluster_leaves(c, list[j]);
        set_parent(c, list[i], node);
        set_parent(c, list[j], node);
        unite(bx[i], bx[j], obx[m]);
        memcpy(c->box + (size_t)node * 6, obx[m], 6 * sizeof(float));
        out[m++] = node;
      } else if (!mutual[i]) {
        memcpy(obx[m], bx[i], 6 * sizeof(float));
        out[m++] = list[i];
      }
    }
    n = m;
    memcpy(list, out, (size_t)n * sizeof(uint32_t));
    memcpy(bx, obx, (size_t)n * sizeof(bx[0]));
  }
  return n;
}

/* delta of two sorted positions: XOR of the (code, global position) keys
 * (_hploc_delta, :114-123; morton_key_delta, bajo/core/morton.mojo:12) */
static uint64_t hdelta(const uint32_t* codes, uint32_t a, uint32_t b) {
  return (((uint64_t)codes[a] << 32) | a) ^ (((uint64_t)codes[b] << 32) | b);
}

/* _hploc_find_parent_id (:126-140): the parent splits at `right` (this range
 * is its left child) or at left - 1 */
static uint32_t find_parent(const uint32_t* codes, uint32_t left, uint32_t right, uint32_t sb, uint32_t se) {
  if (left == sb || (right + 1 != se && hdelta(codes, right, right + 1) < hdelta(codes, left - 1, left)))
    return right;
  return left - 1;
}

/* one merge task over [left, right] split at `split`: the children's lists
 * (packed at left and split, at most 16 entries each) are concatenated,
 * merged, and written back at left */
static void task(hctx* c, uint32_t* clusters, uint32_t left, uint32_t split, uint32_t right, int fin,
                 uint32_t* root) {
  uint32_t list[32];
  int n = 0;
  uint32_t ls = split - left < THRESH ? split - left : THRESH;
  for (uint32_t j = 0; j < ls; ++j)
    if (clusters[left + j] != SENT) list[n++] = clusters[left + j];
  uint32_t rs = right + 1 - split < THRESH ? right + 1 - split : THRESH;
  for (uint32_t j = 0; j < rs; ++j)
    if (clusters[split + j] != SENT) list[n++] = clusters[split + j];
  int before = n;
  n = ploc(c, list, n, fin ? 1 : THRESH);
  for (int j = 0; j < before; ++j) clusters[left + j] = j < n ? list[j] : SENT;
  if (fin) *root = n == 1 ? list[0] : SENT;
}

uint32_t bo_hploc_build(const BoLbvh* k, BoLbvh* o) {
  hctx c;
  memset(&c, 0, sizeof(c));
  c.k = k;
  c.o = o;
  const uint32_t n = k->n_leaves;
  size_t m = k->n_internal ? k->n_internal : 1;
  c.box = (float*)calloc(m * 6, sizeof(float));
  uint32_t* slots = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint32_t* clusters = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (uint32_t i = 0; i < n; ++i) {
    o->leaf_parent[i] = SENT;
    slots[i] = SENT;
    clusters[i] = LEAF | i;
  }
  const uint32_t* codes = k->morton_codes;
  for (uint32_t s = 0; s < k->n_segments; ++s) {
    const uint32_t sb = k->seg_offsets[s], se = k->seg_offsets[s + 1];
    c.counter = 0;
    c.base = k->internal_offsets[s];
    o->roots[s] = se - sb == 1 ? (LEAF | sb) : SENT;
    if (se - sb <= 1) continue;
    /* the threads of the segment's leaves, one after another: each climbs
     * until it is the first to reach a node */
    for (uint32_t i = sb; i < se; ++i) {
      uint32_t left = i, right = i;
      for (;;) {
        uint32_t split, prev;
        if (find_parent(codes, left, right, sb, se) == right) {
          prev = slots[right];
          slots[right] = left;
          if (prev == SENT) break;
          split = right + 1;
          right = prev;
        } else {
          prev = slots[left - 1];
          slots[left - 1] = right;
          if (prev == SENT) break;
          split = left;
          left = prev;
        }
        const int fin = right - left + 1 == se - sb;
        if (right - left + 1 > THRESH || fin) task(&c, clusters, left, split, right, fin, &o->roots[s]);
        if (fin) break;
      }
    }
    if (c.counter != k->internal_offsets[s + 1] - k->internal_offsets[s] || o->roots[s] == SENT) c.err |= 2u;
  }
  free(slots);
  free(clusters);
  free(c.box);
  return c.err;
}
