/* bajo_oracle_wide.c -- TEST INFRASTRUCTURE ONLY: sequential restatement of
 * the BVH2 -> W-wide collapse with fat leaves and of the triangle leaf
 * packing, checking the library's wide build bit for bit.
 *
 * Follows hploc_literature_to_wide_kernel (bajo/bvh/gpu/builder/
 * wide_collapse.mojo:148-644): a wide node rooted at binary node x starts
 * from x's two children, opens the non-fat internal candidate of largest
 * surface area (_encoded_bounds(...).surface_area(), binary_layout.mojo:65,
 * bajo/core/aabb.mojo:47) until W candidates, then opens the largest
 * remaining internal candidates; an opened candidate is replaced by its left
 * child and its right child is appended; candidates with at most four
 * triangles become leaf blocks (_write_hploc_terminal_leaf_block, :67-104,
 * left to right).  Leaf lanes pack [v0][prim][v1 - v0][0][v2 - v0][0]
 * (pack_segmented_triangle_leaf_lanes_kernel, triangle_bvh.mojo:81-148).
 * The reference numbers nodes and leaf blocks with atomics; this restatement
 * and the library both number them in pre-order: a node's own leaf blocks
 * first, then each internal child's subtree in lane order. */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bajo_oracle.h"

#define FAT 4u
#define LEAF_FLAG 0x80000000u
#define IDX_MASK 0x7FFFFFFFu
#define EMPTY 0xFFFFFFFFu

typedef struct {
  const BoLbvh* b;
  const float* verts;
  uint32_t W;
  uint32_t* nw;
  uint32_t* nl;
  float* nodes;
  uint32_t* leaf_indices;
  float* leaf_tris;
  uint32_t* leaf_sorted;
  uint32_t seg_item0;
  uint32_t max_leaf; /* triangles per leaf block (1..4) */
} wctx;

static void ref_box(const wctx* c, uint32_t ref, float out[6]) {
  if (ref & LEAF_FLAG) {
    const float* p = c->b->leaf_bounds + (size_t)c->b->leaf_ids[ref & IDX_MASK] * 6;
    memcpy(out, p, 6 * sizeof(float));
  } else {
    const float* p = c->b->node_bounds + (size_t)(ref & IDX_MASK) * 12;
    for (int k = 0; k < 3; ++k) {
      out[k] = fminf(p[k], p[6 + k]);
      out[3 + k] = fmaxf(p[3 + k], p[9 + k]);
    }
  }
}

static float ref_area(const wctx* c, uint32_t ref) {
  float bx[6];
  ref_box(c, ref, bx);
  float dx = bx[3] - bx[0], dy = bx[4] - bx[1], dz = bx[5] - bx[2];
  return 2.0f * ((dx * dy + dx * dz) + dy * dz);
}

static uint32_t ref_count(const wctx* c, uint32_t ref) {
  return (ref & LEAF_FLAG) ? 1u : c->b->node_leaf_counts[ref & IDX_MASK];
}

static int is_terminal(const wctx* c, uint32_t ref, uint32_t count) {
  return (ref & LEAF_FLAG) || count <= c->max_leaf;
}

static int open_children(const wctx* c, uint32_t x, uint32_t* cand, uint32_t* cnt) {
  const uint32_t* m = c->b->node_meta;
  float ar[8];
  cand[0] = m[(size_t)x * 4 + 1];
  cand[1] = m[(size_t)x * 4 + 2];
  for (int k = 0; k < 2; ++k) {
    cnt[k] = ref_count(c, cand[k]);
    ar[k] = ref_area(c, cand[k]);
  }
  int n = 2;
  for (int phase = 0; phase < 2; ++phase) {
    while (n < (int)c->W) {
      int pos = -1;
      float best = -1.0f;
      for (int k = 0; k < n; ++k) {
        if (cand[k] & LEAF_FLAG) continue;
        if (phase == 0 && cnt[k] <= c->max_leaf) continue;
        if (ar[k] > best) {
          best = ar[k];
          pos = k;
        }
      }
      if (pos < 0) break;
      uint32_t y = cand[pos] & IDX_MASK;
      cand[pos] = m[(size_t)y * 4 + 1];
      cand[n] = m[(size_t)y * 4 + 2];
      cnt[pos] = ref_count(c, cand[pos]);
      cnt[n] = ref_count(c, cand[n]);
      ar[pos] = ref_area(c, cand[pos]);
      ar[n] = ref_area(c, cand[n]);
      ++n;
    }
  }
  return n;
}

/* NW / NL of the collapsed subtree rooted at internal node x (post-order) */
static void counts(wctx* c, uint32_t x) {
  uint32_t cand[8], cnt[8];
  int n = open_children(c, x, cand, cnt);
  uint32_t nodes = 1, leaves = 0;
  for (int k = 0; k < n; ++k) {
    if (is_terminal(c, cand[k], cnt[k])) {
      ++leaves;
    } else {
      uint32_t ci = cand[k] & IDX_MASK;
      counts(c, ci);
      nodes += c->nw[ci];
      leaves += c->nl[ci];
    }
  }
  c->nw[x] = nodes;
  c->nl[x] = leaves;
}

static void write_block(wctx* c, uint32_t ref, uint32_t blk) {
  const uint32_t W = c->W;
  uint32_t stack[FAT + 1];
  int sp = 0;
  uint32_t lane = 0;
  stack[sp++] = ref;
  float* L = c->leaf_tris + (size_t)blk * 12 * W;
  while (sp > 0) {
    uint32_t cur = stack[--sp];
    if (cur & LEAF_FLAG) {
      uint32_t sl = cur & IDX_MASK, item = c->b->leaf_ids[sl];
      const float* v = c->verts + (size_t)item * 9;
      uint32_t prim = item - c->seg_item0;
      float p;
      memcpy(&p, &prim, 4);
      c->leaf_indices[(size_t)blk * W + lane] = item;
      c->leaf_sorted[(size_t)blk * W + lane] = sl;
      L[0 * W + lane] = v[0]; L[1 * W + lane] = v[1]; L[2 * W + lane] = v[2]; L[3 * W + lane] = p;
      L[4 * W + lane] = v[3] - v[0]; L[5 * W + lane] = v[4] - v[1]; L[6 * W + lane] = v[5] - v[2];
      L[7 * W + lane] = 0.0f;
      L[8 * W + lane] = v[6] - v[0]; L[9 * W + lane] = v[7] - v[1]; L[10 * W + lane] = v[8] - v[2];
      L[11 * W + lane] = 0.0f;
      ++lane;
    } else {
      uint32_t y = cur & IDX_MASK;
      stack[sp++] = c->b->node_meta[(size_t)y * 4 + 2];
      stack[sp++] = c->b->node_meta[(size_t)y * 4 + 1];
    }
  }
  for (; lane < W; ++lane) {
    c->leaf_indices[(size_t)blk * W + lane] = EMPTY;
    c->leaf_sorted[(size_t)blk * W + lane] = EMPTY;
    for (uint32_t f = 0; f < 12; ++f) {
      uint32_t e = EMPTY;
      float ef;
      memcpy(&ef, &e, 4);
      L[f * W + lane] = f == 3 ? ef : 0.0f;
    }
  }
}

static void store_lane(float* node, uint32_t W, uint32_t lane, const float bx[6], uint32_t meta) {
  for (int f = 0; f < 6; ++f) node[f * W + lane] = bx[f];
  memcpy(&node[6 * W + lane], &meta, 4);
}

static void store_empty(float* node, uint32_t W, uint32_t lane) {
  float bx[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
  store_lane(node, W, lane, bx, EMPTY);
}

static uint32_t pack_meta(uint32_t data, uint32_t count) { return (count << 26) | (data & 0x03FFFFFFu); }

/* wide node with global id I (local to the segment: I - nb) for binary node x,
 * first leaf block B (global; local B - lb) */
static void emit(wctx* c, uint32_t x, uint32_t I, uint32_t B, uint32_t nb, uint32_t lb) {
  const uint32_t W = c->W;
  float* node = c->nodes + (size_t)I * 7 * W;
  float bx[6];
  uint32_t xc = ref_count(c, x);
  if (is_terminal(c, x, xc)) {
    write_block(c, x, B);
    ref_box(c, x, bx);
    store_lane(node, W, 0, bx, pack_meta(B - lb, xc));
    for (uint32_t j = 1; j < W; ++j) store_empty(node, W, j);
    return;
  }
  uint32_t cand[8], cnt[8];
  int n = open_children(c, x & IDX_MASK, cand, cnt);
  uint32_t leaf_next = B;
  for (int k = 0; k < n; ++k)
    if (is_terminal(c, cand[k], cnt[k])) write_block(c, cand[k], leaf_next++);
  uint32_t own = B, child = I + 1, child_leaf = leaf_next;
  uint32_t child_id[8], child_lb[8];
  for (uint32_t k = 0; k < W; ++k) {
    if ((int)k >= n) {
      store_empty(node, W, k);
      continue;
    }
    ref_box(c, cand[k], bx);
    if (is_terminal(c, cand[k], cnt[k])) {
      store_lane(node, W, k, bx, pack_meta(own - lb, cnt[k]));
      ++own;
    } else {
      uint32_t ci = cand[k] & IDX_MASK;
      store_lane(node, W, k, bx, pack_meta(child - nb, 0));
      child_id[k] = child;
      child_lb[k] = child_leaf;
      child += c->nw[ci];
      child_leaf += c->nl[ci];
    }
  }
  for (int k = 0; k < n; ++k)
    if (!is_terminal(c, cand[k], cnt[k])) emit(c, cand[k], child_id[k], child_lb[k], nb, lb);
}

void bo_wide_build(const BoLbvh* b, const float* verts, uint32_t width, uint32_t max_leaf, float* nodes,
                   uint32_t* leaf_indices, float* leaf_tris, uint32_t* leaf_sorted, uint32_t* node_offsets,
                   uint32_t* leaf_offsets) {
  wctx c;
  memset(&c, 0, sizeof(c));
  c.max_leaf = max_leaf ? max_leaf : FAT;
  c.b = b;
  c.verts = verts;
  c.W = width;
  size_t cap = b->n_leaves ? b->n_leaves : 1;
  c.nw = (uint32_t*)calloc(cap, sizeof(uint32_t));
  c.nl = (uint32_t*)calloc(cap, sizeof(uint32_t));
  c.nodes = nodes;
  c.leaf_indices = leaf_indices;
  c.leaf_tris = leaf_tris;
  c.leaf_sorted = leaf_sorted;
  uint32_t no = 0, lo = 0;
  for (uint32_t s = 0; s < b->n_segments; ++s) {
    node_offsets[s] = no;
    leaf_offsets[s] = lo;
    uint32_t ns = b->seg_offsets[s + 1] - b->seg_offsets[s];
    if (ns == 0) continue;
    uint32_t r = b->roots[s];
    c.seg_item0 = b->seg_offsets[s];
    uint32_t rn, rl;
    if (is_terminal(&c, r, ref_count(&c, r))) {
      rn = rl = 1;
    } else {
      counts(&c, r & IDX_MASK);
      rn = c.nw[r & IDX_MASK];
      rl = c.nl[r & IDX_MASK];
    }
    emit(&c, r, no, lo, no, lo);
    no += rn;
    lo += rl;
  }
  node_offsets[b->n_segments] = no;
  leaf_offsets[b->n_segments] = lo;
  free(c.nw);
  free(c.nl);
}
