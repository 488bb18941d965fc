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
 * The reference hands out node and leaf-block ids with atomics: a node takes
 * its internal children's ids as one contiguous range and its leaf blocks as
 * another (wide_collapse.mojo:551-559), in an order that varies from run to
 * run.  This restatement and the library number them deterministically with
 * the same shape: a node's internal children get consecutive ids in lane
 * order, followed by the descendants of each child in lane order; a node's
 * own leaf blocks come first, then each internal child's subtree's blocks.
 *
 * With octant slots (spatial_slots, :457-521; the CWBVH8 input, W = 8 and at
 * most three triangles per leaf) the candidates are placed in the eight lanes
 * by the greedy centroid-octant assignment, and the node is then encoded as an
 * 80-byte CWBVH8 node (_encode_cwbvh8_node, bajo/bvh/gpu/
 * compressed_bounds_bvh.mojo:84-325) with its triangles packed as 48-byte
 * [e1][0][e2][0][v0][prim] records (pack_segmented_cwbvh_triangles_kernel,
 * :372-404).  The reference reserves each node's triangle range with an atomic
 * counter; here node I's range starts at the first triangle of I's subtree in
 * depth-first lane order (its own leaf lanes, then each internal child's
 * subtree), one of the orders the atomic can produce. */
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
  int spatial;       /* octant slots (W = 8) */
  float* cw_nodes;   /* CWBVH8 output (NULL: plain wide tree) */
  float* cw_tris;
  uint32_t seg_tri0;
} wctx;

static void ref_box(const wctx* c, uint32_t ref, float out[6]) {
  if (ref & LEAF_FLAG) {
    const float* p = c->b->leaf_bounds + (size_t)c->b->leaf_ids[ref & IDX_MASK] * 6;
    memcpy(out, p, 6 * sizeof(float));
  } else {
    const float* p = c->b->node_bounds + (size_t)(ref & IDX_MASK) * 12;
    for (int k = 0; k < 3; ++k) {
      out[k] = bo_fminf(p[k], p[6 + k]);
      out[3 + k] = bo_fmaxf(p[3 + k], p[9 + k]);
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

/* ---- octant slots ------------------------------------------------------- */
/* perm[slot] = candidate placed in that lane, -1 = empty (spatial_slots,
 * wide_collapse.mojo:457-521): repeatedly give the unassigned candidate and
 * free slot of lowest cost (centroid(candidate) - centroid(parent)) . s(slot)
 * their pairing, s(slot) = (-1 if bit 2 else 1, -1 if bit 1 else 1, -1 if bit
 * 0 else 1); candidates, then slots, are scanned in ascending order and the
 * first minimum is kept (strict <, starting from FLT_MAX).  Centroids are
 * (min + max) * 0.5 (aabb.mojo:53).  Should no pair have a cost below FLT_MAX
 * (NaN boxes), the first unassigned candidate takes the first free slot. */
static void octant_slots(const wctx* c, uint32_t x, const uint32_t* cand, int n, int perm[8]) {
  float bx[6], pc[3], cc[8][3];
  ref_box(c, x, bx);
  for (int k = 0; k < 3; ++k) pc[k] = (bx[k] + bx[3 + k]) * 0.5f;
  for (int j = 0; j < n; ++j) {
    ref_box(c, cand[j], bx);
    for (int k = 0; k < 3; ++k) cc[j][k] = (bx[k] + bx[3 + k]) * 0.5f;
  }
  for (int s = 0; s < 8; ++s) perm[s] = -1;
  uint32_t assigned = 0, occupied = 0;
  for (int it = 0; it < n; ++it) {
    float best = FLT_MAX;
    int bc = -1, bs = -1;
    for (int j = 0; j < n; ++j) {
      if (assigned >> j & 1u) continue;
      const float dx = cc[j][0] - pc[0], dy = cc[j][1] - pc[1], dz = cc[j][2] - pc[2];
      for (int s = 0; s < 8; ++s) {
        if (occupied >> s & 1u) continue;
        const float cost = ((s & 4 ? -dx : dx) + (s & 2 ? -dy : dy)) + (s & 1 ? -dz : dz);
        if (cost < best) {
          best = cost;
          bc = j;
          bs = s;
        }
      }
    }
    if (bc < 0) {
      for (bc = 0; assigned >> bc & 1u; ++bc) {
      }
      for (bs = 0; occupied >> bs & 1u; ++bs) {
      }
    }
    assigned |= 1u << bc;
    occupied |= 1u << bs;
    perm[bs] = bc;
  }
}

/* ---- CWBVH8 encoding ------------------------------------------------------ */
/* _power_of_two_scale_exponent (compressed_bounds_bvh.mojo:43-53): the
 * smallest power of two 2^(e - 127) with 255 * 2^(e - 127) >= extent, e in
 * [1, 254]; 127 for an empty extent. */
static uint32_t cw_exponent(float extent) {
  if (extent <= 0.0f) return 127u;
  const float req = extent / 255.0f;
  uint32_t bits;
  memcpy(&bits, &req, 4);
  uint32_t e = (bits >> 23) & 0xFFu;
  if (bits & 0x007FFFFFu) e += 1u;
  return e < 1u ? 1u : (e > 254u ? 254u : e);
}

static float cw_scale(uint32_t e) {
  const uint32_t bits = e << 23;
  float f;
  memcpy(&f, &bits, 4);
  return f;
}

/* floor / ceil to [0, 255] (NaN -> 0) */
static int cw_clamp255(float f) { return f >= 0.0f ? (f <= 255.0f ? (int)f : 255) : 0; }

/* _quantize_lower / _quantize_upper (:61-76): conservative 8-bit planes */
static uint32_t cw_qlo(float value, float start, float scale) {
  int q = cw_clamp255(floorf((value - start) / scale));
  if (fmaf((float)q, scale, start) > value && q > 0) q -= 1;
  return (uint32_t)q;
}

static uint32_t cw_qhi(float value, float start, float scale) {
  int q = cw_clamp255(ceilf((value - start) / scale));
  if (fmaf((float)q, scale, start) < value && q < 255) q += 1;
  return (uint32_t)q;
}

/* 80-byte node from the 8-lane wide node `wn` ([7][8] field-major, meta as
 * bits; internal data = segment-local child ids, leaf count 1..3), written to
 * `out` (20 words: p xyz, exponents | imask << 24, child base, triangle base,
 * two meta words, 12 quantized-plane words).  Node bounds are the minimum /
 * maximum of the valid lanes in lane order (fmin / fmax as a < b ? a : b). */
static void cw_encode_node(const float* wn, uint32_t tri_base, float* out) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  uint32_t meta[8], child_base = 0, n_int = 0, imask = 0, leaf_off = 0, m0 = 0, m1 = 0;
  for (int j = 0; j < 8; ++j) {
    memcpy(&meta[j], &wn[6 * 8 + j], 4);
    if (meta[j] == EMPTY) continue;
    for (int k = 0; k < 3; ++k) {
      const float a = wn[k * 8 + j], b = wn[(3 + k) * 8 + j];
      lo[k] = lo[k] < a ? lo[k] : a;
      hi[k] = hi[k] > b ? hi[k] : b;
    }
    if ((meta[j] >> 26) == 0) {
      if (n_int == 0) child_base = meta[j] & 0x03FFFFFFu;
      ++n_int;
      imask |= 1u << j;
    }
  }
  uint32_t e[3];
  float sc[3];
  for (int k = 0; k < 3; ++k) {
    e[k] = cw_exponent(hi[k] - lo[k]);
    sc[k] = cw_scale(e[k]);
    if (fmaf(255.0f, sc[k], lo[k]) < hi[k] && e[k] < 254u) {
      e[k] += 1u;
      sc[k] = cw_scale(e[k]);
    }
  }
  uint32_t* w = (uint32_t*)out;
  out[0] = lo[0];
  out[1] = lo[1];
  out[2] = lo[2];
  w[3] = e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24);
  w[4] = child_base;
  w[5] = tri_base;
  for (int j = 0; j < 8; ++j) {
    uint32_t byte = 0;
    const uint32_t count = meta[j] >> 26;
    if (meta[j] == EMPTY) {
      byte = 0;
    } else if (count == 0) {
      byte = 0x20u | (24u + (uint32_t)j); /* internal: 001 | slot + 24 */
    } else {
      byte = (((1u << count) - 1u) << 5) | leaf_off; /* unary count | offset */
      leaf_off += count;
    }
    if (j < 4) m0 |= byte << (8 * j);
    else m1 |= byte << (8 * (j - 4));
  }
  w[6] = m0;
  w[7] = m1;
  for (int plane = 0; plane < 6; ++plane) {
    for (int g = 0; g < 2; ++g) {
      uint32_t packed = 0;
      for (int b = 0; b < 4; ++b) {
        const int j = g * 4 + b;
        uint32_t q = 0;
        if (meta[j] != EMPTY) {
          const int k = plane % 3;
          const float v = wn[plane * 8 + j];
          q = plane < 3 ? cw_qlo(v, lo[k], sc[k]) : cw_qhi(v, lo[k], sc[k]);
        }
        packed |= q << (8 * b);
      }
      w[8 + plane * 2 + g] = packed;
    }
  }
}

/* triangles of the binary subtree `ref` (<= 3 leaves), left to right, as
 * CWBVH records at global position `pos` onward */
static uint32_t cw_write_tris(wctx* c, uint32_t ref, uint32_t pos) {
  uint32_t stack[FAT + 1];
  int sp = 0;
  stack[sp++] = ref;
  while (sp > 0) {
    uint32_t cur = stack[--sp];
    if (cur & LEAF_FLAG) {
      uint32_t item = c->b->leaf_ids[cur & IDX_MASK];
      const float* v = c->verts + (size_t)item * 9;
      float* o = c->cw_tris + (size_t)pos * 12;
      uint32_t prim = item - c->seg_tri0;
      o[0] = v[3] - v[0]; o[1] = v[4] - v[1]; o[2] = v[5] - v[2]; o[3] = 0.0f;
      o[4] = v[6] - v[0]; o[5] = v[7] - v[1]; o[6] = v[8] - v[2]; o[7] = 0.0f;
      o[8] = v[0]; o[9] = v[1]; o[10] = v[2];
      memcpy(&o[11], &prim, 4);
      ++pos;
    } else {
      uint32_t y = cur & IDX_MASK;
      stack[sp++] = c->b->node_meta[(size_t)y * 4 + 2];
      stack[sp++] = c->b->node_meta[(size_t)y * 4 + 1];
    }
  }
  return pos;
}

/* wide node with global id I (local to the segment: I - nb) for binary node x:
 * its internal children take ids D, D + 1, ... in lane order and their
 * descendants follow from D + (internal children); its own leaf blocks start
 * at B (global; local B - lb), and T is the first triangle of its subtree
 * (global; CWBVH8 output only) */
static void emit(wctx* c, uint32_t x, uint32_t I, uint32_t D, uint32_t B, uint32_t T, uint32_t nb, uint32_t lb) {
  const uint32_t W = c->W;
  float* node = c->nodes + (size_t)I * 7 * W;
  float bx[6];
  uint32_t xc = ref_count(c, x);
  if (is_terminal(c, x, xc)) {
    if (c->cw_nodes) {
      cw_write_tris(c, x, T);
    } else {
      write_block(c, x, B);
    }
    ref_box(c, x, bx);
    store_lane(node, W, 0, bx, pack_meta(B - lb, xc));
    for (uint32_t j = 1; j < W; ++j) store_empty(node, W, j);
    if (c->cw_nodes) cw_encode_node(node, T - c->seg_tri0, c->cw_nodes + (size_t)I * 20);
    return;
  }
  uint32_t cand[8], cnt[8];
  int n = open_children(c, x & IDX_MASK, cand, cnt);
  int perm[8];
  if (c->spatial) {
    octant_slots(c, x & IDX_MASK, cand, n, perm);
  } else {
    for (uint32_t j = 0; j < W; ++j) perm[j] = (int)j < n ? (int)j : -1;
  }
  uint32_t n_leaf = 0, n_int = 0, own_tris = 0;
  for (int k = 0; k < n; ++k) {
    if (is_terminal(c, cand[k], cnt[k])) {
      ++n_leaf;
      own_tris += cnt[k];
    } else {
      ++n_int;
    }
  }
  uint32_t own = B, own_t = T, child = D, desc = D + n_int, child_leaf = B + n_leaf, child_t = T + own_tris;
  uint32_t kid[8], kid_id[8], kid_desc[8], kid_lb[8], kid_t[8];
  int nk = 0;
  for (uint32_t j = 0; j < W; ++j) {
    const int k = perm[j];
    if (k < 0) {
      store_empty(node, W, j);
      continue;
    }
    ref_box(c, cand[k], bx);
    if (is_terminal(c, cand[k], cnt[k])) {
      if (c->cw_nodes) {
        own_t = cw_write_tris(c, cand[k], own_t);
      } else {
        write_block(c, cand[k], own);
      }
      store_lane(node, W, j, bx, pack_meta(own - lb, cnt[k]));
      ++own;
    } else {
      uint32_t ci = cand[k] & IDX_MASK;
      store_lane(node, W, j, bx, pack_meta(child - nb, 0));
      kid[nk] = cand[k];
      kid_id[nk] = child;
      kid_desc[nk] = desc;
      kid_lb[nk] = child_leaf;
      kid_t[nk] = child_t;
      ++nk;
      ++child;
      desc += c->nw[ci] - 1u;
      child_leaf += c->nl[ci];
      child_t += cnt[k];
    }
  }
  if (c->cw_nodes) cw_encode_node(node, T - c->seg_tri0, c->cw_nodes + (size_t)I * 20);
  for (int i = 0; i < nk; ++i) emit(c, kid[i], kid_id[i], kid_desc[i], kid_lb[i], kid_t[i], nb, lb);
}

static void wide_build(wctx* c, uint32_t* node_offsets, uint32_t* leaf_offsets) {
  const BoLbvh* b = c->b;
  size_t cap = b->n_leaves ? b->n_leaves : 1;
  c->nw = (uint32_t*)calloc(cap, sizeof(uint32_t));
  c->nl = (uint32_t*)calloc(cap, sizeof(uint32_t));
  uint32_t no = 0, lo = 0;
  for (uint32_t s = 0; s < b->n_segments; ++s) {
    node_offsets[s] = no;
    leaf_offsets[s] = lo;
    uint32_t ns = b->seg_offsets[s + 1] - b->seg_offsets[s];
    if (ns == 0) continue;
    uint32_t r = b->roots[s];
    c->seg_item0 = c->seg_tri0 = b->seg_offsets[s];
    uint32_t rn, rl;
    if (is_terminal(c, r, ref_count(c, r))) {
      rn = rl = 1;
    } else {
      counts(c, r & IDX_MASK);
      rn = c->nw[r & IDX_MASK];
      rl = c->nl[r & IDX_MASK];
    }
    emit(c, r, no, no + 1, lo, b->seg_offsets[s], no, lo);
    no += rn;
    lo += rl;
  }
  node_offsets[b->n_segments] = no;
  leaf_offsets[b->n_segments] = lo;
  free(c->nw);
  free(c->nl);
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
  c.nodes = nodes;
  c.leaf_indices = leaf_indices;
  c.leaf_tris = leaf_tris;
  c.leaf_sorted = leaf_sorted;
  wide_build(&c, node_offsets, leaf_offsets);
}

void bo_cwbvh8_build(const BoLbvh* b, const float* verts, float* wide_nodes, float* cw_nodes, float* cw_tris,
                     uint32_t* node_offsets) {
  wctx c;
  memset(&c, 0, sizeof(c));
  c.max_leaf = 3;
  c.spatial = 1;
  c.b = b;
  c.verts = verts;
  c.W = 8;
  c.nodes = wide_nodes;
  c.cw_nodes = cw_nodes;
  c.cw_tris = cw_tris;
  uint32_t* lo = (uint32_t*)calloc((size_t)b->n_segments + 1, sizeof(uint32_t));
  wide_build(&c, node_offsets, lo);
  free(lo);
}
