/*
 * bajo_oracle.c -- CPU oracle for the LBVH build + closest-hit path.
 *
 * TEST INFRASTRUCTURE ONLY (see bajo_oracle.h).  Plain C11 + pthreads,
 * compiled with -O2 -ffp-contract=off so that float arithmetic is rounded
 * exactly as written.  Reference citations are paths inside jgsimard/bajo.
 */
#define _GNU_SOURCE
#include "bajo_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define BO_FLT_MAX FLT_MAX
/* Slack on the far slab distance: a box is entered when
 * t_near <= t_far * (1 + 2^-20).  Keeps the closest hit independent of the
 * traversal order (the reference compares t_near <= t_far exactly,
 * bajo/core/intersect.mojo:213); the CUDA traversal uses the same constant. */
#define BO_SLACK 1.00000095367431640625f

/* ------------------------------------------------------------------------- */
/* persistent worker pool                                                     */
/* ------------------------------------------------------------------------- */
/* The reference's CPU builders run their parallel loops on the Mojo runtime's
 * persistent worker pool (max.algorithm.parallelize,
 * bajo/bvh/cpu/builder/lbvh.mojo:87,112,199,354).  This pool is the same
 * kind of object: worker threads are started once (grown on demand), spin
 * briefly and then sleep between jobs, and a job hands out [0, n) in chunks
 * through an atomic counter.  One job runs at a time; a nested call, or a
 * call from a second host thread while a job runs, executes inline. */
typedef void (*bo_range_fn)(void* ctx, uint32_t begin, uint32_t end);

typedef struct {
  bo_range_fn fn;
  void* ctx;
  uint64_t n, chunk;
  uint64_t next; /* atomic */
} bo_job;

#define BO_POOL_MAX 256
#define BO_POOL_SPIN 20000

static struct {
  pthread_mutex_t mu;     /* sleeping workers and the submitter's wait */
  pthread_cond_t wake, done;
  pthread_mutex_t submit; /* one job at a time */
  uint32_t started;       /* worker threads running (indices 1..started) */
  uint64_t state;         /* (generation << 16) | workers taking part; atomic */
  uint32_t running;       /* workers still inside the current job; atomic */
  bo_job job;
  uint64_t start_state[BO_POOL_MAX + 1];
} g_pool = {PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, PTHREAD_COND_INITIALIZER,
            PTHREAD_MUTEX_INITIALIZER, 0, 0, 0, {0}, {0}};
static __thread int bo_in_pool;

static inline void bo_relax(void) {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#endif
}

static void bo_run_chunks(bo_job* j) {
  for (;;) {
    uint64_t b = __atomic_fetch_add(&j->next, j->chunk, __ATOMIC_RELAXED);
    if (b >= j->n) break;
    uint64_t e = (j->n - b > j->chunk) ? b + j->chunk : j->n;
    j->fn(j->ctx, (uint32_t)b, (uint32_t)e);
  }
}

static void* bo_pool_worker(void* arg) {
  const uint32_t idx = (uint32_t)(uintptr_t)arg;
  uint64_t seen = g_pool.start_state[idx];
  bo_in_pool = 1;
  for (;;) {
    uint64_t st;
    int spins = 0;
    while ((st = __atomic_load_n(&g_pool.state, __ATOMIC_ACQUIRE)) == seen && spins < BO_POOL_SPIN) {
      bo_relax();
      ++spins;
    }
    if (st == seen) {
      pthread_mutex_lock(&g_pool.mu);
      while ((st = __atomic_load_n(&g_pool.state, __ATOMIC_ACQUIRE)) == seen)
        pthread_cond_wait(&g_pool.wake, &g_pool.mu);
      pthread_mutex_unlock(&g_pool.mu);
    }
    seen = st;
    /* generation and participant count are read as one word, so a worker
     * that slept through a job cannot join the next one twice */
    if (idx > (uint32_t)(st & 0xFFFFu)) continue;
    bo_run_chunks(&g_pool.job);
    if (__atomic_sub_fetch(&g_pool.running, 1u, __ATOMIC_ACQ_REL) == 0) {
      pthread_mutex_lock(&g_pool.mu);
      pthread_cond_signal(&g_pool.done);
      pthread_mutex_unlock(&g_pool.mu);
    }
  }
  return NULL;
}

/* Runs fn over [0, n) in chunks on n_threads threads (the caller included). */
static void bo_parallel_for(uint32_t n, uint32_t n_threads, uint32_t chunk,
                            bo_range_fn fn, void* ctx) {
  if (n == 0) return;
  if (chunk == 0) chunk = 1;
  if (n_threads > BO_POOL_MAX + 1) n_threads = BO_POOL_MAX + 1;
  const uint64_t chunks = ((uint64_t)n + chunk - 1) / chunk;
  uint32_t helpers = (uint32_t)((chunks < n_threads ? chunks : n_threads) - 1);
  if (helpers == 0 || bo_in_pool || pthread_mutex_trylock(&g_pool.submit) != 0) {
    fn(ctx, 0, n);
    return;
  }
  const uint64_t cur = __atomic_load_n(&g_pool.state, __ATOMIC_RELAXED);
  while (g_pool.started < helpers) {
    pthread_t th;
    const uint32_t idx = g_pool.started + 1;
    g_pool.start_state[idx] = cur;
    if (pthread_create(&th, NULL, bo_pool_worker, (void*)(uintptr_t)idx) != 0) break;
    pthread_detach(th);
    g_pool.started = idx;
  }
  if (helpers > g_pool.started) helpers = g_pool.started;
  g_pool.job.fn = fn;
  g_pool.job.ctx = ctx;
  g_pool.job.n = n;
  g_pool.job.chunk = chunk;
  g_pool.job.next = 0;
  __atomic_store_n(&g_pool.running, helpers, __ATOMIC_RELAXED);
  const uint64_t next_state = (((cur >> 16) + 1) << 16) | helpers;
  pthread_mutex_lock(&g_pool.mu);
  __atomic_store_n(&g_pool.state, next_state, __ATOMIC_RELEASE);
  pthread_cond_broadcast(&g_pool.wake);
  pthread_mutex_unlock(&g_pool.mu);
  bo_in_pool = 1;
  bo_run_chunks(&g_pool.job);
  bo_in_pool = 0;
  int spins = 0;
  while (__atomic_load_n(&g_pool.running, __ATOMIC_ACQUIRE) != 0 && spins < BO_POOL_SPIN) {
    bo_relax();
    ++spins;
  }
  pthread_mutex_lock(&g_pool.mu);
  while (__atomic_load_n(&g_pool.running, __ATOMIC_ACQUIRE) != 0) pthread_cond_wait(&g_pool.done, &g_pool.mu);
  pthread_mutex_unlock(&g_pool.mu);
  pthread_mutex_unlock(&g_pool.submit);
}

uint32_t bo_minmax_selftest(uint32_t n_random, uint64_t seed) {
  static const float special[] = {0.0f, -0.0f, 1.0f, -1.0f, INFINITY, -INFINITY, NAN, -NAN,
                                  FLT_MIN, -FLT_MIN, FLT_MAX, -FLT_MAX, 1.0e-45f, -1.0e-45f};
  const uint32_t ns = sizeof special / sizeof special[0];
  uint32_t bad = 0;
  uint64_t x = seed * 2862933555777941757ull + 3037000493ull;
  for (uint32_t i = 0; i < ns * ns + n_random; ++i) {
    float a, b;
    if (i < ns * ns) {
      a = special[i / ns];
      b = special[i % ns];
    } else {
      uint32_t ua, ub;
      x = x * 6364136223846793005ull + 1442695040888963407ull;
      ua = (uint32_t)(x >> 32);
      ub = (uint32_t)x;
      if (i & 1) ub = ua ^ (ub & 0x80000000u); /* equal magnitudes, signs vary */
      if ((ua & 0x7F800000u) == 0x7F800000u && (ua & 0x007FFFFFu)) ua |= 0x00400000u; /* quiet NaNs only */
      if ((ub & 0x7F800000u) == 0x7F800000u && (ub & 0x007FFFFFu)) ub |= 0x00400000u;
      memcpy(&a, &ua, 4);
      memcpy(&b, &ub, 4);
    }
    float r[4] = {bo_fminf(a, b), fminf(a, b), bo_fmaxf(a, b), fmaxf(a, b)};
    if (memcmp(&r[0], &r[1], 4) != 0 && !(r[0] != r[0] && r[1] != r[1])) ++bad;
    if (memcmp(&r[2], &r[3], 4) != 0 && !(r[2] != r[2] && r[3] != r[3])) ++bad;
  }
  return bad;
}

/* ------------------------------------------------------------------------- */
/* vector helpers (bajo/core/vec.mojo)                                         */
/* ------------------------------------------------------------------------- */
typedef struct { float x, y, z; } v3;

static inline v3 v3make(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 v3sub(v3 a, v3 b) { return v3make(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 v3add(v3 a, v3 b) { return v3make(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 v3muls(v3 a, float s) { return v3make(a.x * s, a.y * s, a.z * s); }
static inline v3 v3min(v3 a, v3 b) { return v3make(bo_fminf(a.x, b.x), bo_fminf(a.y, b.y), bo_fminf(a.z, b.z)); }
static inline v3 v3max(v3 a, v3 b) { return v3make(bo_fmaxf(a.x, b.x), bo_fmaxf(a.y, b.y), bo_fmaxf(a.z, b.z)); }
/* dot = fma(a.x, b.x, fma(a.y, b.y, a.z * b.z))  -- vec.mojo:440 */
static inline float v3dot(v3 a, v3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
/* cross -- vec.mojo:522-526 */
static inline v3 v3cross(v3 a, v3 b) {
  return v3make(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)),
                fmaf(a.x, b.y, -(a.y * b.x)));
}
/* normalize -- vec.mojo:529-539 */
static inline v3 v3normalize(v3 v) {
  float l = sqrtf(v3dot(v, v));
  float inv_l = (l > 1.0e-20f) ? 1.0f / l : 0.0f;
  return v3muls(v, inv_l);
}
/* safe_inv -- vec.mojo:373-394 */
static inline float safe_inv1(float e) { return (fabsf(e) > 1.0e-20f) ? 1.0f / e : 0.0f; }

static inline v3 load3(const float* p) { return v3make(p[0], p[1], p[2]); }

/* ------------------------------------------------------------------------- */
/* a1: triangle bounds                                                        */
/* ------------------------------------------------------------------------- */
/* bajo/bvh/gpu/triangle_bvh.mojo:680-727: bmin = vmin(vmin(v0,v1),v2). */
void bo_triangle_bounds(const float* verts, uint32_t n, float* b6) {
  for (uint32_t i = 0; i < n; ++i) {
    const float* v = verts + (size_t)9 * i;
    v3 a = load3(v), b = load3(v + 3), c = load3(v + 6);
    v3 mn = v3min(v3min(a, b), c), mx = v3max(v3max(a, b), c);
    float* o = b6 + (size_t)6 * i;
    o[0] = mn.x; o[1] = mn.y; o[2] = mn.z;
    o[3] = mx.x; o[4] = mx.y; o[5] = mx.z;
  }
}

/* ------------------------------------------------------------------------- */
/* a2: segment bounds                                                         */
/* ------------------------------------------------------------------------- */
/* binary_layout.mojo:128-205 -- root AABB and centroid AABB per segment.
 * AABB.invalid() is (+FLT_MAX, -FLT_MAX) (core/aabb.mojo:28); the centroid is
 * (min + max) * 0.5 (core/aabb.mojo:53).  min/max are exact, so the reduction
 * order of the reference's multi-level tree does not change the result. */
void bo_segment_bounds(const float* b6, const uint32_t* so, uint32_t ns, float* out12) {
  for (uint32_t s = 0; s < ns; ++s) {
    v3 bmn = v3make(BO_FLT_MAX, BO_FLT_MAX, BO_FLT_MAX), bmx = v3make(-BO_FLT_MAX, -BO_FLT_MAX, -BO_FLT_MAX);
    v3 cmn = bmn, cmx = bmx;
    for (uint32_t i = so[s]; i < so[s + 1]; ++i) {
      v3 mn = load3(b6 + (size_t)6 * i), mx = load3(b6 + (size_t)6 * i + 3);
      bmn = v3min(bmn, mn);
      bmx = v3max(bmx, mx);
      v3 c = v3muls(v3add(mn, mx), 0.5f);
      cmn = v3min(cmn, c);
      cmx = v3max(cmx, c);
    }
    float* o = out12 + (size_t)12 * s;
    o[0] = bmn.x; o[1] = bmn.y; o[2] = bmn.z; o[3] = bmx.x; o[4] = bmx.y; o[5] = bmx.z;
    o[6] = cmn.x; o[7] = cmn.y; o[8] = cmn.z; o[9] = cmx.x; o[10] = cmx.y; o[11] = cmx.z;
  }
}

/* ------------------------------------------------------------------------- */
/* a3: Morton                                                                 */
/* ------------------------------------------------------------------------- */
/* core/morton.mojo:48-58 */
uint32_t bo_expand_bits_3d(uint32_t n) {
  n = (n ^ (n << 16)) & 0xFF0000FFu;
  n = (n ^ (n << 8)) & 0x0300F00Fu;
  n = (n ^ (n << 4)) & 0x030C30C3u;
  n = (n ^ (n << 2)) & 0x09249249u;
  return n;
}

/* float -> u32 with truncation, clamped to [0, 1023]  (core/morton.mojo:78) */
static inline uint32_t quantize1024(float c) {
  float s = c * 1024.0f;
  uint32_t u;
  if (!(s > 0.0f)) u = 0;                 /* negatives and NaN -> 0 */
  else if (s >= 4294967296.0f) u = 1023;  /* out of u32 range -> saturate */
  else u = (uint32_t)s;
  return u > 1023u ? 1023u : u;
}

/* core/morton.mojo:61-89: code = e(z)<<2 | e(y)<<1 | e(x). */
uint32_t bo_morton3(float x, float y, float z) {
  return (bo_expand_bits_3d(quantize1024(z)) << 2) | (bo_expand_bits_3d(quantize1024(y)) << 1) |
         bo_expand_bits_3d(quantize1024(x));
}

/* core/morton.mojo:22-31: clz64((ca<<32|ia) ^ (cb<<32|ib)), 64 when equal. */
int bo_morton_common_prefix(uint32_t ca, uint32_t ia, uint32_t cb, uint32_t ib) {
  uint64_t x = (((uint64_t)ca << 32) | ia) ^ (((uint64_t)cb << 32) | ib);
  return x ? __builtin_clzll(x) : 64;
}

/* binary_layout.mojo:116-125 */
static uint32_t segment_for_item(const uint32_t* off, uint32_t n_off, uint32_t item) {
  uint32_t lo = 0, hi = n_off - 1;
  while (lo + 1 < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (item < off[mid]) hi = mid; else lo = mid;
  }
  return lo;
}

/* bajo/bvh/gpu/builder/lbvh.mojo:30-62: normalise the leaf centroid over the
 * segment's CENTROID bounds with safe_inv, key = (segment << 32) | morton,
 * value = global item index. */
void bo_morton_keys(const float* b6, const uint32_t* so, uint32_t ns, const float* sb12,
                    uint32_t n, uint64_t* keys, uint32_t* values) {
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t s = segment_for_item(so, ns + 1, i);
    const float* cb = sb12 + (size_t)12 * s + 6;
    v3 cmin = load3(cb), cmax = load3(cb + 3);
    v3 ext = v3sub(cmax, cmin);
    v3 inv = v3make(safe_inv1(ext.x), safe_inv1(ext.y), safe_inv1(ext.z));
    v3 mn = load3(b6 + (size_t)6 * i), mx = load3(b6 + (size_t)6 * i + 3);
    v3 c = v3muls(v3add(mn, mx), 0.5f);
    v3 d = v3sub(c, cmin);
    v3 u = v3make(d.x * inv.x, d.y * inv.y, d.z * inv.z);
    keys[i] = ((uint64_t)s << 32) | bo_morton3(u.x, u.y, u.z);
    values[i] = i;
  }
}

/* ------------------------------------------------------------------------- */
/* a4/a5: stable LSD radix sort, 8-bit digits                                 */
/* ------------------------------------------------------------------------- */
/* bajo/bvh/cpu/builder/lbvh.mojo:36-62 (one counting pass per byte).  Any
 * stable sort yields the same permutation; the digit range [begin_bit,
 * end_bit) mirrors the library's API. */
#define BO_SORT_IMPL(NAME, KT, HASV)                                              \
  void NAME(KT* keys, uint32_t* vals, uint32_t n, int begin_bit, int end_bit) {   \
    if (n == 0) return;                                                           \
    KT* kt = (KT*)malloc(sizeof(KT) * n);                                         \
    uint32_t* vt = HASV ? (uint32_t*)malloc(sizeof(uint32_t) * n) : NULL;         \
    KT* ks = keys; KT* kd = kt;                                                   \
    uint32_t* vs = vals; uint32_t* vd = vt;                                       \
    for (int sh = begin_bit; sh < end_bit; sh += 8) {                             \
      int bits = end_bit - sh < 8 ? end_bit - sh : 8;                             \
      KT mask = (KT)((1u << bits) - 1u);                                          \
      uint32_t cnt[256];                                                          \
      memset(cnt, 0, sizeof cnt);                                                 \
      for (uint32_t i = 0; i < n; ++i) cnt[(ks[i] >> sh) & mask]++;               \
      uint32_t off[256], acc = 0;                                                 \
      for (int b = 0; b < 256; ++b) { off[b] = acc; acc += cnt[b]; }              \
      for (uint32_t i = 0; i < n; ++i) {                                          \
        uint32_t d = (uint32_t)((ks[i] >> sh) & mask);                            \
        uint32_t o = off[d]++;                                                    \
        kd[o] = ks[i];                                                            \
        if (HASV) vd[o] = vs[i];                                                  \
      }                                                                           \
      KT* tk = ks; ks = kd; kd = tk;                                              \
      uint32_t* tv = vs; vs = vd; vd = tv;                                        \
    }                                                                             \
    if (ks != keys) {                                                             \
      memcpy(keys, ks, sizeof(KT) * n);                                           \
      if (HASV) memcpy(vals, vs, sizeof(uint32_t) * n);                           \
    }                                                                             \
    free(kt);                                                                     \
    free(vt);                                                                     \
  }

BO_SORT_IMPL(bo_sort_pairs_u64, uint64_t, 1)
BO_SORT_IMPL(bo_sort_pairs_u32, uint32_t, 1)
static BO_SORT_IMPL(bo_sort_keys_u32_impl, uint32_t, 0)
static BO_SORT_IMPL(bo_sort_keys_u64_impl, uint64_t, 0)
void bo_sort_keys_u32(uint32_t* k, uint32_t n, int b, int e) { bo_sort_keys_u32_impl(k, NULL, n, b, e); }
void bo_sort_keys_u64(uint64_t* k, uint32_t n, int b, int e) { bo_sort_keys_u64_impl(k, NULL, n, b, e); }

/* Multithreaded stable LSD radix sort, the CPU sort baseline.  Each pass is
 * the reference CPU builder's parallel pass (bajo/bvh/cpu/builder/
 * lbvh.mojo:65-110): per-worker digit histograms over contiguous chunks,
 * destinations assigned digit-major then worker-major (which keeps the pass
 * stable), then a parallel scatter.  8-bit digits over [begin_bit, end_bit);
 * scratch from bo_cpu_sort_scratch_bytes (alternate buffers and histograms),
 * so nothing is allocated per call. */
typedef struct {
  const void* ks;
  void* kd;
  const uint32_t* vs;
  uint32_t* vd;
  uint32_t n, workers, shift, mask, key_bytes;
  uint32_t* counts;  /* [workers][256] */
} cpu_sort_ctx;

static inline uint32_t cs_digit(const cpu_sort_ctx* c, uint32_t i) {
  return c->key_bytes == 8 ? (uint32_t)((((const uint64_t*)c->ks)[i] >> c->shift) & c->mask)
                           : (((const uint32_t*)c->ks)[i] >> c->shift) & c->mask;
}
static void cs_hist(void* p, uint32_t b, uint32_t e) {
  cpu_sort_ctx* c = (cpu_sort_ctx*)p;
  for (uint32_t w = b; w < e; ++w) {
    uint32_t* cnt = c->counts + 256 * (size_t)w;
    memset(cnt, 0, 256 * sizeof(uint32_t));
    uint32_t first = (uint32_t)((uint64_t)c->n * w / c->workers), end = (uint32_t)((uint64_t)c->n * (w + 1) / c->workers);
    for (uint32_t i = first; i < end; ++i) cnt[cs_digit(c, i)]++;
  }
}
static void cs_scatter(void* p, uint32_t b, uint32_t e) {
  cpu_sort_ctx* c = (cpu_sort_ctx*)p;
  for (uint32_t w = b; w < e; ++w) {
    uint32_t off[256];
    memcpy(off, c->counts + 256 * (size_t)w, sizeof off);  /* offsets by now */
    uint32_t first = (uint32_t)((uint64_t)c->n * w / c->workers), end = (uint32_t)((uint64_t)c->n * (w + 1) / c->workers);
    if (c->key_bytes == 8) {
      const uint64_t* ks = (const uint64_t*)c->ks;
      uint64_t* kd = (uint64_t*)c->kd;
      for (uint32_t i = first; i < end; ++i) {
        uint32_t o = off[(uint32_t)((ks[i] >> c->shift) & c->mask)]++;
        kd[o] = ks[i];
        if (c->vs) c->vd[o] = c->vs[i];
      }
    } else {
      const uint32_t* ks = (const uint32_t*)c->ks;
      uint32_t* kd = (uint32_t*)c->kd;
      for (uint32_t i = first; i < end; ++i) {
        uint32_t o = off[(ks[i] >> c->shift) & c->mask]++;
        kd[o] = ks[i];
        if (c->vs) c->vd[o] = c->vs[i];
      }
    }
  }
}

size_t bo_cpu_sort_scratch_bytes(uint32_t n, uint32_t key_bytes, int has_values, uint32_t n_threads) {
  if (n_threads == 0) n_threads = 1;
  size_t o = ((size_t)n * key_bytes + 63) & ~(size_t)63;
  if (has_values) o += ((size_t)n * 4 + 63) & ~(size_t)63;
  return o + sizeof(uint32_t) * 256 * (size_t)n_threads;
}

void bo_cpu_sort(void* keys, uint32_t* vals, uint32_t n, uint32_t key_bytes, int begin_bit, int end_bit,
                 uint32_t n_threads, void* scratch) {
  if (n <= 1 || begin_bit >= end_bit) return;
  if (n_threads == 0) n_threads = 1;
  const uint32_t workers = n_threads < n ? n_threads : n;
  unsigned char* sb = (unsigned char*)scratch;
  void* kalt = sb;
  size_t o = ((size_t)n * key_bytes + 63) & ~(size_t)63;
  uint32_t* valt = vals ? (uint32_t*)(sb + o) : NULL;
  if (vals) o += ((size_t)n * 4 + 63) & ~(size_t)63;
  cpu_sort_ctx c;
  c.n = n;
  c.workers = workers;
  c.key_bytes = key_bytes;
  c.counts = (uint32_t*)(sb + o);
  void* ks = keys;
  void* kd = kalt;
  uint32_t* vs = vals;
  uint32_t* vd = valt;
  for (int sh = begin_bit; sh < end_bit; sh += 8) {
    int bits = end_bit - sh < 8 ? end_bit - sh : 8;
    c.ks = ks;
    c.kd = kd;
    c.vs = vs;
    c.vd = vd;
    c.shift = (uint32_t)sh;
    c.mask = (1u << bits) - 1u;
    bo_parallel_for(workers, workers, 1, cs_hist, &c);
    uint32_t acc = 0;
    for (uint32_t b = 0; b <= c.mask; ++b)
      for (uint32_t w = 0; w < workers; ++w) {
        uint32_t cnt = c.counts[256 * (size_t)w + b];
        c.counts[256 * (size_t)w + b] = acc;
        acc += cnt;
      }
    bo_parallel_for(workers, workers, 1, cs_scatter, &c);
    void* tk = ks; ks = kd; kd = tk;
    uint32_t* tv = vs; vs = vd; vd = tv;
  }
  if (ks != keys) {
    memcpy(keys, ks, (size_t)n * key_bytes);
    if (vals) memcpy(vals, vs, (size_t)n * 4);
  }
}

/* 63-bit 3D Morton code, 21 bits per axis (the sort workload's 64-bit keys):
 * u = clamp(u32(c * 2^21), 0, 2^21 - 1) per axis as quantize1024 does with
 * 10 bits (core/morton.mojo:78), code = e(z) << 2 | e(y) << 1 | e(x). */
static inline uint64_t expand_bits_21(uint64_t v) {
  v &= 0x1FFFFFull;
  v = (v | (v << 32)) & 0x001F00000000FFFFull;
  v = (v | (v << 16)) & 0x001F0000FF0000FFull;
  v = (v | (v << 8)) & 0x100F00F00F00F00Full;
  v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}
static inline uint64_t quantize21(float c) {
  float s = c * 2097152.0f;
  if (!(s > 0.0f)) return 0;
  if (s >= 2097151.0f) return 2097151ull;
  return (uint64_t)s;
}
void bo_morton63(const float* xyz, uint32_t n, uint64_t* out) {
  for (uint32_t i = 0; i < n; ++i) {
    const float* p = xyz + (size_t)3 * i;
    out[i] = (expand_bits_21(quantize21(p[2])) << 2) | (expand_bits_21(quantize21(p[1])) << 1) |
             expand_bits_21(quantize21(p[0]));
  }
}

/* ------------------------------------------------------------------------- */
/* a7/a8: Karras topology                                                     */
/* ------------------------------------------------------------------------- */
/* binary_layout.mojo:219-223: internal count per segment = max(count-1, 0). */
void bo_internal_offsets(const uint32_t* so, uint32_t ns, uint32_t* io) {
  io[0] = 0;
  for (uint32_t s = 0; s < ns; ++s) {
    uint32_t c = so[s + 1] - so[s];
    io[s + 1] = io[s] + (c > 0 ? c - 1 : 0);
  }
}

/* lbvh.mojo:221-232 -- delta over segment-local sorted positions, -1 outside */
static inline int cp_(const uint32_t* codes, int64_t len, int64_t i, int64_t j) {
  if (j < 0 || j >= len) return -1;
  return bo_morton_common_prefix(codes[i], (uint32_t)i, codes[j], (uint32_t)j);
}

/* lbvh.mojo:164-191 */
static void find_range(const uint32_t* codes, int64_t len, int64_t i, int64_t* first, int64_t* last) {
  int d_next = cp_(codes, len, i, i + 1);
  int d_prev = cp_(codes, len, i, i - 1);
  int64_t d = (d_next < d_prev) ? -1 : 1;
  int delta_min = cp_(codes, len, i, i - d);
  int64_t lmax = 2;
  while (cp_(codes, len, i, i + lmax * d) > delta_min) {
    lmax <<= 1;
    if (lmax > len * 2) break;
  }
  int64_t l = 0;
  for (int64_t t = lmax >> 1; t > 0; t >>= 1)
    if (cp_(codes, len, i, i + (l + t) * d) > delta_min) l += t;
  int64_t j = i + l * d;
  *first = i < j ? i : j;
  *last = i < j ? j : i;
}

/* lbvh.mojo:194-218 (identical to bajo/bvh/cpu/builder/lbvh.mojo:144-163) */
static int64_t find_split(const uint32_t* codes, int64_t len, int64_t first, int64_t last) {
  int node_prefix = cp_(codes, len, first, last);
  int64_t split = first, step = last - first;
  while (step > 1) {
    step = (step + 1) >> 1;
    int64_t ns = split + step;
    if (ns < last && cp_(codes, len, first, ns) > node_prefix) split = ns;
  }
  return split;
}

static void set_invalid12(float* b) {
  for (int k = 0; k < 2; ++k) {
    b[6 * k + 0] = b[6 * k + 1] = b[6 * k + 2] = BO_FLT_MAX;
    b[6 * k + 3] = b[6 * k + 4] = b[6 * k + 5] = -BO_FLT_MAX;
  }
}

/* lbvh.mojo:235-255 (roots) + 257-329 (one internal node per step) */
void bo_lbvh_topology(const uint32_t* codes_all, const uint32_t* so, const uint32_t* io, uint32_t ns,
                      uint32_t* meta, uint32_t* leaf_parent, uint32_t* leaf_counts, uint32_t* roots,
                      float* node_bounds) {
  for (uint32_t s = 0; s < ns; ++s) {
    uint32_t lb = so[s], le = so[s + 1];
    if (le == lb) roots[s] = BO_SENTINEL;
    else if (le - lb == 1) { roots[s] = BO_LEAF_FLAG | lb; leaf_parent[lb] = BO_SENTINEL; }
    else roots[s] = io[s];
  }
  for (uint32_t s = 0; s < ns; ++s) {
    uint32_t ib = io[s], lb = so[s];
    int64_t len = (int64_t)so[s + 1] - lb;
    const uint32_t* codes = codes_all + lb;
    for (uint32_t i = ib; i < io[s + 1]; ++i) {
      int64_t li = i - ib, first, last;
      if (node_bounds) set_invalid12(node_bounds + (size_t)12 * i);
      find_range(codes, len, li, &first, &last);
      leaf_counts[i] = (uint32_t)(last - first + 1);
      if (first == 0 && last == len - 1) meta[4 * (size_t)i + 0] = BO_SENTINEL;
      int64_t split = find_split(codes, len, first, last);
      uint32_t left = ib + (uint32_t)split, right = ib + (uint32_t)split + 1;
      if (split == first) { left = BO_LEAF_FLAG | (lb + (uint32_t)split); leaf_parent[lb + split] = i; }
      else meta[4 * (size_t)(ib + split) + 0] = i;
      if (split + 1 == last) { right = BO_LEAF_FLAG | (lb + (uint32_t)split + 1); leaf_parent[lb + split + 1] = i; }
      else meta[4 * (size_t)(ib + split + 1) + 0] = i;
      meta[4 * (size_t)i + 1] = left;
      meta[4 * (size_t)i + 2] = right;
      meta[4 * (size_t)i + 3] = lb + (uint32_t)last;
    }
  }
}

/* Top-down restatement following bajo/bvh/cpu/builder/lbvh.mojo:270-315 but
 * numbering nodes with the Karras rule, so it must reproduce
 * bo_lbvh_topology exactly. */
static void topdown_rec(const uint32_t* codes, int64_t len, uint32_t lb, uint32_t ib, uint32_t node,
                        uint32_t parent, int64_t first, int64_t last, uint32_t* meta, uint32_t* lp,
                        uint32_t* lc) {
  for (;;) {
    meta[4 * (size_t)node + 0] = parent;
    lc[node] = (uint32_t)(last - first + 1);
    meta[4 * (size_t)node + 3] = lb + (uint32_t)last;
    int64_t split = find_split(codes, len, first, last);
    uint32_t l, r;
    if (split == first) { l = BO_LEAF_FLAG | (lb + (uint32_t)split); lp[lb + split] = node; }
    else l = ib + (uint32_t)split;
    if (split + 1 == last) { r = BO_LEAF_FLAG | (lb + (uint32_t)split + 1); lp[lb + split + 1] = node; }
    else r = ib + (uint32_t)split + 1;
    meta[4 * (size_t)node + 1] = l;
    meta[4 * (size_t)node + 2] = r;
    if (!(l & BO_LEAF_FLAG)) topdown_rec(codes, len, lb, ib, l, node, first, split, meta, lp, lc);
    if (r & BO_LEAF_FLAG) return;
    parent = node;
    node = r;
    first = split + 1;
  }
}

void bo_lbvh_topology_topdown(const uint32_t* codes_all, const uint32_t* so, const uint32_t* io,
                              uint32_t ns, uint32_t* meta, uint32_t* lp, uint32_t* lc, uint32_t* roots) {
  for (uint32_t s = 0; s < ns; ++s) {
    uint32_t lb = so[s], le = so[s + 1];
    int64_t len = (int64_t)le - lb;
    if (len == 0) { roots[s] = BO_SENTINEL; continue; }
    if (len == 1) { roots[s] = BO_LEAF_FLAG | lb; lp[lb] = BO_SENTINEL; continue; }
    roots[s] = io[s];
    topdown_rec(codes_all + lb, len, lb, io[s], io[s], BO_SENTINEL, 0, len - 1, meta, lp, lc);
  }
}

/* ------------------------------------------------------------------------- */
/* a9: refit                                                                  */
/* ------------------------------------------------------------------------- */
static void child_box(uint32_t ref, const float* lb6, const uint32_t* ids, const float* nb, float out[6]) {
  if (ref & BO_LEAF_FLAG) {
    memcpy(out, lb6 + (size_t)6 * ids[ref & 0x7FFFFFFFu], 6 * sizeof(float));
  } else {
    const float* b = nb + (size_t)12 * ref;
    for (int k = 0; k < 3; ++k) {
      out[k] = bo_fminf(b[k], b[6 + k]);
      out[3 + k] = bo_fmaxf(b[3 + k], b[9 + k]);
    }
  }
}

/* lbvh.mojo:116-161 -- bottom-up climb with an arrival counter.  Processing
 * nodes children-first gives the same values (min/max are exact) and the
 * same final counters (2 per internal node). */
void bo_lbvh_refit(const float* lb6, const uint32_t* ids, const uint32_t* meta, const uint32_t* lp,
                   uint32_t n_leaves, uint32_t n_internal, float* nb, uint32_t* flags) {
  (void)lp;
  (void)n_leaves;
  /* post-order over every tree: iterative, visiting children before parents */
  uint8_t* done = (uint8_t*)calloc(n_internal ? n_internal : 1, 1);
  uint32_t* stack = (uint32_t*)malloc(sizeof(uint32_t) * (n_internal ? n_internal : 1) * 2 + 16);
  for (uint32_t root = 0; root < n_internal; ++root) {
    if (meta[4 * (size_t)root] != BO_SENTINEL || done[root]) continue;
    uint32_t sp = 0;
    stack[sp++] = root;
    while (sp) {
      uint32_t node = stack[sp - 1];
      uint32_t l = meta[4 * (size_t)node + 1], r = meta[4 * (size_t)node + 2];
      int pushed = 0;
      if (!(l & BO_LEAF_FLAG) && !done[l]) { stack[sp++] = l; pushed = 1; }
      if (!(r & BO_LEAF_FLAG) && !done[r]) { stack[sp++] = r; pushed = 1; }
      if (pushed) continue;
      --sp;
      child_box(l, lb6, ids, nb, nb + (size_t)12 * node);
      child_box(r, lb6, ids, nb, nb + (size_t)12 * node + 6);
      flags[node] = 2;
      done[node] = 1;
    }
  }
  free(stack);
  free(done);
}

/* ------------------------------------------------------------------------- */
/* full build                                                                 */
/* ------------------------------------------------------------------------- */
/* bajo/bvh/gpu/builder/lbvh.mojo:332-424 in order: bounds, Morton, sort of the
 * live digits (bits 0..29 and the segment bits), gather low words, roots,
 * topology, refit.  The caller allocates every array in BoLbvh. */
void bo_lbvh_build(const float* verts, const uint32_t* so, uint32_t ns, BoLbvh* o) {
  uint32_t n = so[ns];
  o->n_leaves = n;
  o->n_segments = ns;
  o->seg_offsets = so;
  bo_internal_offsets(so, ns, o->internal_offsets);
  o->n_internal = o->internal_offsets[ns];
  bo_triangle_bounds(verts, n, o->leaf_bounds);
  bo_segment_bounds(o->leaf_bounds, so, ns, o->seg_bounds);
  bo_morton_keys(o->leaf_bounds, so, ns, o->seg_bounds, n, o->sort_keys, o->leaf_ids);
  int seg_bits = 0;
  while (seg_bits < 32 && (ns - 1) >> seg_bits) ++seg_bits;
  bo_sort_pairs_u64(o->sort_keys, o->leaf_ids, n, 0, 32 + seg_bits);
  for (uint32_t i = 0; i < n; ++i) o->morton_codes[i] = (uint32_t)(o->sort_keys[i] & 0xFFFFFFFFu);
  if (o->n_internal == 0) {
    o->node_meta[0] = o->node_meta[1] = o->node_meta[2] = o->node_meta[3] = 0;
    set_invalid12(o->node_bounds);
    o->node_leaf_counts[0] = 0;
    o->node_flags[0] = 0;
  }
  bo_lbvh_topology(o->morton_codes, so, o->internal_offsets, ns, o->node_meta, o->leaf_parent,
                   o->node_leaf_counts, o->roots, o->n_internal ? o->node_bounds : NULL);
  for (uint32_t i = 0; i < o->n_internal; ++i) o->node_flags[i] = 0;
  bo_lbvh_refit(o->leaf_bounds, o->leaf_ids, o->node_meta, o->leaf_parent, n, o->n_internal,
                o->node_bounds, o->node_flags);
}

/* ------------------------------------------------------------------------- */
/* a12: camera                                                                */
/* ------------------------------------------------------------------------- */
/* camera.mojo:77-97 (defocus angle 0 -> zero disk vectors) */
void bo_camera_make(const float o[3], const float t[3], const float up[3], float fov_scale, float out[20]) {
  v3 org = load3(o), tgt = load3(t), wup = load3(up);
  v3 fwd = v3normalize(v3sub(tgt, org));
  v3 right = v3normalize(v3cross(fwd, wup));
  v3 u = v3normalize(v3cross(right, fwd));
  memset(out, 0, 20 * sizeof(float));
  out[0] = org.x; out[1] = org.y; out[2] = org.z;
  out[3] = fwd.x; out[4] = fwd.y; out[5] = fwd.z;
  out[6] = right.x; out[7] = right.y; out[8] = right.z;
  out[9] = u.x; out[10] = u.y; out[11] = u.z;
  out[12] = fov_scale;
  out[13] = 1.0f; /* focus distance */
}

/* camera.mojo:100-116: fov_scale = tan(radians(vfov) / 2) */
void bo_camera_from_vfov(const float o[3], const float t[3], const float up[3], float vfov, float out[20]) {
  float theta = vfov * (float)(3.14159265358979323846 / 180.0);
  bo_camera_make(o, t, up, tanf(theta / 2.0f), out);
}

/* camera.mojo:137-154 make_ray_raster; camera_launch.mojo:34-55 view select */
static void camera_ray(const float* cams, uint32_t idx, uint32_t w, uint32_t h, float inv_h, v3* o, v3* d) {
  uint32_t ppv = w * h;
  uint32_t view = idx / ppv, local = idx - view * ppv;
  const float* c = cams + (size_t)20 * view;
  uint32_t px = local % w, py = local / w;
  float sx = (2.0f * ((float)px + 0.5f) - (float)w) * inv_h;
  float sy = 1.0f - 2.0f * ((float)py + 0.5f) * inv_h;
  float fs = c[12];
  v3 fwd = load3(c + 3), right = load3(c + 6), up = load3(c + 9);
  v3 dir = v3add(v3add(fwd, v3muls(right, sx * fs)), v3muls(up, sy * fs));
  *o = load3(c);
  *d = v3normalize(dir);
}

void bo_camera_rays(const float* cams, uint32_t n, uint32_t w, uint32_t h, float* rays) {
  float inv_h = 1.0f / (float)h;
  for (uint32_t i = 0; i < n; ++i) {
    v3 o, d;
    camera_ray(cams, i, w, h, inv_h, &o, &d);
    rays[0 * (size_t)n + i] = o.x; rays[1 * (size_t)n + i] = o.y; rays[2 * (size_t)n + i] = o.z;
    rays[3 * (size_t)n + i] = 0.0f;
    rays[4 * (size_t)n + i] = d.x; rays[5 * (size_t)n + i] = d.y; rays[6 * (size_t)n + i] = d.z;
    rays[7 * (size_t)n + i] = BO_FLT_MAX;
  }
}

/* ------------------------------------------------------------------------- */
/* a11: ray / box and ray / triangle                                          */
/* ------------------------------------------------------------------------- */
typedef struct {
  v3 o, d, rcp;
  float tmin, tmax;
  int kx, ky, kz;
  float sx, sy, sz;
  int par[3]; /* |d| <= 1e-9 on this axis */
} bo_ray;

static inline float idx3(v3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

/* ray.mojo:86-111 rcp_direction: |d| > 1e-9 ? 1/d : +-1e9 */
static inline float rcp1(float d) {
  const float eps = 1.0e-9f;
  const float large = 1.0f / eps;
  return fabsf(d) > eps ? 1.0f / d : (d < 0.0f ? -large : large);
}

static bo_ray make_ray_od(v3 o, v3 d, float tmin, float tmax) {
  bo_ray r;
  r.o = o;
  r.tmin = tmin;
  r.d = d;
  r.tmax = tmax;
  r.rcp = v3make(rcp1(r.d.x), rcp1(r.d.y), rcp1(r.d.z));
  r.par[0] = !(fabsf(r.d.x) > 1.0e-9f);
  r.par[1] = !(fabsf(r.d.y) > 1.0e-9f);
  r.par[2] = !(fabsf(r.d.z) > 1.0e-9f);
  /* watertight set-up (Woop, Benthin, Wald, JCGT 2(1) 2013, section 3) */
  float ax = fabsf(r.d.x), ay = fabsf(r.d.y), az = fabsf(r.d.z);
  r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  r.kx = r.kz == 2 ? 0 : r.kz + 1;
  r.ky = r.kx == 2 ? 0 : r.kx + 1;
  float dz = idx3(r.d, r.kz);
  if (dz < 0.0f) { int t = r.kx; r.kx = r.ky; r.ky = t; }
  r.sx = idx3(r.d, r.kx) / dz;
  r.sy = idx3(r.d, r.ky) / dz;
  r.sz = 1.0f / dz;
  return r;
}

static bo_ray make_ray(const float* rays, uint32_t n, uint32_t i) {
  return make_ray_od(v3make(rays[i], rays[(size_t)n + i], rays[2 * (size_t)n + i]), v3make(rays[4 * (size_t)n + i], rays[5 * (size_t)n + i], rays[6 * (size_t)n + i]),
                     rays[3 * (size_t)n + i], rays[7 * (size_t)n + i]);
}

/* one slab: (b - o) * rcp, except on axes the ray is parallel to
 * (|d| <= 1e-9), which are tested by containment: [-inf, inf] when the origin
 * lies inside [bmin, bmax], empty otherwise.  The reference's +-1e9 reciprocal
 * (ray.mojo:86-111) gives a ray that runs exactly along a box face an empty
 * slab; containment keeps such rays inside the (closed) box. */
static inline void slab(float bmin, float bmax, float o, float rcp, int par, float* t0, float* t1) {
  if (par) {
    *t0 = bmin <= o ? -INFINITY : INFINITY;
    *t1 = bmax >= o ? INFINITY : -INFINITY;
  } else {
    *t0 = (bmin - o) * rcp;
    *t1 = (bmax - o) * rcp;
  }
}

/* intersect.mojo:193-215 with the far bound scaled by BO_SLACK */
static inline int box_hit(const bo_ray* r, const float* b, float tlimit, float* tnear) {
  float t0x, t1x, t0y, t1y, t0z, t1z;
  slab(b[0], b[3], r->o.x, r->rcp.x, r->par[0], &t0x, &t1x);
  slab(b[1], b[4], r->o.y, r->rcp.y, r->par[1], &t0y, &t1y);
  slab(b[2], b[5], r->o.z, r->rcp.z, r->par[2], &t0z, &t1z);
  float tn = bo_fmaxf(bo_fmaxf(bo_fminf(t0x, t1x), bo_fminf(t0y, t1y)), bo_fmaxf(bo_fminf(t0z, t1z), 0.0f));
  float tf = bo_fminf(bo_fminf(bo_fmaxf(t0x, t1x), bo_fmaxf(t0y, t1y)), bo_fminf(bo_fmaxf(t0z, t1z), tlimit));
  *tnear = tn;
  return tn <= tf * BO_SLACK;
}

typedef struct { float t, u, v; uint32_t prim; v3 n; } bo_hit;

/* closest-hit order: smaller t wins, equal t goes to the lower prim id.  The
 * reference keeps the first-visited candidate on ties (strict t < t_max,
 * intersect.mojo:451). */
static inline int better(float t, uint32_t prim, const bo_hit* h) {
  return t < h->t || (t == h->t && prim < h->prim);
}

/* intersect.mojo:415-459 Moller-Trumbore with precomputed edges */
static inline int tri_mt(const bo_ray* r, v3 v0, v3 e1, v3 e2, float* t, float* u, float* v) {
  v3 p = v3cross(r->d, e2);
  float det = v3dot(e1, p);
  int det_ok = det > 1e-8f || det < -1e-8f;
  float inv_det = 1.0f / det;
  v3 tv = v3sub(r->o, v0);
  float uu = v3dot(tv, p) * inv_det;
  v3 q = v3cross(tv, e1);
  float vv = v3dot(r->d, q) * inv_det;
  float tt = v3dot(e2, q) * inv_det;
  *t = tt; *u = uu; *v = vv;
  return det_ok && uu >= 0.0f && uu <= 1.0f && vv >= 0.0f && (uu + vv) <= 1.0f && tt > r->tmin;
}

/* Woop/Benthin/Wald 2013, algorithm of section 3 (no backface culling):
 * shear to ray space, 2D edge functions without contraction (so a shared edge
 * evaluates to exactly opposite values on both triangles), double-precision
 * re-evaluation when an edge function is exactly zero. */
static inline int tri_wt(const bo_ray* r, v3 v0, v3 v1, v3 v2, float* t, float* u, float* v) {
  v3 A = v3sub(v0, r->o), B = v3sub(v1, r->o), C = v3sub(v2, r->o);
  float Akz = idx3(A, r->kz), Bkz = idx3(B, r->kz), Ckz = idx3(C, r->kz);
  float Ax = idx3(A, r->kx) - r->sx * Akz, Ay = idx3(A, r->ky) - r->sy * Akz;
  float Bx = idx3(B, r->kx) - r->sx * Bkz, By = idx3(B, r->ky) - r->sy * Bkz;
  float Cx = idx3(C, r->kx) - r->sx * Ckz, Cy = idx3(C, r->ky) - r->sy * Ckz;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
  float det = U + V + W;
  if (det == 0.0f) return 0;
  float Az = r->sz * Akz, Bz = r->sz * Bkz, Cz = r->sz * Ckz;
  float T = U * Az + V * Bz + W * Cz;
  float tt = T / det;
  *t = tt;
  *u = V / det;
  *v = W / det;
  return tt > r->tmin;
}

/* one triangle, item id `item`, reported as `prim` */
static inline void test_tri(const bo_ray* r, const float* verts, uint32_t item, uint32_t prim, int mode,
                            bo_hit* h) {
  const float* p = verts + (size_t)9 * item;
  v3 v0 = load3(p), v1 = load3(p + 3), v2 = load3(p + 6);
  v3 e1 = v3sub(v1, v0), e2 = v3sub(v2, v0);
  float t, u, v;
  int ok = mode == BO_TRI_MT ? tri_mt(r, v0, e1, e2, &t, &u, &v) : tri_wt(r, v0, v1, v2, &t, &u, &v);
  if (ok && t < r->tmax && better(t, prim, h)) {
    h->t = t; h->u = u; h->v = v; h->prim = prim;
    h->n = v3normalize(v3cross(e1, e2));
  }
}

static void store_hit(float* hits8, uint32_t i, const bo_hit* h) {
  float* o = hits8 + (size_t)8 * i;
  o[0] = h->u; o[1] = h->v;
  memcpy(&o[2], &h->prim, 4);
  uint32_t inst = BO_EMPTY;
  memcpy(&o[3], &inst, 4);
  o[4] = h->n.x; o[5] = h->n.y; o[6] = h->n.z;
  o[7] = h->t;
}

static bo_hit miss_hit(float tmax) {
  bo_hit h;
  h.t = tmax; h.u = h.v = 0.0f; h.prim = BO_EMPTY; h.n = v3make(0, 0, 0);
  return h;
}

/* Near-first BVH2 closest hit following the two-child loop of
 * bajo/bvh/gpu/trace.mojo:340-428: test both child boxes against the current
 * hit distance, intersect leaf children immediately, continue with the nearer
 * internal child and push the other one if it is still within reach. */
/* st (may be NULL): the five per-ray counters of GpuTraversalStats
 * (bajo/bvh/gpu/trace.mojo:62-90): internal nodes visited, internal children
 * whose box was hit, leaf blocks entered (one triangle each here), triangles
 * tested, deepest stack. */
static bo_hit trace_one(const BoLbvh* bvh, const float* verts, const bo_ray* r, uint32_t seg, int mode,
                        uint32_t* st) {
  bo_hit h = miss_hit(r->tmax);
  uint32_t root = bvh->roots[seg];
  /* prim ids are reported relative to the segment's first item
   * (pack_segmented_triangle_leaf_lanes_kernel, triangle_bvh.mojo:117-120) */
  uint32_t first_item = bvh->seg_offsets ? bvh->seg_offsets[seg] : 0;
  uint32_t nv = 0, nt = 0, nc = 0, ms = 0;
  if (root == BO_SENTINEL) goto done;
  if (root & BO_LEAF_FLAG) {
    uint32_t item = bvh->leaf_ids[root & 0x7FFFFFFFu];
    test_tri(r, verts, item, item - first_item, mode, &h);
    nt++;
    goto done;
  }
  uint32_t stack[128];
  uint32_t sp = 0, cur = root;
  for (;;) {
    nv++;
    const float* b = bvh->node_bounds + (size_t)12 * cur;
    uint32_t c[2] = {bvh->node_meta[4 * (size_t)cur + 1], bvh->node_meta[4 * (size_t)cur + 2]};
    float ct[2];
    int valid[2] = {0, 0};
    /* both child boxes are tested against the same hit distance before any
     * leaf is intersected (_intersect_trace_node_precomputed, trace.mojo:361) */
    int bh[2];
    float tn2[2];
    for (int k = 0; k < 2; ++k) bh[k] = box_hit(r, b + 6 * k, h.t, &tn2[k]);
    for (int k = 0; k < 2; ++k) {
      float tn = tn2[k];
      if (!bh[k]) continue;
      if (c[k] & BO_LEAF_FLAG) {
        uint32_t item = bvh->leaf_ids[c[k] & 0x7FFFFFFFu];
        test_tri(r, verts, item, item - first_item, mode, &h);
        nt++;
      } else {
        valid[k] = 1;
        ct[k] = tn;
        nc++;
      }
    }
    int near = -1;
    if (valid[0]) near = 0;
    if (valid[1] && (near == -1 || ct[1] < ct[0])) near = 1;
    if (near >= 0) {
      int far = 1 - near;
      if (valid[far] && ct[far] <= h.t * BO_SLACK) {
        stack[sp++] = c[far];
        if (sp > ms) ms = sp;
      }
      if (ct[near] <= h.t * BO_SLACK) { cur = c[near]; continue; }
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
done:
  if (st) {
    st[0] = nv;
    st[1] = nc;
    st[2] = nt;
    st[3] = nt;
    st[4] = ms;
  }
  return h;
}

typedef struct {
  const BoLbvh* bvh;
  const float* verts;
  const float* rays;
  uint32_t n;
  int mode;
  float* hits;
  uint32_t n_tris;
} trace_ctx;

static void trace_range(void* p, uint32_t b, uint32_t e) {
  trace_ctx* c = (trace_ctx*)p;
  for (uint32_t i = b; i < e; ++i) {
    bo_ray r = make_ray(c->rays, c->n, i);
    bo_hit h = trace_one(c->bvh, c->verts, &r, 0, c->mode, NULL);
    store_hit(c->hits, i, &h);
  }
}

void bo_trace_bvh2(const BoLbvh* bvh, const float* verts, const float* rays, uint32_t n, int mode,
                   float* hits8, uint32_t n_threads) {
  trace_ctx c = {bvh, verts, rays, n, mode, hits8, 0};
  bo_parallel_for(n, n_threads, 1024, trace_range, &c);
}

void bo_trace_bvh2_stats(const BoLbvh* bvh, const float* verts, const float* rays, uint32_t n, int mode,
                         uint32_t* stats) {
  for (uint32_t i = 0; i < n; ++i) {
    bo_ray r = make_ray(rays, n, i);
    trace_one(bvh, verts, &r, 0, mode, &stats[5 * (size_t)i]);
  }
}

static void brute_range(void* p, uint32_t b, uint32_t e) {
  trace_ctx* c = (trace_ctx*)p;
  for (uint32_t i = b; i < e; ++i) {
    bo_ray r = make_ray(c->rays, c->n, i);
    bo_hit h = miss_hit(r.tmax);
    for (uint32_t t = 0; t < c->n_tris; ++t) test_tri(&r, c->verts, t, t, c->mode, &h);
    store_hit(c->hits, i, &h);
  }
}

void bo_trace_brute(const float* verts, uint32_t n_tris, const float* rays, uint32_t n, int mode,
                    float* hits8, uint32_t n_threads) {
  trace_ctx c = {NULL, verts, rays, n, mode, hits8, n_tris};
  bo_parallel_for(n, n_threads, 64, brute_range, &c);
}

/* ------------------------------------------------------------------------- */
/* two-level trees                                                            */
/* ------------------------------------------------------------------------- */
/* AABB.apply_transform (bajo/core/aabb.mojo:101-139) of each instance's BLAS
 * root box (seg_bounds[12 b .. 12 b + 6)), written as [min, max, min]; an
 * empty box (min > max) stays empty */
void bo_tlas_instance_boxes(const float* seg_bounds, uint32_t n_blas, const float* xf, const uint32_t* blas,
                            uint32_t n, float* out9) {
  for (uint32_t i = 0; i < n; ++i) {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    uint32_t b = blas[i];
    if (b < n_blas) {
      const float* lb = seg_bounds + (size_t)b * 12;
      const float* r = xf + (size_t)i * 12;
      if (lb[0] <= lb[3]) {
        for (int k = 0; k < 3; ++k) mn[k] = mx[k] = r[4 * k + 3];
        for (int col = 0; col < 3; ++col)
          for (int k = 0; k < 3; ++k) {
            float m = r[4 * k + col], a = m * lb[col], c = m * lb[3 + col];
            mn[k] = mn[k] + bo_fminf(a, c);
            mx[k] = mx[k] + bo_fmaxf(a, c);
          }
      }
    }
    float* o = out9 + (size_t)i * 9;
    o[0] = mn[0]; o[1] = mn[1]; o[2] = mn[2];
    o[3] = mx[0]; o[4] = mx[1]; o[5] = mx[2];
    o[6] = mn[0]; o[7] = mn[1]; o[8] = mn[2];
  }
}

typedef struct {
  const BoLbvh* top;
  const BoLbvh* blas;
  const float* blas_verts;
  const float* inv;
  const uint32_t* blas_idx;
  uint32_t n_inst;
  int mode, any;
} tlas_ctx;

typedef struct { bo_hit h; uint32_t inst; int hit; } tl_hit;

/* one instance leaf (tlas.mojo:54-136): the ray in BLAS space (Affine3.ray,
 * transform.mojo:155-211), the BLAS walk with the current hit distance as
 * t_max, a closer hit promoted with its instance */
static int tlas_leaf(const tlas_ctx* c, const bo_ray* r, uint32_t sorted, tl_hit* th) {
  uint32_t inst = c->top->leaf_ids[sorted];
  uint32_t b = c->blas_idx[inst];
  const float* m = c->inv + (size_t)inst * 12;
  v3 o = v3make(fmaf(m[0], r->o.x, fmaf(m[1], r->o.y, fmaf(m[2], r->o.z, m[3]))),
                fmaf(m[4], r->o.x, fmaf(m[5], r->o.y, fmaf(m[6], r->o.z, m[7]))),
                fmaf(m[8], r->o.x, fmaf(m[9], r->o.y, fmaf(m[10], r->o.z, m[11]))));
  v3 d = v3make(fmaf(m[0], r->d.x, fmaf(m[1], r->d.y, m[2] * r->d.z)),
                fmaf(m[4], r->d.x, fmaf(m[5], r->d.y, m[6] * r->d.z)),
                fmaf(m[8], r->d.x, fmaf(m[9], r->d.y, m[10] * r->d.z)));
  bo_ray lr = make_ray_od(o, d, r->tmin, c->any ? r->tmax : th->h.t);
  bo_hit lh = trace_one(c->blas, c->blas_verts, &lr, b, c->mode, NULL);
  if (lh.prim == BO_EMPTY) return 0;
  th->h = lh;
  th->inst = inst;
  th->hit = 1;
  return 1;
}

/* the binary near-first loop of trace_one over the top-level tree */
static tl_hit tlas_one(const tlas_ctx* c, const bo_ray* r) {
  tl_hit th;
  th.h = miss_hit(r->tmax);
  th.inst = BO_EMPTY;
  th.hit = 0;
  const BoLbvh* t = c->top;
  uint32_t root = t->roots[0];
  if (root == BO_SENTINEL) return th;
  if (root & BO_LEAF_FLAG) {
    tlas_leaf(c, r, root & 0x7FFFFFFFu, &th);
    return th;
  }
  uint32_t stack[128];
  uint32_t sp = 0, cur = root;
  for (;;) {
    const float* b = t->node_bounds + (size_t)12 * cur;
    uint32_t ch[2] = {t->node_meta[4 * (size_t)cur + 1], t->node_meta[4 * (size_t)cur + 2]};
    float lim0 = c->any ? r->tmax : th.h.t;
    int bh[2];
    float tn[2];
    for (int k = 0; k < 2; ++k) bh[k] = box_hit(r, b + 6 * k, lim0, &tn[k]);
    int valid[2] = {0, 0};
    for (int k = 0; k < 2; ++k) {
      if (!bh[k]) continue;
      if (ch[k] & BO_LEAF_FLAG) {
        if (tlas_leaf(c, r, ch[k] & 0x7FFFFFFFu, &th) && c->any) return th;
      } else {
        valid[k] = 1;
      }
    }
    int near = -1;
    if (valid[0]) near = 0;
    if (valid[1] && (near == -1 || tn[1] < tn[0])) near = 1;
    if (near >= 0) {
      float lim = (c->any ? r->tmax : th.h.t) * BO_SLACK;
      int far = 1 - near;
      if (valid[far] && tn[far] <= lim) stack[sp++] = ch[far];
      if (tn[near] <= lim) {
        cur = ch[near];
        continue;
      }
    }
    if (sp == 0) break;
    cur = stack[--sp];
  }
  return th;
}

static void tlas_store(const tlas_ctx* c, float* hits8, uint32_t i, const tl_hit* th) {
  float* o = hits8 + (size_t)8 * i;
  memset(o, 0, 8 * sizeof(float));
  uint32_t prim = th->hit ? th->h.prim : BO_EMPTY;
  float t = th->h.t;
  v3 n = v3make(0, 0, 0);
  if (c->any) {
    if (th->hit) {
      t = 0.0f;
      prim = BO_EMPTY;
    }
  } else if (th->hit) {
    o[0] = th->h.u;
    o[1] = th->h.v;
    const float* m = c->inv + (size_t)th->inst * 12;
    v3 ln = th->h.n; /* normalize(cross(e1, e2)) of the BLAS triangle */
    /* normal_from_inverse (transform.mojo:224-257) */
    n = v3normalize(v3make(fmaf(m[0], ln.x, fmaf(m[4], ln.y, m[8] * ln.z)),
                           fmaf(m[1], ln.x, fmaf(m[5], ln.y, m[9] * ln.z)),
                           fmaf(m[2], ln.x, fmaf(m[6], ln.y, m[10] * ln.z))));
  }
  memcpy(&o[2], &prim, 4);
  memcpy(&o[3], &th->inst, 4);
  o[4] = n.x; o[5] = n.y; o[6] = n.z; o[7] = t;
}

void bo_trace_tlas(const BoLbvh* top, const BoLbvh* blas, const float* blas_verts, const float* inv,
                   const uint32_t* blas_idx, uint32_t n_inst, const float* rays, uint32_t n, int any, int mode,
                   float* hits8) {
  tlas_ctx c = {top, blas, blas_verts, inv, blas_idx, n_inst, mode, any};
  for (uint32_t i = 0; i < n; ++i) {
    bo_ray r = make_ray(rays, n, i);
    tl_hit th = tlas_one(&c, &r);
    tlas_store(&c, hits8, i, &th);
  }
}

/* ------------------------------------------------------------------------- */
/* CWBVH8 traversal                                                           */
/* ------------------------------------------------------------------------- */

/* intersect_ray_tri_edges_scaled (bajo/core/intersect.mojo:462-505):
 * determinant-scaled Moller-Trumbore; the candidate passes when
 * |det| > 1e-8, 0 <= u', v', u' + v' <= |det| and t_min|det| < t' < t_max|det| */
static inline int tri_scaled(v3 o, v3 d, v3 v0, v3 e1, v3 e2, float tmax, float tmin, float* ad, float* ts,
                             float* us, float* vs) {
  v3 p = v3cross(d, e2);
  float det = v3dot(e1, p);
  int pos = det >= 0.0f;
  float a = pos ? det : -det;
  v3 tv = v3sub(o, v0);
  float un = v3dot(tv, p);
  v3 q = v3cross(tv, e1);
  float vn = v3dot(d, q), tn = v3dot(e2, q);
  float u = pos ? un : -un, v = pos ? vn : -vn, t = pos ? tn : -tn;
  *ad = a; *ts = t; *us = u; *vs = v;
  return a > 1e-8f && u >= 0.0f && u <= a && v >= 0.0f && (u + v) <= a && t > tmin * a && t < tmax * a;
}

static inline float cw_exp_scale(uint32_t e) {
  uint32_t bits = (e & 0xFFu) << 23;
  float f;
  memcpy(&f, &bits, 4);
  return f;
}

/* trace_cwbvh8_triangles (bajo/bvh/gpu/triangle_bvh.mojo:1010-1104) with the
 * node decode of _intersect_cwbvh8_node_tasks (compressed_bounds_bvh.mojo:
 * 469-576) and the record test of _intersect_cwbvh_triangle
 * (triangle_bvh.mojo:962-1007).  Node groups hold hit internal children in
 * bits 24..31 (slot + 24, slot XOR the inverted ray octant) and the node's
 * imask in bits 0..7; triangle groups hold hit triangles in bits 0..23,
 * relative to the node's triangle base; both are consumed highest bit first.
 * Any-hit returns t = 0 and prim = EMPTY on the first triangle hit.  *err
 * records an out-of-range node or triangle, a revisit beyond n_nodes or a full
 * stack (64 groups); the ray then stops. */
static bo_hit cwbvh8_one(const float* nodes, const float* tris, uint32_t n_nodes, uint32_t n_tris,
                         const bo_ray* r, int any, uint32_t* err) {
  bo_hit h = miss_hit(r->tmax);
  if (n_nodes == 0) return h;
  uint32_t sb[64], sm[64];
  int sp = 0;
  uint32_t sign = (r->d.x < 0.0f ? 4u : 0u) | (r->d.y < 0.0f ? 2u : 0u) | (r->d.z < 0.0f ? 1u : 0u);
  uint32_t oi = 7u - sign;
  uint32_t nbase = 0, nmask = 1u << 31, tbase = 0, tmask = 0, visits = 0;
  for (;;) {
    if (nmask > 0x00FFFFFFu) {
      uint32_t gm = nmask;
      int bit = 31 - __builtin_clz(nmask);
      nmask &= ~(1u << bit);
      if (nmask > 0x00FFFFFFu) {
        if (sp >= 64) { *err |= 2u; break; }
        sb[sp] = nbase;
        sm[sp] = nmask;
        ++sp;
      }
      uint32_t slot = ((uint32_t)bit - 24u) ^ oi;
      uint32_t rel = (uint32_t)__builtin_popcount(gm & ((1u << slot) - 1u));
      uint32_t ni = nbase + rel;
      if (ni >= n_nodes || ++visits > n_nodes) { *err |= 1u; break; }
      const float* nd = nodes + (size_t)ni * 20;
      const uint32_t* w = (const uint32_t*)nd;
      float px = nd[0], py = nd[1], pz = nd[2];
      uint32_t ei = w[3];
      float sx = cw_exp_scale(ei), sy = cw_exp_scale(ei >> 8), sz = cw_exp_scale(ei >> 16);
      uint32_t imask = ei >> 24;
      float tlim = any ? r->tmax : h.t;
      float idx = sx * r->rcp.x, idy = sy * r->rcp.y, idz = sz * r->rcp.z;
      float ox = (px - r->o.x) * r->rcp.x, oy = (py - r->o.y) * r->rcp.y, oz = (pz - r->o.z) * r->rcp.z;
      uint32_t hm = 0;
      for (int j = 0; j < 8; ++j) {
        int g = j >> 2, sh = (j & 3) * 8;
        float qlx = (float)((w[8 + 0 + g] >> sh) & 0xFFu), qly = (float)((w[8 + 2 + g] >> sh) & 0xFFu);
        float qlz = (float)((w[8 + 4 + g] >> sh) & 0xFFu), qhx = (float)((w[8 + 6 + g] >> sh) & 0xFFu);
        float qhy = (float)((w[8 + 8 + g] >> sh) & 0xFFu), qhz = (float)((w[8 + 10 + g] >> sh) & 0xFFu);
        float nx = r->d.x < 0.0f ? qhx : qlx, fx = r->d.x < 0.0f ? qlx : qhx;
        float ny = r->d.y < 0.0f ? qhy : qly, fy = r->d.y < 0.0f ? qly : qhy;
        float nz = r->d.z < 0.0f ? qhz : qlz, fz = r->d.z < 0.0f ? qlz : qhz;
        float tnx = fmaf(nx, idx, ox), tny = fmaf(ny, idy, oy), tnz = fmaf(nz, idz, oz);
        float tfx = fmaf(fx, idx, ox), tfy = fmaf(fy, idy, oy), tfz = fmaf(fz, idz, oz);
        /* fmaxf / fminf: the reference's select-based fmax / fmin
         * (bajo/core/utils.mojo:60-70) give the same comparison unless an
         * operand is NaN */
        float tn = bo_fmaxf(bo_fmaxf(tnx, tny), bo_fmaxf(tnz, 0.0f));
        float tf = bo_fminf(bo_fminf(tfx, tfy), bo_fminf(tfz, tlim));
        uint32_t byte = (w[6 + g] >> sh) & 0xFFu;
        if (byte != 0 && tn <= tf) {
          uint32_t bi = byte & 0x1Fu;
          if (imask >> j & 1u) bi ^= oi;
          hm |= (byte >> 5) << bi;
        }
      }
      nbase = w[4];
      nmask = (hm & 0xFF000000u) | imask;
      tbase = w[5];
      tmask = hm & 0x00FFFFFFu;
    } else {
      tbase = nbase;
      tmask = nmask;
      nmask = 0;
    }
    while (tmask != 0) {
      int bit = 31 - __builtin_clz(tmask);
      tmask &= ~(1u << bit);
      uint32_t ti = tbase + (uint32_t)bit;
      if (ti >= n_tris) { *err |= 1u; return h; }
      const float* tr = tris + (size_t)ti * 12;
      v3 e1 = load3(tr), e2 = load3(tr + 4), v0 = load3(tr + 8);
      float ad, ts, us, vs;
      if (!tri_scaled(r->o, r->d, v0, e1, e2, h.t, r->tmin, &ad, &ts, &us, &vs)) continue;
      if (any) {
        h = miss_hit(0.0f);
        return h;
      }
      float inv = 1.0f / ad;
      h.t = ts * inv;
      h.u = us * inv;
      h.v = vs * inv;
      memcpy(&h.prim, &tr[11], 4);
      h.n = v3normalize(v3cross(e1, e2));
    }
    if (nmask <= 0x00FFFFFFu) {
      if (sp == 0) break;
      --sp;
      nbase = sb[sp];
      nmask = sm[sp];
    }
  }
  return h;
}

typedef struct {
  const float* nodes;
  const float* tris;
  uint32_t n_nodes, n_tris;
  const float* rays;
  uint32_t n;
  int any;
  float* hits;
  uint32_t* err;
} cw_ctx;

static void cw_range(void* p, uint32_t b, uint32_t e) {
  cw_ctx* c = (cw_ctx*)p;
  for (uint32_t i = b; i < e; ++i) {
    bo_ray r = make_ray(c->rays, c->n, i);
    uint32_t err = 0;
    bo_hit h = cwbvh8_one(c->nodes, c->tris, c->n_nodes, c->n_tris, &r, c->any, &err);
    store_hit(c->hits, i, &h);
    if (c->err) c->err[i] = err;
  }
}

void bo_trace_cwbvh8(const float* nodes, uint32_t n_nodes, const float* tris, uint32_t n_tris, const float* rays,
                     uint32_t n, int any_hit, float* hits8, uint32_t* err, uint32_t n_threads) {
  cw_ctx c = {nodes, tris, n_nodes, n_tris, rays, n, any_hit, hits8, err};
  bo_parallel_for(n, n_threads, 1024, cw_range, &c);
}

/* ------------------------------------------------------------------------- */
/* reference CPU builder (timed CPU baseline)                                 */
/* ------------------------------------------------------------------------- */
typedef struct { uint32_t code, item; } bo_mitem;

typedef struct {
  const float* verts;
  uint32_t n;
  float* bounds6;
  float cmin[3], inv[3];
  bo_mitem* pairs;
  /* radix */
  bo_mitem* src;
  bo_mitem* dst;
  int shift;
  uint32_t workers;
  uint32_t* counts;  /* workers x 256 */
  uint32_t* offsets; /* workers x 256 */
} cpu_build_ctx;

static void cb_bounds(void* p, uint32_t b, uint32_t e) {
  cpu_build_ctx* c = (cpu_build_ctx*)p;
  bo_triangle_bounds(c->verts + (size_t)9 * b, e - b, c->bounds6 + (size_t)6 * b);
}

/* bajo/bvh/cpu/builder/lbvh.mojo:190-199 morton_worker */
static void cb_morton(void* p, uint32_t b, uint32_t e) {
  cpu_build_ctx* c = (cpu_build_ctx*)p;
  for (uint32_t i = b; i < e; ++i) {
    const float* bb = c->bounds6 + (size_t)6 * i;
    float cx = (bb[0] + bb[3]) * 0.5f, cy = (bb[1] + bb[4]) * 0.5f, cz = (bb[2] + bb[5]) * 0.5f;
    c->pairs[i].code = bo_morton3((cx - c->cmin[0]) * c->inv[0], (cy - c->cmin[1]) * c->inv[1],
                                  (cz - c->cmin[2]) * c->inv[2]);
    c->pairs[i].item = i;
  }
}

/* bajo/bvh/cpu/builder/lbvh.mojo:65-112: per-worker histograms over
 * contiguous chunks, offsets assigned bucket-major then worker-major (stable). */
static void cb_hist(void* p, uint32_t b, uint32_t e) {
  cpu_build_ctx* c = (cpu_build_ctx*)p;
  for (uint32_t w = b; w < e; ++w) {
    uint32_t* cnt = c->counts + 256 * (size_t)w;
    memset(cnt, 0, 256 * sizeof(uint32_t));
    uint32_t first = (uint32_t)((uint64_t)c->n * w / c->workers), end = (uint32_t)((uint64_t)c->n * (w + 1) / c->workers);
    for (uint32_t i = first; i < end; ++i) cnt[(c->src[i].code >> c->shift) & 0xFF]++;
  }
}
static void cb_scatter(void* p, uint32_t b, uint32_t e) {
  cpu_build_ctx* c = (cpu_build_ctx*)p;
  for (uint32_t w = b; w < e; ++w) {
    uint32_t off[256];
    memcpy(off, c->offsets + 256 * (size_t)w, sizeof off);
    uint32_t first = (uint32_t)((uint64_t)c->n * w / c->workers), end = (uint32_t)((uint64_t)c->n * (w + 1) / c->workers);
    for (uint32_t i = first; i < end; ++i) c->dst[off[(c->src[i].code >> c->shift) & 0xFF]++] = c->src[i];
  }
}

typedef struct {
  const bo_mitem* pairs;
  int64_t len;
  BoCpuNode* nodes;
  uint32_t* item_indices;
  const float* bounds6;
  uint32_t next; /* next free node id (frontier collection, then task bases) */
} cpu_tree_ctx;

static int cp_pairs(const bo_mitem* p, int64_t len, int64_t i, int64_t j) {
  if (j < 0 || j >= len) return -1;
  return bo_morton_common_prefix(p[i].code, (uint32_t)i, p[j].code, (uint32_t)j);
}
/* bajo/bvh/cpu/builder/lbvh.mojo:144-163 */
static int64_t split_pairs(const bo_mitem* p, int64_t len, int64_t first, int64_t last) {
  int np = cp_pairs(p, len, first, last);
  int64_t split = first, step = last - first;
  while (step > 1) {
    step = (step + 1) >> 1;
    int64_t ns = split + step;
    if (ns < last && cp_pairs(p, len, first, ns) > np) split = ns;
  }
  return split;
}

static void node_set_box(BoCpuNode* nd, const float* mn, const float* mx) {
  for (int k = 0; k < 3; ++k) { nd->bmin[k] = mn[k]; nd->bmax[k] = mx[k]; }
}

/* bajo/bvh/cpu/builder/lbvh.mojo:252-267 (leaf, leaf_size 1) and 401-437 */
/* Node ids: the reference takes each child pair from one shared atomic
 * counter (lbvh.mojo:414).  A frontier task over c leaves allocates exactly
 * 2 (c - 1) nodes, so each task here draws from its own contiguous range
 * (`next`), assigned in task order: the layout the shared counter produces
 * when the tasks run one after another, without its cache-line traffic. */
static void cpu_build_rec(cpu_tree_ctx* c, uint32_t node, int64_t first, int64_t count, uint32_t* next) {
  BoCpuNode* nd = &c->nodes[node];
  if (count <= 1) {
    const float* b = c->bounds6 + (size_t)6 * c->item_indices[first];
    node_set_box(nd, b, b + 3);
    nd->left_or_first = (uint32_t)first;
    nd->count = (uint32_t)count;
    return;
  }
  int64_t last = first + count - 1;
  int64_t split = split_pairs(c->pairs, c->len, first, last);
  int64_t lc = split - first + 1;
  uint32_t left = *next;
  *next += 2u;
  cpu_build_rec(c, left, first, lc, next);
  cpu_build_rec(c, left + 1, split + 1, count - lc, next);
  BoCpuNode* L = &c->nodes[left];
  BoCpuNode* R = &c->nodes[left + 1];
  float mn[3], mx[3];
  for (int k = 0; k < 3; ++k) { mn[k] = bo_fminf(L->bmin[k], R->bmin[k]); mx[k] = bo_fmaxf(L->bmax[k], R->bmax[k]); }
  node_set_box(nd, mn, mx);
  nd->left_or_first = left;
  nd->count = 0;
}

typedef struct { uint32_t node; int64_t first, count; uint32_t base; } frontier_task;
typedef struct { cpu_tree_ctx* t; frontier_task* tasks; } frontier_ctx;

static void cpu_collect(cpu_tree_ctx* c, uint32_t node, int64_t first, int64_t count, int depth,
                        frontier_task* out, uint32_t* n_out) {
  if (count <= 1 || depth == 0) {
    out[(*n_out)++] = (frontier_task){node, first, count, 0};
    return;
  }
  int64_t last = first + count - 1;
  int64_t split = split_pairs(c->pairs, c->len, first, last);
  int64_t lc = split - first + 1;
  uint32_t left = c->next;
  c->next += 2;
  c->nodes[node].left_or_first = left;
  c->nodes[node].count = 0;
  cpu_collect(c, left, first, lc, depth - 1, out, n_out);
  cpu_collect(c, left + 1, split + 1, count - lc, depth - 1, out, n_out);
}

static void frontier_worker(void* p, uint32_t b, uint32_t e) {
  frontier_ctx* f = (frontier_ctx*)p;
  for (uint32_t k = b; k < e; ++k) {
    frontier_task t = f->tasks[k];
    for (int64_t i = t.first; i < t.first + t.count; ++i) f->t->item_indices[i] = f->t->pairs[i].item;
    uint32_t next = t.base;
    cpu_build_rec(f->t, t.node, t.first, t.count, &next);
  }
}

static void refit_frontier(BoCpuNode* nodes, uint32_t node, int depth) {
  BoCpuNode* nd = &nodes[node];
  if (depth == 0 || nd->count != 0) return;
  uint32_t l = nd->left_or_first;
  refit_frontier(nodes, l, depth - 1);
  refit_frontier(nodes, l + 1, depth - 1);
  for (int k = 0; k < 3; ++k) {
    nd->bmin[k] = bo_fminf(nodes[l].bmin[k], nodes[l + 1].bmin[k]);
    nd->bmax[k] = bo_fmaxf(nodes[l].bmax[k], nodes[l + 1].bmax[k]);
  }
}

/* Scratch of one build: leaf bounds, Morton pairs and their sort buffer, and
 * the per-worker radix histograms and offsets (256 each). */
static size_t cpu_scratch_layout(uint32_t n, uint32_t workers, size_t* off_pairs, size_t* off_scratch,
                                 size_t* off_counts, size_t* off_offsets) {
  size_t o = ((sizeof(float) * 6 * (size_t)n) + 63) & ~(size_t)63;
  *off_pairs = o;
  o += (sizeof(bo_mitem) * (size_t)n + 63) & ~(size_t)63;
  *off_scratch = o;
  o += (sizeof(bo_mitem) * (size_t)n + 63) & ~(size_t)63;
  *off_counts = o;
  o += sizeof(uint32_t) * 256 * (size_t)workers;
  *off_offsets = o;
  o += sizeof(uint32_t) * 256 * (size_t)workers;
  return o;
}

size_t bo_cpu_lbvh_scratch_bytes(uint32_t n, uint32_t n_threads) {
  size_t a, b, c, d;
  if (n_threads == 0) n_threads = 1;
  return cpu_scratch_layout(n, n_threads < n ? n_threads : (n ? n : 1), &a, &b, &c, &d);
}

/* bajo/bvh/cpu/builder/lbvh.mojo:166-216 + 318-359 */
uint32_t bo_cpu_build_lbvh_scratch(const float* verts, uint32_t n, uint32_t n_threads, BoCpuNode* nodes,
                                   uint32_t* item_indices, void* scratch) {
  if (n == 0) return 0;
  if (n_threads == 0) n_threads = 1;
  uint32_t workers = n_threads < n ? n_threads : n;
  size_t off_pairs, off_scratch, off_counts, off_offsets;
  cpu_scratch_layout(n, workers, &off_pairs, &off_scratch, &off_counts, &off_offsets);
  unsigned char* sb = (unsigned char*)scratch;
  cpu_build_ctx c;
  memset(&c, 0, sizeof c);
  c.verts = verts;
  c.n = n;
  c.bounds6 = (float*)sb;
  bo_parallel_for(n, n_threads, 8192, cb_bounds, &c);
  /* centroid bounds grown serially over the items, as
   * update_node_bounds_and_centroid_bounds does (builder.mojo:133-147) */
  float cmn[3] = {BO_FLT_MAX, BO_FLT_MAX, BO_FLT_MAX}, cmx[3] = {-BO_FLT_MAX, -BO_FLT_MAX, -BO_FLT_MAX};
  for (uint32_t i = 0; i < n; ++i) {
    const float* b = c.bounds6 + (size_t)6 * i;
    for (int k = 0; k < 3; ++k) {
      float cc = (b[k] + b[3 + k]) * 0.5f;
      cmn[k] = bo_fminf(cmn[k], cc);
      cmx[k] = bo_fmaxf(cmx[k], cc);
    }
  }
  for (int k = 0; k < 3; ++k) { c.cmin[k] = cmn[k]; c.inv[k] = safe_inv1(cmx[k] - cmn[k]); }
  bo_mitem* pairs = (bo_mitem*)(sb + off_pairs);
  bo_mitem* scratch_pairs = (bo_mitem*)(sb + off_scratch);
  c.pairs = pairs;
  bo_parallel_for(n, n_threads, 8192, cb_morton, &c);
  /* stable LSD radix over the 32-bit code, workers over contiguous chunks */
  c.workers = workers;
  c.counts = (uint32_t*)(sb + off_counts);
  c.offsets = (uint32_t*)(sb + off_offsets);
  bo_mitem* src = pairs;
  bo_mitem* dst = scratch_pairs;
  for (int sh = 0; sh < 32; sh += 8) {
    c.src = src;
    c.dst = dst;
    c.shift = sh;
    bo_parallel_for(workers, workers, 1, cb_hist, &c);
    uint32_t acc = 0;
    for (int b = 0; b < 256; ++b)
      for (uint32_t w = 0; w < workers; ++w) { c.offsets[256 * w + b] = acc; acc += c.counts[256 * w + b]; }
    bo_parallel_for(workers, workers, 1, cb_scatter, &c);
    bo_mitem* t = src; src = dst; dst = t;
  }
  /* four passes: the sorted pairs are back in `pairs` */
  cpu_tree_ctx t;
  t.pairs = pairs;
  t.len = n;
  t.nodes = nodes;
  t.item_indices = item_indices;
  t.bounds6 = c.bounds6;
  t.next = 1;
  frontier_task tasks[16];
  uint32_t nt = 0;
  cpu_collect(&t, 0, 0, n, 3, tasks, &nt);
  for (uint32_t k = 0; k < nt; ++k) {
    tasks[k].base = t.next;
    t.next += tasks[k].count > 1 ? 2u * (uint32_t)(tasks[k].count - 1) : 0u;
  }
  frontier_ctx f = {&t, tasks};
  bo_parallel_for(nt, n_threads, 1, frontier_worker, &f);
  refit_frontier(nodes, 0, 3);
  return t.next;
}

uint32_t bo_cpu_build_lbvh(const float* verts, uint32_t n, uint32_t n_threads, BoCpuNode* nodes,
                           uint32_t* item_indices) {
  if (n == 0) return 0;
  void* scratch = malloc(bo_cpu_lbvh_scratch_bytes(n, n_threads));
  if (!scratch) return 0;
  uint32_t used = bo_cpu_build_lbvh_scratch(verts, n, n_threads, nodes, item_indices, scratch);
  free(scratch);
  return used;
}

typedef struct {
  const BoCpuNode* nodes;
  const uint32_t* items;
  const float* verts;
  const float* rays;
  uint32_t n;
  int mode;
  float* hits;
} cpu_trace_ctx;

static void cpu_trace_range(void* p, uint32_t b, uint32_t e) {
  cpu_trace_ctx* c = (cpu_trace_ctx*)p;
  for (uint32_t i = b; i < e; ++i) {
    bo_ray r = make_ray(c->rays, c->n, i);
    bo_hit h = miss_hit(r.tmax);
    uint32_t stack[128], sp = 0;
    uint32_t cur = 0;
    float tn0;
    float rb[6];
    const BoCpuNode* root = &c->nodes[0];
    for (int k = 0; k < 3; ++k) { rb[k] = root->bmin[k]; rb[3 + k] = root->bmax[k]; }
    if (box_hit(&r, rb, h.t, &tn0)) {
      for (;;) {
        const BoCpuNode* nd = &c->nodes[cur];
        if (nd->count) {
          for (uint32_t k = 0; k < nd->count; ++k) {
            uint32_t item = c->items[nd->left_or_first + k];
            test_tri(&r, c->verts, item, item, c->mode, &h);
          }
        } else {
          uint32_t l = nd->left_or_first;
          float tl, tr;
          float bl[6], br[6];
          for (int k = 0; k < 3; ++k) {
            bl[k] = c->nodes[l].bmin[k]; bl[3 + k] = c->nodes[l].bmax[k];
            br[k] = c->nodes[l + 1].bmin[k]; br[3 + k] = c->nodes[l + 1].bmax[k];
          }
          int hl = box_hit(&r, bl, h.t, &tl), hr = box_hit(&r, br, h.t, &tr);
          if (hl && hr) {
            uint32_t nearc = tl <= tr ? l : l + 1, farc = tl <= tr ? l + 1 : l;
            stack[sp++] = farc;
            cur = nearc;
            continue;
          }
          if (hl) { cur = l; continue; }
          if (hr) { cur = l + 1; continue; }
        }
        if (!sp) break;
        cur = stack[--sp];
      }
    }
    store_hit(c->hits, i, &h);
  }
}

void bo_cpu_trace(const BoCpuNode* nodes, const uint32_t* items, const float* verts, const float* rays,
                  uint32_t n, int mode, float* hits8, uint32_t n_threads) {
  cpu_trace_ctx c = {nodes, items, verts, rays, n, mode, hits8};
  bo_parallel_for(n, n_threads, 1024, cpu_trace_range, &c);
}

/* ========================================================================= */
/* Wavefront path tracer (PATH / NEE / MIS), restated per path               */
/* ========================================================================= */
/* The GPU renderer runs one kernel per bounce over queues; every path is
 * independent and owns its random streams, so a per-path loop that adds the
 * same contributions in the same order (bounce b: the hit's emission or sky,
 * then the shadow ray's light) produces the same per-sample radiance.
 * References: bajo/rt/gpu/common_kernels.mojo:22-136 (primary, resolve),
 * bajo/rt/gpu/scene_trace.mojo:41-369,586 (trace, shadow),
 * bajo/rt/gpu/path_shading.mojo:261-590 (NEE, MIS emission, Lambertian),
 * bajo/rt/shading.mojo:92-118, bajo/rt/common.mojo:12-67,
 * bajo/rt/lighting.mojo:7-39, bajo/rt/wavefront_contract.mojo:107-133. */

/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11); counter
 * (0, 0, stage, path_id), key = seed: the first block of the stream owned by
 * the (path, stage) pair.  24-bit uniforms in [0, 1). */
void bo_rt_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void bo_rt_uniform4(uint64_t seed, uint32_t path_id, uint32_t stage, float out[4]) {
  const uint32_t ctr[4] = {0u, 0u, stage, path_id};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t x[4];
  bo_rt_philox4x32_10(ctr, key, x);
  uint32_t c0 = x[0], c1 = x[1], c2 = x[2], c3 = x[3];
  const float s = 1.0f / 16777216.0f;
  out[0] = (float)(c0 >> 8) * s; out[1] = (float)(c1 >> 8) * s;
  out[2] = (float)(c2 >> 8) * s; out[3] = (float)(c3 >> 8) * s;
}

/* sin / cos of 2*pi*u: nearest quarter turn, Taylor series on |a| <= pi/4. */
void bo_rt_sincos_turns(float u, float* s_out, float* c_out) {
  const float qf = floorf(u * 4.0f + 0.5f);
  const int q = (int)qf & 3;
  const float r = u - qf * 0.25f;
  const float a = r * 6.28318530717958647692f;
  const float a2 = a * a;
  float s = fmaf(a2, 1.0f / 362880.0f, -1.0f / 5040.0f);
  s = fmaf(a2, s, 1.0f / 120.0f);
  s = fmaf(a2, s, -1.0f / 6.0f);
  s = fmaf(a2, s, 1.0f);
  s = a * s;
  float c = fmaf(a2, -1.0f / 3628800.0f, 1.0f / 40320.0f);
  c = fmaf(a2, c, -1.0f / 720.0f);
  c = fmaf(a2, c, 1.0f / 24.0f);
  c = fmaf(a2, c, -0.5f);
  c = fmaf(a2, c, 1.0f);
  if (q == 0) { *s_out = s; *c_out = c; }
  else if (q == 1) { *s_out = c; *c_out = -s; }
  else if (q == 2) { *s_out = -s; *c_out = -c; }
  else { *s_out = -c; *c_out = s; }
}

#define BO_MAT_LAMBERTIAN 0u
#define BO_MAT_METAL 1u
#define BO_MAT_DIELECTRIC 2u
#define BO_MAT_EMISSIVE 3u
#define BO_LIGHT_STRIDE 16
static const float BO_INV_PI = 0.3183098861837907f;

static inline v3 vmul(v3 a, v3 b) { return v3make(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vneg(v3 a) { return v3make(-a.x, -a.y, -a.z); }
static inline v3 vdivs(v3 a, float s) { return v3make(a.x / s, a.y / s, a.z / s); }
static inline float power_heuristic(float a, float b) {
  float a2 = a * a, b2 = b * b, den = a2 + b2;
  return den > 0.0f ? a2 / den : 0.0f;
}

/* series_log2 / series_exp2 / series_pow: the CUDA sampling.cuh functions,
 * operation for operation (atanh series of log2 on [sqrt(1/2), sqrt(2)),
 * Taylor series of 2^f on |f| <= 1/2) */
static float series_log2(float x) {
  uint32_t bits;
  memcpy(&bits, &x, 4);
  int e = (int)((bits >> 23) & 0xFFu) - 127;
  uint32_t mb = (bits & 0x007FFFFFu) | 0x3F800000u;
  float m;
  memcpy(&m, &mb, 4);
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float poly = 1.0f + s2 * (0.333333333f + s2 * (0.2f + s2 * (0.142857143f + s2 * 0.111111111f)));
  return (float)e + ((2.0f * s) * poly) * 1.44269504f;
}

static float series_exp2(float z) {
  if (z < -126.0f) return 0.0f;
  if (z > 127.0f) z = 127.0f;
  float k = rintf(z);
  float y = (z - k) * 0.693147181f;
  float p = 1.0f + y * (1.0f + y * (0.5f + y * (0.166666667f + y * (0.0416666667f + y * (0.00833333333f +
                                                                     y * (0.00138888889f + y * 0.000198412698f))))));
  uint32_t sb = (uint32_t)((int)k + 127) << 23;
  float sc;
  memcpy(&sc, &sb, 4);
  return p * sc;
}

static float series_pow(float x, float y) {
  if (y == 0.0f) return 1.0f;
  if (!(x >= 1.17549435e-38f)) return 0.0f;
  return series_exp2(y * series_log2(x));
}

float bo_rt_series_pow(float x, float y) { return series_pow(x, y); }

static v3 v3reflect(v3 v, v3 n) {
  float k = 2.0f * v3dot(v, n);
  return v3make(v.x - k * n.x, v.y - k * n.y, v.z - k * n.z);
}

typedef struct { v3 dir, weight; float pdf; int delta, ok; } bo_bsdf;

/* _sample_metal / _evaluate_metal (bajo/rt/shading.mojo:29-56,122-161) */
static bo_bsdf sample_metal(v3 d, v3 normal, v3 albedo, float fuzz, float u, float v) {
  bo_bsdf r;
  v3 reflected = v3normalize(v3reflect(v3normalize(d), normal));
  int smooth = fuzz <= 1.0e-4f;
  r.delta = smooth;
  if (smooth) {
    r.dir = reflected;
    r.weight = albedo;
    r.pdf = 1.0f;
    r.ok = v3dot(reflected, normal) > 0.0f;
    return r;
  }
  float exponent = bo_fmaxf(2.0f / (fuzz * fuzz) - 2.0f, 0.0f);
  float cos_t = series_pow(u, 1.0f / (exponent + 1.0f));
  float sin_t = sqrtf(bo_fmaxf(1.0f - cos_t * cos_t, 0.0f));
  float sp, cp;
  bo_rt_sincos_turns(v, &sp, &cp);
  v3 helper = fabsf(reflected.y) > 0.99f ? v3make(1.0f, 0.0f, 0.0f) : v3make(0.0f, 1.0f, 0.0f);
  v3 tangent = v3normalize(v3cross(helper, reflected));
  v3 bitangent = v3cross(reflected, tangent);
  v3 dir = v3normalize(v3add(v3add(v3muls(tangent, cp * sin_t), v3muls(bitangent, sp * sin_t)),
                             v3muls(reflected, cos_t)));
  v3 dn = v3normalize(dir);
  int surface_valid = v3dot(normal, dn) > 0.0f;
  float lobe_cos = bo_fmaxf(v3dot(reflected, dn), 0.0f);
  float lobe = series_pow(lobe_cos, exponent);
  int valid = surface_valid && lobe_cos > 0.0f;
  float value_scale = valid ? ((exponent + 2.0f) * lobe) / 6.28318531f : 0.0f;
  float pdf = valid ? ((exponent + 1.0f) * lobe) / 6.28318531f : 0.0f;
  float scos = bo_fmaxf(v3dot(normal, dir), 0.0f);
  r.ok = pdf > 0.0f && scos > 0.0f;
  float scale = scos / (r.ok ? pdf : 1.0f);
  r.dir = dir;
  r.weight = v3muls(v3muls(albedo, value_scale), scale);
  r.pdf = pdf;
  return r;
}

/* _sample_dielectric (bajo/rt/shading.mojo:165-198), refract and the
 * Schlick reflectance (:235-258) */
static bo_bsdf sample_dielectric(v3 d, v3 normal, float ior, int front, float u) {
  bo_bsdf r;
  float ri = front ? 1.0f / ior : ior;
  v3 ud = v3normalize(d);
  float cos_t = bo_fminf(v3dot(vneg(ud), normal), 1.0f);
  float sin_t = sqrtf(bo_fmaxf(1.0f - cos_t * cos_t, 0.0f));
  int cannot = ri * sin_t > 1.0f;
  float root = (1.0f - ri) / (1.0f + ri);
  float r2 = root * root;
  float x = 1.0f - cos_t;
  float x2 = x * x;
  float x5 = (x2 * x2) * x;
  float refl = fmaf(1.0f - r2, x5, r2);
  int rs = cannot || refl > u;
  v3 out;
  if (rs) {
    out = v3reflect(ud, normal);
  } else {
    float ct = bo_fminf(v3dot(vneg(ud), normal), 1.0f);
    v3 perp = v3make(ri * (ud.x + ct * normal.x), ri * (ud.y + ct * normal.y), ri * (ud.z + ct * normal.z));
    float par = -sqrtf(fabsf(1.0f - v3dot(perp, perp)));
    out = v3make(perp.x + par * normal.x, perp.y + par * normal.y, perp.z + par * normal.z);
  }
  r.dir = v3normalize(out);
  r.weight = v3make(1.0f, 1.0f, 1.0f);
  r.pdf = rs ? (cannot ? 1.0f : refl) : 1.0f - refl;
  r.delta = 1;
  r.ok = 1;
  return r;
}

/* LightStore (bajo/rt/types.mojo:190-247, 490-525) */
int bo_rt_build_lights(const float* v, const uint32_t* surf, uint32_t n, const float* em, float* out,
                       uint32_t max_lights, uint32_t* n_lights, float* total_weight) {
  uint32_t* tri = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  float* w = (float*)malloc(sizeof(float) * (n ? n : 1));
  uint32_t count = 0;
  float total = 0.0f;
  for (uint32_t i = 0; i < n; ++i) {
    if ((surf[i] >> 28) != BO_MAT_EMISSIVE) continue;
    const float* p = v + (size_t)9 * i;
    v3 v0 = load3(p), e1 = v3sub(load3(p + 3), v0), e2 = v3sub(load3(p + 6), v0);
    v3 c = v3cross(e1, e2);
    float area = 0.5f * sqrtf(v3dot(c, c));
    const float* L = em + 3 * (size_t)(surf[i] & 0x0FFFFFFFu);
    float imp = bo_fmaxf(((L[0] + L[1]) + L[2]) / 3.0f, 0.0f);
    float wt = area * imp;
    if (wt > 0.0f) {
      total += wt;
      tri[count] = i;
      w[count] = wt;
      ++count;
    }
  }
  if (count > max_lights) { free(tri); free(w); return 1; }
  float* prob = (float*)malloc(sizeof(float) * (count ? count : 1));
  float* scaled = (float*)malloc(sizeof(float) * (count ? count : 1));
  uint32_t* alias = (uint32_t*)malloc(sizeof(uint32_t) * (count ? count : 1));
  uint32_t* small = (uint32_t*)malloc(sizeof(uint32_t) * (count ? count : 1));
  uint32_t* large = (uint32_t*)malloc(sizeof(uint32_t) * (count ? count : 1));
  uint32_t ns = 0, nl = 0;
  for (uint32_t i = 0; i < count; ++i) { prob[i] = 1.0f; alias[i] = 0; }
  if (count > 0 && total > 0.0f) {
    for (uint32_t i = 0; i < count; ++i) {
      alias[i] = i;
      scaled[i] = w[i] * (float)count / total;
      if (scaled[i] < 1.0f) small[ns++] = i; else large[nl++] = i;
    }
    while (ns > 0 && nl > 0) {
      uint32_t si = small[--ns], li = large[--nl];
      prob[si] = scaled[si];
      alias[si] = li;
      scaled[li] = scaled[li] + scaled[si] - 1.0f;
      if (scaled[li] < 1.0f) small[ns++] = li; else large[nl++] = li;
    }
    while (ns > 0) { uint32_t i = small[--ns]; prob[i] = 1.0f; alias[i] = i; }
    while (nl > 0) { uint32_t i = large[--nl]; prob[i] = 1.0f; alias[i] = i; }
  }
  for (uint32_t k = 0; k < count; ++k) {
    float* r = out + (size_t)k * BO_LIGHT_STRIDE;
    memcpy(r, v + (size_t)9 * tri[k], 9 * sizeof(float));
    const float* L = em + 3 * (size_t)(surf[tri[k]] & 0x0FFFFFFFu);
    r[9] = L[0]; r[10] = L[1]; r[11] = L[2];
    r[12] = prob[k];
    memcpy(&r[13], &alias[k], 4);
    r[14] = 0.0f; r[15] = 0.0f;
  }
  *n_lights = count;
  *total_weight = total;
  free(tri); free(w); free(prob); free(scaled); free(alias); free(small); free(large);
  return 0;
}

/* any hit on (tmin, tmax): boxes culled against the ray's t_max */
static int any_hit(const BoLbvh* bvh, const float* verts, const bo_ray* r) {
  bo_hit h = miss_hit(r->tmax);
  uint32_t root = bvh->roots[0];
  if (root == BO_SENTINEL) return 0;
  if (root & BO_LEAF_FLAG) {
    uint32_t item = bvh->leaf_ids[root & 0x7FFFFFFFu];
    test_tri(r, verts, item, item, BO_TRI_WATERTIGHT, &h);
    return h.prim != BO_EMPTY;
  }
  uint32_t stack[128], sp = 0, cur = root;
  for (;;) {
    const float* b = bvh->node_bounds + (size_t)12 * cur;
    uint32_t c[2] = {bvh->node_meta[4 * (size_t)cur + 1], bvh->node_meta[4 * (size_t)cur + 2]};
    for (int k = 0; k < 2; ++k) {
      float tn;
      if (!box_hit(r, b + 6 * k, r->tmax, &tn)) continue;
      if (c[k] & BO_LEAF_FLAG) {
        uint32_t item = bvh->leaf_ids[c[k] & 0x7FFFFFFFu];
        test_tri(r, verts, item, item, BO_TRI_WATERTIGHT, &h);
        if (h.prim != BO_EMPTY) return 1;
      } else {
        stack[sp++] = c[k];
      }
    }
    if (sp == 0) return 0;
    cur = stack[--sp];
  }
}

typedef struct {
  const BoLbvh* bvh;
  const float* verts;
  const uint32_t* surfaces;
  const float* lambertians;
  const float* emissives;
  const float* lights;
  uint32_t n_lights;
  float total_weight;
  const float* metals;      /* 4 per metal (may be NULL) */
  const float* dielectrics; /* 1 per dielectric (may be NULL) */
  const float* cam;
  uint32_t width, height, spp, max_depth;
  uint64_t seed;
  int algorithm;
  float* sample_radiance; /* 3 per path, path_id order */
  /* compressed 8-wide tree (NULL: trace bvh): bajo/rt/gpu/prepared_scene.mojo:29-33 */
  const float* cw_nodes;
  const float* cw_tris;
  uint32_t cw_n_nodes, cw_n_tris;
} rt_ctx;

/* closest hit / occlusion of one path ray through the scene's tree: the
 * binary LBVH (watertight, ties to the lowest id) or the CWBVH8 walk of
 * trace_cwbvh8_triangles (its own visiting order and tie rule) */
static bo_hit rt_closest(const rt_ctx* c, const bo_ray* r) {
  if (c->cw_nodes) {
    uint32_t err = 0;
    return cwbvh8_one(c->cw_nodes, c->cw_tris, c->cw_n_nodes, c->cw_n_tris, r, 0, &err);
  }
  return trace_one(c->bvh, c->verts, r, 0, BO_TRI_WATERTIGHT, NULL);
}
static int rt_occluded(const rt_ctx* c, const bo_ray* r) {
  if (c->cw_nodes) {
    uint32_t err = 0;
    return cwbvh8_one(c->cw_nodes, c->cw_tris, c->cw_n_nodes, c->cw_n_tris, r, 1, &err).t == 0.0f;
  }
  return any_hit(c->bvh, c->verts, r);
}

static inline uint32_t st_bsdf(uint32_t b) { return (0u << 30) | (b + 1); }
static inline uint32_t st_roulette(uint32_t b) { return (1u << 30) | (b + 1); }
static inline uint32_t st_light(uint32_t b) { return (2u << 30) | (b + 1); }

static void rt_path(const rt_ctx* c, uint32_t path_id, float out[3]) {
  const float* cam = c->cam;
  float r[4];
  bo_rt_uniform4(c->seed, path_id, 0, r);
  uint32_t pixel = path_id / c->spp;
  uint32_t px = pixel % c->width, py = pixel / c->width;
  float st, ct;
  bo_rt_sincos_turns(r[0], &st, &ct);
  float lr = sqrtf(r[1]);
  float lens_u = lr * ct, lens_v = lr * st;
  float w = (float)c->width, h = (float)c->height;
  float aspect = w / h;
  float sx = (((float)px + r[2]) / w) * 2.0f - 1.0f;
  float sy = 1.0f - (((float)py + r[3]) / h) * 2.0f;
  v3 origin = load3(cam), fwd = load3(cam + 3), right = load3(cam + 6), up = load3(cam + 9);
  float fs = cam[12], focus = cam[13];
  v3 du = load3(cam + 14), dv = load3(cam + 17);
  v3 inner = v3add(v3add(fwd, v3muls(right, (sx * aspect) * fs)), v3muls(up, sy * fs));
  v3 focal = v3add(origin, v3make(focus * inner.x, focus * inner.y, focus * inner.z));
  v3 ro = v3add(v3add(origin, v3make(lens_u * du.x, lens_u * du.y, lens_u * du.z)),
                v3make(lens_v * dv.x, lens_v * dv.y, lens_v * dv.z));
  v3 o = ro, d = v3normalize(v3sub(focal, ro));
  float tmin = 0.001f, tmax = BO_FLT_MAX;
  v3 T = v3make(1.0f, 1.0f, 1.0f);
  float prev_pdf = 0.0f;
  int delta = 1;
  float rad[3] = {0.0f, 0.0f, 0.0f};
  for (uint32_t b = 0; b < c->max_depth; ++b) {
    bo_ray ray = make_ray_od(o, d, tmin, tmax);
    bo_hit hit = rt_closest(c, &ray);
    if (hit.prim == BO_EMPTY) {
      v3 un = v3normalize(d);
      float a = 0.5f * (un.y + 1.0f);
      v3 sk = v3make((1.0f - a) * 1.0f + a * 0.5f, (1.0f - a) * 1.0f + a * 0.7f, (1.0f - a) * 1.0f + a * 1.0f);
      v3 add = vmul(T, sk);
      rad[0] += add.x; rad[1] += add.y; rad[2] += add.z;
      break;
    }
    float t = hit.t;
    v3 outward = hit.n;
    int front = v3dot(d, outward) < 0.0f;
    v3 normal = front ? outward : vneg(outward);
    uint32_t surface = c->surfaces[hit.prim];
    uint32_t kind = surface >> 28, midx = surface & 0x0FFFFFFFu;
    v3 p = v3make(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
    if (kind == BO_MAT_EMISSIVE) {
      if (front) {
        v3 L = load3(c->emissives + 3 * (size_t)midx);
        float wgt = 1.0f;
        if (c->algorithm == 3 && b > 0 && !delta) wgt = 0.0f;
        if (c->algorithm == 4 && b > 0 && !delta) {
          float lc = bo_fmaxf(v3dot(normal, vneg(v3normalize(d))), 0.0f);
          float lpdf = 0.0f;
          if (lc > 0.0f && c->total_weight > 0.0f) {
            float d2 = (t * t) * v3dot(d, d);
            lpdf = (d2 * ((L.x + L.y) + L.z)) / ((3.0f * lc) * c->total_weight);
          }
          wgt = power_heuristic(prev_pdf, lpdf);
        }
        v3 TL = vmul(T, L);
        rad[0] += TL.x * wgt; rad[1] += TL.y * wgt; rad[2] += TL.z * wgt;
      }
      break;
    }
    if (kind == BO_MAT_METAL || kind == BO_MAT_DIELECTRIC) {
      /* _gpu_rt_shade_one for METAL / DIELECTRIC (path_shading.mojo:690-786):
       * no light sample; the continuation carries the sample's pdf and delta */
      if (b + 1 >= c->max_depth) break;
      float u[4];
      bo_rt_uniform4(c->seed, path_id, st_bsdf(b), u);
      bo_bsdf sm;
      if (kind == BO_MAT_METAL) {
        const float* m = c->metals + 4 * (size_t)midx;
        sm = sample_metal(d, normal, load3(m), m[3], u[0], u[1]);
      } else {
        sm = sample_dielectric(d, normal, c->dielectrics[midx], front, u[0]);
      }
      if (!sm.ok) break;
      v3 Tm = vmul(T, sm.weight);
      if (b + 1 >= 5u) {
        float mm = bo_fmaxf(Tm.x, bo_fmaxf(Tm.y, Tm.z));
        if (mm <= 0.0f) break;
        float survival = bo_fminf(bo_fmaxf(mm, 0.05f), 0.95f);
        float rr[4];
        bo_rt_uniform4(c->seed, path_id, st_roulette(b), rr);
        if (rr[0] >= survival) break;
        Tm = vdivs(Tm, survival);
      }
      o = p; d = sm.dir; tmin = 0.001f; tmax = BO_FLT_MAX; T = Tm; prev_pdf = sm.pdf; delta = sm.delta;
      continue;
    }
    if (kind != BO_MAT_LAMBERTIAN) break;
    v3 albedo = load3(c->lambertians + 3 * (size_t)midx);
    int want_shadow = 0;
    v3 sh_c = v3make(0, 0, 0);
    bo_ray shadow;
    if ((c->algorithm == 3 || c->algorithm == 4) && c->n_lights > 0 && c->total_weight > 0.0f) {
      float u[4];
      bo_rt_uniform4(c->seed, path_id, st_light(b), u);
      float as = u[0] * (float)c->n_lights;
      uint32_t li = (uint32_t)as;
      float frac = as - (float)li;
      const float* lrec = c->lights + (size_t)li * BO_LIGHT_STRIDE;
      if (frac > lrec[12]) memcpy(&li, &lrec[13], 4);
      lrec = c->lights + (size_t)li * BO_LIGHT_STRIDE;
      v3 p0 = load3(lrec), e1 = v3sub(load3(lrec + 3), p0), e2 = v3sub(load3(lrec + 6), p0);
      v3 av = v3cross(e1, e2);
      float tas = v3dot(av, av);
      if (tas > 0.0f) {
        v3 ln = vdivs(av, sqrtf(tas));
        float ru = sqrtf(u[1]);
        float b1 = ru * (1.0f - u[2]);
        float b2 = ru - b1;
        v3 lp = v3add(v3add(p0, v3muls(e1, b1)), v3muls(e2, b2));
        v3 tl = v3sub(lp, p);
        float d2 = v3dot(tl, tl);
        if (d2 > 1.0e-8f) {
          float dist = sqrtf(d2);
          v3 dir = vdivs(tl, dist);
          float scos = bo_fmaxf(v3dot(normal, dir), 0.0f);
          float lcos = bo_fmaxf(v3dot(ln, vneg(dir)), 0.0f);
          float smax = dist - 0.002f;
          if (scos > 0.0f && lcos > 0.0f && smax > 0.001f) {
            v3 E = load3(lrec + 9);
            float lpdf = (d2 * ((E.x + E.y) + E.z)) / ((3.0f * lcos) * c->total_weight);
            float bpdf = bo_fmaxf(v3dot(normal, v3normalize(dir)), 0.0f) * BO_INV_PI;
            if (lpdf > 0.0f && bpdf > 0.0f) {
              float wgt = c->algorithm == 4 ? power_heuristic(lpdf, bpdf) : 1.0f;
              float scale = (scos * wgt) / lpdf;
              if (scale > 0.0f) {
                v3 value = v3muls(albedo, BO_INV_PI);
                v3 tv = vmul(vmul(T, value), E);
                want_shadow = 1;
                sh_c = v3muls(tv, scale);
                shadow = make_ray_od(p, dir, 0.001f, smax);
              }
            }
          }
        }
      }
    }
    int alive = 0;
    v3 nd = v3make(0, 0, 0), Tn = T;
    float pdf = 0.0f;
    if (b + 1 < c->max_depth) {
      float u[4];
      bo_rt_uniform4(c->seed, path_id, st_bsdf(b), u);
      float s2, c2;
      bo_rt_sincos_turns(u[0], &s2, &c2);
      float z = 1.0f - 2.0f * u[1];
      float radius = sqrtf(bo_fmaxf(1.0f - z * z, 0.0f));
      v3 sd = v3add(normal, v3make(radius * c2, radius * s2, z));
      if (fabsf(sd.x) < 1.0e-8f && fabsf(sd.y) < 1.0e-8f && fabsf(sd.z) < 1.0e-8f) sd = normal;
      nd = v3normalize(sd);
      pdf = bo_fmaxf(v3dot(normal, v3normalize(nd)), 0.0f) * BO_INV_PI;
      Tn = vmul(T, albedo);
      alive = 1;
      if (b + 1 >= 5u) {
        float m = bo_fmaxf(Tn.x, bo_fmaxf(Tn.y, Tn.z));
        if (m <= 0.0f) alive = 0;
        else {
          float survival = bo_fminf(bo_fmaxf(m, 0.05f), 0.95f);
          float rr[4];
          bo_rt_uniform4(c->seed, path_id, st_roulette(b), rr);
          if (rr[0] >= survival) alive = 0;
          else Tn = vdivs(Tn, survival);
        }
      }
    }
    if (want_shadow && !rt_occluded(c, &shadow)) {
      rad[0] += sh_c.x; rad[1] += sh_c.y; rad[2] += sh_c.z;
    }
    if (!alive) break;
    o = p; d = nd; tmin = 0.001f; tmax = BO_FLT_MAX; T = Tn; prev_pdf = pdf; delta = 0;
  }
  out[0] = rad[0]; out[1] = rad[1]; out[2] = rad[2];
}

typedef struct { const rt_ctx* c; } rt_job;

static void rt_range(void* p, uint32_t b, uint32_t e) {
  const rt_ctx* c = ((rt_job*)p)->c;
  for (uint32_t i = b; i < e; ++i) rt_path(c, i, c->sample_radiance + 3 * (size_t)i);
}

/* tree of the next bo_render call (set by bo_render_cwbvh8 around it) */
static __thread struct {
  const float* nodes;
  const float* tris;
  uint32_t n_nodes, n_tris;
} g_render_cw;

/* bo_render: pixels (3 f32, mean over samples in sample order) and optional
 * per-sample radiance.  Scene arrays as in BajoRtScene. */
void bo_render(const BoLbvh* bvh, const float* verts, const uint32_t* surfaces, const float* lambertians,
               const float* emissives, const float* metals, const float* dielectrics, const float* lights,
               uint32_t n_lights, float total_weight,
               const float* cam, uint32_t width, uint32_t height, uint32_t spp, uint32_t max_depth, uint64_t seed,
               int algorithm, float* pixels, float* sample_radiance, uint32_t n_threads) {
  uint64_t n_paths = (uint64_t)width * height * spp;
  float* rad = sample_radiance ? sample_radiance : (float*)malloc(sizeof(float) * 3 * n_paths);
  rt_ctx c = {bvh, verts, surfaces, lambertians, emissives, lights, n_lights, total_weight, metals, dielectrics, cam,
              width, height, spp, max_depth, seed, algorithm, rad, g_render_cw.nodes, g_render_cw.tris,
              g_render_cw.n_nodes, g_render_cw.n_tris};
  rt_job job = {&c};
  bo_parallel_for((uint32_t)n_paths, n_threads, 256, rt_range, &job);
  float scale = 1.0f / (float)spp;
  for (uint64_t px = 0; px < (uint64_t)width * height; ++px) {
    float r = 0.0f, g = 0.0f, b = 0.0f;
    for (uint32_t s = 0; s < spp; ++s) {
      const float* v = rad + 3 * (px * spp + s);
      r += v[0]; g += v[1]; b += v[2];
    }
    pixels[3 * px + 0] = r * scale;
    pixels[3 * px + 1] = g * scale;
    pixels[3 * px + 2] = b * scale;
  }
  if (!sample_radiance) free(rad);
}

/* bo_render through a compressed 8-wide tree (bajo_cwbvh8_build of the
 * scene's single-segment tree): the reference's default triangle scene
 * (prepared_scene.mojo:32-33,52-53). */
void bo_render_cwbvh8(const float* cw_nodes, uint32_t cw_n_nodes, const float* cw_tris, uint32_t cw_n_tris,
                      const float* verts, const uint32_t* surfaces, const float* lambertians, const float* emissives,
                      const float* metals, const float* dielectrics, const float* lights, uint32_t n_lights,
                      float total_weight, const float* cam, uint32_t width, uint32_t height, uint32_t spp,
                      uint32_t max_depth, uint64_t seed, int algorithm, float* pixels, float* sample_radiance,
                      uint32_t n_threads) {
  g_render_cw.nodes = cw_nodes;
  g_render_cw.tris = cw_tris;
  g_render_cw.n_nodes = cw_n_nodes;
  g_render_cw.n_tris = cw_n_tris;
  bo_render(NULL, verts, surfaces, lambertians, emissives, metals, dielectrics, lights, n_lights, total_weight, cam,
            width, height, spp, max_depth, seed, algorithm, pixels, sample_radiance, n_threads);
  g_render_cw.nodes = NULL;
  g_render_cw.tris = NULL;
  g_render_cw.n_nodes = g_render_cw.n_tris = 0;
}

/* ========================================================================= */
/* Batched primary + bounce trace over a segmented LBVH                      */
/* ========================================================================= */
static inline uint32_t st_bsdf0(void) { return (0u << 30) | 1u; }

/* _sample_lambertian (bajo/rt/shading.mojo:92-118), same operations as the
 * CUDA lambertian_dir */
static v3 lambertian_dir(v3 normal, float u, float v) {
  float st, ct;
  bo_rt_sincos_turns(u, &st, &ct);
  float z = 1.0f - 2.0f * v;
  float rad = sqrtf(bo_fmaxf(1.0f - z * z, 0.0f));
  v3 sd = v3add(normal, v3make(rad * ct, rad * st, z));
  if (fabsf(sd.x) < 1.0e-8f && fabsf(sd.y) < 1.0e-8f && fabsf(sd.z) < 1.0e-8f) sd = normal;
  return v3normalize(sd);
}

typedef struct {
  const BoLbvh* bvh;
  const float* verts;
  const float* cams;
  uint32_t cam_stride, width, height;
  uint64_t seed;
  int mode;
  float *t0, *t1;
  uint32_t *p0, *p1;
  uint32_t view_base; /* global view of segment 0 (random streams, camera) */
} batch_ctx;

static void batch_range(void* p, uint32_t b, uint32_t e) {
  const batch_ctx* c = (const batch_ctx*)p;
  const uint32_t ppv = c->width * c->height;
  const float inv_h = 1.0f / (float)c->height;
  for (uint32_t i = b; i < e; ++i) {
    uint32_t view = i / ppv, local = i - view * ppv;
    const uint32_t gview = c->view_base + view;
    const uint32_t gi = gview * ppv + local; /* the ray's index in the whole batch */
    const float* cam = c->cams + (size_t)gview * c->cam_stride;
    uint32_t px = local % c->width, py = local / c->width;
    float sx = (2.0f * ((float)px + 0.5f) - (float)c->width) * inv_h;
    float sy = 1.0f - 2.0f * ((float)py + 0.5f) * inv_h;
    float fs = cam[12];
    v3 d = v3normalize(v3add(v3add(load3(cam + 3), v3muls(load3(cam + 6), sx * fs)), v3muls(load3(cam + 9), sy * fs)));
    v3 o = load3(cam);
    bo_ray r = make_ray_od(o, d, 0.0f, BO_FLT_MAX);
    bo_hit h = trace_one(c->bvh, c->verts, &r, view, c->mode, NULL);
    c->t0[i] = h.t;
    c->p0[i] = h.prim;
    float bt = BO_FLT_MAX;
    uint32_t bp = BO_EMPTY;
    if (h.prim != BO_EMPTY) {
      v3 normal = v3dot(d, h.n) < 0.0f ? h.n : vneg(h.n);
      float u[4];
      bo_rt_uniform4(c->seed, gi, st_bsdf0(), u);
      v3 dir = lambertian_dir(normal, u[0], u[1]);
      v3 p = v3make(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
      bo_ray r2 = make_ray_od(p, dir, 0.001f, BO_FLT_MAX);
      bo_hit h2 = trace_one(c->bvh, c->verts, &r2, view, c->mode, NULL);
      bt = h2.t;
      bp = h2.prim;
    }
    c->t1[i] = bt;
    c->p1[i] = bp;
  }
}

void bo_trace_batch(const BoLbvh* bvh, const float* verts, const float* cams, uint32_t cam_stride, uint32_t width,
                    uint32_t height, uint64_t seed, int mode, float* t0, uint32_t* p0, float* t1, uint32_t* p1,
                    uint32_t n_threads) {
  bo_trace_batch_views(bvh, verts, cams, cam_stride, width, height, seed, mode, 0, t0, p0, t1, p1, n_threads);
}

void bo_trace_batch_views(const BoLbvh* bvh, const float* verts, const float* cams, uint32_t cam_stride,
                          uint32_t width, uint32_t height, uint64_t seed, int mode, uint32_t view_base, float* t0,
                          uint32_t* p0, float* t1, uint32_t* p1, uint32_t n_threads) {
  batch_ctx c = {bvh, verts, cams, cam_stride, width, height, seed, mode, t0, t1, p0, p1, view_base};
  uint32_t n = bvh->n_segments * width * height;
  bo_parallel_for(n, n_threads, 512, batch_range, &c);
}
