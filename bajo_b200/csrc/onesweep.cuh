// onesweep.cuh -- stable LSD radix sort, one scatter kernel per digit (8
// bits, or 10 bits for small 64-bit-key sorts) with decoupled look-back
// (Merrill & Garland / Adinets & Merrill "Onesweep").
//
// Restates the reference's onesweep (bajo/sort/gpu/onesweep.mojo:31-328) for
// sm_100a, with these changes:
//  - keys are staged in shared memory with their own type, so 64-bit keys are
//    sorted correctly (the reference stages them through UInt32 shared memory,
//    onesweep.mojo:244,311,321, which truncates 64-bit keys);
//  - digit ranking finds a key's peers with one ballot per digit bit, like
//    the reference (bajo/sort/gpu/utils.mojo:46-103); the match instruction
//    it replaces was measured twice as slow per pass on B200;
//  - the look-back loads a batch of predecessor flags at once and is bounded
//    by elapsed time (BAJO_STATUS_LOOKBACK_TIMEOUT) instead of spinning
//    forever one flag at a time (onesweep.mojo:246-270);
//  - the per-pass global digit offsets are scanned inside each scatter CTA
//    (one fewer launch than scan_global, onesweep.mojo:102);
//  - two look-back regions alternate between passes and every pass clears the
//    other region's slots, so only the first region needs a memset;
//  - several tile shapes and two digit widths are compiled and chosen at run
//    time (tuning table);
//  - any digit range [begin_bit, end_bit) can be sorted, so constant key bits
//    cost no pass.
#pragma once

#include <type_traits>

#include "bajo_common.cuh"

namespace bajo {
namespace onesweep {

constexpr uint32_t kRadix = 256;
constexpr uint32_t kFlagAgg = 1u << 30;   // tile aggregate published
constexpr uint32_t kFlagInc = 2u << 30;   // inclusive prefix published
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr uint64_t kLookbackTimeoutNs = 200ull * 1000ull * 1000ull;  // 200 ms
constexpr int kLookbackBatch = 8;

template <typename K>
struct KeyTraits;
template <>
struct KeyTraits<uint32_t> {
  static constexpr uint32_t kMax = 0xFFFFFFFFu;
};
template <>
struct KeyTraits<uint64_t> {
  static constexpr uint64_t kMax = 0xFFFFFFFFFFFFFFFFull;
};

// ---------------------------------------------------------------------------
// Tile shapes, digit widths and pass kernels.  Variants 4-6 of the 32-bit
// keys and 5-6 of the 64-bit keys run onesweep_early_pass_kernel (variant 5
// is the built-in choice from 2^20 and 2^19 keys); the others run
// onesweep_pass_kernel or its wide-digit form.  Smaller tiles give small sorts more CTAs.  max_log2n:
// the largest sort (log2 of n) a variant may serve, which bounds the
// look-back memory a workspace must hold.  bits: digit width.  Variant 4 of the 64-bit keys sorts 10-bit
// digits, so the 30 live bits of single-scene LBVH keys take three passes
// instead of four, but each pass does 1,024 digits of per-tile work.
// Measured on B200 (30-bit keys + 32-bit values): 2^14 keys 54.8 vs 60.2 us
// (best 8-bit variant), 2^16 68.3 vs 59.3, 2^18 87.8 vs 71.3; inside the
// LBVH build 2^15 triangles 78.8 vs 80.9 us, 2^16 85-87 vs 85.0.
// ---------------------------------------------------------------------------
constexpr int kNumVariants = 7;  // the largest variant count of any key type
struct Shape {
  int block, kpt, max_log2n, bits, early, lb, match;  // early: onesweep_early_pass_kernel (8-bit digits);
                                                      // lb: look-back flags per round trip (0: kLookbackBatch);
                                                      // match: early pass peers by ballots (0) or shared OR
                                                      // (1; 2: two alternating masks and the run by atomics)
};
template <typename K>
struct Shapes;
template <>
struct Shapes<uint32_t> {
  static constexpr int count = 7;
  static constexpr Shape v[count] = {{512, 12, 30, 8, 0, 0}, {256, 12, 30, 8, 0, 0}, {256, 8, 24, 8, 0, 0},
                                     {256, 4, 20, 8, 0, 0},  {256, 20, 30, 8, 1, 8, 2}, {256, 24, 30, 8, 1, 8, 2},
                                     {256, 32, 30, 8, 1, 8, 2}};
};
constexpr int kEarlyU32Default = 5;  // Shapes<uint32_t>::v[5]
constexpr int kEarlyU64Default = 5;  // Shapes<uint64_t>::v[5]

template <>
struct Shapes<uint64_t> {
  static constexpr int count = 7;
  static constexpr Shape v[count] = {{512, 8, 30, 8}, {256, 8, 30, 8}, {256, 5, 24, 8}, {256, 3, 20, 8},
                                     {256, 4, 18, 10}, {256, 16, 30, 8, 1, 8, 2}, {256, 12, 30, 8, 1, 8, 2}};
};

constexpr uint32_t ceil_log2(uint32_t n) {
  uint32_t l = 0;
  while (l < 32 && (1ull << l) < n) ++l;
  return l;
}
template <typename K>
constexpr bool variant_allowed(int v, uint32_t n) {
  return v >= 0 && v < Shapes<K>::count && ceil_log2(n) <= (uint32_t)Shapes<K>::v[v].max_log2n;
}
template <typename K>
constexpr uint32_t variant_tile(int v) {
  return (uint32_t)(Shapes<K>::v[v].block * Shapes<K>::v[v].kpt);
}
template <typename K>
constexpr uint32_t variant_bits(int v) {
  return (uint32_t)Shapes<K>::v[v].bits;
}
constexpr uint32_t passes_for(int begin_bit, int end_bit, uint32_t bits) {
  return (uint32_t)((end_bit - begin_bit + (int)bits - 1) / (int)bits);
}
// look-back words one region needs for n keys: the largest tiles x digits of
// any allowed variant
template <typename K>
constexpr size_t lookback_words(uint32_t n) {
  size_t w = 0;
  for (int v = 0; v < Shapes<K>::count; ++v) {
    if (!variant_allowed<K>(v, n)) continue;
    const size_t t = ((size_t)n + variant_tile<K>(v) - 1) / variant_tile<K>(v);
    const size_t x = (t ? t : 1) * ((size_t)1 << variant_bits<K>(v));
    if (x > w) w = x;
  }
  return w;
}
// digits per pass of the widest allowed variant (sizes the histograms)
template <typename K>
constexpr uint32_t max_radix(uint32_t n) {
  uint32_t r = 256;
  for (int v = 0; v < Shapes<K>::count; ++v)
    if (variant_allowed<K>(v, n) && (1u << variant_bits<K>(v)) > r) r = 1u << variant_bits<K>(v);
  return r;
}

// Process-wide tuning table: variant per (key bytes, values, log2 n).  A
// negative entry means "use the built-in choice".
int tuned_variant(int key_bytes, bool has_values, uint32_t n);

template <typename K, bool HAS_V>
inline int choose_variant(uint32_t n, int sm_count) {
  int v = tuned_variant((int)sizeof(K), HAS_V, n);
  if (variant_allowed<K>(v, n)) return v;
  // built-in: the largest tile that still gives every SM two tiles
  // built-in: 10-bit digits for small 64-bit-key sorts (measured faster up
  // to 2^15 keys), else the largest 8-bit tile that still gives every SM two
  // tiles
  if (sizeof(K) == 8 && HAS_V && n <= (1u << 15) && variant_allowed<K>(4, n)) return 4;
  // 32-bit keys from 2^20 on: the early-count pass, 256 x 24 keys (measured
  // fastest on B200 at 2^20-2^28, keys and pairs)
  if (sizeof(K) == 4 && n >= (1u << 20) && variant_allowed<K>(kEarlyU32Default, n)) return kEarlyU32Default;
  // 64-bit keys from 2^19 on: the early-count pass, 256 x 16 keys
  if (sizeof(K) == 8 && n >= (1u << 19) && variant_allowed<K>(kEarlyU64Default, n)) return kEarlyU64Default;
  for (int c = 0; c < Shapes<K>::count; ++c) {
    if (!variant_allowed<K>(c, n) || variant_bits<K>(c) != 8) continue;
    if ((n + variant_tile<K>(c) - 1) / variant_tile<K>(c) >= (uint32_t)(2 * sm_count)) return c;
  }
  for (int c = Shapes<K>::count - 1; c >= 0; --c)
    if (variant_allowed<K>(c, n) && variant_bits<K>(c) == 8) return c;
  return 0;
}

// Lanes of the warp whose BITS-bit label equals this lane's: one ballot per
// label bit (full-rate vote instructions; no match instruction).
template <int BITS>
__device__ __forceinline__ uint32_t match_label(uint32_t label) {
  uint32_t peers = 0xFFFFFFFFu;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    const bool set = (label >> b) & 1u;
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, set);
    peers &= set ? m : ~m;
  }
  return peers;
}

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= (uint32_t)o) v += u;
  }
  return v;
}

// Exclusive scan of one value per thread over threads [0, 256) of the block.
// Every thread of the block must call it (threads >= 256 pass anything).
template <int BLOCK>
__device__ __forceinline__ uint32_t scan256_exclusive(uint32_t v, uint32_t* tmp8) {
  static_assert(BLOCK >= 256, "needs 256 threads");
  const uint32_t tid = threadIdx.x;
  uint32_t inc = 0;
  if (tid < 256) {
    inc = warp_inclusive_scan(v);
    if ((tid & 31) == 31) tmp8[tid >> 5] = inc;
  }
  __syncthreads();
  uint32_t excl = 0;
  if (tid < 256) {
    uint32_t w = tid >> 5, add = 0;
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) add += (k < w) ? tmp8[k] : 0u;
    excl = add + inc - v;
  }
  __syncthreads();
  return excl;
}

// ---------------------------------------------------------------------------
// Global digit histogram of every pass in one read of the keys
// (global_histogram, onesweep.mojo:31-99).  Grid-strided over the keys;
// warps own private shared histogram copies to limit contention.
// ---------------------------------------------------------------------------
constexpr int kHistBlock = 256;
constexpr int kHistCopies = 4;  // copies per pass inside a CTA

// Shared copies per pass of a histogram of 2^digit_bits digits.
__host__ __device__ constexpr uint32_t hist_copies(uint32_t digit_bits) { return digit_bits > 8 ? 2u : (uint32_t)kHistCopies; }
constexpr size_t hist_smem(uint32_t passes, uint32_t digit_bits) {
  return (size_t)passes * hist_copies(digit_bits) * (1u << digit_bits) * 4;
}

template <typename K>
__global__ void __launch_bounds__(kHistBlock) global_histogram_kernel(const K* __restrict__ keys, uint32_t n,
                                                                      uint32_t begin_bit, uint32_t n_passes,
                                                                      uint32_t end_bit, uint32_t digit_bits,
                                                                      uint32_t* __restrict__ ghist) {
  extern __shared__ uint32_t s_hist[];  // n_passes * copies * 2^digit_bits
  const uint32_t radix = 1u << digit_bits, copies = hist_copies(digit_bits);
  const uint32_t words = n_passes * copies * radix;
  for (uint32_t i = threadIdx.x; i < words; i += kHistBlock) s_hist[i] = 0;
  __syncthreads();
  const uint32_t copy = (threadIdx.x >> 5) % copies;
  uint32_t* h = s_hist + copy * radix;
  const uint32_t pstride = copies * radix;
  auto count = [&](K k) {
    uint32_t* hp = h;
    for (uint32_t p = 0, sh = begin_bit; p < n_passes; ++p, sh += digit_bits, hp += pstride) {
      const uint32_t bits = min(digit_bits, end_bit - sh);
      atomicAdd(&hp[(uint32_t)(k >> sh) & ((1u << bits) - 1u)], 1u);
    }
  };
  const uint32_t stride = gridDim.x * kHistBlock;
  const uint32_t g = blockIdx.x * kHistBlock + threadIdx.x;
  // 16-byte loads (two in flight per thread) over the aligned bulk, single
  // keys over the rest; the keys are read once, so the loads stream past L1
  constexpr uint32_t kVec = 16 / sizeof(K);
  const uint32_t head = (uint32_t)((((uintptr_t)keys + 15) & ~(uintptr_t)15) - (uintptr_t)keys) / sizeof(K);
  const uint32_t h0 = min(head, n);
  const uint32_t nvec = (n - h0) / kVec;
  const uint4* kv = reinterpret_cast<const uint4*>(keys + h0);
  uint32_t i = g;
  for (; i + stride < nvec; i += 2 * stride) {
    const uint4 a = __ldcs(kv + i), b = __ldcs(kv + i + stride);
    const K* ka = reinterpret_cast<const K*>(&a);
    const K* kb = reinterpret_cast<const K*>(&b);
#pragma unroll
    for (uint32_t j = 0; j < kVec; ++j) count(ka[j]);
#pragma unroll
    for (uint32_t j = 0; j < kVec; ++j) count(kb[j]);
  }
  for (; i < nvec; i += stride) {
    const uint4 a = __ldcs(kv + i);
    const K* ka = reinterpret_cast<const K*>(&a);
#pragma unroll
    for (uint32_t j = 0; j < kVec; ++j) count(ka[j]);
  }
  for (uint32_t q = g; q < h0; q += stride) count(keys[q]);                           // unaligned head
  for (uint32_t q = h0 + nvec * kVec + g; q < n; q += stride) count(keys[q]);  // ragged tail
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < n_passes * radix; q += kHistBlock) {
    uint32_t p = q / radix, d = q % radix, sum = 0;
    for (uint32_t c = 0; c < copies; ++c) sum += s_hist[(p * copies + c) * radix + d];
    if (sum) atomicAdd(&ghist[p * radix + d], sum);
  }
}

// ---------------------------------------------------------------------------
// One digit pass (digit_binning, onesweep.mojo:121-328).
//
// The pass is bound by shared-memory instruction issue, so every per-key
// shared access is counted: ranking costs one match, one shuffle and one
// shared atomic by the run leader; the per-(warp, digit) start is a single
// lookup; key and value are staged together (one 8- or 16-byte store and
// load); the scatter looks up one destination base per key.
// ---------------------------------------------------------------------------
template <typename K, bool HAS_V>
struct Staged;
template <>
struct Staged<uint32_t, false> {
  using T = uint32_t;
  __device__ static T pack(uint32_t k, uint32_t) { return k; }
  __device__ static uint32_t key(T t) { return t; }
  __device__ static uint32_t val(T) { return 0; }
};
template <>
struct Staged<uint32_t, true> {
  using T = uint2;
  __device__ static T pack(uint32_t k, uint32_t v) { return make_uint2(k, v); }
  __device__ static uint32_t key(T t) { return t.x; }
  __device__ static uint32_t val(T t) { return t.y; }
};
template <>
struct Staged<uint64_t, false> {
  using T = uint64_t;
  __device__ static T pack(uint64_t k, uint32_t) { return k; }
  __device__ static uint64_t key(T t) { return t; }
  __device__ static uint32_t val(T) { return 0; }
};
template <>
struct Staged<uint64_t, true> {
  using T = uint4;
  __device__ static T pack(uint64_t k, uint32_t v) {
    return make_uint4((uint32_t)k, (uint32_t)(k >> 32), v, 0u);
  }
  __device__ static uint64_t key(T t) { return ((uint64_t)t.y << 32) | t.x; }
  __device__ static uint32_t val(T t) { return t.z; }
};

template <typename K, bool HAS_V, int BLOCK, int KPT>
struct BinSmem {
  using T = typename Staged<K, HAS_V>::T;
  static constexpr int kWarps = BLOCK / 32;
  static constexpr int kTile = BLOCK * KPT;
  union {
    T staged[kTile];
    uint32_t warp_hist[kWarps * kRadix];  // per (warp, digit): count, then start
  } u;
  uint32_t digit_offset[kRadix];
  uint32_t scan_tmp[8];
  uint32_t tile;
  uint32_t abort;  // a look-back wait timed out: publish, skip the scatter
};

__device__ __forceinline__ void prefetch_l2_bulk(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// lookback: this pass's flags; lookback_next: the other region, whose slot of
// this tile is cleared for the next pass.
template <typename K, bool HAS_V, bool EMIT_LOW32, int BLOCK, int KPT, int LB = kLookbackBatch>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) onesweep_pass_kernel(
    const K* __restrict__ keys_in, K* __restrict__ keys_out, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ vals_out, uint32_t* __restrict__ low32_out, const uint32_t* __restrict__ ghist,
    uint32_t* __restrict__ lookback, uint32_t* __restrict__ lookback_next, uint32_t* __restrict__ tile_counter,
    uint32_t* __restrict__ status, uint32_t n, uint32_t shift, uint32_t digit_mask) {
  using S = BinSmem<K, HAS_V, BLOCK, KPT>;
  using ST = Staged<K, HAS_V>;
  constexpr int kWarps = S::kWarps;
  constexpr uint32_t kTile = S::kTile;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& s = *reinterpret_cast<S*>(smem_raw);

  const uint32_t tid = threadIdx.x;
  const uint32_t lane = tid & 31, warp = tid >> 5;

  for (uint32_t i = tid; i < kWarps * kRadix; i += BLOCK) s.u.warp_hist[i] = 0;
  if (tid == 0) {
    s.tile = atomicAdd(tile_counter, 1u);  // tiles in launch order
    s.abort = 0;
  }
  __syncthreads();
  const uint32_t tile = s.tile;
  const uint32_t tile_base = tile * kTile;
  const uint32_t valid = min(kTile, n - tile_base);
  if (HAS_V && tid == 0 && (((uintptr_t)(vals_in + tile_base)) & 15) == 0)
    prefetch_l2_bulk(vals_in + tile_base, (valid * 4u) & ~15u);  // values are read after the look-back
  if (lookback_next && tid < kRadix) lookback_next[tile * kRadix + tid] = 0;

  // warp-striped load: key i of this thread sits at tile position
  // warp*32*KPT + 32*i + lane, so (warp, i, lane) order is position order.
  K key[KPT];
  const uint32_t pos0 = tile_base + warp * 32 * KPT + lane;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    uint32_t p = pos0 + 32 * i;
    key[i] = (p < n) ? keys_in[p] : KeyTraits<K>::kMax;
  }

  // rank every key among equal digits of its warp, in position order
  uint32_t* wh = s.u.warp_hist + warp * kRadix;
  const uint32_t lt = lanemask_lt();
  uint32_t rank[KPT];
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t d = (uint32_t)(key[i] >> shift) & digit_mask;
    const uint32_t peers = match_label<8>(d);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t before = 0;
    if (lane == leader) before = atomicAdd(&wh[d], (uint32_t)__popc(peers));
    before = __shfl_sync(0xFFFFFFFFu, before, leader);
    rank[i] = before + __popc(peers & lt);
  }
  __syncthreads();

  // per digit: tile total, publish the tile aggregate
  uint32_t total = 0, agg = 0, gcount = 0;
  if (tid < kRadix) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) total += s.u.warp_hist[w * kRadix + tid];
    agg = total - ((tid == digit_mask) ? (kTile - valid) : 0u);  // padding keys carry the top digit
    uint32_t word = agg | (tile == 0 ? kFlagInc : kFlagAgg);
    st_relaxed_gpu(&lookback[tile * kRadix + tid], word);
    gcount = ghist[tid];
  }
  const uint32_t tstart = scan256_exclusive<BLOCK>(total, s.scan_tmp);
  const uint32_t gstart = scan256_exclusive<BLOCK>(gcount, s.scan_tmp);
  if (tid < kRadix) {
    // per (warp, digit) start inside the tile: tile start of the digit plus
    // the counts of the earlier warps
    uint32_t run = tstart;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = s.u.warp_hist[w * kRadix + tid];
      s.u.warp_hist[w * kRadix + tid] = run;
      run += c;
    }
  }
  __syncthreads();
  // tile-local sorted position of every key (rank becomes the position)
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t d = (uint32_t)(key[i] >> shift) & digit_mask;
    rank[i] += s.u.warp_hist[warp * kRadix + d];
  }

  // Decoupled look-back, one thread per digit.  The flags of up to LB
  // predecessors are loaded at once (independent loads), so a chain of ready
  // aggregates costs one L2 round trip per batch.
  if (tid < kRadix) {
    uint32_t excl = 0;
    if (tile > 0) {
      int32_t k = (int32_t)tile - 1;
      uint32_t spins = 0;
      uint64_t t0 = 0;
      while (k >= 0) {
        uint32_t f[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q)
          f[q] = (k - q >= 0) ? ld_relaxed_gpu(&lookback[(uint32_t)(k - q) * kRadix + tid]) : kFlagInc;
        int consumed = 0;
        bool done = false;
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          if (done || consumed != q) continue;  // stop at the first flag not ready
          const uint32_t flag = f[q] & kFlagMask;
          if (flag == kFlagInc) {
            excl += f[q] & kValueMask;
            done = true;
          } else if (flag == kFlagAgg) {
            excl += f[q] & kValueMask;
            ++consumed;
          }
        }
        if (done) break;
        k -= consumed;
        if (consumed > 0) {
          spins = 0;
          continue;
        }
        // not ready: back off, give up after kLookbackTimeoutNs
        if (spins == 0) t0 = global_timer_ns();
        ++spins;
        if ((spins & 63u) == 0 && global_timer_ns() - t0 > kLookbackTimeoutNs) {
          raise_status(status, BAJO_STATUS_LOOKBACK_TIMEOUT);
          s.abort = 1;
          break;
        }
        __nanosleep(spins < 64 ? 32 : 256);
      }
      st_relaxed_gpu(&lookback[tile * kRadix + tid], ((excl + agg) & kValueMask) | kFlagInc);
    }
    s.digit_offset[tid] = gstart + excl - tstart;
  }
  __syncthreads();
  // The successors are released (inclusive prefixes published); without a
  // complete prefix the scatter addresses are unknown, so write nothing.
  if (s.abort) return;

  // stage key (+ value) at its tile-local position (the barrier above also
  // ends every read of warp_hist, which the staging overwrites)
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    uint32_t v = 0;
    if constexpr (HAS_V) {
      const uint32_t p = pos0 + 32 * i;
      v = (p < n) ? vals_in[p] : 0u;
    }
    s.u.staged[rank[i]] = ST::pack(key[i], v);
  }
  __syncthreads();

  // scatter: consecutive tile slots of one digit go to consecutive addresses
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t j = tid + i * BLOCK;
    if (j < valid) {
      const auto e = s.u.staged[j];
      const K k = ST::key(e);
      const uint32_t d = (uint32_t)(k >> shift) & digit_mask;
      const uint32_t dst = s.digit_offset[d] + j;
      if (dst < n) {  // holds whenever the digit counts are consistent
        keys_out[dst] = k;
        if constexpr (HAS_V) vals_out[dst] = ST::val(e);
        if constexpr (EMIT_LOW32) low32_out[dst] = (uint32_t)k;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// One digit pass with early counts (8-bit digits; threads below 256: one per
// digit).  The same result as onesweep_pass_kernel, in another order:
//  1. every warp counts its keys' digits into its own shared histogram (one
//     shared atomic per key, no ranking yet);
//  2. thread d sums digit d over the warps, publishes the tile's aggregate
//     at once (successors' look-backs need not wait for this tile's ranking)
//     and turns the warp counts into each warp's first tile position of d;
//  3. ranking: per key one match over the warp's digits, one shared load of
//     the warp's running position of the digit and, by the highest peer,
//     one shared store of the advanced position (no atomic, no shuffle);
//  4. keys (and values) staged in tile order;
//  5. the look-back (thread d), after the ranking, when the predecessors'
//     prefixes are most likely complete, many predecessors' flags per round
//     trip;
//  6. the scatter of digit runs.
// ---------------------------------------------------------------------------
template <typename K, bool HAS_V, int BLOCK, int KPT>
struct EarlySmem {
  using T = typename Staged<K, HAS_V>::T;
  static constexpr int kWarps = BLOCK / 32;
  static constexpr int kTile = BLOCK * KPT;
  union {
    T staged[kTile];
    struct {
      uint32_t warp_run[kWarps * kRadix];  // per (warp, digit): count, then running tile position
      uint32_t match[2][kWarps * kRadix];  // per (warp, digit): lanes whose key has the digit (MATCH 1, 2)
    } r;
  } u;
  uint32_t digit_offset[kRadix];
  uint32_t scan_tmp[8];
  uint32_t tile;
  uint32_t abort;
};

template <typename K, bool HAS_V, bool EMIT_LOW32, int BLOCK, int KPT, int LB = kLookbackBatch, int MATCH = 0>
__global__ void __launch_bounds__(BLOCK, BLOCK >= 512 ? 1 : (KPT >= 32 ? 2 : 3)) onesweep_early_pass_kernel(
    const K* __restrict__ keys_in, K* __restrict__ keys_out, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ vals_out, uint32_t* __restrict__ low32_out, const uint32_t* __restrict__ ghist,
    uint32_t* __restrict__ lookback, uint32_t* __restrict__ lookback_next, uint32_t* __restrict__ tile_counter,
    uint32_t* __restrict__ status, uint32_t n, uint32_t shift, uint32_t digit_mask) {
  static_assert(BLOCK % (int)kRadix == 0, "threads below kRadix: one per digit");
  using S = EarlySmem<K, HAS_V, BLOCK, KPT>;
  using ST = Staged<K, HAS_V>;
  constexpr int kWarps = S::kWarps;
  constexpr uint32_t kTile = S::kTile;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& s = *reinterpret_cast<S*>(smem_raw);

  const uint32_t tid = threadIdx.x;
  const uint32_t lane = tid & 31, warp = tid >> 5;

  for (uint32_t q = tid; q < kWarps * kRadix; q += BLOCK) {
    s.u.r.warp_run[q] = 0;
    if constexpr (MATCH >= 1) s.u.r.match[0][q] = 0;
    if constexpr (MATCH == 2) s.u.r.match[1][q] = 0;
  }
  if (tid == 0) {
    s.tile = atomicAdd(tile_counter, 1u);  // tiles in launch order
    s.abort = 0;
  }
  __syncthreads();
  const uint32_t tile = s.tile;
  const uint32_t tile_base = tile * kTile;
  const uint32_t valid = min(kTile, n - tile_base);
  if (HAS_V && tid == 0 && (((uintptr_t)(vals_in + tile_base)) & 15) == 0)
    prefetch_l2_bulk(vals_in + tile_base, (valid * 4u) & ~15u);  // values are read after the look-back
  if (lookback_next && tid < kRadix) lookback_next[tile * kRadix + tid] = 0;

  // warp-striped load: key i of this thread sits at tile position
  // warp*32*KPT + 32*i + lane, so (warp, i, lane) order is position order.
  K key[KPT];
  const uint32_t pos0 = tile_base + warp * 32 * KPT + lane;
  const bool full = valid == kTile;  // every tile but the last: no bounds checks
  if (full) {
#pragma unroll
    for (int i = 0; i < KPT; ++i) key[i] = keys_in[pos0 + 32 * i];
  } else {
#pragma unroll
    for (int i = 0; i < KPT; ++i) {
      const uint32_t p = pos0 + 32 * i;
      key[i] = (p < n) ? keys_in[p] : KeyTraits<K>::kMax;
    }
  }
  // 1. the warp's digit counts
  uint32_t* wr = s.u.r.warp_run + warp * kRadix;
  uint32_t* wm = s.u.r.match[0] + warp * kRadix;
#pragma unroll
  for (int i = 0; i < KPT; ++i) atomicAdd(&wr[(uint32_t)(key[i] >> shift) & digit_mask], 1u);
  __syncthreads();

  // 2. thread d: the tile's count of digit d, published at once, and each
  // warp's first tile position of d
  uint32_t cw[kWarps], total = 0, agg = 0, gcount = 0;
  if (tid < kRadix) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      cw[w] = s.u.r.warp_run[w * kRadix + tid];
      total += cw[w];
    }
    agg = total - ((tid == digit_mask) ? (kTile - valid) : 0u);  // padding keys: the top digit
    st_relaxed_gpu(&lookback[tile * kRadix + tid], agg | (tile == 0 ? kFlagInc : kFlagAgg));
    gcount = ghist[tid];
  }
  const uint32_t tstart = scan256_exclusive<BLOCK>(total, s.scan_tmp);
  const uint32_t gstart = scan256_exclusive<BLOCK>(gcount, s.scan_tmp);
  if (tid < kRadix) {
    uint32_t run = tstart;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      s.u.r.warp_run[w * kRadix + tid] = run;
      run += cw[w];
    }
  }
  __syncthreads();

  // 3. ranks: tile positions, in position order within every digit
  const uint32_t lt = lanemask_lt();
  uint32_t rank[KPT];
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t d = (uint32_t)(key[i] >> shift) & digit_mask;
    if constexpr (MATCH == 2) {
      // masks alternate between two arrays, so a mask cleared here is next
      // written two keys later, after the next key's warp barrier; the
      // run moves by the lowest peer's atomic add (atomics on one word keep
      // their order), whose old value the peers take by shuffle
      uint32_t* m = s.u.r.match[i & 1] + warp * kRadix;
      atomicOr(&m[d], 1u << lane);
      __syncwarp();
      const uint32_t peers = m[d];
      const uint32_t leader = __ffs(peers) - 1;
      uint32_t at = 0;
      if (lane == leader) {
        at = atomicAdd(&wr[d], (uint32_t)__popc(peers));
        m[d] = 0u;
      }
      rank[i] = __shfl_sync(0xFFFFFFFFu, at, leader) + __popc(peers & lt);
      continue;
    }
    uint32_t peers;
    if constexpr (MATCH == 1) {  // every lane ORs its bit into the digit's mask
      atomicOr(&wm[d], 1u << lane);
      __syncwarp();
      peers = wm[d];
    } else {
      peers = match_label<8>(d);
    }
    const uint32_t at = wr[d];
    rank[i] = at + __popc(peers & lt);
    __syncwarp();  // every peer has read the run (and the mask) before they change
    if ((peers >> lane) == 1u) {  // the highest peer advances the run
      wr[d] = at + __popc(peers);
      if constexpr (MATCH == 1) wm[d] = 0u;
    }
    __syncwarp();
  }

  __syncthreads();  // every warp has ranked: warp_run is not read again
  // 4. stage key (+ value) at its tile position (so the look-back below runs
  // with few live registers, and the value loads overlap it)
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    uint32_t v = 0;
    if constexpr (HAS_V) {
      const uint32_t p = pos0 + 32 * i;
      v = (full || p < n) ? vals_in[p] : 0u;
    }
    s.u.staged[rank[i]] = ST::pack(key[i], v);
  }

  // 5. decoupled look-back, thread d (as in onesweep_pass_kernel)
  if (tid < kRadix) {
    uint32_t excl = 0;
    if (tile > 0) {
      int32_t k = (int32_t)tile - 1;
      uint32_t spins = 0;
      uint64_t t0 = 0;
      while (k >= 0) {
        uint32_t f[LB];
#pragma unroll
        for (int q = 0; q < LB; ++q)
          f[q] = (k - q >= 0) ? ld_relaxed_gpu(&lookback[(uint32_t)(k - q) * kRadix + tid]) : kFlagInc;
        int consumed = 0;
        bool done = false;
#pragma unroll
        for (int q = 0; q < LB; ++q) {
          if (done || consumed != q) continue;  // stop at the first flag not ready
          const uint32_t flag = f[q] & kFlagMask;
          if (flag == kFlagInc) {
            excl += f[q] & kValueMask;
            done = true;
          } else if (flag == kFlagAgg) {
            excl += f[q] & kValueMask;
            ++consumed;
          }
        }
        if (done) break;
        k -= consumed;
        if (consumed > 0) {
          spins = 0;
          continue;
        }
        if (spins == 0) t0 = global_timer_ns();
        ++spins;
        if ((spins & 63u) == 0 && global_timer_ns() - t0 > kLookbackTimeoutNs) {
          raise_status(status, BAJO_STATUS_LOOKBACK_TIMEOUT);
          s.abort = 1;
          break;
        }
        __nanosleep(spins < 64 ? 32 : 256);
      }
      st_relaxed_gpu(&lookback[tile * kRadix + tid], ((excl + agg) & kValueMask) | kFlagInc);
    }
    s.digit_offset[tid] = gstart + excl - tstart;
  }
  __syncthreads();  // the staged tile and the digit offsets are complete
  if (s.abort) return;

  // 6. scatter digit runs
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t j = tid + i * BLOCK;
    if (full || j < valid) {
      const auto e = s.u.staged[j];
      const K k = ST::key(e);
      const uint32_t d = (uint32_t)(k >> shift) & digit_mask;
      const uint32_t dst = s.digit_offset[d] + j;
      if (dst < n) {  // holds whenever the digit counts are consistent
        keys_out[dst] = k;
        if constexpr (HAS_V) vals_out[dst] = ST::val(e);
        if constexpr (EMIT_LOW32) low32_out[dst] = (uint32_t)k;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// One pass over wide digits (2^RBITS = 1,024 digits): the same steps as
// onesweep_pass_kernel, reorganised for many digits per thread.
//  - per-(warp, digit) counters are 16-bit (a tile holds fewer than 65,536
//    keys) and warp private, so the run leader updates them without an
//    atomic;
//  - each thread owns DPT consecutive digits: it publishes and reads their
//    look-back flags with 16-byte loads and stores, and walks the
//    predecessors of all of them in one loop;
//  - the tile scans of the digit totals are one block scan of per-thread
//    sums.
// ---------------------------------------------------------------------------
template <typename K, bool HAS_V, int BLOCK, int KPT, int RBITS>
struct WideBinSmem {
  using T = typename Staged<K, HAS_V>::T;
  static constexpr int kWarps = BLOCK / 32;
  static constexpr int kTile = BLOCK * KPT;
  static constexpr int R = 1 << RBITS;
  static_assert(kTile < 65536, "16-bit per-warp counters");
  union {
    T staged[kTile];
    uint16_t warp_hist[kWarps * R];  // per (warp, digit): count, then start
  } u;
  uint32_t digit_offset[R];
  uint32_t scan_tmp[2][kWarps];
  uint32_t tile;
  uint32_t abort;
};

__device__ __forceinline__ void st_relaxed_gpu_v4(uint32_t* p, uint4 v) {
  asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z),
               "r"(v.w)
               : "memory");
}
__device__ __forceinline__ uint4 ld_relaxed_gpu_v4(const uint32_t* p) {
  uint4 v;
  asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p)
               : "memory");
  return v;
}

// exclusive block scans of two values per thread
template <int BLOCK>
__device__ __forceinline__ void scan2_exclusive(uint32_t a, uint32_t b, uint32_t* tmpa, uint32_t* tmpb,
                                                uint32_t& ea, uint32_t& eb) {
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t ia = warp_inclusive_scan(a), ib = warp_inclusive_scan(b);
  if (lane == 31) {
    tmpa[warp] = ia;
    tmpb[warp] = ib;
  }
  __syncthreads();
  uint32_t sa = 0, sb = 0;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; ++w)
    if (w < (int)warp) {
      sa += tmpa[w];
      sb += tmpb[w];
    }
  ea = sa + ia - a;
  eb = sb + ib - b;
  __syncthreads();
}

template <typename K, bool HAS_V, bool EMIT_LOW32, int BLOCK, int KPT, int RBITS>
__global__ void __launch_bounds__(BLOCK) onesweep_wide_pass_kernel(
    const K* __restrict__ keys_in, K* __restrict__ keys_out, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ vals_out, uint32_t* __restrict__ low32_out, const uint32_t* __restrict__ ghist,
    uint32_t* __restrict__ lookback, uint32_t* __restrict__ lookback_next, uint32_t* __restrict__ tile_counter,
    uint32_t* __restrict__ status, uint32_t n, uint32_t shift, uint32_t digit_mask) {
  using S = WideBinSmem<K, HAS_V, BLOCK, KPT, RBITS>;
  using ST = Staged<K, HAS_V>;
  constexpr int R = S::R, kWarps = S::kWarps;
  constexpr uint32_t kTile = S::kTile;
  constexpr int DPT = R / BLOCK;  // consecutive digits per thread
  static_assert(DPT % 4 == 0, "digits are handled in groups of four");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& s = *reinterpret_cast<S*>(smem_raw);
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  {
    uint4* z = reinterpret_cast<uint4*>(s.u.warp_hist);
    for (uint32_t i = tid; i < kWarps * R * 2 / 16; i += BLOCK) z[i] = make_uint4(0, 0, 0, 0);
  }
  if (tid == 0) {
    s.tile = atomicAdd(tile_counter, 1u);  // tiles in launch order
    s.abort = 0;
  }
  __syncthreads();
  const uint32_t tile = s.tile;
  const uint32_t tile_base = tile * kTile;
  const uint32_t valid = min(kTile, n - tile_base);
  const uint32_t d0 = tid * DPT;
  if (lookback_next) {
#pragma unroll
    for (int g = 0; g < DPT / 4; ++g)
      reinterpret_cast<uint4*>(lookback_next + (size_t)tile * R + d0)[g] = make_uint4(0, 0, 0, 0);
  }

  K key[KPT];
  const uint32_t pos0 = tile_base + warp * 32 * KPT + lane;
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t p = pos0 + 32 * i;
    key[i] = (p < n) ? keys_in[p] : KeyTraits<K>::kMax;
  }
  // rank among equal digits of the warp, in position order
  uint16_t* wh = s.u.warp_hist + warp * R;
  const uint32_t lt = lanemask_lt();
  uint32_t rank[KPT];
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t d = (uint32_t)(key[i] >> shift) & digit_mask;
    const uint32_t peers = match_label<RBITS>(d);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t before = 0;
    if (lane == leader) {  // one leader per digit value: no two lanes share a counter
      before = wh[d];
      wh[d] = (uint16_t)(before + __popc(peers));
    }
    __syncwarp();
    before = __shfl_sync(0xFFFFFFFFu, before, leader);
    rank[i] = before + __popc(peers & lt);
  }
  __syncthreads();

  // this thread's digits: tile totals, published aggregates, global counts
  uint32_t total[DPT], agg[DPT], gc[DPT];
  uint32_t tsum = 0, gsum = 0;
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    const uint32_t d = d0 + j;
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) t += s.u.warp_hist[w * R + d];
    total[j] = t;
    agg[j] = t - ((d == digit_mask) ? (kTile - valid) : 0u);  // padding keys carry the top digit
    gc[j] = ghist[d];
    tsum += t;
    gsum += gc[j];
  }
  {
    const uint32_t f = tile == 0 ? kFlagInc : kFlagAgg;
#pragma unroll
    for (int g = 0; g < DPT / 4; ++g)
      st_relaxed_gpu_v4(lookback + (size_t)tile * R + d0 + 4 * g,
                        make_uint4(agg[4 * g] | f, agg[4 * g + 1] | f, agg[4 * g + 2] | f, agg[4 * g + 3] | f));
  }
  uint32_t tbase, gbase;
  scan2_exclusive<BLOCK>(tsum, gsum, s.scan_tmp[0], s.scan_tmp[1], tbase, gbase);
  uint32_t tstart[DPT], gstart[DPT];
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    tstart[j] = tbase;
    gstart[j] = gbase;
    tbase += total[j];
    gbase += gc[j];
  }
  // per (warp, digit) start inside the tile
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    const uint32_t d = d0 + j;
    uint32_t run = tstart[j];
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t c = s.u.warp_hist[w * R + d];
      s.u.warp_hist[w * R + d] = (uint16_t)run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t d = (uint32_t)(key[i] >> shift) & digit_mask;
    rank[i] += s.u.warp_hist[warp * R + d];
  }

  // decoupled look-back over the predecessors, all DPT digits together:
  // a step consumes one predecessor once every pending digit's flag there
  // is published
  uint32_t excl[DPT];
#pragma unroll
  for (int j = 0; j < DPT; ++j) excl[j] = 0;
  if (tile > 0) {
    constexpr uint32_t kAll = (DPT >= 32) ? 0xFFFFFFFFu : ((1u << DPT) - 1u);
    uint32_t done = 0;  // bit j: digit j has reached an inclusive prefix
    int32_t k = (int32_t)tile - 1;
    uint32_t spins = 0;
    uint64_t t0 = 0;
    while (done != kAll && k >= 0) {
      uint32_t f[DPT];
#pragma unroll
      for (int g = 0; g < DPT / 4; ++g) {
        const uint4 v = ld_relaxed_gpu_v4(lookback + (size_t)k * R + d0 + 4 * g);
        f[4 * g] = v.x;
        f[4 * g + 1] = v.y;
        f[4 * g + 2] = v.z;
        f[4 * g + 3] = v.w;
      }
      bool ready = true;
#pragma unroll
      for (int j = 0; j < DPT; ++j)
        if (!((done >> j) & 1u) && !(f[j] & kFlagMask)) ready = false;
      if (ready) {
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
          if ((done >> j) & 1u) continue;
          excl[j] += f[j] & kValueMask;
          if ((f[j] & kFlagMask) == kFlagInc) done |= 1u << j;
        }
        --k;
        spins = 0;
        continue;
      }
      // not ready: back off, give up after kLookbackTimeoutNs
      if (spins == 0) t0 = global_timer_ns();
      ++spins;
      if ((spins & 63u) == 0 && global_timer_ns() - t0 > kLookbackTimeoutNs) {
        raise_status(status, BAJO_STATUS_LOOKBACK_TIMEOUT);
        s.abort = 1;
        break;
      }
      __nanosleep(spins < 64 ? 32 : 256);
    }
#pragma unroll
    for (int g = 0; g < DPT / 4; ++g)
      st_relaxed_gpu_v4(lookback + (size_t)tile * R + d0 + 4 * g,
                        make_uint4(((excl[4 * g] + agg[4 * g]) & kValueMask) | kFlagInc,
                                   ((excl[4 * g + 1] + agg[4 * g + 1]) & kValueMask) | kFlagInc,
                                   ((excl[4 * g + 2] + agg[4 * g + 2]) & kValueMask) | kFlagInc,
                                   ((excl[4 * g + 3] + agg[4 * g + 3]) & kValueMask) | kFlagInc));
  }
#pragma unroll
  for (int j = 0; j < DPT; ++j) s.digit_offset[d0 + j] = gstart[j] + excl[j] - tstart[j];
  __syncthreads();
  // without a complete prefix the scatter addresses are unknown: write nothing
  if (s.abort) return;

#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    uint32_t v = 0;
    if constexpr (HAS_V) {
      const uint32_t p = pos0 + 32 * i;
      v = (p < n) ? vals_in[p] : 0u;
    }
    s.u.staged[rank[i]] = ST::pack(key[i], v);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < KPT; ++i) {
    const uint32_t j = tid + i * BLOCK;
    if (j < valid) {
      const auto e = s.u.staged[j];
      const K k = ST::key(e);
      const uint32_t d = (uint32_t)(k >> shift) & digit_mask;
      const uint32_t dst = s.digit_offset[d] + j;
      if (dst < n) {  // holds whenever the digit counts are consistent
        keys_out[dst] = k;
        if constexpr (HAS_V) vals_out[dst] = ST::val(e);
        if constexpr (EMIT_LOW32) low32_out[dst] = (uint32_t)k;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host-side plan
// ---------------------------------------------------------------------------
inline uint32_t num_passes(int begin_bit, int end_bit) { return (uint32_t)((end_bit - begin_bit + 7) / 8); }

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Workspace of one sort: [status | ghist | tile counters (P) | look-back
// region 0 | look-back region 1 | keys_alt | vals_alt].  ghist holds P
// histograms of up to max_radix digits, a look-back region lookback_words
// flags (both sized for every variant the size allows).  ghist, the
// counters and region 0 must start zeroed (one memset of zero_bytes from
// off_ghist); region 1 is cleared by the first pass.
// An optional `extra` region (caller data that must also start zeroed) sits
// between the status word and ghist, inside the zeroed range.
struct Plan {
  uint32_t n, passes, radix;
  size_t lb_words;
  size_t off_extra, off_zero, off_ghist, off_counters, off_lookback, zero_bytes, off_keys_alt, off_vals_alt, total;
};

// passes: the 8-bit digit passes of the sorted bit range (every allowed
// variant needs at most as many).
constexpr Plan make_plan_words(uint32_t n, uint32_t key_bytes, bool has_values, uint32_t passes, uint32_t radix,
                               size_t lb_words, size_t extra_zero_bytes = 0) {
  Plan p{};
  p.n = n;
  p.passes = passes;
  p.radix = radix;
  p.lb_words = lb_words;
  size_t o = 256;  // status word
  p.off_extra = o;
  p.off_zero = o;
  o += (extra_zero_bytes + 15) & ~(size_t)15;
  p.off_ghist = o;
  o += (size_t)passes * radix * 4;
  p.off_counters = o;
  o += (size_t)passes * 4;
  o = (o + 15) & ~(size_t)15;
  p.off_lookback = o;
  p.zero_bytes = o + lb_words * 4 - p.off_zero;
  o += 2 * lb_words * 4;
  o = align256(o);
  p.off_keys_alt = o;
  o = align256(o + (size_t)n * key_bytes);
  p.off_vals_alt = o;
  if (has_values) o = align256(o + (size_t)n * 4);
  p.total = o;
  return p;
}

template <typename K>
constexpr Plan make_plan(uint32_t n, bool has_values, uint32_t passes, size_t extra_zero_bytes = 0) {
  return make_plan_words(n, (uint32_t)sizeof(K), has_values, passes, max_radix<K>(n), lookback_words<K>(n),
                         extra_zero_bytes);
}

template <typename K, bool HAS_V, bool EMIT_LOW32, int V>
inline cudaError_t launch_variant(const K* kin, K* kout, const uint32_t* vin, uint32_t* vout, uint32_t* low32,
                                  const uint32_t* ghist, uint32_t* lb, uint32_t* lb_next, uint32_t* counter,
                                  uint32_t* status, uint32_t n, uint32_t shift, uint32_t digit_mask,
                                  cudaStream_t stream) {
  constexpr int B = Shapes<K>::v[V].block;
  constexpr int KPT = Shapes<K>::v[V].kpt;
  constexpr int BITS = Shapes<K>::v[V].bits;
  constexpr bool EARLY = Shapes<K>::v[V].early != 0;
  constexpr int LB = Shapes<K>::v[V].lb > 0 ? Shapes<K>::v[V].lb : kLookbackBatch;
  constexpr int MATCH = Shapes<K>::v[V].match;
  using Smem = typename std::conditional<
      EARLY, EarlySmem<K, HAS_V, B, KPT>,
      typename std::conditional<BITS == 8, BinSmem<K, HAS_V, B, KPT>,
                                WideBinSmem<K, HAS_V, B, KPT, (BITS == 8 ? 10 : BITS)>>::type>::type;
  auto kern = [] {
    if constexpr (EARLY) return onesweep_early_pass_kernel<K, HAS_V, EMIT_LOW32, B, KPT, LB, MATCH>;
    else if constexpr (BITS == 8) return onesweep_pass_kernel<K, HAS_V, EMIT_LOW32, B, KPT, LB>;
    else return onesweep_wide_pass_kernel<K, HAS_V, EMIT_LOW32, B, KPT, BITS>;
  }();
  const size_t smem = sizeof(Smem);
  static bool configured[64] = {};  // per template instance and device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || !configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) configured[dev] = true;
  }
  const uint32_t tiles = (n + B * KPT - 1) / (B * KPT);
  kern<<<tiles, B, smem, stream>>>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter, status, n, shift,
                                   digit_mask);
  return cudaGetLastError();
}

template <typename K, bool HAS_V, bool EMIT_LOW32>
inline cudaError_t launch_pass(int variant, const K* kin, K* kout, const uint32_t* vin, uint32_t* vout,
                               uint32_t* low32, const uint32_t* ghist, uint32_t* lb, uint32_t* lb_next,
                               uint32_t* counter, uint32_t* status, uint32_t n, uint32_t shift, uint32_t digit_mask,
                               cudaStream_t stream) {
  switch (variant) {
    case 1:
      return launch_variant<K, HAS_V, EMIT_LOW32, 1>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                     status, n, shift, digit_mask, stream);
    case 2:
      return launch_variant<K, HAS_V, EMIT_LOW32, 2>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                     status, n, shift, digit_mask, stream);
    case 3:
      return launch_variant<K, HAS_V, EMIT_LOW32, 3>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                     status, n, shift, digit_mask, stream);
    case 4:
      if constexpr (Shapes<K>::count > 4)
        return launch_variant<K, HAS_V, EMIT_LOW32, 4>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                       status, n, shift, digit_mask, stream);
      return cudaErrorInvalidValue;
    case 5:
      if constexpr (Shapes<K>::count > 5)
        return launch_variant<K, HAS_V, EMIT_LOW32, 5>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                       status, n, shift, digit_mask, stream);
      return cudaErrorInvalidValue;
    case 6:
      if constexpr (Shapes<K>::count > 6)
        return launch_variant<K, HAS_V, EMIT_LOW32, 6>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                       status, n, shift, digit_mask, stream);
      return cudaErrorInvalidValue;
    default:
      return launch_variant<K, HAS_V, EMIT_LOW32, 0>(kin, kout, vin, vout, low32, ghist, lb, lb_next, counter,
                                                     status, n, shift, digit_mask, stream);
  }
}

// Runs every digit pass of [begin_bit, end_bit) over keys that start in
// (k0, v0); the workspace gives the other buffer (k1, v1).  The histograms in
// the workspace must already hold the counts of every pass in the variant's
// digit width (pass p at ghist + p * 2^bits), and ghist, the counters and
// look-back region 0 must be zero.  Returns through
// *result_in_first whether the sorted keys ended in (k0, v0).  `variant`
// selects the tile shape (it must be allowed for p.n); pass_events, when
// given, receive one record after each pass.
template <typename K, bool HAS_V>
inline cudaError_t run_passes(K* k0, uint32_t* v0, K* k1, uint32_t* v1, uint32_t* low32_last, const Plan& p,
                              unsigned char* ws, int begin_bit, int end_bit, cudaStream_t stream,
                              bool* result_in_first, int variant, cudaEvent_t* pass_events = nullptr) {
  if (!variant_allowed<K>(variant, p.n)) return cudaErrorInvalidValue;
  const uint32_t bits_v = variant_bits<K>(variant), radix = 1u << bits_v;
  const uint32_t passes = passes_for(begin_bit, end_bit, bits_v);
  const size_t tiles = ((size_t)p.n + variant_tile<K>(variant) - 1) / variant_tile<K>(variant);
  if (passes > p.passes || radix > p.radix || tiles * radix > p.lb_words) return cudaErrorInvalidValue;
  uint32_t* status = reinterpret_cast<uint32_t*>(ws);
  uint32_t* ghist = reinterpret_cast<uint32_t*>(ws + p.off_ghist);
  uint32_t* counters = reinterpret_cast<uint32_t*>(ws + p.off_counters);
  uint32_t* region[2] = {reinterpret_cast<uint32_t*>(ws + p.off_lookback),
                         reinterpret_cast<uint32_t*>(ws + p.off_lookback) + p.lb_words};
  K* src = k0;
  K* dst = k1;
  uint32_t* vs = v0;
  uint32_t* vd = v1;
  for (uint32_t pass = 0; pass < passes; ++pass) {
    uint32_t sh = (uint32_t)begin_bit + bits_v * pass;
    uint32_t bits = min(bits_v, (uint32_t)end_bit - sh);
    uint32_t mask = (1u << bits) - 1u;
    uint32_t* lb = region[pass & 1];
    uint32_t* lb_next = (pass + 1 < passes) ? region[(pass + 1) & 1] : nullptr;
    cudaError_t e;
    bool last = pass + 1 == passes;
    if (last && low32_last)
      e = launch_pass<K, HAS_V, true>(variant, src, dst, vs, vd, low32_last, ghist + pass * radix, lb, lb_next,
                                      counters + pass, status, p.n, sh, mask, stream);
    else
      e = launch_pass<K, HAS_V, false>(variant, src, dst, vs, vd, nullptr, ghist + pass * radix, lb, lb_next,
                                       counters + pass, status, p.n, sh, mask, stream);
    if (e != cudaSuccess) return e;
    if (pass_events && (e = cudaEventRecord(pass_events[pass], stream)) != cudaSuccess) return e;
    K* t = src;
    src = dst;
    dst = t;
    uint32_t* tv = vs;
    vs = vd;
    vd = tv;
  }
  *result_in_first = (src == k0);
  return cudaSuccess;
}

}  // namespace onesweep
}  // namespace bajo
