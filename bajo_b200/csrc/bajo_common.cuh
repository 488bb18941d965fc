// bajo_common.cuh -- shared device helpers for the sm_100a LBVH / traversal
// library.  The float helpers restate bajo/core/vec.mojo with the same
// rounding: this library is compiled with -fmad=false, so a product followed
// by a sum is rounded twice unless fmaf() is spelled out, exactly where the
// reference spells fma() (bajo/core/vec.mojo:440, :523-525).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cfloat>

#include "../../include/bajo_b200.h"

namespace bajo {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;   // LBVH_SENTINEL, bajo/bvh/constants.mojo:6
constexpr uint32_t kLeafFlag = 0x80000000u;   // _BVH_LEAF_FLAG, bajo/bvh/tagged_ref.mojo:3
constexpr uint32_t kIndexMask = 0x7FFFFFFFu;  // _BVH_INDEX_MASK, tagged_ref.mojo:4
constexpr uint32_t kEmpty = 0xFFFFFFFFu;      // EMPTY_LANE / MISS_PRIM, constants.mojo:19-20
// Slack on the far slab distance (t_near <= t_far * (1 + 2^-20)): keeps the
// closest hit independent of the traversal order.  Same constant in the oracle.
constexpr float kSlack = 1.00000095367431640625f;

struct f3 {
  float x, y, z;
};

__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return mk(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return mk(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
// dot = fma(a.x, b.x, fma(a.y, b.y, a.z * b.z))   (vec.mojo:440)
__device__ __forceinline__ float dot(f3 a, f3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
// vec.mojo:522-526
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return mk(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}
// vec.mojo:529-539
__device__ __forceinline__ f3 normalize(f3 v) {
  float l = sqrtf(dot(v, v));
  float inv_l = (l > 1.0e-20f) ? 1.0f / l : 0.0f;
  return v * inv_l;
}
// vec.mojo:373-394
__device__ __forceinline__ float safe_inv1(float e) { return (fabsf(e) > 1.0e-20f) ? 1.0f / e : 0.0f; }
__device__ __forceinline__ float comp(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Order-preserving float <-> uint32 map, so that exact float min/max
// reductions can use integer atomics.
__device__ __forceinline__ uint32_t float_to_ordered(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u) {
  uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
  return __uint_as_float(b);
}

// core/morton.mojo:48-58
__device__ __forceinline__ uint32_t expand_bits_3d(uint32_t n) {
  n = (n ^ (n << 16)) & 0xFF0000FFu;
  n = (n ^ (n << 8)) & 0x0300F00Fu;
  n = (n ^ (n << 4)) & 0x030C30C3u;
  n = (n ^ (n << 2)) & 0x09249249u;
  return n;
}
// float -> u32 truncation clamped to [0, 1023]   (core/morton.mojo:78)
__device__ __forceinline__ uint32_t quantize1024(float c) {
  uint32_t u = __float2uint_rz(c * 1024.0f);  // saturates: negatives/NaN -> 0
  return u > 1023u ? 1023u : u;
}
// core/morton.mojo:61-89
__device__ __forceinline__ uint32_t morton3(float x, float y, float z) {
  return (expand_bits_3d(quantize1024(z)) << 2) | (expand_bits_3d(quantize1024(y)) << 1) |
         expand_bits_3d(quantize1024(x));
}

// binary_layout.mojo:116-125: segment containing item (offsets has n_off
// entries, the last one is the total).
__device__ __forceinline__ uint32_t segment_for_item(const uint32_t* __restrict__ off, uint32_t n_off,
                                                     uint32_t item) {
  uint32_t lo = 0, hi = n_off - 1;
  while (lo + 1 < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (item < __ldg(off + mid)) hi = mid;
    else lo = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t lane_id() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Fetch-add with acquire-release semantics at GPU scope: the writes before it
// are visible to whoever reads its result, and the writes released by an
// earlier atomic whose value it reads are visible after it.
__device__ __forceinline__ uint32_t atomic_add_acq_rel_gpu(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ uint32_t atomic_add_acquire_gpu(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.add.acquire.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
// Release / acquire fence among the threads of one CTA (the message-passing
// pattern of a shared-memory arrival counter: data, fence, counter on one
// side; counter, fence, data on the other).  Lighter than the sequentially
// consistent fence that __threadfence_block() issues.
__device__ __forceinline__ void fence_acq_rel_cta() { asm volatile("fence.acq_rel.cta;" ::: "memory"); }

__device__ __forceinline__ void red_add_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float2 ld_relaxed_gpu_f2(const float* p) {
  float2 v;
  asm volatile("ld.relaxed.gpu.global.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_gpu_f2(float* p, float x, float y) {
  asm volatile("st.relaxed.gpu.global.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(x), "f"(y) : "memory");
}
__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded wait for a flag another thread publishes: spins with acquire loads
// until any of `bits` is set in *p, for at most limit_ns (global timer).
// Returns false when the limit ran out; the caller then reports a status and
// returns instead of waiting further.  Every wait on another thread's flag in
// this library goes through a bound like this one.
__device__ __forceinline__ bool wait_bits_acquire(const uint32_t* p, uint32_t bits, uint64_t limit_ns) {
  if (ld_acquire_gpu(p) & bits) return true;
  const uint64_t t0 = global_timer_ns();
  while (!(ld_acquire_gpu(p) & bits))
    if (global_timer_ns() - t0 > limit_ns) return false;
  return true;
}

// Device status word bits (read back by bajo_workspace_status).
__device__ __forceinline__ void raise_status(uint32_t* status, uint32_t bit) {
  if (status) atomicOr(status, bit);
}

}  // namespace bajo
