// sampling.cuh -- random streams and direction sampling shared by the path
// tracer and the batched trace.
//
// Random numbers: every (path, stage) pair owns a Philox-4x32-10 stream
// (Salmon et al., SC'11) keyed by the seed with counter (0, 0, stage,
// path_id) -- the reference's (path_id << 32) | stage subsequence
// (bajo/rt/wavefront_contract.mojo:107-133); each stage uses at most the four
// floats of its first block.  Angles use sincos_turns, a polynomial the
// oracle restates operation for operation, so results are bit-identical.
#pragma once

#include "bajo_common.cuh"

namespace bajo {
namespace smp {

// stage domains (wavefront_contract.mojo:32-133)
__device__ __forceinline__ uint32_t stage_bsdf(uint32_t b) { return (0u << 30) | (b + 1); }
__device__ __forceinline__ uint32_t stage_roulette(uint32_t b) { return (1u << 30) | (b + 1); }
__device__ __forceinline__ uint32_t stage_light(uint32_t b) { return (2u << 30) | (b + 1); }

// Philox-4x32-10: 10 rounds of the multiply-xor bijection with Weyl key bumps.
__device__ __forceinline__ float4 uniform4(uint64_t seed, uint32_t path_id, uint32_t stage) {
  uint32_t c0 = 0, c1 = 0, c2 = stage, c3 = path_id;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  const float s = 1.0f / 16777216.0f;  // 24-bit uniforms in [0, 1)
  return make_float4((float)(c0 >> 8) * s, (float)(c1 >> 8) * s, (float)(c2 >> 8) * s, (float)(c3 >> 8) * s);
}

// sin and cos of 2*pi*u for u in [0, 1): reduce to the nearest quarter turn,
// evaluate the Taylor series of sin and cos on |a| <= pi/4 (terms to a^9 and
// a^10, truncation below 2e-9), rotate by the quadrant.
__device__ __forceinline__ void sincos_turns(float u, float& s_out, float& c_out) {
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
  if (q == 0) { s_out = s; c_out = c; }
  else if (q == 1) { s_out = c; c_out = -s; }
  else if (q == 2) { s_out = -s; c_out = -c; }
  else { s_out = -c; c_out = s; }
}

// Lambertian direction (_sample_lambertian, bajo/rt/shading.mojo:92-118):
// normal + a uniform point on the unit sphere, normalised; the normal itself
// when the sum is (near) zero.
__device__ __forceinline__ f3 lambertian_dir(f3 normal, float u, float v) {
  float st, ct;
  sincos_turns(u, st, ct);
  const float z = 1.0f - 2.0f * v;
  const float rad = sqrtf(fmaxf(1.0f - z * z, 0.0f));
  f3 sd = normal + mk(rad * ct, rad * st, z);
  if (fabsf(sd.x) < 1.0e-8f && fabsf(sd.y) < 1.0e-8f && fabsf(sd.z) < 1.0e-8f) sd = normal;
  return normalize(sd);
}

}  // namespace smp
}  // namespace bajo
