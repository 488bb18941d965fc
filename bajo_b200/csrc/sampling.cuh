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

// x^y for x in [0, 1] and y >= 0 (the metal lobe's powers), from two
// series evaluated with + - * / only, so the oracle's C gives the same bits:
//  - log2 x: x = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh s,
//    s = (m - 1) / (m + 1), |s| < 0.172, series 2 (s + s^3/3 + ... + s^9/9)
//    (truncation below 3e-9);
//  - 2^z: z = k + f with k = rint(z), |f| <= 1/2; e^(f ln 2) by its Taylor
//    series to the 7th power (truncation below 2e-9), scaled by 2^k.
// Relative error about 1e-6 against the exact power; 0^y = 0 (y > 0), x^0 = 1.
__device__ __forceinline__ float series_log2(float x) {
  const uint32_t bits = __float_as_uint(x);
  int e = (int)((bits >> 23) & 0xFFu) - 127;
  float m = __uint_as_float((bits & 0x007FFFFFu) | 0x3F800000u);
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  const float poly = 1.0f + s2 * (0.333333333f + s2 * (0.2f + s2 * (0.142857143f + s2 * 0.111111111f)));
  return (float)e + ((2.0f * s) * poly) * 1.44269504f;
}

__device__ __forceinline__ float series_exp2(float z) {
  if (z < -126.0f) return 0.0f;
  if (z > 127.0f) z = 127.0f;
  const float k = rintf(z);
  const float y = (z - k) * 0.693147181f;
  const float p =
      1.0f + y * (1.0f + y * (0.5f + y * (0.166666667f + y * (0.0416666667f + y * (0.00833333333f +
                                                                                  y * (0.00138888889f +
                                                                                       y * 0.000198412698f))))));
  return p * __uint_as_float((uint32_t)((int)k + 127) << 23);
}

__device__ __forceinline__ float series_pow(float x, float y) {
  if (y == 0.0f) return 1.0f;
  if (!(x >= 1.17549435e-38f)) return 0.0f;  // 0, subnormals and NaN
  return series_exp2(y * series_log2(x));
}

// reflect (bajo/rt/shading.mojo:227-232): v - (2 (v . n)) n
__device__ __forceinline__ f3 reflect(f3 v, f3 n) {
  const float k = 2.0f * dot(v, n);
  return mk(v.x - k * n.x, v.y - k * n.y, v.z - k * n.z);
}

struct BsdfSample {
  f3 dir, weight;
  float pdf;
  bool delta, ok;
};

// _sample_metal with _evaluate_metal (bajo/rt/shading.mojo:29-56,122-161):
// mirror reflection for fuzz <= 1e-4, otherwise a Phong-type lobe of exponent
// 2 / fuzz^2 - 2 around it (angles by sincos_turns, powers by series_pow)
__device__ __forceinline__ BsdfSample sample_metal(f3 d, f3 normal, f3 albedo, float fuzz, float u, float v) {
  BsdfSample r;
  const f3 reflected = normalize(reflect(normalize(d), normal));
  const bool smooth = fuzz <= 1.0e-4f;
  r.delta = smooth;
  if (smooth) {
    r.dir = reflected;
    r.weight = albedo;
    r.pdf = 1.0f;
    r.ok = dot(reflected, normal) > 0.0f;
    return r;
  }
  const float exponent = fmaxf(2.0f / (fuzz * fuzz) - 2.0f, 0.0f);
  const float cos_t = series_pow(u, 1.0f / (exponent + 1.0f));
  const float sin_t = sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f));
  float sp, cp;
  sincos_turns(v, sp, cp);
  const f3 helper = fabsf(reflected.y) > 0.99f ? mk(1.0f, 0.0f, 0.0f) : mk(0.0f, 1.0f, 0.0f);
  const f3 tangent = normalize(cross(helper, reflected));
  const f3 bitangent = cross(reflected, tangent);
  const f3 dir = normalize((tangent * (cp * sin_t) + bitangent * (sp * sin_t)) + reflected * cos_t);
  // evaluation at dir
  const f3 dn = normalize(dir);
  const bool surface_valid = dot(normal, dn) > 0.0f;
  const float lobe_cos = fmaxf(dot(reflected, dn), 0.0f);
  const float lobe = series_pow(lobe_cos, exponent);
  const bool valid = surface_valid && lobe_cos > 0.0f;
  const float value_scale = valid ? ((exponent + 2.0f) * lobe) / 6.28318531f : 0.0f;
  const float pdf = valid ? ((exponent + 1.0f) * lobe) / 6.28318531f : 0.0f;
  const float scos = fmaxf(dot(normal, dir), 0.0f);
  r.ok = pdf > 0.0f && scos > 0.0f;
  const float scale = scos / (r.ok ? pdf : 1.0f);
  r.dir = dir;
  r.weight = (albedo * value_scale) * scale;
  r.pdf = pdf;
  return r;
}

// _sample_dielectric (bajo/rt/shading.mojo:165-198) with refract and the
// Schlick reflectance (:235-258): reflect when refraction is impossible or
// with the reflectance's probability, else refract; weight 1
__device__ __forceinline__ BsdfSample sample_dielectric(f3 d, f3 normal, float ior, bool front, float u) {
  BsdfSample r;
  const float ri = front ? 1.0f / ior : ior;
  const f3 ud = normalize(d);
  const float cos_t = fminf(dot(mk(-ud.x, -ud.y, -ud.z), normal), 1.0f);
  const float sin_t = sqrtf(fmaxf(1.0f - cos_t * cos_t, 0.0f));
  const bool cannot = ri * sin_t > 1.0f;
  const float root = (1.0f - ri) / (1.0f + ri);
  const float r2 = root * root;
  const float x = 1.0f - cos_t;
  const float x2 = x * x;
  const float x5 = (x2 * x2) * x;
  const float refl = fmaf(1.0f - r2, x5, r2);
  const bool rs = cannot || refl > u;
  f3 out;
  if (rs) {
    out = reflect(ud, normal);
  } else {
    const float ct = fminf(dot(mk(-ud.x, -ud.y, -ud.z), normal), 1.0f);
    const f3 perp = mk(ri * (ud.x + ct * normal.x), ri * (ud.y + ct * normal.y), ri * (ud.z + ct * normal.z));
    const float par = -sqrtf(fabsf(1.0f - dot(perp, perp)));
    out = mk(perp.x + par * normal.x, perp.y + par * normal.y, perp.z + par * normal.z);
  }
  r.dir = normalize(out);
  r.weight = mk(1.0f, 1.0f, 1.0f);
  r.pdf = rs ? (cannot ? 1.0f : refl) : 1.0f - refl;
  r.delta = true;
  r.ok = true;
  return r;
}

}  // namespace smp
}  // namespace bajo
