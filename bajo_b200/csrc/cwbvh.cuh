// cwbvh.cuh -- the device walk of the compressed 8-wide BVH (CWBVH8): shared
// by its closest-hit / any-hit entry points (cwbvh.cu) and the wavefront path
// tracer's CWBVH8 policy (rt.cu).  See cwbvh.cu for the restated reference.
#pragma once

#include "traverse.cuh"

namespace bajo {
namespace cw {

constexpr int kBlock = 128;
constexpr int kStack = 64;  // node groups; one per level of the wide tree at most

struct Tree {
  const float4* nodes;
  const float4* tris;
  uint32_t n_nodes;  // bound on node references and visits
  uint32_t n_tris;   // bound on triangle references
};

struct Hit {
  float t, u, v;
  uint32_t prim, tri;
};

// byte b of w as an exact float: 2^23 + q (one byte permute) minus 2^23
__device__ __forceinline__ float qbyte(uint32_t w, int b) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + b)) - 8388608.0f;
}

template <bool ANY>
__device__ __forceinline__ Hit trace(f3 o, f3 d, float tmin, float tmax, const Tree& tr, uint32_t* status) {
  Hit h;
  h.t = tmax;
  h.u = h.v = 0.0f;
  h.prim = kEmpty;
  h.tri = kEmpty;
  if (tr.n_nodes == 0) return h;
  const f3 rcp = mk(trav::rcp1(d.x), trav::rcp1(d.y), trav::rcp1(d.z));
  const bool negx = d.x < 0.0f, negy = d.y < 0.0f, negz = d.z < 0.0f;
  const uint32_t oi = 7u - ((negx ? 4u : 0u) | (negy ? 2u : 0u) | (negz ? 1u : 0u));
  uint2 stack[kStack];
  int sp = 0;
  uint32_t nbase = 0, nmask = 0x80000000u, tbase = 0, tmask = 0, visits = 0;
  // a corrupt tree ends the walk; the status bit is raised after the loop,
  // which keeps the atomic out of the loop's code
  uint32_t fail = 0;
  for (;;) {
    if (nmask > 0x00FFFFFFu) {
      const uint32_t gm = nmask;
      const int bit = 31 - __clz(nmask);
      nmask &= ~(1u << bit);
      if (nmask > 0x00FFFFFFu) {
        if (sp >= kStack) {
          fail = BAJO_STATUS_STACK_OVERFLOW;
          break;
        }
        stack[sp++] = make_uint2(nbase, nmask);
      }
      const uint32_t slot = ((uint32_t)bit - 24u) ^ oi;
      const uint32_t ni = nbase + (uint32_t)__popc(gm & ((1u << slot) - 1u));
      if (ni >= tr.n_nodes || ++visits > tr.n_nodes) {
        fail = BAJO_STATUS_BAD_TOPOLOGY;
        break;
      }
      const float4* nd = tr.nodes + (size_t)ni * 5;
      const float4 n0 = __ldg(nd + 0), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3),
                   n4 = __ldg(nd + 4);
      const uint32_t ei = __float_as_uint(n0.w);
      const float idx = __uint_as_float((ei & 0xFFu) << 23) * rcp.x;
      const float idy = __uint_as_float(((ei >> 8) & 0xFFu) << 23) * rcp.y;
      const float idz = __uint_as_float(((ei >> 16) & 0xFFu) << 23) * rcp.z;
      const float ox = (n0.x - o.x) * rcp.x, oy = (n0.y - o.y) * rcp.y, oz = (n0.z - o.z) * rcp.z;
      const uint32_t imask = ei >> 24;
      const float tlim = ANY ? tmax : h.t;
      // near / far planes per axis, by the ray's direction sign
      const uint32_t q[12] = {__float_as_uint(n2.x), __float_as_uint(n2.y), __float_as_uint(n2.z),
                              __float_as_uint(n2.w), __float_as_uint(n3.x), __float_as_uint(n3.y),
                              __float_as_uint(n3.z), __float_as_uint(n3.w), __float_as_uint(n4.x),
                              __float_as_uint(n4.y), __float_as_uint(n4.z), __float_as_uint(n4.w)};
      const uint32_t meta[2] = {__float_as_uint(n1.z), __float_as_uint(n1.w)};
      uint32_t hm = 0;
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        // four lanes at once: bit position (low 5 bits, XOR the inverted
        // octant on internal lanes) and child bits (top 3 bits) of each byte
        const uint32_t inner = ((((imask >> (4 * g)) & 0xFu) * 0x00204081u) & 0x01010101u) * oi;
        const uint32_t bit4 = (meta[g] ^ inner) & 0x1F1F1F1Fu, kids4 = (meta[g] >> 5) & 0x07070707u;
        const uint32_t nxw = negx ? q[6 + g] : q[0 + g], fxw = negx ? q[0 + g] : q[6 + g];
        const uint32_t nyw = negy ? q[8 + g] : q[2 + g], fyw = negy ? q[2 + g] : q[8 + g];
        const uint32_t nzw = negz ? q[10 + g] : q[4 + g], fzw = negz ? q[4 + g] : q[10 + g];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const float tnx = __fmaf_rn(qbyte(nxw, b), idx, ox), tfx = __fmaf_rn(qbyte(fxw, b), idx, ox);
          const float tny = __fmaf_rn(qbyte(nyw, b), idy, oy), tfy = __fmaf_rn(qbyte(fyw, b), idy, oy);
          const float tnz = __fmaf_rn(qbyte(nzw, b), idz, oz), tfz = __fmaf_rn(qbyte(fzw, b), idz, oz);
          const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
          const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tlim));
          if (tn <= tf) hm |= __byte_perm(kids4, 0u, 0x4440u + b) << __byte_perm(bit4, 0u, 0x4440u + b);
        }
      }
      nbase = __float_as_uint(n1.x);
      nmask = (hm & 0xFF000000u) | imask;
      tbase = __float_as_uint(n1.y);
      tmask = hm & 0x00FFFFFFu;
    } else {
      tbase = nbase;
      tmask = nmask;
      nmask = 0;
    }
    while (tmask != 0u) {
      const int bit = 31 - __clz(tmask);
      tmask &= ~(1u << bit);
      const uint32_t ti = tbase + (uint32_t)bit;
      if (ti >= tr.n_tris) {
        fail = BAJO_STATUS_BAD_TOPOLOGY;
        break;
      }
      const float4* rec = tr.tris + (size_t)ti * 3;
      const float4 a = __ldg(rec + 0), b = __ldg(rec + 1), c = __ldg(rec + 2);
      const f3 e1 = mk(a.x, a.y, a.z), e2 = mk(b.x, b.y, b.z);
      const f3 p = cross(d, e2);
      const float det = dot(e1, p);
      const bool pos = det >= 0.0f;
      const float ad = pos ? det : -det;
      const f3 tv = o - mk(c.x, c.y, c.z);
      const float un = dot(tv, p);
      const f3 qv = cross(tv, e1);
      const float vn = dot(d, qv), tn = dot(e2, qv);
      const float us = pos ? un : -un, vs = pos ? vn : -vn, ts = pos ? tn : -tn;
      if (!(ad > 1e-8f && us >= 0.0f && us <= ad && vs >= 0.0f && (us + vs) <= ad && ts > tmin * ad &&
            ts < h.t * ad))
        continue;
      if (ANY) {
        h.t = 0.0f;
        return h;
      }
      const float inv = 1.0f / ad;
      h.t = ts * inv;
      h.u = us * inv;
      h.v = vs * inv;
      h.prim = __float_as_uint(c.w);
      h.tri = ti;
    }
    if (fail) break;
    if (nmask <= 0x00FFFFFFu) {
      if (sp == 0) break;
      --sp;
      nbase = stack[sp].x;
      nmask = stack[sp].y;
    }
  }
  if (fail) raise_status(status, fail);
  return h;
}

}  // namespace cw
}  // namespace bajo
