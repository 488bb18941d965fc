// mlp.cuh -- device pieces of the path-guiding network shared by the MLP
// kernels (mlp.cu) and the guided wavefront shading kernel (rt.cu).
//
// Network: features (64) = one-blob(position, 3 x 16 bins) ++ one-blob(normal,
// octahedral coordinates, 2 x 8 bins); three hidden layers of 64 with ReLU;
// output 20 = 4 lobes x (mean xyz, log kappa, weight logit).
// Parameter layout (floats / halves): W1[64x64] b1[64] W2 b2 W3 b3 W4[32x64]
// b4[32] (rows 20..31 of W4 and b4 are zero), weights row-major [out][in].
//
// Dense layers run on the 5th-generation tensor cores (namespace tc below:
// tcgen05.mma with FP32 accumulators in tensor memory) in the guided shading,
// the batched forward of bajo_mlp_forward_tc and the training gradient.  The
// warp-level mma.sync m16n8k16 kernels (f16 inputs, f32 accumulation) remain
// as bajo_mlp_forward / bajo_mlp_grad, the comparison for the tcgen05 ones.
// mma.sync fragment layouts (PTX ISA), g = lane / 4, t = lane % 4:
//   A (16x16): a0a1 = (g, 2t..2t+1), a2a3 = (g+8, 2t..), a4a5 = (g, 2t+8..),
//              a6a7 = (g+8, 2t+8..)
//   B (16x8):  b0b1 = (k 2t..2t+1, n g), b2b3 = (k 2t+8.., n g)
//   C (16x8):  c0c1 = (g, 2t..2t+1), c2c3 = (g+8, 2t..2t+1)
// The C fragments of n-tiles 2j and 2j+1 are exactly the A fragment of k-tile
// j, so a layer's output feeds the next layer without leaving registers.
#pragma once

#include <cuda_fp16.h>

#include "bajo_common.cuh"

namespace bajo {
namespace mlp {

constexpr int kIn = 64, kHid = 64, kOut = 20, kOutPad = 32, kLobes = 4;
constexpr int kLayerSize = kHid * kIn + kHid;  // 4160
__host__ __device__ constexpr int kOffW(int l) { return l * kLayerSize; }
__host__ __device__ constexpr int kOffB(int l) {
  return l < 3 ? l * kLayerSize + kHid * kIn : 3 * kLayerSize + kOutPad * kHid;
}
constexpr int kParams = 3 * kLayerSize + kOutPad * kHid + kOutPad;  // 14560
constexpr int kPosBins = 16, kDirBins = 8;
constexpr float kPi = 3.14159265358979323846f;
constexpr float kLogKappaMin = -2.0f, kLogKappaMax = 8.0f;

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
  __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}
// saturating pack for gradients: FP16 overflows at 65504
__device__ __forceinline__ uint32_t pack_h2_sat(float lo, float hi) {
  const float m = 65000.0f;
  return pack_h2(fminf(fmaxf(lo, -m), m), fminf(fmaxf(hi, -m), m));
}
__device__ __forceinline__ uint32_t ld32(const __half* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ void st32(__half* p, uint32_t v) { *reinterpret_cast<uint32_t*>(p) = v; }

// ---------------------------------------------------------------------------
// encoding
// ---------------------------------------------------------------------------
// One-blob encoding (Mueller et al., "Neural Importance Sampling", 2019) with a
// hat kernel one bin wide: v in [0, 1] lands on the two nearest bin centres
// with linear weights; bin value k of the blob.
__device__ __forceinline__ void blob_bins(float v, int bins, int& i0, int& i1, float& f) {
  v = fminf(fmaxf(v, 0.0f), 1.0f);
  const float s = v * (float)bins - 0.5f;
  const float fl = floorf(s);
  f = s - fl;
  i0 = max((int)fl, 0);
  i1 = min((int)fl + 1, bins - 1);
}
__device__ __forceinline__ float blob_value(int k, int i0, int i1, float f) {
  return (k == i0 ? 1.0f - f : 0.0f) + (k == i1 ? f : 0.0f);
}

// octahedral coordinates of a unit normal in [0, 1]^2 (no transcendentals)
__device__ __forceinline__ void octahedral(float nx, float ny, float nz, float& u, float& v) {
  const float l1 = fabsf(nx) + fabsf(ny) + fabsf(nz);
  float x = l1 > 0.0f ? nx / l1 : 0.0f, y = l1 > 0.0f ? ny / l1 : 0.0f;
  if (nz < 0.0f) {
    const float ax = fabsf(x), ay = fabsf(y);
    x = (1.0f - ay) * (x >= 0.0f ? 1.0f : -1.0f);
    y = (1.0f - ax) * (y >= 0.0f ? 1.0f : -1.0f);
  }
  u = x * 0.5f + 0.5f;
  v = y * 0.5f + 0.5f;
}

// Encoding group `grp` (0..2 position axes, 3..4 normal coordinates) of one
// sample, written as half pairs into its 64-feature row.
__device__ __forceinline__ void encode_group(int grp, const float* p, const float* n, const float* box,
                                             __half* row) {
  float v;
  int bins, col;
  if (grp < 3) {
    const float ext = box[3 + grp] - box[grp];
    v = ext > 0.0f ? (p[grp] - box[grp]) / ext : 0.5f;
    bins = kPosBins;
    col = grp * kPosBins;
  } else {
    float u, w;
    octahedral(n[0], n[1], n[2], u, w);
    v = grp == 3 ? u : w;
    bins = kDirBins;
    col = 3 * kPosBins + (grp - 3) * kDirBins;
  }
  int i0, i1;
  float f;
  blob_bins(v, bins, i0, i1, f);
  for (int k = 0; k < bins; k += 2) st32(row + col + k, pack_h2(blob_value(k, i0, i1, f), blob_value(k + 1, i0, i1, f)));
}

// every group of one sample's row
__device__ __forceinline__ void encode_row(const float* p, const float* n, const float* box, __half* row) {
#pragma unroll 1
  for (int grp = 0; grp < 5; ++grp) encode_group(grp, p, n, box, row);
}

// ---------------------------------------------------------------------------
// network in shared memory and the per-warp forward pass
// ---------------------------------------------------------------------------
// Shared-memory row strides: 64-wide FP16 tiles use 72 halves (144 B), so the
// 8 rows a fragment load touches fall in distinct banks (a 128-byte stride
// would put all 8 in one bank); 32-wide FP16 tiles use 40 halves; FP32
// output tiles 36 floats.
constexpr int kLd = 72, kLd32 = 40, kOutLd = 36;

struct Net {
  __half W[3][kHid * kLd];    // hidden layers, [out][in]
  __half W4[kOutPad * kLd];   // output layer, [out][in]
  float B[3][kHid];
  float B4[kOutPad];
};

template <int THREADS>
__device__ void load_net(Net& s, const __half* __restrict__ p16) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(p16);
  for (int i = threadIdx.x; i < kHid * kIn / 2; i += THREADS) {
    const int dst = (i >> 5) * (kLd / 2) + (i & 31);  // 32 words per source row
    for (int l = 0; l < 3; ++l) reinterpret_cast<uint32_t*>(s.W[l])[dst] = src[kOffW(l) / 2 + i];
  }
  for (int i = threadIdx.x; i < kOutPad * kHid / 2; i += THREADS)
    reinterpret_cast<uint32_t*>(s.W4)[(i >> 5) * (kLd / 2) + (i & 31)] = src[kOffW(3) / 2 + i];
  for (int i = threadIdx.x; i < kHid; i += THREADS)
    for (int l = 0; l < 3; ++l) s.B[l][i] = __half2float(p16[kOffB(l) + i]);
  for (int i = threadIdx.x; i < kOutPad; i += THREADS) s.B4[i] = __half2float(p16[kOffB(3) + i]);
}

// A fragments (4 k-tiles of 16) of the 16 rows from row0 of a [rows x kLd] tile
__device__ __forceinline__ void load_afrag64(const __half* t, int row0, uint32_t a[4][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const int c = 16 * kt + 2 * tq;
    a[kt][0] = ld32(t + (row0 + g) * kLd + c);
    a[kt][1] = ld32(t + (row0 + g + 8) * kLd + c);
    a[kt][2] = ld32(t + (row0 + g) * kLd + c + 8);
    a[kt][3] = ld32(t + (row0 + g + 8) * kLd + c + 8);
  }
}

__device__ __forceinline__ void store_afrag64(__half* t, int row0, const uint32_t a[4][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const int c = 16 * kt + 2 * tq;
    st32(t + (row0 + g) * kLd + c, a[kt][0]);
    st32(t + (row0 + g + 8) * kLd + c, a[kt][1]);
    st32(t + (row0 + g) * kLd + c + 8, a[kt][2]);
    st32(t + (row0 + g + 8) * kLd + c + 8, a[kt][3]);
  }
}

// one dense layer on MT m-tiles of 16 rows: acc[m][n-tile] = A x W^T + b,
// W [out][in] with row stride kLd; each B fragment is loaded once for all
// m-tiles
template <int MT, int NT>
__device__ __forceinline__ void dense(const uint32_t a[MT][4][4], const __half* W, const float* bias,
                                      float acc[MT][NT][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const float b0 = bias[8 * j + 2 * tq], b1 = bias[8 * j + 2 * tq + 1];
#pragma unroll
    for (int m = 0; m < MT; ++m) {
      acc[m][j][0] = b0;
      acc[m][j][1] = b1;
      acc[m][j][2] = b0;
      acc[m][j][3] = b1;
    }
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      uint32_t b[2];
      const __half* w = W + (8 * j + g) * kLd + 16 * kt + 2 * tq;
      b[0] = ld32(w);
      b[1] = ld32(w + 8);
#pragma unroll
      for (int m = 0; m < MT; ++m) mma16816(acc[m][j], a[m][kt], b);
    }
  }
}

// ReLU on the C fragments of 8 n-tiles, repacked as the 4 A k-tiles
__device__ __forceinline__ void relu_to_afrag(const float acc[8][4], uint32_t a[4][4]) {
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const float* lo = acc[2 * kt];
    const float* hi = acc[2 * kt + 1];
    a[kt][0] = pack_h2(fmaxf(lo[0], 0.0f), fmaxf(lo[1], 0.0f));
    a[kt][1] = pack_h2(fmaxf(lo[2], 0.0f), fmaxf(lo[3], 0.0f));
    a[kt][2] = pack_h2(fmaxf(hi[0], 0.0f), fmaxf(hi[1], 0.0f));
    a[kt][3] = pack_h2(fmaxf(hi[2], 0.0f), fmaxf(hi[3], 0.0f));
  }
}

// Forward of MT m-tiles (rows row0 .. row0 + 16 MT - 1) of the feature tile
// `x` ([rows x kLd]); hidden activations go to keep[0..2] (same layout) when
// keep is non-null; the 32 padded outputs to out[row * kOutLd + c].
template <int MT>
__device__ __forceinline__ void forward_tile(const Net& s, const __half* x, int row0, __half* const* keep,
                                             float* out) {
  uint32_t a[MT][4][4];
  float acc[MT][8][4];
#pragma unroll
  for (int m = 0; m < MT; ++m) load_afrag64(x, row0 + 16 * m, a[m]);
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    dense<MT, 8>(a, s.W[l], s.B[l], acc);
#pragma unroll
    for (int m = 0; m < MT; ++m) {
      relu_to_afrag(acc[m], a[m]);
      if (keep) store_afrag64(keep[l], row0 + 16 * m, a[m]);
    }
  }
  float o[MT][4][4];
  dense<MT, 4>(a, s.W4, s.B4, o);
  const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = 8 * j + 2 * tq, r = row0 + 16 * m + g;
      *reinterpret_cast<float2*>(&out[r * kOutLd + c]) = make_float2(o[m][j][0], o[m][j][1]);
      *reinterpret_cast<float2*>(&out[(r + 8) * kOutLd + c]) = make_float2(o[m][j][2], o[m][j][3]);
    }
}

// Per-warp working set of the warp-autonomous forward: 32 feature rows and
// their 32 outputs.  A warp encodes, evaluates and consumes its own rows, so
// no block-wide barrier is needed after the weights are loaded.
struct WarpTile {
  __half x[32 * kLd];
  float out[32 * kOutLd];
};

// ---------------------------------------------------------------------------
// The network on the 5th-generation tensor cores (tcgen05), used by the
// batched forward (mlp.cu) and the guided shading kernel (rt.cu).  NT tiles of
// 128 rows per CTA of 128 NT threads: thread t owns row t % 128 of tile t /
// 128.  Each layer is five tcgen05.mma per tile (kind::f16, M = 128, N = 64 or
// 32, K = 16; FP16 operands in shared memory, FP32 accumulator in tensor
// memory) issued by thread 0 and committed to one mbarrier; then every warp
// reads its 32 accumulator lanes (tcgen05.ld 32x32b), applies ReLU while it
// packs to FP16 (cvt.rn.relu.f16x2.f32) and writes the next layer's operand
// in place.  The biases ride in the MMA: every operand row carries a
// constant 1 in column 64 (columns 65-79 zero) and every weight row its bias
// there, so K = 80 and the epilogue adds nothing (the biases are FP16 values,
// so 1 x bias is exact in the FP32 sum).  Operands use the canonical
// interleaved (no swizzle) K-major layout: 8 x 8 core matrices of 128 bytes,
// the 10 cores of one 8-row group side by side along K, so the leading (K)
// byte offset is 128 and the stride (8-row) byte offset 1,280.
// ---------------------------------------------------------------------------
namespace tc {

constexpr int kRows = 128;
constexpr int kK = 80;                          // 64 inputs, the constant 1, zero padding
constexpr int kKCores = kK / 8;                 // core matrices along K
constexpr uint32_t kTileBytes = kRows * kK * 2;  // one operand tile
constexpr uint32_t kColsPerTile = 64;           // one layer's FP32 accumulator (N <= 64)
constexpr uint64_t kWaitNs = 200ull * 1000ull * 1000ull;

// byte offset of element (r, k) of an [rows][kK] FP16 operand in core layout
__device__ __forceinline__ uint32_t core_off(int r, int k) {
  return (uint32_t)(((r >> 3) * kKCores + (k >> 3)) * 128 + ((r & 7) << 4) + ((k & 7) << 1));
}
// shared-memory matrix descriptor: start >> 4, leading byte offset 128 >> 4,
// stride byte offset (kKCores x 128) >> 4, descriptor version 1 (bit 46), no
// swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)((kKCores * 128u) >> 4) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B FP16
// (bits 7-12 = 0), both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at
// bit 24
__host__ __device__ constexpr uint32_t instr_desc(uint32_t n) {
  return (1u << 4) | ((n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {  // at most kWaitNs
  if (bar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (!bar_try_wait(bar, parity))
    if (global_timer_ns() - t0 > kWaitNs) return false;
  return true;
}
// 32 consecutive FP32 accumulator columns of this thread's lane, waited for
// in the same statement (so no use of r can be scheduled before the wait)
__device__ __forceinline__ void tmem_ld32_wait(uint32_t taddr, uint32_t r[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory, before the tensor cores read them
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// max(lo, 0) and max(hi, 0) rounded to FP16 and packed (lo in the low half)
__device__ __forceinline__ uint32_t relu_pack(uint32_t lo, uint32_t hi) {
  uint32_t d;
  asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(d) : "r"(hi), "r"(lo));
  return d;
}

// The network's weights in core layout, each row's bias in column 64.
struct __align__(128) Weights {
  __half w[3][kHid * kK];   // hidden layers [out][in | bias | 0]
  __half w4[kOutPad * kK];  // output layer
};

template <int THREADS>
__device__ void load_weights(Weights& s, const __half* __restrict__ p16) {
  if ((reinterpret_cast<uintptr_t>(p16) & 15u) == 0) {
    // 16-byte chunks: 8 inputs of a row, the (bias, 0 x 7) chunk or zeros;
    // every layer's rows start on 16 bytes (4160 halves apart, rows of 64)
    constexpr int kChunks = kK / 8, kHidden = 3 * kHid * kChunks, kTotal = kHidden + kOutPad * kChunks;
    const uint4* src = reinterpret_cast<const uint4*>(p16);
#pragma unroll 4
    for (int c = threadIdx.x; c < kTotal; c += THREADS) {
      const int l = c < kHidden ? c / (kHid * kChunks) : 3;
      const int rc = c < kHidden ? c % (kHid * kChunks) : c - kHidden;
      const int o = rc / kChunks, kg = rc % kChunks;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (kg < kIn / 8) v = src[(kOffW(l) + o * kIn) / 8 + kg];
      else if (kg == kIn / 8) v.x = (uint32_t)__half_as_ushort(p16[kOffB(l) + o]);
      unsigned char* dst = reinterpret_cast<unsigned char*>(l < 3 ? s.w[l] : s.w4);
      *reinterpret_cast<uint4*>(dst + core_off(o, 8 * kg)) = v;
    }
    return;
  }
  const uint32_t* src = reinterpret_cast<const uint32_t*>(p16);
  for (int i = threadIdx.x; i < kHid * kK / 2; i += THREADS) {
    const int o = (2 * i) / kK, k = (2 * i) % kK;  // pairs (k, k + 1) of row o
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      uint32_t v;
      if (k < kIn) v = src[(kOffW(l) + o * kIn + k) / 2];
      else if (k == kIn) v = (uint32_t)__half_as_ushort(p16[kOffB(l) + o]);  // (bias, 0)
      else v = 0u;
      *reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(s.w[l]) + core_off(o, k)) = v;
    }
  }
  for (int i = threadIdx.x; i < kOutPad * kK / 2; i += THREADS) {
    const int o = (2 * i) / kK, k = (2 * i) % kK;
    uint32_t v;
    if (k < kIn) v = src[(kOffW(3) + o * kIn + k) / 2];
    else if (k == kIn) v = (uint32_t)__half_as_ushort(p16[kOffB(3) + o]);
    else v = 0u;
    *reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(s.w4) + core_off(o, k)) = v;
  }
}

// The 64 one-blob features of one sample as 32 FP16 pairs.
__device__ __forceinline__ void encode_pairs(const float* p, const float* n, const float* box, uint32_t f[32]) {
#pragma unroll
  for (int grp = 0; grp < 5; ++grp) {
    float v;
    int bins, col;
    if (grp < 3) {
      const float ext = box[3 + grp] - box[grp];
      v = ext > 0.0f ? (p[grp] - box[grp]) / ext : 0.5f;
      bins = kPosBins;
      col = grp * kPosBins;
    } else {
      float u, w;
      octahedral(n[0], n[1], n[2], u, w);
      v = grp == 3 ? u : w;
      bins = kDirBins;
      col = 3 * kPosBins + (grp - 3) * kDirBins;
    }
    int i0, i1;
    float fr;
    blob_bins(v, bins, i0, i1, fr);
#pragma unroll
    for (int k = 0; k < kPosBins; k += 2)
      if (k < bins) f[(col + k) >> 1] = pack_h2(blob_value(k, i0, i1, fr), blob_value(k + 1, i0, i1, fr));
  }
}
// row r's features into a tile in core layout (one 16-byte store per 8),
// with the constant 1 in column 64 and zeros up to 79
__device__ __forceinline__ void store_features(unsigned char* tile, int r, const uint32_t f[32]) {
#pragma unroll
  for (int q = 0; q < 8; ++q)
    *reinterpret_cast<uint4*>(tile + core_off(r, 8 * q)) = make_uint4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
  *reinterpret_cast<uint4*>(tile + core_off(r, kIn)) = make_uint4(0x3C00u, 0u, 0u, 0u);  // FP16 1.0, zeros
  *reinterpret_cast<uint4*>(tile + core_off(r, kIn + 8)) = make_uint4(0u, 0u, 0u, 0u);
}

// Prologue of a CTA: the mbarrier (count 1) and `cols` tensor-memory columns
// (a power of two from 32 to 512; warp 0 allocates); returns their address.
// Every thread must call it.
__device__ __forceinline__ uint32_t setup_cols(uint32_t bar, uint32_t* s_tmem, uint32_t cols) {
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(s_tmem)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  return *s_tmem;
}
// Epilogue: frees the columns once no thread reads them.  Every thread must call it.
__device__ __forceinline__ void teardown_cols(uint32_t tmem, uint32_t cols) {
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}
// NT tiles of 128 rows: NT x 64 columns
template <int NT>
__device__ __forceinline__ uint32_t setup(uint32_t bar, uint32_t* s_tmem) {
  return setup_cols(bar, s_tmem, NT * kColsPerTile);
}
template <int NT>
__device__ __forceinline__ void teardown(uint32_t tmem) {
  teardown_cols(tmem, NT * kColsPerTile);
}

// The network on the NT tiles at `act` (kTileBytes apart, features already
// written by their row threads); the calling thread's row's 20 outputs land
// in `out`.  Every thread must call it; false (in every thread) when the
// tensor cores never signalled completion (status bit raised, the launch
// should stop).
template <int NT>
__device__ __forceinline__ bool forward(const Weights& w, unsigned char* act, uint32_t tmem, uint32_t bar,
                                        uint32_t& phase, float out[kOut], uint32_t* status) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tile = tid / kRows, r = tid % kRows;
  const uint32_t trow = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)tile * kColsPerTile;
  unsigned char* const mine = act + (size_t)tile * kTileBytes;
  const uint32_t act_addr = saddr(act);
#pragma unroll 1
  for (int l = 0; l < 4; ++l) {
    const uint32_t nn = l < 3 ? (uint32_t)kHid : (uint32_t)kOutPad;
    fence_async_smem();
    fence_before_sync();
    __syncthreads();  // the operands are written; the previous layer's accumulators are read
    fence_after_sync();
    if (tid == 0) {
      const uint32_t w_addr = l < 3 ? saddr(w.w[l]) : saddr(w.w4);
#pragma unroll
      for (int t = 0; t < NT; ++t)
#pragma unroll
        for (int ks = 0; ks < kK / 16; ++ks)  // K = 16 per instruction: two cores along K
          mma_f16(tmem + (uint32_t)t * kColsPerTile, smem_desc(act_addr + (uint32_t)t * kTileBytes + 256u * ks),
                  smem_desc(w_addr + 256u * ks), instr_desc(nn), ks > 0);
      commit(bar);
    }
    const bool done = bar_wait(bar, phase);
    if (__syncthreads_or(!done)) {
      if (tid == 0) raise_status(status, BAJO_STATUS_WAIT_TIMEOUT);
      bar_wait(bar, phase);  // once more, so that no MMA is in flight when the caller frees the memory
      return false;
    }
    phase ^= 1u;
    fence_after_sync();
    if (l < 3) {
#pragma unroll
      for (int c0 = 0; c0 < kHid; c0 += 32) {
        uint32_t v[32];
        tmem_ld32_wait(trow + (uint32_t)c0, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          *reinterpret_cast<uint4*>(mine + core_off(r, c0 + 8 * q)) =
              make_uint4(relu_pack(v[8 * q], v[8 * q + 1]), relu_pack(v[8 * q + 2], v[8 * q + 3]),
                         relu_pack(v[8 * q + 4], v[8 * q + 5]), relu_pack(v[8 * q + 6], v[8 * q + 7]));
      }
    } else {
      uint32_t v[32];
      tmem_ld32_wait(trow, v);
#pragma unroll
      for (int c = 0; c < kOut; ++c) out[c] = __uint_as_float(v[c]);
    }
  }
  fence_before_sync();
  __syncthreads();  // every operand read is done: the caller may overwrite the tiles
  fence_after_sync();
  return true;
}

}  // namespace tc

// ---------------------------------------------------------------------------
// vMF mixture: mean = m / len, len = sqrt(|m|^2 + 1e-12) (so d mean / dm =
// (I - mean mean^T) / len exactly), kappa = exp(clamp(s, -2, 8)),
// weights = softmax(logits);
// pdf(w) = sum_k pi_k kappa_k / (2 pi (1 - e^-2kappa)) exp(kappa (mu.w - 1)).
// ---------------------------------------------------------------------------
struct Mixture {
  float pi[kLobes], mu[kLobes][3], kap[kLobes], norm[kLobes], len[kLobes];
};

__device__ __forceinline__ void mixture_from_outputs(const float* o, Mixture& m) {
  float mx = -FLT_MAX;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, o[5 * k + 4]);
  float z = 0.0f;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    m.pi[k] = expf(o[5 * k + 4] - mx);
    z += m.pi[k];
  }
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    m.pi[k] /= z;
    const float x = o[5 * k], y = o[5 * k + 1], w = o[5 * k + 2];
    m.len[k] = sqrtf(x * x + y * y + w * w + 1e-12f);
    m.mu[k][0] = x / m.len[k];
    m.mu[k][1] = y / m.len[k];
    m.mu[k][2] = w / m.len[k];
    m.kap[k] = expf(fminf(fmaxf(o[5 * k + 3], kLogKappaMin), kLogKappaMax));
    m.norm[k] = m.kap[k] / (2.0f * kPi * (-expm1f(-2.0f * m.kap[k])));
  }
}

__device__ __forceinline__ float mixture_pdf(const Mixture& m, const float* d) {
  float q = 0.0f;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    const float c = m.mu[k][0] * d[0] + m.mu[k][1] * d[1] + m.mu[k][2] * d[2];
    q += m.pi[k] * m.norm[k] * expf(m.kap[k] * (c - 1.0f));
  }
  return q;
}

// Loss -weight * log pdf(dir) of one sample and its gradient w.r.t. the 20
// raw outputs.
__device__ __forceinline__ float mixture_nll_grad(const float* o, const float* dir, float weight, float* grad) {
  Mixture m;
  mixture_from_outputs(o, m);
  float v[kLobes], c[kLobes];
  float q = 0.0f;
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    c[k] = m.mu[k][0] * dir[0] + m.mu[k][1] * dir[1] + m.mu[k][2] * dir[2];
    v[k] = m.norm[k] * expf(m.kap[k] * (c[k] - 1.0f));
    q += m.pi[k] * v[k];
  }
  q = fmaxf(q, 1e-30f);
#pragma unroll
  for (int k = 0; k < kLobes; ++k) {
    const float r = m.pi[k] * v[k] / q;
    grad[5 * k + 4] = weight * (m.pi[k] - r);
    const float kap = m.kap[k];
    const float dlogv_ds = 1.0f - 2.0f * kap * expf(-2.0f * kap) / (-expm1f(-2.0f * kap)) + kap * (c[k] - 1.0f);
    const bool clamped = o[5 * k + 3] < kLogKappaMin || o[5 * k + 3] > kLogKappaMax;
    grad[5 * k + 3] = clamped ? 0.0f : -weight * r * dlogv_ds;
#pragma unroll
    for (int a = 0; a < 3; ++a) grad[5 * k + a] = -weight * r * kap * (dir[a] - m.mu[k][a] * c[k]) / m.len[k];
  }
  return -weight * logf(q);
}

// ---------------------------------------------------------------------------
// training-record buffer written by the guided tracer: 256-byte header (u32
// count, u32 first record of the current chunk), then arrays on 256-byte
// boundaries
// ---------------------------------------------------------------------------
struct RecordLayout {
  size_t pos, nrm, dir, weight, sidx, tn, snap, wpre, total;
};

inline RecordLayout record_layout(uint32_t cap) {
  auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  RecordLayout L;
  size_t o = 256;
  const size_t c = cap;
  L.pos = o;
  o = a256(o + 12 * c);
  L.nrm = o;
  o = a256(o + 12 * c);
  L.dir = o;
  o = a256(o + 12 * c);
  L.weight = o;
  o = a256(o + 4 * c);
  L.sidx = o;
  o = a256(o + 4 * c);
  L.tn = o;
  o = a256(o + 12 * c);
  L.snap = o;
  o = a256(o + 12 * c);
  L.wpre = o;
  o = a256(o + 4 * c);
  L.total = o;
  return L;
}

}  // namespace mlp
}  // namespace bajo
