// mlp.cu -- kernels of the path-guiding network: batched forward, the
// vMF-mixture negative-log-likelihood gradient (forward recompute +
// backpropagation, weight gradients on the tensor cores), Adam, and the
// training loop over the records the guided tracer writes.  The network, its
// encoding and the mixture math live in mlp.cuh.  New on this path (the
// reference has no guiding); the CPU FP64 oracle checks outputs and
// gradients.
#include <cmath>

#include "mlp.cuh"

namespace bajo {
int sm_count();

namespace mlp {

constexpr int kWarps = 8, kThreads = 256, kRows = 16 * kWarps;  // 128 rows per CTA tile

// feature rows of a tile: 5 encoding groups per row spread over the block;
// rows past the end are zero.  Row j reads sample (offset + j) % count when
// `wrap`, else sample j.
__device__ void encode_tile(__half* x, const float* __restrict__ pos, const float* __restrict__ nrm,
                            const float* box, uint64_t row_base, uint32_t rows, uint32_t offset, uint32_t count,
                            bool wrap) {
  for (int w = threadIdx.x; w < kRows * 5; w += kThreads) {
    const int r = w / 5, grp = w % 5;
    const uint64_t j = row_base + r;
    __half* row = x + r * kLd;
    if (j < rows) {
      const uint64_t i = wrap ? ((uint64_t)offset + j) % count : j;
      const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
      const float q[3] = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
      encode_group(grp, p, q, box, row);
    } else {
      const int col = grp < 3 ? grp * kPosBins : 3 * kPosBins + (grp - 3) * kDirBins;
      const int bins = grp < 3 ? kPosBins : kDirBins;
      for (int k = 0; k < bins; k += 2) st32(row + col + k, 0u);
    }
  }
}

struct FwdSmem {
  Net net;
  WarpTile tile[kWarps];
};

// warp-autonomous: every warp encodes 32 samples (one per lane), runs them
// through the network and writes their outputs
__global__ void __launch_bounds__(kThreads, 2) forward_kernel(const __half* __restrict__ p16,
                                                              const float* __restrict__ pos,
                                                              const float* __restrict__ nrm, const float* box,
                                                              uint32_t n, float* __restrict__ out20) {
  extern __shared__ __align__(16) unsigned char raw[];
  FwdSmem& s = *reinterpret_cast<FwdSmem*>(raw);
  load_net<kThreads>(s.net, p16);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpTile& t = s.tile[warp];
  const uint64_t warps = (uint64_t)gridDim.x * kWarps;
  for (uint64_t base = ((uint64_t)blockIdx.x * kWarps + warp) * 32; base < n; base += warps * 32) {
    const uint64_t i = base + lane;
    __half* row = t.x + lane * kLd;
    if (i < n) {
      const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
      const float q[3] = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
      encode_row(p, q, box, row);
    } else {
      for (int k = 0; k < kIn; k += 2) st32(row + k, 0u);
    }
    __syncwarp();
    forward_tile<2>(s.net, t.x, 0, nullptr, t.out);
    __syncwarp();
    for (int k = lane; k < 32 * kOut; k += 32) {
      const int r = k / kOut, c = k % kOut;
      if (base + r < n) out20[(base + r) * kOut + c] = t.out[r * kOutLd + c];
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// gradient of sum_j -w_j log pdf_j(dir_j) over a batch of rows.
// Persistent CTAs; each warp owns fixed 16x8 tiles of every weight gradient
// and accumulates them in registers over all of the CTA's row tiles; bias
// gradients in shared memory; one atomicAdd per element at the end.
// Rows j < min(n_rows, count) read sample (offset + j) % count when a device
// count is given (the training records; count = min(*d_count, count_cap)),
// else sample j.
// ---------------------------------------------------------------------------
constexpr float kGradScale = 256.0f;  // keeps FP16 dL/dz away from underflow

// dW[out][in] tile (16 out x 8 in) += dZ^T x A over the tile's 128 rows:
// A operand (m = out, k = row) = dz[row][out]; B operand (k = row, n = in) =
// act[row][in].
__device__ __forceinline__ uint32_t pk2(__half lo, __half hi) {
  __half2 h;
  h.x = lo;
  h.y = hi;
  return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ void dw_tile(const __half* dz, int dz_ld, int out0, const __half* act, int in0,
                                        float c[4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
#pragma unroll 2
  for (int kt = 0; kt < kRows / 16; ++kt) {
    const int r = 16 * kt + 2 * tq;
    uint32_t a[4], b[2];
    a[0] = pk2(dz[r * dz_ld + out0 + g], dz[(r + 1) * dz_ld + out0 + g]);
    a[1] = pk2(dz[r * dz_ld + out0 + g + 8], dz[(r + 1) * dz_ld + out0 + g + 8]);
    a[2] = pk2(dz[(r + 8) * dz_ld + out0 + g], dz[(r + 9) * dz_ld + out0 + g]);
    a[3] = pk2(dz[(r + 8) * dz_ld + out0 + g + 8], dz[(r + 9) * dz_ld + out0 + g + 8]);
    b[0] = pk2(act[r * kLd + in0 + g], act[(r + 1) * kLd + in0 + g]);
    b[1] = pk2(act[(r + 8) * kLd + in0 + g], act[(r + 9) * kLd + in0 + g]);
    mma16816(c, a, b);
  }
}

struct TrainSmem {
  Net net;
  __half WT[3][kIn * kLd];     // transposes [in][out]
  __half W4T[kHid * kLd32];    // [in][out]
  __half act[4][kRows * kLd];  // X, A1, A2, A3 of the tile, row-major
  __half dz[kRows * kLd];      // dZ of the layer being reduced
  __half g[kRows * kLd32];     // scaled dL/dout
  float out[kRows * kOutLd];   // outputs of the tile
  float db[4][kHid];
  float loss;
};

__global__ void __launch_bounds__(kThreads) train_kernel(const __half* __restrict__ p16,
                                                         const float* __restrict__ pos,
                                                         const float* __restrict__ nrm,
                                                         const float* __restrict__ dir,
                                                         const float* __restrict__ weight, const float* box,
                                                         uint32_t n_rows, uint32_t offset,
                                                         const uint32_t* __restrict__ d_count, uint32_t count_cap,
                                                         float* __restrict__ grad32, float* __restrict__ loss_out) {
  extern __shared__ __align__(16) unsigned char raw[];
  TrainSmem& s = *reinterpret_cast<TrainSmem*>(raw);
  load_net<kThreads>(s.net, p16);
  for (int i = threadIdx.x; i < kHid * kIn; i += kThreads)
    for (int l = 0; l < 3; ++l) s.WT[l][(i % kIn) * kLd + i / kIn] = p16[kOffW(l) + i];
  for (int i = threadIdx.x; i < kOutPad * kHid; i += kThreads)
    s.W4T[(i % kHid) * kLd32 + i / kHid] = p16[kOffW(3) + i];
  for (int i = threadIdx.x; i < 4 * kHid; i += kThreads) (&s.db[0][0])[i] = 0.0f;
  if (threadIdx.x == 0) s.loss = 0.0f;
  const bool wrap = d_count != nullptr;
  const uint32_t count = wrap ? min(*d_count, count_cap) : n_rows;
  const uint32_t rows = wrap ? min(n_rows, count) : n_rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
  const int row0 = warp * 16;
  __half* const keep[3] = {s.act[1], s.act[2], s.act[3]};
  // weight-gradient tiles of this warp: hidden layers 64x64 = 4 x 8 tiles of
  // 16x8 (out tile warp / 2, in tiles 4 * (warp % 2) + q); output layer
  // 32x64 = 2 x 8 tiles (tile 2 * warp + t: out tile / 8, in tile % 8)
  float dw[3][4][4] = {};
  float dw4[2][4] = {};
  for (uint64_t base = (uint64_t)blockIdx.x * kRows; base < rows; base += (uint64_t)gridDim.x * kRows) {
    __syncthreads();
    encode_tile(s.act[0], pos, nrm, box, base, rows, offset, count, wrap);
    __syncthreads();
    forward_tile<1>(s.net, s.act[0], row0, keep, s.out);
    __syncwarp();
    // dL/dout of the warp's rows, lanes 0..15 one row each
    if (lane < 16) {
      const int r = row0 + lane;
      const uint64_t j = base + r;
      float gr[kOut];
      float l = 0.0f;
      if (j < rows) {
        const uint64_t i = wrap ? ((uint64_t)offset + j) % count : j;
        const float d[3] = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
        l = mixture_nll_grad(&s.out[r * kOutLd], d, weight[i], gr);
      } else {
        for (int k = 0; k < kOut; ++k) gr[k] = 0.0f;
      }
      for (int k = 0; k < kOutPad; k += 2)
        st32(&s.g[r * kLd32 + k], pack_h2_sat(k < kOut ? gr[k] * kGradScale : 0.0f,
                                                 k + 1 < kOut ? gr[k + 1] * kGradScale : 0.0f));
      if (l != 0.0f) atomicAdd(&s.loss, l);
    }
    __syncwarp();
    uint32_t ga[2][4];  // G as A fragments (k = 32 outputs = 2 k-tiles)
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      const int c = 16 * kt + 2 * tq;
      ga[kt][0] = ld32(&s.g[(row0 + g) * kLd32 + c]);
      ga[kt][1] = ld32(&s.g[(row0 + g + 8) * kLd32 + c]);
      ga[kt][2] = ld32(&s.g[(row0 + g) * kLd32 + c + 8]);
      ga[kt][3] = ld32(&s.g[(row0 + g + 8) * kLd32 + c + 8]);
    }
    __syncthreads();  // every warp's G and activations are in shared memory
    for (int t2 = 0; t2 < 2; ++t2) {
      const int tile = warp * 2 + t2;
      dw_tile(s.g, kLd32, 16 * (tile / 8), s.act[3], 8 * (tile % 8), dw4[t2]);
    }
    if (threadIdx.x < kOutPad) {
      float acc = 0.0f;
      for (int r = 0; r < kRows; ++r) acc += __half2float(s.g[r * kLd32 + threadIdx.x]);
      s.db[3][threadIdx.x] += acc;
    }
    // dA3 = G x W4: B operand (k = out, n = in) = W4T[in][out]
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
      for (int kt = 0; kt < 2; ++kt) {
        uint32_t b[2];
        const __half* w = s.W4T + (8 * j + g) * kLd32 + 16 * kt + 2 * tq;
        b[0] = ld32(w);
        b[1] = ld32(w + 8);
        mma16816(acc[j], ga[kt], b);
      }
    }
    for (int l = 2; l >= 0; --l) {
      __syncthreads();  // the previous layer's readers of s.dz are done
      // dZ_l = dA_{l+1} * (A_{l+1} > 0), row-major for the weight gradient
      const __half* A = s.act[l + 1];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = 8 * j + 2 * tq;
        const __half2 lo = *reinterpret_cast<const __half2*>(&A[(row0 + g) * kLd + c]);
        const __half2 hi = *reinterpret_cast<const __half2*>(&A[(row0 + g + 8) * kLd + c]);
        if (!(__low2float(lo) > 0.0f)) acc[j][0] = 0.0f;
        if (!(__high2float(lo) > 0.0f)) acc[j][1] = 0.0f;
        if (!(__low2float(hi) > 0.0f)) acc[j][2] = 0.0f;
        if (!(__high2float(hi) > 0.0f)) acc[j][3] = 0.0f;
        st32(&s.dz[(row0 + g) * kLd + c], pack_h2_sat(acc[j][0], acc[j][1]));
        st32(&s.dz[(row0 + g + 8) * kLd + c], pack_h2_sat(acc[j][2], acc[j][3]));
      }
      __syncthreads();
      for (int qd = 0; qd < 4; ++qd)
        dw_tile(s.dz, kLd, 16 * (warp / 2), s.act[l], 8 * (4 * (warp % 2) + qd), dw[l][qd]);
      if (threadIdx.x < kHid) {
        float sacc = 0.0f;
        for (int r = 0; r < kRows; ++r) sacc += __half2float(s.dz[r * kLd + threadIdx.x]);
        s.db[l][threadIdx.x] += sacc;
      }
      if (l == 0) break;
      // dA_l = dZ_l x W_l: A = the warp's dZ_l rows, B (k = out, n = in) = WT[in][out]
      uint32_t a[4][4];
      load_afrag64(s.dz, row0, a);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          uint32_t b[2];
          const __half* w = s.WT[l] + (8 * j + g) * kLd + 16 * kt + 2 * tq;
          b[0] = ld32(w);
          b[1] = ld32(w + 8);
          mma16816(acc[j], a[kt], b);
        }
      }
    }
  }
  __syncthreads();
  // flush the weight-gradient tiles (C fragments) and biases, unscaled
  const float inv = 1.0f / kGradScale;
  for (int l = 0; l < 3; ++l)
    for (int qd = 0; qd < 4; ++qd) {
      const int out0 = 16 * (warp / 2), in0 = 8 * (4 * (warp % 2) + qd);
      float* G = grad32 + kOffW(l);
      atomicAdd(&G[(out0 + g) * kIn + in0 + 2 * tq], dw[l][qd][0] * inv);
      atomicAdd(&G[(out0 + g) * kIn + in0 + 2 * tq + 1], dw[l][qd][1] * inv);
      atomicAdd(&G[(out0 + g + 8) * kIn + in0 + 2 * tq], dw[l][qd][2] * inv);
      atomicAdd(&G[(out0 + g + 8) * kIn + in0 + 2 * tq + 1], dw[l][qd][3] * inv);
    }
  for (int t2 = 0; t2 < 2; ++t2) {
    const int tile = warp * 2 + t2, out0 = 16 * (tile / 8), in0 = 8 * (tile % 8);
    float* G = grad32 + kOffW(3);
    atomicAdd(&G[(out0 + g) * kHid + in0 + 2 * tq], dw4[t2][0] * inv);
    atomicAdd(&G[(out0 + g) * kHid + in0 + 2 * tq + 1], dw4[t2][1] * inv);
    atomicAdd(&G[(out0 + g + 8) * kHid + in0 + 2 * tq], dw4[t2][2] * inv);
    atomicAdd(&G[(out0 + g + 8) * kHid + in0 + 2 * tq + 1], dw4[t2][3] * inv);
  }
  for (int i = threadIdx.x; i < kHid; i += kThreads)
    for (int l = 0; l < 3; ++l) atomicAdd(&grad32[kOffB(l) + i], s.db[l][i] * inv);
  for (int i = threadIdx.x; i < kOutPad; i += kThreads) atomicAdd(&grad32[kOffB(3) + i], s.db[3][i] * inv);
  if (threadIdx.x == 0 && loss_out) atomicAdd(loss_out, s.loss);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; FP16 copies refreshed.
// grad_scale multiplies the raw gradient; the padded rows of the output layer
// stay zero.
// With `clear`, the gradient (and *loss, when given) is zeroed after use, so
// that the next gradient launch may accumulate without a memset.
__global__ void adam_kernel(float* __restrict__ p32, __half* __restrict__ p16, float* __restrict__ grad,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float bc1, float bc2, float grad_scale, bool clear, float* __restrict__ loss) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  if (clear && i == 0 && loss) *loss = 0.0f;
  const bool pad_w = i >= kOffW(3) && i < kOffB(3) && (i - kOffW(3)) / kHid >= kOut;
  const bool pad_b = i >= kOffB(3) && i - kOffB(3) >= kOut;
  if (pad_w || pad_b) {
    p32[i] = 0.0f;
    p16[i] = __float2half(0.0f);
    if (clear) grad[i] = 0.0f;
    return;
  }
  const float gr = grad[i] * grad_scale;
  if (clear) grad[i] = 0.0f;
  const float mi = b1 * m[i] + (1.0f - b1) * gr;
  const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
  m[i] = mi;
  v[i] = vi;
  const float w = p32[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  p32[i] = w;
  p16[i] = __float2half(w);
}

uint32_t grid_for(uint64_t rows) {
  uint64_t grid = (rows + kRows - 1) / kRows;
  const uint64_t cap = (uint64_t)sm_count();
  if (grid > cap) grid = cap;
  return grid ? (uint32_t)grid : 1u;
}

cudaError_t launch_grad(const __half* p16, const float* pos, const float* nrm, const float* dir, const float* w,
                        const float* box, uint32_t n, uint32_t offset, const uint32_t* d_count, uint32_t count_cap,
                        float* grad, float* loss, cudaStream_t st) {
  static_assert(sizeof(TrainSmem) <= 227 * 1024, "training tile exceeds shared memory");
  const size_t smem = sizeof(TrainSmem);
  cudaError_t e = cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st)) != cudaSuccess) return e;
  if (loss && (e = cudaMemsetAsync(loss, 0, sizeof(float), st)) != cudaSuccess) return e;
  if (n == 0) return cudaSuccess;
  train_kernel<<<grid_for(n), kThreads, smem, st>>>(p16, pos, nrm, dir, w, box, n, offset, d_count, count_cap, grad,
                                                    loss);
  return cudaGetLastError();
}

cudaError_t launch_adam(float* p32, __half* p16, float* grad, float* m, float* v, uint32_t step, float lr,
                        float b1, float b2, float eps, float grad_scale, cudaStream_t st, bool clear = false,
                        float* loss = nullptr) {
  const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
  adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(p32, p16, grad, m, v, lr, b1, b2, eps, bc1, bc2, grad_scale,
                                                     clear, loss);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Forward on the 5th-generation tensor cores (tcgen05): tc::forward (mlp.cuh)
// over 128-row tiles, one CTA of 128 threads per resident slot.
// ---------------------------------------------------------------------------
namespace tc {

struct __align__(128) FwdSmem {
  Weights w;
  __half a[kRows * kK];  // the tile's features, activations, then staged outputs
  unsigned long long bar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(kRows) forward_tc_kernel(const __half* __restrict__ p16,
                                                             const float* __restrict__ pos,
                                                             const float* __restrict__ nrm, const float* box,
                                                             uint32_t n, float* __restrict__ out20,
                                                             uint32_t* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char raw[];
  FwdSmem& s = *reinterpret_cast<FwdSmem*>(raw);
  const int tid = threadIdx.x;
  load_weights<kRows>(s.w, p16);
  const uint32_t bar = saddr(&s.bar);
  const uint32_t tmem = setup<1>(bar, &s.tmem);
  uint32_t phase = 0;
  unsigned char* const abytes = reinterpret_cast<unsigned char*>(s.a);
  for (uint64_t base = (uint64_t)blockIdx.x * kRows; base < n; base += (uint64_t)gridDim.x * kRows) {
    {
      uint32_t f[32];
      const uint64_t i = base + tid;
      if (i < n) {
        const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        const float q[3] = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
        encode_pairs(p, q, box, f);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) f[j] = 0u;
      }
      store_features(abytes, tid, f);
    }
    float o[kOut];
    if (!forward<1>(s.w, abytes, tmem, bar, phase, o, status)) break;
    // the tile's outputs, staged row-major in the (now unread) operand buffer
    // and written out coalesced
    float* stage = reinterpret_cast<float*>(s.a);
#pragma unroll
    for (int c = 0; c < kOut; ++c) stage[tid * kOut + c] = o[c];
    __syncthreads();
    const uint64_t rows = min((uint64_t)kRows, (uint64_t)n - base);
    for (uint32_t k = tid; k < rows * kOut; k += kRows) out20[base * kOut + k] = stage[k];
    __syncthreads();  // the next tile's features overwrite the staged outputs
  }
  teardown<1>(tmem);
}

// ---------------------------------------------------------------------------
// Gradient of sum_j -w_j log pdf_j(dir_j) on the tensor cores.  Per 128-row
// tile: the forward with every layer's input A_l kept in shared memory
// (A_0 = the features), D_3 = dL/dout per row, then for l = 3..0
//   dW_l += D_l^T A_l   (M = 64 outputs, N = 80: 64 inputs, the column of
//                        ones (its bias) and zeros, K = 128 rows)
//   dA_l  = D_l W_l     (M = 128 rows, N = 64 inputs, K = outputs of l; l > 0)
//   D_{l-1} = dA_l where A_l > 0.
// The same shared-memory tiles serve both products.  A core matrix of a
// [rows][features] tile holds 8 rows x 8 features, the 8 features of a row
// in 16 contiguous bytes: K-major when the rows are M (the forward, dA_l),
// MN-major when the rows are K (dW_l).  Likewise the weights' [out][in] tiles
// are K-major with N = out (forward) and MN-major with N = in (dA_l).
// The weight gradients accumulate in tensor memory over all of the CTA's
// tiles (an M = 64 accumulator holds row 16 q + i in lane 32 q + i) and are
// added to the global gradient once, unscaled, at the end.
// ---------------------------------------------------------------------------
constexpr int kDCols = 64;                           // columns of the D tiles (dL/dout uses 20)
constexpr uint32_t kDBytes = kRows * kDCols * 2;     // 16 KB
constexpr uint32_t kDSbo = (kDCols / 8) * 128;       // bytes between 8-row groups of a D tile
constexpr uint32_t kActSbo = kKCores * 128;          // ... of an activation tile (1280)
constexpr uint32_t kGradCols = 512;                  // tensor memory of a CTA
__host__ __device__ constexpr uint32_t dw_col(int l) { return 64u + 96u * (uint32_t)l; }  // 80 columns each
static_assert(dw_col(3) + 96 <= kGradCols, "weight-gradient accumulators exceed tensor memory");

__device__ __forceinline__ uint32_t d_off(int r, int k) {
  return (uint32_t)(((r >> 3) * (kDCols / 8) + (k >> 3)) * 128 + ((r & 7) << 4) + ((k & 7) << 1));
}
// matrix descriptor with explicit leading / stride byte offsets (no swizzle)
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: D FP32, A and B FP16, A MN-major (bit 15)
// and B MN-major (bit 16) when asked
__host__ __device__ constexpr uint32_t idesc(uint32_t m, uint32_t n, bool a_mn, bool b_mn) {
  return (1u << 4) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

struct __align__(128) GradSmem {
  Weights w;
  unsigned char act[4][kTileBytes];  // A_0 (features), A_1..A_3; ones in column 64
  unsigned char d3[kDBytes];         // dL/dout x kGradScale (columns 20..63 zero)
  unsigned char d[kDBytes];          // D_2, D_1, D_0 in turn
  unsigned long long bar;
  uint32_t tmem;
  float loss;
};

// the operands are written (generic proxy) and the accumulators read
__device__ __forceinline__ void before_mma() {
  fence_async_smem();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
}
// true in every thread once the committed MMAs completed; false in every
// thread (status raised, in-flight MMAs waited for once more) on a timeout
__device__ __forceinline__ bool after_mma(uint32_t bar, uint32_t& phase, uint32_t* status) {
  const bool done = bar_wait(bar, phase);
  if (__syncthreads_or(!done)) {
    if (threadIdx.x == 0) raise_status(status, BAJO_STATUS_WAIT_TIMEOUT);
    bar_wait(bar, phase);
    return false;
  }
  phase ^= 1u;
  fence_after_sync();
  return true;
}

__global__ void __launch_bounds__(kRows, 1) grad_tc_kernel(const __half* __restrict__ p16,
                                                          const float* __restrict__ pos,
                                                          const float* __restrict__ nrm,
                                                          const float* __restrict__ dir,
                                                          const float* __restrict__ weight, const float* box,
                                                          uint32_t n_rows, uint32_t offset,
                                                          const uint32_t* __restrict__ d_count, uint32_t count_cap,
                                                          float* __restrict__ grad32, float* __restrict__ loss_out,
                                                          uint32_t* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char raw[];
  GradSmem& s = *reinterpret_cast<GradSmem*>(raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  load_weights<kRows>(s.w, p16);
  // the ones column of A_1..A_3 and the zero columns of D_3 (written once)
#pragma unroll
  for (int l = 1; l < 4; ++l) {
    *reinterpret_cast<uint4*>(s.act[l] + core_off(tid, kIn)) = make_uint4(0x3C00u, 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(s.act[l] + core_off(tid, kIn + 8)) = make_uint4(0u, 0u, 0u, 0u);
  }
#pragma unroll
  for (int q = 0; q < kDCols / 8; ++q) *reinterpret_cast<uint4*>(s.d3 + d_off(tid, 8 * q)) = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) s.loss = 0.0f;
  const uint32_t bar = saddr(&s.bar);
  const uint32_t tmem = setup_cols(bar, &s.tmem, kGradCols);
  const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);  // this thread's lane
  const uint32_t a_addr[4] = {saddr(s.act[0]), saddr(s.act[1]), saddr(s.act[2]), saddr(s.act[3])};
  const uint32_t w_addr[4] = {saddr(s.w.w[0]), saddr(s.w.w[1]), saddr(s.w.w[2]), saddr(s.w.w4)};
  const uint32_t d3_addr = saddr(s.d3), d_addr = saddr(s.d);
  const bool wrap = d_count != nullptr;
  const uint32_t count = wrap ? min(*d_count, count_cap) : n_rows;
  const uint32_t rows = wrap ? min(n_rows, count) : n_rows;
  uint32_t phase = 0;
  bool ok = true, any = false;
  float my_loss = 0.0f;
  for (uint64_t base = (uint64_t)blockIdx.x * kRows; base < rows; base += (uint64_t)gridDim.x * kRows) {
    const uint64_t j = base + tid;
    const bool valid = j < rows;
    const uint64_t i = valid ? (wrap ? ((uint64_t)offset + j) % count : j) : 0;
    {
      uint32_t f[32];
      if (valid) {
        const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        const float q[3] = {nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]};
        encode_pairs(p, q, box, f);
      } else {
#pragma unroll
        for (int k = 0; k < 32; ++k) f[k] = 0u;
      }
      store_features(s.act[0], tid, f);
    }
    // forward: layer l reads A_l, writes A_{l+1} (l < 3) or the outputs
    float o[kOut];
#pragma unroll 1
    for (int l = 0; l < 4 && ok; ++l) {
      before_mma();
      if (tid == 0) {
#pragma unroll
        for (int ks = 0; ks < kK / 16; ++ks)
          mma_f16(tmem, desc(a_addr[l] + 256u * ks, 128u, kActSbo), desc(w_addr[l] + 256u * ks, 128u, kActSbo),
                  idesc(kRows, l < 3 ? kHid : kOutPad, false, false), ks > 0);
        commit(bar);
      }
      if (!(ok = after_mma(bar, phase, status))) break;
      if (l < 3) {
#pragma unroll
        for (int c0 = 0; c0 < kHid; c0 += 32) {
          uint32_t v[32];
          tmem_ld32_wait(trow + (uint32_t)c0, v);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            *reinterpret_cast<uint4*>(s.act[l + 1] + core_off(tid, c0 + 8 * q)) =
                make_uint4(relu_pack(v[8 * q], v[8 * q + 1]), relu_pack(v[8 * q + 2], v[8 * q + 3]),
                           relu_pack(v[8 * q + 4], v[8 * q + 5]), relu_pack(v[8 * q + 6], v[8 * q + 7]));
        }
      } else {
        uint32_t v[32];
        tmem_ld32_wait(trow, v);
#pragma unroll
        for (int c = 0; c < kOut; ++c) o[c] = __uint_as_float(v[c]);
      }
    }
    if (!ok) break;
    // D_3: this row's dL/dout, scaled (columns 0..23 rewritten, 20..23 zero)
    {
      float gr[kOut];
      if (valid) {
        const float dd[3] = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
        my_loss += mixture_nll_grad(o, dd, weight[i], gr);
      } else {
#pragma unroll
        for (int k = 0; k < kOut; ++k) gr[k] = 0.0f;
      }
      uint32_t h[12];
#pragma unroll
      for (int k = 0; k < 12; ++k)
        h[k] = pack_h2_sat(2 * k < kOut ? gr[2 * k] * kGradScale : 0.0f,
                           2 * k + 1 < kOut ? gr[2 * k + 1] * kGradScale : 0.0f);
#pragma unroll
      for (int q = 0; q < 3; ++q)
        *reinterpret_cast<uint4*>(s.d3 + d_off(tid, 8 * q)) = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2],
                                                                           h[4 * q + 3]);
    }
    // backward
#pragma unroll 1
    for (int l = 3; l >= 0; --l) {
      before_mma();
      if (tid == 0) {
        const uint32_t dl = l == 3 ? d3_addr : d_addr;
        // dW_l (+)= D_l^T A_l: D_l MN-major (M = out: 128 B apart; K = rows:
        // 8-row groups kDSbo apart), A_l MN-major (N = in: 128 B; K: kActSbo)
#pragma unroll
        for (int ks = 0; ks < kRows / 16; ++ks)
          mma_f16(tmem + dw_col(l), desc(dl + 2u * kDSbo * ks, kDSbo, 128u),
                  desc(a_addr[l] + 2u * kActSbo * ks, kActSbo, 128u), idesc(64, 80, true, true), (ks > 0) || any);
        if (l > 0) {
          // dA_l = D_l W_l: D_l K-major (K = out: 128 B; M = rows: kDSbo),
          // W_l MN-major (N = in: 128 B apart; K = out: 8-row groups kActSbo apart)
          const int k_out = l == 3 ? kOutPad : kHid;
          for (int ks = 0; ks < k_out / 16; ++ks)
            mma_f16(tmem, desc(dl + 256u * ks, 128u, kDSbo), desc(w_addr[l] + 2u * kActSbo * ks, kActSbo, 128u),
                    idesc(kRows, kIn, false, true), ks > 0);
        }
        commit(bar);
      }
      if (!(ok = after_mma(bar, phase, status))) break;
      if (l > 0) {
        // D_{l-1} = dA_l where A_l > 0 (FP16, saturated)
#pragma unroll
        for (int c0 = 0; c0 < kIn; c0 += 32) {
          uint32_t v[32];
          tmem_ld32_wait(trow + (uint32_t)c0, v);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint4 a4 = *reinterpret_cast<const uint4*>(s.act[l] + core_off(tid, c0 + 8 * q));
            const uint32_t av[4] = {a4.x, a4.y, a4.z, a4.w};
            uint32_t h[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const __half2 a = *reinterpret_cast<const __half2*>(&av[k]);
              const float lo = __low2float(a) > 0.0f ? __uint_as_float(v[8 * q + 2 * k]) : 0.0f;
              const float hi = __high2float(a) > 0.0f ? __uint_as_float(v[8 * q + 2 * k + 1]) : 0.0f;
              h[k] = pack_h2_sat(lo, hi);
            }
            *reinterpret_cast<uint4*>(s.d + d_off(tid, c0 + 8 * q)) = make_uint4(h[0], h[1], h[2], h[3]);
          }
        }
      }
    }
    if (!ok) break;
    any = true;
  }
  // loss of the CTA's rows
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) my_loss += __shfl_xor_sync(0xFFFFFFFFu, my_loss, k);
  if (lane == 0 && my_loss != 0.0f) atomicAdd(&s.loss, my_loss);
  // flush the weight gradients: warp q reads lanes 32 q.., whose lanes 0..15
  // hold rows 16 q + lane (column 64 = the bias); staged row-major in the
  // (now unread) activation tiles, then added with coalesced 16-byte atomics
  if (ok && any) {
    float* stage = reinterpret_cast<float*>(s.act[0]);  // [4][64][kStageLd], 80 KB
    constexpr int kStageLd = 80;
    static_assert(4 * 64 * kStageLd * 4 <= 4 * kTileBytes, "gradient staging exceeds the activation tiles");
    const int out = 16 * warp + lane;
#pragma unroll 1
    for (int l = 0; l < 4; ++l)
#pragma unroll 1
      for (int c0 = 0; c0 < 96; c0 += 32) {  // columns 0..95 (80..95 unused)
        uint32_t v[32];
        tmem_ld32_wait(trow + dw_col(l) + (uint32_t)c0, v);
        if (lane < 16) {
          float4* dst = reinterpret_cast<float4*>(stage + (l * 64 + out) * kStageLd + c0);
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (c0 + 4 * q < kStageLd)
              dst[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                   __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
        }
      }
    __syncthreads();
    const float inv = 1.0f / kGradScale;
    // per layer: rows x 16 chunks of 4 weights, then rows / 4 chunks of biases
    for (int l = 0; l < 4; ++l) {
      const int rows_l = l < 3 ? kHid : kOutPad;
      const float* sl = stage + l * 64 * kStageLd;
      float4* W = reinterpret_cast<float4*>(grad32 + kOffW(l));
      for (int c = tid; c < rows_l * (kIn / 4); c += kRows) {
        const int o = c / (kIn / 4), k = 4 * (c % (kIn / 4));
        const float* x = sl + o * kStageLd + k;
        atomicAdd(&W[c], make_float4(x[0] * inv, x[1] * inv, x[2] * inv, x[3] * inv));
      }
      float4* B = reinterpret_cast<float4*>(grad32 + kOffB(l));
      for (int c = tid; c < rows_l / 4; c += kRows) {
        const float* x = sl + 4 * c * kStageLd + kIn;
        atomicAdd(&B[c], make_float4(x[0] * inv, x[kStageLd] * inv, x[2 * kStageLd] * inv, x[3 * kStageLd] * inv));
      }
    }
  }
  __syncthreads();
  if (tid == 0 && loss_out && s.loss != 0.0f) atomicAdd(loss_out, s.loss);
  teardown_cols(tmem, kGradCols);
}

// One CTA per SM (its tensor memory takes all 512 columns), tiles strided.
cudaError_t launch_grad(const __half* p16, const float* pos, const float* nrm, const float* dir, const float* w,
                        const float* box, uint32_t n, uint32_t offset, const uint32_t* d_count, uint32_t count_cap,
                        float* grad, float* loss, uint32_t* status, cudaStream_t st, bool zero = true) {
  static_assert(sizeof(GradSmem) <= 227 * 1024, "gradient tile exceeds shared memory");
  // the weight gradients are added with 16-byte atomics
  if ((reinterpret_cast<uintptr_t>(grad) & 15u) != 0) return cudaErrorMisalignedAddress;
  const size_t smem = sizeof(GradSmem);
  static bool attr_set[64] = {};  // one attribute call per device (the value never changes)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    e = cudaFuncSetAttribute(grad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  if (zero) {
    if ((e = cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st)) != cudaSuccess) return e;
    if (loss && (e = cudaMemsetAsync(loss, 0, sizeof(float), st)) != cudaSuccess) return e;
  }
  if (n == 0) return cudaSuccess;
  grad_tc_kernel<<<grid_for(n), kRows, smem, st>>>(p16, pos, nrm, dir, w, box, n, offset, d_count, count_cap, grad,
                                                   loss, status);
  return cudaGetLastError();
}

}  // namespace tc

}  // namespace mlp
}  // namespace bajo

extern "C" {

int32_t bajo_mlp_param_count(uint32_t* count) {
  if (!count) return BAJO_ERR_INVALID_ARGUMENT;
  *count = bajo::mlp::kParams;
  return BAJO_OK;
}

int32_t bajo_mlp_forward(const void* d_params16, const float* d_pos, const float* d_nrm, uint32_t n,
                         const float* d_box6, float* d_out20, void* stream) {
  using namespace bajo::mlp;
  if (!d_params16 || !d_box6 || (n && (!d_pos || !d_nrm || !d_out20))) return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  const size_t smem = sizeof(FwdSmem);
  if (cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return BAJO_ERR_CUDA;
  uint64_t grid = ((uint64_t)n + 32 * kWarps - 1) / (32 * kWarps);
  if (grid > 2 * (uint64_t)bajo::sm_count()) grid = 2 * (uint64_t)bajo::sm_count();
  forward_kernel<<<(uint32_t)grid, kThreads, smem, (cudaStream_t)stream>>>((const __half*)d_params16, d_pos, d_nrm,
                                                                         d_box6, n, d_out20);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_mlp_forward_tc(const void* d_params16, const float* d_pos, const float* d_nrm, uint32_t n,
                            const float* d_box6, float* d_out20, uint32_t* d_status, void* stream) {
  using namespace bajo::mlp;
  if (!d_params16 || !d_box6 || (n && (!d_pos || !d_nrm || !d_out20))) return BAJO_ERR_INVALID_ARGUMENT;
  if (n == 0) return BAJO_OK;
  const size_t smem = sizeof(tc::FwdSmem);
  if (cudaFuncSetAttribute(tc::forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return BAJO_ERR_CUDA;
  // one CTA per resident slot: shared memory bounds them (each holds its own
  // copy of the weights and a 16 KB tile), tensor memory (64 of 512 columns)
  // does not
  static int per_sm[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return BAJO_ERR_CUDA;
  if (dev < 0 || dev >= 64) dev = 0;
  if (per_sm[dev] == 0) {
    int sm_bytes = 0;
    cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    per_sm[dev] = max(1, min(8, sm_bytes / (int)(smem + 1024)));
  }
  uint64_t grid = ((uint64_t)n + tc::kRows - 1) / tc::kRows;
  if (grid > (uint64_t)per_sm[dev] * bajo::sm_count()) grid = (uint64_t)per_sm[dev] * bajo::sm_count();
  tc::forward_tc_kernel<<<(uint32_t)grid, tc::kRows, smem, (cudaStream_t)stream>>>(
      (const __half*)d_params16, d_pos, d_nrm, d_box6, n, d_out20, d_status);
  return cudaGetLastError() == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_mlp_grad(const void* d_params16, const float* d_pos, const float* d_nrm, const float* d_dir,
                      const float* d_weight, uint32_t n, const float* d_box6, float* d_grad32, float* d_loss,
                      void* stream) {
  using namespace bajo::mlp;
  if (!d_params16 || !d_box6 || !d_grad32 || (n && (!d_pos || !d_nrm || !d_dir || !d_weight)))
    return BAJO_ERR_INVALID_ARGUMENT;
  const cudaError_t e = launch_grad((const __half*)d_params16, d_pos, d_nrm, d_dir, d_weight, d_box6, n, 0, nullptr,
                                    0, d_grad32, d_loss, (cudaStream_t)stream);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_mlp_grad_tc(const void* d_params16, const float* d_pos, const float* d_nrm, const float* d_dir,
                         const float* d_weight, uint32_t n, const float* d_box6, float* d_grad32, float* d_loss,
                         uint32_t* d_status, void* stream) {
  using namespace bajo::mlp;
  if (!d_params16 || !d_box6 || !d_grad32 || (n && (!d_pos || !d_nrm || !d_dir || !d_weight)))
    return BAJO_ERR_INVALID_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(d_grad32) & 15u) != 0) return BAJO_ERR_INVALID_ARGUMENT;
  const cudaError_t e = tc::launch_grad((const __half*)d_params16, d_pos, d_nrm, d_dir, d_weight, d_box6, n, 0,
                                        nullptr, 0, d_grad32, d_loss, d_status, (cudaStream_t)stream);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_mlp_adam(float* d_params32, void* d_params16, const float* d_grad32, float* d_m, float* d_v,
                      uint32_t step, float lr, float beta1, float beta2, float eps, float grad_scale, void* stream) {
  if (!d_params32 || !d_params16 || !d_grad32 || !d_m || !d_v || step == 0) return BAJO_ERR_INVALID_ARGUMENT;
  // clear = false: the gradient is only read
  const cudaError_t e = bajo::mlp::launch_adam(d_params32, (__half*)d_params16, const_cast<float*>(d_grad32), d_m,
                                               d_v, step, lr, beta1, beta2, eps, grad_scale, (cudaStream_t)stream);
  return e == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_guide_records_size(uint32_t capacity, size_t* bytes) {
  if (!bytes) return BAJO_ERR_INVALID_ARGUMENT;
  *bytes = bajo::mlp::record_layout(capacity).total;
  return BAJO_OK;
}

int32_t bajo_guide_train(BajoGuideNet* net, const void* d_records, uint32_t record_capacity, const float* d_box6,
                         uint32_t batch, uint32_t steps, float lr, void* stream) {
  using namespace bajo::mlp;
  if (!net || !net->params32 || !net->params16 || !net->adam_m || !net->adam_v || !net->grad || !d_records ||
      !d_box6 || record_capacity == 0 || batch == 0 || (reinterpret_cast<uintptr_t>(net->grad) & 15u) != 0)
    return BAJO_ERR_INVALID_ARGUMENT;
  const RecordLayout L = record_layout(record_capacity);
  const unsigned char* r = (const unsigned char*)d_records;
  cudaStream_t st = (cudaStream_t)stream;
  for (uint32_t s = 0; s < steps; ++s) {
    const uint32_t offset = (uint32_t)((uint64_t)net->step * batch % 0xFFFFFFFFull);
    cudaError_t e = tc::launch_grad((const __half*)net->params16, (const float*)(r + L.pos),
                                    (const float*)(r + L.nrm), (const float*)(r + L.dir), (const float*)(r + L.weight),
                                    d_box6, batch, offset, (const uint32_t*)r, record_capacity, net->grad, net->loss,
                                    net->status, st, s == 0);
    if (e != cudaSuccess) return BAJO_ERR_CUDA;
    net->step += 1;
    // Adam clears the gradient and the loss for the next step's accumulation;
    // the last step's stay readable
    e = launch_adam(net->params32, (__half*)net->params16, net->grad, net->adam_m, net->adam_v, net->step, lr, 0.9f,
                    0.999f, 1e-8f, 1.0f / (float)batch, st, s + 1 < steps, net->loss);
    if (e != cudaSuccess) return BAJO_ERR_CUDA;
  }
  return BAJO_OK;
}

}  // extern "C"
