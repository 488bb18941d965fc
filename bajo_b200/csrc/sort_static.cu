// sort_static.cu -- a radix sort entry point that allocates nothing.
//
// Some callers of this library cannot call cudaMalloc or hand the library a
// workspace: a host that owns every device allocation itself and passes only
// the buffers it computes on (for example a plugin host or a language runtime
// whose device arena is fixed at start-up), or a real-time frame loop where an
// allocation would stall the device.  bajo_sort_pairs_u32_noalloc serves them:
// its scratch (alternate key / value buffers, digit histograms, look-back
// flags) lives in one file-scope __device__ array of fixed size, so the caller
// passes only the keys and values.
//
// Costs and rules:
//  - every GPU that loads the library holds kNoAllocScratchBytes of device
//    memory for this array until the process exits;
//  - n is limited to BAJO_SORT_NOALLOC_MAX_KEYS; larger calls are rejected
//    with BAJO_ERR_TOO_LARGE before any device work;
//  - all calls on a device share the one array: calls whose device work
//    overlaps (different streams, or several host threads) race on it and
//    must be serialised by the caller;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  Calls made outside a capture look the
//    address up again (a host-side table lookup), so a device reset, after
//    which the module and its array may be loaded elsewhere, is picked up by
//    the next uncaptured call; captured calls use the address cached last.
#include <mutex>

#include "onesweep.cuh"

namespace bajo {

int sm_count();

namespace {

constexpr uint32_t kNoAllocMaxKeys = BAJO_SORT_NOALLOC_MAX_KEYS;
constexpr uint32_t kNoAllocPasses = 4;  // 32-bit keys, 8-bit digits

// Scratch layout of a 32-bit key / 32-bit value sort of kNoAllocMaxKeys keys
// (onesweep::make_plan): status word, histograms, tile counters, look-back
// flags, alternate keys, alternate values.  Computed at compile time so the
// array has a fixed size; smaller sorts use a prefix-compatible, smaller plan.
constexpr size_t kNoAllocScratchBytes =
    onesweep::make_plan<uint32_t>(kNoAllocMaxKeys, true, kNoAllocPasses).total;
static_assert(kNoAllocScratchBytes == BAJO_SORT_NOALLOC_SCRATCH_BYTES,
              "the header's scratch size must follow the sort plan");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// names a host-side stand-in, not device memory, so the address must come
// from cudaGetSymbolAddress with the device current.
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {};

cudaError_t noalloc_scratch(cudaStream_t stream, void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(stream, &capture);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev] || capture == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace bajo

extern "C" int32_t bajo_sort_pairs_u32_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, int32_t begin_bit,
                                               int32_t end_bit, uint32_t* d_status, void* stream_) {
  using namespace bajo;
  if (begin_bit < 0 || end_bit > 32 || begin_bit > end_bit) return BAJO_ERR_INVALID_ARGUMENT;
  if (n > kNoAllocMaxKeys) return BAJO_ERR_TOO_LARGE;
  if (n > 0 && (!d_keys || !d_vals)) return BAJO_ERR_INVALID_ARGUMENT;
  const uint32_t passes = onesweep::num_passes(begin_bit, end_bit);
  const onesweep::Plan p = onesweep::make_plan<uint32_t>(n, true, passes);
  if (p.total > kNoAllocScratchBytes) return BAJO_ERR_TOO_LARGE;
  cudaStream_t stream = (cudaStream_t)stream_;
  void* base = nullptr;
  if (noalloc_scratch(stream, &base) != cudaSuccess) return BAJO_ERR_CUDA;
  unsigned char* w = (unsigned char*)base;
  // the array keeps the previous call's contents: clear the status word and
  // every counter / flag that must start at zero
  if (cudaMemsetAsync(w, 0, 4, stream) != cudaSuccess) return BAJO_ERR_CUDA;
  if (n > 1 && passes > 0) {
    if (cudaMemsetAsync(w + p.off_zero, 0, p.zero_bytes, stream) != cudaSuccess) return BAJO_ERR_CUDA;
    uint32_t* ghist = (uint32_t*)(w + p.off_ghist);
    const size_t hsmem = onesweep::hist_smem(passes, 8);  // 32-bit keys: 8-bit digits only
    uint32_t grid = (n + onesweep::kHistBlock * 16 - 1) / (onesweep::kHistBlock * 16);
    const uint32_t max_grid = (uint32_t)sm_count() * 4;
    if (grid > max_grid) grid = max_grid;
    if (grid == 0) grid = 1;
    onesweep::global_histogram_kernel<uint32_t><<<grid, onesweep::kHistBlock, hsmem, stream>>>(
        d_keys, n, (uint32_t)begin_bit, passes, (uint32_t)end_bit, 8u, ghist);
    if (cudaGetLastError() != cudaSuccess) return BAJO_ERR_CUDA;
    uint32_t* kalt = (uint32_t*)(w + p.off_keys_alt);
    uint32_t* valt = (uint32_t*)(w + p.off_vals_alt);
    bool in_first = true;
    const int variant = onesweep::choose_variant<uint32_t, true>(n, sm_count());
    if (onesweep::run_passes<uint32_t, true>(d_keys, d_vals, kalt, valt, nullptr, p, w, begin_bit, end_bit, stream,
                                             &in_first, variant) != cudaSuccess)
      return BAJO_ERR_CUDA;
    if (!in_first) {
      if (cudaMemcpyAsync(d_keys, kalt, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
          cudaMemcpyAsync(d_vals, valt, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
        return BAJO_ERR_CUDA;
    }
  }
  if (d_status && cudaMemcpyAsync(d_status, w, 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    return BAJO_ERR_CUDA;
  return BAJO_OK;
}
