// sort.cu -- C ABI of the standalone onesweep radix sort and the workspace
// status helpers.  Kernels live in onesweep.cuh.
#include <atomic>
#include <mutex>

#include "onesweep.cuh"

namespace bajo {

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = v > 0 ? v : 148;
  }
  return cached[dev];
}

namespace onesweep {

// Tuning table: [64-bit keys][has values][ceil log2 n] -> variant, -1 = the
// built-in choice.  Written by the autotuner through bajo_sort_tuning_set.
static std::atomic<int8_t> g_tuning[2][2][33];
static std::once_flag g_tuning_once;

static void tuning_init() {
  std::call_once(g_tuning_once, [] {
    for (auto& a : g_tuning)
      for (auto& b : a)
        for (auto& c : b) c.store(-1);
  });
}

int tuned_variant(int key_bytes, bool has_values, uint32_t n) {
  tuning_init();
  return g_tuning[key_bytes == 8][has_values ? 1 : 0][ceil_log2(n)].load(std::memory_order_relaxed);
}

}  // namespace onesweep

namespace {

template <typename K, bool HAS_V>
int32_t sort_impl(K* keys, uint32_t* vals, uint32_t n, int32_t begin_bit, int32_t end_bit, void* ws,
                  size_t ws_bytes, void* stream_) {
  constexpr int kBits = (int)sizeof(K) * 8;
  if (begin_bit < 0 || end_bit > kBits || begin_bit > end_bit) return BAJO_ERR_INVALID_ARGUMENT;
  if (n > BAJO_SORT_MAX_KEYS) return BAJO_ERR_TOO_LARGE;
  if (n > 0 && (!keys || (HAS_V && !vals))) return BAJO_ERR_INVALID_ARGUMENT;
  if (!ws) return BAJO_ERR_INVALID_ARGUMENT;
  const uint32_t passes = onesweep::num_passes(begin_bit, end_bit);
  const onesweep::Plan p = onesweep::make_plan<K>(n, HAS_V, passes);
  if (ws_bytes < p.total) return BAJO_ERR_WORKSPACE_TOO_SMALL;
  if (n <= 1 || passes == 0) return BAJO_OK;
  cudaStream_t stream = (cudaStream_t)stream_;
  unsigned char* w = (unsigned char*)ws;
  if (cudaMemsetAsync(w + p.off_zero, 0, p.zero_bytes, stream) != cudaSuccess) return BAJO_ERR_CUDA;
  const int variant = onesweep::choose_variant<K, HAS_V>(n, sm_count());
  const uint32_t bits = onesweep::variant_bits<K>(variant);
  const uint32_t vpasses = onesweep::passes_for(begin_bit, end_bit, bits);
  uint32_t* ghist = (uint32_t*)(w + p.off_ghist);
  const size_t hsmem = onesweep::hist_smem(vpasses, bits);
  uint32_t grid = (n + onesweep::kHistBlock * 16 - 1) / (onesweep::kHistBlock * 16);
  uint32_t max_grid = (uint32_t)sm_count() * 8;
  if (grid > max_grid) grid = max_grid;
  if (grid == 0) grid = 1;
  if (hsmem > 48 * 1024 &&
      cudaFuncSetAttribute(onesweep::global_histogram_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)hsmem) != cudaSuccess)
    return BAJO_ERR_CUDA;
  onesweep::global_histogram_kernel<K><<<grid, onesweep::kHistBlock, hsmem, stream>>>(
      keys, n, (uint32_t)begin_bit, vpasses, (uint32_t)end_bit, bits, ghist);
  if (cudaGetLastError() != cudaSuccess) return BAJO_ERR_CUDA;
  K* kalt = (K*)(w + p.off_keys_alt);
  uint32_t* valt = HAS_V ? (uint32_t*)(w + p.off_vals_alt) : nullptr;
  bool in_first = true;
  if (onesweep::run_passes<K, HAS_V>(keys, vals, kalt, valt, nullptr, p, w, begin_bit, end_bit, stream,
                                     &in_first, variant) != cudaSuccess)
    return BAJO_ERR_CUDA;
  if (!in_first) {
    // odd pass count: bring the result back into the caller's buffers
    if (cudaMemcpyAsync(keys, kalt, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return BAJO_ERR_CUDA;
    if (HAS_V && cudaMemcpyAsync(vals, valt, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
      return BAJO_ERR_CUDA;
  }
  return BAJO_OK;
}

}  // namespace
}  // namespace bajo

extern "C" {

int32_t bajo_workspace_status(const void* ws, void* stream, uint32_t* status) {
  if (!ws || !status) return BAJO_ERR_INVALID_ARGUMENT;
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return BAJO_ERR_CUDA;
  if (cudaMemcpy(status, ws, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return BAJO_ERR_CUDA;
  return BAJO_OK;
}

int32_t bajo_workspace_status_clear(void* ws, void* stream) {
  if (!ws) return BAJO_ERR_INVALID_ARGUMENT;
  return cudaMemsetAsync(ws, 0, 4, (cudaStream_t)stream) == cudaSuccess ? BAJO_OK : BAJO_ERR_CUDA;
}

int32_t bajo_sort_workspace_size(uint32_t n, uint32_t key_bytes, int32_t has_values, int32_t begin_bit,
                                 int32_t end_bit, size_t* bytes) {
  using namespace bajo::onesweep;
  if (!bytes || (key_bytes != 4 && key_bytes != 8)) return BAJO_ERR_INVALID_ARGUMENT;
  if (begin_bit < 0 || end_bit > (int)key_bytes * 8 || begin_bit > end_bit) return BAJO_ERR_INVALID_ARGUMENT;
  if (n > BAJO_SORT_MAX_KEYS) return BAJO_ERR_TOO_LARGE;
  const uint32_t passes = num_passes(begin_bit, end_bit);
  *bytes = key_bytes == 4 ? make_plan<uint32_t>(n, has_values != 0, passes).total
                          : make_plan<uint64_t>(n, has_values != 0, passes).total;
  return BAJO_OK;
}

int32_t bajo_sort_tuning_set(uint32_t key_bytes, int32_t has_values, uint32_t log2n, int32_t variant) {
  using namespace bajo::onesweep;
  if ((key_bytes != 4 && key_bytes != 8) || log2n > 32 || variant < -1 ||
      variant >= (key_bytes == 4 ? Shapes<uint32_t>::count : Shapes<uint64_t>::count))
    return BAJO_ERR_INVALID_ARGUMENT;
  if (variant >= 0) {
    const uint32_t n = log2n >= 32 ? 0xFFFFFFFFu : (1u << log2n);
    if (key_bytes == 4 ? !variant_allowed<uint32_t>(variant, n) : !variant_allowed<uint64_t>(variant, n))
      return BAJO_ERR_INVALID_ARGUMENT;
  }
  tuned_variant(4, false, 1);  // initialise the table
  g_tuning[key_bytes == 8][has_values ? 1 : 0][log2n].store((int8_t)variant);
  return BAJO_OK;
}

int32_t bajo_sort_tuning_get(uint32_t key_bytes, int32_t has_values, uint32_t n, int32_t* variant) {
  using namespace bajo::onesweep;
  if ((key_bytes != 4 && key_bytes != 8) || !variant) return BAJO_ERR_INVALID_ARGUMENT;
  const int sms = bajo::sm_count();
  *variant = key_bytes == 4 ? (has_values ? choose_variant<uint32_t, true>(n, sms)
                                          : choose_variant<uint32_t, false>(n, sms))
                            : (has_values ? choose_variant<uint64_t, true>(n, sms)
                                          : choose_variant<uint64_t, false>(n, sms));
  return BAJO_OK;
}

int32_t bajo_sort_keys_u32(uint32_t* k, uint32_t n, int32_t b, int32_t e, void* ws, size_t wb, void* s) {
  return bajo::sort_impl<uint32_t, false>(k, nullptr, n, b, e, ws, wb, s);
}
int32_t bajo_sort_pairs_u32(uint32_t* k, uint32_t* v, uint32_t n, int32_t b, int32_t e, void* ws, size_t wb,
                            void* s) {
  return bajo::sort_impl<uint32_t, true>(k, v, n, b, e, ws, wb, s);
}
int32_t bajo_sort_keys_u64(uint64_t* k, uint32_t n, int32_t b, int32_t e, void* ws, size_t wb, void* s) {
  return bajo::sort_impl<uint64_t, false>(k, nullptr, n, b, e, ws, wb, s);
}
int32_t bajo_sort_pairs_u64(uint64_t* k, uint32_t* v, uint32_t n, int32_t b, int32_t e, void* ws, size_t wb,
                            void* s) {
  return bajo::sort_impl<uint64_t, true>(k, v, n, b, e, ws, wb, s);
}

const char* bajo_version(void) { return "bajo_b200 0.1 (sm_100a)"; }

}  // extern "C"
