// Fuzzy union without caller-provided scratch (msc_fuzzy_union_noalloc).
//
// Some callers cannot hand the library a scratch buffer: code running under a memory manager
// that owns all device memory (a framework's caching allocator, a serving process that reserves
// its HBM up front and gives plug-ins no allocator), or a hot loop where cudaMalloc/cudaFree —
// which may synchronise the device — are not acceptable.  This entry point runs the same kernels
// as msc_fuzzy_union but takes its scratch from a fixed array in the library's own device memory,
// so it allocates nothing.  Its size bounds the problems it accepts (see msc_b200.h).
#include <mutex>
#include <unordered_map>

#include "kernels.cuh"

namespace msc {

namespace {

// Scratch of the no-allocation union: large enough for union_workspace_bytes(n, k) whenever
// n <= MSC_NOALLOC_MAX_CELLS and n·k <= MSC_NOALLOC_MAX_ENTRIES (checked on every call).
// Every GPU that loads the library holds this array until the process exits.
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(20) << 20;      // 20 MiB
static __device__ __align__(256) unsigned char g_union_scratch[NOALLOC_SCRATCH_BYTES];

// Host code cannot use g_union_scratch as a device address; the address is looked up once per
// device (with that device current) and cached.
int scratch_address(void** out) {
  static std::mutex mu;
  static std::unordered_map<int, void*> cache;
  int dev = -1;
  MSC_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) {
    *out = it->second;
    return MSC_OK;
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_union_scratch);
  if (e != cudaSuccess || p == nullptr) {
    set_error("cudaGetSymbolAddress(g_union_scratch) failed on device %d: %s", dev,
              cudaGetErrorString(e));
    return MSC_ERR_CUDA;
  }
  cache[dev] = p;
  *out = p;
  return MSC_OK;
}

}  // namespace
}  // namespace msc

using namespace msc;

extern "C" int msc_fuzzy_union_noalloc(const int32_t* knn_idx_dev, const float* w_dev, int64_t n,
                                       int32_t k, int64_t* indptr_dev, int32_t* indices_dev,
                                       float* data_dev, int64_t* nnz_dev, void* stream) {
  if (n < 1 || k < 1 || k > MSC_MAX_K) {
    set_error("msc_fuzzy_union_noalloc: bad n=%lld / k=%d", (long long)n, k);
    return MSC_ERR_INVALID_ARG;
  }
  if (n > MSC_NOALLOC_MAX_CELLS || n * int64_t(k) > MSC_NOALLOC_MAX_ENTRIES) {
    set_error("msc_fuzzy_union_noalloc: n=%lld, n*k=%lld exceed the fixed scratch "
              "(n <= %d, n*k <= %d); use msc_fuzzy_union with a workspace",
              (long long)n, (long long)(n * k), MSC_NOALLOC_MAX_CELLS, MSC_NOALLOC_MAX_ENTRIES);
    return MSC_ERR_INVALID_ARG;
  }
  if (!knn_idx_dev || !w_dev || !indptr_dev || !indices_dev || !data_dev) {
    set_error("msc_fuzzy_union_noalloc: NULL pointer argument");
    return MSC_ERR_INVALID_ARG;
  }
  const size_t need = union_workspace_bytes(n, k);
  if (need > NOALLOC_SCRATCH_BYTES) {
    set_error("msc_fuzzy_union_noalloc: needs %zu bytes of scratch, the fixed array has %zu",
              need, NOALLOC_SCRATCH_BYTES);
    return MSC_ERR_INVALID_ARG;
  }
  void* scratch = nullptr;
  MSC_TRY(scratch_address(&scratch));
  // launch_union clears the counters it needs at zero before use; the rest of the array is
  // written before it is read, so the previous call's contents do not matter
  return launch_union(0, knn_idx_dev, w_dev, nullptr, n, k, indptr_dev, indices_dev, data_dev,
                      nnz_dev, scratch, NOALLOC_SCRATCH_BYTES, static_cast<cudaStream_t>(stream));
}
