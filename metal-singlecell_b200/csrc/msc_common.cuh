// Shared definitions of the msc_b200 CUDA library: status plumbing, the workspace carver, the
// tile plan shared by the candidate kernels, and small exact-arithmetic helpers.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stddef.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "msc_b200.h"          // include/ is on the include path

namespace msc {

// ------------------------------------------------------------------------------------------------
// host-side error plumbing
// ------------------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
const char* last_error();

// kernels launched by this library (counted after every launch)
extern std::atomic<long long> g_launch_count;

// optional CUDA-event marks between pipeline stages (process-global instrumentation)
void stage_mark(cudaStream_t st, int stage);

#define MSC_CUDA_TRY(expr)                                                                     \
  do {                                                                                         \
    cudaError_t _e = (expr);                                                                   \
    if (_e != cudaSuccess) {                                                                   \
      ::msc::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__,      \
                       __LINE__);                                                              \
      return MSC_ERR_CUDA;                                                                     \
    }                                                                                          \
  } while (0)

#define MSC_LAUNCH_CHECK()                                                                     \
  do {                                                                                         \
    ::msc::g_launch_count.fetch_add(1, std::memory_order_relaxed);                             \
    cudaError_t _e = cudaGetLastError();                                                       \
    if (_e != cudaSuccess) {                                                                   \
      ::msc::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(_e), __FILE__,  \
                       __LINE__);                                                              \
      return MSC_ERR_CUDA;                                                                     \
    }                                                                                          \
  } while (0)

#define MSC_TRY(expr)                                                                          \
  do {                                                                                         \
    int _s = (expr);                                                                           \
    if (_s != MSC_OK) return _s;                                                               \
  } while (0)

// ------------------------------------------------------------------------------------------------
// Workspace carver: the same sequence of take() calls sizes the workspace (base == nullptr) and
// later hands out the pieces; every piece is 256-byte aligned.
// ------------------------------------------------------------------------------------------------
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base(static_cast<char*>(b)) {}
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
  size_t bytes() const { return (off + 255) & ~size_t(255); }
};

// ------------------------------------------------------------------------------------------------
// Tile plan.  Cells of sample s (original rows [off_s, off_s + n_s)) are laid out in "packed"
// row space at [poff_s, poff_s + pad(n_s)), pad = multiple of SEG_PAD, so that no 128-row query
// tile and no key tile (64/128/256 rows) straddles two samples.
// ------------------------------------------------------------------------------------------------
constexpr int SEG_PAD = 256;
constexpr int QTILE = 128;

struct WorkItem {
  int32_t qrow0;      // packed row of the first query of this tile
  int32_t nq;         // valid queries in the tile (<= 128)
  int32_t key0;       // packed row of the sample's first key
  int32_t nkeys;      // valid keys of the sample (n_s)
  int32_t orig_off;   // original row of the sample's first cell
  int32_t qorig0;     // original row of the tile's first query (orig_off + qrow0 - key0)
  int32_t pad0, pad1;
};

// per-row statistics of the query operand, for the certification bound
struct QStat {
  double sq;          // Σ z_t² (z = scaled, centred row), exact in FP64
  float hi;           // |a_hi|  (norm of the rounded operand)
  float lo;           // |a_lo|  (norm of the second split term; 0 for one-term precisions)
  float res;          // |z - a_hi - a_lo|  (what the operand terms do not represent)
  float pad;
};

// maxima over all keys (float bits, values >= 0, combined with atomicMax on the bit pattern)
struct KeyMax {
  unsigned hi, lo, res, nerr, sq, pad0, pad1, pad2;
};

// device-side control block written by the kernels and read back by the host
struct Ctl {
  int64_t stats[MSC_STATS_LEN];
  int32_t item_counter;     // dynamic work distribution of the persistent candidate kernels
  int32_t n_items;
  int32_t n_fail;           // rows that failed certification
  int32_t timeout_flag;
  double colsum_scale;      // scale factor f applied to the centred rows (power of two)
  unsigned max_sq_bits;     // max Σ z² over rows (before scaling), float bits
  int32_t n_refine;         // rows compacted for the BF16x3 refine pass
  int32_t n_items_refine;   // query tiles of the refine pass
  int32_t tc_counter[3];    // item counters of the tensor-core launches (main, refine, near)
  int32_t refine_split;     // work items per refine item (key ranges), 1 = not split
  int32_t n_items_refine_eff;   // n_items_refine × refine_split
  int32_t ordered_ok;           // 1: every work item's sorted visit list fits (prune.cu)
  int32_t pad2[2];
};

// ------------------------------------------------------------------------------------------------
// device helpers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float exp_f32(float z) {
  // exp of a float32 argument, evaluated in FP64 and rounded once to float32
  return __double2float_rn(exp(static_cast<double>(z)));
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned* addr, float v) {
  atomicMax(addr, __float_as_uint(v));
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }

constexpr unsigned FULL = 0xffffffffu;
constexpr float F_INF = __builtin_huge_valf();

__host__ __device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// number of SMs of the current device (cached per device)
int num_sms();

// Raise a kernel's dynamic shared-memory cap (cudaFuncAttributeMaxDynamicSharedMemorySize) to at
// least `bytes`, never lowering it.  The attribute is per function and process-wide: when host
// threads launch the same kernel with different sizes, one thread setting a smaller cap between
// another's set and launch makes that launch fail ("too many resources requested").  Raising only,
// under one lock, leaves every cap at the largest size any caller asked for.
cudaError_t raise_smem_cap_fn(const void* func, size_t bytes);
template <typename K>
inline cudaError_t raise_smem_cap(K* kern, size_t bytes) {
  return raise_smem_cap_fn(reinterpret_cast<const void*>(kern), bytes);
}

// Blocks of `threads` threads and `smem` dynamic shared-memory bytes that fit on one SM at once
// (the occupancy query, cached per kernel, device and shape; at least 1).  A grid-stride kernel
// launched with more blocks than the SMs hold runs a second, partly filled wave.
int resident_blocks_fn(const void* func, int threads, size_t smem);
template <typename K>
inline int resident_grid(K* kern, int threads, size_t smem, int64_t work_blocks) {
  const int64_t full = int64_t(num_sms()) *
                       resident_blocks_fn(reinterpret_cast<const void*>(kern), threads, smem);
  return int(max64(1, min64(work_blocks, full)));
}

}  // namespace msc
