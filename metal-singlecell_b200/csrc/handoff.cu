// Edge preparation of the UMAP layout, on the device, from a connectivities CSR that is already in
// HBM (the hand-off from the neighbour graph to its first consumer, without a host round trip).
//
// Reference: metalsinglecell embedding.py.  `umap()` first drops the edges too weak to be sampled
// once over the run (`_prune_weak_edges`, embedding.py:255-267: keep w >= max(w) / n_epochs, the
// division in float32 — NumPy 2 keeps a float32 scalar divided by a Python float in float32), then
// takes the kept graph as COO in CSR order (`graph.tocoo()`, embedding.py:115) and derives each
// edge's sampling period (`_make_epochs_per_sample`, embedding.py:123-137, in FP64:
// n_epochs / (n_epochs · (w / max w)), -1 for an edge never sampled).
//
// Kernels: (1) the largest weight (a max of non-negative float32 values, exact in any order);
// (2) kept entries per row; (3) exclusive scan into the kept graph's row pointers; (4) per row,
// the kept entries compacted in their CSR order with their row, column, weight and period.
#include "kernels.cuh"

namespace msc {

namespace {

constexpr int HW = 8;        // warps per block in the warp-per-row kernels

__global__ void weight_max_kernel(const float* __restrict__ data, const int64_t* __restrict__ nnz,
                                  unsigned* __restrict__ wmax_bits) {
  const int64_t m = *nnz;
  float mx = 0.f;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < m;
       e += int64_t(gridDim.x) * blockDim.x)
    mx = fmaxf(mx, data[e]);
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
  if (lane_id() == 0 && mx > 0.f) atomic_max_nonneg(wmax_bits, mx);
}

__device__ __forceinline__ float keep_threshold(const unsigned* wmax_bits, int n_epochs) {
  return __fdiv_rn(__uint_as_float(*wmax_bits), float(n_epochs));
}

__global__ void __launch_bounds__(HW * 32)
kept_count_kernel(const int64_t* __restrict__ indptr, const float* __restrict__ data, int64_t n,
                  int n_epochs, const unsigned* __restrict__ wmax_bits,
                  int32_t* __restrict__ kept) {
  const float thr = keep_threshold(wmax_bits, n_epochs);
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int64_t a = indptr[i], b = indptr[i + 1];
    int c = 0;
    for (int64_t e = a + lane; e < b; e += 32) c += data[e] >= thr ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
    if (lane == 0) kept[i] = c;
  }
}

__global__ void __launch_bounds__(HW * 32)
compact_kernel(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
               const float* __restrict__ data, int64_t n, int n_epochs,
               const unsigned* __restrict__ wmax_bits, const int64_t* __restrict__ out_ptr,
               int32_t* __restrict__ rows, int32_t* __restrict__ cols,
               float* __restrict__ weights, double* __restrict__ eps) {
  const float thr = keep_threshold(wmax_bits, n_epochs);
  // the kept graph's largest weight is the input's (the largest entry is always kept)
  const double wmax = double(__uint_as_float(*wmax_bits));
  const double ne = double(n_epochs);
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int64_t a = indptr[i], b = indptr[i + 1];
    int64_t o = out_ptr[i];
    for (int64_t e0 = a; e0 < b; e0 += 32) {
      const int64_t e = e0 + lane;
      const float w = e < b ? data[e] : 0.f;
      const bool keep = e < b && w >= thr;
      const unsigned m = __ballot_sync(FULL, keep);
      if (keep) {
        const int64_t p = o + __popc(m & ((1u << lane) - 1u));
        rows[p] = int32_t(i);
        cols[p] = indices[e];
        weights[p] = w;
        const double ns = __dmul_rn(ne, __ddiv_rn(double(w), wmax));
        eps[p] = ns > 0.0 ? __ddiv_rn(ne, ns) : -1.0;
      }
      o += __popc(m);
    }
  }
}

struct EdgeWs {
  unsigned* wmax;
  int32_t* kept;
  int64_t* scan;
};

EdgeWs carve_edges(Carver& c, int64_t n) {
  EdgeWs w;
  w.wmax = c.take<unsigned>(8);
  w.kept = c.take<int32_t>(n);
  w.scan = c.take<int64_t>(scan_i32_scratch_elems(n));
  return w;
}

}  // namespace

size_t umap_edges_workspace_bytes(int64_t n) {
  Carver c(nullptr);
  carve_edges(c, n);
  return c.bytes();
}

int launch_umap_edges(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n,
                      int n_epochs, int64_t* out_ptr, int32_t* rows, int32_t* cols,
                      float* weights, double* eps, void* ws, cudaStream_t st) {
  Carver c(ws);
  EdgeWs w = carve_edges(c, n);
  MSC_CUDA_TRY(cudaMemsetAsync(w.wmax, 0, sizeof(unsigned), st));
  const int sms = num_sms();
  weight_max_kernel<<<sms * 4, 256, 0, st>>>(data, indptr + n, w.wmax);
  MSC_LAUNCH_CHECK();
  const int g = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, HW), int64_t(sms) * 16)));
  kept_count_kernel<<<g, HW * 32, 0, st>>>(indptr, data, n, n_epochs, w.wmax, w.kept);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl_i32(w.kept, n, out_ptr, w.scan, st));
  compact_kernel<<<g, HW * 32, 0, st>>>(indptr, indices, data, n, n_epochs, w.wmax, out_ptr, rows,
                                        cols, weights, eps);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
