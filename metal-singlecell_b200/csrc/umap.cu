// UMAP fuzzy-set pieces and the distances CSR.
//
// Reference: umap-learn 0.5.12 `fuzzy_simplicial_set` as metalsinglecell calls it
// (neighbors.py:742-753: set_op_mix_ratio=1, local_connectivity=1) and the distances graph of
// neighbors.py:755-759.  umap-learn keeps its bisection state in float32 (numba locals); these
// kernels fix that arithmetic exactly — float32 state, sums in column order, IEEE float32
// division, exp evaluated in FP64 and rounded once to float32 — so that the results are
// reproducible bit for bit against the CPU restatement.
#include "kernels.cuh"

namespace msc {

namespace {

constexpr float SMOOTH_K_TOLERANCE = 1e-5f;
constexpr double MIN_K_DIST_SCALE = 1e-3;
constexpr int SK_THREADS = 128;

// FP64 sum of all n·k distances: per-block partials, then one block adds them in order
__global__ void dist_sum_partial_kernel(const float* __restrict__ dist, int64_t total,
                                        double* __restrict__ partial) {
  __shared__ double red[256];
  double a = 0.0;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x)
    a += double(dist[e]);
  red[threadIdx.x] = a;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void dist_sum_final_kernel(const double* __restrict__ partial, int nb,
                                      double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0.0;
    for (int b = 0; b < nb; ++b) a += partial[b];
    *out = a;
  }
}

__global__ void __launch_bounds__(SK_THREADS)
smooth_knn_kernel(const float* __restrict__ dist, int64_t n, int k, float local_connectivity,
                  const double* __restrict__ gsum, float* __restrict__ sigma,
                  float* __restrict__ rho_out) {
  extern __shared__ float sd[];                    // [SK_THREADS][k]
  const int64_t row0 = int64_t(blockIdx.x) * SK_THREADS;
  const int nrows = int(min64(SK_THREADS, n - row0));
  for (int e = threadIdx.x; e < nrows * k; e += SK_THREADS) sd[e] = dist[row0 * k + e];
  __syncthreads();
  if (threadIdx.x >= nrows) return;
  const int64_t i = row0 + threadIdx.x;
  const float* D = sd + threadIdx.x * k;
  const double target = log2(double(k));
  // rho
  int nz = 0;
  for (int j = 0; j < k; ++j) nz += D[j] > 0.f;
  const int index = int(floor(double(local_connectivity)));
  const double interpolation = double(local_connectivity) - index;
  auto nth_nonzero = [&](int r) -> float {      // r-th (1-based) non-zero in row order
    int c = 0;
    for (int j = 0; j < k; ++j)
      if (D[j] > 0.f && ++c == r) return D[j];
    return 0.f;
  };
  float rho = 0.f;
  if (double(nz) >= double(local_connectivity)) {
    if (index > 0) {
      rho = nth_nonzero(index);
      if (interpolation > double(SMOOTH_K_TOLERANCE)) {
        float nxt = nth_nonzero(index + 1);
        rho = __double2float_rn(double(rho) + interpolation * double(nxt - rho));
      }
    } else {
      rho = __double2float_rn(interpolation * double(nth_nonzero(1)));
    }
  } else if (nz > 0) {
    float m = 0.f;
    for (int j = 0; j < k; ++j) if (D[j] > 0.f) m = fmaxf(m, D[j]);
    rho = m;
  }
  // bisection for sigma (float32 state, column order)
  float lo = 0.f, hi = __int_as_float(0x7f800000), mid = 1.f;
  for (int it = 0; it < 64; ++it) {
    float psum = 0.f;
    for (int j = 1; j < k; ++j) {
      const float dd = __fsub_rn(D[j], rho);
      if (dd > 0.f) psum = __fadd_rn(psum, exp_f32(-__fdiv_rn(dd, mid)));
      else psum = __fadd_rn(psum, 1.f);
    }
    const double p64 = double(psum);
    if (fabs(p64 - target) < double(SMOOTH_K_TOLERANCE)) break;
    if (p64 > target) {
      hi = mid;
      mid = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
    } else {
      lo = mid;
      if (isinf(hi)) mid = __fmul_rn(mid, 2.f);
      else mid = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
    }
  }
  float result = mid;
  if (rho > 0.f) {
    float rs = 0.f;
    for (int j = 0; j < k; ++j) rs = __fadd_rn(rs, D[j]);
    const double fl = MIN_K_DIST_SCALE * (double(rs) / double(k));
    if (double(result) < fl) result = __double2float_rn(fl);
  } else {
    const double fl = MIN_K_DIST_SCALE * (*gsum / (double(n) * double(k)));
    if (double(result) < fl) result = __double2float_rn(fl);
  }
  sigma[i] = result;
  rho_out[i] = rho;
}

__global__ void membership_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist,
                                  const float* __restrict__ sigma, const float* __restrict__ rho,
                                  int64_t n, int k, float* __restrict__ w) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n * k;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / k;
    float val;
    if (idx[e] == i) {
      val = 0.f;
    } else {
      const float dd = __fsub_rn(dist[e], rho[i]);
      const float sg = sigma[i];
      if (dd <= 0.f || sg == 0.f) val = 1.f;
      else val = exp_f32(-__fdiv_rn(dd, sg));
    }
    w[e] = val;
  }
}

// distances CSR (neighbors.py:755-759): row i holds knn columns 1..k-1 sorted by column index;
// a warp per row computes each entry's rank among the row's columns (columns are distinct)
constexpr int DC_WARPS = 8;
__global__ void __launch_bounds__(DC_WARPS * 32)
distances_csr_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist, int64_t n,
                     int k, int64_t* __restrict__ indptr, int32_t* __restrict__ indices,
                     float* __restrict__ data) {
  __shared__ int32_t cols_all[DC_WARPS][MSC_MAX_K];
  const int lane = lane_id(), wib = warp_id();
  int32_t* cols = cols_all[wib];
  const int m = k - 1;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    for (int e = lane; e < m; e += 32) cols[e] = idx[i * k + 1 + e];
    __syncwarp();
    for (int e = lane; e < m; e += 32) {
      const int32_t c = cols[e];
      int r = 0;
      for (int f = 0; f < m; ++f) r += cols[f] < c;
      indices[i * m + r] = c;
      data[i * m + r] = dist[i * k + 1 + e];
    }
    if (lane == 0) indptr[i] = i * m;
    if (lane == 0 && i == n - 1) indptr[n] = n * m;
    __syncwarp();
  }
}

// gauss: σ_i² = median of the squared distances to the k-1 other neighbours (FP64)
__global__ void __launch_bounds__(DC_WARPS * 32)
gauss_sigma_kernel(const float* __restrict__ dist, int64_t n, int k, double* __restrict__ sig2) {
  __shared__ double sq_all[DC_WARPS][MSC_MAX_K];
  const int lane = lane_id(), wib = warp_id();
  double* sq = sq_all[wib];
  const int m = k - 1;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    for (int e = lane; e < m; e += 32) {
      const double v = double(dist[i * k + 1 + e]);
      sq[e] = v * v;
    }
    __syncwarp();
    // the values at sorted positions (m-1)/2 and m/2, ties by position
    double lo_v = 0.0, hi_v = 0.0;
    for (int e = lane; e < m; e += 32) {
      const double v = sq[e];
      int r = 0;
      for (int f = 0; f < m; ++f) r += (sq[f] < v) || (sq[f] == v && f < e);
      if (r == (m - 1) / 2) lo_v = v;
      if (r == m / 2) hi_v = v;
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo_v += __shfl_xor_sync(FULL, lo_v, o);
      hi_v += __shfl_xor_sync(FULL, hi_v, o);
    }
    if (lane == 0) sig2[i] = m == 0 ? 0.0 : ((m & 1) ? lo_v : (lo_v + hi_v) * 0.5);
    __syncwarp();
  }
}

}  // namespace

int launch_smooth_knn(const float* dist, int64_t n, int k, float local_connectivity,
                      float* sigma, float* rho, double* gsum, cudaStream_t st) {
  // gsum: workspace of >= 1 + 1024 doubles (total at [0], partials after)
  const int nb = int(std::min<int64_t>(1024, std::max<int64_t>(1, ceil_div(n * k, 4096))));
  dist_sum_partial_kernel<<<nb, 256, 0, st>>>(dist, n * k, gsum + 1);
  MSC_LAUNCH_CHECK();
  dist_sum_final_kernel<<<1, 32, 0, st>>>(gsum + 1, nb, gsum);
  MSC_LAUNCH_CHECK();
  const size_t smem = size_t(SK_THREADS) * k * sizeof(float);
  if (smem > 48 * 1024)
    MSC_CUDA_TRY(raise_smem_cap(smooth_knn_kernel, smem));
  smooth_knn_kernel<<<unsigned(ceil_div(n, SK_THREADS)), SK_THREADS, smem, st>>>(
      dist, n, k, local_connectivity, gsum, sigma, rho);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_membership(const int32_t* idx, const float* dist, const float* sigma,
                      const float* rho, int64_t n, int k, float* w, cudaStream_t st) {
  int blocks = int(std::min<int64_t>(ceil_div(n * k, 256), int64_t(num_sms()) * 16));
  membership_kernel<<<std::max(blocks, 1), 256, 0, st>>>(idx, dist, sigma, rho, n, k, w);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_distances_csr(const int32_t* idx, const float* dist, int64_t n, int k,
                         int64_t* indptr, int32_t* indices, float* data, cudaStream_t st) {
  int blocks = int(std::min<int64_t>(ceil_div(n, DC_WARPS), int64_t(num_sms()) * 16));
  distances_csr_kernel<<<std::max(blocks, 1), DC_WARPS * 32, 0, st>>>(idx, dist, n, k, indptr,
                                                                       indices, data);
  MSC_LAUNCH_CHECK();
  if (n == 0) return MSC_OK;
  return MSC_OK;
}

int launch_gauss_sigma(const float* dist, int64_t n, int k, double* sig2, cudaStream_t st) {
  int blocks = int(std::min<int64_t>(ceil_div(n, DC_WARPS), int64_t(num_sms()) * 16));
  gauss_sigma_kernel<<<std::max(blocks, 1), DC_WARPS * 32, 0, st>>>(dist, n, k, sig2);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
