// Batch-balanced kNN: metalsinglecell `neighbors.bbknn` (neighbors.py:491-559) and its trimming
// `_trim_graph` (neighbors.py:465-488), called by `pp.bbknn` (pp.py:809-833).
//
// Every cell gets, for every batch b, its kk_b = min(k, n_b) nearest cells of b (a cell of b finds
// itself at distance 0); the K = Σ kk_b entries of a cell are merged by (distance, index) and go
// through the same fuzzy simplicial set as pp.neighbors.  The reference scans each batch by brute
// force in FP32 (the n × n_b Gram matrix, neighbors.py:525-537); here the lists are exact:
//
//   layout   cells grouped by batch as the key side, batch b at packed rows [poff_b, poff_b + n_b)
//            (ascending cell index, each batch padded to SEG_PAD rows), and every cell once more
//            in a query region [P1, P1 + n) whose positions are never key columns, so the
//            candidate kernel's self-exclusion never drops a cell's own copy;
//   operands one centring (the mean of all cells) and one FP16 scale for both sides;
//   scan     per batch, one launch of the tensor-core candidate kernel in its row-list mode:
//            query tiles of 128 listed cells against the batch's key range, k' candidates per
//            cell and the k'-th value bounding every key left out;
//   re-rank  FP32 direct differences of the candidates, FP64 at the kk-th boundary, order by
//            (FP64 squared distance, index), and the same certificate as the self-kNN path; the
//            cells it cannot certify take an FP64 scan of the batch;
//   merge    every cell's K entries sorted by (float32 distance, index).
//
// The distances graph drops the diagonal and every zero distance (neighbors.py:554-557); the
// trimming keeps an entry (i, j) of value v when v != 0, v >= θ_i and v >= θ_j, θ_i being the
// trim-th largest stored value of row i when the row stores more than `trim` entries, else 0.
#include <algorithm>

#include "kernels.cuh"
#include "msc_warpsort.cuh"

namespace msc {

namespace {

constexpr int BB_T = 256;
constexpr int BB_WARPS = BB_T / 32;
constexpr int BB_COLMEAN_NB = 256;

__host__ __device__ __forceinline__ int64_t bb_grid(int64_t units, int per_block) {
  return (units + per_block - 1) / per_block;
}

// ---- layout -------------------------------------------------------------------------------------

__global__ void bb_query_region_kernel(int64_t n, int64_t p1, int32_t* __restrict__ perm,
                                       int32_t* __restrict__ qmap) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    perm[p1 + i] = int32_t(i);
    qmap[i] = int32_t(p1 + i);
  }
}

__global__ void bb_flag_kernel(const int32_t* __restrict__ codes, int64_t n, int b,
                               int32_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    flag[i] = codes[i] == b ? 1 : 0;
}

// cells of batch b to [poff, poff + nb) in ascending cell order; a cell beyond the stated count
// (codes and counts that disagree) is not placed, so no write leaves the batch's rows
__global__ void bb_place_kernel(const int32_t* __restrict__ codes, int64_t n, int b,
                                const int64_t* __restrict__ S, int64_t poff, int64_t nb,
                                int32_t* __restrict__ perm) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (codes[i] != b) continue;
    const int64_t r = S[i];
    if (r < nb) perm[poff + r] = int32_t(i);
  }
}

__global__ void bb_set_i32_kernel(int32_t* __restrict__ p, int32_t v) { *p = v; }

// query tiles of batch b: 128 listed cells each against the batch's keys
__global__ void bb_items_kernel(int64_t n, int64_t poff, int64_t nb, WorkItem* __restrict__ items) {
  const int64_t nt = (n + QTILE - 1) / QTILE;
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < nt;
       t += int64_t(gridDim.x) * blockDim.x) {
    WorkItem w;
    w.qrow0 = int32_t(t * QTILE);
    w.nq = int32_t(min64(QTILE, n - t * QTILE));
    w.key0 = int32_t(poff);
    w.nkeys = int32_t(nb);
    w.orig_off = 0;
    w.qorig0 = 0;
    w.pad0 = 0;
    w.pad1 = 0;
    items[t] = w;
  }
}

// ---- exact re-rank of one batch's candidates ----------------------------------------------------

__device__ __forceinline__ double bb_d2_f64(const float* xs, const float* __restrict__ y, int d) {
  double acc = 0.0;
  for (int t = 0; t < d; ++t) {
    const double df = double(xs[t]) - double(y[t]);
    acc += df * df;
  }
  return acc;
}
__device__ __forceinline__ float bb_d2_f32(const float* xs, const float* __restrict__ y, int d) {
  float acc = 0.f;
  for (int t = 0; t < d; ++t) {
    const float df = xs[t] - y[t];
    acc = fmaf(df, df, acc);
  }
  return acc;
}

// One warp per cell i: its k' candidates in batch b (original rows, -1 = none) → the kk nearest
// by (FP64 d², index) into columns [col0, col0 + kk) of row i; uncertified cells to fail_rows.
__global__ void __launch_bounds__(BB_T)
bb_rerank_kernel(const float* __restrict__ X, int d, int64_t n, int64_t p1,
                 const int32_t* __restrict__ cand_idx, const float* __restrict__ cand_thr,
                 int kprime, const QStat* __restrict__ qs, const KeyMax* __restrict__ km,
                 const Ctl* __restrict__ ctl, int prec, int kmma, int64_t nb, int kk, int K,
                 int col0, int32_t* __restrict__ knn_idx, float* __restrict__ knn_dist,
                 int32_t* __restrict__ fail_rows, int32_t* __restrict__ nfail,
                 int64_t* __restrict__ n_cert_out) {
  __shared__ __align__(16) float xs_all[BB_WARPS][MSC_MAX_D];
  const int lane = lane_id(), wib = warp_id();
  float* xs = xs_all[wib];
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const KeyMax kmv = *km;
  const double f = op_scale(prec, ctl);
  const double f2 = f * f;
  const double delta = double(d + 4) * 0x1p-24;
  const double INF = __longlong_as_double(0x7ff0000000000000ll);
  int64_t n_cert = 0;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    for (int t = lane; t < d; t += 32) xs[t] = X[i * d + t];
    __syncwarp();
    int c0 = lane < kprime ? cand_idx[i * kprime + lane] : -1;
    int c1 = lane + 32 < kprime ? cand_idx[i * kprime + lane + 32] : -1;
    double v0 = c0 >= 0 ? double(bb_d2_f32(xs, X + int64_t(c0) * d, d)) : INF;
    double v1 = c1 >= 0 ? double(bb_d2_f32(xs, X + int64_t(c1) * d, d)) : INF;
    int i0 = c0 >= 0 ? c0 : INT32_MAX, i1 = c1 >= 0 ? c1 : INT32_MAX;
    warp_sort64_d(v0, i0, v1, i1);
    const double B = __shfl_sync(FULL, kk - 1 < 32 ? v0 : v1, (kk - 1) & 31);
    // FP64 for the window of FP32 values within B·(1+3δ)
    const double lim = B * (1.0 + 3.0 * delta) + 1e-300;
    const bool w0 = i0 != INT32_MAX && v0 <= lim;
    const bool w1 = i1 != INT32_MAX && v1 <= lim;
    double g0 = w0 ? bb_d2_f64(xs, X + int64_t(i0) * d, d) : INF;
    double g1 = w1 ? bb_d2_f64(xs, X + int64_t(i1) * d, d) : INF;
    int h0 = w0 ? i0 : INT32_MAX, h1 = w1 ? i1 : INT32_MAX;
    warp_sort64_d(g0, h0, g1, h1);
    const double Dk = __shfl_sync(FULL, kk - 1 < 32 ? g0 : g1, (kk - 1) & 31);
    bool cert;
    if (nb <= kprime) {
      cert = true;                                     // every key of the batch is a candidate
    } else {
      const QStat q = qs[p1 + i];
      const double eps = cert_eps(q, kmv, prec, kmma, d);
      cert = f2 * Dk < q.sq + double(cand_thr[i]) - eps;
    }
    int32_t* oi = knn_idx + i * K + col0;
    float* od = knn_dist + i * K + col0;
    if (lane < kk) {
      oi[lane] = h0 == INT32_MAX ? int32_t(i) : h0;
      od[lane] = __double2float_rn(sqrt(g0));
    }
    if (lane + 32 < kk) {
      oi[lane + 32] = h1 == INT32_MAX ? int32_t(i) : h1;
      od[lane + 32] = __double2float_rn(sqrt(g1));
    }
    if (lane == 0) {
      if (cert) ++n_cert;
      else fail_rows[atomicAdd(nfail, 1)] = int32_t(i);
    }
    __syncwarp();
  }
  if (lane == 0 && n_cert)
    atomicAdd(reinterpret_cast<unsigned long long*>(n_cert_out), (unsigned long long)n_cert);
}

// FP64 scan of batch b for the listed cells (every cell when rows == nullptr): the kk (<= 128)
// nearest keys by (d², index) into columns [col0, col0 + kk)
__global__ void __launch_bounds__(BB_T)
bb_scan_kernel(const float* __restrict__ X, int d, int64_t n, const int32_t* __restrict__ perm,
               int64_t poff, int64_t nb, const int32_t* __restrict__ rows,
               const int32_t* __restrict__ nrows, int kk, int K, int col0,
               int32_t* __restrict__ knn_idx, float* __restrict__ knn_dist,
               int64_t* __restrict__ n_scanned) {
  __shared__ __align__(16) float xs_all[BB_WARPS][MSC_MAX_D];
  const int lane = lane_id(), wib = warp_id();
  float* xs = xs_all[wib];
  const int64_t count = rows ? int64_t(*nrows) : n;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const double INF = __longlong_as_double(0x7ff0000000000000ll);
  int64_t done = 0;
  for (int64_t w = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; w < count;
       w += nwarps) {
    const int64_t i = rows ? int64_t(rows[w]) : w;
    for (int t = lane; t < d; t += 32) xs[t] = X[i * d + t];
    __syncwarp();
    WarpTop128 top;
    top.init();
    for (int64_t base = 0; base < nb; base += 32) {
      const int64_t jj = base + lane;
      double v = INF;
      int vi = INT32_MAX;
      if (jj < nb) {
        const int32_t c = perm[poff + jj];
        if (c >= 0) {
          v = bb_d2_f64(xs, X + int64_t(c) * d, d);
          vi = c;
        }
      }
      top.offer(v, vi, kk);
    }
    int32_t* oi = knn_idx + i * K + col0;
    float* od = knn_dist + i * K + col0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int r = s * 32 + lane;
      if (r < kk) {
        oi[r] = top.ai[s] == INT32_MAX ? int32_t(i) : top.ai[s];
        od[r] = __double2float_rn(sqrt(top.a[s]));
      }
    }
    ++done;
    __syncwarp();
  }
  if (lane == 0 && done)
    atomicAdd(reinterpret_cast<unsigned long long*>(n_scanned), (unsigned long long)done);
}

// every row's K (<= 128) entries in (float32 distance, index) order: each entry's rank is the
// number of entries before it
__global__ void __launch_bounds__(BB_T)
bb_merge_kernel(int64_t n, int K, int32_t* __restrict__ knn_idx, float* __restrict__ knn_dist) {
  __shared__ float dv_all[BB_WARPS][128];
  __shared__ int32_t iv_all[BB_WARPS][128];
  const int lane = lane_id(), wib = warp_id();
  float* dv = dv_all[wib];
  int32_t* iv = iv_all[wib];
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    for (int e = lane; e < K; e += 32) {
      dv[e] = knn_dist[i * K + e];
      iv[e] = knn_idx[i * K + e];
    }
    __syncwarp();
    for (int e = lane; e < K; e += 32) {
      const float de = dv[e];
      const int32_t ie = iv[e];
      int r = 0;
      for (int g = 0; g < K; ++g)
        r += (dv[g] < de || (dv[g] == de && (iv[g] < ie || (iv[g] == ie && g < e)))) ? 1 : 0;
      knn_idx[i * K + r] = ie;
      knn_dist[i * K + r] = de;
    }
    __syncwarp();
  }
}

// ---- distances graph ---------------------------------------------------------------------------

__device__ __forceinline__ bool bb_dist_kept(int32_t j, float v, int64_t i) {
  return int64_t(j) != i && v != 0.f;
}

__global__ void bb_dist_count_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist,
                                     int64_t n, int K, int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    int c = 0;
    for (int e = 0; e < K; ++e) c += bb_dist_kept(idx[i * K + e], dist[i * K + e], i) ? 1 : 0;
    cnt[i] = c;
  }
}

// row i's kept entries in column order (the columns of a row are distinct)
__global__ void __launch_bounds__(BB_T)
bb_dist_fill_kernel(const int32_t* __restrict__ idx, const float* __restrict__ dist, int64_t n,
                    int K, const int64_t* __restrict__ indptr, int32_t* __restrict__ indices,
                    float* __restrict__ data) {
  __shared__ int32_t col_all[BB_WARPS][128];
  const int lane = lane_id(), wib = warp_id();
  int32_t* col = col_all[wib];
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    for (int e = lane; e < K; e += 32) {
      const int32_t j = idx[i * K + e];
      col[e] = bb_dist_kept(j, dist[i * K + e], i) ? j : -1;
    }
    __syncwarp();
    const int64_t base = indptr[i];
    for (int e = lane; e < K; e += 32) {
      const int32_t j = col[e];
      if (j < 0) continue;
      int r = 0;
      for (int g = 0; g < K; ++g) r += (col[g] >= 0 && col[g] < j) ? 1 : 0;
      indices[base + r] = j;
      data[base + r] = dist[i * K + e];
    }
    __syncwarp();
  }
}

// ---- trimming ----------------------------------------------------------------------------------

// float -> unsigned with the same order (negative values below positive ones)
__device__ __forceinline__ uint32_t ord_key(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_val(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// θ_i = the trim-th largest stored value of row i when the row stores more than `trim` entries,
// else 0: the largest key t with #{v : key(v) >= t} >= trim, found bit by bit from the top
__global__ void __launch_bounds__(BB_T)
trim_theta_kernel(const int64_t* __restrict__ indptr, const float* __restrict__ data, int64_t n,
                  int trim, float* __restrict__ theta) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int64_t a = indptr[i], b = indptr[i + 1];
    if (b - a <= trim) {
      if (lane == 0) theta[i] = 0.f;
      continue;
    }
    uint32_t t = 0;
    for (int bit = 31; bit >= 0; --bit) {
      const uint32_t test = t | (1u << bit);
      int64_t c = 0;
      for (int64_t e = a + lane; e < b; e += 32) c += ord_key(data[e]) >= test ? 1 : 0;
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
      if (c >= trim) t = test;
    }
    if (lane == 0) theta[i] = ord_val(t);
  }
}

__device__ __forceinline__ bool trim_kept(float v, float ti, float tj) {
  return v != 0.f && v >= ti && v >= tj;
}

__global__ void trim_count_kernel(const int64_t* __restrict__ indptr,
                                  const int32_t* __restrict__ indices,
                                  const float* __restrict__ data, int64_t n,
                                  const float* __restrict__ theta, int32_t* __restrict__ cnt) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const float ti = theta[i];
    int c = 0;
    for (int64_t e = indptr[i]; e < indptr[i + 1]; ++e)
      c += trim_kept(data[e], ti, theta[indices[e]]) ? 1 : 0;
    cnt[i] = c;
  }
}

// the kept entries of each row, in their stored order
__global__ void __launch_bounds__(BB_T)
trim_fill_kernel(const int64_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                 const float* __restrict__ data, int64_t n, const float* __restrict__ theta,
                 const int64_t* __restrict__ out_ptr, int32_t* __restrict__ out_idx,
                 float* __restrict__ out_data) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int64_t a = indptr[i], b = indptr[i + 1];
    const float ti = theta[i];
    int64_t o = out_ptr[i];
    for (int64_t e0 = a; e0 < b; e0 += 32) {
      const int64_t e = e0 + lane;
      bool keep = false;
      int32_t j = 0;
      float v = 0.f;
      if (e < b) {
        j = indices[e];
        v = data[e];
        keep = trim_kept(v, ti, theta[j]);
      }
      const unsigned m = __ballot_sync(FULL, keep);
      if (keep) {
        const int64_t at = o + __popc(m & ((1u << lane) - 1u));
        out_idx[at] = j;
        out_data[at] = v;
      }
      o += __popc(m);
    }
  }
}

int grid_for(int64_t units, int per_block) {
  return int(std::max<int64_t>(1, std::min<int64_t>(bb_grid(units, per_block),
                                                    int64_t(num_sms()) * 16)));
}

}  // namespace

// ---- host side ---------------------------------------------------------------------------------

BbPlan bb_plan(int64_t n, int d, const int64_t* counts, int nb, int kwb, int prec) {
  BbPlan P;
  P.n = n;
  P.d = d;
  P.nb = nb;
  P.kwb = kwb;
  P.prec = prec;
  P.K = 0;
  P.kk_max = 0;
  P.p1 = 0;
  P.max_nb = 0;
  for (int b = 0; b < nb; ++b) {
    const int kk = int(std::min<int64_t>(kwb, counts[b]));
    P.K += kk;
    P.kk_max = std::max(P.kk_max, kk);
    P.p1 += round_up(std::max<int64_t>(counts[b], 1), SEG_PAD);
    P.max_nb = std::max(P.max_nb, counts[b]);
  }
  P.npk = P.p1 + round_up(n, QTILE);
  // candidates: the one-term tensor-core scan with the self-kNN path's over-fetch for k = kk+1
  P.candidates = P.kk_max + 1 <= 64 && prec != PREC_FP32 && d <= MSC_MAX_D;
  P.kprime = 0;
  if (P.candidates) {
    // over-fetch: the certificate compares the kk-th neighbour with the k'-th candidate, a wide
    // margin already at k' = 32 for the usual kk = 3 (the self path's k' = 48 is sized for the
    // 15th neighbour); wider lists for larger kk
    P.kprime = prec == PREC_BF16X3 ? std::min(64, std::max(32, P.kk_max + 9))
                                   : std::min(64, std::max(32, P.kk_max + 16));
    P.L = op_layout(prec, d);
    P.cfg = tc_default_config(prec, d, P.kprime);
    if (P.cfg.pair || !tc_config_ok(P.cfg, P.L.kp, P.kprime)) P.candidates = false;
  }
  P.ntiles = ceil_div(n, QTILE);
  return P;
}

size_t bb_workspace_bytes(const BbPlan& P) {
  BbWs w;
  return bb_carve(P, nullptr, w);
}

size_t bb_carve(const BbPlan& P, void* base, BbWs& w) {
  Carver c(base);
  w.ctl = c.take<Ctl>(1);
  w.km = c.take<KeyMax>(1);
  w.seg = c.take<SegDesc>(1);
  w.nfail = c.take<int32_t>(1);
  w.counters = c.take<int32_t>(std::max(P.nb, 1));
  w.perm = c.take<int32_t>(P.npk);
  w.qmap = c.take<int32_t>(P.n);
  w.flag = c.take<int32_t>(P.n);
  w.S = c.take<int64_t>(P.n + 1);
  w.scan = c.take<int64_t>(scan_i32_scratch_elems(P.n));
  w.fail_rows = c.take<int32_t>(P.n);
  w.mean = c.take<double>(P.d);
  w.partial = c.take<double>(colmean_partial_elems(1, P.d, BB_COLMEAN_NB));
  if (P.candidates) {
    const size_t el = P.prec == PREC_FP16 ? sizeof(__half) : sizeof(__nv_bfloat16);
    w.Aop = c.take<char>(size_t(round_up(P.n, QTILE)) * P.L.kp * el);
    w.Bop = c.take<char>(size_t(P.p1) * P.L.kp * el);
    w.qs = c.take<QStat>(P.npk);
    w.items = c.take<WorkItem>(std::max<int64_t>(P.ntiles, 1));
    w.cand_idx = c.take<int32_t>(size_t(P.n) * P.kprime);
    w.cand_thr = c.take<float>(P.n);
  } else {
    w.Aop = w.Bop = nullptr;
    w.qs = nullptr;
    w.items = nullptr;
    w.cand_idx = nullptr;
    w.cand_thr = nullptr;
  }
  return c.bytes();
}

int run_bbknn(const BbPlan& P, const BbWs& w, const float* X, const int32_t* codes,
              const int64_t* counts, int32_t* knn_idx, float* knn_dist, cudaStream_t st) {
  MSC_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(Ctl), st));
  MSC_CUDA_TRY(cudaMemsetAsync(w.km, 0, sizeof(KeyMax), st));
  MSC_CUDA_TRY(cudaMemsetAsync(w.counters, 0, sizeof(int32_t) * std::max(P.nb, 1), st));
  MSC_CUDA_TRY(cudaMemsetAsync(w.perm, 0xFF, sizeof(int32_t) * P.npk, st));
  const int g = grid_for(P.n, BB_T);
  // layout: batch segments, then the query region
  int64_t poff = 0;
  for (int b = 0; b < P.nb; ++b) {
    bb_flag_kernel<<<g, BB_T, 0, st>>>(codes, P.n, b, w.flag);
    MSC_LAUNCH_CHECK();
    MSC_TRY(scan_excl_i32(w.flag, P.n, w.S, w.scan, st));
    bb_place_kernel<<<g, BB_T, 0, st>>>(codes, P.n, b, w.S, poff, counts[b], w.perm);
    MSC_LAUNCH_CHECK();
    poff += round_up(std::max<int64_t>(counts[b], 1), SEG_PAD);
  }
  bb_query_region_kernel<<<g, BB_T, 0, st>>>(P.n, P.p1, w.perm, w.qmap);
  MSC_LAUNCH_CHECK();
  const int gw = grid_for(P.n, BB_WARPS);                 // one warp per cell
  if (P.candidates) {
    // one centring and one scale for both sides
    MSC_TRY(launch_single_segment(w.seg, P.n, st));
    MSC_TRY(launch_colmean(X, w.seg, 1, P.n, P.d, w.partial, BB_COLMEAN_NB, w.mean,
                           &w.ctl->stats[MSC_STAT_NONFINITE], st));
    if (P.prec == PREC_FP16) MSC_TRY(launch_maxnorm(X, w.seg, 1, w.mean, P.d, P.n, w.ctl, st));
    MSC_TRY(launch_pack_tc(P.prec, X, w.perm, w.seg, 1, w.mean, P.d, P.p1, nullptr, nullptr, 0,
                           nullptr, w.Bop, w.qs, w.km, w.ctl, st));
    // the query operand: every cell, listed through qmap (the listed-row count in ctl)
    bb_set_i32_kernel<<<1, 1, 0, st>>>(&w.ctl->n_refine, int32_t(P.n));
    MSC_LAUNCH_CHECK();
    MSC_CUDA_TRY(cudaMemsetAsync(w.Aop, 0,
                                 size_t(round_up(P.n, QTILE)) * P.L.kp *
                                     (P.prec == PREC_FP16 ? sizeof(__half) : sizeof(__nv_bfloat16)),
                                 st));
    MSC_TRY(launch_pack_tc(P.prec, X, w.perm, w.seg, 1, w.mean, P.d, P.npk, w.qmap,
                           &w.ctl->n_refine, P.n, w.Aop, nullptr, w.qs, nullptr, w.ctl, st));
  }
  poff = 0;
  int col0 = 0;
  for (int b = 0; b < P.nb; ++b) {
    const int64_t nbk = counts[b];
    const int kk = int(std::min<int64_t>(P.kwb, nbk));
    if (kk > 0) {
      if (P.candidates) {
        bb_items_kernel<<<grid_for(P.ntiles, BB_T), BB_T, 0, st>>>(P.n, poff, nbk, w.items);
        MSC_LAUNCH_CHECK();
        // the query operand's map spans its zero-filled tail rows too (no box beyond the rows)
        MSC_TRY(launch_knn_tc(P.prec, P.cfg, w.Aop, w.Bop, round_up(P.n, QTILE), P.p1, P.L.kp,
                              P.L.kmma, w.items, P.ntiles, w.perm, w.qmap, nullptr,
                              &w.counters[b], w.ctl,
                              P.kprime, w.cand_idx, w.cand_thr, P.kprime, st));
        MSC_CUDA_TRY(cudaMemsetAsync(w.nfail, 0, sizeof(int32_t), st));
        bb_rerank_kernel<<<gw, BB_T, 0, st>>>(X, P.d, P.n, P.p1, w.cand_idx, w.cand_thr,
                                              P.kprime, w.qs, w.km, w.ctl, P.prec, P.L.kmma, nbk,
                                              kk, P.K, col0, knn_idx, knn_dist, w.fail_rows,
                                              w.nfail, &w.ctl->stats[MSC_STAT_CERTIFIED]);
        MSC_LAUNCH_CHECK();
        bb_scan_kernel<<<gw, BB_T, 0, st>>>(X, P.d, P.n, w.perm, poff, nbk, w.fail_rows,
                                            w.nfail, kk, P.K, col0, knn_idx, knn_dist,
                                            &w.ctl->stats[MSC_STAT_RESCANNED]);
        MSC_LAUNCH_CHECK();
      } else {
        bb_scan_kernel<<<gw, BB_T, 0, st>>>(X, P.d, P.n, w.perm, poff, nbk, nullptr, nullptr,
                                            kk, P.K, col0, knn_idx, knn_dist,
                                            &w.ctl->stats[MSC_STAT_RESCANNED]);
        MSC_LAUNCH_CHECK();
      }
    }
    col0 += kk;
    poff += round_up(std::max<int64_t>(nbk, 1), SEG_PAD);
  }
  bb_merge_kernel<<<gw, BB_T, 0, st>>>(P.n, P.K, knn_idx, knn_dist);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

size_t bb_distances_workspace_bytes(int64_t n) {
  Carver c(nullptr);
  c.take<int32_t>(n);
  c.take<int64_t>(scan_i32_scratch_elems(n));
  return c.bytes();
}

int launch_bb_distances(const int32_t* idx, const float* dist, int64_t n, int K, int64_t* indptr,
                        int32_t* indices, float* data, void* ws, cudaStream_t st) {
  Carver c(ws);
  int32_t* cnt = c.take<int32_t>(n);
  int64_t* scan = c.take<int64_t>(scan_i32_scratch_elems(n));
  bb_dist_count_kernel<<<grid_for(n, BB_T), BB_T, 0, st>>>(idx, dist, n, K, cnt);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl_i32(cnt, n, indptr, scan, st));
  bb_dist_fill_kernel<<<grid_for(n, BB_WARPS), BB_T, 0, st>>>(idx, dist, n, K, indptr, indices,
                                                              data);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

size_t trim_workspace_bytes(int64_t n) {
  Carver c(nullptr);
  c.take<float>(n);
  c.take<int32_t>(n);
  c.take<int64_t>(scan_i32_scratch_elems(n));
  return c.bytes();
}

int launch_trim(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n,
                int trim, int64_t* out_ptr, int32_t* out_idx, float* out_data, void* ws,
                cudaStream_t st) {
  Carver c(ws);
  float* theta = c.take<float>(n);
  int32_t* cnt = c.take<int32_t>(n);
  int64_t* scan = c.take<int64_t>(scan_i32_scratch_elems(n));
  trim_theta_kernel<<<grid_for(n, BB_WARPS), BB_T, 0, st>>>(indptr, data, n, trim, theta);
  MSC_LAUNCH_CHECK();
  trim_count_kernel<<<grid_for(n, BB_T), BB_T, 0, st>>>(indptr, indices, data, n, theta, cnt);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl_i32(cnt, n, out_ptr, scan, st));
  trim_fill_kernel<<<grid_for(n, BB_WARPS), BB_T, 0, st>>>(indptr, indices, data, n, theta,
                                                           out_ptr, out_idx, out_data);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
