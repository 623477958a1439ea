// Exact re-rank of the candidates and the certificate that they contain the true neighbours.
//
// Reference counterpart: the fp32 direct-difference recompute of the selected neighbours
// (metalsinglecell neighbors.py:120-123) and the host sort by distance with self first
// (neighbors.py:129-131; ties by index as in neighbors.py:457-461).  The reference ranks on fp16
// and accepts ~0.99 recall; here every row is either proven exact or re-scanned exactly:
//
//   1. FP32 direct differences Σ(x_t − y_t)² for all k' candidates (one lane per candidate);
//   2. the (k−1)-th smallest FP32 value B bounds the answer;
//   3. candidates within B·(1+3δ) (δ = (d+4)·2⁻²⁴, the FP32 sum's relative error bound) are
//      recomputed in FP64 and ordered by (FP64 distance, index) — FP64 only breaks ties at the
//      k-th boundary, and gives the returned distances float32(sqrt(d²₆₄)).  Usually the window
//      holds k−1 … 32 candidates: B then comes from a sort of the 64 values alone, the window's
//      ids are compacted into lanes 0..m−1 for one FP64 pass and a 32-pair sort.  Otherwise (a
//      wider window, or NaN) all 64 (value, index) pairs are sorted, then the window's FP64
//      values.  Both give the same set, the same FP64 values and the same order;
//   4. certificate: every key outside the candidate list has approximate value v̂ ≥ T (the
//      k'-th smallest kept), so its true squared distance is ≥ (|z_x|² + T − ε)/f² where ε
//      bounds |v̂ − v| from the operand residual norms recorded by the packing kernel.  If the
//      (k−1)-th FP64 distance is strictly below that, the row is exact; otherwise the row goes
//      to the FP64 full scan below.
#include "kernels.cuh"
#include "msc_select.cuh"
#include "msc_warpsort.cuh"

namespace msc {

namespace {

constexpr int RR_WARPS = 8;

__device__ __forceinline__ double d2_f64(const float* xs, const float* __restrict__ y, int d) {
  double acc = 0.0;
  for (int t = 0; t < d; ++t) {
    double df = double(xs[t]) - double(y[t]);
    acc += df * df;
  }
  return acc;
}

// One lane's share of the FP32 squared distance of a shared-memory row xs and row y when the 4
// lanes of a group split the row (part = lane & 3 takes every 4th 8-byte pair, or every 4th
// element of a row that is not 8-byte aligned); the group then sums the four shares.  The warp
// reads 8 candidate rows per instruction in 32-byte pieces instead of an 8-byte piece of each of
// 32 rows.  Any summation order of the d positive terms stays within the (d+4)·2^-24 relative
// bound the re-rank window assumes.
__device__ __forceinline__ float group_part_d2_f32(const float* xs, const float* __restrict__ y,
                                                   int d, int part) {
  float a0 = 0.f, a1 = 0.f;
  if ((reinterpret_cast<uintptr_t>(y) & 7) == 0) {
    const float2* y2 = reinterpret_cast<const float2*>(y);
    const float2* x2 = reinterpret_cast<const float2*>(xs);
    const int h = d >> 1;
    for (int t = part; t < h; t += 4) {
      const float2 u = y2[t], p = x2[t];
      const float e0 = p.x - u.x, e1 = p.y - u.y;
      a0 = fmaf(e0, e0, a0);
      a1 = fmaf(e1, e1, a1);
    }
    if ((d & 1) && part == 0) {
      const float e = xs[d - 1] - y[d - 1];
      a0 = fmaf(e, e, a0);
    }
  } else {
    for (int t = part; t < d; t += 4) {
      const float e = xs[t] - y[t];
      a0 = fmaf(e, e, a0);
    }
  }
  return a0 + a1;
}

__device__ __forceinline__ float out_dist(double d2, int cosine) {
  return cosine ? __double2float_rn(d2 * 0.5) : __double2float_rn(sqrt(d2));
}

__global__ void __launch_bounds__(RR_WARPS * 32, 4)
rerank_kernel(const float* __restrict__ X, int d, const int32_t* __restrict__ perm,
              const SegDesc* __restrict__ seg, int nseg,
              int64_t npacked, const int32_t* __restrict__ cand_idx,
              const float* __restrict__ cand_thr, int cand_stride, int kprime,
              const QStat* __restrict__ qs, const KeyMax* __restrict__ km, Ctl* __restrict__ ctl,
              int prec, int kmma, int k, int cosine, int32_t* __restrict__ knn_idx,
              float* __restrict__ knn_dist, int32_t* __restrict__ fail_rows,
              const int32_t* __restrict__ rows, const int32_t* __restrict__ nrows,
              int32_t* __restrict__ fail_flags) {
  __shared__ __align__(16) float xs_all[RR_WARPS][MSC_MAX_D];
  __shared__ int wsc_all[RR_WARPS][32];                 // a row's window, compacted
  const int lane = lane_id(), wib = warp_id();
  float* xs = xs_all[wib];
  const int kk = k - 1;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  // key-side maxima and the scale
  const KeyMax kmv = *km;
  const double f = op_scale(prec, ctl);
  const double f2 = f * f;
  const double delta = double(d + 4) * 0x1p-24;
  int64_t n_cert = 0, n_ties = 0;
  const int64_t count = rows ? int64_t(*nrows) : npacked;
  for (int64_t wq = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; wq < count;
       wq += nwarps) {
    const int64_t p = rows ? int64_t(rows[wq]) : wq;
    const int64_t i = perm[p];                          // original row
    if (i < 0) continue;                                // padding (warp-uniform)
    const int s = find_seg(seg, nseg, p);
    const int64_t ns = seg[s].n;
    for (int t = lane; t < d; t += 32) xs[t] = X[i * d + t];
    __syncwarp();
    if (kk == 0) {
      if (lane == 0) { knn_idx[i * k] = int32_t(i); knn_dist[i * k] = 0.f; ++n_cert; }
      continue;
    }
    // 1. FP32 distances of the candidates (lane: slots lane and lane+32), eight candidates at a
    //    time, four lanes each; candidate c's value goes to lane c & 31, slot c >> 5
    int c0 = lane < kprime ? cand_idx[i * cand_stride + lane] : -1;
    int c1 = lane + 32 < kprime ? cand_idx[i * cand_stride + lane + 32] : -1;
    float e0 = __int_as_float(0x7f800000), e1 = __int_as_float(0x7f800000);
    {
      const int part = lane & 3, grp = lane >> 2;
      for (int r = 0; r < kprime; r += 8) {              // warp-uniform
        const int c = r + grp;
        // the candidate ids sit in lanes c & 31 of c0 (c < 32) or c1
        const int id0 = __shfl_sync(FULL, c0, c & 31), id1 = __shfl_sync(FULL, c1, c & 31);
        const int cid = c < kprime ? (c < 32 ? id0 : id1) : -1;
        float v = cid >= 0 ? group_part_d2_f32(xs, X + int64_t(cid) * d, d, part) : 0.f;
        v += __shfl_xor_sync(FULL, v, 1);                // the group's four shares
        v += __shfl_xor_sync(FULL, v, 2);
        if (cid < 0) v = __int_as_float(0x7f800000);
        const int rb = r & 31;                            // lanes rb .. rb+7 receive this round
        const float got = __shfl_sync(FULL, v, ((lane - rb) & 7) * 4);
        if (lane >= rb && lane < rb + 8) {
          if (r < 32) e0 = got; else e1 = got;
        }
      }
    }
    // 2.-3. B = the (k-1)-th smallest FP32 value; the window = the candidates within B's rounding
    //    bound, recomputed in FP64 (summed in dimension order) and ordered by (FP64 value, index).
    //    Fast path (no NaN, k-1 <= window <= 32): B from a values-only sort, the window's ids
    //    compacted into lanes 0..m-1, one FP64 pass and a 32-pair sort.  The window holds the same
    //    candidates and the same FP64 values as on the general path (two 64-pair sorts), so the
    //    outputs are the same.
    const double INF = __longlong_as_double(0x7ff0000000000000ll);
    double g0 = INF, g1 = INF, Dk = INF;
    int h0 = INT32_MAX, h1 = INT32_MAX, m = 0;
    bool fast = false;
    if (!__any_sync(FULL, isnan(e0) || isnan(e1))) {
      float s0 = e0, s1 = e1;
      warp_sort64_f(s0, s1);
      const float Bf = __shfl_sync(FULL, kk - 1 < 32 ? s0 : s1, (kk - 1) & 31);
      const double limf = double(Bf) * (1.0 + 3.0 * delta) + 1e-300;
      const bool w0 = c0 >= 0 && double(e0) <= limf;
      const bool w1 = c1 >= 0 && double(e1) <= limf;
      const unsigned b0 = __ballot_sync(FULL, w0), b1 = __ballot_sync(FULL, w1);
      m = __popc(b0) + __popc(b1);
      if (m >= kk && m <= 32) {                          // warp-uniform
        int* wsc = wsc_all[wib];
        const unsigned lt = (1u << lane) - 1u;
        if (w0) wsc[__popc(b0 & lt)] = c0;
        if (w1) wsc[__popc(b0) + __popc(b1 & lt)] = c1;
        __syncwarp();
        int cw = lane < m ? wsc[lane] : INT32_MAX;
        double gw = lane < m ? d2_f64(xs, X + int64_t(cw) * d, d) : INF;
        __syncwarp();                                    // wsc is read before the next row
        warp_sort32_d(gw, cw);
        g0 = gw; h0 = cw;
        Dk = __shfl_sync(FULL, g0, kk - 1);
        fast = true;
      }
    }
    if (!fast) {
      // general path: sort all 64 (FP32 value, index) pairs, then the window's FP64 values
      double v0 = e0, v1 = e1;
      int i0 = c0 >= 0 ? c0 : INT32_MAX, i1 = c1 >= 0 ? c1 : INT32_MAX;
      warp_sort64_d(v0, i0, v1, i1);
      const float se0 = float(v0), se1 = float(v1);
      const float B = __shfl_sync(FULL, kk - 1 < 32 ? se0 : se1, (kk - 1) & 31);
      const double lim = double(B) * (1.0 + 3.0 * delta) + 1e-300;
      const bool w0 = i0 != INT32_MAX && double(se0) <= lim;
      const bool w1 = i1 != INT32_MAX && double(se1) <= lim;
      g0 = w0 ? d2_f64(xs, X + int64_t(i0) * d, d) : INF;
      g1 = w1 ? d2_f64(xs, X + int64_t(i1) * d, d) : INF;
      m = __popc(__ballot_sync(FULL, w0)) + __popc(__ballot_sync(FULL, w1));
      h0 = i0; h1 = i1;
      warp_sort64_d(g0, h0, g1, h1);
      Dk = __shfl_sync(FULL, kk - 1 < 32 ? g0 : g1, (kk - 1) & 31);
    }
    // 4. certificate
    bool cert;
    const int nvalid = int(min64(ns - 1, kprime));
    if (ns - 1 <= kprime) {
      cert = true;                                      // every key is a candidate
    } else {
      const QStat q = qs[p];
      const double eps = cert_eps(q, kmv, prec, kmma, d);
      const double T = double(cand_thr[i]);
      cert = f2 * Dk < q.sq + T - eps;
    }
    (void)nvalid;
    // outputs
    if (lane == 0) {
      knn_idx[i * k] = int32_t(i);
      knn_dist[i * k] = 0.f;
    }
    // a slot without a valid candidate (only possible with non-finite input) is filled with the
    // row itself so that every index stays in range for the graph stages
    if (lane < kk) {
      knn_idx[i * k + 1 + lane] = h0 == INT32_MAX ? int32_t(i) : h0;
      knn_dist[i * k + 1 + lane] = out_dist(g0, cosine);
    }
    if (lane + 32 < kk) {
      knn_idx[i * k + 33 + lane] = h1 == INT32_MAX ? int32_t(i) : h1;
      knn_dist[i * k + 33 + lane] = out_dist(g1, cosine);
    }
    if (lane == 0) {
      n_ties += m - kk;
      if (cert) {
        ++n_cert;
      } else if (fail_flags) {
        fail_flags[p] = 1;                              // to the refine pass
      } else {
        int slot = atomicAdd(&ctl->n_fail, 1);
        fail_rows[slot] = int32_t(p);                   // packed row, to the FP64 scan
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    if (n_cert) atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->stats[MSC_STAT_CERTIFIED]),
                          (unsigned long long)n_cert);
    if (n_ties) atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->stats[MSC_STAT_FP64_TIES]),
                          (unsigned long long)n_ties);
  }
}

// ------------------------------------------------------------------------------------------------
// FP64 full scan of one row per warp: all keys of the row's sample, ordered by (d², index), with
// a warp-distributed sorted list of 32·SLOTS (SLOTS per lane) merged 32 keys at a time; SLOTS = 4,
// 8 or 16 covers k - 1 up to 128, 256 or 512.
// ------------------------------------------------------------------------------------------------
template <int SLOTS>
__global__ void __launch_bounds__(RR_WARPS * 32)
fp64_scan_kernel(const float* __restrict__ X, int d, const int32_t* __restrict__ perm,
                 const SegDesc* __restrict__ seg, int nseg,
                 const int32_t* __restrict__ fail_rows, Ctl* __restrict__ ctl, int k, int cosine,
                 int32_t* __restrict__ knn_idx, float* __restrict__ knn_dist) {
  __shared__ __align__(16) float xs_all[RR_WARPS][MSC_MAX_D];
  const int lane = lane_id(), wib = warp_id();
  float* xs = xs_all[wib];
  const int kk = k - 1;
  const int nfail = ctl->n_fail;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const double INF = __longlong_as_double(0x7ff0000000000000ll);
  int64_t done = 0;
  for (int64_t w = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; w < nfail; w += nwarps) {
    const int64_t p = fail_rows[w];                      // packed row
    const int sg = find_seg(seg, nseg, p);
    const int64_t off = seg[sg].off, ns = seg[sg].n;
    const int64_t i = perm[p];                           // original row
    for (int t = lane; t < d; t += 32) xs[t] = X[i * d + t];
    __syncwarp();
    WarpTop<SLOTS> top;
    top.init();
    for (int64_t base = 0; base < ns; base += 32) {
      const int64_t jj = base + lane;
      double v = INF;
      int vi = INT32_MAX;
      if (jj < ns && off + jj != i) {
        v = d2_f64(xs, X + (off + jj) * d, d);
        vi = int(off + jj);
      }
      top.offer(v, vi, kk);
    }
    if (lane == 0) { knn_idx[i * k] = int32_t(i); knn_dist[i * k] = 0.f; }
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) {
      const int r = s * 32 + lane;
      if (r < kk) {
        knn_idx[i * k + 1 + r] = top.ai[s] == INT32_MAX ? int32_t(i) : top.ai[s];
        knn_dist[i * k + 1 + r] = out_dist(top.a[s], cosine);
      }
    }
    ++done;
    __syncwarp();
  }
  if (lane == 0 && done)
    atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->stats[MSC_STAT_RESCANNED]),
              (unsigned long long)done);
}

// every valid packed row goes to the FP64 scan (n_neighbors beyond the candidate kernels)
__global__ void all_rows_fail_kernel(const int32_t* __restrict__ perm, int64_t npacked,
                                     int32_t* __restrict__ fail_rows, Ctl* __restrict__ ctl) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x)
    if (perm[p] >= 0) fail_rows[atomicAdd(&ctl->n_fail, 1)] = int32_t(p);
}

// refine pass: the flagged rows, in packed order, as a compact query list
__global__ void compact_flags_kernel(const int32_t* __restrict__ flags,
                                     const int64_t* __restrict__ S, int64_t npacked,
                                     int32_t* __restrict__ qmap, Ctl* __restrict__ ctl) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    if (flags[p]) qmap[S[p]] = int32_t(p);
    if (p == 0) {
      ctl->n_refine = int32_t(S[npacked]);
      ctl->stats[MSC_STAT_REFINED] = S[npacked];
    }
  }
}

// query tiles of at most QTILE listed rows, never spanning two samples (one thread: the list is
// short and the tile count is written once)
__global__ void refine_items_kernel(const SegDesc* __restrict__ seg, int nseg,
                                    const int64_t* __restrict__ S, WorkItem* __restrict__ items,
                                    Ctl* __restrict__ ctl, int split, int max_split_items) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int32_t n = 0;
  for (int s = 0; s < nseg; ++s) {
    const int64_t cs = S[seg[s].poff], ce = S[seg[s].poff + seg[s].n];
    for (int64_t q = cs; q < ce; q += QTILE) {
      WorkItem w;
      w.qrow0 = int32_t(q);
      w.nq = int32_t(min64(QTILE, ce - q));
      w.key0 = int32_t(seg[s].poff);
      w.nkeys = int32_t(seg[s].n);
      w.orig_off = int32_t(seg[s].off);
      w.qorig0 = 0;
      w.pad0 = w.pad1 = 0;
      items[n++] = w;
    }
  }
  ctl->n_items_refine = n;
  // few refine items (the usual case) would leave most SMs idle: split each over key ranges
  const int sp = (split > 1 && n <= max_split_items) ? split : 1;
  ctl->refine_split = sp;
  ctl->n_items_refine_eff = n * sp;
}

}  // namespace

int launch_all_rows_fail(const int32_t* perm, int64_t npacked, int32_t* fail_rows, Ctl* ctl,
                         cudaStream_t st) {
  int blocks = int(std::min<int64_t>(ceil_div(npacked, 256), int64_t(num_sms()) * 8));
  all_rows_fail_kernel<<<std::max(blocks, 1), 256, 0, st>>>(perm, npacked, fail_rows, ctl);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_rerank(const float* X, int d, const int32_t* perm, const SegDesc* seg, int nseg,
                  int64_t npacked,
                  const int32_t* cand_idx, const float* cand_thr, int cand_stride, int kprime,
                  const QStat* qs, const KeyMax* km, int prec, int kmma, int k, int cosine,
                  int32_t* knn_idx, float* knn_dist, int32_t* fail_rows, Ctl* ctl,
                  const int32_t* rows, const int32_t* nrows, int64_t max_rows,
                  int32_t* fail_flags, cudaStream_t st) {
  if (kprime > 64 || k - 1 > 64) {
    set_error("rerank: kprime=%d / k=%d beyond 64", kprime, k);
    return MSC_ERR_UNSUPPORTED;
  }
  const int64_t n_work = rows ? max_rows : npacked;
  int blocks = int(std::min<int64_t>(ceil_div(n_work, RR_WARPS), int64_t(num_sms()) * 8));
  rerank_kernel<<<std::max(blocks, 1), RR_WARPS * 32, 0, st>>>(
      X, d, perm, seg, nseg, npacked, cand_idx, cand_thr, cand_stride, kprime, qs, km, ctl, prec,
      kmma, k, cosine, knn_idx, knn_dist, fail_rows, rows, nrows, fail_flags);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_refine_plan(const int32_t* flags, int64_t npacked, const SegDesc* seg, int nseg,
                       int32_t* qmap, WorkItem* items, int64_t* S, int64_t* scan_scratch,
                       Ctl* ctl, int split, int max_split_items, cudaStream_t st) {
  MSC_TRY(scan_excl_i32(flags, npacked, S, scan_scratch, st));
  int blocks = int(std::min<int64_t>(ceil_div(npacked, 256), int64_t(num_sms()) * 8));
  compact_flags_kernel<<<std::max(blocks, 1), 256, 0, st>>>(flags, S, npacked, qmap, ctl);
  MSC_LAUNCH_CHECK();
  refine_items_kernel<<<1, 32, 0, st>>>(seg, nseg, S, items, ctl, split, max_split_items);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_fp64_scan(const float* X, int d, const int32_t* perm, const SegDesc* seg, int nseg,
                     const int32_t* fail_rows, int64_t max_rows, int k, int cosine,
                     int32_t* knn_idx, float* knn_dist, Ctl* ctl, cudaStream_t st) {
  if (k - 1 > 512) {
    set_error("fp64 scan: k=%d beyond 513", k);
    return MSC_ERR_UNSUPPORTED;
  }
  const int blocks = std::max(
      1, int(std::min<int64_t>(ceil_div(max_rows, RR_WARPS), int64_t(num_sms()) * 8)));
  if (k - 1 <= 128)
    fp64_scan_kernel<4><<<blocks, RR_WARPS * 32, 0, st>>>(X, d, perm, seg, nseg, fail_rows, ctl,
                                                          k, cosine, knn_idx, knn_dist);
  else if (k - 1 <= 256)
    fp64_scan_kernel<8><<<blocks, RR_WARPS * 32, 0, st>>>(X, d, perm, seg, nseg, fail_rows, ctl,
                                                          k, cosine, knn_idx, knn_dist);
  else
    fp64_scan_kernel<16><<<blocks, RR_WARPS * 32, 0, st>>>(X, d, perm, seg, nseg, fail_rows, ctl,
                                                           k, cosine, knn_idx, knn_dist);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
