// Input preparation for the candidate kernels.
//
// The reference ranks neighbours on a scaled fp16 Gram form |x|²+|y|²−2x·y
// (metalsinglecell neighbors.py:99-103,117-118) and, in its exact helper, centres the data first
// because the Gram form cancels catastrophically on large magnitudes (neighbors.py:423-441).
// Here every sample is centred on its own column mean (FP64), scaled by a power of two (FP16
// only), and rounded into the operand format of the chosen precision.  The squared norm of each
// key is folded into the key operand so that one GEMM yields v = |y|² − 2x·y directly:
//
//   one-term (FP16 / BF16):  A = [a | 1 1 1 | 0…]                B = [−2b | s1 s2 s3 | 0…]
//   three-term BF16 split:   A = [a_hi | a_hi | a_lo | 1 1 1 | 0…]
//                            B = [−2b_hi | −2b_lo | −2b_hi | s1 s2 s3 | 0…]
//   FP32 SIMT:               A = fp32(z), plus fp32 |z|² per row
//
// s1+s2+s3 is a three-term split of Σ z² (FP64).  The kernels also record, per row, the norms of
// what the operands represent and of what they miss, and the maxima over keys; the re-rank turns
// these into a rigorous bound on |v̂ − v| that certifies each row's candidate set.
#include "kernels.cuh"

namespace msc {

// ------------------------------------------------------------------------------------------------
// cosine: x̂ = float32(x · 1/sqrt(Σ x_t²)), the sum in FP64 in dimension order (thread per row)
// ------------------------------------------------------------------------------------------------
__global__ void normalize_rows_kernel(const float* __restrict__ X, float* __restrict__ Xn,
                                      int64_t n, int d, int64_t* nonfinite) {
  int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= n) return;
  const float* x = X + i * d;
  double s = 0.0;
  int bad = 0;
  for (int t = 0; t < d; ++t) {
    double v = x[t];
    bad |= !isfinite(v);
    s += v * v;
  }
  double r = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
  float* y = Xn + i * d;
  for (int t = 0; t < d; ++t) y[t] = __double2float_rn(double(x[t]) * r);
  if (bad) atomicAdd(reinterpret_cast<unsigned long long*>(nonfinite), 1ull);
}

int launch_normalize(const float* X, float* Xn, int64_t n, int d, int64_t* nonfinite,
                     cudaStream_t st) {
  normalize_rows_kernel<<<unsigned(ceil_div(n, 256)), 256, 0, st>>>(X, Xn, n, d, nonfinite);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// ------------------------------------------------------------------------------------------------
// per-sample column means: block (b, s) sums rows [b·chunk, (b+1)·chunk) of sample s in FP64;
// the finalize kernel adds the partials in block order, so the result is deterministic.
// ------------------------------------------------------------------------------------------------
__global__ void colsum_partial_kernel(const float* __restrict__ X, const SegDesc* __restrict__ seg,
                                      int d, int nb, double* __restrict__ partial,
                                      int64_t* nonfinite) {
  const int s = blockIdx.y, b = blockIdx.x;
  const int64_t off = seg[s].off, ns = seg[s].n;
  const int64_t chunk = (ns + nb - 1) / nb;
  const int64_t r0 = off + min64(ns, b * chunk);
  const int64_t r1 = off + min64(ns, (b + 1) * chunk);
  const int P = int(blockDim.x) / d;          // row phases (d <= blockDim.x)
  const int t = threadIdx.x % d, p = threadIdx.x / d;
  __shared__ double red[256];
  double acc = 0.0;
  int bad = 0;
  if (p < P) {
    for (int64_t r = r0 + p; r < r1; r += P) {
      float v = X[r * d + t];
      bad |= !isfinite(v);
      acc += double(v);
    }
    red[p * d + t] = acc;
  }
  __syncthreads();
  if (threadIdx.x < d) {
    double a = 0.0;
    for (int q = 0; q < P; ++q) a += red[q * d + threadIdx.x];
    partial[(int64_t(s) * nb + b) * d + threadIdx.x] = a;
  }
  if (bad) atomicAdd(reinterpret_cast<unsigned long long*>(nonfinite), 1ull);
}

__global__ void colmean_finalize_kernel(const double* __restrict__ partial,
                                        const SegDesc* __restrict__ seg, int nseg, int d, int nb,
                                        double* __restrict__ mean) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nseg * d) return;
  int s = i / d, t = i % d;
  double a = 0.0;
  for (int b = 0; b < nb; ++b) a += partial[(int64_t(s) * nb + b) * d + t];
  mean[i] = seg[s].n > 0 ? a / double(seg[s].n) : 0.0;
}

size_t colmean_partial_elems(int nseg, int d, int nb) { return size_t(nseg) * nb * d; }

int launch_colmean(const float* X, const SegDesc* seg, int nseg, int64_t max_seg_n, int d,
                   double* partial, int nb, double* mean, int64_t* nonfinite, cudaStream_t st) {
  if (d > 256) { set_error("colmean: d=%d > 256", d); return MSC_ERR_UNSUPPORTED; }
  (void)max_seg_n;
  dim3 grid(nb, nseg);
  colsum_partial_kernel<<<grid, 256, 0, st>>>(X, seg, d, nb, partial, nonfinite);
  MSC_LAUNCH_CHECK();
  colmean_finalize_kernel<<<unsigned(ceil_div(int64_t(nseg) * d, 256)), 256, 0, st>>>(
      partial, seg, nseg, d, nb, mean);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// ------------------------------------------------------------------------------------------------
// max over rows of Σ (x − c)² (FP64, rounded up) — sizes the FP16 scale factor
// ------------------------------------------------------------------------------------------------
__global__ void maxnorm_kernel(const float* __restrict__ X, const SegDesc* __restrict__ seg,
                               int nseg, const double* __restrict__ mean, int d, int64_t npacked,
                               Ctl* ctl) {
  float m = 0.f;
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    int s = find_seg(seg, nseg, p);
    int64_t j = p - seg[s].poff;
    if (j >= seg[s].n) continue;
    const float* x = X + (seg[s].off + j) * d;
    const double* c = mean + int64_t(s) * d;
    double acc = 0.0;
    for (int t = 0; t < d; ++t) {
      double z = double(x[t]) - c[t];
      acc += z * z;
    }
    m = fmaxf(m, __double2float_ru(acc));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(&ctl->max_sq_bits, __float_as_uint(m));
}

int launch_maxnorm(const float* X, const SegDesc* seg, int nseg, const double* mean, int d,
                   int64_t npacked, Ctl* ctl, cudaStream_t st) {
  int blocks = int(std::min<int64_t>(ceil_div(npacked, 256), int64_t(num_sms()) * 8));
  maxnorm_kernel<<<std::max(blocks, 1), 256, 0, st>>>(X, seg, nseg, mean, d, npacked, ctl);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// ------------------------------------------------------------------------------------------------
// operand packing: one warp per packed row (grid-stride), lanes over dimensions
// ------------------------------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T to_op(double v);
template <> __device__ __forceinline__ __half to_op<__half>(double v) { return __double2half(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_op<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}
__device__ __forceinline__ double op_val(__half v) { return double(__half2float(v)); }
__device__ __forceinline__ double op_val(__nv_bfloat16 v) { return double(__bfloat162float(v)); }

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}


// block-level max of 5 non-negative fields, then one atomicMax per field per block
__device__ __forceinline__ void block_keymax(float (&m)[5], KeyMax* km) {
  __shared__ float red[5][32];
  const int lane = lane_id(), w = warp_id();
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    float v = m[f];
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL, v, o));
    if (lane == 0) red[f][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    float v = 0.f;
    for (int i = 0; i < int(blockDim.x >> 5); ++i) v = fmaxf(v, red[threadIdx.x][i]);
    unsigned* dst = &km->hi;
    atomicMax(dst + threadIdx.x, __float_as_uint(v));
  }
}

// Operand rows of the tensor-core candidate kernel.  Packed row p (original row perm[p]) goes to
// output row p, or — with a row list — list entry q (packed row rows[q], q < *nrows) goes to
// output row q.  Aop / Bop may each be null (that side is not written); the key-side statistics
// (qs, km) are written with the key side.
template <class T, int SPLIT>
__global__ void pack_tc_kernel(const float* __restrict__ X, const int32_t* __restrict__ perm,
                               const SegDesc* __restrict__ seg, int nseg,
                               const double* __restrict__ mean, int d, int kp, int prec,
                               int64_t npacked, const int32_t* __restrict__ rows,
                               const int32_t* __restrict__ nrows, T* __restrict__ Aop,
                               T* __restrict__ Bop, QStat* __restrict__ qs,
                               KeyMax* __restrict__ km, const Ctl* __restrict__ ctl,
                               double pad_term) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const double f = op_scale(prec, ctl);
  const T zero = to_op<T>(0.0);
  const T one = to_op<T>(1.0);
  const T padt = to_op<T>(pad_term);
  const int kd = SPLIT * d;                     // first column after the data terms
  const int64_t count = rows ? int64_t(*nrows) : npacked;
  float mx[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int64_t q = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; q < count;
       q += nwarps) {
    const int64_t p = rows ? int64_t(rows[q]) : q;
    const int s = find_seg(seg, nseg, p);
    const int64_t orow = perm[p];
    const bool valid = orow >= 0;
    const double* c = mean + int64_t(s) * d;
    T* arow = Aop ? Aop + q * kp : nullptr;
    T* brow = Bop ? Bop + q * kp : nullptr;
    double sq = 0.0, nh = 0.0, nl = 0.0, nr = 0.0;
    for (int t = lane; t < d; t += 32) {
      double z = valid ? (double(X[orow * d + t]) - c[t]) * f : 0.0;
      T hi = to_op<T>(z);
      double hv = op_val(hi);
      T lo = to_op<T>(SPLIT == 3 ? z - hv : 0.0);
      double lv = SPLIT == 3 ? op_val(lo) : 0.0;
      double r = z - hv - lv;
      sq += z * z;
      nh += hv * hv;
      nl += lv * lv;
      nr += r * r;
      if (SPLIT == 3) {
        if (arow) { arow[t] = hi; arow[d + t] = hi; arow[2 * d + t] = lo; }
        if (brow) {
          brow[t] = to_op<T>(-2.0 * hv); brow[d + t] = to_op<T>(-2.0 * lv);
          brow[2 * d + t] = to_op<T>(-2.0 * hv);
        }
      } else {
        if (arow) arow[t] = hi;
        if (brow) brow[t] = to_op<T>(-2.0 * hv);
      }
    }
    sq = warp_sum_d(sq); nh = warp_sum_d(nh); nl = warp_sum_d(nl); nr = warp_sum_d(nr);
    const T t1 = to_op<T>(sq);
    const double s1 = op_val(t1);
    const T t2 = to_op<T>(sq - s1);
    const double s2 = op_val(t2);
    const T t3 = to_op<T>(sq - s1 - s2);
    const double s3 = op_val(t3);
    const double nerr = fabs(sq - s1 - s2 - s3);
    for (int col = kd + lane; col < kp; col += 32) {
      const int jj = col - kd;
      if (arow) arow[col] = (jj < 3 && valid) ? one : zero;
      if (brow) {
        T v = zero;
        if (jj == 0) v = valid ? t1 : padt;
        if (jj == 1) v = valid ? t2 : padt;
        if (jj == 2) v = valid ? t3 : padt;
        brow[col] = v;
      }
    }
    if (lane == 0 && qs) {
      QStat qq;
      qq.sq = sq;
      qq.hi = __double2float_ru(sqrt(nh));
      qq.lo = __double2float_ru(sqrt(nl));
      qq.res = __double2float_ru(sqrt(nr));
      qq.pad = 0.f;
      qs[p] = qq;
      if (valid) {
        mx[0] = fmaxf(mx[0], qq.hi);
        mx[1] = fmaxf(mx[1], qq.lo);
        mx[2] = fmaxf(mx[2], qq.res);
        mx[3] = fmaxf(mx[3], __double2float_ru(nerr));
        mx[4] = fmaxf(mx[4], __double2float_ru(sq));
      }
    }
  }
  if (km) block_keymax(mx, km);
}

int launch_pack_tc(int prec, const float* X, const int32_t* perm, const SegDesc* seg, int nseg,
                   const double* mean, int d, int64_t npacked, const int32_t* rows,
                   const int32_t* nrows, int64_t max_rows, void* Aop, void* Bop, QStat* qs,
                   KeyMax* km, const Ctl* ctl, cudaStream_t st) {
  const OpLayout L = op_layout(prec, d);
  const int64_t n_out = rows ? max_rows : npacked;
  int blocks = int(std::min<int64_t>(ceil_div(n_out, 8), int64_t(num_sms()) * 16));
  blocks = std::max(blocks, 1);
  switch (prec) {
    case PREC_BF16X3:
      pack_tc_kernel<__nv_bfloat16, 3><<<blocks, 256, 0, st>>>(
          X, perm, seg, nseg, mean, d, L.kp, prec, npacked, rows, nrows,
          static_cast<__nv_bfloat16*>(Aop), static_cast<__nv_bfloat16*>(Bop), qs, km, ctl,
          PAD_NORM_TERM_BF16);
      break;
    case PREC_BF16:
      pack_tc_kernel<__nv_bfloat16, 1><<<blocks, 256, 0, st>>>(
          X, perm, seg, nseg, mean, d, L.kp, prec, npacked, rows, nrows,
          static_cast<__nv_bfloat16*>(Aop), static_cast<__nv_bfloat16*>(Bop), qs, km, ctl,
          PAD_NORM_TERM_BF16);
      break;
    case PREC_FP16:
      pack_tc_kernel<__half, 1><<<blocks, 256, 0, st>>>(
          X, perm, seg, nseg, mean, d, L.kp, prec, npacked, rows, nrows,
          static_cast<__half*>(Aop), static_cast<__half*>(Bop), qs, km, ctl, PAD_NORM_TERM_FP16);
      break;
    default:
      set_error("pack_tc: bad precision %d", prec);
      return MSC_ERR_INVALID_ARG;
  }
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// FP32 SIMT operands: A32 = fp32(z) (row stride dpad, zero padded), sq32 = fp32(Σ z²)
__global__ void pack_fp32_kernel(const float* __restrict__ X, const int32_t* __restrict__ perm,
                                 const SegDesc* __restrict__ seg, int nseg, const double* __restrict__ mean, int d, int dpad,
                                 int64_t npacked, float* __restrict__ A32,
                                 float* __restrict__ sq32, QStat* __restrict__ qs,
                                 KeyMax* __restrict__ km) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  float mx[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  for (int64_t p = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; p < npacked;
       p += nwarps) {
    const int s = find_seg(seg, nseg, p);
    const int64_t orow = perm[p];
    const bool valid = orow >= 0;
    const double* c = mean + int64_t(s) * d;
    double sq = 0.0, nh = 0.0, nr = 0.0;
    for (int t = lane; t < dpad; t += 32) {
      double z = (valid && t < d) ? double(X[orow * d + t]) - c[t] : 0.0;
      float a = __double2float_rn(z);
      double r = z - double(a);
      sq += z * z;
      nh += double(a) * double(a);
      nr += r * r;
      A32[p * dpad + t] = a;
    }
    sq = warp_sum_d(sq); nh = warp_sum_d(nh); nr = warp_sum_d(nr);
    if (lane == 0) {
      const float s32 = valid ? __double2float_rn(sq) : PAD_SQ_FP32;
      sq32[p] = s32;
      QStat q;
      q.sq = sq;
      q.hi = __double2float_ru(sqrt(nh));
      q.lo = 0.f;
      q.res = __double2float_ru(sqrt(nr));
      q.pad = 0.f;
      qs[p] = q;
      if (valid) {
        mx[0] = fmaxf(mx[0], q.hi);
        mx[2] = fmaxf(mx[2], q.res);
        mx[3] = fmaxf(mx[3], __double2float_ru(fabs(sq - double(s32))));
        mx[4] = fmaxf(mx[4], __double2float_ru(sq));
      }
    }
  }
  block_keymax(mx, km);
}

int launch_pack_fp32(const float* X, const int32_t* perm, const SegDesc* seg, int nseg,
                     const double* mean, int d, int dpad, int64_t npacked, float* A32, float* sq32,
                     QStat* qs, KeyMax* km, cudaStream_t st) {
  int blocks = int(std::min<int64_t>(ceil_div(npacked, 8), int64_t(num_sms()) * 16));
  pack_fp32_kernel<<<std::max(blocks, 1), 256, 0, st>>>(X, perm, seg, nseg, mean, d, dpad,
                                                        npacked, A32, sq32, qs, km);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// ------------------------------------------------------------------------------------------------
// tile plan on the device
// ------------------------------------------------------------------------------------------------
__global__ void single_segment_kernel(SegDesc* seg, int64_t n) {
  SegDesc s;
  s.off = 0;
  s.n = n;
  s.poff = 0;
  s.padlen = ((n + SEG_PAD - 1) / SEG_PAD) * SEG_PAD;
  s.tile0 = 0;
  s.ntiles = (n + QTILE - 1) / QTILE;
  s.ptile0 = 0;
  s.pad1 = 0;
  *seg = s;
}

int launch_single_segment(SegDesc* seg, int64_t n, cudaStream_t st) {
  single_segment_kernel<<<1, 1, 0, st>>>(seg, n);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// one work item per 128-row query tile; largest samples first so the persistent kernels'
// dynamic scheduler ends with the short items
__global__ void build_items_kernel(const SegDesc* __restrict__ seg, int nseg, int64_t n_items,
                                   int rows, WorkItem* __restrict__ items, Ctl* ctl) {
  int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (t == 0) ctl->n_items = int32_t(n_items);
  if (t >= n_items) return;
  const bool pair = rows != QTILE;
  // segment of item t: last with first item <= t
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if ((pair ? seg[mid].ptile0 : seg[mid].tile0) <= t) lo = mid; else hi = mid - 1;
  }
  const SegDesc s = seg[lo];
  const int64_t q = t - (pair ? s.ptile0 : s.tile0);
  WorkItem w;
  w.qrow0 = int32_t(s.poff + q * rows);
  w.nq = int32_t(min64(rows, s.n - q * rows));
  w.key0 = int32_t(s.poff);
  w.nkeys = int32_t(s.n);
  w.orig_off = int32_t(s.off);
  w.qorig0 = int32_t(s.off + q * rows);
  w.pad0 = w.pad1 = 0;
  items[t] = w;
}

int launch_build_items(const SegDesc* seg, int nseg, int64_t n_items, int rows, WorkItem* items,
                       Ctl* ctl, cudaStream_t st) {
  if (rows != QTILE && rows != 2 * QTILE) {
    set_error("work items of %d rows", rows);
    return MSC_ERR_INVALID_ARG;
  }
  build_items_kernel<<<unsigned(std::max<int64_t>(1, ceil_div(n_items, 256))), 256, 0, st>>>(
      seg, nseg, n_items, rows, items, ctl);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
