// Key-tile pruning for the tensor-core candidate kernel: the pairs of (query tile, key tile) that
// cannot contribute a candidate are never computed.
//
// The reference computes every distance of a row block (neighbors.py:114-119); so does the plain
// form here.  An exact kNN does not need to: a key whose squared distance to row x is provably
// above x's running k'-th value can never enter x's candidate list.  This file proves it per tile
// pair with bounding balls:
//
//   1. near pass: the candidate kernel visits only each query tile's own key tile (the cells are
//      in locality order) and returns every row's k'-th smallest value thr_x.
//      R_x = thr_x + |z_x|² + 3·eps_x bounds, in the scaled space z of the operands, the squared
//      distance below which x can still take a key (eps_x = the certificate's bound on the
//      operand and accumulation error, see rerank.cu);
//   2. outliers: rows whose R_x is far above their sample's mean R (cells in no dense region)
//      move to the end of their sample, so that the balls of the tiles of regular rows stay
//      tight; the order is otherwise kept (stable partition), and so are the locality-tree leaves;
//   3. balls: every 32-row block of packed rows gets two balls (split at the first leaf boundary
//      inside the block), every 128-row query tile and every 256-row block one ball; centres are
//      float, radii are rounded up so that each ball holds all of its rows;
//   4. plan: key tile K is skipped for query tile Q when every ball u of Q and every ball w of K
//      are separated: |c_u − c_w| − r_u − r_w = L > 0 and f²·L² > max R over u's rows.  Then every
//      (x, y) with x in Q, y in K has v(x,y) = |z_x − z_y|² − |z_x|² > thr_x + 3·eps_x, so the
//      approximate value the kernel would compute is above thr_x + 2·eps_x; the k' keys behind
//      thr_x are never skipped, so the final k'-th value T_x <= thr_x + 2·eps_x, and the
//      certificate's premise (every key outside the list has approximate value >= T_x) holds for
//      skipped keys exactly as for scanned ones.  Near tiles are always visited.
//
// Each query tile gets a bit mask over its sample's key tiles (set = visit, near tiles excluded);
// the candidate kernel walks its near tiles first and then the set bits in ascending order.
#include <cstdlib>

#include "kernels.cuh"

namespace msc {

namespace {

constexpr int PR_T = 256;

// summed over plans while profiling: key tiles visited beyond the near tiles, all such tiles,
// tiles that failed level 1, tiles that reached the pair tests, pair tests
__device__ unsigned long long g_prune_tiles[5];
constexpr int SUB = 32;          // rows per sub-block (two balls each)
constexpr float NO_BALL = -1.f;  // radius of a ball without rows
constexpr double OUTLIER_FACTOR = 4.0;   // default; MSC_B200_OUTLIER_FACTOR overrides (tuning)

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// R per packed position of the near-pass layout (+inf where the row has no finite threshold;
// padding rows get NaN and are never read as rows)
__global__ void row_radius_kernel(const int32_t* __restrict__ perm, int64_t npacked,
                                  const float* __restrict__ cand_thr,
                                  const QStat* __restrict__ qs, const KeyMax* __restrict__ km,
                                  int prec, int kmma, int d, double* __restrict__ rpos) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int32_t i = perm[p];
    if (i < 0) { rpos[p] = __longlong_as_double(0x7ff8000000000000ll); continue; }
    const double thr = cand_thr[i];
    const QStat q = qs[p];
    const double r = thr + q.sq + 3.0 * cert_eps(q, *km, prec, kmma, d);
    rpos[p] = r < 1e300 ? r : __longlong_as_double(0x7ff0000000000000ll);
  }
}

// mean of the finite R of every sample, in two steps with a fixed summation order: MEAN_CHUNKS
// blocks per sample (grid y = sample) each sum a fixed slice, then one thread per sample adds the
// slices in order
constexpr int MEAN_CHUNKS = 64;
__global__ void sample_mean_partial_kernel(const SegDesc* __restrict__ seg, int nseg,
                                           const double* __restrict__ rpos,
                                           double2* __restrict__ part) {
  __shared__ double ssum[PR_T / 32], scnt[PR_T / 32];
  for (int sidx = blockIdx.y; sidx < nseg; sidx += gridDim.y) {
    const SegDesc s = seg[sidx];
    const int64_t per = (s.n + MEAN_CHUNKS - 1) / MEAN_CHUNKS;
    const int64_t j0 = int64_t(blockIdx.x) * per, j1 = min64(s.n, j0 + per);
    double sum = 0.0, cnt = 0.0;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
      const double r = rpos[s.poff + j];
      if (r < 1e300) { sum += r; cnt += 1.0; }
    }
    sum = warp_sum_d(sum);
    cnt = warp_sum_d(cnt);
    __syncthreads();
    if (lane_id() == 0) { ssum[warp_id()] = sum; scnt[warp_id()] = cnt; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < int(blockDim.x >> 5); ++w) { a += ssum[w]; b += scnt[w]; }
      part[int64_t(sidx) * MEAN_CHUNKS + blockIdx.x] = make_double2(a, b);
    }
  }
}
__global__ void sample_mean_final_kernel(const double2* __restrict__ part, int nseg,
                                         double* __restrict__ mean_out) {
  for (int sidx = blockIdx.x * blockDim.x + threadIdx.x; sidx < nseg;
       sidx += gridDim.x * blockDim.x) {
    double a = 0.0, b = 0.0;
    for (int c = 0; c < MEAN_CHUNKS; ++c) {
      const double2 v = part[int64_t(sidx) * MEAN_CHUNKS + c];
      a += v.x;
      b += v.y;
    }
    mean_out[sidx] = b > 0.0 ? a / b : __longlong_as_double(0x7ff0000000000000ll);
  }
}

__global__ void regular_flag_kernel(const int32_t* __restrict__ perm, int64_t npacked,
                                    const SegDesc* __restrict__ seg, int nseg,
                                    const double* __restrict__ rpos,
                                    const double* __restrict__ mean, double factor,
                                    int32_t* __restrict__ reg) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    if (perm[p] < 0) { reg[p] = 0; continue; }
    const double m = mean[find_seg(seg, nseg, p)];
    reg[p] = rpos[p] > factor * m ? 0 : 1;                // NaN / inf mean: regular
  }
}

// stable partition inside every sample: regular rows first, then the outliers (leaf OUTLIER_LEAF)
// The seed of a row lies strictly above thr + 2·eps: the near pass's k' keys keep values at or
// below thr + 2·eps in the scan of the new layout (the operands of a row are the same; each value is within eps of
// the exact one), so the row's final k'-th value cannot exceed it.
__global__ void partition_kernel(const int32_t* __restrict__ perm, const int32_t* __restrict__ leaf,
                                 const double* __restrict__ rpos, int64_t npacked,
                                 const SegDesc* __restrict__ seg, int nseg,
                                 const int32_t* __restrict__ reg, const int64_t* __restrict__ S,
                                 const float* __restrict__ cand_thr, const QStat* __restrict__ qs,
                                 const KeyMax* __restrict__ km, int prec, int kmma, int d, int bn,
                                 int32_t* __restrict__ perm2, int32_t* __restrict__ leaf2,
                                 double* __restrict__ rpos2, float* __restrict__ seed2,
                                 int32_t* __restrict__ iperm, int4* __restrict__ excl) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const SegDesc s = seg[find_seg(seg, nseg, p)];
    int64_t pos = p;
    int32_t lf = leaf[p];
    if (p < s.poff + s.n) {
      const int64_t before = S[p] - S[s.poff];                 // regular rows before p
      if (reg[p]) {
        pos = s.poff + before;
      } else {
        const int64_t nreg = S[s.poff + s.n] - S[s.poff];
        pos = s.poff + nreg + (p - s.poff) - before;
        lf = OUTLIER_LEAF;
      }
    }
    const int32_t i = perm[p];
    float sd = F_INF;
    if (i >= 0) {
      const double t = double(cand_thr[i]) + 2.0 * cert_eps(qs[p], *km, prec, kmma, d);
      if (t < 1e300) sd = nextafterf(__double2float_ru(t), F_INF);   // strictly above
    }
    perm2[pos] = i;
    leaf2[pos] = lf;
    rpos2[pos] = rpos[p];
    seed2[pos] = sd;
    int4 ex = make_int4(0, 0, 0, 0);
    if (i >= 0) {
      iperm[i] = int32_t(pos);
      // the near pass scored row i against key tile diag of its query tile (bn rows); those keys
      // are a run of regular rows and a run of outliers in the new order
      const int64_t qt = (p - s.poff) / QTILE;
      const int64_t a = s.poff + (qt * QTILE / bn) * bn, b = min64(a + bn, s.poff + s.n);
      const int64_t ra = S[a] - S[s.poff], rb = S[b] - S[s.poff];
      const int64_t nreg = S[s.poff + s.n] - S[s.poff];
      ex = make_int4(int(s.poff + ra), int(s.poff + rb), int(s.poff + nreg + (a - s.poff) - ra),
                     int(s.poff + nreg + (b - s.poff) - rb));
    }
    excl[pos] = ex;
  }
}

// One ball per group of G packed rows (G = 128 or 256): centre = float(mean of the rows), radius =
// max distance to that centre, rounded up.  One warp per group; lane t sums dimensions t, t+32, ...
template <int G>
__global__ void group_ball_kernel(const float* __restrict__ X, int d, int dp,
                                  const int32_t* __restrict__ perm, int64_t ngroups,
                                  float* __restrict__ centre, float* __restrict__ radius) {
  const int lane = lane_id();
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; g < ngroups;
       g += warps) {
    double s[4] = {0, 0, 0, 0};
    int cnt = 0;
    for (int r = 0; r < G; ++r) {
      const int32_t i = perm[g * G + r];
      if (i < 0) continue;
      ++cnt;
      for (int j = 0; j < 4; ++j) {
        const int t = lane + 32 * j;
        if (t < d) s[j] += X[int64_t(i) * d + t];
      }
    }
    float c[4];
    for (int j = 0; j < 4; ++j) {
      const int t = lane + 32 * j;
      c[j] = (cnt && t < d) ? float(s[j] / cnt) : 0.f;
      if (t < dp) centre[g * dp + t] = c[j];
    }
    double mx = 0.0;
    for (int r = 0; r < G; ++r) {
      const int32_t i = perm[g * G + r];
      if (i < 0) continue;
      double a = 0.0;
      for (int j = 0; j < 4; ++j) {
        const int t = lane + 32 * j;
        if (t < d) {
          const double u = double(X[int64_t(i) * d + t]) - double(c[j]);
          a += u * u;
        }
      }
      mx = fmax(mx, warp_sum_d(a));
    }
    if (lane == 0)
      radius[g] = cnt ? __double2float_ru(sqrt(mx) * (1.0 + 0x1p-40)) : NO_BALL;
  }
}

// Two balls per 32-row block, split at the first row whose leaf differs from the block's first
// row (rows of one leaf are close, rows of two leaves may lie in two clusters), and the block's
// max R.  Ball 2b covers rows [0, m), ball 2b+1 rows [m, 32).
__global__ void sub_ball_kernel(const float* __restrict__ X, int d, int dp,
                                const int32_t* __restrict__ perm,
                                const int32_t* __restrict__ leaf,
                                const double* __restrict__ rpos, int64_t nsub,
                                float* __restrict__ centre, float* __restrict__ radius,
                                double* __restrict__ rsub) {
  const int lane = lane_id();
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t b = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; b < nsub; b += warps) {
    const int64_t p0 = b * SUB;
    const int32_t my_i = perm[p0 + lane];
    const int32_t my_leaf = leaf[p0 + lane];
    const int32_t leaf0 = __shfl_sync(FULL, my_leaf, 0);
    const unsigned diff = __ballot_sync(FULL, my_leaf != leaf0);
    const int m = diff ? __ffs(diff) - 1 : SUB;
    // the block's max R over its rows (unknown radius = +inf)
    double rv = 0.0;
    if (my_i >= 0) {
      const double r = rpos[p0 + lane];
      rv = r < 1e300 ? r : __longlong_as_double(0x7ff0000000000000ll);
    }
    rv = warp_max_d(rv);
    if (lane == 0) rsub[b] = rv;
    for (int h = 0; h < 2; ++h) {
      const int r0 = h ? m : 0, r1 = h ? SUB : m;
      double s[4] = {0, 0, 0, 0};
      int cnt = 0;
      for (int r = r0; r < r1; ++r) {
        const int32_t i = __shfl_sync(FULL, my_i, r);
        if (i < 0) continue;
        ++cnt;
        for (int j = 0; j < 4; ++j) {
          const int t = lane + 32 * j;
          if (t < d) s[j] += X[int64_t(i) * d + t];
        }
      }
      float c[4];
      float* cdst = centre + (2 * b + h) * dp;
      for (int j = 0; j < 4; ++j) {
        const int t = lane + 32 * j;
        c[j] = (cnt && t < d) ? float(s[j] / cnt) : 0.f;
        if (t < dp) cdst[t] = c[j];
      }
      double mx = 0.0;
      for (int r = r0; r < r1; ++r) {
        const int32_t i = __shfl_sync(FULL, my_i, r);
        if (i < 0) continue;
        double a = 0.0;
        for (int j = 0; j < 4; ++j) {
          const int t = lane + 32 * j;
          if (t < d) {
            const double u = double(X[int64_t(i) * d + t]) - double(c[j]);
            a += u * u;
          }
        }
        mx = fmax(mx, warp_sum_d(a));
      }
      if (lane == 0)
        radius[2 * b + h] = cnt ? __double2float_ru(sqrt(mx) * (1.0 + 0x1p-40)) : NO_BALL;
    }
  }
}

// Are the balls (cu, ru) and (cw, rw) so far apart that no row of u can take a key of w?  R = max
// R over u's rows (z-space), f2 = square of the operand scale.  An empty ball is separated from
// everything; an unknown R (inf / NaN) from nothing.  Centres are n4 float4 (zero padded); the
// FP32 distance is lowered by its rounding bound (d+8 units of 2^-23 relative) before the test.
__device__ __forceinline__ bool separated(const float* __restrict__ cu, float ru, double R,
                                          const float* __restrict__ cw, float rw, int n4, int d,
                                          double f2) {
  if (ru < 0.f || rw < 0.f) return true;
  if (!(R < 1e300)) return false;
  const float4* a = reinterpret_cast<const float4*>(cu);
  const float4* b = reinterpret_cast<const float4*>(cw);
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll 4
  for (int t = 0; t < n4; ++t) {
    const float4 x = a[t], y = b[t];
    const float e0 = x.x - y.x, e1 = x.y - y.y, e2 = x.z - y.z, e3 = x.w - y.w;
    s0 = fmaf(e0, e0, s0);
    s1 = fmaf(e1, e1, s1);
    s2 = fmaf(e2, e2, s2);
    s3 = fmaf(e3, e3, s3);
  }
  const float s = (s0 + s1) + (s2 + s3);
  const double lo = double(s) * (1.0 - double(d + 8) * 0x1p-23);
  const double L = sqrt(lo) - double(ru) - double(rw);
  return L > 0.0 && f2 * L * L > R * (1.0 + 1e-9);
}

// One warp per query tile (work item).  Level 1, lane = key tile: the query tile's ball against
// the 256-row ball holding the key tile.  The key tiles of a 32-tile chunk that fail it go to
// level 2 together: (a) every query sub-ball against the key tile's ball, (b) every key sub-ball
// against the query tile's ball — a sub-ball separated there is separated from every sub-ball of
// the other side — with the (key tile, sub-ball) tests spread over the lanes; then, per key tile
// left, the remaining sub-ball pairs, one pair per lane.
constexpr int PLAN_WARPS = 4;
constexpr int PLAN_WORDS = 8;     // mask words (256 key tiles) per warp task
constexpr int PLAN_MAX_PAIRS = 32;  // sub-ball pairs tested per key tile (one per lane);
                                    // MSC_B200_PLAN_PAIRS overrides (tuning)
__global__ void __launch_bounds__(PLAN_WARPS * 32, 6)
plan_kernel(const WorkItem* __restrict__ items, int64_t n_items, int bn, int d, int dp,
            const Ctl* ctl, int prec, const float* __restrict__ qc, const float* __restrict__ qr,
            const float* __restrict__ kc, const float* __restrict__ kr,
            const float* __restrict__ sc, const float* __restrict__ sr,
            const double* __restrict__ rsub, int words, uint32_t* __restrict__ mask, int prof,
            int max_pairs) {
  extern __shared__ float4 sm4[];
  __shared__ unsigned ubits_all[PLAN_WARPS][32], wbits_all[PLAN_WARPS][32];
  const int lane = lane_id(), wib = warp_id();
  float* qball = reinterpret_cast<float*>(sm4) + wib * (9 * dp);   // [0]: tile, [1..8]: sub-balls
  unsigned* ubits = ubits_all[wib];
  unsigned* wbits = wbits_all[wib];
  const int n4 = dp / 4;
  const double f = op_scale(prec, ctl);
  const double f2 = f * f;
  const int64_t warps = int64_t(gridDim.x) * PLAN_WARPS;
  const int nv = 2 * max(1, bn / SUB);          // key sub-balls per key tile
  long long nvis = 0, ntot = 0, nl1 = 0, npt = 0, npr = 0;
  // tasks = (query tile, block of PLAN_WORDS mask words): the level-2 work of a query tile varies
  // widely, so whole tiles per warp would leave most SMs idle behind the slowest few
  const int nblk = (words + PLAN_WORDS - 1) / PLAN_WORDS;
  const int64_t ntasks = n_items * nblk;
  // consecutive warps take consecutive query tiles of the same key-tile block, so the key-side
  // centres they read are shared through L1
  for (int64_t task = int64_t(blockIdx.x) * PLAN_WARPS + wib; task < ntasks; task += warps) {
    const int wblk = int(task / n_items);
    const int64_t it = task - int64_t(wblk) * n_items;
    const WorkItem w = items[it];
    const int64_t qt = w.qrow0 / QTILE;          // 128-row tile of packed rows
    const int64_t sb0 = int64_t(w.qrow0) / SUB;  // its first 32-row block
    __syncwarp();
    for (int t = lane; t < dp; t += 32) qball[t] = qc[qt * dp + t];
    for (int u = 0; u < 8; ++u)
      for (int t = lane; t < dp; t += 32) qball[(1 + u) * dp + t] = sc[(2 * sb0 + u) * dp + t];
    __syncwarp();
    const float rq = qr[qt];
    double Rq = 0.0;
    for (int j = 0; j < 4; ++j) Rq = fmax(Rq, rsub[sb0 + j]);    // rsub is >= 0 or +inf
    const int nkt = (w.nkeys + bn - 1) / bn;
    const int diag = (w.qrow0 - w.key0) / bn;
    const int lo = max(0, diag - 2), hi = min(nkt - 1, diag + 2);
    uint32_t* out = mask + it * int64_t(words);
    const int wend = min(words, (wblk + 1) * PLAN_WORDS);
    for (int base = wblk * PLAN_WORDS * 32; base < wend * 32; base += 32) {
      const int kt = base + lane;
      bool l1 = false;                           // not separated at level 1
      if (kt < nkt && (kt < lo || kt > hi)) {
        const int64_t g = (int64_t(w.key0) + int64_t(kt) * bn) / 256;
        l1 = !separated(qball, rq, Rq, kc + g * dp, kr[g], n4, d, f2);
      }
      const uint32_t fm = __ballot_sync(FULL, l1);
      uint32_t bits = 0u;
      if (fm) {
        const int nf = __popc(fm);
        nl1 += nf;
        ubits[lane] = 0u;
        wbits[lane] = 0u;
        __syncwarp();
        // (a) query sub-ball u of failing tile i
        for (int x = lane; x < 8 * nf; x += 32) {
          const int i = x >> 3, u = x & 7;
          const int kti = base + __fns(fm, 0, i + 1);
          const int64_t g = (int64_t(w.key0) + int64_t(kti) * bn) / 256;
          if (!separated(qball + (1 + u) * dp, sr[2 * sb0 + u], rsub[sb0 + (u >> 1)],
                         kc + g * dp, kr[g], n4, d, f2))
            atomicOr(&ubits[i], 1u << u);
        }
        __syncwarp();
        // (b) key sub-ball v of failing tile i, only for the tiles (a) left open (a tile with no
        // open query sub-ball is skipped whatever (b) finds)
        const uint32_t fo = __ballot_sync(FULL, lane < nf && ubits[lane] != 0u);
        const int no = __popc(fo);
        for (int x = lane; x < nv * no; x += 32) {
          const int io = x / nv, v = x - io * nv;
          const int i = __fns(fo, 0, io + 1);
          const int kti = base + __fns(fm, 0, i + 1);
          const int64_t kb0 = (int64_t(w.key0) + int64_t(kti) * bn) / SUB;
          const float rw = sr[2 * kb0 + v];
          if (rw >= 0.f && !separated(qball, rq, Rq, sc + (2 * kb0 + v) * dp, rw, n4, d, f2))
            atomicOr(&wbits[i], 1u << v);
        }
        __syncwarp();
        for (int i = 0; i < nf; ++i) {
          const uint32_t ub = ubits[i], wb = wbits[i];
          if (!ub || !wb) continue;                 // warp-uniform
          const int kti = base + __fns(fm, 0, i + 1);
          const int64_t kb0 = (int64_t(w.key0) + int64_t(kti) * bn) / SUB;
          const int nu = __popc(ub), npair = nu * __popc(wb);
          // many overlapping sub-ball pairs: the tiles share a cluster, and testing every pair
          // would almost always end in a visit anyway
          if (npair > max_pairs) {
            bits |= 1u << (kti - base);
            continue;
          }
          ++npt;
          npr += npair;
          bool hit = false;
          for (int pr = lane; pr < npair && !hit; pr += 32) {
            const int u = __fns(ub, 0, pr % nu + 1), vv = __fns(wb, 0, pr / nu + 1);
            hit = !separated(qball + (1 + u) * dp, sr[2 * sb0 + u], rsub[sb0 + (u >> 1)],
                             sc + (2 * kb0 + vv) * dp, sr[2 * kb0 + vv], n4, d, f2);
          }
          if (__any_sync(FULL, hit)) bits |= 1u << (kti - base);
        }
      }
      if (lane == 0) {
        out[base >> 5] = bits;
        nvis += __popc(bits);
      }
    }
    if (wblk == 0) ntot += nkt - (hi - lo + 1);
  }
  if (prof && lane == 0) {
    atomicAdd(&g_prune_tiles[0], (unsigned long long)nvis);
    atomicAdd(&g_prune_tiles[1], (unsigned long long)ntot);
    atomicAdd(&g_prune_tiles[2], (unsigned long long)nl1);
    atomicAdd(&g_prune_tiles[3], (unsigned long long)npt);
    atomicAdd(&g_prune_tiles[4], (unsigned long long)npr);
  }
}


// Point test of the kept pairs, one block per (256-key tile, item slice): a key tile whose bounding
// ball is wide (cells of two clusters, or outliers spread over the whole sample) fails the ball
// tests for almost every query tile even when no key of it is near.  Here every key is a ball of
// radius 0: the pair is skipped when every key y satisfies |c_Q − y| − r_Q = L > 0 and
// f²·L² > R_Q (c_Q, r_Q the query tile's ball, R_Q the largest R of its rows), the plan's own
// separation rule.  The tile's keys are staged once in shared memory, dimension-major (a warp's
// 32 keys of one dimension hit 32 banks); the query tiles that kept the tile are listed, and each
// warp takes whole query tiles from the list: its lanes test 8 keys each and stop at the first key
// that is not separated.  A pair every key clears has its bit taken out of the mask.
constexpr int POINT_T = 256;
constexpr int POINT_SLICES = 2;    // item slices per key tile (the long lists of outlier tiles)
constexpr int POINT_LIST = 2048;   // listed query tiles per round
__global__ void __launch_bounds__(POINT_T)
point_test_kernel(const float* __restrict__ X, int d, int dp, const int32_t* __restrict__ perm,
                  const WorkItem* __restrict__ items, int64_t n_items, int bn, int words,
                  const Ctl* ctl, int prec, const float* __restrict__ qc,
                  const float* __restrict__ qr, const double* __restrict__ rsub,
                  uint32_t* __restrict__ mask, int64_t nkt_all, int prof) {
  extern __shared__ float ys[];                       // [d][256] this tile's keys
  __shared__ int32_t list[POINT_LIST];
  __shared__ int nlist, next;
  __shared__ unsigned pad_bits[256 / 32];             // keys that are padding rows
  const int tid = threadIdx.x, lane = lane_id(), wib = warp_id();
  constexpr int NW = POINT_T / 32;
  const double f = op_scale(prec, ctl);
  const double f2 = f * f;
  const double shrink = 1.0 - double(d + 8) * 0x1p-23;
  long long cleared = 0;
  if (tid < 256 / 32) pad_bits[tid] = 0u;
  for (int64_t gb = blockIdx.x; gb < nkt_all * POINT_SLICES; gb += gridDim.x) {   // block-uniform
    const int64_t g = gb / POINT_SLICES;
    const int slice = int(gb - g * POINT_SLICES);
    const int64_t p0 = g * 256;
    __syncthreads();                                   // the previous tile's keys are done with
    // keys: a warp per row (coalesced), dimension-major in shared memory
    for (int r = wib; r < 256; r += NW) {
      const int32_t i = perm[p0 + r];
      for (int t = lane; t < d; t += 32) ys[t * 256 + r] = i < 0 ? 0.f : X[int64_t(i) * d + t];
      const unsigned pb = __ballot_sync(FULL, i < 0);  // warp-uniform i: all lanes agree
      if (lane == 0) atomicOr(&pad_bits[r >> 5], (pb ? 1u : 0u) << (r & 31));
    }
    for (int64_t base = slice; base < n_items; base += int64_t(POINT_SLICES) * POINT_LIST) {
      __syncthreads();
      if (tid == 0) { nlist = 0; next = 0; }
      __syncthreads();
      for (int j = tid; j < POINT_LIST; j += POINT_T) {
        const int64_t it = base + int64_t(j) * POINT_SLICES;
        if (it < n_items) {
          const WorkItem w = items[it];
          const int64_t rel = p0 - w.key0;
          if (rel >= 0 && rel < w.nkeys) {
            const int kt = int(rel / bn);
            if (mask[it * words + (kt >> 5)] & (1u << (kt & 31)))
              list[atomicAdd(&nlist, 1)] = int32_t(it);
          }
        }
      }
      __syncthreads();
      const int nl = nlist;
      for (;;) {                                       // warp-uniform: a query tile per warp
        int k = 0;
        if (lane == 0) k = atomicAdd(&next, 1);
        k = __shfl_sync(FULL, k, 0);
        if (k >= nl) break;
        const int32_t it = list[k];
        const WorkItem w = items[it];
        const int64_t qt = w.qrow0 / QTILE, sb0 = w.qrow0 / SUB;
        double R = 0.0;
        for (int j = 0; j < 4; ++j) R = fmax(R, rsub[sb0 + j]);
        const float rq = qr[qt];
        if (!(rq >= 0.f) || !(R < 1e300)) continue;     // nothing provable for this tile
        const float* c = qc + qt * dp;
        bool all = true;
        for (int kk = 0; kk < 8 && all; ++kk) {          // keys lane + 32·kk
          const int key = lane + 32 * kk;
          bool sep = true;
          if (!((pad_bits[key >> 5] >> (key & 31)) & 1u)) {
            float acc = 0.f;
            for (int t = 0; t < d; ++t) {
              const float u = c[t] - ys[t * 256 + key];
              acc = fmaf(u, u, acc);
            }
            const double L = sqrt(double(acc) * shrink) - double(rq);
            sep = L > 0.0 && f2 * L * L > R * (1.0 + 1e-9);
          }
          all = __all_sync(FULL, sep);
        }
        if (all && lane == 0) {
          const int kt = int((p0 - w.key0) / bn);
          atomicAnd(&mask[int64_t(it) * words + (kt >> 5)], ~(1u << (kt & 31)));
          ++cleared;
        }
      }
    }
    __syncthreads();
    if (tid < 256 / 32) pad_bits[tid] = 0u;            // for the next tile
  }
  if (prof && cleared) atomicAdd(&g_prune_tiles[0], (unsigned long long)(-cleared));
}

// Visit mask of every work item of the refine pass (the rows whose one-term certificate failed,
// re-scanned with the three-term split).  A refine item holds up to 128 such rows from anywhere in
// their sample; its mask is the union of its rows' query-tile masks and near tiles.  This stays
// exact for the refine values v3 if each row's
// one-term error bound, in the unscaled space, covers the three-term one (eps1 >= f²·eps3): the
// skipped keys have v > (thr + 3·eps1)/f², the near-pass keys (never skipped) v <= (thr + eps1)/f²,
// so every skipped key's v3 lies above the refine threshold.  An item with a row where that fails
// scans every key tile.
__global__ void refine_mask_kernel(const WorkItem* __restrict__ items3,
                                   const int32_t* __restrict__ n_items3,
                                   const int32_t* __restrict__ qmap,
                                   const SegDesc* __restrict__ seg, int nseg,
                                   const uint32_t* __restrict__ mask, int words, int bn,
                                   const QStat* __restrict__ qs, const KeyMax* __restrict__ km,
                                   const QStat* __restrict__ qs3, const KeyMax* __restrict__ km3,
                                   const Ctl* __restrict__ ctl, int prec, int kmma, int kmma3,
                                   int d, uint32_t* __restrict__ mask3) {
  const int lane = lane_id();
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int nitems = *n_items3;
  const double f = op_scale(prec, ctl);
  const KeyMax K1 = *km, K3 = *km3;
  for (int64_t r = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; r < nitems; r += warps) {
    const WorkItem w = items3[r];
    const int nkt = (w.nkeys + bn - 1) / bn;
    bool ok = true;
    for (int j = lane; j < w.nq; j += 32) {
      const int32_t p = qmap[w.qrow0 + j];
      ok = ok && cert_eps(qs[p], K1, prec, kmma, d) >= f * f * cert_eps(qs3[p], K3, PREC_BF16X3, kmma3, d);
    }
    ok = __all_sync(FULL, ok);
    uint32_t* out = mask3 + r * int64_t(words);
    for (int wi = lane; wi < words; wi += 32) {
      uint32_t acc = 0u;
      if (!ok) {
        acc = 0xffffffffu;
      } else {
        for (int j = 0; j < w.nq; ++j) {
          const int32_t p = qmap[w.qrow0 + j];
          const SegDesc sg = seg[find_seg(seg, nseg, p)];
          const int64_t mi = sg.tile0 + (p - sg.poff) / QTILE;       // its query tile's item
          acc |= mask[mi * words + wi];
          const int dj = int(((p - sg.poff) / QTILE * QTILE) / bn);    // that tile's near range
          const int l0 = max(0, dj - 2) - wi * 32, h0 = min(nkt - 1, dj + 2) - wi * 32;
          for (int b = max(0, l0); b <= min(31, h0); ++b) acc |= 1u << b;
        }
      }
      // never beyond the sample (refine walks have no near phase: the item's own near tiles
      // stay in the mask)
      for (int b = 0; b < 32; ++b) {
        const int kt = wi * 32 + b;
        if (kt >= nkt) acc &= ~(1u << b);
      }
      out[wi] = acc;
    }
  }
}

// Merge of a split refine pass: warp per refine row; the S·k' entries of its S work items, the k'
// smallest kept (ties: lower lane, then lower slot).  The threshold is the k'-th smallest: each
// work item's list holds k' values at or below its own k'-th value, so the merged k'-th value is
// at most every work item's, and every key a work item dropped is at least that item's.
__global__ void refine_merge_kernel(const WorkItem* __restrict__ items3,
                                    const int32_t* __restrict__ n_items3,
                                    const Ctl* __restrict__ ctl, const int32_t* __restrict__ qmap,
                                    const int32_t* __restrict__ perm,
                                    const int2* __restrict__ part,
                                    const float* __restrict__ part_thr, int kprime,
                                    int32_t* __restrict__ cand_idx, float* __restrict__ cand_thr) {
  const int S = ctl->refine_split;
  if (S <= 1) return;
  const int lane = lane_id();
  const int nitems = *n_items3;
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int per = (S * kprime + 31) / 32;              // entries per lane (<= 16)
  for (int64_t x = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
       x < int64_t(nitems) * QTILE; x += warps) {
    const int r = int(x / QTILE), j = int(x % QTILE);
    const WorkItem w = items3[r];
    if (j >= w.nq) continue;                          // warp-uniform
    float v[16];
    int id[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      v[t] = F_INF;
      id[t] = -1;
      const int e = lane + 32 * t;
      if (t < per && e < S * kprime) {
        const int s = e / kprime, slot = e - s * kprime;
        const int2 pe = part[((int64_t(r) * S + s) * QTILE + j) * kprime + slot];
        if (pe.y >= 0) { v[t] = __int_as_float(pe.x); id[t] = pe.y; }
      }
    }
    const int64_t orow = perm[qmap[w.qrow0 + j]];
    float kth = F_INF;
    for (int o = 0; o < kprime; ++o) {
      float bv = F_INF;
      int bt = 16;
#pragma unroll
      for (int t = 0; t < 16; ++t)
        if (v[t] < bv) { bv = v[t]; bt = t; }
      // warp argmin of (value, lane)
      float mv = bv;
      int ml = lane;
      for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(FULL, mv, off);
        const int ol = __shfl_xor_sync(FULL, ml, off);
        if (ov < mv || (ov == mv && ol < ml)) { mv = ov; ml = ol; }
      }
      int out = -1;
      if (lane == ml && bt < 16) {
#pragma unroll
        for (int t = 0; t < 16; ++t)
          if (t == bt) { out = id[t]; v[t] = F_INF; }
      }
      out = __shfl_sync(FULL, out, ml);
      if (lane == 0) cand_idx[orow * kprime + o] = mv < F_INF ? out : -1;
      kth = mv;
    }
    if (lane == 0) cand_thr[orow] = kth;
  }
}

// ---- sorted visit lists of the main scan ----

// |z|² + 3·eps of every packed row of the final layout: the part of the row's radius
// R = threshold + roff that stays fixed while the scan lowers the threshold (as R is formed from
// the near pass's threshold in row_radius_kernel)
__global__ void row_offset_kernel(const int32_t* __restrict__ perm, int64_t npacked,
                                  const QStat* __restrict__ qs, const KeyMax* __restrict__ km,
                                  int prec, int kmma, int d, double* __restrict__ roff) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    if (perm[p] < 0) { roff[p] = 0.0; continue; }
    const QStat q = qs[p];
    roff[p] = q.sq + 3.0 * cert_eps(q, *km, prec, kmma, d);
  }
}

// kept far tiles per work item (warp per item)
__global__ void visit_count_kernel(const uint32_t* __restrict__ mask, int64_t n_items, int words,
                                   int32_t* __restrict__ cnt) {
  const int lane = lane_id();
  const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t it = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; it < n_items;
       it += warps) {
    int c = 0;
    for (int wi = lane; wi < words; wi += 32) c += __popc(mask[it * words + wi]);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
    if (lane == 0) cnt[it] = c;
  }
}

// Claim order of the main scan's work items, costliest first.  Cost = the far tiles the plan kept
// (every item also scans its few near tiles), in COST_BUCKETS buckets of 2^shift tiles.  The
// persistent CTAs claim items in this order, so the long items (rows whose radius reaches many
// key tiles) start first instead of ending the launch on a few SMs.
constexpr int COST_BUCKETS = 256;
__global__ void cost_hist_kernel(const int32_t* __restrict__ cnt, int64_t n_items, int shift,
                                 int32_t* __restrict__ hist) {
  __shared__ int32_t h[COST_BUCKETS];
  for (int b = threadIdx.x; b < COST_BUCKETS; b += blockDim.x) h[b] = 0;
  __syncthreads();
  for (int64_t it = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; it < n_items;
       it += int64_t(gridDim.x) * blockDim.x)
    atomicAdd(&h[min(COST_BUCKETS - 1, cnt[it] >> shift)], 1);
  __syncthreads();
  for (int b = threadIdx.x; b < COST_BUCKETS; b += blockDim.x)
    if (h[b]) atomicAdd(&hist[b], h[b]);
}
// one block of COST_BUCKETS threads: hist[b] := items in buckets above b (descending offsets)
__global__ void cost_offsets_kernel(int32_t* __restrict__ hist) {
  __shared__ int32_t h[COST_BUCKETS];
  const int b = threadIdx.x;
  h[b] = hist[b];
  __syncthreads();
  int32_t above = 0;
  for (int j = b + 1; j < COST_BUCKETS; ++j) above += h[j];
  hist[b] = above;
}
__global__ void cost_scatter_kernel(const int32_t* __restrict__ cnt, int64_t n_items, int shift,
                                    int32_t* __restrict__ off, int32_t* __restrict__ order) {
  for (int64_t it = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; it < n_items;
       it += int64_t(gridDim.x) * blockDim.x) {
    const int b = min(COST_BUCKETS - 1, cnt[it] >> shift);
    order[atomicAdd(&off[b], 1)] = int32_t(it);
  }
}

constexpr int VO_T = 256;            // threads per block of the order kernel
constexpr int VO_SORT_MAX = 8192;    // longest list sorted (longer ones keep tile order)

// One block per work item: its kept far tiles (the set bits of its mask) in order of the distance
// between the 128-row query tile's ball centre and the 256-row key ball's centre (ties by tile):
// nearest first, so the rows' thresholds fall early and later tiles rarely insert.  Each entry
// carries a stop bound: the smallest need over it and every later entry, need = f²·L²,
// L = |c_Q − c_K|·sqrt(1 − e) − r_Q − r_K (the float distance lowered by its rounding bound e as in
// separated()), rounded down, 0 when L <= 0; need <= f²·|x − y|² for every row x of the tile and
// key y of the key tile (unscaled coordinates, f = the operand scale), so once an entry's bound
// exceeds every row's radius, no later tile can give a row a candidate.
__global__ void __launch_bounds__(VO_T)
visit_order_kernel(const WorkItem* __restrict__ items, int64_t n_items, int bn, int d, int dp,
                   const Ctl* __restrict__ ctl, int prec, const float* __restrict__ qc,
                   const float* __restrict__ qr, const float* __restrict__ kc,
                   const float* __restrict__ kr, const uint32_t* __restrict__ mask, int words,
                   const int64_t* __restrict__ voff, int64_t cap,
                   unsigned long long* __restrict__ vlist, int32_t* __restrict__ ok_flag) {
  extern __shared__ unsigned long long vo_keys[];                 // [VO_SORT_MAX] dist | pos
  int32_t* vo_kt = reinterpret_cast<int32_t*>(vo_keys + VO_SORT_MAX);   // [VO_SORT_MAX]
  float* vo_need = reinterpret_cast<float*>(vo_kt + VO_SORT_MAX);       // [VO_SORT_MAX]
  float* qcen = vo_need + VO_SORT_MAX;                                  // [dp]
  int32_t* wpre = reinterpret_cast<int32_t*>(qcen + dp);                // [words + 1]
  const bool fits = voff[n_items] <= cap;
  if (blockIdx.x == 0 && threadIdx.x == 0) *ok_flag = fits ? 1 : 0;
  if (!fits) return;
  const double f = op_scale(prec, ctl);
  const double f2 = f * f;
  const double e = double(d + 8) * 0x1p-23;
  const int n4 = dp / 4;
  for (int64_t it = blockIdx.x; it < n_items; it += gridDim.x) {
    const WorkItem w = items[it];
    const int64_t o = voff[it];
    const int c = int(voff[it + 1] - o);
    if (c == 0) continue;                                         // block-uniform
    const int64_t qt = w.qrow0 / QTILE;
    __syncthreads();
    for (int t = threadIdx.x; t < dp; t += VO_T) qcen[t] = qc[qt * dp + t];
    // exclusive prefix of the words' bit counts (one thread; words is small)
    if (threadIdx.x == 0) {
      int a = 0;
      for (int wi = 0; wi < words; ++wi) { wpre[wi] = a; a += __popc(mask[it * words + wi]); }
      wpre[words] = a;
    }
    __syncthreads();
    const float rq = qr[qt];
    const bool sorted = c <= VO_SORT_MAX;
    for (int wi = threadIdx.x; wi < words; wi += VO_T) {
      uint32_t bits = mask[it * words + wi];
      int pos = wpre[wi];
      while (bits) {
        const int b = __ffs(bits) - 1;
        bits &= bits - 1u;
        const int kt = wi * 32 + b;
        if (!sorted) {                  // tile order, no stop bound (-inf never ends a walk)
          vlist[o + pos] = (static_cast<unsigned long long>(__float_as_uint(-F_INF)) << 32) |
                           uint32_t(kt);
          ++pos;
          continue;
        }
        const int64_t g = (int64_t(w.key0) + int64_t(kt) * bn) / 256;
        const float rk = kr[g];
        float dist = 0.f, need = F_INF;
        if (rq >= 0.f && rk >= 0.f) {
          const float4* a4 = reinterpret_cast<const float4*>(qcen);
          const float4* b4 = reinterpret_cast<const float4*>(kc + g * dp);
          float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
          for (int t = 0; t < n4; ++t) {
            const float4 x = a4[t], y = b4[t];
            const float e0 = x.x - y.x, e1 = x.y - y.y, e2 = x.z - y.z, e3 = x.w - y.w;
            s0 = fmaf(e0, e0, s0);
            s1 = fmaf(e1, e1, s1);
            s2 = fmaf(e2, e2, s2);
            s3 = fmaf(e3, e3, s3);
          }
          const float sum = (s0 + s1) + (s2 + s3);
          dist = sum;
          const double L = sqrt(double(sum) * (1.0 - e)) - double(rq) - double(rk);
          need = L > 0.0 ? __double2float_rd(f2 * L * L * (1.0 - 1e-12)) : 0.f;
        } else {
          dist = F_INF;                 // a ball without rows: no candidate, last
        }
        vo_kt[pos] = kt;
        vo_need[pos] = need;
        vo_keys[pos] = (static_cast<unsigned long long>(__float_as_uint(dist)) << 32) |
                       uint32_t(pos);
        ++pos;
      }
    }
    if (!sorted) continue;                                        // block-uniform
    int P2 = 1;
    while (P2 < c) P2 <<= 1;
    __syncthreads();
    for (int t = c + threadIdx.x; t < P2; t += VO_T) vo_keys[t] = ~0ull;
    __syncthreads();
    // dist >= 0, so the float bits order as the values do; pos breaks ties in tile order
    for (int kk = 2; kk <= P2; kk <<= 1) {
      for (int jj = kk >> 1; jj > 0; jj >>= 1) {
        for (int t = threadIdx.x; t < P2; t += VO_T) {
          const int u = t ^ jj;
          if (u > t) {
            const unsigned long long a = vo_keys[t], b = vo_keys[u];
            const bool up = (t & kk) == 0;
            if ((a > b) == up) { vo_keys[t] = b; vo_keys[u] = a; }
          }
        }
        __syncthreads();
      }
    }
    // suffix minimum of the stop bounds along the sorted order (one thread), then the entries
    if (threadIdx.x == 0) {
      float m = F_INF;
      for (int j = c - 1; j >= 0; --j) {
        const int p = int(uint32_t(vo_keys[j]));
        m = fminf(m, vo_need[p]);
        vlist[o + j] = (static_cast<unsigned long long>(__float_as_uint(m)) << 32) |
                       uint32_t(vo_kt[p]);
      }
    }
  }
}

int grid_for(int64_t n) {
  return int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, PR_T), int64_t(num_sms()) * 8)));
}

}  // namespace

int prune_mask_words(int64_t max_seg, int bn) {
  return int(ceil_div(ceil_div(max_seg, bn), 32));
}

PruneWs carve_prune(Carver& c, int64_t npacked, int nseg, int d, int64_t n_items, int words,
                    int64_t n, int kprime) {
  PruneWs w{};
  w.leaf = c.take<int32_t>(npacked);
  w.leaf2 = c.take<int32_t>(npacked);
  w.perm2 = c.take<int32_t>(npacked);
  w.reg = c.take<int32_t>(npacked);
  w.S = c.take<int64_t>(npacked + 1);
  w.scan_scratch = c.take<int64_t>(scan_i32_scratch_elems(npacked));
  w.rpos = c.take<double>(npacked);
  w.rpos2 = c.take<double>(npacked);
  w.mean = c.take<double>(nseg);
  w.mean_part = c.take<double2>(size_t(nseg) * MEAN_CHUNKS);
  const int64_t nq = npacked / QTILE, nk = npacked / 256, ns = npacked / SUB;
  const int dp = int(round_up(d, 4));
  w.qc = c.take<float>(size_t(nq) * dp);
  w.qr = c.take<float>(nq);
  w.kc = c.take<float>(size_t(nk) * dp);
  w.kr = c.take<float>(nk);
  w.sc = c.take<float>(size_t(2 * ns) * dp);
  w.sr = c.take<float>(2 * ns);
  w.rsub = c.take<double>(ns);
  w.mask = c.take<uint32_t>(size_t(n_items) * words);
  w.mask3 = c.take<uint32_t>(size_t(n_items) * words);
  w.cand_val = c.take<float>(size_t(n) * kprime);
  w.iperm = c.take<int32_t>(n);
  w.excl = c.take<int4>(npacked);
  w.max_split_items = int(std::min<int64_t>(256, n_items));
  const int64_t prow = int64_t(w.max_split_items) * REFINE_SPLIT * QTILE;
  w.part = c.take<int2>(size_t(prow) * kprime);
  w.part_thr = c.take<float>(prow);
  w.seed = c.take<float>(npacked);
  w.roff = c.take<double>(npacked);
  w.vcnt = c.take<int32_t>(n_items);
  w.claim = c.take<int32_t>(n_items);
  w.chist = c.take<int32_t>(COST_BUCKETS);
  w.voff = c.take<int64_t>(n_items + 1);
  w.vscan = c.take<int64_t>(scan_i32_scratch_elems(n_items));
  // kept far tiles of all work items: at most every key tile of every work item; beyond a
  // quarter of that (pruning keeps a few percent on large samples) the mask walk takes over
  const int64_t all = n_items * int64_t(words) * 32;
  w.vcap = std::min<int64_t>(all, std::max<int64_t>(int64_t(16) << 20, all / 4));
  w.vlist = c.take<unsigned long long>(w.vcap);
  return w;
}

int launch_prune_partition(const float* X, int d, const SegDesc* seg, int nseg, int64_t npacked,
                           int32_t* perm, const float* cand_thr, const QStat* qs,
                           const KeyMax* km, int prec, int kmma, int bn, const PruneWs& w,
                           cudaStream_t st) {
  (void)X;
  const int grid = grid_for(npacked);
  row_radius_kernel<<<grid, PR_T, 0, st>>>(perm, npacked, cand_thr, qs, km, prec, kmma, d, w.rpos);
  MSC_LAUNCH_CHECK();
  sample_mean_partial_kernel<<<dim3(MEAN_CHUNKS, std::min(nseg, 65535)), PR_T, 0, st>>>(
      seg, nseg, w.rpos, w.mean_part);
  MSC_LAUNCH_CHECK();
  sample_mean_final_kernel<<<(nseg + 127) / 128, 128, 0, st>>>(w.mean_part, nseg, w.mean);
  MSC_LAUNCH_CHECK();
  double factor = OUTLIER_FACTOR;
  if (const char* env = std::getenv("MSC_B200_OUTLIER_FACTOR")) {
    const double v = std::atof(env);
    if (v > 1.0) factor = v;
  }
  regular_flag_kernel<<<grid, PR_T, 0, st>>>(perm, npacked, seg, nseg, w.rpos, w.mean, factor,
                                             w.reg);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl_i32(w.reg, npacked, w.S, w.scan_scratch, st));
  partition_kernel<<<grid, PR_T, 0, st>>>(perm, w.leaf, w.rpos, npacked, seg, nseg, w.reg, w.S,
                                          cand_thr, qs, km, prec, kmma, d, bn, w.perm2,
                                          w.leaf2, w.rpos2, w.seed, w.iperm, w.excl);
  MSC_LAUNCH_CHECK();
  MSC_CUDA_TRY(cudaMemcpyAsync(perm, w.perm2, sizeof(int32_t) * npacked,
                               cudaMemcpyDeviceToDevice, st));
  return MSC_OK;
}

int prune_counters(unsigned long long* out) {
  MSC_CUDA_TRY(cudaMemcpyFromSymbol(out, g_prune_tiles, sizeof(unsigned long long) * 5));
  return MSC_OK;
}
int prune_counters_clear() {
  const unsigned long long z[5] = {0, 0, 0, 0, 0};
  MSC_CUDA_TRY(cudaMemcpyToSymbol(g_prune_tiles, z, sizeof(z)));
  return MSC_OK;
}

int launch_prune_plan(const float* X, int d, int64_t npacked, const int32_t* perm,
                      const WorkItem* items, int64_t n_items, int bn, const Ctl* ctl, int prec,
                      const PruneWs& w, int words, cudaStream_t st) {
  if (d > 128 || bn > 256 || (npacked % 256) != 0) {
    set_error("prune plan: unsupported shape (d=%d, bn=%d)", d, bn);
    return MSC_ERR_INVALID_ARG;
  }
  const int64_t nq = npacked / QTILE, nk = npacked / 256, ns = npacked / SUB;
  const int dp = int(round_up(d, 4));
  const int wgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(nq, 8), num_sms() * 16)));
  group_ball_kernel<QTILE><<<wgrid, PR_T, 0, st>>>(X, d, dp, perm, nq, w.qc, w.qr);
  MSC_LAUNCH_CHECK();
  group_ball_kernel<256><<<wgrid, PR_T, 0, st>>>(X, d, dp, perm, nk, w.kc, w.kr);
  MSC_LAUNCH_CHECK();
  const int sgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(ns, 8), num_sms() * 16)));
  sub_ball_kernel<<<sgrid, PR_T, 0, st>>>(X, d, dp, perm, w.leaf2, w.rpos2, ns, w.sc, w.sr, w.rsub);
  MSC_LAUNCH_CHECK();
  const size_t smem = size_t(PLAN_WARPS) * 9 * dp * sizeof(float);
  int max_pairs = PLAN_MAX_PAIRS;
  if (const char* env = std::getenv("MSC_B200_PLAN_PAIRS")) max_pairs = std::max(0, std::atoi(env));
  const int64_t ntasks = n_items * ceil_div(words, PLAN_WORDS);
  const int pgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(ntasks, PLAN_WARPS),
                                                              int64_t(num_sms()) * 32)));
  plan_kernel<<<pgrid, PLAN_WARPS * 32, smem, st>>>(items, n_items, bn, d, dp, ctl, prec, w.qc,
                                                    w.qr, w.kc, w.kr, w.sc, w.sr, w.rsub, words,
                                                    w.mask, profiling_enabled() ? 1 : 0,
                                                    max_pairs);
  MSC_LAUNCH_CHECK();
  // point test of the kept pairs, opt-in (MSC_B200_POINT_TEST=1).  Measured at 1.3M × 50: far
  // tiles kept 2.63 M → 1.63 M and main scan 33.4 → 28.0 ms, but the test itself costs ~15 ms
  // (every key of a separated pair is checked over all d dimensions on the CUDA cores), so the
  // graph takes 81.0 ms against 72.6 without it
  const char* pt_env = std::getenv("MSC_B200_POINT_TEST");
  if ((pt_env && *pt_env == '1') && bn == 256) {
    const size_t psmem = size_t(256) * d * sizeof(float);
    MSC_CUDA_TRY(raise_smem_cap(point_test_kernel, psmem));
    const int64_t nblk = nk * POINT_SLICES;
    const int ptgrid = int(std::max<int64_t>(1, std::min<int64_t>(nblk, int64_t(num_sms()) * 8)));
    point_test_kernel<<<ptgrid, POINT_T, psmem, st>>>(X, d, dp, perm, items, n_items, bn, words,
                                                      ctl, prec, w.qc, w.qr, w.rsub, w.mask, nk,
                                                      profiling_enabled() ? 1 : 0);
    MSC_LAUNCH_CHECK();
  }
  return MSC_OK;
}

int launch_claim_order(int64_t n_items, int words, const PruneWs& w, cudaStream_t st) {
  const int cgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n_items, 8),
                                                              int64_t(num_sms()) * 8)));
  visit_count_kernel<<<cgrid, PR_T, 0, st>>>(w.mask, n_items, words, w.vcnt);
  MSC_LAUNCH_CHECK();
  int shift = 0;
  while ((int64_t(words) * 32 >> shift) >= COST_BUCKETS) ++shift;
  MSC_CUDA_TRY(cudaMemsetAsync(w.chist, 0, sizeof(int32_t) * COST_BUCKETS, st));
  const int hgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n_items, PR_T),
                                                              int64_t(num_sms()) * 2)));
  cost_hist_kernel<<<hgrid, PR_T, 0, st>>>(w.vcnt, n_items, shift, w.chist);
  MSC_LAUNCH_CHECK();
  cost_offsets_kernel<<<1, COST_BUCKETS, 0, st>>>(w.chist);
  MSC_LAUNCH_CHECK();
  cost_scatter_kernel<<<hgrid, PR_T, 0, st>>>(w.vcnt, n_items, shift, w.chist, w.claim);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_visit_order(const WorkItem* items, int64_t n_items, int bn, int d, int64_t npacked,
                       const int32_t* perm, const Ctl* ctl, Ctl* ctl_w, int prec, int kmma,
                       const QStat* qs, const KeyMax* km, const PruneWs& w, int words,
                       cudaStream_t st, bool* built) {
  *built = false;
  // opt-in (MSC_B200_ORDERED=1): on clustered 50-dimensional data the nearest-ball-first order
  // left the insertions per row and the scanned tiles almost unchanged (the rows of one cluster
  // are nearly equidistant), and building the lists cost about what the main scan saved
  const char* env = std::getenv("MSC_B200_ORDERED");
  if (!(env && *env == '1')) return MSC_OK;
  const int dp = int(round_up(d, 4));
  const size_t smem = size_t(VO_SORT_MAX) * 16 + size_t(dp) * 4 + size_t(words + 1) * 4;
  if (bn != 256 || d > 128 || smem > size_t(200) * 1024) return MSC_OK;
  row_offset_kernel<<<grid_for(npacked), PR_T, 0, st>>>(perm, npacked, qs, km, prec, kmma, d,
                                                        w.roff);
  MSC_LAUNCH_CHECK();
  const int cgrid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n_items, 8),
                                                              int64_t(num_sms()) * 8)));
  visit_count_kernel<<<cgrid, PR_T, 0, st>>>(w.mask, n_items, words, w.vcnt);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl_i32(w.vcnt, n_items, w.voff, w.vscan, st));
  MSC_CUDA_TRY(raise_smem_cap(visit_order_kernel, smem));
  const int ogrid = int(std::max<int64_t>(1, std::min<int64_t>(n_items, int64_t(num_sms()) * 4)));
  visit_order_kernel<<<ogrid, VO_T, smem, st>>>(items, n_items, bn, d, dp, ctl, prec, w.qc, w.qr,
                                                w.kc, w.kr, w.mask, words, w.voff, w.vcap,
                                                w.vlist, &ctl_w->ordered_ok);
  MSC_LAUNCH_CHECK();
  *built = true;
  return MSC_OK;
}

int launch_refine_mask(const WorkItem* items3, const int32_t* n_items3, const int32_t* qmap,
                       int64_t max_items, const SegDesc* seg, int nseg, int bn, int words,
                       const QStat* qs, const KeyMax* km, const QStat* qs3, const KeyMax* km3,
                       const Ctl* ctl, int prec, int kmma, int kmma3, int d, const PruneWs& w,
                       cudaStream_t st) {
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(max_items, 8),
                                                             int64_t(num_sms()) * 8)));
  refine_mask_kernel<<<grid, PR_T, 0, st>>>(items3, n_items3, qmap, seg, nseg, w.mask, words, bn,
                                            qs, km, qs3, km3, ctl, prec, kmma, kmma3, d, w.mask3);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

int launch_refine_merge(const WorkItem* items3, const int32_t* n_items3, const Ctl* ctl,
                        const int32_t* qmap, const int32_t* perm, int64_t max_rows,
                        const PruneWs& w, int kprime, int32_t* cand_idx, float* cand_thr,
                        cudaStream_t st) {
  const int64_t rows = std::min<int64_t>(max_rows, int64_t(w.max_split_items) * QTILE);
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(rows, 8),
                                                             int64_t(num_sms()) * 8)));
  refine_merge_kernel<<<grid, PR_T, 0, st>>>(items3, n_items3, ctl, qmap, perm, w.part,
                                             w.part_thr, kprime, cand_idx, cand_thr);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
