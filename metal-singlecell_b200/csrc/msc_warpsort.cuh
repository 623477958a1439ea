// Warp-wide ordering of (FP64 value, index) pairs: bitonic sorts of 32 and 64 pairs held one or
// two per lane, and a sorted list of the 32·SLOTS smallest pairs seen so far (SLOTS per lane)
// that a full scan feeds 32 pairs at a time.  Pairs order by (value, index): the (distance, index) rule
// of every neighbour list in this library.
#pragma once

#include "msc_common.cuh"

namespace msc {

__device__ __forceinline__ bool dless(double av, int ai, double bv, int bi) {
  return av < bv || (av == bv && ai < bi);
}
__device__ __forceinline__ void cmpx_d(double& v, int& i, int j, bool keep_min) {
  double ov = __shfl_xor_sync(FULL, v, j);
  int oi = __shfl_xor_sync(FULL, i, j);
  bool take = keep_min ? dless(ov, oi, v, i) : dless(v, i, ov, oi);
  if (take) { v = ov; i = oi; }
}
__device__ __forceinline__ void warp_sort32_d(double& v, int& i) {
  const int lane = lane_id();
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) cmpx_d(v, i, j, ((lane & j) == 0) == ((lane & k) == 0));
}
__device__ __forceinline__ void warp_merge32_d(double& v, int& i) {
  const int lane = lane_id();
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) cmpx_d(v, i, j, (lane & j) == 0);
}
// lo/hi := elementwise min/max of a and reversed b (both ascending), lexicographic
__device__ __forceinline__ void min_rev_d(double av, int ai, double bv, int bi, double& lv, int& li,
                                          double& hv, int& hi) {
  const int lane = lane_id();
  double rv = __shfl_sync(FULL, bv, 31 - lane);
  int ri = __shfl_sync(FULL, bi, 31 - lane);
  if (dless(rv, ri, av, ai)) { lv = rv; li = ri; hv = av; hi = ai; }
  else { lv = av; li = ai; hv = rv; hi = ri; }
}
// sort 64 pairs held as (v0,i0) lane-slot 0 and (v1,i1) lane-slot 1
__device__ __forceinline__ void warp_sort64_d(double& v0, int& i0, double& v1, int& i1) {
  warp_sort32_d(v0, i0);
  warp_sort32_d(v1, i1);
  double lv, hv; int li, hi;
  min_rev_d(v0, i0, v1, i1, lv, li, hv, hi);
  warp_merge32_d(lv, li);
  warp_merge32_d(hv, hi);
  v0 = lv; i0 = li; v1 = hv; i1 = hi;
}

// The same networks on float values alone (no index): fminf / fmaxf, one shuffle per step.  For
// values without NaN the multiset is sorted exactly; ties need no index since only the values are
// kept.
__device__ __forceinline__ void cmpx_f(float& v, int j, bool keep_min) {
  const float ov = __shfl_xor_sync(FULL, v, j);
  v = keep_min ? fminf(v, ov) : fmaxf(v, ov);
}
__device__ __forceinline__ void warp_sort32_f(float& v) {
  const int lane = lane_id();
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) cmpx_f(v, j, ((lane & j) == 0) == ((lane & k) == 0));
}
__device__ __forceinline__ void warp_merge32_f(float& v) {
  const int lane = lane_id();
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) cmpx_f(v, j, (lane & j) == 0);
}
// 64 values held as v0 (lane-slot 0) and v1 (lane-slot 1), ascending over (slot, lane)
__device__ __forceinline__ void warp_sort64_f(float& v0, float& v1) {
  warp_sort32_f(v0);
  warp_sort32_f(v1);
  const float r = __shfl_sync(FULL, v1, 31 - lane_id());
  float lo = fminf(v0, r), hi = fmaxf(v0, r);
  warp_merge32_f(lo);
  warp_merge32_f(hi);
  v0 = lo;
  v1 = hi;
}

// The `kk` (<= 32·SLOTS) smallest pairs offered so far, ascending: entry s·32 + lane in slot s of
// lane `lane`.  offer() takes one pair per lane; a batch with no pair below the current kk-th
// costs one vote.  A batch is sorted and cascaded through the slots from the last: each step
// splits (slot, carry) into its lower and upper 32 pairs, keeps the upper in the slot's successor
// and carries the lower on; the 32 pairs above the last slot are dropped.
template <int SLOTS>
struct WarpTop {
  static_assert(SLOTS >= 1 && SLOTS <= 16, "1..16 slots of 32");
  double a[SLOTS];
  int ai[SLOTS];
  double thr;          // the kk-th smallest so far (+inf until kk pairs were offered)
  int thri;
  __device__ __forceinline__ void init() {
    const double INF = __longlong_as_double(0x7ff0000000000000ll);
#pragma unroll
    for (int s = 0; s < SLOTS; ++s) { a[s] = INF; ai[s] = INT32_MAX; }
    thr = INF;
    thri = INT32_MAX;
  }
  __device__ __forceinline__ void offer(double v, int vi, int kk) {
    if (!__any_sync(FULL, dless(v, vi, thr, thri))) return;
    warp_sort32_d(v, vi);
    double c, u;
    int ci, ui;
    min_rev_d(a[SLOTS - 1], ai[SLOTS - 1], v, vi, c, ci, u, ui);
    warp_merge32_d(c, ci);                       // the lower 32 of (last slot, batch)
#pragma unroll
    for (int s = SLOTS - 2; s >= 0; --s) {
      double lo, hi;
      int li, hi_i;
      min_rev_d(a[s], ai[s], c, ci, lo, li, hi, hi_i);
      warp_merge32_d(lo, li);
      warp_merge32_d(hi, hi_i);
      a[s + 1] = hi;
      ai[s + 1] = hi_i;
      c = lo;
      ci = li;
    }
    a[0] = c;
    ai[0] = ci;
    const int slot = (kk - 1) >> 5, src = (kk - 1) & 31;
    double tv = a[0];
    int ti = ai[0];
#pragma unroll
    for (int s = 1; s < SLOTS; ++s)
      if (s == slot) { tv = a[s]; ti = ai[s]; }
    thr = __shfl_sync(FULL, tv, src);
    thri = __shfl_sync(FULL, ti, src);
  }
};
using WarpTop128 = WarpTop<4>;

}  // namespace msc
