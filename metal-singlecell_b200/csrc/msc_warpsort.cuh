// Warp-wide ordering of (FP64 value, index) pairs: bitonic sorts of 32 and 64 pairs held one or
// two per lane, and a sorted list of the 128 smallest pairs seen so far (four per lane) that a
// full scan feeds 32 pairs at a time.  Pairs order by (value, index): the (distance, index) rule
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

// The `kk` (<= 128) smallest pairs offered so far, ascending: entry s·32 + lane in slot s of
// lane `lane`.  offer() takes one pair per lane; a batch with no pair below the current kk-th
// costs one vote.
struct WarpTop128 {
  double a[4];
  int ai[4];
  double thr;          // the kk-th smallest so far (+inf until kk pairs were offered)
  int thri;
  __device__ __forceinline__ void init() {
    const double INF = __longlong_as_double(0x7ff0000000000000ll);
#pragma unroll
    for (int s = 0; s < 4; ++s) { a[s] = INF; ai[s] = INT32_MAX; }
    thr = INF;
    thri = INT32_MAX;
  }
  __device__ __forceinline__ void offer(double v, int vi, int kk) {
    if (!__any_sync(FULL, dless(v, vi, thr, thri))) return;
    warp_sort32_d(v, vi);
    double z, u; int zi, ui;
    min_rev_d(a[3], ai[3], v, vi, z, zi, u, ui);
    warp_merge32_d(z, zi);
    // cascade: (a2, z) -> (w2, slot3), (a1, w2) -> (w1, slot2), (a0, w1) -> (slot0, slot1)
    double lw, hw; int lwi, hwi;
    min_rev_d(a[2], ai[2], z, zi, lw, lwi, hw, hwi);
    warp_merge32_d(lw, lwi); warp_merge32_d(hw, hwi);
    a[3] = hw; ai[3] = hwi;
    double lw1, hw1; int lwi1, hwi1;
    min_rev_d(a[1], ai[1], lw, lwi, lw1, lwi1, hw1, hwi1);
    warp_merge32_d(lw1, lwi1); warp_merge32_d(hw1, hwi1);
    a[2] = hw1; ai[2] = hwi1;
    double lw0, hw0; int lwi0, hwi0;
    min_rev_d(a[0], ai[0], lw1, lwi1, lw0, lwi0, hw0, hwi0);
    warp_merge32_d(lw0, lwi0); warp_merge32_d(hw0, hwi0);
    a[0] = lw0; ai[0] = lwi0; a[1] = hw0; ai[1] = hwi0;
    const int slot = (kk - 1) >> 5, src = (kk - 1) & 31;
    double tv = slot == 0 ? a[0] : slot == 1 ? a[1] : slot == 2 ? a[2] : a[3];
    int ti = slot == 0 ? ai[0] : slot == 1 ? ai[1] : slot == 2 ? ai[2] : ai[3];
    thr = __shfl_sync(FULL, tv, src);
    thri = __shfl_sync(FULL, ti, src);
  }
};

}  // namespace msc
