// Per-row top-k selection shared by the candidate kernels (FP32 SIMT and tcgen05 epilogue).
//
// One thread owns one query row (in the tcgen05 epilogue this is forced: TMEM lane i is row i).
// A thread filters its row's distances against the row's current threshold (the k'-th smallest
// value kept so far); the rare survivors are appended to a small per-row buffer in shared memory.
// When any lane's buffer is nearly full the whole warp compacts: for each row with pending
// entries, the warp loads the buffer across its 32 lanes, sorts it with a shuffle bitonic network
// and merges it into the row's sorted list (also held across the lanes during the merge), then
// publishes the new threshold.  This replaces the reference's one-thread-per-row register
// insertion (`topk_rows`, metalsinglecell neighbors.py:25-49), which rescans k entries per insert.
#pragma once

#include "msc_common.cuh"

namespace msc {

// --- warp bitonic primitives on (value, payload) pairs, ascending ------------------------------

__device__ __forceinline__ void cmpx(float& v, int& i, int j, bool keep_min) {
  float ov = __shfl_xor_sync(FULL, v, j);
  int oi = __shfl_xor_sync(FULL, i, j);
  bool take = keep_min ? (ov < v) : (ov > v);
  if (take) { v = ov; i = oi; }
}

// sort 32 values (one per lane) ascending
__device__ __forceinline__ void warp_sort32(float& v, int& i) {
  const int lane = lane_id();
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      bool up = (lane & k) == 0;
      bool lower = (lane & j) == 0;
      cmpx(v, i, j, lower == up);
    }
  }
}

// sort a bitonic sequence of 32 (one per lane) ascending
__device__ __forceinline__ void warp_merge32(float& v, int& i) {
  const int lane = lane_id();
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) cmpx(v, i, j, (lane & j) == 0);
}

// (v, i) := elementwise min / max of (a) and reversed (b); both inputs sorted ascending
__device__ __forceinline__ void min_rev(float av, int ai, float bv, int bi, float& lv, int& li,
                                        float& hv, int& hi) {
  const int lane = lane_id();
  float rv = __shfl_sync(FULL, bv, 31 - lane);
  int ri = __shfl_sync(FULL, bi, 31 - lane);
  if (rv < av) { lv = rv; li = ri; hv = av; hi = ai; }
  else { lv = av; li = ai; hv = rv; hi = ri; }
}

// --- the row selector -----------------------------------------------------------------------------
//
// Shared memory layout (slot-major so that the 32 rows of a warp hit 32 banks):
//   lv/li[KPL][ROWS]  sorted list per row (ascending; +inf / -1 padding)
//   bv/bi[CB][ROWS]   append buffer per row
// KPL is 32 or 64 (list length >= k'); CB is 16 or 32.
template <int KPL, int CB, int ROWS>
struct RowSelect {
  static_assert(KPL == 32 || KPL == 64, "list length 32 or 64");
  static_assert(CB == 8 || CB == 16 || CB == 32, "buffer 8, 16 or 32");
  __host__ __device__ static constexpr size_t smem_bytes() { return size_t(KPL + CB) * ROWS * 8; }

  float* lv; int* li; float* bv; int* bi;
  int row;        // this thread's row within the ROWS rows
  int kth;        // k'-1: position of the threshold in the sorted list
  float thr;
  int cnt;

  __device__ void bind(void* smem, int row_, int kprime) {
    lv = static_cast<float*>(smem);
    li = reinterpret_cast<int*>(lv + KPL * ROWS);
    bv = reinterpret_cast<float*>(li + KPL * ROWS);
    bi = reinterpret_cast<int*>(bv + CB * ROWS);
    row = row_;
    kth = kprime - 1;
  }

  // every owner thread resets its own row
  __device__ void reset(float init_thr = F_INF) {
#pragma unroll 4
    for (int s = 0; s < KPL; ++s) {
      lv[s * ROWS + row] = __int_as_float(0x7f800000);
      li[s * ROWS + row] = -1;
    }
    thr = init_thr;
    cnt = 0;
  }

  __device__ __forceinline__ void append(float v, int col) {
    bv[cnt * ROWS + row] = v;
    bi[cnt * ROWS + row] = col;
    ++cnt;
  }

  // warp-collective: merge every pending buffer of this warp's 32 rows into its list
  __device__ void compact() {
    const int lane = lane_id();
    const int row0 = row - lane;           // rows of a warp are consecutive
    unsigned pending = __ballot_sync(FULL, cnt > 0);
    while (pending) {
      const int r = __ffs(pending) - 1;
      pending &= pending - 1;
      const int rr = row0 + r;
      const int cr = __shfl_sync(FULL, cnt, r);
      float nv = __int_as_float(0x7f800000);
      int ni = -1;
      if (lane < cr) { nv = bv[lane * ROWS + rr]; ni = bi[lane * ROWS + rr]; }
      warp_sort32(nv, ni);
      float newthr;
      if (KPL == 32) {
        float av = lv[lane * ROWS + rr];
        int ai = li[lane * ROWS + rr];
        float zv, hv; int zi, hi;
        min_rev(av, ai, nv, ni, zv, zi, hv, hi);
        warp_merge32(zv, zi);
        lv[lane * ROWS + rr] = zv;
        li[lane * ROWS + rr] = zi;
        newthr = __shfl_sync(FULL, zv, kth & 31);
      } else {
        float a0 = lv[lane * ROWS + rr], a1 = lv[(32 + lane) * ROWS + rr];
        int i0 = li[lane * ROWS + rr], i1 = li[(32 + lane) * ROWS + rr];
        float zv, hv; int zi, hi;
        min_rev(a1, i1, nv, ni, zv, zi, hv, hi);   // 32 smallest of (a1 ∪ new), bitonic
        warp_merge32(zv, zi);
        float wv, uv; int wi, ui;
        min_rev(a0, i0, zv, zi, wv, wi, uv, ui);   // split a0 ∪ z into low / high halves
        warp_merge32(wv, wi);
        warp_merge32(uv, ui);
        lv[lane * ROWS + rr] = wv;
        li[lane * ROWS + rr] = wi;
        lv[(32 + lane) * ROWS + rr] = uv;
        li[(32 + lane) * ROWS + rr] = ui;
        float t0 = __shfl_sync(FULL, wv, kth & 31);
        float t1 = __shfl_sync(FULL, uv, kth & 31);
        newthr = kth < 32 ? t0 : t1;
      }
      if (lane == r) { thr = fminf(thr, newthr); cnt = 0; }
    }
    __syncwarp();
  }

  // Offer 32 consecutive candidate columns col0..col0+31 of this row (warp-collective).
  // Columns equal to `self` or >= `limit` are never kept.
  __device__ __forceinline__ void push32(const float (&v)[32], int col0, int self, int limit) {
    float m0 = fminf(fminf(v[0], v[1]), fminf(v[2], v[3]));
    float m1 = fminf(fminf(v[4], v[5]), fminf(v[6], v[7]));
    float m2 = fminf(fminf(v[8], v[9]), fminf(v[10], v[11]));
    float m3 = fminf(fminf(v[12], v[13]), fminf(v[14], v[15]));
    float m4 = fminf(fminf(v[16], v[17]), fminf(v[18], v[19]));
    float m5 = fminf(fminf(v[20], v[21]), fminf(v[22], v[23]));
    float m6 = fminf(fminf(v[24], v[25]), fminf(v[26], v[27]));
    float m7 = fminf(fminf(v[28], v[29]), fminf(v[30], v[31]));
    float m = fminf(fminf(fminf(m0, m1), fminf(m2, m3)), fminf(fminf(m4, m5), fminf(m6, m7)));
    if (__any_sync(FULL, m < thr)) {
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        const int c = col0 + e;
        if (v[e] < thr && c != self && c < limit) append(v[e], c);
        if ((e & 7) == 7) {
          if (__any_sync(FULL, cnt > CB - 8)) compact();
        }
      }
    }
  }

  // Offer one value (used by tails); warp-collective.  Keeps the invariant cnt <= CB - 8 between
  // calls that push32 relies on.
  __device__ __forceinline__ void push1(float v, int c, int self, int limit) {
    if (v < thr && c != self && c < limit) append(v, c);
    if (__any_sync(FULL, cnt > CB - 8)) compact();
  }

  // warp-collective: flush the buffers and write every row's first KOUT list entries and the
  // threshold value (list[k'-1]) of the warp's rows to global memory.
  __device__ void finish(int* out_idx, float* out_thr, int out_stride, int64_t first_out_row,
                         int nvalid_rows, int kout) {
    compact();
    const int lane = lane_id();
    const int row0 = row - lane;
    for (int r = 0; r < 32; ++r) {
      const int rr = row0 + r;
      const int64_t orow = first_out_row + r;
      if (r >= nvalid_rows) break;
      for (int s = lane; s < kout; s += 32) out_idx[orow * out_stride + s] = li[s * ROWS + rr];
      if (lane == 0) out_thr[orow] = lv[kth * ROWS + rr];
    }
    __syncwarp();
  }
};

}  // namespace msc
