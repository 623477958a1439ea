// Per-row top-k selection shared by the candidate kernels (FP32 SIMT and tcgen05 epilogue).
//
// One thread owns one query row (in the tcgen05 epilogue this is forced: TMEM lane i is row i).
// It filters its row's values against the row's threshold (the k'-th smallest kept so far) in
// three levels — the minimum of a 32-column chunk, then of eleven groups of ≤3 columns, then single
// columns — so that the common case costs one vote per chunk.  Survivors are appended to a small
// per-row buffer in shared memory.  When any lane's buffer is nearly full, every lane compacts its
// own row at once: an insertion sort of the buffer, then a merge with the row's sorted k' list that
// keeps the k' smallest and yields the new threshold.  This replaces the reference's
// one-thread-per-row register insertion (`topk_rows`, metalsinglecell neighbors.py:25-49), which
// rescans all k entries on every insert.
#pragma once

#include "msc_common.cuh"

namespace msc {

// three-input minimum (PTX min.f32 with three sources, sm_100 and later); NaN inputs are ignored
// like fminf
__device__ __forceinline__ float min3f(float a, float b, float c) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fminf(fminf(a, b), c);
#endif
}

// --- the row selector -----------------------------------------------------------------------------
//
// Shared memory layout (slot-major so that the 32 rows of a warp hit 32 banks):
//   lv/li[KPL][ROWS]  sorted list per row (ascending; +inf / -1 padding), k' <= KPL entries used
//   bv/bi[CB][ROWS]   append buffer per row
template <int KPL, int CB, int ROWS>
struct RowSelect {
  static_assert(KPL == 32 || KPL == 64, "list length 32 or 64");
  static_assert(CB >= 8 && CB <= 64, "buffer 8..64");
  __host__ __device__ static constexpr size_t smem_bytes() { return size_t(KPL + CB) * ROWS * 8; }

  float* lv; int* li; float* bv; int* bi;
  int row;        // this thread's row within the ROWS rows
  int kp;         // k'
  float thr;      // this list's k'-th value
  float thr_f;    // filter threshold: min(thr, seed, the partner list's published thr)
  // An upper bound on the row's final k'-th value known before the scan (from an earlier pass
  // over a subset of its keys), +inf if none.  Values at or above it are never kept; the list's
  // threshold reported by finish() is min(list[k'-1], seed), so every value not in the list is
  // at least the reported threshold even if fewer than k' values passed the filter.
  float seed = F_INF;
  int cnt;
  // When two selectors split one row's columns, each publishes its threshold here (shared memory)
  // and filters against the smaller of the two: the k'-th smallest of the union is at most either
  // list's k'-th value, so nothing it drops can belong to the union's k' smallest.
  float* pub_own = nullptr;
  const float* pub_other = nullptr;
  int n_hot = 0, n_compact = 0, n_append = 0;   // counters for the pipeline profile

  __device__ void bind(void* smem, int row_, int kprime) {
    lv = static_cast<float*>(smem);
    li = reinterpret_cast<int*>(lv + KPL * ROWS);
    bv = reinterpret_cast<float*>(li + KPL * ROWS);
    bi = reinterpret_cast<int*>(bv + CB * ROWS);
    row = row_;
    kp = kprime;
  }

  // every owner thread resets its own row
  __device__ void reset() {
    for (int s = 0; s < KPL; ++s) {
      lv[s * ROWS + row] = F_INF;
      li[s * ROWS + row] = -1;
    }
    thr = F_INF;
    thr_f = F_INF;
    seed = F_INF;
    cnt = 0;
  }

  __device__ __forceinline__ void set_seed(float s) {
    seed = s;
    thr_f = fminf(thr_f, s);
  }

  // take the partner's latest published threshold
  __device__ __forceinline__ void refresh() {
    thr_f = fminf(thr, seed);
    if (pub_other) thr_f = fminf(thr_f, *reinterpret_cast<const volatile float*>(pub_other));
  }

  __device__ __forceinline__ void append(float v, int col) {
    bv[cnt * ROWS + row] = v;
    bi[cnt * ROWS + row] = col;
    ++cnt;
    ++n_append;
  }

  // This thread's row only (no warp collectives): merge the buffer into the sorted list.
  __device__ __noinline__ void compact_own() {
    const int n = cnt;
    if (n == 0) return;
    ++n_compact;
    float* B = bv + row;
    int* BI = bi + row;
    float* L = lv + row;
    int* LI = li + row;
    // insertion sort of the buffer (n <= CB)
    for (int i = 1; i < n; ++i) {
      const float x = B[i * ROWS];
      const int xi = BI[i * ROWS];
      int j = i - 1;
      while (j >= 0 && B[j * ROWS] > x) {
        B[(j + 1) * ROWS] = B[j * ROWS];
        BI[(j + 1) * ROWS] = BI[j * ROWS];
        --j;
      }
      B[(j + 1) * ROWS] = x;
      BI[(j + 1) * ROWS] = xi;
    }
    // how many of the k' smallest of (list ∪ buffer) come from each
    int a = 0, b = 0;
    float la = L[0], lb = B[0];
    for (int p = 0; p < kp; ++p) {
      if (lb < la) {
        ++b;
        lb = b < n ? B[b * ROWS] : F_INF;
      } else {
        ++a;
        la = a < KPL ? L[a * ROWS] : F_INF;
      }
    }
    // merge backwards in place: every list slot written has already been consumed
    int ia = a - 1, ib = b - 1;
    for (int p = kp - 1; p >= 0; --p) {
      if (ib >= 0 && (ia < 0 || B[ib * ROWS] > L[ia * ROWS])) {
        L[p * ROWS] = B[ib * ROWS];
        LI[p * ROWS] = BI[ib * ROWS];
        --ib;
      } else {
        L[p * ROWS] = L[ia * ROWS];
        LI[p * ROWS] = LI[ia * ROWS];
        --ia;
      }
    }
    thr = L[(kp - 1) * ROWS];
    cnt = 0;
    if (pub_own) *reinterpret_cast<volatile float*>(pub_own) = thr;
    thr_f = thr;
    refresh();
  }

  // Merge another selector's sorted list for the same row (same layout, base `other`) into this
  // one, keeping the k' smallest.  The buffer must be empty (after flush()).
  __device__ void merge_from(const void* other) {
    const float* O = static_cast<const float*>(other) + row;
    const int* OI = reinterpret_cast<const int*>(static_cast<const float*>(other) + KPL * ROWS) + row;
    float* L = lv + row;
    int* LI = li + row;
    int a = 0, b = 0;
    float la = L[0], lb = O[0];
    for (int p = 0; p < kp; ++p) {
      if (lb < la) {
        ++b;
        lb = b < kp ? O[b * ROWS] : F_INF;
      } else {
        ++a;
        la = a < kp ? L[a * ROWS] : F_INF;
      }
    }
    int ia = a - 1, ib = b - 1;
    for (int p = kp - 1; p >= 0; --p) {
      if (ib >= 0 && (ia < 0 || O[ib * ROWS] > L[ia * ROWS])) {
        L[p * ROWS] = O[ib * ROWS];
        LI[p * ROWS] = OI[ib * ROWS];
        --ib;
      } else {
        L[p * ROWS] = L[ia * ROWS];
        LI[p * ROWS] = LI[ia * ROWS];
        --ia;
      }
    }
    thr = L[(kp - 1) * ROWS];
    thr_f = thr;
  }

  // Offer 32 consecutive candidate columns col0..col0+31 of this row (warp-collective).
  // Columns equal to `self` or >= `limit` are never kept.  Invariant between calls: cnt <= CB-3.
  __device__ __forceinline__ void push32(const float (&v)[32], int col0, int self, int limit) {
    float g[11];
#pragma unroll
    for (int q = 0; q < 10; ++q) g[q] = min3f(v[3 * q], v[3 * q + 1], v[3 * q + 2]);
    g[10] = fminf(v[30], v[31]);
    const float n0 = min3f(g[0], g[1], g[2]), n1 = min3f(g[3], g[4], g[5]);
    const float n2 = min3f(g[6], g[7], g[8]), n3 = fminf(g[9], g[10]);
    const float mn = fminf(min3f(n0, n1, n2), n3);
    if (!__any_sync(FULL, mn < thr_f)) return;
    ++n_hot;
#pragma unroll
    for (int q = 0; q < 11; ++q) {
      if (__any_sync(FULL, g[q] < thr_f)) {
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const int e = 3 * q + t;
          if (e < 32) {
            const int c = col0 + e;
            if (v[e] < thr_f && c != self && c < limit) append(v[e], c);
          }
        }
        if (__any_sync(FULL, cnt > CB - 3)) compact_own();
      }
    }
  }

  // Offer one value (tails); warp-collective; keeps cnt <= CB-3.
  __device__ __forceinline__ void push1(float v, int c, int self, int limit) {
    if (v < thr_f && c != self && c < limit) append(v, c);
    if (__any_sync(FULL, cnt > CB - 3)) compact_own();
  }

  __device__ void flush() { compact_own(); }

  // warp-collective: flush and write the first `kout` list entries and the threshold value
  // (list[k'-1]) of the warp's first `nvalid_rows` rows.  Columns are packed positions; the
  // warp's rows are query rows first_row.. (packed positions, or through qmap when the queries
  // are a compacted row list); perm maps packed positions to original rows (the output row and
  // the stored neighbour ids).
  __device__ void finish(int* out_idx, float* out_thr, int out_stride,
                         const int32_t* __restrict__ perm, const int32_t* __restrict__ qmap,
                         int64_t first_row, int nvalid_rows, int kout) {
    compact_own();
    __syncwarp();
    const int lane = lane_id();
    const int row0 = row - lane;
    for (int r = 0; r < nvalid_rows; ++r) {
      const int rr = row0 + r;
      const int64_t prow = qmap ? int64_t(qmap[first_row + r]) : first_row + r;
      const int64_t orow = perm[prow];
      const float sd = __shfl_sync(FULL, seed, r);
      for (int s = lane; s < kout; s += 32) {
        const int c = li[s * ROWS + rr];
        out_idx[orow * out_stride + s] = c >= 0 ? perm[c] : -1;
      }
      if (lane == 0) out_thr[orow] = fminf(lv[(kp - 1) * ROWS + rr], sd);
    }
    __syncwarp();
  }
};

}  // namespace msc
