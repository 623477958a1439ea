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


// --- the row top-k' of the tensor-core epilogue ---------------------------------------------------
//
// The same three-level filter as above, but a value that passes replaces the row's current
// k'-th value at once.  The k' (value, column) pairs of a row sit unsorted in shared memory in 8
// groups of KH/8 slots; each thread keeps, in registers, every group's largest value and its slot,
// and which group holds the overall largest (the row's threshold).  An insertion overwrites that
// slot, re-reads that one group (KH/8 independent loads) and re-takes two small maxima — a short
// dependency chain, where a binary heap's sift-down is a chain of up to log2(k') dependent
// shared-memory round trips.  The candidates' order does not matter to the callers (the re-rank
// sorts them).
//
// Shared memory (slot-major, so the 32 rows of a warp hit 32 banks whatever slot each lane is at):
//   hv[KH][ROWS]   values: +inf while free, -inf in slots >= k'
//   hc[KH][ROWS]   columns (-1 while free); kept apart so that reading values is conflict-free
template <int KH, int ROWS>
struct RowTopK {
  static_assert(KH == 32 || KH == 48 || KH == 64, "32, 48 or 64 slots");
  static constexpr int G = 8;           // groups
  static constexpr int GS = KH / G;     // slots per group
  __host__ __device__ static constexpr size_t smem_bytes() { return size_t(KH) * ROWS * 8; }

  float* hv;
  int* hc;
  int row;        // this thread's row within the ROWS rows
  int kp;         // k' (<= KH)
  float gmax[G];  // largest value of each group
  int gstar;      // group of the overall largest
  float thr;      // the k'-th smallest value kept (+inf while fewer than k' are kept)
  float thr_f;    // filter threshold: min(thr, seed, the partner's published threshold)
  // An upper bound on the row's final k'-th value known before the scan (from an earlier pass
  // over a subset of its keys), +inf if none.  Values at or above it are never kept; the
  // threshold reported by finish() is min(thr, seed), so every value not kept is at least the
  // reported threshold even if fewer than k' values passed the filter.
  float seed = F_INF;
  // When two selectors split one row's columns, each publishes its threshold here (shared
  // memory) and filters against the smaller of the two: the k'-th smallest of the union is at
  // most either one's k'-th value, so nothing it drops can belong to the union's k' smallest.
  float* pub_own = nullptr;
  const float* pub_other = nullptr;
  // columns never offered again: [ex_r0, ex_r1) and [ex_o0, ex_o1) (keys whose values an earlier
  // pass already put into the list this one was loaded from)
  int ex_r0 = 0, ex_r1 = 0, ex_o0 = 0, ex_o1 = 0;
  int n_hot = 0, n_compact = 0, n_append = 0;   // counters for the pipeline profile
  bool prof = false;                            // also time the hot path (clock64)
  long long c_hot = 0, n_rounds = 0;

  __device__ __forceinline__ void bind(void* smem, int row_, int kprime) {
    hv = static_cast<float*>(smem);
    hc = reinterpret_cast<int*>(hv + KH * ROWS);
    row = row_;
    kp = kprime;
  }

  // the group maxima and the overall largest, from shared memory
  __device__ __forceinline__ void rescan_all() {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      float m = hv[(g * GS) * ROWS + row];
#pragma unroll
      for (int t = 1; t < GS; ++t) m = fmaxf(m, hv[(g * GS + t) * ROWS + row]);
      gmax[g] = m;
    }
    take_max();
  }

  __device__ __forceinline__ void take_max() {
    float m = gmax[0];
    int gs = 0;
#pragma unroll
    for (int g = 1; g < G; ++g)
      if (gmax[g] > m) { m = gmax[g]; gs = g; }
    thr = m;
    gstar = gs;
  }

  __device__ __forceinline__ void reset() {
    for (int s = 0; s < KH; ++s) {
      hv[s * ROWS + row] = s < kp ? F_INF : -F_INF;
      hc[s * ROWS + row] = -1;
    }
#pragma unroll
    for (int g = 0; g < G; ++g) gmax[g] = g * GS < kp ? F_INF : -F_INF;
    thr = F_INF;
    gstar = 0;
    thr_f = F_INF;
    seed = F_INF;
  }

  __device__ __forceinline__ void set_seed(float s) {
    seed = s;
    thr_f = fminf(thr_f, s);
  }

  __device__ __forceinline__ void refresh() {
    thr_f = fminf(thr, seed);
    if (pub_other) thr_f = fminf(thr_f, *reinterpret_cast<const volatile float*>(pub_other));
  }

  // warp-collective: load the lists an earlier pass wrote with finish() for the warp's first
  // nvalid_rows rows (packed rows first_row + r): k' values and original rows per row, the rows
  // mapped to packed positions through iperm.  The lanes read one row's list at a time (coalesced),
  // several rows in flight; then every lane takes its own row's group maxima.
  __device__ __forceinline__ void load_warp(const float* __restrict__ vals,
                                            const int32_t* __restrict__ idx,
                                            const int32_t* __restrict__ iperm,
                                            const int32_t* __restrict__ perm, int64_t first_row,
                                            int nvalid_rows, int stride) {
    const int lane = lane_id();
    const int row0 = row - lane;
    const int64_t my_orow = lane < nvalid_rows ? int64_t(perm[first_row + lane]) : 0;
#pragma unroll 4
    for (int r = 0; r < nvalid_rows; ++r) {
      const int64_t orow = __shfl_sync(FULL, my_orow, r);
      for (int s = lane; s < kp; s += 32) {
        const float v = vals[orow * stride + s];
        const int32_t c = idx[orow * stride + s];
        hv[s * ROWS + row0 + r] = v;
        hc[s * ROWS + row0 + r] = c >= 0 ? iperm[c] : -1;
      }
    }
    __syncwarp();
    if (lane < nvalid_rows) {
      rescan_all();
      if (pub_own) *reinterpret_cast<volatile float*>(pub_own) = thr;
      refresh();
    }
  }

  __device__ __forceinline__ static unsigned span_bits(int col0, int a, int b) {
    const int lo = max(a - col0, 0), hi = min(b - col0, 32);
    if (hi <= lo) return 0u;
    const unsigned upto = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
    return upto & ~((1u << lo) - 1u);
  }

  // (v, col) replaces the largest kept value (v < thr): the group holding it is read (its
  // largest is the slot equal to the group's maximum), the slot overwritten, the group's and the
  // overall maxima re-taken
  __device__ __forceinline__ void insert(float v, int col) {
    ++n_append;
    const int base = gstar * GS;
    float x[GS];
#pragma unroll
    for (int t = 0; t < GS; ++t) x[t] = hv[(base + t) * ROWS + row];
    int ts = GS - 1;
#pragma unroll
    for (int t = GS - 2; t >= 0; --t)
      if (x[t] == thr) ts = t;                  // the first slot holding the maximum
    hv[(base + ts) * ROWS + row] = v;
    hc[(base + ts) * ROWS + row] = col;
    float m = v;
#pragma unroll
    for (int t = 0; t < GS; ++t)
      if (t != ts) m = fmaxf(m, x[t]);
#pragma unroll
    for (int g = 0; g < G; ++g)
      if (g == gstar) gmax[g] = m;
    take_max();
    if (pub_own) *reinterpret_cast<volatile float*>(pub_own) = thr;
    refresh();
  }

  // Merge another selector of the same row (same layout, base `other`) into this one.  Nothing is
  // published meanwhile: the partner reads this row's published threshold as +inf until the next
  // tile.  Entries in the excluded ranges are skipped: both were loaded with the same earlier
  // candidates, so this one holds its own copy or has dropped the key for k' better ones.
  __device__ __forceinline__ void merge_from(const void* other) {
    const float* OV = static_cast<const float*>(other) + row;
    const int* OC = reinterpret_cast<const int*>(static_cast<const float*>(other) + KH * ROWS) + row;
    float* keep = pub_own;
    pub_own = nullptr;
    for (int s = 0; s < kp; ++s) {
      const float v = OV[s * ROWS];
      const int c = OC[s * ROWS];
      const bool loaded = (c >= ex_r0 && c < ex_r1) || (c >= ex_o0 && c < ex_o1);
      if (v < thr && !loaded) insert(v, c);
    }
    pub_own = keep;
  }

  // the e-th of 32 register values without indexing the register array (a 5-level select tree)
  __device__ __forceinline__ static float pick32(const float (&v)[32], int e) {
    float a[16], b[8], c[4], d[2];
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = (e & 1) ? v[2 * i + 1] : v[2 * i];
#pragma unroll
    for (int i = 0; i < 8; ++i) b[i] = (e & 2) ? a[2 * i + 1] : a[2 * i];
#pragma unroll
    for (int i = 0; i < 4; ++i) c[i] = (e & 4) ? b[2 * i + 1] : b[2 * i];
#pragma unroll
    for (int i = 0; i < 2; ++i) d[i] = (e & 8) ? c[2 * i + 1] : c[2 * i];
    return (e & 16) ? d[1] : d[0];
  }

  // Offer 32 consecutive candidate columns col0..col0+31 of this row (warp-collective).
  // Columns equal to `self` or >= `limit` are never kept.  Every lane first marks its values
  // below the threshold; then the lanes insert their next marked value together, so that the
  // sift-downs of the warp's 32 rows run side by side instead of one lane after another.
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
    const long long t_hot = prof ? clock64() : 0;
    unsigned m = 0u;
    if (mn < thr_f) {
#pragma unroll
      for (int e = 0; e < 32; ++e) m |= (v[e] < thr_f ? 1u : 0u) << e;
      const int ds = self - col0;
      if (ds >= 0 && ds < 32) m &= ~(1u << ds);
      const int dl = limit - col0;
      if (dl < 32) m &= dl <= 0 ? 0u : ((1u << dl) - 1u);
      m &= ~(span_bits(col0, ex_r0, ex_r1) | span_bits(col0, ex_o0, ex_o1));
    }
    while (__any_sync(FULL, m != 0u)) {
      ++n_rounds;
      if (m) {
        const int e = __ffs(m) - 1;
        m &= m - 1u;
        const float x = pick32(v, e);
        if (x < thr_f) insert(x, col0 + e);
      }
    }
    if (prof) c_hot += clock64() - t_hot;
  }

  __device__ __forceinline__ void push1(float v, int c, int self, int limit) {
    if (v < thr_f && c != self && c < limit) insert(v, c);
  }

  __device__ __forceinline__ void flush() {}

  // warp-collective: the first nvalid_rows rows of the warp into part (k' (value, original row)
  // per row, rows at part_row0 + r) and part_thr (min(thr, seed)), for a later merge
  __device__ __forceinline__ void finish_partial(int2* part, float* part_thr, int64_t part_row0,
                                 const int32_t* __restrict__ perm, int nvalid_rows, int kout) {
    __syncwarp();
    const int lane = lane_id();
    const int row0 = row - lane;
#pragma unroll 4
    for (int r = 0; r < nvalid_rows; ++r) {
      const int rr = row0 + r;
      const float sd = __shfl_sync(FULL, seed, r);
      int2* out = part + (part_row0 + r) * kout;
      for (int s = lane; s < kout; s += 32) {
        const int c = hc[s * ROWS + rr];
        out[s] = make_int2(__float_as_int(hv[s * ROWS + rr]), c >= 0 ? perm[c] : -1);
      }
      const float th = __shfl_sync(FULL, thr, r);
      if (lane == 0) part_thr[part_row0 + r] = fminf(th, sd);
    }
    __syncwarp();
  }

  // warp-collective: write the k' kept columns (slot order) and the threshold min(thr, seed) of
  // the warp's first `nvalid_rows` rows; columns are packed positions mapped to original rows
  // through perm (see RowSelect::finish)
  __device__ __forceinline__ void finish(int* out_idx, float* out_thr, int out_stride,
                         const int32_t* __restrict__ perm, const int32_t* __restrict__ qmap,
                         int64_t first_row, int nvalid_rows, int kout, float* out_val = nullptr) {
    __syncwarp();
    const int lane = lane_id();
    const int row0 = row - lane;
    int64_t my_orow = 0;
    if (lane < nvalid_rows)
      my_orow = perm[qmap ? int64_t(qmap[first_row + lane]) : first_row + lane];
#pragma unroll 4
    for (int r = 0; r < nvalid_rows; ++r) {
      const int rr = row0 + r;
      const int64_t orow = __shfl_sync(FULL, my_orow, r);
      const float sd = __shfl_sync(FULL, seed, r);
      for (int s = lane; s < kout; s += 32) {
        const int c = hc[s * ROWS + rr];
        out_idx[orow * out_stride + s] = c >= 0 ? perm[c] : -1;
        if (out_val) out_val[orow * out_stride + s] = hv[s * ROWS + rr];
      }
      const float th = __shfl_sync(FULL, thr, r);
      if (lane == 0) out_thr[orow] = fminf(th, sd);
    }
    __syncwarp();
  }
};


}  // namespace msc
