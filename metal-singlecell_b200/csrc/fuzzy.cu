// Symmetrisation of the kNN graph into a CSR matrix, on the device.
//
// Reference: umap-learn's fuzzy union inside `fuzzy_simplicial_set` (called at metalsinglecell
// neighbors.py:742-753 with set_op_mix_ratio=1):  A = coo(memberships) with zeros eliminated,
// P = A + Aᵀ − A∘Aᵀ, zeros eliminated, CSR with sorted indices.  SciPy performs that in float32, so
// P_ij = fl(fl(a + b) − fl(a·b)) with a = A_ij, b = A_ji (a missing entry counts as 0 and leaves
// the other value unchanged).  The same structure machinery serves method='gauss', whose value of a
// pair is the symmetric locally scaled Gaussian kernel.
//
// Stages (all integer work is exact, so the CSR structure is bit-exact):
//   1. count: indeg[j] += 1 per kept edge i→j (a warp walks 32 rows' lists in memory order);
//   2. exclusive scan of the in-degrees → row i's segment of the record array at i·k + rptr[i]:
//      k slots for its own list, then its reverse records;
//   3. fill: every kept edge i→j written into row j's segment as one 8-byte reverse record
//      (slot from an atomic cursor — order within the segment is arbitrary);
//   4. per row: its own list (read straight from the kNN arrays) and its reverse records sorted by
//      key = (column << 1 | reverse) — a warp bitonic network in registers up to 128 entries
//      (inline with the row's neighbours), up to 512 in a second warp-per-row pass, a block
//      network beyond — then the pairs merged (a column present in both directions) and
//      the unique entries written left-justified into the segment;
//   5. exclusive scan of the unique counts → indptr; 6. copy into indices / data.
#include "kernels.cuh"

namespace msc {

namespace {

constexpr int UW = 8;            // warps per block in the warp-per-row kernels
constexpr int BLK_SMEM_MAX = 8192;

// ------------------------------------------------------------------------------------------------
// exclusive scan of int32 counts into int64 offsets (out has n+1 entries); deterministic
// ------------------------------------------------------------------------------------------------
constexpr int SCAN_T = 1024, SCAN_E = 4, SCAN_B = SCAN_T * SCAN_E;

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* sh, int64_t& total) {
  // sh: 32 entries
  const int lane = lane_id(), w = warp_id();
  int64_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int64_t s = lane < int(blockDim.x >> 5) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(FULL, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  int64_t base = w > 0 ? sh[w - 1] : 0;
  __syncthreads();
  return base + x - v;
}

template <class T>
__global__ void scan_reduce_kernel(const T* __restrict__ in, int64_t n, int64_t* __restrict__ bsum) {
  __shared__ int64_t sh[32];
  const int64_t b0 = int64_t(blockIdx.x) * SCAN_B;
  int64_t s = 0;
  for (int e = 0; e < SCAN_E; ++e) {
    int64_t i = b0 + int64_t(e) * SCAN_T + threadIdx.x;
    if (i < n) s += int64_t(in[i]);
  }
  int64_t total;
  block_excl_scan(s, sh, total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

template <class T>
__global__ void scan_apply_kernel(const T* __restrict__ in, int64_t n,
                                  const int64_t* __restrict__ boff, int64_t* __restrict__ out) {
  __shared__ int64_t sh[32];
  const int64_t b0 = int64_t(blockIdx.x) * SCAN_B;
  int64_t v[SCAN_E];
  int64_t s = 0;
  const int64_t base_i = b0 + int64_t(threadIdx.x) * SCAN_E;     // contiguous per thread
  for (int e = 0; e < SCAN_E; ++e) {
    int64_t i = base_i + e;
    v[e] = i < n ? int64_t(in[i]) : 0;
    s += v[e];
  }
  int64_t total;
  int64_t pre = block_excl_scan(s, sh, total) + (boff ? boff[blockIdx.x] : 0);
  for (int e = 0; e < SCAN_E; ++e) {
    int64_t i = base_i + e;
    if (i < n) out[i] = pre;
    pre += v[e];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = pre;
}

size_t scan_scratch_elems(int64_t n) {
  size_t tot = 0;
  int64_t m = n;
  while (m > SCAN_B) {
    int64_t nb = ceil_div(m, SCAN_B);
    tot += size_t(nb) + 1 + size_t(nb) + 1;   // block sums and their offsets
    m = nb;
  }
  return tot + 8;
}

template <class T>
int scan_excl(const T* in, int64_t n, int64_t* out, int64_t* scratch, cudaStream_t st) {
  const int64_t nb = ceil_div(std::max<int64_t>(n, 1), SCAN_B);
  if (nb == 1) {
    scan_apply_kernel<T><<<1, SCAN_T, 0, st>>>(in, n, nullptr, out);
    MSC_LAUNCH_CHECK();
    return MSC_OK;
  }
  int64_t* bsum = scratch;
  int64_t* boff = scratch + nb + 1;
  scan_reduce_kernel<T><<<unsigned(nb), SCAN_T, 0, st>>>(in, n, bsum);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl<int64_t>(bsum, nb, boff, scratch + 2 * (nb + 1), st));
  scan_apply_kernel<T><<<unsigned(nb), SCAN_T, 0, st>>>(in, n, boff, out);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

// ------------------------------------------------------------------------------------------------
// stages 1 and 3: flat passes over the kNN lists, a warp per 32 rows
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool kept(int mode, int t, float v) {
  // umap: memberships > 0 (self has 0); gauss: every neighbour but self (column 0)
  return mode == 0 ? (v > 0.f) : (t > 0);
}

// The lanes of a warp walk the k·32 list entries of 32 consecutive rows in memory order (coalesced
// loads).  Entry x of the group is row x / k, position x % k; the division is a multiply-shift,
// exact for x < 32·k and k <= 129 (x·ceil(2^22 / k) >> 22 = floor(x / k), checked exhaustively).
__host__ __device__ __forceinline__ uint32_t div_magic(int k) {
  return uint32_t(((uint64_t(1) << 22) + uint64_t(k) - 1) / uint64_t(k));
}

template <class F>
__device__ __forceinline__ void for_each_kept_edge(int mode, const int32_t* __restrict__ idx,
                                                   const float* __restrict__ vals, int64_t n, int k,
                                                   uint32_t magic, F&& f) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; g * 32 < n;
       g += nwarps) {
    const int64_t r0 = g * 32;
    const int ne = int(min64(32, n - r0)) * k;
    const int64_t e0 = r0 * k;
    for (int x = lane; x < ne; x += 32) {
      const int r = int((uint32_t(x) * magic) >> 22);
      const int t = x - r * k;
      const int64_t i = r0 + r;
      const int32_t j = idx[e0 + x];
      const float v = vals[e0 + x];
      if (j != i && j >= 0 && j < n && kept(mode, t, v)) f(i, j, v);
    }
  }
}

__global__ void __launch_bounds__(256)
rev_count_kernel(int mode, const int32_t* __restrict__ idx, const float* __restrict__ vals,
                 int64_t n, int k, uint32_t magic, int32_t* __restrict__ indeg) {
  for_each_kept_edge(mode, idx, vals, n, k, magic,
                     [&](int64_t, int32_t j, float) { atomicAdd(&indeg[j], 1); });
}

// Row i's segment of the record array starts at i·k + rptr[i] (rptr = exclusive scan of the
// in-degrees): k slots for its own list, then its reverse records (i' → i, in any order).
__global__ void __launch_bounds__(256)
rev_fill_kernel(int mode, const int32_t* __restrict__ idx, const float* __restrict__ vals,
                int64_t n, int k, uint32_t magic, const int64_t* __restrict__ rptr,
                int32_t* __restrict__ cursor, int2* __restrict__ rec) {
  for_each_kept_edge(mode, idx, vals, n, k, magic, [&](int64_t i, int32_t j, float v) {
    const int64_t slot = int64_t(j) * k + rptr[j] + k + atomicAdd(&cursor[j], 1);
    rec[slot] = make_int2(int((uint32_t(i) << 1) | 1u), __float_as_int(v));
  });
}

// value of a merged entry (row i, column c); a/b = forward/reverse record values.  The gauss
// kernel is kept out of line: the umap merge paths stay small
__device__ __noinline__ float gauss_pair(int64_t i, uint32_t c, bool has_a, float a, float b,
                                         const double* __restrict__ sig2);
__device__ __forceinline__ float pair_value(int mode, int64_t i, uint32_t c, bool has_a, float a,
                                            bool has_b, float b, const double* __restrict__ sig2) {
  if (mode == 0) {
    if (has_a && has_b) return __fsub_rn(__fadd_rn(a, b), __fmul_rn(a, b));
    return has_a ? a : b;
  }
  return gauss_pair(i, c, has_a, a, b, sig2);
}
__device__ __noinline__ float gauss_pair(int64_t i, uint32_t c, bool has_a, float a, float b,
                                         const double* __restrict__ sig2) {
  const float dd = has_a ? a : b;                 // the pair's distance (same from both ends)
  const double d2 = double(dd) * double(dd);
  const double si2 = sig2[i], sc2 = sig2[c];
  const double num = (2.0 * sqrt(si2)) * sqrt(sc2);
  const double den = si2 + sc2;
  if (!(den > 0.0)) return 0.f;
  return __double2float_rn(sqrt(num / den) * exp(-d2 / den));
}

// ------------------------------------------------------------------------------------------------
// stage 4, warp tier: a row of L <= 32·W entries (its k list positions + its reverse records) is
// held W keys per lane, sorted by a warp bitonic network (registers and shuffles), merged and
// written back left-justified into its own segment.  Key = column << 1 | reverse, so the forward
// and the reverse record of one column sort next to each other, forward first.
// ------------------------------------------------------------------------------------------------
constexpr uint32_t SENT = 0xffffffffu;    // empty position: sorts last, never written

template <int W>
__device__ __forceinline__ void warp_bitonic(uint32_t (&key)[W], float (&val)[W]) {
  const int lane = lane_id();
#pragma unroll
  for (int size = 2; size <= 32 * W; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {                      // partner in the same lane, another register
        const int rs = stride >> 5;
#pragma unroll
        for (int w = 0; w < W; ++w) {
          if ((w & rs) == 0) {
            const int w2 = w | rs;
            const bool up = ((w * 32 + lane) & size) == 0;
            if ((key[w] > key[w2]) == up) {
              const uint32_t tk = key[w]; key[w] = key[w2]; key[w2] = tk;
              const float tv = val[w]; val[w] = val[w2]; val[w2] = tv;
            }
          }
        }
      } else {                                 // partner in lane ^ stride, same register
#pragma unroll
        for (int w = 0; w < W; ++w) {
          const uint32_t ok = __shfl_xor_sync(FULL, key[w], stride);
          const float ov = __shfl_xor_sync(FULL, val[w], stride);
          const bool up = ((w * 32 + lane) & size) == 0;
          const bool lower = (lane & stride) == 0;
          if (lower == up ? ok < key[w] : ok > key[w]) { key[w] = ok; val[w] = ov; }
        }
      }
    }
  }
}

template <int W>
__device__ __forceinline__ int merge_row_regs(int mode, int64_t i, int k, int L, int64_t n,
                                              const int32_t* __restrict__ idx,
                                              const float* __restrict__ vals, int2* seg,
                                              const double* __restrict__ sig2) {
  const int lane = lane_id();
  uint32_t key[W];
  float val[W];
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const int p = w * 32 + lane;
    key[w] = SENT;
    val[w] = 0.f;
    if (p < k) {
      const int32_t j = idx[i * k + p];
      const float v = vals[i * k + p];
      if (j != i && j >= 0 && j < n && kept(mode, p, v)) { key[w] = uint32_t(j) << 1; val[w] = v; }
    } else if (p < L) {
      const int2 r = seg[p];
      key[w] = uint32_t(r.x);
      val[w] = __int_as_float(r.y);
    }
  }
  __syncwarp();                                 // every record is read before any is rewritten
  warp_bitonic<W>(key, val);
  int written = 0;
  uint32_t carry_col = SENT;                     // column of the previous register's lane 31
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const uint32_t kk = key[w];
    const uint32_t col = kk >> 1;
    uint32_t left = __shfl_up_sync(FULL, kk == SENT ? SENT : col, 1);
    if (lane == 0) left = carry_col;
    uint32_t rk = __shfl_down_sync(FULL, kk, 1);
    float rv = __shfl_down_sync(FULL, val[w], 1);
    if (w + 1 < W) {
      const uint32_t nk = __shfl_sync(FULL, key[w + 1 < W ? w + 1 : w], 0);
      const float nv = __shfl_sync(FULL, val[w + 1 < W ? w + 1 : w], 0);
      if (lane == 31) { rk = nk; rv = nv; }
    } else if (lane == 31) {
      rk = SENT;
    }
    carry_col = __shfl_sync(FULL, kk == SENT ? SENT : col, 31);
    const bool first = kk != SENT && left != col;
    float out = 0.f;
    if (first) {
      if (rk != SENT && (rk >> 1) == col) {
        out = pair_value(mode, i, col, true, val[w], true, rv, sig2);
      } else {
        const bool rev = kk & 1u;
        out = pair_value(mode, i, col, !rev, val[w], rev, val[w], sig2);
      }
    }
    const unsigned m = __ballot_sync(FULL, first);
    if (first) seg[written + __popc(m & ((1u << lane) - 1u))] = make_int2(int(col), __float_as_int(out));
    written += __popc(m);
  }
  return written;
}

constexpr int WARP_MAX = 128;    // longest row the warp tier sorts (4 keys per lane)
constexpr int MID_MAX = 512;     // longest row the mid tier sorts (16 keys per lane)

// rows of 65..128 entries are rare: their sort stays out of line, so that the common paths (one or
// two keys per lane) keep a small instruction footprint
__device__ __noinline__ int merge_row_regs4(int mode, int64_t i, int k, int L, int64_t n,
                                            const int32_t* __restrict__ idx,
                                            const float* __restrict__ vals, int2* seg,
                                            const double* __restrict__ sig2) {
  return merge_row_regs<4>(mode, i, k, L, n, idx, vals, seg, sig2);
}

// A warp takes 32 consecutive rows at a time: their segment offsets come in one coalesced load,
// then the rows are merged one after another.
__global__ void __launch_bounds__(UW * 32)
merge_warp_kernel(int mode, int64_t n, int k, const int32_t* __restrict__ idx,
                  const float* __restrict__ vals, const int64_t* __restrict__ rptr,
                  int2* __restrict__ rec, const double* __restrict__ sig2,
                  int32_t* __restrict__ uniq, int32_t* __restrict__ big_rows,
                  int32_t* __restrict__ n_big) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; g * 32 < n;
       g += nwarps) {
    const int64_t r0 = g * 32;
    const int nr = int(min64(32, n - r0));
    const int64_t my_p0 = lane < nr ? rptr[r0 + lane] : 0;
    const int64_t my_p1 = lane < nr ? rptr[r0 + lane + 1] : 0;
    int my_u = 0;
    for (int j = 0; j < nr; ++j) {
      const int64_t i = r0 + j;
      const int64_t p0 = __shfl_sync(FULL, my_p0, j);
      const int L = k + int(__shfl_sync(FULL, my_p1, j) - p0);
      int2* seg = rec + i * k + p0;
      int u;
      if (L <= 32) {
        u = merge_row_regs<1>(mode, i, k, L, n, idx, vals, seg, sig2);
      } else if (L <= 64) {
        u = merge_row_regs<2>(mode, i, k, L, n, idx, vals, seg, sig2);
      } else if (L <= WARP_MAX) {
        u = merge_row_regs4(mode, i, k, L, n, idx, vals, seg, sig2);
      } else {
        // a long row goes to the mid or block tier: its own list into the first k slots of its
        // segment (the block tier sorts the segment in place)
        for (int t = lane; t < k; t += 32) {
          const int32_t jj = idx[i * k + t];
          const float v = vals[i * k + t];
          const bool ok = jj != i && jj >= 0 && jj < n && kept(mode, t, v);
          seg[t] = make_int2(int(ok ? (uint32_t(jj) << 1) : SENT), __float_as_int(v));
        }
        if (lane == 0) big_rows[atomicAdd(n_big, 1)] = int32_t(i);
        continue;
      }
      if (lane == j) my_u = u;
    }
    // rows of the block tier write their own count there
    const int64_t p0 = my_p0, p1 = my_p1;
    if (lane < nr && k + int(p1 - p0) <= WARP_MAX) uniq[r0 + lane] = my_u;
  }
}

// mid tier: a warp per listed long row of up to MID_MAX entries, sorted in registers (8 or 16
// keys per lane); longer rows are listed again for the block tier.  (Rows of 129..512 entries in
// the block tier -- a 1024-thread block with a barrier per network stage for a few hundred keys --
// took 1.7 ms at 1.3M cells.)
constexpr int MID_W = 8;         // warps per block
__global__ void __launch_bounds__(MID_W * 32)
merge_mid_kernel(int mode, int64_t n, int k, const int32_t* __restrict__ idx,
                 const float* __restrict__ vals, const int64_t* __restrict__ rptr,
                 int2* __restrict__ rec, const double* __restrict__ sig2,
                 int32_t* __restrict__ uniq, const int32_t* __restrict__ big_rows,
                 const int32_t* __restrict__ n_big, int32_t* __restrict__ huge_rows,
                 int32_t* __restrict__ n_huge) {
  const int lane = lane_id();
  const int nb = *n_big;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; r < nb; r += nwarps) {
    const int64_t i = big_rows[r];
    const int64_t p0 = rptr[i];
    const int L = k + int(rptr[i + 1] - p0);
    int2* seg = rec + i * k + p0;
    int u;
    if (L <= 256) {
      u = merge_row_regs<8>(mode, i, k, L, n, idx, vals, seg, sig2);
    } else if (L <= MID_MAX) {
      u = merge_row_regs<16>(mode, i, k, L, n, idx, vals, seg, sig2);
    } else {
      if (lane == 0) huge_rows[atomicAdd(n_huge, 1)] = int32_t(i);
      continue;
    }
    if (lane == 0) uniq[i] = u;
  }
}

// block tier: one block per long row; ascending-only bitonic network over the next power of two
// (positions >= L act as +inf and never move), in shared memory when the row fits, else in place
// in its segment
__global__ void __launch_bounds__(1024)
merge_block_kernel(int mode, int k, const int32_t* __restrict__ big_rows,
                   const int32_t* __restrict__ n_big, const int64_t* __restrict__ rptr,
                   int2* __restrict__ rec, const double* __restrict__ sig2,
                   int32_t* __restrict__ uniq) {
  extern __shared__ unsigned char smem[];
  const int nb = *n_big;
  for (int r = blockIdx.x; r < nb; r += gridDim.x) {
    const int64_t i = big_rows[r];
    const int64_t b = i * k + rptr[i];
    const int64_t L = k + (rptr[i + 1] - rptr[i]);
    int2* seg = rec + b;
    const bool in_smem = L <= BLK_SMEM_MAX;
    int2* S = in_smem ? reinterpret_cast<int2*>(smem) : seg;
    if (in_smem)
      for (int64_t e = threadIdx.x; e < L; e += blockDim.x) S[e] = seg[e];
    __syncthreads();
    int64_t P = 1;
    while (P < L) P <<= 1;
    for (int64_t kk = 2; kk <= P; kk <<= 1) {
      for (int64_t j = kk >> 1; j > 0; j >>= 1) {
        const bool flip = j == (kk >> 1);
        for (int64_t q = threadIdx.x; q < P / 2; q += blockDim.x) {
          const int64_t lo = (q / j) * 2 * j + (q % j);
          const int64_t hi = flip ? (lo ^ (kk - 1)) : lo + j;
          if (hi < L && uint32_t(S[hi].x) < uint32_t(S[lo].x)) {
            const int2 t = S[lo]; S[lo] = S[hi]; S[hi] = t;
          }
        }
        __syncthreads();
      }
    }
    // merge + left-justify by warp 0 (in place is safe: write position <= read position)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      int64_t written = 0;
      uint32_t prev_col = SENT;                    // the previous chunk may already be rewritten
      for (int64_t e0 = 0; e0 < L; e0 += 32) {
        const int64_t e = e0 + lane;
        const uint32_t kk = e < L ? uint32_t(S[e].x) : SENT;
        const float v = e < L ? __int_as_float(S[e].y) : 0.f;
        const uint32_t col = kk >> 1;
        uint32_t left = __shfl_up_sync(FULL, kk == SENT ? SENT : col, 1);
        if (lane == 0) left = prev_col;
        const bool first = kk != SENT && left != col;
        float out = 0.f;
        if (first) {
          const uint32_t nk = e + 1 < L ? uint32_t(S[e + 1].x) : SENT;
          if (nk != SENT && (nk >> 1) == col) {
            out = pair_value(mode, i, col, true, v, true, __int_as_float(S[e + 1].y), sig2);
          } else {
            const bool rev = kk & 1u;
            out = pair_value(mode, i, col, !rev, v, rev, v, sig2);
          }
        }
        const unsigned m = __ballot_sync(FULL, first);
        prev_col = __shfl_sync(FULL, kk == SENT ? SENT : col, 31);
        __syncwarp();                       // all reads of this chunk precede its writes
        if (first) seg[written + __popc(m & ((1u << lane) - 1u))] = make_int2(int(col), __float_as_int(out));
        __syncwarp();
        written += __popc(m);
      }
      if (lane == 0) uniq[i] = int32_t(written);
    }
    __syncthreads();
  }
}

// stage 6: copy the unique entries of every row to the output CSR
__global__ void __launch_bounds__(UW * 32)
emit_kernel(int64_t n, int k, const int64_t* __restrict__ rptr,
            const int64_t* __restrict__ outptr, const int2* __restrict__ rec,
            int32_t* __restrict__ indices, float* __restrict__ data) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int2* seg = rec + i * k + rptr[i];
    const int64_t o = outptr[i];
    const int64_t m = outptr[i + 1] - o;
    for (int64_t e = lane; e < m; e += 32) {
      const int2 r = seg[e];
      indices[o + e] = r.x;
      data[o + e] = __int_as_float(r.y);
    }
  }
}

__global__ void copy_nnz_kernel(const int64_t* __restrict__ outptr, int64_t n,
                                int64_t* __restrict__ nnz) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *nnz = outptr[n];
}

struct UnionWs {
  int32_t *indeg, *cursor, *nbig, *uniq, *big, *huge;
  int64_t *rptr, *scan;
  int2* rec;
};

UnionWs carve_union(Carver& c, int64_t n, int k) {
  UnionWs w;
  w.indeg = c.take<int32_t>(n);
  w.cursor = c.take<int32_t>(n);
  w.nbig = c.take<int32_t>(8);
  w.uniq = c.take<int32_t>(n);
  w.big = c.take<int32_t>(n);
  w.huge = c.take<int32_t>(n);
  w.rptr = c.take<int64_t>(n + 1);
  w.scan = c.take<int64_t>(scan_scratch_elems(n));
  // every row's k own slots plus at most n·k reverse records in all (n·(k-1) when every list
  // holds its own cell, as kNN lists do)
  w.rec = c.take<int2>(size_t(2) * size_t(n) * size_t(k));
  return w;
}

}  // namespace

size_t union_workspace_bytes(int64_t n, int k) {
  Carver c(nullptr);
  carve_union(c, n, k);
  return c.bytes();
}

int launch_union(int mode, const int32_t* idx, const float* vals, const double* sig2, int64_t n,
                 int k, int64_t* indptr, int32_t* indices, float* data, int64_t* nnz_dev,
                 void* ws, size_t ws_bytes, cudaStream_t st) {
  if (ws_bytes < union_workspace_bytes(n, k)) {
    set_error("fuzzy union: workspace %zu < %zu bytes", ws_bytes, union_workspace_bytes(n, k));
    return MSC_ERR_WORKSPACE;
  }
  if (n >= (int64_t(1) << 31)) { set_error("n >= 2^31"); return MSC_ERR_UNSUPPORTED; }
  if (k < 1 || k > MSC_MAX_K) { set_error("fuzzy union: k=%d out of range", k); return MSC_ERR_INVALID_ARG; }
  Carver c(ws);
  UnionWs w = carve_union(c, n, k);
  // in-degrees, cursors and the long-row counter are contiguous at the start: one memset
  MSC_CUDA_TRY(cudaMemsetAsync(w.indeg, 0, reinterpret_cast<char*>(w.uniq) - reinterpret_cast<char*>(w.indeg), st));
  const int sms = num_sms();
  const uint32_t magic = div_magic(k);
  const int g1 = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), int64_t(sms) * 8)));
  rev_count_kernel<<<g1, 256, 0, st>>>(mode, idx, vals, n, k, magic, w.indeg);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl<int32_t>(w.indeg, n, w.rptr, w.scan, st));
  rev_fill_kernel<<<g1, 256, 0, st>>>(mode, idx, vals, n, k, magic, w.rptr, w.cursor, w.rec);
  MSC_LAUNCH_CHECK();
  const int g2 = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, UW), int64_t(sms) * 16)));
  merge_warp_kernel<<<g2, UW * 32, 0, st>>>(mode, n, k, idx, vals, w.rptr, w.rec, sig2, w.uniq,
                                             w.big, w.nbig);
  MSC_LAUNCH_CHECK();
  // rows longer than WARP_MAX: a warp each up to MID_MAX (nbig[0] listed), then the longest
  // (nbig[1] listed) a block each
  merge_mid_kernel<<<sms * 4, MID_W * 32, 0, st>>>(mode, n, k, idx, vals, w.rptr, w.rec, sig2,
                                                   w.uniq, w.big, w.nbig, w.huge, w.nbig + 1);
  MSC_LAUNCH_CHECK();
  const size_t bsm = size_t(BLK_SMEM_MAX) * sizeof(int2);
  MSC_CUDA_TRY(raise_smem_cap(merge_block_kernel, bsm));
  merge_block_kernel<<<sms, 1024, bsm, st>>>(mode, k, w.huge, w.nbig + 1, w.rptr, w.rec, sig2,
                                             w.uniq);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl<int32_t>(w.uniq, n, indptr, w.scan, st));
  emit_kernel<<<g2, UW * 32, 0, st>>>(n, k, w.rptr, indptr, w.rec, indices, data);
  MSC_LAUNCH_CHECK();
  if (nnz_dev) {
    copy_nnz_kernel<<<1, 32, 0, st>>>(indptr, n, nnz_dev);
    MSC_LAUNCH_CHECK();
  }
  return MSC_OK;
}

// exclusive scan of n int32 values into n + 1 int64 values (out[n] = total), deterministic
size_t scan_i32_scratch_elems(int64_t n) { return scan_scratch_elems(n); }
int scan_excl_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* scratch, cudaStream_t st) {
  return scan_excl<int32_t>(in, n, out, scratch, st);
}

}  // namespace msc
