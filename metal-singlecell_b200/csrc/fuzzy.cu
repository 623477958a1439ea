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
//   1. count: fwd[i] = kept entries of row i; indeg[j] += 1 per kept edge i→j;
//   2. exclusive scan of fwd+indeg → per-row segment offsets;
//   3. fill: row i's own entries, then every edge i→j scattered into row j's segment as a
//      "reverse" record (slot from an atomic cursor — order within the segment is arbitrary);
//   4. per row: sort the records by key = (column << 1 | reverse) — warp rank sort up to 256,
//      block bitonic beyond — then merge the pairs (a column present in both directions) and
//      write the unique entries left-justified;
//   5. exclusive scan of the unique counts → indptr; 6. copy into indices / data.
#include "kernels.cuh"

namespace msc {

namespace {

constexpr int UW = 8;            // warps per block in the warp-per-row kernels
constexpr int WARP_MAX = 256;    // longest row the warp tier sorts
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
// stages 1 and 3
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool kept(int mode, int t, float v) {
  // umap: memberships > 0 (self has 0); gauss: every neighbour but self (column 0)
  return mode == 0 ? (v > 0.f) : (t > 0);
}

__global__ void count_kernel(int mode, const int32_t* __restrict__ idx,
                             const float* __restrict__ vals, int64_t n, int k,
                             int32_t* __restrict__ fwd, int32_t* __restrict__ indeg) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    int c = 0;
    for (int t = 0; t < k; ++t) {
      const int64_t e = i * k + t;
      const int32_t j = idx[e];
      if (j != i && j >= 0 && j < n && kept(mode, t, vals[e])) {
        ++c;
        atomicAdd(&indeg[j], 1);
      }
    }
    fwd[i] = c;
  }
}

__global__ void seglen_kernel(const int32_t* __restrict__ fwd, const int32_t* __restrict__ indeg,
                              int64_t n, int32_t* __restrict__ len) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    len[i] = fwd[i] + indeg[i];
}

__global__ void fill_kernel(int mode, const int32_t* __restrict__ idx,
                            const float* __restrict__ vals, int64_t n, int k,
                            const int64_t* __restrict__ segptr, const int32_t* __restrict__ fwd,
                            int32_t* __restrict__ cursor, uint32_t* __restrict__ rkey,
                            float* __restrict__ rval) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    int64_t own = segptr[i];
    for (int t = 0; t < k; ++t) {
      const int64_t e = i * k + t;
      const int32_t j = idx[e];
      const float v = vals[e];
      if (j == i || j < 0 || j >= n || !kept(mode, t, v)) continue;
      rkey[own] = uint32_t(j) << 1;
      rval[own] = v;
      ++own;
      const int64_t slot = segptr[j] + fwd[j] + atomicAdd(&cursor[j], 1);
      rkey[slot] = (uint32_t(i) << 1) | 1u;
      rval[slot] = v;
    }
  }
}

// value of a merged entry (row i, column c); a/b = forward/reverse record values
__device__ __forceinline__ float pair_value(int mode, int64_t i, uint32_t c, bool has_a, float a,
                                            bool has_b, float b, const double* __restrict__ sig2) {
  if (mode == 0) {
    if (has_a && has_b) return __fsub_rn(__fadd_rn(a, b), __fmul_rn(a, b));
    return has_a ? a : b;
  }
  const float dd = has_a ? a : b;                 // the pair's distance (same from both ends)
  const double d2 = double(dd) * double(dd);
  const double si2 = sig2[i], sc2 = sig2[c];
  const double num = (2.0 * sqrt(si2)) * sqrt(sc2);
  const double den = si2 + sc2;
  if (!(den > 0.0)) return 0.f;
  return __double2float_rn(sqrt(num / den) * exp(-d2 / den));
}

// ------------------------------------------------------------------------------------------------
// stage 4, warp tier: rows of length <= WARP_MAX; longer rows are queued for the block tier
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(UW * 32)
merge_warp_kernel(int mode, int64_t n, const int64_t* __restrict__ segptr,
                  uint32_t* __restrict__ rkey, float* __restrict__ rval,
                  const double* __restrict__ sig2, int32_t* __restrict__ uniq,
                  int32_t* __restrict__ big_rows, int32_t* __restrict__ n_big) {
  __shared__ uint32_t sk_all[UW][WARP_MAX];
  __shared__ float sv_all[UW][WARP_MAX];
  const int lane = lane_id(), wib = warp_id();
  uint32_t* sk = sk_all[wib];
  float* sv = sv_all[wib];
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int64_t b = segptr[i];
    const int L = int(segptr[i + 1] - b);
    if (L > WARP_MAX) {
      if (lane == 0) big_rows[atomicAdd(n_big, 1)] = int32_t(i);
      continue;
    }
    // rank sort into shared memory (keys are distinct within a row)
    for (int e = lane; e < L; e += 32) {
      const uint32_t key = rkey[b + e];
      int r = 0;
      for (int f = 0; f < L; ++f) r += rkey[b + f] < key;
      sk[r] = key;
      sv[r] = rval[b + e];
    }
    __syncwarp();
    // merge pairs and write unique entries left-justified
    int written = 0;
    uint32_t prev_col = 0xffffffffu;               // column of the previous chunk's last entry
    for (int e0 = 0; e0 < L; e0 += 32) {
      const int e = e0 + lane;
      bool uniq_e = false;
      uint32_t col = 0xffffffffu;
      float val = 0.f;
      const uint32_t left = __shfl_up_sync(FULL, e < L ? (sk[e] >> 1) : 0xffffffffu, 1);
      if (e < L) {
        const uint32_t key = sk[e];
        col = key >> 1;
        const bool second = (lane == 0 ? prev_col : left) == col;
        if (!second) {
          uniq_e = true;
          const bool rev = key & 1u;
          const bool nxt = e + 1 < L && (sk[e + 1] >> 1) == col;
          if (nxt) val = pair_value(mode, i, col, true, sv[e], true, sv[e + 1], sig2);
          else val = pair_value(mode, i, col, !rev, sv[e], rev, sv[e], sig2);
        }
      }
      const unsigned m = __ballot_sync(FULL, uniq_e);
      const int pos = written + __popc(m & ((1u << lane) - 1u));
      prev_col = __shfl_sync(FULL, col, 31);
      __syncwarp();
      if (uniq_e) {
        rkey[b + pos] = col;
        rval[b + pos] = val;
      }
      written += __popc(m);
    }
    if (lane == 0) uniq[i] = written;
    __syncwarp();
  }
}

// block tier: one block per long row; ascending-only bitonic network over the next power of two
// (positions >= L act as +inf and never move), in shared memory when the row fits, else in place
// in global memory
__global__ void __launch_bounds__(1024)
merge_block_kernel(int mode, const int32_t* __restrict__ big_rows, const int32_t* __restrict__ n_big,
                   const int64_t* __restrict__ segptr, uint32_t* __restrict__ rkey,
                   float* __restrict__ rval, const double* __restrict__ sig2,
                   int32_t* __restrict__ uniq) {
  extern __shared__ unsigned char smem[];
  const int nb = *n_big;
  for (int r = blockIdx.x; r < nb; r += gridDim.x) {
    const int64_t i = big_rows[r];
    const int64_t b = segptr[i];
    const int64_t L = segptr[i + 1] - b;
    const bool in_smem = L <= BLK_SMEM_MAX;
    uint32_t* K = in_smem ? reinterpret_cast<uint32_t*>(smem) : rkey + b;
    float* V = in_smem ? reinterpret_cast<float*>(smem + BLK_SMEM_MAX * 4) : rval + b;
    if (in_smem) {
      for (int64_t e = threadIdx.x; e < L; e += blockDim.x) { K[e] = rkey[b + e]; V[e] = rval[b + e]; }
    }
    __syncthreads();
    int64_t P = 1;
    while (P < L) P <<= 1;
    for (int64_t kk = 2; kk <= P; kk <<= 1) {
      for (int64_t j = kk >> 1; j > 0; j >>= 1) {
        const bool flip = j == (kk >> 1);
        for (int64_t q = threadIdx.x; q < P / 2; q += blockDim.x) {
          const int64_t lo = (q / j) * 2 * j + (q % j);
          const int64_t hi = flip ? (lo ^ (kk - 1)) : lo + j;
          if (hi < L && K[hi] < K[lo]) {
            uint32_t tk = K[lo]; K[lo] = K[hi]; K[hi] = tk;
            float tv = V[lo]; V[lo] = V[hi]; V[hi] = tv;
          }
        }
        __syncthreads();
      }
    }
    // merge + left-justify by warp 0 (in place is safe: write position <= read position)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      int64_t written = 0;
      uint32_t prev_col = 0xffffffffu;             // the previous chunk may already be rewritten
      for (int64_t e0 = 0; e0 < L; e0 += 32) {
        const int64_t e = e0 + lane;
        bool uniq_e = false;
        uint32_t col = 0xffffffffu;
        float val = 0.f;
        const uint32_t left = __shfl_up_sync(FULL, e < L ? (K[e] >> 1) : 0xffffffffu, 1);
        if (e < L) {
          const uint32_t key = K[e];
          col = key >> 1;
          const bool second = (lane == 0 ? prev_col : left) == col;
          if (!second) {
            uniq_e = true;
            const bool rev = key & 1u;
            const bool nxt = e + 1 < L && (K[e + 1] >> 1) == col;
            if (nxt) val = pair_value(mode, i, col, true, V[e], true, V[e + 1], sig2);
            else val = pair_value(mode, i, col, !rev, V[e], rev, V[e], sig2);
          }
        }
        const unsigned m = __ballot_sync(FULL, uniq_e);
        const int64_t pos = written + __popc(m & ((1u << lane) - 1u));
        prev_col = __shfl_sync(FULL, col, 31);
        __syncwarp();                       // all reads of this chunk precede its writes
        if (uniq_e) { rkey[b + pos] = col; rval[b + pos] = val; }
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
emit_kernel(int64_t n, const int64_t* __restrict__ segptr, const int64_t* __restrict__ outptr,
            const uint32_t* __restrict__ rkey, const float* __restrict__ rval,
            int32_t* __restrict__ indices, float* __restrict__ data) {
  const int lane = lane_id();
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t i = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
    const int64_t b = segptr[i], o = outptr[i];
    const int64_t m = outptr[i + 1] - o;
    for (int64_t e = lane; e < m; e += 32) {
      indices[o + e] = int32_t(rkey[b + e]);
      data[o + e] = rval[b + e];
    }
  }
}

__global__ void copy_nnz_kernel(const int64_t* __restrict__ outptr, int64_t n,
                                int64_t* __restrict__ nnz) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *nnz = outptr[n];
}

struct UnionWs {
  int32_t *fwd, *indeg, *cursor, *len, *uniq, *big, *nbig;
  int64_t *segptr, *scan;
  uint32_t* rkey;
  float* rval;
};

UnionWs carve_union(Carver& c, int64_t n, int k) {
  UnionWs w;
  w.fwd = c.take<int32_t>(n);
  w.indeg = c.take<int32_t>(n);
  w.cursor = c.take<int32_t>(n);
  w.nbig = c.take<int32_t>(8);
  w.len = c.take<int32_t>(n);
  w.uniq = c.take<int32_t>(n);
  w.big = c.take<int32_t>(n);
  w.segptr = c.take<int64_t>(n + 1);
  w.scan = c.take<int64_t>(scan_scratch_elems(n));
  const size_t e2 = size_t(2) * size_t(n) * size_t(std::max(k - 1, 1));
  w.rkey = c.take<uint32_t>(e2);
  w.rval = c.take<float>(e2);
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
  Carver c(ws);
  UnionWs w = carve_union(c, n, k);
  // fwd, indeg, cursor and the big-row counter are contiguous at the start: one memset
  MSC_CUDA_TRY(cudaMemsetAsync(w.fwd, 0, reinterpret_cast<char*>(w.len) - reinterpret_cast<char*>(w.fwd), st));
  const int sms = num_sms();
  const int g1 = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), sms * 8)));
  count_kernel<<<g1, 256, 0, st>>>(mode, idx, vals, n, k, w.fwd, w.indeg);
  MSC_LAUNCH_CHECK();
  seglen_kernel<<<g1, 256, 0, st>>>(w.fwd, w.indeg, n, w.len);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl<int32_t>(w.len, n, w.segptr, w.scan, st));
  fill_kernel<<<g1, 256, 0, st>>>(mode, idx, vals, n, k, w.segptr, w.fwd, w.cursor, w.rkey,
                                  w.rval);
  MSC_LAUNCH_CHECK();
  const int g2 = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, UW), sms * 16)));
  merge_warp_kernel<<<g2, UW * 32, 0, st>>>(mode, n, w.segptr, w.rkey, w.rval, sig2, w.uniq,
                                             w.big, w.nbig);
  MSC_LAUNCH_CHECK();
  const size_t bsm = size_t(BLK_SMEM_MAX) * 8;
  MSC_CUDA_TRY(cudaFuncSetAttribute(merge_block_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, int(bsm)));
  merge_block_kernel<<<sms, 1024, bsm, st>>>(mode, w.big, w.nbig, w.segptr, w.rkey, w.rval, sig2,
                                             w.uniq);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl<int32_t>(w.uniq, n, indptr, w.scan, st));
  emit_kernel<<<g2, UW * 32, 0, st>>>(n, w.segptr, indptr, w.rkey, w.rval, indices, data);
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
