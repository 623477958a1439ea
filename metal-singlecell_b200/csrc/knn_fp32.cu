// Plain FP32 SIMT candidate kernel: the "FP32 GPU form" the tensor-core path is measured against.
//
// It computes the same v = |y|² − 2x·y ranking values as the tensor-core kernel (centred FP32
// operands, FP32 FMA accumulation) and keeps the k' smallest per row with the shared row selector,
// so the n×n matrix never leaves shared memory.  Persistent: one block per SM takes 128-row query
// tiles from a device work list and sweeps the tile's sample key by key tile.
//
// With a pruning plan (prune.cu) the same kernel runs as a near pass (every query tile against its
// own 256-key tile) and then as a pruned main pass (the near 256-key tiles and those the plan's
// mask keeps, each swept as four 64-key tiles), so that the FP32 form can be compared with the
// 16-bit tensor-core forms at the same pruning.
//
// Reference counterpart: the fp16 Gram tile + `topk_rows` kernel of metalsinglecell
// neighbors.py:114-119 (which materialises a block×n distance matrix in device memory).
#include "kernels.cuh"
#include "msc_select.cuh"

namespace msc {

namespace {

constexpr int F_BM = 128;     // query rows per tile
constexpr int F_BN = 64;      // keys per tile
constexpr int F_THREADS = 256;
constexpr int V_STRIDE = F_BN + 4;

constexpr int F_BIG = 256;    // key tiles of the pruning plan
constexpr int F_SUB = F_BIG / F_BN;

// The 64-key tiles of one work item: every tile in order (plain form), or the plan's 256-key
// tiles — the near ones first (the query tile's own, then alternately right and left, two each
// side), then the far ones whose mask bit is set — each split into its 64-key tiles; the near
// pass takes the own 256-key tile only.
struct FpWalk {
  int nkeys, nsmall, nbig, diag, lo, hi, np, j;
  const uint32_t* mask;
  int words, w;
  uint32_t cur;
  int big, sub;
  bool plain;
  __device__ __forceinline__ void init(const WorkItem& item, const uint32_t* m, int nw, bool near) {
    nkeys = item.nkeys;
    nsmall = (nkeys + F_BN - 1) / F_BN;
    plain = m == nullptr && !near;
    nbig = (nkeys + F_BIG - 1) / F_BIG;
    diag = (item.qrow0 - item.key0) / F_BIG;
    lo = max(0, diag - 2);
    hi = min(nbig - 1, diag + 2);
    np = near ? 1 : hi - lo + 1;
    j = 0;
    mask = near ? nullptr : m;
    words = nw;
    w = 0;
    cur = mask ? mask[0] : 0u;
    big = -1;
    sub = F_SUB;
  }
  __device__ __forceinline__ int near_at(int t) const {
    const int left = diag - lo, right = hi - diag, m = min(left, right);
    if (t == 0) return diag;
    if (t <= 2 * m) return (t & 1) ? diag + ((t + 1) >> 1) : diag - (t >> 1);
    return right > left ? diag + (t - m) : diag - (t - m);
  }
  __device__ __forceinline__ int next_big() {
    if (j < np) return near_at(j++);
    if (!mask) return -1;
    for (;;) {
      while (cur == 0u) {
        if (++w >= words) return -1;
        cur = mask[w];
      }
      const int b = __ffs(cur) - 1;
      cur &= cur - 1u;
      const int bt = w * 32 + b;
      if (bt < nbig) return bt;
    }
  }
  // the next 64-key tile, or -1
  __device__ __forceinline__ int next() {
    if (plain) return j < nsmall ? j++ : -1;
    for (;;) {
      if (big >= 0 && sub < F_SUB) {
        const int kt = big * F_SUB + sub++;
        if (kt < nsmall) return kt;
        continue;
      }
      big = next_big();
      sub = 0;
      if (big < 0) return -1;
    }
  }
};

template <int KPL, int CB>
struct FpSmem {
  static size_t bytes(int dpad) {
    size_t a = size_t(dpad) * F_BM * 4;          // As[t][row]
    size_t b = 2 * size_t(dpad) * F_BN * 4;      // Bs[2][t][key]
    size_t sq = 2 * size_t(F_BN) * 4;            // key norms
    size_t v = size_t(F_BM) * V_STRIDE * 4;      // V[row][key]
    return a + b + sq + v + RowSelect<KPL, CB, F_BM>::smem_bytes() + 64;
  }
};

template <int KPL, int CB>
__global__ void __launch_bounds__(F_THREADS, 1)
knn_fp32_kernel(const float* __restrict__ A32, const float* __restrict__ sq32, int dpad,
                const WorkItem* __restrict__ items, const int32_t* __restrict__ perm,
                Ctl* __restrict__ ctl, int kprime, int32_t* __restrict__ cand_idx,
                float* __restrict__ cand_thr, int cand_stride, const uint32_t* __restrict__ mask,
                int words, int near_only, const float* __restrict__ seed,
                int32_t* __restrict__ counter, int n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* As = reinterpret_cast<float*>(smem_raw);
  float* Bs = As + size_t(dpad) * F_BM;
  float* Sq = Bs + 2 * size_t(dpad) * F_BN;
  float* V = Sq + 2 * F_BN;
  void* sel_mem = V + size_t(F_BM) * V_STRIDE;
  __shared__ int s_item;

  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;        // GEMM: rows 8ty.., keys 4tx..
  const bool selector = tid < F_BM;              // warps 0-3 own one row each
  RowSelect<KPL, CB, F_BM> sel;
  sel.bind(sel_mem, selector ? tid : 0, kprime);
  for (;;) {
    if (tid == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= n_items) break;
    const WorkItem w = items[it];
    // query tile, transposed into As[t][row]: a thread reads 4 consecutive dimensions of one row
    // (float4) and writes them to 4 consecutive t-rows; neighbouring threads take neighbouring
    // rows, so the shared-memory stores hit distinct banks
    for (int e = tid; e < F_BM * (dpad >> 2); e += F_THREADS) {
      const int r = e % F_BM, tq = e / F_BM;
      const float4 a = *reinterpret_cast<const float4*>(A32 + (int64_t(w.qrow0) + r) * dpad + 4 * tq);
      As[(4 * tq + 0) * F_BM + r] = a.x;
      As[(4 * tq + 1) * F_BM + r] = a.y;
      As[(4 * tq + 2) * F_BM + r] = a.z;
      As[(4 * tq + 3) * F_BM + r] = a.w;
    }
    if (selector) {
      sel.reset();
      if (seed && tid < w.nq) sel.set_seed(seed[int64_t(w.qrow0) + tid]);
    }
    FpWalk walk;
    walk.init(w, mask ? mask + int64_t(it) * words : nullptr, words, near_only != 0);
    // first key tile
    auto load_b = [&](int kt, int buf) {
      const int64_t k0 = int64_t(w.key0) + int64_t(kt) * F_BN;
      float* B = Bs + size_t(buf) * dpad * F_BN;
      for (int e = (tid & 127); e < F_BN * (dpad >> 2); e += 128) {
        const int kr = e % F_BN, tq = e / F_BN;
        const float4 b = *reinterpret_cast<const float4*>(A32 + (k0 + kr) * dpad + 4 * tq);
        B[(4 * tq + 0) * F_BN + kr] = b.x;
        B[(4 * tq + 1) * F_BN + kr] = b.y;
        B[(4 * tq + 2) * F_BN + kr] = b.z;
        B[(4 * tq + 3) * F_BN + kr] = b.w;
      }
      if ((tid & 127) < F_BN) Sq[buf * F_BN + (tid & 127)] = sq32[k0 + (tid & 127)];
    };
    int kt = walk.next();
    if (tid >= F_BM && kt >= 0) load_b(kt, 0);
    __syncthreads();
    // neighbour ids are packed positions here; finish() maps them to original rows
    const int self_base = w.qrow0;
    const int limit = w.key0 + w.nkeys;
    for (int step = 0; kt >= 0; ++step) {
      const int nxt = walk.next();                 // every thread walks the same sequence
      const int buf = step & 1;
      const float* B = Bs + size_t(buf) * dpad * F_BN;
      float acc[8][4];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
      for (int t = 0; t < dpad; ++t) {
        const float4 a0 = *reinterpret_cast<const float4*>(As + t * F_BM + 8 * ty);
        const float4 a1 = *reinterpret_cast<const float4*>(As + t * F_BM + 8 * ty + 4);
        const float4 b = *reinterpret_cast<const float4*>(B + t * F_BN + 4 * tx);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        const float bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], bb[j], acc[i][j]);
      }
      const float4 sq4 = *reinterpret_cast<const float4*>(Sq + buf * F_BN + 4 * tx);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        float4 o;
        o.x = fmaf(-2.f, acc[i][0], sq4.x);
        o.y = fmaf(-2.f, acc[i][1], sq4.y);
        o.z = fmaf(-2.f, acc[i][2], sq4.z);
        o.w = fmaf(-2.f, acc[i][3], sq4.w);
        *reinterpret_cast<float4*>(V + (8 * ty + i) * V_STRIDE + 4 * tx) = o;
      }
      __syncthreads();
      if (selector) {
        const int col0 = w.key0 + kt * F_BN;
#pragma unroll
        for (int h = 0; h < F_BN; h += 32) {
          float v[32];
#pragma unroll
          for (int e = 0; e < 32; e += 4) {
            const float4 q = *reinterpret_cast<const float4*>(V + tid * V_STRIDE + h + e);
            v[e] = q.x; v[e + 1] = q.y; v[e + 2] = q.z; v[e + 3] = q.w;
          }
          sel.push32(v, col0 + h, self_base + tid, limit);
        }
      } else if (nxt >= 0) {
        load_b(nxt, buf ^ 1);
      }
      __syncthreads();
      kt = nxt;
    }
    if (selector) {
      const int wrow0 = tid & ~31;
      const int nvalid = min(32, w.nq - wrow0);
      if (nvalid > 0)
        sel.finish(cand_idx, cand_thr, cand_stride, perm, nullptr, int64_t(w.qrow0) + wrow0, nvalid,
                   kprime);
      else
        sel.flush();
    }
    __syncthreads();
  }
}

template <int KPL, int CB>
int launch_fp32_t(const float* A32, const float* sq32, int d, int dpad, const WorkItem* items,
                  int64_t n_items, const int32_t* perm, Ctl* ctl, int kprime, int32_t* cand_idx,
                  float* cand_thr, int cand_stride, cudaStream_t st, const FpPrune& pr) {
  (void)d;
  const size_t smem = FpSmem<KPL, CB>::bytes(dpad);
  auto kern = knn_fp32_kernel<KPL, CB>;
  MSC_CUDA_TRY(raise_smem_cap(kern, smem));
  int grid = int(std::min<int64_t>(n_items, num_sms()));
  MSC_CUDA_TRY(cudaMemsetAsync(pr.counter, 0, sizeof(int32_t), st));
  kern<<<std::max(grid, 1), F_THREADS, smem, st>>>(A32, sq32, dpad, items, perm, ctl, kprime,
                                                   cand_idx, cand_thr, cand_stride, pr.mask,
                                                   pr.words, pr.near_only ? 1 : 0, pr.seed,
                                                   pr.counter, int(n_items));
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace

int launch_knn_fp32(const float* A32, const float* sq32, int d, int dpad, const WorkItem* items,
                    int64_t n_items, const int32_t* perm, Ctl* ctl, int kprime,
                    int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st,
                    const FpPrune* prune) {
  FpPrune pr{};
  if (prune) pr = *prune;
  if (!pr.counter) pr.counter = &ctl->item_counter;
  if (kprime <= 32)
    return launch_fp32_t<32, 32>(A32, sq32, d, dpad, items, n_items, perm, ctl, kprime, cand_idx,
                                 cand_thr, cand_stride, st, pr);
  if (kprime <= 64)
    return launch_fp32_t<64, 32>(A32, sq32, d, dpad, items, n_items, perm, ctl, kprime, cand_idx,
                                 cand_thr, cand_stride, st, pr);
  set_error("kprime=%d > 64 is not supported by the candidate kernels", kprime);
  return MSC_ERR_UNSUPPORTED;
}

}  // namespace msc
