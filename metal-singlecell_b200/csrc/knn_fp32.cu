// Plain FP32 SIMT candidate kernel: the "FP32 GPU form" the tensor-core path is measured against.
//
// It computes the same v = |y|² − 2x·y ranking values as the tensor-core kernel (centred FP32
// operands, FP32 FMA accumulation) and keeps the k' smallest per row with the shared row selector,
// so the n×n matrix never leaves shared memory.  Persistent: one block per SM takes 128-row query
// tiles from a device work list and sweeps the tile's sample key by key tile.
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
                float* __restrict__ cand_thr, int cand_stride) {
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
  const int n_items = ctl->n_items;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(&ctl->item_counter, 1);
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
    if (selector) sel.reset();
    const int nkt = (w.nkeys + F_BN - 1) / F_BN;
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
    if (tid >= F_BM) load_b(0, 0);
    __syncthreads();
    // neighbour ids are packed positions here; finish() maps them to original rows
    const int self_base = w.qrow0;
    const int limit = w.key0 + w.nkeys;
    for (int kt = 0; kt < nkt; ++kt) {
      const int buf = kt & 1;
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
      } else if (kt + 1 < nkt) {
        load_b(kt + 1, buf ^ 1);
      }
      __syncthreads();
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
                  float* cand_thr, int cand_stride, cudaStream_t st) {
  (void)d;
  const size_t smem = FpSmem<KPL, CB>::bytes(dpad);
  auto kern = knn_fp32_kernel<KPL, CB>;
  MSC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(smem)));
  int grid = int(std::min<int64_t>(n_items, num_sms()));
  kern<<<std::max(grid, 1), F_THREADS, smem, st>>>(A32, sq32, dpad, items, perm, ctl, kprime,
                                                   cand_idx, cand_thr, cand_stride);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace

int launch_knn_fp32(const float* A32, const float* sq32, int d, int dpad, const WorkItem* items,
                    int64_t n_items, const int32_t* perm, Ctl* ctl, int kprime,
                    int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st) {
  if (kprime <= 32)
    return launch_fp32_t<32, 32>(A32, sq32, d, dpad, items, n_items, perm, ctl, kprime, cand_idx,
                                 cand_thr, cand_stride, st);
  if (kprime <= 64)
    return launch_fp32_t<64, 32>(A32, sq32, d, dpad, items, n_items, perm, ctl, kprime, cand_idx,
                                 cand_thr, cand_stride, st);
  set_error("kprime=%d > 64 is not supported by the candidate kernels", kprime);
  return MSC_ERR_UNSUPPORTED;
}

}  // namespace msc
