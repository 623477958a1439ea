// Locality order of the cells: a deterministic bisection tree built on the GPU.
//
// The candidate kernels filter every key against the row's running k'-th value.  With cells in
// arbitrary order a row's list keeps improving through the whole scan (about k'·ln(n/k')
// insertions per row), and a 32-row warp takes the slow path whenever any of its rows does.
// Scanning first the keys that are near the query tile's rows brings every threshold close to its
// final value within a few key tiles.  This file computes that order; the packed operands are
// laid out in it, and each query tile scans its own key tile first and then outwards.  The
// neighbour graph does not depend on the order (candidates are re-ranked exactly and certified).
//
// The tree: every node (a range of packed positions inside one sample) larger than LEAF rows is
// split in two around two far-apart cells — a = the cell farthest from the node's first cell,
// b = the cell farthest from a — each cell going to the side of the nearer of the two (ties to
// a's side); a degenerate split (all on one side) halves the range instead.  Farthest-point
// choices break distance ties by the lower position (64-bit atomicMax of distance bits and
// inverted position), and the partition is stable, so the order is a pure function of the input.
// A fixed number of levels runs without host synchronisation (graph-capturable); nodes at or
// below LEAF rows are left as they are.
#include "kernels.cuh"

namespace msc {

namespace {

constexpr int OR_T = 256;

__device__ __forceinline__ float row_d2(const float* __restrict__ X, int d, int64_t a, int64_t b) {
  const float* x = X + a * d;
  const float* y = X + b * d;
  float acc = 0.f;
  for (int t = 0; t < d; ++t) {
    const float df = x[t] - y[t];
    acc = fmaf(df, df, acc);
  }
  return acc;
}

__device__ __forceinline__ unsigned long long far_key(float d2, int64_t p) {
  // d2 >= 0 (or NaN): its bits order like its value; the lower position wins a tie
  return (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) |
         (0xFFFFFFFFull - static_cast<unsigned long long>(p));
}
__device__ __forceinline__ int64_t far_pos(unsigned long long key) {
  return int64_t(0xFFFFFFFFull - (key & 0xFFFFFFFFull));
}

// identity order inside each sample; node = the sample's valid rows, padding rows are size 0
__global__ void order_init_kernel(const SegDesc* __restrict__ seg, int nseg, int64_t npacked,
                                  int32_t* __restrict__ perm, int32_t* __restrict__ ns,
                                  int32_t* __restrict__ ne) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int s = find_seg(seg, nseg, p);
    const int64_t j = p - seg[s].poff;
    if (j < seg[s].n) {
      perm[p] = int32_t(seg[s].off + j);
      ns[p] = int32_t(seg[s].poff);
      ne[p] = int32_t(seg[s].poff + seg[s].n);
    } else {
      perm[p] = -1;
      ns[p] = int32_t(p);
      ne[p] = int32_t(p);
    }
  }
}

__global__ void far_a_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
                             const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
                             const int32_t* __restrict__ ne, unsigned long long* __restrict__ best) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int s = ns[p], e = ne[p];
    if (e - s <= leaf) continue;
    atomicMax(&best[s], far_key(row_d2(X, d, perm[p], perm[s]), p));
  }
}

__global__ void far_b_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
                             const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
                             const int32_t* __restrict__ ne, const unsigned long long* __restrict__ best_a,
                             float* __restrict__ da, unsigned long long* __restrict__ best_b) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int s = ns[p], e = ne[p];
    if (e - s <= leaf) continue;
    const float v = row_d2(X, d, perm[p], perm[far_pos(best_a[s])]);
    da[p] = v;
    atomicMax(&best_b[s], far_key(v, p));
  }
}

__global__ void side_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
                            const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
                            const int32_t* __restrict__ ne, const float* __restrict__ da,
                            const unsigned long long* __restrict__ best_b,
                            int32_t* __restrict__ side) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int s = ns[p], e = ne[p];
    int v = 0;
    if (e - s > leaf) {
      const float db = row_d2(X, d, perm[p], perm[far_pos(best_b[s])]);
      v = da[p] > db ? 1 : 0;                    // nearer to b: second half
    }
    side[p] = v;
  }
}

__global__ void scatter_kernel(int64_t npacked, int leaf, const int32_t* __restrict__ perm,
                               const int32_t* __restrict__ ns, const int32_t* __restrict__ ne,
                               const int32_t* __restrict__ side, const int64_t* __restrict__ S,
                               int32_t* __restrict__ perm2, int32_t* __restrict__ ns2,
                               int32_t* __restrict__ ne2) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x) {
    const int s = ns[p], e = ne[p];
    int64_t pos = p;
    int cs = s, ce = e;
    if (e - s > leaf) {
      const int64_t c1 = S[e] - S[s];
      const int64_t c0 = int64_t(e - s) - c1;
      if (c0 == 0 || c1 == 0) {
        const int mid = s + (e - s) / 2;         // degenerate: halve the range
        if (p < mid) ce = mid; else cs = mid;
      } else {
        const int64_t r1 = S[p] - S[s];          // side-1 cells before p in the node
        if (side[p]) {
          pos = s + c0 + r1;
          cs = int(s + c0);
        } else {
          pos = s + (p - s) - r1;
          ce = int(s + c0);
        }
      }
    }
    perm2[pos] = perm[p];
    ns2[pos] = cs;
    ne2[pos] = ce;
  }
}

}  // namespace

size_t order_workspace_bytes(int64_t npacked) {
  Carver c(nullptr);
  c.take<int32_t>(npacked);                       // second permutation
  c.take<int32_t>(npacked);                       // node start, node end (two copies each)
  c.take<int32_t>(npacked);
  c.take<int32_t>(npacked);
  c.take<int32_t>(npacked);
  c.take<unsigned long long>(npacked);            // farthest cells per node
  c.take<unsigned long long>(npacked);
  c.take<float>(npacked);                         // distance to a
  c.take<int32_t>(npacked);                       // side
  c.take<int64_t>(npacked + 1);                   // scan of side
  c.take<int64_t>(scan_i32_scratch_elems(npacked));
  return c.bytes();
}

int launch_order(const float* X, int d, const SegDesc* seg, int nseg, int64_t npacked, int levels,
                 int leaf, int32_t* perm, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (ws_bytes < order_workspace_bytes(npacked)) {
    set_error("order: workspace %zu < %zu bytes", ws_bytes, order_workspace_bytes(npacked));
    return MSC_ERR_WORKSPACE;
  }
  Carver c(ws);
  int32_t* perm2 = c.take<int32_t>(npacked);
  int32_t* nsA = c.take<int32_t>(npacked);
  int32_t* neA = c.take<int32_t>(npacked);
  int32_t* nsB = c.take<int32_t>(npacked);
  int32_t* neB = c.take<int32_t>(npacked);
  unsigned long long* best_a = c.take<unsigned long long>(npacked);
  unsigned long long* best_b = c.take<unsigned long long>(npacked);
  float* da = c.take<float>(npacked);
  int32_t* side = c.take<int32_t>(npacked);
  int64_t* S = c.take<int64_t>(npacked + 1);
  int64_t* scratch = c.take<int64_t>(scan_i32_scratch_elems(npacked));
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(npacked, OR_T),
                                                              int64_t(num_sms()) * 8)));
  order_init_kernel<<<grid, OR_T, 0, st>>>(seg, nseg, npacked, perm, nsA, neA);
  MSC_LAUNCH_CHECK();
  int32_t *pc = perm, *pn = perm2, *sc = nsA, *ec = neA, *sn = nsB, *en = neB;
  for (int l = 0; l < levels; ++l) {
    MSC_CUDA_TRY(cudaMemsetAsync(best_a, 0, sizeof(unsigned long long) * npacked, st));
    MSC_CUDA_TRY(cudaMemsetAsync(best_b, 0, sizeof(unsigned long long) * npacked, st));
    far_a_kernel<<<grid, OR_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, best_a);
    MSC_LAUNCH_CHECK();
    far_b_kernel<<<grid, OR_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, best_a, da, best_b);
    MSC_LAUNCH_CHECK();
    side_kernel<<<grid, OR_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, da, best_b, side);
    MSC_LAUNCH_CHECK();
    MSC_TRY(scan_excl_i32(side, npacked, S, scratch, st));
    scatter_kernel<<<grid, OR_T, 0, st>>>(npacked, leaf, pc, sc, ec, side, S, pn, sn, en);
    MSC_LAUNCH_CHECK();
    std::swap(pc, pn);
    std::swap(sc, sn);
    std::swap(ec, en);
  }
  if (pc != perm)
    MSC_CUDA_TRY(cudaMemcpyAsync(perm, pc, sizeof(int32_t) * npacked, cudaMemcpyDeviceToDevice, st));
  return MSC_OK;
}

}  // namespace msc
