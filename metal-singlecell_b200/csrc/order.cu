// Locality order of the cells: a bisection tree built on the GPU.
//
// The candidate kernels filter every key against the row's running k'-th value.  With cells in
// arbitrary order a row's list keeps improving through the whole scan (about k'·ln(n/k')
// insertions per row), and a 32-row warp takes the slow path whenever any of its rows does.
// Scanning first the keys that are near the query tile's rows brings every threshold close to its
// final value within a few key tiles.  The order also decides how tight the bounding balls of the
// tiles are, which is what lets whole tiles of keys be skipped.  This file computes that order;
// the packed operands are laid out in it.  The neighbour graph does not depend on the order
// (candidates are re-ranked exactly and certified).
//
// The tree: every node (a range of packed positions inside one sample) larger than LEAF rows is
// split in two by 2-means.  It starts from two far-apart cells — a = the cell farthest from the
// node's first cell, b = the cell farthest from a (distance ties to the lower position) — assigns
// every cell to the nearer of the two (ties to a's side), then moves a and b to the means of their
// sides; on the first LLOYD_LEVELS levels the means take LLOYD_STEPS more 2-means steps over a
// sample of the node's cells; then every cell is assigned to the nearer mean.  The assignment to
// the means follows the gaps between clusters instead of the bisector of two extreme (often
// outlying) cells; the extra steps matter at the top of the tree, where a node holds many
// clusters and the bisector of the first means cuts through some of them (measured at 1.3M × 50,
// 200 clusters: far key tiles kept by the pruning plan 3.42 M → 2.63 M, main scan 44.8 → 40.9 ms,
// for 0.6 ms more ordering).  The caller may give the rows projected onto a few random directions
// for the lower levels (Xp, from level proj_from on): those levels split inside one cluster, and
// each of their passes then reads a fraction of a row.
// A degenerate split (all on one side) halves the range instead; the partition is stable.  The
// side means are summed with floating-point atomics, so a cell almost equidistant from both means
// may fall on either side from run to run; the graph is the same either way.  A fixed number of
// levels runs without host synchronisation (graph-capturable); nodes at or below LEAF rows are
// left as they are and are the leaves of the tree.
#include <cstdlib>

#include "kernels.cuh"

namespace msc {

namespace {

constexpr int OR_T = 256;
// More 2-means steps on the first LLOYD_LEVELS levels (lloyd_node_kernel), on up to
// LLOYD_SAMPLES_MAX rows of every split node (MSC_B200_LLOYD_LEVELS / MSC_B200_LLOYD_STEPS override
// the level count and the steps: tuning).  With one step, a mixture of well-separated clusters is
// cut into many fragments whose pieces share leaves and tiles; their bounding balls then span
// clusters and the pruning plan keeps those tiles for almost every query tile.
constexpr int LLOYD_LEVELS = 8;
constexpr int LLOYD_STEPS = 5;
constexpr int LLOYD_SAMPLES_MAX = 512;
constexpr size_t LLOYD_SMEM_MAX = 200 * 1024;
// ... and only while the largest sample's nodes hold at least this many cells: smaller nodes are
// parts of one or a few clusters, and the launches would cost a small graph more than they save
constexpr int64_t LLOYD_MIN_NODE = 8192;

// The row passes of a level (far_a, far_b, side, reassign, side_sum) run ROW_T-thread blocks:
// with their row tiles, ten to eleven blocks fit on an SM.
constexpr int ROW_T = 128;
constexpr int ROW_W = ROW_T / 32;

// One warp's 32 rows, 32 dimensions at a time: row r's dimensions c..c+31 in tile[r][0..31]
// (dimensions at or past d, and rows < 0, hold zeros).  Lanes load a row together (one coalesced
// line per row and chunk), then each lane reads its own row back from the tile in pairs: a stride
// of 34 floats keeps the rows 8-byte aligned, and the 16 lanes of each half-warp phase of a
// 64-bit read then cover the 32 banks once.  A thread reading its row alone, one float per load,
// keeps 32 rows' lines live per warp and thrashes L1.
constexpr int TILE_S = 34;
using RowTile = float[32][TILE_S];
// per warp: one or two rows of reference values (the far cell, or the two side means),
// zero-padded to whole 32-dimension chunks
using RefRows = float[2][MSC_MAX_D];

// stage dimensions c..c+31 of the lanes' rows (row < 0: zeros); sixteen loads are issued before
// their stores so that a warp keeps sixteen lines in flight
__device__ __forceinline__ void stage_rows(const float* __restrict__ X, int d, int c, int32_t row,
                                           RowTile& tile) {
  const int t = c + lane_id();
#pragma unroll
  for (int r0 = 0; r0 < 32; r0 += 16) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int32_t rr = __shfl_sync(FULL, row, r0 + u);
      v[u] = (rr >= 0 && t < d) ? X[int64_t(rr) * d + t] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) tile[r0 + u][lane_id()] = v[u];
  }
  __syncwarp();
}

// Σ_j (tile[lane][j] − ref[c + j])² over the chunk's 32 dimensions, added to acc in order
__device__ __forceinline__ float chunk_d2(const RowTile& tile, const float* ref, int c, float acc) {
#pragma unroll
  for (int j = 0; j < 32; j += 2) {
    const float2 x = *reinterpret_cast<const float2*>(&tile[lane_id()][j]);
    const float2 y = *reinterpret_cast<const float2*>(&ref[c + j]);
    const float dx = x.x - y.x, dy = x.y - y.y;
    acc = fmaf(dx, dx, acc);
    acc = fmaf(dy, dy, acc);
  }
  return acc;
}

// squared distance between the lane's row and row `other`, summed over t = 0..d-1 in order
// (the same sum as a plain loop over the two rows: the padding adds exact zeros); lanes with
// row < 0 return 0.  When the warp's active lanes share `other` (a warp inside one node: all but
// the warps that straddle a node boundary) that row is staged once in ref[0]; otherwise every
// lane reads its own through L1.
__device__ __forceinline__ float warp_row_d2(const float* __restrict__ X, int d, int32_t row,
                                             int64_t other, RowTile& tile, RefRows& ref) {
  const unsigned act = __ballot_sync(FULL, row >= 0);
  float acc = 0.f;
  if (act == 0) return acc;
  const int64_t o0 = __shfl_sync(FULL, other, __ffs(act) - 1);
  const bool uni = __all_sync(FULL, row < 0 || other == o0);
  if (uni) {
    for (int t = lane_id(); t < MSC_MAX_D; t += 32) ref[0][t] = t < d ? X[o0 * d + t] : 0.f;
    __syncwarp();
  }
  for (int c = 0; c < d; c += 32) {
    stage_rows(X, d, c, row, tile);
    if (row >= 0) {
      if (uni) {
        acc = chunk_d2(tile, ref[0], c, acc);
      } else {
        const float* y = X + other * d + c;
        const int tn = min(32, d - c);
        for (int j = 0; j < tn; ++j) {
          const float df = tile[lane_id()][j] - y[j];
          acc = fmaf(df, df, acc);
        }
      }
    }
    __syncwarp();
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

// atomicMax of key into best[s]; the lanes of a warp that share node s combine first (positions
// are contiguous, so a warp almost always lies inside one node and issues a single atomic)
__device__ __forceinline__ void warp_far_max(unsigned long long* best, int s, bool active,
                                             unsigned long long key) {
  const int s0 = __shfl_sync(FULL, s, 0);
  if (__all_sync(FULL, active && s == s0)) {
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_xor_sync(FULL, key, o);
      key = other > key ? other : key;
    }
    if (lane_id() == 0) atomicMax(&best[s0], key);
  } else if (active) {
    atomicMax(&best[s], key);
  }
}

// The loops below keep the 32 lanes of a warp on 32 consecutive positions (warp-uniform trip
// counts) so that warp_far_max can combine them and warp_row_d2 can stage their rows.
__global__ void __launch_bounds__(ROW_T)
far_a_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
             const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
             const int32_t* __restrict__ ne, unsigned long long* __restrict__ best) {
  __shared__ __align__(16) RowTile tiles[ROW_W];
  __shared__ __align__(16) RefRows refs[ROW_W];
  RowTile& tile = tiles[warp_id()];
  RefRows& ref = refs[warp_id()];
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t b = blockIdx.x * int64_t(blockDim.x) + (threadIdx.x & ~31); b < npacked;
       b += stride) {
    const int64_t p = b + lane_id();
    int s = 0, e = 0;
    if (p < npacked) { s = ns[p]; e = ne[p]; }
    const bool active = p < npacked && e - s > leaf;
    const int32_t row = active ? perm[p] : -1;
    const float v = warp_row_d2(X, d, row, active ? perm[s] : 0, tile, ref);
    warp_far_max(best, s, active, active ? far_key(v, p) : 0ull);
  }
}

__global__ void __launch_bounds__(ROW_T)
far_b_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
             const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
             const int32_t* __restrict__ ne, const unsigned long long* __restrict__ best_a,
             float* __restrict__ da, unsigned long long* __restrict__ best_b) {
  __shared__ __align__(16) RowTile tiles[ROW_W];
  __shared__ __align__(16) RefRows refs[ROW_W];
  RowTile& tile = tiles[warp_id()];
  RefRows& ref = refs[warp_id()];
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t b = blockIdx.x * int64_t(blockDim.x) + (threadIdx.x & ~31); b < npacked;
       b += stride) {
    const int64_t p = b + lane_id();
    int s = 0, e = 0;
    if (p < npacked) { s = ns[p]; e = ne[p]; }
    const bool active = p < npacked && e - s > leaf;
    const int32_t row = active ? perm[p] : -1;
    const float v = warp_row_d2(X, d, row, active ? perm[far_pos(best_a[s])] : 0, tile, ref);
    if (active) da[p] = v;
    warp_far_max(best_b, s, active, active ? far_key(v, p) : 0ull);
  }
}

__global__ void __launch_bounds__(ROW_T)
side_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
            const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
            const int32_t* __restrict__ ne, const float* __restrict__ da,
            const unsigned long long* __restrict__ best_b, int32_t* __restrict__ side) {
  __shared__ __align__(16) RowTile tiles[ROW_W];
  __shared__ __align__(16) RefRows refs[ROW_W];
  RowTile& tile = tiles[warp_id()];
  RefRows& ref = refs[warp_id()];
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t b = blockIdx.x * int64_t(blockDim.x) + (threadIdx.x & ~31); b < npacked;
       b += stride) {
    const int64_t p = b + lane_id();
    int s = 0, e = 0;
    if (p < npacked) { s = ns[p]; e = ne[p]; }
    const bool active = p < npacked && e - s > leaf;
    const int32_t row = active ? perm[p] : -1;
    const float db = warp_row_d2(X, d, row, active ? perm[far_pos(best_b[s])] : 0, tile, ref);
    if (p < npacked) side[p] = active && da[p] > db ? 1 : 0;   // nearer to b: second half
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

// first position of every node that is split at this level
__global__ void split_start_kernel(int64_t npacked, int leaf, const int32_t* __restrict__ ns,
                                   const int32_t* __restrict__ ne, int32_t* __restrict__ flag) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x)
    flag[p] = (ns[p] == p && ne[p] - ns[p] > leaf) ? 1 : 0;
}

// Per split node and side: Σ x and the count.  Each warp takes a contiguous range of 32-position
// tasks (consecutive tasks mostly lie in one node); lane t owns dimensions t, t+32, ... (PER of
// them: d <= 32·PER) and keeps FP64 sums for the node it is in, handed on with one atomic per
// (node, side, dimension) when the node changes.  A task whose active positions share one node
// stages its 32 rows chunk by chunk and adds the columns from shared memory (in FP32 over the
// task's rows, then into the FP64 sums); a task that straddles nodes adds row by row from global
// memory.  At the end the warps of a block that finish in the same node combine in shared memory,
// so at the top levels, where every warp is in one of a few nodes, a block issues one set of
// atomics.  acc layout per node: [2][d] sums, then [2] counts.
constexpr int SUM_SLOT = 2 * MSC_MAX_D + 2;
template <int PER>
__global__ void __launch_bounds__(ROW_T)
side_sum_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
                const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
                const int32_t* __restrict__ ne, const int64_t* __restrict__ S,
                const int32_t* __restrict__ side, double* __restrict__ acc) {
  __shared__ __align__(16) RowTile tiles[ROW_W];
  __shared__ double part[ROW_W][SUM_SLOT];
  __shared__ int64_t part_node[ROW_W];
  RowTile& tile = tiles[warp_id()];
  const int lane = lane_id(), wib = warp_id();
  const int64_t ntask = (npacked + 31) / 32;
  const int64_t nwarp = int64_t(gridDim.x) * ROW_W, gw = int64_t(blockIdx.x) * ROW_W + wib;
  const int64_t t0 = ntask * gw / nwarp, t1 = ntask * (gw + 1) / nwarp;
  double s0[PER], s1[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) { s0[j] = 0.0; s1[j] = 0.0; }
  double c0 = 0, c1 = 0;
  int64_t cur = -1;                          // node id being accumulated
  auto flush = [&]() {
    if (cur < 0) return;
    double* a = acc + cur * (2 * d + 2);
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int t = lane + 32 * j;
      if (t < d) {
        if (s0[j] != 0.0) atomicAdd(&a[t], s0[j]);
        if (s1[j] != 0.0) atomicAdd(&a[d + t], s1[j]);
      }
      s0[j] = 0; s1[j] = 0;
    }
    if (lane == 0) {
      if (c0 != 0) atomicAdd(&a[2 * d], c0);
      if (c1 != 0) atomicAdd(&a[2 * d + 1], c1);
    }
    c0 = 0; c1 = 0;
  };
  for (int64_t tk = t0; tk < t1; ++tk) {     // warp-uniform
    const int64_t p = tk * 32 + lane;
    int64_t id = -1;
    int32_t row = -1;
    int sd = 0;
    if (p < npacked) {
      const int st = ns[p];
      if (ne[p] - st > leaf) {
        id = S[st];
        row = perm[p];
        sd = side[p];
      }
    }
    const unsigned act = __ballot_sync(FULL, id >= 0);
    if (act == 0) continue;
    const int64_t id0 = __shfl_sync(FULL, id, __ffs(act) - 1);
    if (__all_sync(FULL, id < 0 || id == id0)) {
      if (id0 != cur) { flush(); cur = id0; }
      const unsigned m1 = __ballot_sync(FULL, id >= 0 && sd != 0);
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        if (32 * j < d) {                    // warp-uniform
          stage_rows(X, d, 32 * j, row, tile);
          float f0 = 0.f, f1 = 0.f;
#pragma unroll
          for (int r = 0; r < 32; ++r) {
            const float v = tile[r][lane];
            if ((m1 >> r) & 1u) f1 += v; else f0 += v;
          }
          s0[j] += f0;
          s1[j] += f1;
          __syncwarp();
        }
      }
      c1 += __popc(m1);
      c0 += __popc(act & ~m1);
    } else {
      for (int r = 0; r < 32; ++r) {
        const int64_t idr = __shfl_sync(FULL, id, r);
        if (idr < 0) continue;               // warp-uniform
        const int32_t rw = __shfl_sync(FULL, row, r);
        const bool one = __shfl_sync(FULL, sd, r) != 0;
        if (idr != cur) { flush(); cur = idr; }
        const float* x = X + int64_t(rw) * d;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
          const int t = lane + 32 * j;
          if (t < d) {
            if (one) s1[j] += x[t]; else s0[j] += x[t];
          }
        }
        if (one) c1 += 1.0; else c0 += 1.0;
      }
    }
  }
  // the last node's sums go to the block
  if (cur >= 0) {
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int t = lane + 32 * j;
      if (t < d) { part[wib][t] = s0[j]; part[wib][d + t] = s1[j]; }
    }
    if (lane == 0) { part[wib][2 * d] = c0; part[wib][2 * d + 1] = c1; }
  }
  if (lane == 0) part_node[wib] = cur;
  __syncthreads();
  if (wib == 0) {
    // consecutive warps in the same node: one atomic per value per node
    int w0 = 0;
    while (w0 < ROW_W) {
      const int64_t nd = part_node[w0];
      int w1 = w0 + 1;
      while (w1 < ROW_W && part_node[w1] == nd) ++w1;
      if (nd >= 0) {
        double* a = acc + nd * (2 * d + 2);
        for (int t = lane; t < 2 * d + 2; t += 32) {
          double v = 0.0;
          for (int w = w0; w < w1; ++w) v += part[w][t];
          if (v != 0.0) atomicAdd(&a[t], v);
        }
      }
      w0 = w1;
    }
  }
}

// The first assignment and the side sums in one pass over the rows (d <= 32·PER, PER <= 2): a
// warp stages a task's 32 rows whole (every 32-dimension chunk), takes each row's distance to b
// (the same sum as warp_row_d2), writes the row's side (nearer to b: 1; as side_kernel), and adds
// the columns of each side's rows from the same tiles.  Task ranges, node hand-off and the block
// combine are those of side_sum_kernel.
template <int PER>
__global__ void __launch_bounds__(ROW_T)
side_fused_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
                  const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
                  const int32_t* __restrict__ ne, const int64_t* __restrict__ S,
                  const float* __restrict__ da, const unsigned long long* __restrict__ best_b,
                  int32_t* __restrict__ side, double* __restrict__ acc) {
  constexpr int SLOT = 2 * 32 * PER + 2;
  __shared__ __align__(16) RowTile tiles[ROW_W][PER];
  __shared__ __align__(16) float refs[ROW_W][32 * PER];
  __shared__ double part[ROW_W][SLOT];
  __shared__ int64_t part_node[ROW_W];
  const int lane = lane_id(), wib = warp_id();
  float* ref = refs[wib];
  const int64_t ntask = (npacked + 31) / 32;
  const int64_t nwarp = int64_t(gridDim.x) * ROW_W, gw = int64_t(blockIdx.x) * ROW_W + wib;
  const int64_t t0 = ntask * gw / nwarp, t1 = ntask * (gw + 1) / nwarp;
  double s0[PER], s1[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) { s0[j] = 0.0; s1[j] = 0.0; }
  double c0 = 0, c1 = 0;
  int64_t cur = -1;                          // node id being accumulated
  auto flush = [&]() {
    if (cur < 0) return;
    double* a = acc + cur * (2 * d + 2);
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int t = lane + 32 * j;
      if (t < d) {
        if (s0[j] != 0.0) atomicAdd(&a[t], s0[j]);
        if (s1[j] != 0.0) atomicAdd(&a[d + t], s1[j]);
      }
      s0[j] = 0; s1[j] = 0;
    }
    if (lane == 0) {
      if (c0 != 0) atomicAdd(&a[2 * d], c0);
      if (c1 != 0) atomicAdd(&a[2 * d + 1], c1);
    }
    c0 = 0; c1 = 0;
  };
  for (int64_t tk = t0; tk < t1; ++tk) {     // warp-uniform
    const int64_t p = tk * 32 + lane;
    int64_t id = -1, other = 0;
    int32_t row = -1;
    if (p < npacked) {
      const int st = ns[p];
      if (ne[p] - st > leaf) {
        id = S[st];
        row = perm[p];
        other = perm[far_pos(best_b[st])];
      }
    }
    const unsigned act = __ballot_sync(FULL, id >= 0);
    if (act == 0) {
      if (p < npacked) side[p] = 0;
      continue;
    }
    const int src = __ffs(act) - 1;
    const int64_t id0 = __shfl_sync(FULL, id, src);
    const bool uni = __all_sync(FULL, id < 0 || id == id0);
#pragma unroll
    for (int j = 0; j < PER; ++j)
      if (32 * j < d) stage_rows(X, d, 32 * j, row, tiles[wib][j]);
    float db = 0.f;
    if (uni) {
      const int64_t o0 = __shfl_sync(FULL, other, src);
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        const int t = lane + 32 * j;
        ref[t] = t < d ? X[o0 * d + t] : 0.f;
      }
      __syncwarp();
      if (row >= 0) {
#pragma unroll
        for (int j = 0; j < PER; ++j)
          if (32 * j < d) db = chunk_d2(tiles[wib][j], ref, 32 * j, db);
      }
    } else if (row >= 0) {
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        if (32 * j < d) {
          const float* y = X + other * d + 32 * j;
          const int tn = min(32, d - 32 * j);
          for (int jj = 0; jj < tn; ++jj) {
            const float df = tiles[wib][j][lane][jj] - y[jj];
            db = fmaf(df, df, db);
          }
        }
      }
    }
    const int sd = (row >= 0 && da[p] > db) ? 1 : 0;
    if (p < npacked) side[p] = sd;
    const unsigned m1 = __ballot_sync(FULL, sd != 0);
    if (uni) {
      if (id0 != cur) { flush(); cur = id0; }
#pragma unroll
      for (int j = 0; j < PER; ++j) {
        if (32 * j < d) {                    // warp-uniform
          float f0 = 0.f, f1 = 0.f;
#pragma unroll
          for (int r = 0; r < 32; ++r) {
            const float v = tiles[wib][j][r][lane];
            if ((m1 >> r) & 1u) f1 += v; else f0 += v;
          }
          s0[j] += f0;
          s1[j] += f1;
        }
      }
      c1 += __popc(m1);
      c0 += __popc(act & ~m1);
    } else {
      for (int r = 0; r < 32; ++r) {
        const int64_t idr = __shfl_sync(FULL, id, r);
        if (idr < 0) continue;               // warp-uniform
        const bool one = (m1 >> r) & 1u;
        if (idr != cur) { flush(); cur = idr; }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
          if (lane + 32 * j < d) {
            const float v = tiles[wib][j][r][lane];
            if (one) s1[j] += v; else s0[j] += v;
          }
        }
        if (one) c1 += 1.0; else c0 += 1.0;
      }
    }
    __syncwarp();                            // tiles and ref are restaged by the next task
  }
  // the last node's sums go to the block
  if (cur >= 0) {
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int t = lane + 32 * j;
      if (t < d) { part[wib][t] = s0[j]; part[wib][d + t] = s1[j]; }
    }
    if (lane == 0) { part[wib][2 * d] = c0; part[wib][2 * d + 1] = c1; }
  }
  if (lane == 0) part_node[wib] = cur;
  __syncthreads();
  if (wib == 0) {
    int w0 = 0;
    while (w0 < ROW_W) {
      const int64_t nd = part_node[w0];
      int w1 = w0 + 1;
      while (w1 < ROW_W && part_node[w1] == nd) ++w1;
      if (nd >= 0) {
        double* a = acc + nd * (2 * d + 2);
        for (int t = lane; t < 2 * d + 2; t += 32) {
          double v = 0.0;
          for (int w = w0; w < w1; ++w) v += part[w][t];
          if (v != 0.0) atomicAdd(&a[t], v);
        }
      }
      w0 = w1;
    }
  }
}

// second assignment: the nearer of the two side means (ties to side 0), in FP32 with each mean
// rounded once from its FP64 sum / count; a side left empty by the first assignment keeps it.  A
// warp inside one node stages the two means once in ref.
__global__ void __launch_bounds__(ROW_T)
reassign_kernel(const float* __restrict__ X, int d, int64_t npacked, int leaf,
                const int32_t* __restrict__ perm, const int32_t* __restrict__ ns,
                const int32_t* __restrict__ ne, const int64_t* __restrict__ S,
                const double* __restrict__ acc, int32_t* __restrict__ side) {
  __shared__ __align__(16) RowTile tiles[ROW_W];
  __shared__ __align__(16) RefRows refs[ROW_W];
  RowTile& tile = tiles[warp_id()];
  RefRows& ref = refs[warp_id()];
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t b = blockIdx.x * int64_t(blockDim.x) + (threadIdx.x & ~31); b < npacked;
       b += stride) {
    const int64_t p = b + lane_id();
    const double* a = nullptr;
    double i0 = 0.0, i1 = 0.0;
    int64_t slot = -1;
    int32_t row = -1;
    if (p < npacked) {
      const int st = ns[p];
      if (ne[p] - st > leaf) {
        slot = S[st];
        a = acc + slot * (2 * d + 2);
        const double n0 = a[2 * d], n1 = a[2 * d + 1];
        if (n0 != 0.0 && n1 != 0.0) {
          i0 = 1.0 / n0;
          i1 = 1.0 / n1;
          row = perm[p];
        }
      }
    }
    const unsigned act = __ballot_sync(FULL, row >= 0);
    if (act == 0) continue;                  // warp-uniform
    const int src = __ffs(act) - 1;
    const int64_t slot0 = __shfl_sync(FULL, slot, src);
    const bool uni = __all_sync(FULL, row < 0 || slot == slot0);
    if (uni) {
      const double* a0 = acc + slot0 * (2 * d + 2);
      const double j0 = __shfl_sync(FULL, i0, src), j1 = __shfl_sync(FULL, i1, src);
      for (int t = lane_id(); t < MSC_MAX_D; t += 32) {
        ref[0][t] = t < d ? float(a0[t] * j0) : 0.f;
        ref[1][t] = t < d ? float(a0[d + t] * j1) : 0.f;
      }
      __syncwarp();
    }
    float d0 = 0.f, d1 = 0.f;
    for (int c = 0; c < d; c += 32) {
      stage_rows(X, d, c, row, tile);
      if (row >= 0) {
        if (uni) {
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const float2 x = *reinterpret_cast<const float2*>(&tile[lane_id()][j]);
            const float2 m0 = *reinterpret_cast<const float2*>(&ref[0][c + j]);
            const float2 m1 = *reinterpret_cast<const float2*>(&ref[1][c + j]);
            float u = x.x - m0.x;
            d0 = fmaf(u, u, d0);
            u = x.y - m0.y;
            d0 = fmaf(u, u, d0);
            u = x.x - m1.x;
            d1 = fmaf(u, u, d1);
            u = x.y - m1.y;
            d1 = fmaf(u, u, d1);
          }
        } else {
          const int tn = min(32, d - c);
          for (int j = 0; j < tn; ++j) {
            const float v = tile[lane_id()][j];
            const float u0 = v - float(a[c + j] * i0), u1 = v - float(a[d + c + j] * i1);
            d0 = fmaf(u0, u0, d0);
            d1 = fmaf(u1, u1, d1);
          }
        }
      }
      __syncwarp();
    }
    if (row >= 0) side[p] = d0 > d1 ? 1 : 0;
  }
}

// start position of every split node of the level (its id: the scan of the split starts)
__global__ void node_start_kernel(int64_t npacked, const int32_t* __restrict__ flag,
                                  const int64_t* __restrict__ SN, int32_t* __restrict__ start) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x)
    if (flag[p]) start[SN[p]] = int32_t(p);
}

// More 2-means steps for the split nodes of a top level, one CTA per node: up to m_max of the
// node's rows (every (size/m)-th position) are staged in shared memory and the two side means,
// starting from the sums in acc, are moved `steps` times to the means of the staged rows nearer to
// each; the result replaces the node's sums (as means with counts of one) for the reassignment
// of every row.  A step that leaves a side empty ends the node's steps with the means before it.
constexpr int LLOYD_T = 256;
__global__ void __launch_bounds__(LLOYD_T)
lloyd_node_kernel(const float* __restrict__ X, int d, int64_t npacked,
                  const int32_t* __restrict__ perm, const int32_t* __restrict__ ne,
                  const int64_t* __restrict__ SN, const int32_t* __restrict__ start,
                  double* __restrict__ acc, int steps, int m_max) {
  extern __shared__ float xs[];                        // [m][d]
  __shared__ float mu[2][MSC_MAX_D];
  __shared__ int rows[LLOYD_SAMPLES_MAX], sides[LLOYD_SAMPLES_MAX];
  __shared__ int cnt[2];
  const int tid = threadIdx.x, lane = lane_id(), wib = warp_id();
  constexpr int NW = LLOYD_T / 32;
  const int64_t nodes = SN[npacked];
  for (int64_t b = blockIdx.x; b < nodes; b += gridDim.x) {     // block-uniform
    const int64_t s = start[b], size = int64_t(ne[s]) - s;
    const int m = int(min64(m_max, size));
    const int64_t stp = size / m;
    double* a = acc + b * (2 * d + 2);
    const double n0 = a[2 * d], n1 = a[2 * d + 1];
    if (n0 == 0.0 || n1 == 0.0) continue;
    for (int q = tid; q < 2 * d; q += LLOYD_T) {
      const int h = q >= d, t = q - h * d;
      mu[h][t] = float(a[q] / (h ? n1 : n0));
    }
    for (int j = tid; j < m; j += LLOYD_T) rows[j] = perm[s + int64_t(j) * stp];
    __syncthreads();
    // a warp per sample row (coalesced), four rows in flight per warp
    for (int j0 = wib * 4; j0 < m; j0 += NW * 4) {
      float v[4][4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int j = j0 + u, t = lane + 32 * c;
          v[u][c] = (j < m && t < d) ? X[int64_t(rows[j]) * d + t] : 0.f;
        }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int j = j0 + u, t = lane + 32 * c;
          if (j < m && t < d) xs[j * d + t] = v[u][c];
        }
    }
    __syncthreads();
    for (int it = 0; it < steps; ++it) {
      if (tid < 2) cnt[tid] = 0;
      __syncthreads();
      for (int j = tid; j < m; j += LLOYD_T) {
        float d0 = 0.f, d1 = 0.f;
        for (int t = 0; t < d; ++t) {
          const float x = xs[j * d + t];
          const float u0 = x - mu[0][t], u1 = x - mu[1][t];
          d0 = fmaf(u0, u0, d0);
          d1 = fmaf(u1, u1, d1);
        }
        const int sd = d0 > d1 ? 1 : 0;
        sides[j] = sd;
        atomicAdd(&cnt[sd], 1);
      }
      __syncthreads();
      const int c0 = cnt[0], c1 = cnt[1];
      if (c0 == 0 || c1 == 0) break;                 // block-uniform
      float s0 = 0.f, s1 = 0.f;
      if (tid < d) {
        for (int j = 0; j < m; ++j) {
          const float x = xs[j * d + tid];
          if (sides[j]) s1 += x; else s0 += x;
        }
      }
      __syncthreads();                                // every distance read mu
      if (tid < d) {
        mu[0][tid] = s0 / float(c0);
        mu[1][tid] = s1 / float(c1);
      }
      __syncthreads();
    }
    for (int q = tid; q < 2 * d; q += LLOYD_T) {
      const int h = q >= d, t = q - h * d;
      a[q] = double(mu[h][t]);
    }
    if (tid == 0) { a[2 * d] = 1.0; a[2 * d + 1] = 1.0; }
    __syncthreads();
  }
}

// Rows projected onto ORDER_PROJ_D random directions for the tree (entries ±1 from a fixed hash:
// a random sign matrix keeps the pairwise distances to within a small factor with high
// probability, which is all that choosing 2-means splits needs).  Each pass of a tree level then
// reads ORDER_PROJ_D floats per row instead of d; the balls, the plan and every distance of the
// graph use the exact rows.
__device__ __forceinline__ float proj_sign(int t, int j) {
  uint32_t h = uint32_t(t) * 0x9E3779B1u ^ (uint32_t(j) + 0x7F4A7C15u) * 0x85EBCA77u;
  h ^= h >> 15; h *= 0x2C1B3C6Du; h ^= h >> 12; h *= 0x297A2D39u; h ^= h >> 15;
  return (h & 1u) ? 1.f : -1.f;
}
__global__ void __launch_bounds__(256)
project_kernel(const float* __restrict__ X, int64_t n, int d, float* __restrict__ Y) {
  __shared__ float R[MSC_MAX_D][ORDER_PROJ_D];
  for (int e = threadIdx.x; e < d * ORDER_PROJ_D; e += blockDim.x)
    R[e / ORDER_PROJ_D][e % ORDER_PROJ_D] = proj_sign(e / ORDER_PROJ_D, e % ORDER_PROJ_D);
  __syncthreads();
  const int64_t total = n * ORDER_PROJ_D;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < total;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / ORDER_PROJ_D;
    const int j = int(e - i * ORDER_PROJ_D);
    const float* x = X + i * d;
    float acc = 0.f;
    for (int t = 0; t < d; ++t) acc = fmaf(x[t], R[t][j], acc);
    Y[e] = acc;
  }
}

// leaf of every packed position: the first position of its final node (-1: padding rows)
__global__ void leaf_id_kernel(int64_t npacked, const int32_t* __restrict__ perm,
                               const int32_t* __restrict__ ns, int32_t* __restrict__ leaf_out) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < npacked;
       p += int64_t(gridDim.x) * blockDim.x)
    leaf_out[p] = perm[p] >= 0 ? ns[p] : -1;
}

}  // namespace


// split nodes at one level: each holds more than `leaf` rows
inline int64_t max_split_nodes(int64_t npacked, int leaf) { return npacked / (leaf + 1) + 1; }

size_t order_workspace_bytes(int64_t npacked, int d, int leaf) {
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
  c.take<int32_t>(npacked);                       // split-node starts
  c.take<int64_t>(npacked + 1);                   // their scan: node ids
  c.take<double>(size_t(max_split_nodes(npacked, leaf)) * (2 * d + 2));   // side sums, counts
  c.take<int32_t>(size_t(max_split_nodes(npacked, leaf)));            // split-node starts by id
  return c.bytes();
}

int launch_order(const float* X, int d, const SegDesc* seg, int nseg, int64_t npacked, int levels,
                 int leaf, int32_t* perm, int32_t* leaf_out, void* ws, size_t ws_bytes,
                 cudaStream_t st, int64_t max_seg, const float* Xp, int dp, int proj_from) {
  const float* X0 = X;
  const int d0 = d;
  if (ws_bytes < order_workspace_bytes(npacked, d, leaf)) {
    set_error("order: workspace %zu < %zu bytes", ws_bytes, order_workspace_bytes(npacked, d, leaf));
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
  int32_t* sflag = c.take<int32_t>(npacked);
  int64_t* SN = c.take<int64_t>(npacked + 1);
  const size_t acc_elems = size_t(max_split_nodes(npacked, leaf)) * (2 * d + 2);
  double* acc = c.take<double>(acc_elems);
  int32_t* nstart = c.take<int32_t>(size_t(max_split_nodes(npacked, leaf)));
  const int grid = int(std::max<int64_t>(1, std::min<int64_t>(ceil_div(npacked, OR_T),
                                                              int64_t(num_sms()) * 8)));
  // the row passes: one wave of resident blocks each (a grid-stride grid of more blocks than the
  // SMs hold ran a second, partly filled wave)
  const int64_t wb = ceil_div(npacked, ROW_T);
  const int g_far_a = resident_grid(far_a_kernel, ROW_T, 0, wb);
  const int g_far_b = resident_grid(far_b_kernel, ROW_T, 0, wb);
  const int g_side = resident_grid(side_kernel, ROW_T, 0, wb);
  const int g_reassign = resident_grid(reassign_kernel, ROW_T, 0, wb);
  const int64_t sb = ceil_div(ceil_div(npacked, 32), ROW_W);
  const int g_fused1 = resident_grid(side_fused_kernel<1>, ROW_T, 0, sb);
  const int g_fused2 = resident_grid(side_fused_kernel<2>, ROW_T, 0, sb);
  const int g_sum4 = resident_grid(side_sum_kernel<4>, ROW_T, 0, sb);
  int lloyd_levels = LLOYD_LEVELS, lloyd_steps = LLOYD_STEPS;
  if (const char* e = std::getenv("MSC_B200_LLOYD_LEVELS")) lloyd_levels = std::max(0, std::atoi(e));
  if (const char* e = std::getenv("MSC_B200_LLOYD_STEPS")) lloyd_steps = std::max(0, std::atoi(e));
  const int m_max = int(std::min<size_t>(LLOYD_SAMPLES_MAX, LLOYD_SMEM_MAX / (sizeof(float) * d)));
  const size_t lsmem = size_t(m_max) * d * sizeof(float);
  if (lloyd_levels > 0 && lloyd_steps > 0) MSC_CUDA_TRY(raise_smem_cap(lloyd_node_kernel, lsmem));
  order_init_kernel<<<grid, OR_T, 0, st>>>(seg, nseg, npacked, perm, nsA, neA);
  MSC_LAUNCH_CHECK();
  int32_t *pc = perm, *pn = perm2, *sc = nsA, *ec = neA, *sn = nsB, *en = neB;
  for (int l = 0; l < levels; ++l) {
    // the exact rows on the top levels, where a split separates clusters; the projected rows below
    X = (Xp && l >= proj_from) ? Xp : X0;
    d = (Xp && l >= proj_from) ? dp : d0;
    // the level's split nodes and their ids (from the node bounds alone)
    split_start_kernel<<<grid, OR_T, 0, st>>>(npacked, leaf, sc, ec, sflag);
    MSC_LAUNCH_CHECK();
    MSC_TRY(scan_excl_i32(sflag, npacked, SN, scratch, st));
    MSC_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * acc_elems, st));
    MSC_CUDA_TRY(cudaMemsetAsync(best_a, 0, sizeof(unsigned long long) * npacked, st));
    MSC_CUDA_TRY(cudaMemsetAsync(best_b, 0, sizeof(unsigned long long) * npacked, st));
    far_a_kernel<<<g_far_a, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, best_a);
    MSC_LAUNCH_CHECK();
    far_b_kernel<<<g_far_b, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, best_a, da, best_b);
    MSC_LAUNCH_CHECK();
    // the nearer of a and b, then the side sums for one 2-means step (one pass for d <= 64)
    if (d <= 32) {
      side_fused_kernel<1><<<g_fused1, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, SN, da,
                                                        best_b, side, acc);
    } else if (d <= 64) {
      side_fused_kernel<2><<<g_fused2, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, SN, da,
                                                        best_b, side, acc);
    } else {
      side_kernel<<<g_side, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, da, best_b, side);
      MSC_LAUNCH_CHECK();
      side_sum_kernel<4><<<g_sum4, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, SN, side, acc);
    }
    MSC_LAUNCH_CHECK();
    if (l < lloyd_levels && lloyd_steps > 0 && (max_seg >> l) >= LLOYD_MIN_NODE) {
      node_start_kernel<<<grid, OR_T, 0, st>>>(npacked, sflag, SN, nstart);
      MSC_LAUNCH_CHECK();
      // a CTA per split node (every sample of a batch has its own nodes at every level); CTAs
      // beyond the level's node count return at once
      const int64_t nb = std::min<int64_t>(max_split_nodes(npacked, leaf), int64_t(num_sms()) * 4);
      lloyd_node_kernel<<<unsigned(std::max<int64_t>(1, nb)), LLOYD_T, lsmem, st>>>(
          X, d, npacked, pc, ec, SN, nstart, acc, lloyd_steps, m_max);
      MSC_LAUNCH_CHECK();
    }
    reassign_kernel<<<g_reassign, ROW_T, 0, st>>>(X, d, npacked, leaf, pc, sc, ec, SN, acc, side);
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
  if (leaf_out) {
    leaf_id_kernel<<<grid, OR_T, 0, st>>>(npacked, perm, sc, leaf_out);
    MSC_LAUNCH_CHECK();
  }
  return MSC_OK;
}

int launch_project(const float* X, int64_t n, int d, float* Y, cudaStream_t st) {
  const int grid = int(std::max<int64_t>(
      1, std::min<int64_t>(ceil_div(n * ORDER_PROJ_D, 256), int64_t(num_sms()) * 8)));
  project_kernel<<<grid, 256, 0, st>>>(X, n, d, Y);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
