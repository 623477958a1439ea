// Uniform-grid (cell-list) exact kNN and fixed-radius search of 2-D / 3-D coordinates: the
// spatial index of metalsinglecell's neighbors._knn_grid / _radius_grid (neighbors.py:143-417),
// which gr.spatial_neighbors_knn / _radius (gr.py:186-255) and spatial.spatial_neighbors
// (spatial.py:13-44) call.
//
// Arithmetic (the reference grid kernel's, neighbors.py:180-183, fixed so that every row follows
// it): d² = fl(fl(dx²) + fl(dy²)) [+ fl(dz²)], dx = fl(x_p − x_q), no fused multiply-add;
// distance = correctly rounded float32 sqrt(d²); kNN order (distance, index) with self first;
// radius test r_lo² ≤ d² ≤ r_hi² with r² rounded once to float32 (neighbors.py:301-302).
//
// Build, all on the device:
//   sp_bbox   per-axis minimum / maximum (order-preserving integer atomics), non-finite count
//   sp_plan   one thread: cell side, cells per axis (at most 4n + 16 cells), FP64 geometry
//   sp_bin    cell of every point (FP64 floor of (x − o) / cs), cell counts, chunk counts
//   scans     cell starts, chunk starts
//   sp_place  points in cell order as float4 (x, y, z, index bits)
//   sp_chunks chunk → (cell, first sorted position); a chunk is ≤ 32 points of one cell
// Search: one warp per chunk (persistent grid), one lane per query, candidates of a run of
// cells staged through shared memory and read by every lane (broadcast reads).
//   kNN: shells R = 0, 1, 2, ... of cells around the chunk's cell; each lane keeps its k − 1
//        best (distance, index) keys sorted in registers; it is done once its (k−1)-th distance
//        is provably below the distance to every cell outside the scanned box (FP64 bound with a
//        margin that covers float32 rounding), so every row is exact without a fallback pass.
//   radius: every cell within ring = ceil(D / cs) of the chunk's cell, D = radius plus a margin
//        that covers rounding; a count pass, a scan, a fill pass in the same walk order, then
//        each row's columns put in ascending order (rank sort).
#include <climits>

#include "kernels.cuh"

namespace msc {

namespace {

constexpr int SP_T = 128;                 // threads per block of the search kernels
constexpr int SP_W = SP_T / 32;
constexpr int SP_STAGE = 64;              // candidates staged per warp per round
constexpr int SORT_TILE = 256;            // columns staged per warp by the row sort
constexpr int SORT_E = 4;                 // entries ranked per lane per group

struct SpGrid {
  double o[3];          // origin (per-axis minimum)
  double cs;            // cell side
  double eps_abs;       // absolute slack of FP64 geometry
  double reach;         // radius search: D
  int32_t g[3];         // cells per axis (1 on an unused axis)
  int32_t ring;         // radius search: cells scanned on each side
  int64_t ncells;
  int32_t status;       // 0 ok, 1 non-finite coordinates, 2 plan failed
  int32_t pad;
};

__device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ __forceinline__ unsigned f2o(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// mm[0..2] = ordered minima, mm[3..5] = ordered maxima (initialised to 0xffffffff / 0)
__global__ void sp_bbox_kernel(const float* __restrict__ X, int64_t n, int d,
                               unsigned* __restrict__ mm, unsigned long long* __restrict__ nonfinite) {
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  unsigned long long bad = 0;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    for (int a = 0; a < d; ++a) {
      float v = X[i * d + a];
      if (!isfinite(v)) { ++bad; continue; }
      lo[a] = fminf(lo[a], v);
      hi[a] = fmaxf(hi[a], v);
    }
  }
  for (int a = 0; a < d; ++a) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
    }
  }
  for (int off = 16; off > 0; off >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, off);
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < d; ++a) {
      if (lo[a] <= hi[a]) {
        atomicMin(&mm[a], f2o(lo[a]));
        atomicMax(&mm[3 + a], f2o(hi[a]));
      }
    }
    if (bad) atomicAdd(nonfinite, bad);
  }
}

// mode 0: kNN (k), mode 1: radius (reach = D > 0)
__global__ void sp_plan_kernel(const unsigned* __restrict__ mm,
                               const unsigned long long* __restrict__ nonfinite, int64_t n, int d,
                               int mode, int k, double reach, SpGrid* __restrict__ G) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  SpGrid g{};
  g.reach = reach;
  if (*nonfinite) { g.status = 1; *G = g; return; }
  double ext[3] = {0, 0, 0};
  double mag = 0;
  int eff = 0;
  for (int a = 0; a < 3; ++a) {
    if (a < d) {
      const double lo = double(o2f(mm[a])), hi = double(o2f(mm[3 + a]));
      g.o[a] = lo;
      ext[a] = hi - lo;
      mag = fmax(mag, fmax(fabs(lo), fabs(hi)));
      if (ext[a] > 0) ++eff;
    } else {
      g.o[a] = 0;
    }
  }
  double cs;
  if (mode == 0) {
    if (eff == 0) {
      cs = 1.0;
    } else {
      double vol = 1.0;
      for (int a = 0; a < 3; ++a) if (ext[a] > 0) vol *= ext[a];
      const double target = double(k > 4 ? 2 * k : 8);
      cs = pow(target * vol / double(n), 1.0 / eff);
    }
  } else {
    cs = reach > 0 ? reach * (1.0 + 1e-6) : 1.0;
  }
  const double cap = 4.0 * double(n) + 16.0;
  double cells = 0;
  bool ok = false;
  for (int it = 0; it < 200; ++it) {
    cells = 1;
    for (int a = 0; a < 3; ++a) cells *= ext[a] > 0 ? ceil(ext[a] / cs) + 1.0 : 1.0;
    if (cells <= cap) { ok = true; break; }
    if (!isfinite(cells) || !(cs > 0)) {
      // a cell side so small that the cell count overflows: restart from two cells per axis
      cs = fmax(fmax(ext[0], ext[1]), ext[2]) * 0.5;
      continue;
    }
    cs *= pow(cells / cap, 1.0 / (eff > 0 ? eff : 1)) * (1.0 + 1e-9);
  }
  if (!ok || !(cs > 0) || !isfinite(cs)) { g.status = 2; *G = g; return; }
  for (int a = 0; a < 3; ++a) g.g[a] = ext[a] > 0 ? int32_t(ceil(ext[a] / cs) + 1.0) : 1;
  g.ncells = int64_t(g.g[0]) * g.g[1] * g.g[2];
  g.cs = cs;
  g.eps_abs = 1e-12 * (mag + cs);
  if (mode == 1) {
    const double r = reach / cs + 1e-7;
    int ring = int(ceil(r));
    int gmax = max(g.g[0], max(g.g[1], g.g[2]));
    g.ring = max(1, min(ring, gmax));
  }
  *G = g;
}

__device__ __forceinline__ int cell_axis(float x, const SpGrid& g, int a) {
  const double t = floor((double(x) - g.o[a]) / g.cs);
  int c = t < 0 ? 0 : (t > double(g.g[a] - 1) ? g.g[a] - 1 : int(t));
  return c;
}

__device__ __forceinline__ int64_t cell_of(const float* p, int d, const SpGrid& g) {
  const int cx = cell_axis(p[0], g, 0);
  const int cy = cell_axis(p[1], g, 1);
  const int cz = d == 3 ? cell_axis(p[2], g, 2) : 0;
  return (int64_t(cz) * g.g[1] + cy) * g.g[0] + cx;
}

__global__ void sp_bin_kernel(const float* __restrict__ X, int64_t n, int d,
                              const SpGrid* __restrict__ G, int64_t* __restrict__ cell,
                              int32_t* __restrict__ count) {
  const SpGrid g = *G;
  if (g.status) return;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t c = cell_of(X + i * d, d, g);
    cell[i] = c;
    atomicAdd(&count[c], 1);
  }
}

__global__ void sp_chunk_count_kernel(const int32_t* __restrict__ count, const SpGrid* __restrict__ G,
                                      int32_t* __restrict__ nchunk) {
  const int64_t nc = G->status ? 0 : G->ncells;
  for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < nc;
       c += int64_t(gridDim.x) * blockDim.x)
    nchunk[c] = (count[c] + 31) >> 5;
}

__global__ void sp_place_kernel(const float* __restrict__ X, int64_t n, int d,
                                const SpGrid* __restrict__ G, const int64_t* __restrict__ cell,
                                const int64_t* __restrict__ cell_start, int32_t* __restrict__ cursor,
                                float4* __restrict__ pts) {
  if (G->status) return;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t c = cell[i];
    const int64_t pos = cell_start[c] + atomicAdd(&cursor[c], 1);
    const float* p = X + i * d;
    pts[pos] = make_float4(p[0], p[1], d == 3 ? p[2] : 0.f, __int_as_float(int(i)));
  }
}

// chunk j → (its cell, its first sorted position): the cell is the last c with
// chunk_start[c] <= j (binary search), so a cell with many points spreads over many threads
__global__ void sp_chunks_kernel(const int64_t* __restrict__ cell_start,
                                 const int64_t* __restrict__ chunk_start, int64_t cap,
                                 int2* __restrict__ chunks) {
  const int64_t total = chunk_start[cap];
  for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < total;
       j += int64_t(gridDim.x) * blockDim.x) {
    int64_t lo = 0, hi = cap;                 // chunk_start[lo] <= j < chunk_start[hi]
    while (hi - lo > 1) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (chunk_start[mid] <= j) lo = mid; else hi = mid;
    }
    chunks[j] = make_int2(int(lo), int(cell_start[lo] + (j - chunk_start[lo]) * 32));
  }
}

template <int D>
__device__ __forceinline__ float sq_dist(const float4& p, const float4& q) {
  const float dx = __fsub_rn(p.x, q.x);
  float s = __fmul_rn(dx, dx);
  const float dy = __fsub_rn(p.y, q.y);
  s = __fadd_rn(s, __fmul_rn(dy, dy));
  if (D == 3) {
    const float dz = __fsub_rn(p.z, q.z);
    s = __fadd_rn(s, __fmul_rn(dz, dz));
  }
  return s;
}

__device__ __forceinline__ bool key_less(float s, int i, float ts, int ti) {
  return s < ts || (s == ts && i < ti);
}

// d² above this cannot give a distance ≤ top: (next float above top)², rounded up
__device__ __forceinline__ float prefilter(float top) {
  if (top < 0.f) return -1.f;
  if (isinf(top)) return INFINITY;
  const float up = __uint_as_float(__float_as_uint(top) + 1u);
  return __fmul_ru(up, up);
}

// Stage the points [a, b) through the warp's shared buffer; f(candidate) runs on every lane.
template <class F>
__device__ __forceinline__ void scan_run(const float4* __restrict__ pts, int64_t a, int64_t b,
                                         float4* stage, int lane, F&& f) {
  for (int64_t base = a; base < b; base += SP_STAGE) {
    const int cnt = int(imin64(SP_STAGE, b - base));
    __syncwarp();
    for (int j = lane; j < cnt; j += 32) stage[j] = pts[base + j];
    __syncwarp();
    for (int t = 0; t < cnt; ++t) f(stage[t]);
  }
}

template <int K, int D>
__global__ void __launch_bounds__(SP_T)
sp_knn_kernel(const float4* __restrict__ pts, const int64_t* __restrict__ cell_start,
              const int2* __restrict__ chunks, const int64_t* __restrict__ chunk_start,
              const SpGrid* __restrict__ G, int k, int32_t* __restrict__ out_idx,
              float* __restrict__ out_dist, unsigned long long* __restrict__ counters) {
  __shared__ float4 stage_all[SP_W][SP_STAGE];
  const SpGrid g = *G;
  if (g.status) return;
  const int lane = threadIdx.x & 31;
  float4* stage = stage_all[threadIdx.x >> 5];
  const int64_t nchunks = chunk_start[g.ncells];
  const int64_t wid = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int m = k - 1;
  unsigned long long evals = 0, expanded = 0;
  for (int64_t ch = wid; ch < nchunks; ch += nw) {
    const int2 c = chunks[ch];
    const int64_t qend = imin64(int64_t(c.y) + 32, cell_start[int64_t(c.x) + 1]);
    const int64_t qpos = int64_t(c.y) + lane;
    const bool active = qpos < qend;
    const float4 q = active ? pts[qpos] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int qi = active ? __float_as_int(q.w) : -1;
    const int cx = int(int64_t(c.x) % g.g[0]);
    const int cy = int((int64_t(c.x) / g.g[0]) % g.g[1]);
    const int cz = int(int64_t(c.x) / (int64_t(g.g[0]) * g.g[1]));
    float s[K];
    int id[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const bool sent = j < K - m;
      s[j] = sent ? -1.f : INFINITY;
      id[j] = sent ? -1 : INT_MAX;
    }
    float t2 = prefilter(s[K - 1]);
    bool done = !active;
    const int rmax = max(max(cx, g.g[0] - 1 - cx),
                         max(max(cy, g.g[1] - 1 - cy), D == 3 ? max(cz, g.g[2] - 1 - cz) : 0));
    auto visit = [&](const float4& p) {
      if (done) return;
      const float d2 = sq_dist<D>(p, q);
      const int pid = __float_as_int(p.w);
      ++evals;
      if (d2 <= t2 && pid != qi) {
        const float sd = __fsqrt_rn(d2);
        if (key_less(sd, pid, s[K - 1], id[K - 1])) {
#pragma unroll
          for (int j = K - 1; j > 0; --j) {
            const bool lp = key_less(sd, pid, s[j - 1], id[j - 1]);
            const bool lc = key_less(sd, pid, s[j], id[j]);
            const float ns = lp ? s[j - 1] : (lc ? sd : s[j]);
            const int ni = lp ? id[j - 1] : (lc ? pid : id[j]);
            s[j] = ns;
            id[j] = ni;
          }
          if (key_less(sd, pid, s[0], id[0])) { s[0] = sd; id[0] = pid; }
          t2 = prefilter(s[K - 1]);
        }
      }
    };
    auto run = [&](int y, int z, int x0, int x1) {
      x0 = max(x0, 0);
      x1 = min(x1, g.g[0] - 1);
      if (x0 > x1 || y < 0 || y >= g.g[1] || z < 0 || z >= g.g[2]) return;
      const int64_t row = (int64_t(z) * g.g[1] + y) * g.g[0];
      scan_run(pts, cell_start[row + x0], cell_start[row + x1 + 1], stage, lane, visit);
    };
    for (int R = 0;; ++R) {
      const int zlo = D == 3 ? -R : 0, zhi = D == 3 ? R : 0;
      for (int dz = zlo; dz <= zhi; ++dz) {
        for (int dy = -R; dy <= R; ++dy) {
          const bool full = (dy == -R || dy == R || (D == 3 && (dz == -R || dz == R)));
          if (full) {
            run(cy + dy, cz + dz, cx - R, cx + R);
          } else {
            run(cy + dy, cz + dz, cx - R, cx - R);
            run(cy + dy, cz + dz, cx + R, cx + R);
          }
        }
      }
      if (!done) {
        // distance from the query to the nearest face of the box of cells within R that has
        // points beyond it; a box that reaches the grid's edge on a side bounds nothing there
        double bound = INFINITY;
        const int cc[3] = {cx, cy, cz};
        const float qq[3] = {q.x, q.y, q.z};
#pragma unroll
        for (int a = 0; a < D; ++a) {
          if (cc[a] - R > 0)
            bound = fmin(bound, double(qq[a]) - (g.o[a] + double(cc[a] - R) * g.cs));
          if (cc[a] + R < g.g[a] - 1)
            bound = fmin(bound, (g.o[a] + double(cc[a] + R + 1) * g.cs) - double(qq[a]));
        }
        if (isinf(bound) || double(s[K - 1]) < bound * (1.0 - 4e-6) - g.eps_abs) {
          done = true;
          if (R >= 2) ++expanded;
        }
      }
      if (__all_sync(0xffffffffu, done) || R >= rmax) break;
    }
    if (active) {
      int32_t* oi = out_idx + int64_t(qi) * k;
      float* od = out_dist + int64_t(qi) * k;
      oi[0] = qi;
      od[0] = 0.f;
#pragma unroll
      for (int j = 0; j < K; ++j) {
        if (j >= K - m) {
          oi[1 + j - (K - m)] = id[j];
          od[1 + j - (K - m)] = s[j];
        }
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    evals += __shfl_xor_sync(0xffffffffu, evals, off);
    expanded += __shfl_xor_sync(0xffffffffu, expanded, off);
  }
  if (lane == 0) {
    atomicAdd(&counters[0], evals);
    atomicAdd(&counters[1], expanded);
  }
}

// Radius search.  pass 0 counts into count[qi]; pass 1 writes (column, distance) from
// indptr[qi] in the same walk order.
template <int D>
__global__ void __launch_bounds__(SP_T)
sp_radius_kernel(const float4* __restrict__ pts, const int64_t* __restrict__ cell_start,
                 const int2* __restrict__ chunks, const int64_t* __restrict__ chunk_start,
                 const SpGrid* __restrict__ G, float r2lo, float r2hi, int pass,
                 int32_t* __restrict__ count, const int64_t* __restrict__ indptr,
                 int32_t* __restrict__ col, float* __restrict__ val,
                 unsigned long long* __restrict__ counters) {
  __shared__ float4 stage_all[SP_W][SP_STAGE];
  const SpGrid g = *G;
  if (g.status) return;
  const int lane = threadIdx.x & 31;
  float4* stage = stage_all[threadIdx.x >> 5];
  const int64_t nchunks = chunk_start[g.ncells];
  const int64_t wid = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int R = g.ring;
  unsigned long long evals = 0;
  for (int64_t ch = wid; ch < nchunks; ch += nw) {
    const int2 c = chunks[ch];
    const int64_t qend = imin64(int64_t(c.y) + 32, cell_start[int64_t(c.x) + 1]);
    const int64_t qpos = int64_t(c.y) + lane;
    const bool active = qpos < qend;
    const float4 q = active ? pts[qpos] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int qi = active ? __float_as_int(q.w) : -1;
    const int cx = int(int64_t(c.x) % g.g[0]);
    const int cy = int((int64_t(c.x) / g.g[0]) % g.g[1]);
    const int cz = int(int64_t(c.x) / (int64_t(g.g[0]) * g.g[1]));
    int64_t w = (pass == 1 && active) ? indptr[qi] : 0;
    int32_t cnt = 0;
    auto visit = [&](const float4& p) {
      if (!active) return;
      const float d2 = sq_dist<D>(p, q);
      const int pid = __float_as_int(p.w);
      ++evals;
      if (pid != qi && d2 <= r2hi && d2 >= r2lo) {
        if (pass == 1) {
          col[w] = pid;
          val[w] = __fsqrt_rn(d2);
          ++w;
        }
        ++cnt;
      }
    };
    const int zlo = D == 3 ? max(cz - R, 0) : 0, zhi = D == 3 ? min(cz + R, g.g[2] - 1) : 0;
    const int x0 = max(cx - R, 0), x1 = min(cx + R, g.g[0] - 1);
    for (int z = zlo; z <= zhi; ++z) {
      for (int y = max(cy - R, 0); y <= min(cy + R, g.g[1] - 1); ++y) {
        const int64_t row = (int64_t(z) * g.g[1] + y) * g.g[0];
        scan_run(pts, cell_start[row + x0], cell_start[row + x1 + 1], stage, lane, visit);
      }
    }
    if (pass == 0 && active) count[qi] = cnt;
  }
  for (int off = 16; off > 0; off >>= 1) evals += __shfl_xor_sync(0xffffffffu, evals, off);
  if (lane == 0) atomicAdd(&counters[0], evals);
}

// Columns of every row in ascending order (they are distinct within a row): the rank of an
// entry is the number of smaller columns in its row.  One warp per row.
__global__ void __launch_bounds__(SP_T)
sp_sort_rows_kernel(const int64_t* __restrict__ indptr, int64_t n, const int32_t* __restrict__ col_in,
                    const float* __restrict__ val_in, int32_t* __restrict__ col_out,
                    float* __restrict__ val_out) {
  __shared__ int32_t tile_all[SP_W][SORT_TILE];
  const int lane = threadIdx.x & 31;
  int32_t* tile = tile_all[threadIdx.x >> 5];
  const int64_t wid = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t row = wid; row < n; row += nw) {
    const int64_t a = indptr[row];
    const int64_t m = indptr[row + 1] - a;
    for (int64_t g0 = 0; g0 < m; g0 += 32 * SORT_E) {
      int32_t mine[SORT_E];
      int64_t rank[SORT_E];
#pragma unroll
      for (int e = 0; e < SORT_E; ++e) {
        const int64_t j = g0 + lane + 32 * e;
        mine[e] = j < m ? col_in[a + j] : INT_MAX;
        rank[e] = 0;
      }
      for (int64_t t0 = 0; t0 < m; t0 += SORT_TILE) {
        const int cnt = int(imin64(SORT_TILE, m - t0));
        __syncwarp();
        for (int j = lane; j < cnt; j += 32) tile[j] = col_in[a + t0 + j];
        __syncwarp();
        for (int t = 0; t < cnt; ++t) {
          const int32_t v = tile[t];
#pragma unroll
          for (int e = 0; e < SORT_E; ++e) rank[e] += v < mine[e];
        }
      }
#pragma unroll
      for (int e = 0; e < SORT_E; ++e) {
        const int64_t j = g0 + lane + 32 * e;
        if (j < m) {
          col_out[a + rank[e]] = mine[e];
          val_out[a + rank[e]] = val_in[a + j];
        }
      }
    }
  }
}

// FP64 edge lengths of a CSR graph from float64 coordinates (gr.py:32-34): squares summed axis
// by axis in order, correctly rounded sqrt.  One warp per row.
__global__ void sp_edge_len_kernel(const double* __restrict__ X, int d,
                                   const int64_t* __restrict__ indptr, int64_t n,
                                   const int32_t* __restrict__ cols, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t row = wid; row < n; row += nw) {
    const double* xi = X + row * d;
    for (int64_t e = indptr[row] + lane; e < indptr[row + 1]; e += 32) {
      const double* xj = X + int64_t(cols[e]) * d;
      double acc = 0;
      for (int a = 0; a < d; ++a) {
        const double t = __dsub_rn(xi[a], xj[a]);
        const double t2 = __dmul_rn(t, t);
        acc = a == 0 ? t2 : __dadd_rn(acc, t2);
      }
      out[e] = __dsqrt_rn(acc);
    }
  }
}

__global__ void sp_init_kernel(unsigned* mm, unsigned long long* nonfinite, unsigned long long* counters) {
  if (threadIdx.x < 3) { mm[threadIdx.x] = 0xffffffffu; mm[3 + threadIdx.x] = 0u; }
  if (threadIdx.x == 0) { *nonfinite = 0; counters[0] = 0; counters[1] = 0; }
}

__global__ void sp_stats_kernel(const SpGrid* __restrict__ G, const unsigned long long* __restrict__ nonfinite,
                                const unsigned long long* __restrict__ counters,
                                const int64_t* __restrict__ chunk_start, int64_t* __restrict__ stats) {
  if (threadIdx.x != 0) return;
  const SpGrid g = *G;
  stats[MSC_SP_STAT_NONFINITE] = int64_t(*nonfinite);
  stats[MSC_SP_STAT_STATUS] = g.status;
  stats[MSC_SP_STAT_CELLS] = g.status ? 0 : g.ncells;
  stats[MSC_SP_STAT_CHUNKS] = g.status ? 0 : chunk_start[g.ncells];
  stats[MSC_SP_STAT_EVALS] = int64_t(counters[0]);
  stats[MSC_SP_STAT_EXPANDED] = int64_t(counters[1]);
  stats[MSC_SP_STAT_RING] = g.status ? 0 : g.ring;
  stats[MSC_SP_STAT_CELL_SIDE] = g.status ? 0 : int64_t(__double_as_longlong(g.cs));
}

struct SpWs {
  SpGrid* G;
  unsigned* mm;
  unsigned long long* nonfinite;
  unsigned long long* counters;
  int64_t* cell;          // [n]
  int32_t* count;         // [cap]
  int32_t* cursor;        // [cap]
  int32_t* nchunk;        // [cap]
  int64_t* cell_start;    // [cap + 1]
  int64_t* chunk_start;   // [cap + 1]
  int64_t* scan_scratch;
  float4* pts;            // [n]
  int2* chunks;           // [cap + n / 32 + 1]
};

int64_t cell_cap(int64_t n) { return 4 * n + 16; }

SpWs carve(Carver& c, int64_t n) {
  const int64_t cap = cell_cap(n);
  SpWs w;
  w.G = c.take<SpGrid>(1);
  w.mm = c.take<unsigned>(8);
  w.nonfinite = c.take<unsigned long long>(1);
  w.counters = c.take<unsigned long long>(2);
  w.cell = c.take<int64_t>(n);
  w.count = c.take<int32_t>(cap);
  w.cursor = c.take<int32_t>(cap);
  w.nchunk = c.take<int32_t>(cap);
  w.cell_start = c.take<int64_t>(cap + 1);
  w.chunk_start = c.take<int64_t>(cap + 1);
  w.scan_scratch = c.take<int64_t>(scan_i32_scratch_elems(cap));
  w.pts = c.take<float4>(n);
  w.chunks = c.take<int2>(cap + n / 32 + 1);
  return w;
}


unsigned flat_grid(int64_t items, int threads) {
  const int64_t b = (items + threads - 1) / threads;
  return unsigned(std::max<int64_t>(1, std::min<int64_t>(b, int64_t(num_sms()) * 16)));
}

// The grid: bounding box, plan, binning, cell-ordered points, chunks.  The cell table is sized
// for the cap; the plan never uses more cells than that.
int build_grid(const float* X, int64_t n, int d, int mode, int k, double reach, const SpWs& w,
               cudaStream_t st) {
  const int64_t cap = cell_cap(n);
  sp_init_kernel<<<1, 32, 0, st>>>(w.mm, w.nonfinite, w.counters);
  MSC_LAUNCH_CHECK();
  sp_bbox_kernel<<<flat_grid(n, 256), 256, 0, st>>>(X, n, d, w.mm, w.nonfinite);
  MSC_LAUNCH_CHECK();
  sp_plan_kernel<<<1, 32, 0, st>>>(w.mm, w.nonfinite, n, d, mode, k, reach, w.G);
  MSC_LAUNCH_CHECK();
  MSC_CUDA_TRY(cudaMemsetAsync(w.count, 0, sizeof(int32_t) * cap, st));
  MSC_CUDA_TRY(cudaMemsetAsync(w.cursor, 0, sizeof(int32_t) * cap, st));
  MSC_CUDA_TRY(cudaMemsetAsync(w.nchunk, 0, sizeof(int32_t) * cap, st));
  sp_bin_kernel<<<flat_grid(n, 256), 256, 0, st>>>(X, n, d, w.G, w.cell, w.count);
  MSC_LAUNCH_CHECK();
  sp_chunk_count_kernel<<<flat_grid(cap, 256), 256, 0, st>>>(w.count, w.G, w.nchunk);
  MSC_LAUNCH_CHECK();
  // scans over the whole cap: cells the plan does not use hold zero counts, so
  // cell_start[ncells] = n and chunk_start[ncells] = the number of chunks
  MSC_TRY(scan_excl_i32(w.count, cap, w.cell_start, w.scan_scratch, st));
  MSC_TRY(scan_excl_i32(w.nchunk, cap, w.chunk_start, w.scan_scratch, st));
  sp_place_kernel<<<flat_grid(n, 256), 256, 0, st>>>(X, n, d, w.G, w.cell, w.cell_start, w.cursor,
                                                      w.pts);
  MSC_LAUNCH_CHECK();
  sp_chunks_kernel<<<flat_grid(cap + n / 32 + 1, 256), 256, 0, st>>>(w.cell_start, w.chunk_start,
                                                                       cap, w.chunks);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

unsigned search_grid(int64_t n) {
  // persistent: enough warps for every chunk of a uniform layout, at most 8 blocks per SM
  const int64_t warps = n / 16 + 1;
  const int64_t blocks = (warps + SP_W - 1) / SP_W;
  return unsigned(std::max<int64_t>(1, std::min<int64_t>(blocks, int64_t(num_sms()) * 8)));
}

template <int K>
int launch_knn_k(const SpWs& w, int64_t n, int d, int k, int32_t* idx, float* dist, cudaStream_t st) {
  if (d == 2)
    sp_knn_kernel<K, 2><<<search_grid(n), SP_T, 0, st>>>(w.pts, w.cell_start, w.chunks,
                                                         w.chunk_start, w.G, k, idx, dist,
                                                         w.counters);
  else
    sp_knn_kernel<K, 3><<<search_grid(n), SP_T, 0, st>>>(w.pts, w.cell_start, w.chunks,
                                                         w.chunk_start, w.G, k, idx, dist,
                                                         w.counters);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace

size_t spatial_knn_workspace_bytes(int64_t n) {
  Carver c(nullptr);
  carve(c, n);
  return c.bytes();
}

int launch_spatial_knn(const float* X, int64_t n, int d, int k, int32_t* idx, float* dist,
                       int64_t* stats, void* ws, cudaStream_t st) {
  Carver c(ws);
  const SpWs w = carve(c, n);
  MSC_TRY(build_grid(X, n, d, 0, k, 0.0, w, st));
  const int m = k - 1;
  if (m <= 8) MSC_TRY(launch_knn_k<8>(w, n, d, k, idx, dist, st));
  else if (m <= 16) MSC_TRY(launch_knn_k<16>(w, n, d, k, idx, dist, st));
  else if (m <= 32) MSC_TRY(launch_knn_k<32>(w, n, d, k, idx, dist, st));
  else MSC_TRY(launch_knn_k<64>(w, n, d, k, idx, dist, st));
  sp_stats_kernel<<<1, 32, 0, st>>>(w.G, w.nonfinite, w.counters, w.chunk_start, stats);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

size_t spatial_radius_workspace_bytes(int64_t n) {
  Carver c(nullptr);
  carve(c, n);
  c.take<int32_t>(n);                     // per-row counts
  return c.bytes();
}

int launch_spatial_radius_count(const float* X, int64_t n, int d, double radius, double min_radius,
                                int64_t* indptr, int64_t* stats, void* ws, cudaStream_t st) {
  Carver c(ws);
  const SpWs w = carve(c, n);
  int32_t* rowcnt = c.take<int32_t>(n);
  const double reach = radius * (1.0 + 1e-6);
  MSC_TRY(build_grid(X, n, d, 1, 0, reach, w, st));
  MSC_CUDA_TRY(cudaMemsetAsync(rowcnt, 0, sizeof(int32_t) * n, st));
  const float r2hi = float(radius * radius), r2lo = float(min_radius * min_radius);
  if (d == 2)
    sp_radius_kernel<2><<<search_grid(n), SP_T, 0, st>>>(w.pts, w.cell_start, w.chunks,
                                                         w.chunk_start, w.G, r2lo, r2hi, 0, rowcnt,
                                                         nullptr, nullptr, nullptr, w.counters);
  else
    sp_radius_kernel<3><<<search_grid(n), SP_T, 0, st>>>(w.pts, w.cell_start, w.chunks,
                                                         w.chunk_start, w.G, r2lo, r2hi, 0, rowcnt,
                                                         nullptr, nullptr, nullptr, w.counters);
  MSC_LAUNCH_CHECK();
  MSC_TRY(scan_excl_i32(rowcnt, n, indptr, w.scan_scratch, st));
  sp_stats_kernel<<<1, 32, 0, st>>>(w.G, w.nonfinite, w.counters, w.chunk_start, stats);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

size_t spatial_radius_fill_scratch_bytes(int64_t nnz) {
  Carver c(nullptr);
  c.take<int32_t>(nnz);
  c.take<float>(nnz);
  return c.bytes();
}

int launch_spatial_radius_fill(int64_t n, int d, double radius, double min_radius,
                               const int64_t* indptr, int64_t nnz, int32_t* cols, float* dist,
                               void* ws, void* scratch, cudaStream_t st) {
  Carver c(ws);
  const SpWs w = carve(c, n);
  Carver s(scratch);
  int32_t* col_tmp = s.take<int32_t>(nnz);
  float* val_tmp = s.take<float>(nnz);
  const float r2hi = float(radius * radius), r2lo = float(min_radius * min_radius);
  if (nnz > 0) {
    if (d == 2)
      sp_radius_kernel<2><<<search_grid(n), SP_T, 0, st>>>(w.pts, w.cell_start, w.chunks,
                                                           w.chunk_start, w.G, r2lo, r2hi, 1,
                                                           nullptr, indptr, col_tmp, val_tmp,
                                                           w.counters);
    else
      sp_radius_kernel<3><<<search_grid(n), SP_T, 0, st>>>(w.pts, w.cell_start, w.chunks,
                                                           w.chunk_start, w.G, r2lo, r2hi, 1,
                                                           nullptr, indptr, col_tmp, val_tmp,
                                                           w.counters);
    MSC_LAUNCH_CHECK();
    sp_sort_rows_kernel<<<search_grid(n * 8), SP_T, 0, st>>>(indptr, n, col_tmp, val_tmp, cols,
                                                             dist);
    MSC_LAUNCH_CHECK();
  }
  return MSC_OK;
}

int launch_spatial_edge_lengths(const double* X, int64_t n, int d, const int64_t* indptr,
                                const int32_t* cols, double* out, cudaStream_t st) {
  sp_edge_len_kernel<<<flat_grid(n * 32, 256), 256, 0, st>>>(X, d, indptr, n, cols, out);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

}  // namespace msc
