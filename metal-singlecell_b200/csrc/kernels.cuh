// Internal declarations shared by the msc_b200 translation units (not part of the C ABI).
#pragma once

#include "msc_common.cuh"

namespace msc {

// internal precision ids (same values as the MSC_PREC_* ABI constants)
constexpr int PREC_FP32 = MSC_PREC_FP32;
constexpr int PREC_BF16X3 = MSC_PREC_BF16X3;
constexpr int PREC_FP16 = MSC_PREC_FP16;
constexpr int PREC_BF16 = MSC_PREC_BF16;

// norm term written into padded key rows: their v = Σ terms is larger than any real v
constexpr double PAD_NORM_TERM_FP16 = 65504.0;
constexpr double PAD_NORM_TERM_BF16 = 1.0e30;
constexpr float PAD_SQ_FP32 = 1.0e30f;

// one sample ("segment") of the input
struct SegDesc {
  int64_t off;      // first original row
  int64_t n;        // cells
  int64_t poff;     // first packed row
  int64_t padlen;   // packed rows (n rounded up to SEG_PAD)
  int64_t tile0;    // index of the sample's first 128-row query tile
  int64_t ntiles;   // query tiles of the sample
  int64_t ptile0;   // index of the sample's first 256-row query tile (CTA-pair work items)
  int64_t pad1;
};

__device__ __forceinline__ int find_seg(const SegDesc* seg, int nseg, int64_t p) {
  // last segment with poff <= p
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (seg[mid].poff <= p) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// operand layout of a precision: elements per packed row loaded (multiple of 64) and the K
// extent the MMAs cover (multiple of 16)
struct OpLayout {
  int split;    // 1 or 3 (data terms)
  int kdata;    // split·d + 3 norm terms
  int kp;       // load width, multiple of 64 elements (128-byte swizzle atoms)
  int kmma;     // K covered by the MMAs, multiple of 16
};
inline OpLayout op_layout(int prec, int d) {
  OpLayout L;
  L.split = prec == PREC_BF16X3 ? 3 : 1;
  L.kdata = L.split * d + 3;
  L.kp = int(round_up(L.kdata, 64));
  L.kmma = int(round_up(L.kdata, 16));
  return L;
}

// ---- prep.cu ----
int launch_normalize(const float* X, float* Xn, int64_t n, int d, int64_t* nonfinite,
                     cudaStream_t st);
int launch_colmean(const float* X, const SegDesc* seg, int nseg, int64_t max_seg_n, int d,
                   double* partial, int nb, double* mean, int64_t* nonfinite, cudaStream_t st);
size_t colmean_partial_elems(int nseg, int d, int nb);
int launch_maxnorm(const float* X, const SegDesc* seg, int nseg, const double* mean, int d,
                   int64_t npacked, Ctl* ctl, cudaStream_t st);
// packed row p holds original row perm[p] (-1: padding) of the sample seg[find_seg(p)]
// rows/nrows: pack only the listed packed rows (device count, at most max_rows) into output rows
// 0..; null: every packed row.  Aop or Bop may be null; qs/km (key statistics) may be null.
int launch_pack_tc(int prec, const float* X, const int32_t* perm, const SegDesc* seg, int nseg,
                   const double* mean, int d, int64_t npacked, const int32_t* rows,
                   const int32_t* nrows, int64_t max_rows, void* Aop, void* Bop, QStat* qs,
                   KeyMax* km, const Ctl* ctl, cudaStream_t st);
int launch_pack_fp32(const float* X, const int32_t* perm, const SegDesc* seg, int nseg,
                     const double* mean, int d, int dpad, int64_t npacked, float* A32, float* sq32,
                     QStat* qs, KeyMax* km, cudaStream_t st);
// locality order (order.cu): perm[p] for every packed row, cells of a sample permuted so that
// near cells are near in packed order; levels = 0 gives the identity order
size_t order_workspace_bytes(int64_t npacked);
int launch_order(const float* X, int d, const SegDesc* seg, int nseg, int64_t npacked, int levels,
                 int leaf, int32_t* perm, void* ws, size_t ws_bytes, cudaStream_t st);
size_t scan_i32_scratch_elems(int64_t n);
int scan_excl_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* scratch, cudaStream_t st);
int launch_single_segment(SegDesc* seg, int64_t n, cudaStream_t st);
// one work item per `rows` (128 or 256) query rows of every sample
int launch_build_items(const SegDesc* seg, int nseg, int64_t n_items, int rows, WorkItem* items,
                       Ctl* ctl, cudaStream_t st);

// ---- knn_fp32.cu ----
int launch_knn_fp32(const float* A32, const float* sq32, int d, int dpad, const WorkItem* items,
                    int64_t n_items, const int32_t* perm, Ctl* ctl, int kprime,
                    int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st);

// ---- knn_tc.cu ----
struct TcConfig {
  int bn;        // key tile rows (32, 64, 128, 256)
  int stages;    // smem pipeline depth of the key tiles
  int kpl;       // selector list length (32 / 64)
  int cb;        // selector buffer (16 / 32)
  int epi;       // epilogue warps: 4 (one per TMEM lane quarter) or 8 (two, splitting the columns)
  int pair;      // 1: CTA pairs (cta_group::2, M=256, each CTA stages half of every key tile)
};
bool tc_config_ok(const TcConfig& c, int kp, int kprime);
int launch_wait_selftest(uint64_t limit_ns, int32_t* out, cudaStream_t st);
int tc_counters(unsigned long long* out, int max);
int tc_counters_clear();
bool profiling_enabled();
TcConfig tc_default_config(int prec, int d, int kprime);
int launch_knn_tc(int prec, const TcConfig& cfg, const void* Aop, const void* Bop,
                  int64_t a_rows, int64_t b_rows, int kp, int kmma, const WorkItem* items,
                  int64_t n_items, const int32_t* perm, const int32_t* qmap,
                  const int32_t* n_items_dev, int32_t* counter, Ctl* ctl, int kprime,
                  int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st);

// ---- rerank.cu ----
int launch_rerank(const float* X, int d, const int32_t* perm, const SegDesc* seg, int nseg,
                  int64_t npacked,
                  const int32_t* cand_idx, const float* cand_thr, int cand_stride, int kprime,
                  const QStat* qs, const KeyMax* km, int prec, int kmma, int k, int cosine,
                  int32_t* knn_idx, float* knn_dist, int32_t* fail_rows, Ctl* ctl,
                  const int32_t* rows, const int32_t* nrows, int64_t max_rows,
                  int32_t* fail_flags, cudaStream_t st);
// refine plan: compact the flagged packed rows (sorted) into qmap, count them (ctl->n_refine)
// and cut them into per-sample query tiles (items, ctl->n_items_refine); S: npacked+1 int64
int launch_refine_plan(const int32_t* flags, int64_t npacked, const SegDesc* seg, int nseg,
                       int32_t* qmap, WorkItem* items, int64_t* S, int64_t* scan_scratch,
                       Ctl* ctl, cudaStream_t st);
int launch_all_rows_fail(const int32_t* perm, int64_t npacked, int32_t* fail_rows, Ctl* ctl,
                         cudaStream_t st);
int launch_fp64_scan(const float* X, int d, const int32_t* perm, const SegDesc* seg, int nseg,
                     const int32_t* fail_rows, int64_t max_rows, int k, int cosine,
                     int32_t* knn_idx, float* knn_dist, Ctl* ctl, cudaStream_t st);

// ---- umap.cu ----
int launch_smooth_knn(const float* dist, int64_t n, int k, float local_connectivity,
                      float* sigma, float* rho, double* gsum, cudaStream_t st);
int launch_membership(const int32_t* idx, const float* dist, const float* sigma,
                      const float* rho, int64_t n, int k, float* w, cudaStream_t st);
int launch_distances_csr(const int32_t* idx, const float* dist, int64_t n, int k,
                         int64_t* indptr, int32_t* indices, float* data, cudaStream_t st);
int launch_gauss_sigma(const float* dist, int64_t n, int k, double* sig2, cudaStream_t st);

// ---- fuzzy.cu ----
size_t union_workspace_bytes(int64_t n, int k);
// mode 0: umap fuzzy union of memberships w; mode 1: gauss kernel from distances + sig2
int launch_union(int mode, const int32_t* idx, const float* vals, const double* sig2,
                 int64_t n, int k, int64_t* indptr, int32_t* indices, float* data,
                 int64_t* nnz_dev, void* ws, size_t ws_bytes, cudaStream_t st);

}  // namespace msc
