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

// operand scale f (a power of two): FP16 keeps max Σ z² at or below 2^14, the others use 1
__device__ __forceinline__ double op_scale(int prec, const Ctl* ctl) {
  if (prec != PREC_FP16) return 1.0;
  float mx = __uint_as_float(ctl->max_sq_bits);
  if (!(mx > 0.f)) return 1.0;
  int e = int(floor(0.5 * log2(16384.0 / double(mx))));
  e = max(-60, min(60, e));
  return ldexp(1.0, e);
}

// Bound on |v̂ − v| for query row q against any key (z-space): v = |z_y|² − 2 z_x·z_y exactly, v̂
// what the candidate kernel computes from the rounded operands.  Covers the operand residuals
// (Cauchy–Schwarz), the norm-split error, the FP32 accumulation of kmma products (or of the FP32
// SIMT dot product) and an FP64 slack.
__device__ __forceinline__ double cert_eps(const QStat& q, const KeyMax& km, int prec, int kmma,
                                           int d) {
  const double Kh = __uint_as_float(km.hi), Kl = __uint_as_float(km.lo);
  const double Kr = __uint_as_float(km.res), Kn = __uint_as_float(km.nerr);
  const double Ks = __uint_as_float(km.sq);
  const double qh = q.hi, ql = q.lo, qr = q.res;
  const double dot_err = ql * Kl + (qh + ql) * Kr + qr * (Kh + Kl) + qr * Kr;
  double acc_err;
  if (prec == PREC_FP32)
    acc_err = 0x1p-23 * ((2.0 * d + 4.0) * qh * Kh + 2.0 * Ks);
  else
    acc_err = double(kmma) * 0x1p-22 * (2.0 * (qh + ql) * (Kh + Kl) + Ks);
  return 2.0 * dot_err + Kn + acc_err + 0x1p-40 * (q.sq + Ks);
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
// leaf_out (optional): per packed position, the first position of its leaf (-1: padding)
size_t order_workspace_bytes(int64_t npacked, int d, int leaf);
// the tree runs on the rows projected onto ORDER_PROJ_D random sign directions when d is larger
constexpr int ORDER_PROJ_D = 16;
int launch_project(const float* X, int64_t n, int d, float* Y, cudaStream_t st);
// max_seg: the largest sample (the extra 2-means steps run only on levels whose nodes are large)
// Xp (optional): the rows projected onto dp dimensions, used from level proj_from on
int launch_order(const float* X, int d, const SegDesc* seg, int nseg, int64_t npacked, int levels,
                 int leaf, int32_t* perm, int32_t* leaf_out, void* ws, size_t ws_bytes,
                 cudaStream_t st, int64_t max_seg, const float* Xp = nullptr, int dp = 0,
                 int proj_from = 0);
size_t scan_i32_scratch_elems(int64_t n);
int scan_excl_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* scratch, cudaStream_t st);
int launch_single_segment(SegDesc* seg, int64_t n, cudaStream_t st);
// one work item per `rows` (128 or 256) query rows of every sample
int launch_build_items(const SegDesc* seg, int nseg, int64_t n_items, int rows, WorkItem* items,
                       Ctl* ctl, cudaStream_t st);

// ---- prune.cu ----
constexpr int32_t OUTLIER_LEAF = -2;   // leaf id of the rows moved to the end of their sample
struct PruneWs {
  int32_t* leaf;      // locality-tree leaf per packed position (near-pass layout)
  int32_t* leaf2;     // the same after the partition
  int32_t* perm2;
  int32_t* reg;
  int64_t* S;
  int64_t* scan_scratch;
  double* rpos;       // R per packed position
  double* rpos2;
  double* mean;       // per sample
  double2* mean_part; // per sample and slice: partial sums of R and counts
  float *qc, *qr;     // 128-row balls: centres [npacked/128][d], radii
  float *kc, *kr;     // 256-row balls
  float *sc, *sr;     // two balls per 32-row block
  double* rsub;       // max R per 32-row block
  uint32_t* mask;     // visit bits per work item
  uint32_t* mask3;    // visit bits per work item of the refine pass
  float* seed;        // per packed row (final layout): bound on its final k'-th value
  float* cand_val;    // n × k' near-pass candidate values
  int32_t* iperm;     // original row -> packed position (final layout)
  int4* excl;         // per packed row (final layout): the key ranges the near pass scored
  int2* part;         // refine split: k' (value, row) per row per work item
  float* part_thr;
  int max_split_items;
  // sorted visit lists of the main scan (see VisitOrder)
  double* roff;       // per packed row (final layout): |z|² + 3·eps
  int32_t* vcnt;      // per work item: kept far tiles
  int64_t* voff;      // per work item: first entry (n_items + 1)
  int64_t* vscan;     // scan scratch over the work items
  unsigned long long* vlist;
  int64_t vcap;       // entries vlist holds
  int32_t* claim;      // main-scan claim order of the work items (costliest first)
  int32_t* chist;      // its bucket counts / offsets
};
int prune_mask_words(int64_t max_seg, int bn);
PruneWs carve_prune(Carver& c, int64_t npacked, int nseg, int d, int64_t n_items, int words,
                    int64_t n, int kprime);
// after the near pass (key tiles of bn rows): R per row, outliers to the end of each sample
// (perm is rewritten), the inverse permutation and every row's near-pass key ranges
int launch_prune_partition(const float* X, int d, const SegDesc* seg, int nseg, int64_t npacked,
                           int32_t* perm, const float* cand_thr, const QStat* qs,
                           const KeyMax* km, int prec, int kmma, int bn, const PruneWs& w,
                           cudaStream_t st);
// balls of the final layout and the visit mask of every work item
int launch_prune_plan(const float* X, int d, int64_t npacked, const int32_t* perm,
                      const WorkItem* items, int64_t n_items, int bn, const Ctl* ctl, int prec,
                      const PruneWs& w, int words, cudaStream_t st);
// sorted visit lists of the main scan from the plan's masks (after launch_prune_plan): false in
// *built when the shape does not allow them (the mask walk is used)
// the main scan's claim order (PruneWs::claim): work items by their kept far tiles, most first
int launch_claim_order(int64_t n_items, int words, const PruneWs& w, cudaStream_t st);
int launch_visit_order(const WorkItem* items, int64_t n_items, int bn, int d, int64_t npacked,
                       const int32_t* perm, const Ctl* ctl, Ctl* ctl_w, int prec, int kmma,
                       const QStat* qs, const KeyMax* km, const PruneWs& w, int words,
                       cudaStream_t st, bool* built);
// visit masks of the refine pass's work items (from the main pass's masks)
int launch_refine_mask(const WorkItem* items3, const int32_t* n_items3, const int32_t* qmap,
                       int64_t max_items, const SegDesc* seg, int nseg, int bn, int words,
                       const QStat* qs, const KeyMax* km, const QStat* qs3, const KeyMax* km3,
                       const Ctl* ctl, int prec, int kmma, int kmma3, int d, const PruneWs& w,
                       cudaStream_t st);
// after a split refine pass: every refine row's k' smallest of its work items' lists
int launch_refine_merge(const WorkItem* items3, const int32_t* n_items3, const Ctl* ctl,
                        const int32_t* qmap, const int32_t* perm, int64_t max_rows,
                        const PruneWs& w, int kprime, int32_t* cand_idx, float* cand_thr,
                        cudaStream_t st);
constexpr int REFINE_SPLIT = 8;
int prune_counters(unsigned long long* out);
int prune_counters_clear();

// ---- knn_fp32.cu ----
// the FP32 SIMT form under a pruning plan: a near pass (own 256-key tile only), or a main pass
// over the near 256-key tiles and the mask's far ones with per-row seeds; counter: the launch's
// work-item counter (zeroed by the launcher)
struct FpPrune {
  const uint32_t* mask;
  int words;
  bool near_only;
  const float* seed;
  int32_t* counter;
};
int launch_knn_fp32(const float* A32, const float* sq32, int d, int dpad, const WorkItem* items,
                    int64_t n_items, const int32_t* perm, Ctl* ctl, int kprime,
                    int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st,
                    const FpPrune* prune = nullptr);

// The near pass's candidates handed to the main pass: the near pass writes val (and the usual
// candidate rows); the main pass loads them as every row's starting list and never offers the
// keys the near pass scored again (excl: two packed-position ranges per row).
struct NearInit {
  float* val;              // n × k' values
  const int32_t* idx;      // n × k' original rows (the near pass's candidate rows)
  const int32_t* iperm;    // original row -> packed position of the main pass
  const int4* excl;        // per packed row of the main pass: [x, y) and [z, w)
};

// The refine pass split over key ranges (prune.cu): split_dev (device int) work items per refine
// item; each writes its rows' lists to part (k' entries per row) and part_thr, merged afterwards.
struct RefineSplit {
  const int32_t* split_dev;
  int2* part;
  float* part_thr;
};

// Main scan after a pruning plan: every work item's kept far key tiles, nearest (by ball centres)
// first, each entry carrying a stop bound (bound bits << 32 | key tile): a lower bound on the
// squared operand-space distance between the query tile's rows and the keys of that tile and of
// every later tile (-inf: the list is unsorted and never ends a walk).  The producer walks the
// near tiles and then this list, and ends the item's walk at the first entry whose bound exceeds
// every row's current radius R = threshold + roff.
struct VisitOrder {
  const unsigned long long* list;
  const int64_t* off;
  const double* roff;
  const int32_t* ok;      // device flag: the lists were built (else the mask walk)
};

// ---- knn_tc.cu ----
// Work items are claimed dynamically by the persistent CTAs, in index order or (reverse) from the
// last one down.  Batches pack their largest samples first, so index order starts the longest
// items first; a single pruned sample keeps its costliest query tiles (the outlier rows, scanned
// against every key) at its end, so it claims in reverse.
struct TcConfig {
  int bn;        // key tile rows (32, 64, 128, 256)
  int stages;    // smem pipeline depth of the key tiles
  int kpl;       // slots of the per-row candidate list (32 / 48 / 64), >= k'
  int cb;        // 16 or 32; kept in the tile code for compatibility, no longer used
  int epi;       // epilogue warps: 4 (one per TMEM lane quarter) or 8 (two, splitting the columns)
  int pair;      // 1: CTA pairs (cta_group::2, M=256, each CTA stages half of every key tile)
  // CTAs per SM: 1, or 2 (one accumulator and one query buffer each, at most 128 registers per
  // thread), so that every scheduler runs two epilogue warps of different rows
  int ctas = 1;
};
bool tc_config_ok(const TcConfig& c, int kp, int kprime);
int list_slots(int kprime);
int launch_wait_selftest(uint64_t limit_ns, int32_t* out, cudaStream_t st);
int tc_counters(unsigned long long* out, int max);
int tc_counters_clear();
bool profiling_enabled();
TcConfig tc_default_config(int prec, int d, int kprime);
int launch_knn_tc(int prec, const TcConfig& cfg, const void* Aop, const void* Bop,
                  int64_t a_rows, int64_t b_rows, int kp, int kmma, const WorkItem* items,
                  int64_t n_items, const int32_t* perm, const int32_t* qmap,
                  const int32_t* n_items_dev, int32_t* counter, Ctl* ctl, int kprime,
                  int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st,
                  const uint32_t* mask = nullptr, int mask_words = 0, bool near_only = false,
                  bool reverse = false, const float* seed = nullptr,
                  const NearInit* init = nullptr, const RefineSplit* split = nullptr,
                  const VisitOrder* order = nullptr, const int32_t* claim = nullptr);

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
// split > 1: when there are at most max_split_items refine items, each becomes `split` work
// items over key ranges (ctl->refine_split, ctl->n_items_refine_eff)
int launch_refine_plan(const int32_t* flags, int64_t npacked, const SegDesc* seg, int nseg,
                       int32_t* qmap, WorkItem* items, int64_t* S, int64_t* scan_scratch,
                       Ctl* ctl, int split, int max_split_items, cudaStream_t st);
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
// ---- handoff.cu ----
size_t umap_edges_workspace_bytes(int64_t n);
int launch_umap_edges(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n,
                      int n_epochs, int64_t* out_ptr, int32_t* rows, int32_t* cols,
                      float* weights, double* eps, void* ws, cudaStream_t st);
size_t union_workspace_bytes(int64_t n, int k);
// mode 0: umap fuzzy union of memberships w; mode 1: gauss kernel from distances + sig2
int launch_union(int mode, const int32_t* idx, const float* vals, const double* sig2,
                 int64_t n, int k, int64_t* indptr, int32_t* indices, float* data,
                 int64_t* nnz_dev, void* ws, size_t ws_bytes, cudaStream_t st);


// ---- bbknn.cu ----
// batch-balanced kNN (neighbors.py:491-559): plan from the per-batch cell counts
struct BbPlan {
  int64_t n;
  int d, nb, kwb, prec;
  int K;              // Σ_b min(kwb, n_b): entries per cell
  int kk_max;
  int64_t p1;         // key rows (batches, each padded to SEG_PAD)
  int64_t npk;        // p1 + the query region
  int64_t max_nb;
  int64_t ntiles;     // 128-cell query tiles
  bool candidates;    // tensor-core candidates + certificate, else the FP64 scan for every cell
  int kprime;
  OpLayout L;
  TcConfig cfg;
};
struct BbWs {
  Ctl* ctl;
  KeyMax* km;
  SegDesc* seg;
  int32_t* nfail;
  int32_t* counters;
  int32_t* perm;
  int32_t* qmap;
  int32_t* flag;
  int64_t* S;
  int64_t* scan;
  int32_t* fail_rows;
  double* mean;
  double* partial;
  void* Aop;
  void* Bop;
  QStat* qs;
  WorkItem* items;
  int32_t* cand_idx;
  float* cand_thr;
};
BbPlan bb_plan(int64_t n, int d, const int64_t* counts, int nb, int kwb, int prec);
size_t bb_carve(const BbPlan& P, void* base, BbWs& w);
size_t bb_workspace_bytes(const BbPlan& P);
int run_bbknn(const BbPlan& P, const BbWs& w, const float* X, const int32_t* codes,
              const int64_t* counts, int32_t* knn_idx, float* knn_dist, cudaStream_t st);
size_t bb_distances_workspace_bytes(int64_t n);
int launch_bb_distances(const int32_t* idx, const float* dist, int64_t n, int K, int64_t* indptr,
                        int32_t* indices, float* data, void* ws, cudaStream_t st);
size_t trim_workspace_bytes(int64_t n);
int launch_trim(const int64_t* indptr, const int32_t* indices, const float* data, int64_t n,
                int trim, int64_t* out_ptr, int32_t* out_idx, float* out_data, void* ws,
                cudaStream_t st);
// ---- spatial.cu ----
size_t spatial_knn_workspace_bytes(int64_t n);
int launch_spatial_knn(const float* X, int64_t n, int d, int k, int32_t* idx, float* dist,
                       int64_t* stats, void* ws, cudaStream_t st);
size_t spatial_radius_workspace_bytes(int64_t n);
int launch_spatial_radius_count(const float* X, int64_t n, int d, double radius, double min_radius,
                                int64_t* indptr, int64_t* stats, void* ws, cudaStream_t st);
size_t spatial_radius_fill_scratch_bytes(int64_t nnz);
int launch_spatial_radius_fill(int64_t n, int d, double radius, double min_radius,
                               const int64_t* indptr, int64_t nnz, int32_t* cols, float* dist,
                               void* ws, void* scratch, cudaStream_t st);
int launch_spatial_edge_lengths(const double* X, int64_t n, int d, const int64_t* indptr,
                                const int32_t* cols, double* out, cudaStream_t st);

}  // namespace msc
