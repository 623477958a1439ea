// C ABI of the library: argument checks, workspace layout and the stream-ordered pipelines.
//
//   msc_neighbors  = kNN + distances CSR + connectivities   (metalsinglecell neighbors.py:727-760)
//   msc_knn        = kNN only                                (neighbors.py:698-724 / 82-132)
//   msc_batched_*  = kNN of many samples in one persistent launch
//   msc_smooth_knn_dist / msc_membership / msc_fuzzy_union / msc_gauss_connectivities /
//   msc_distances_csr = the individual graph stages
//   msc_bbknn_*    = batch-balanced kNN lists, their distances graph, and the trimming of the
//                    connectivities                     (neighbors.py:491-559, 465-488)
//
// Nothing here allocates device memory: every buffer is carved out of the caller's workspace.
#include <map>
#include <mutex>
#include <tuple>
#include <vector>
#include <algorithm>
#include <unordered_map>

#include <cstdlib>

#include <nvtx3/nvToolsExt.h>

#include "kernels.cuh"

namespace msc {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}
const char* last_error() { return g_err.c_str(); }

std::atomic<long long> g_launch_count{0};

// ---- stage timing: events recorded between pipeline stages when enabled ----
namespace {
constexpr int MAX_MARKS = 16;
struct StageTimer {
  bool on = false;
  cudaEvent_t ev[MAX_MARKS] = {};
  int last = -1;           // highest mark recorded in the current call
  std::mutex mu;
};
StageTimer& timer() {
  static StageTimer t;
  return t;
}
}  // namespace

bool profiling_enabled() { return timer().on; }

// NVTX ranges over the same stages, on the host timeline (the enqueue of each stage), for users
// of Nsight tools; with no tool attached the calls return at once.  A mark ends the previous
// stage's range and opens the next one's; the entry points close what is left open.
namespace {
const char* const kStageNames[] = {"msc: prep",
                                   "msc: near pass",
                                   "msc: pruning plan",
                                   "msc: candidates",
                                   "msc: re-rank + FP64 scan",
                                   "msc: CSR + rho/sigma + memberships",
                                   "msc: fuzzy union"};
constexpr int N_STAGE_NAMES = int(sizeof(kStageNames) / sizeof(kStageNames[0]));
thread_local nvtxRangeId_t g_range = 0;
thread_local bool g_range_open = false;

void stage_range_close() {
  if (g_range_open) {
    nvtxRangeEnd(g_range);
    g_range_open = false;
  }
}

// closes the open stage range when an entry point returns, on every path
struct StageRangeGuard {
  ~StageRangeGuard() { stage_range_close(); }
};
}  // namespace

void stage_mark(cudaStream_t st, int stage) {
  stage_range_close();
  if (stage >= 0 && stage < N_STAGE_NAMES) {
    g_range = nvtxRangeStartA(kStageNames[stage]);
    g_range_open = true;
  }
  StageTimer& t = timer();
  if (!t.on || stage < 0 || stage >= MAX_MARKS) return;
  if (!t.ev[stage] && cudaEventCreate(&t.ev[stage]) != cudaSuccess) return;
  cudaEventRecord(t.ev[stage], st);
  if (stage == 0) t.last = 0;
  else t.last = std::max(t.last, stage);
}

int num_sms() {
  static std::mutex mu;
  static std::unordered_map<int, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int v = 148;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) v = 148;
  cache[dev] = v;
  return v;
}

cudaError_t raise_smem_cap_fn(const void* func, size_t bytes) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, func);
  if (e != cudaSuccess) return e;
  if (fa.maxDynamicSharedSizeBytes >= 0 && size_t(fa.maxDynamicSharedSizeBytes) >= bytes)
    return cudaSuccess;
  return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
}

int resident_blocks_fn(const void* func, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  const auto key = std::make_tuple(func, dev, threads, smem);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int v = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, func, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    v = 1;
  }
  v = std::max(1, v);
  cache[key] = v;
  return v;
}

namespace {

constexpr int COLMEAN_NB = 256;

struct Problem {
  int64_t n = 0;          // total cells
  int d = 0, k = 0, metric = 0, prec = 0, kprime = 0;
  int nseg = 1;
  int64_t npacked = 0;    // packed rows
  int64_t ntiles = 0;     // 128-row query tiles
  int64_t nptiles = 0;    // 256-row query tiles (CTA-pair work items)
  int64_t max_seg = 0;
  bool candidates = true; // false: every row takes the FP64 scan (k-1 > 64)
  OpLayout L{};
  int dpad = 0;
  // refine pass (one-term FP16/BF16 candidates): rows that fail the certificate re-run through
  // the BF16x3 candidate kernel before the FP64 scan takes what is left
  bool refine = false;
  OpLayout L3{};
  // key-tile pruning of the tensor-core scan (prune.cu): workspace carved, mask words per item
  bool prune = false;
  int prune_words = 0;
};

struct KnnWs {
  Ctl* ctl;
  KeyMax* km;
  SegDesc* seg;
  WorkItem* items;
  double* mean;
  double* partial;
  float* Xn;
  void* Aop;
  void* Bop;
  float* A32;
  float* sq32;
  QStat* qs;
  int32_t* cand_idx;
  float* cand_thr;
  int32_t* fail_rows;
  int32_t* perm;          // packed row -> original row (-1: padding)
  float* Xo;              // the rows projected for the locality order (d > ORDER_PROJ_D)
  void* order_ws;
  size_t order_ws_bytes;
  // refine pass
  int32_t* flags;         // per packed row: failed the first certificate
  int64_t* S;             // scan of flags (npacked + 1)
  int64_t* scan_scratch;
  int32_t* qmap;          // refine query row -> packed row
  WorkItem* items3;
  void* A3;               // BF16x3 query operand of the listed rows
  void* B3;               // BF16x3 key operand of every packed row
  QStat* qs3;
  KeyMax* km3;
  PruneWs pr;
};

int default_kprime(int prec, int k) {
  // over-fetch sized to each precision's certificate.  FP32 and the three-term BF16 split have
  // error bounds far below typical neighbour gaps, but the k'-th candidate must still clear the
  // k-th neighbour by the bound: at 1.3M cells k' = k+8 left ~0.04% of the rows to the FP64 scan,
  // k' = 32 none.  One-term FP16/BF16 need a wider margin.
  if (prec == PREC_FP32) return std::min(64, std::max(k - 1, k + 8));
  if (prec == PREC_BF16X3) return std::min(64, std::max(32, k + 8));
  return std::min(64, std::max(48, k + 15));
}

int check_common(int64_t n, int d, int k, int metric, int prec, int kprime,
                 int max_k = MSC_MAX_K) {
  if (n < 1 || n >= (int64_t(1) << 30)) { set_error("n=%lld out of range", (long long)n); return MSC_ERR_INVALID_ARG; }
  if (d < 1 || d > MSC_MAX_D) { set_error("d=%d must be in [1, %d]", d, MSC_MAX_D); return MSC_ERR_INVALID_ARG; }
  if (k < 1) { set_error("n_neighbors=%d must be at least 1", k); return MSC_ERR_INVALID_ARG; }
  if (k > max_k) {
    // a valid request (any k <= n is), above the widest list the kernels keep
    set_error("n_neighbors=%d is above the supported %d", k, max_k);
    return MSC_ERR_UNSUPPORTED;
  }
  if (metric != MSC_METRIC_EUCLIDEAN && metric != MSC_METRIC_COSINE) { set_error("unknown metric %d", metric); return MSC_ERR_INVALID_ARG; }
  if (prec < 0 || prec > 3) { set_error("unknown precision %d", prec); return MSC_ERR_INVALID_ARG; }
  if (kprime != 0 && (kprime < k - 1 || kprime > 64)) {
    set_error("kprime=%d must be 0 or in [n_neighbors-1=%d, 64]", kprime, k - 1);
    return MSC_ERR_INVALID_ARG;
  }
  return MSC_OK;
}

// key-tile pruning: samples from this size on, key tiles of this many rows, mask size cap
constexpr int64_t PRUNE_MIN_CELLS = 4096;
constexpr int PRUNE_BN = 256;
constexpr int64_t PRUNE_MASK_MAX = int64_t(2) << 30;

int make_problem(Problem& P, int64_t n, int d, int k, int metric, int prec, int kprime,
                 const int64_t* offsets, int nseg, int max_k = MSC_MAX_K) {
  MSC_TRY(check_common(n, d, k, metric, prec, kprime, max_k));
  P.n = n; P.d = d; P.k = k; P.metric = metric; P.prec = prec;
  P.kprime = kprime ? kprime : default_kprime(prec, k);
  P.candidates = (k - 1) <= 64;
  if (P.candidates) P.kprime = std::max(P.kprime, k - 1);
  P.nseg = nseg;
  P.L = op_layout(prec, d);
  P.dpad = int(round_up(d, 4));
  if (offsets) {
    if (offsets[0] != 0 || offsets[nseg] != n) { set_error("offsets must run from 0 to n"); return MSC_ERR_INVALID_ARG; }
    P.npacked = 0; P.ntiles = 0; P.nptiles = 0; P.max_seg = 0;
    for (int s = 0; s < nseg; ++s) {
      const int64_t ns = offsets[s + 1] - offsets[s];
      if (ns < k) { set_error("sample %d has %lld cells < n_neighbors=%d", s, (long long)ns, k); return MSC_ERR_INVALID_ARG; }
      P.npacked += round_up(ns, SEG_PAD);
      P.ntiles += ceil_div(ns, QTILE);
      P.nptiles += ceil_div(ns, 2 * QTILE);
      P.max_seg = std::max(P.max_seg, ns);
    }
  } else {
    if (n < k) { set_error("n_neighbors=%d > n=%lld", k, (long long)n); return MSC_ERR_INVALID_ARG; }
    P.npacked = round_up(n, SEG_PAD);
    P.ntiles = ceil_div(n, QTILE);
    P.nptiles = ceil_div(n, 2 * QTILE);
    P.max_seg = n;
  }
  if (P.npacked >= (int64_t(1) << 31)) { set_error("too many packed rows"); return MSC_ERR_UNSUPPORTED; }
  if (P.candidates && prec != PREC_FP32) {
    TcConfig c = tc_default_config(prec, d, P.kprime);
    if (!tc_config_ok(c, P.L.kp, P.kprime)) {
      // the operand row is too wide for a resident query tile at this precision: the FP32
      // candidate kernel takes over (the result is exact either way; MSC_STAT_PRECISION says)
      P.prec = PREC_FP32;
      P.kprime = kprime ? kprime : default_kprime(PREC_FP32, k);
      P.kprime = std::max(P.kprime, k - 1);
      P.L = op_layout(PREC_FP32, d);
    }
  }
  if (P.candidates && k > 1 && (P.prec == PREC_FP16 || P.prec == PREC_BF16)) {
    P.L3 = op_layout(PREC_BF16X3, d);
    P.refine = tc_config_ok(tc_default_config(PREC_BF16X3, d, P.kprime), P.L3.kp, P.kprime);
  }
  // Pruning pays once a sample spans many key tiles beyond the near ones; its mask (one bit per
  // 256-key tile per 128-row query tile) is capped at 2 GB.  MSC_B200_PRUNE=0 turns it off.  The
  // plain FP32 form scans every key unless MSC_B200_PRUNE_FP32=1 (the same plan, for comparing
  // the forms at equal pruning).
  const char* env32 = std::getenv("MSC_B200_PRUNE_FP32");
  const bool prune32 = env32 && *env32 == '1';
  if (P.candidates && k > 1 && (P.prec != PREC_FP32 || prune32) &&
      P.max_seg >= PRUNE_MIN_CELLS) {
    const char* env = std::getenv("MSC_B200_PRUNE");
    const int words = prune_mask_words(P.max_seg, PRUNE_BN);
    if (!(env && *env == '0') && double(P.ntiles) * words * 4.0 <= double(PRUNE_MASK_MAX)) {
      P.prune = true;
      P.prune_words = words;
    }
  }
  return MSC_OK;
}

// leaves of the locality tree (order.cu) hold at most this many rows
constexpr int ORDER_LEAF = 256;
// first tree level on the projected rows: the levels above split the sample between clusters, and
// there the exact rows keep whole clusters together.  Measured at 1.3M × 50 (graph / far key tiles
// kept): exact rows throughout 72.3 ms / 2.63 M; projected from level 10 70.95 ms / 2.79 M, from
// level 8 71.07 ms / 2.84 M, every level 76.0 ms / 3.91 M.
constexpr int ORDER_PROJ_FROM = 10;

KnnWs carve_knn(Carver& c, const Problem& P) {
  KnnWs w{};
  w.ctl = c.take<Ctl>(1);
  w.km = c.take<KeyMax>(1);
  w.seg = c.take<SegDesc>(P.nseg);
  w.items = c.take<WorkItem>(P.ntiles);
  w.mean = c.take<double>(size_t(P.nseg) * P.d);
  w.partial = c.take<double>(colmean_partial_elems(P.nseg, P.d, COLMEAN_NB));
  w.Xn = P.metric == MSC_METRIC_COSINE ? c.take<float>(size_t(P.n) * P.d) : nullptr;
  if (P.prec == PREC_FP32) {
    w.A32 = c.take<float>(size_t(P.npacked) * P.dpad);
    w.sq32 = c.take<float>(P.npacked);
  } else {
    w.Aop = c.take<uint16_t>(size_t(P.npacked) * P.L.kp);
    w.Bop = c.take<uint16_t>(size_t(P.npacked) * P.L.kp);
  }
  w.qs = c.take<QStat>(P.npacked);
  w.cand_idx = c.take<int32_t>(size_t(P.n) * P.kprime);
  w.cand_thr = c.take<float>(P.n);
  w.fail_rows = c.take<int32_t>(P.n);
  w.perm = c.take<int32_t>(P.npacked);
  // the order's rows: projected when d > ORDER_PROJ_D
  w.Xo = P.d > ORDER_PROJ_D ? c.take<float>(size_t(P.n) * ORDER_PROJ_D) : nullptr;
  w.order_ws_bytes = order_workspace_bytes(P.npacked, std::max(P.d, ORDER_PROJ_D), ORDER_LEAF);
  w.order_ws = c.take<unsigned char>(w.order_ws_bytes);
  if (P.refine) {
    w.flags = c.take<int32_t>(P.npacked);
    w.S = c.take<int64_t>(P.npacked + 1);
    w.scan_scratch = c.take<int64_t>(scan_i32_scratch_elems(P.npacked));
    w.qmap = c.take<int32_t>(P.n);
    w.items3 = c.take<WorkItem>(P.ntiles);
    w.A3 = c.take<uint16_t>(size_t(P.n) * P.L3.kp);
    w.B3 = c.take<uint16_t>(size_t(P.npacked) * P.L3.kp);
    w.qs3 = c.take<QStat>(P.npacked);
    w.km3 = c.take<KeyMax>(1);
  }
  if (P.prune)
    w.pr = carve_prune(c, P.npacked, P.nseg, P.d, P.ntiles, P.prune_words, P.n, P.kprime);
  return w;
}

// Levels of the locality tree (order.cu) for the tensor-core path: enough halvings to bring the
// largest sample to leaves of ORDER_LEAF rows, plus slack for uneven splits.  The FP32 SIMT kernel
// scans keys in plain order, so it keeps the identity order.  MSC_B200_ORDER=0 turns it off.
int order_levels(const Problem& P, bool tc) {
  if (!tc || P.max_seg <= 2 * ORDER_LEAF) return 0;
  const char* env = std::getenv("MSC_B200_ORDER");
  if (env && *env == '0') return 0;
  int l = 0;
  while ((int64_t(ORDER_LEAF) << l) < P.max_seg) ++l;
  // uneven 2-means splits leave some nodes above the leaf size after l levels; four more levels
  // split them (MSC_B200_ORDER_EXTRA overrides the four: tuning)
  int extra = 4;
  if (const char* e = std::getenv("MSC_B200_ORDER_EXTRA")) extra = std::max(0, std::atoi(e));
  return std::min(28, l + extra);
}

int decode_tile_config(int32_t code, const Problem& P, TcConfig& cfg) {
  cfg = tc_default_config(P.prec, P.d, P.kprime);
  if (code == 0) {
    // tuning override for the automatic choice (same encoding as tile_config)
    const char* env = std::getenv("MSC_B200_TILE_CONFIG");
    if (env && *env) code = int32_t(std::strtol(env, nullptr, 0));
  }
  if (code == 0) return MSC_OK;
  TcConfig c{code & 0xfff, (code >> 12) & 0xff, list_slots(P.kprime), (code >> 20) & 0x7f,
             (code >> 27) & 1 ? 8 : 4, (code >> 28) & 1, (code >> 29) & 1 ? 2 : 1};
  if (!tc_config_ok(c, P.L.kp, P.kprime)) {
    set_error("tile_config 0x%x (bn=%d stages=%d cb=%d epi=%d pair=%d ctas=%d) is not valid here",
              code, c.bn, c.stages, c.cb, c.epi, c.pair, c.ctas);
    return MSC_ERR_INVALID_ARG;
  }
  cfg = c;
  return MSC_OK;
}

int launch_set_stat(Ctl* ctl, int idx, int64_t v, cudaStream_t st);

// The kNN pipeline after the sample table (w.seg) is in place.
int run_knn(const Problem& P, const KnnWs& w, const float* X, int32_t* knn_idx, float* knn_dist,
            int32_t tile_code, cudaStream_t st) {
  stage_mark(st, 0);
  MSC_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(Ctl), st));
  MSC_CUDA_TRY(cudaMemsetAsync(w.km, 0, sizeof(KeyMax), st));
  MSC_TRY(launch_set_stat(w.ctl, MSC_STAT_PRECISION, P.candidates ? P.prec : -1, st));
  const bool cosine = P.metric == MSC_METRIC_COSINE;
  const float* Xu = X;
  if (cosine) {
    MSC_TRY(launch_normalize(X, w.Xn, P.n, P.d, &w.ctl->stats[MSC_STAT_NONFINITE], st));
    Xu = w.Xn;
  }
  const bool tc = P.candidates && P.k > 1 && P.prec != PREC_FP32;
  TcConfig cfg{};
  if (tc) MSC_TRY(decode_tile_config(tile_code, P, cfg));
  const bool pair_items = tc && cfg.pair;
  const int64_t n_items = pair_items ? P.nptiles : P.ntiles;
  MSC_TRY(launch_build_items(w.seg, P.nseg, n_items, pair_items ? 2 * QTILE : QTILE, w.items, w.ctl,
                             st));
  // pruning needs single-CTA work items over 256-key tiles (or the FP32 SIMT kernel)
  const bool prune = P.prune && tc && !cfg.pair && cfg.bn == PRUNE_BN;
  const bool prune32 = P.prune && P.candidates && P.k > 1 && P.prec == PREC_FP32;
  // the tree's lower levels on projected rows (MSC_B200_ORDER_PROJ=<level>: the first level on
  // them, 0 = all, negative = none; tuning)
  const int levels = order_levels(P, tc || prune32);
  int proj_from = ORDER_PROJ_FROM;
  if (const char* pe = std::getenv("MSC_B200_ORDER_PROJ")) proj_from = std::atoi(pe);
  const bool proj = w.Xo && levels > proj_from && proj_from >= 0;
  if (proj) MSC_TRY(launch_project(Xu, P.n, P.d, w.Xo, st));
  MSC_TRY(launch_order(Xu, P.d, w.seg, P.nseg, P.npacked, levels,
                       ORDER_LEAF, w.perm, (prune || prune32) ? w.pr.leaf : nullptr, w.order_ws,
                       w.order_ws_bytes, st, P.max_seg, proj ? w.Xo : nullptr, ORDER_PROJ_D,
                       proj_from));
  if (!P.candidates) {
    MSC_TRY(launch_all_rows_fail(w.perm, P.npacked, w.fail_rows, w.ctl, st));
    MSC_TRY(launch_fp64_scan(Xu, P.d, w.perm, w.seg, P.nseg, w.fail_rows, P.n, P.k, cosine,
                             knn_idx, knn_dist, w.ctl, st));
    return MSC_OK;
  }
  MSC_TRY(launch_colmean(Xu, w.seg, P.nseg, P.max_seg, P.d, w.partial, COLMEAN_NB, w.mean,
                         cosine ? nullptr : &w.ctl->stats[MSC_STAT_NONFINITE], st));
  if (P.k > 1) {
    if (P.prec == PREC_FP32) {
      MSC_TRY(launch_pack_fp32(Xu, w.perm, w.seg, P.nseg, w.mean, P.d, P.dpad, P.npacked, w.A32,
                               w.sq32, w.qs, w.km, st));
      stage_mark(st, 1);
      if (prune32) {
        // the same near pass -> radius -> outliers -> re-pack -> plan as the tensor-core forms
        const FpPrune near{nullptr, 0, true, nullptr, &w.ctl->tc_counter[2]};
        MSC_TRY(launch_knn_fp32(w.A32, w.sq32, P.d, P.dpad, w.items, P.ntiles, w.perm, w.ctl,
                                P.kprime, w.cand_idx, w.cand_thr, P.kprime, st, &near));
        stage_mark(st, 2);
        MSC_TRY(launch_prune_partition(Xu, P.d, w.seg, P.nseg, P.npacked, w.perm, w.cand_thr,
                                       w.qs, w.km, P.prec, P.L.kmma, PRUNE_BN, w.pr, st));
        MSC_CUDA_TRY(cudaMemsetAsync(w.km, 0, sizeof(KeyMax), st));
        MSC_TRY(launch_pack_fp32(Xu, w.perm, w.seg, P.nseg, w.mean, P.d, P.dpad, P.npacked,
                                 w.A32, w.sq32, w.qs, w.km, st));
        const int words32 = prune_mask_words(P.max_seg, PRUNE_BN);
        MSC_TRY(launch_prune_plan(Xu, P.d, P.npacked, w.perm, w.items, P.ntiles, PRUNE_BN, w.ctl,
                                  P.prec, w.pr, words32, st));
        stage_mark(st, 3);
        const FpPrune main32{w.pr.mask, words32, false, w.pr.seed, &w.ctl->tc_counter[0]};
        MSC_TRY(launch_knn_fp32(w.A32, w.sq32, P.d, P.dpad, w.items, P.ntiles, w.perm, w.ctl,
                                P.kprime, w.cand_idx, w.cand_thr, P.kprime, st, &main32));
      } else {
        stage_mark(st, 2);
        stage_mark(st, 3);
        MSC_TRY(launch_knn_fp32(w.A32, w.sq32, P.d, P.dpad, w.items, P.ntiles, w.perm, w.ctl,
                                P.kprime, w.cand_idx, w.cand_thr, P.kprime, st));
      }
    } else {
      if (P.prec == PREC_FP16)
        MSC_TRY(launch_maxnorm(Xu, w.seg, P.nseg, w.mean, P.d, P.npacked, w.ctl, st));
      MSC_TRY(launch_pack_tc(P.prec, Xu, w.perm, w.seg, P.nseg, w.mean, P.d, P.npacked,
                             nullptr, nullptr, 0, w.Aop, w.Bop, w.qs, w.km, w.ctl, st));
      stage_mark(st, 1);
      const uint32_t* mask = nullptr;
      int words = 0;
      bool ordered = false;
      const int32_t* claim = nullptr;
      const NearInit init{w.pr.cand_val, w.cand_idx, w.pr.iperm, w.pr.excl};
      if (prune) {
        // near pass -> per-row radius -> outliers to the end of each sample -> operands of the
        // new order -> balls and the visit mask of every query tile
        MSC_TRY(launch_knn_tc(P.prec, cfg, w.Aop, w.Bop, P.npacked, P.npacked, P.L.kp,
                              P.L.kmma, w.items, n_items, w.perm, nullptr, nullptr,
                              &w.ctl->tc_counter[2], w.ctl, P.kprime, w.cand_idx, w.cand_thr,
                              P.kprime, st, nullptr, 0, true, false, nullptr, &init));
        stage_mark(st, 2);
        MSC_TRY(launch_prune_partition(Xu, P.d, w.seg, P.nseg, P.npacked, w.perm, w.cand_thr,
                                       w.qs, w.km, P.prec, P.L.kmma, cfg.bn, w.pr, st));
        MSC_CUDA_TRY(cudaMemsetAsync(w.km, 0, sizeof(KeyMax), st));
        MSC_TRY(launch_pack_tc(P.prec, Xu, w.perm, w.seg, P.nseg, w.mean, P.d, P.npacked,
                               nullptr, nullptr, 0, w.Aop, w.Bop, w.qs, w.km, w.ctl, st));
        words = prune_mask_words(P.max_seg, cfg.bn);
        MSC_TRY(launch_prune_plan(Xu, P.d, P.npacked, w.perm, w.items, n_items, cfg.bn, w.ctl,
                                  P.prec, w.pr, words, st));
        mask = w.pr.mask;
        // MSC_B200_CLAIM_ORDER=0: claim in index order (reversed) instead (tuning)
        const char* co = std::getenv("MSC_B200_CLAIM_ORDER");
        if (!(co && *co == '0')) {
          MSC_TRY(launch_claim_order(n_items, words, w.pr, st));
          claim = w.pr.claim;
        }
        MSC_TRY(launch_visit_order(w.items, n_items, cfg.bn, P.d, P.npacked, w.perm, w.ctl,
                                   w.ctl, P.prec, P.L.kmma, w.qs, w.km, w.pr, words, st,
                                   &ordered));
      } else {
        stage_mark(st, 2);
      }
      stage_mark(st, 3);
      const VisitOrder order{w.pr.vlist, w.pr.voff, w.pr.roff, &w.ctl->ordered_ok};
      MSC_TRY(launch_knn_tc(P.prec, cfg, w.Aop, w.Bop, P.npacked, P.npacked, P.L.kp, P.L.kmma,
                            w.items, n_items, w.perm, nullptr, nullptr, &w.ctl->tc_counter[0],
                            w.ctl, P.kprime, w.cand_idx, w.cand_thr, P.kprime, st, mask, words,
                            false, prune && P.nseg == 1, prune ? w.pr.seed : nullptr,
                            prune ? &init : nullptr, nullptr,
                            ordered ? &order : nullptr, claim));
    }
  }
  stage_mark(st, 4);
  if (P.refine) MSC_CUDA_TRY(cudaMemsetAsync(w.flags, 0, sizeof(int32_t) * P.npacked, st));
  MSC_TRY(launch_rerank(Xu, P.d, w.perm, w.seg, P.nseg, P.npacked, w.cand_idx, w.cand_thr,
                        P.kprime, P.kprime, w.qs, w.km, P.prec, P.L.kmma, P.k, cosine, knn_idx,
                        knn_dist, w.fail_rows, w.ctl, nullptr, nullptr, 0,
                        P.refine ? w.flags : nullptr, st));
  if (P.refine) {
    // the rows the one-term candidates could not certify, again with the three-term split
    // with pruning, a small refine set is split over key ranges (prune.cu)
    const bool split = prune;
    MSC_TRY(launch_refine_plan(w.flags, P.npacked, w.seg, P.nseg, w.qmap, w.items3, w.S,
                               w.scan_scratch, w.ctl, split ? REFINE_SPLIT : 1,
                               split ? w.pr.max_split_items : 0, st));
    MSC_CUDA_TRY(cudaMemsetAsync(w.km3, 0, sizeof(KeyMax), st));
    MSC_TRY(launch_pack_tc(PREC_BF16X3, Xu, w.perm, w.seg, P.nseg, w.mean, P.d, P.npacked,
                           nullptr, nullptr, 0, nullptr, w.B3, w.qs3, w.km3, w.ctl, st));
    MSC_TRY(launch_pack_tc(PREC_BF16X3, Xu, w.perm, w.seg, P.nseg, w.mean, P.d, P.npacked,
                           w.qmap, &w.ctl->n_refine, P.n, w.A3, nullptr, nullptr, nullptr, w.ctl,
                           st));
    const TcConfig cfg3 = tc_default_config(PREC_BF16X3, P.d, P.kprime);
    const uint32_t* mask3 = nullptr;
    int words3 = 0;
    if (prune && !cfg3.pair && cfg3.bn == PRUNE_BN) {
      words3 = prune_mask_words(P.max_seg, cfg3.bn);
      MSC_TRY(launch_refine_mask(w.items3, &w.ctl->n_items_refine, w.qmap, P.ntiles, w.seg,
                                 P.nseg, cfg3.bn, words3, w.qs, w.km, w.qs3, w.km3, w.ctl,
                                 P.prec, P.L.kmma, P.L3.kmma, P.d, w.pr, st));
      mask3 = w.pr.mask3;
    }
    const RefineSplit rs{&w.ctl->refine_split, split ? w.pr.part : nullptr,
                         split ? w.pr.part_thr : nullptr};
    const int64_t max_work = split ? std::max<int64_t>(P.ntiles,
                                                       int64_t(w.pr.max_split_items) * REFINE_SPLIT)
                                   : P.ntiles;
    MSC_TRY(launch_knn_tc(PREC_BF16X3, cfg3, w.A3, w.B3, P.n, P.npacked, P.L3.kp, P.L3.kmma,
                          w.items3, max_work, w.perm, w.qmap, &w.ctl->n_items_refine_eff,
                          &w.ctl->tc_counter[1], w.ctl, P.kprime, w.cand_idx, w.cand_thr,
                          P.kprime, st, mask3, words3, false, false, nullptr, nullptr,
                          split ? &rs : nullptr));
    if (split)
      MSC_TRY(launch_refine_merge(w.items3, &w.ctl->n_items_refine, w.ctl, w.qmap, w.perm, P.n,
                                  w.pr, P.kprime, w.cand_idx, w.cand_thr, st));
    MSC_TRY(launch_rerank(Xu, P.d, w.perm, w.seg, P.nseg, P.npacked, w.cand_idx, w.cand_thr,
                          P.kprime, P.kprime, w.qs3, w.km3, PREC_BF16X3, P.L3.kmma, P.k, cosine,
                          knn_idx, knn_dist, w.fail_rows, w.ctl, w.qmap, &w.ctl->n_refine, P.n,
                          nullptr, st));
  }
  MSC_TRY(launch_fp64_scan(Xu, P.d, w.perm, w.seg, P.nseg, w.fail_rows, P.n, P.k, cosine,
                           knn_idx, knn_dist, w.ctl, st));
  stage_mark(st, 5);
  return MSC_OK;
}

int copy_stats(const KnnWs& w, int64_t* stats_dev, cudaStream_t st) {
  if (stats_dev)
    MSC_CUDA_TRY(cudaMemcpyAsync(stats_dev, w.ctl->stats, sizeof(int64_t) * MSC_STATS_LEN,
                                 cudaMemcpyDeviceToDevice, st));
  return MSC_OK;
}

struct GraphWs {
  float* sigma;
  float* rho;
  float* w;
  double* gsum;
  double* sig2;
  void* uws;
  size_t uws_bytes;
};

GraphWs carve_graph(Carver& c, int64_t n, int k, int method) {
  GraphWs g{};
  if (method == MSC_METHOD_UMAP) {
    g.sigma = c.take<float>(n);
    g.rho = c.take<float>(n);
    g.w = c.take<float>(size_t(n) * k);
    g.gsum = c.take<double>(1 + 1024);
  } else {
    g.sig2 = c.take<double>(n);
  }
  g.uws_bytes = union_workspace_bytes(n, k);
  g.uws = c.take<unsigned char>(g.uws_bytes);
  return g;
}

__global__ void set_stat_kernel(Ctl* ctl, int idx, int64_t v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) ctl->stats[idx] = v;
}
int launch_set_stat(Ctl* ctl, int idx, int64_t v, cudaStream_t st) {
  set_stat_kernel<<<1, 32, 0, st>>>(ctl, idx, v);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

__global__ void store_nnz_kernel(const int64_t* __restrict__ indptr, int64_t n, Ctl* ctl) {
  if (threadIdx.x == 0 && blockIdx.x == 0) ctl->stats[MSC_STAT_CONN_NNZ] = indptr[n];
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

bool bad_ptr(const void* p, const char* name) {
  if (p) return false;
  set_error("%s is NULL", name);
  return true;
}

}  // namespace
}  // namespace msc

using namespace msc;

extern "C" {

int msc_version(void) { return 10000; }
const char* msc_last_error(void) { return msc::last_error(); }

long long msc_launch_count(void) { return msc::g_launch_count.load(); }

int msc_profile_enable(int on) {
  timer().on = on != 0;
  timer().last = -1;
  if (on) {
    MSC_TRY(tc_counters_clear());
    return prune_counters_clear();
  }
  return MSC_OK;
}

int msc_profile_counters(unsigned long long* out, int max_counters) {
  if (!out || max_counters < 1) { set_error("out/max_counters invalid"); return MSC_ERR_INVALID_ARG; }
  MSC_CUDA_TRY(cudaDeviceSynchronize());
  MSC_TRY(tc_counters(out, max_counters));
  unsigned long long pt[5];
  MSC_TRY(prune_counters(pt));
  for (int i = 0; i < 2 && 10 + i < max_counters; ++i) out[10 + i] = pt[i];
  for (int i = 2; i < 5 && 10 + i < max_counters; ++i) out[10 + i] = pt[i];
  return MSC_OK;
}

int msc_profile_read(float* ms_out, int max_stages) {
  StageTimer& t = timer();
  if (!ms_out || max_stages < 1) { set_error("ms_out/max_stages invalid"); return -MSC_ERR_INVALID_ARG; }
  int n = 0;
  for (int s = 1; s <= t.last && n < max_stages; ++s, ++n) {
    float ms = -1.f;
    if (t.ev[s] && t.ev[s - 1]) {
      cudaEventSynchronize(t.ev[s]);
      if (cudaEventElapsedTime(&ms, t.ev[s - 1], t.ev[s]) != cudaSuccess) ms = -1.f;
    }
    ms_out[n] = ms;
  }
  return n;
}

int msc_selftest_wait_timeout(int64_t limit_ns, int32_t* out_dev, void* stream) {
  if (limit_ns < 1000 || limit_ns > int64_t(10) * 1000000000ll || !out_dev) {
    set_error("limit_ns must be in [1 us, 10 s] and out_dev non-NULL");
    return MSC_ERR_INVALID_ARG;
  }
  return launch_wait_selftest(uint64_t(limit_ns), out_dev, as_stream(stream));
}

size_t msc_knn_workspace_bytes(int64_t n, int32_t d, int32_t k, int32_t metric, int32_t precision,
                               int32_t kprime) {
  Problem P;
  if (make_problem(P, n, d, k, metric, precision, kprime, nullptr, 1, MSC_MAX_K_KNN) != MSC_OK)
    return 0;
  Carver c(nullptr);
  carve_knn(c, P);
  return c.bytes();
}

int msc_knn(const float* X_dev, int64_t n, int32_t d, int32_t k, int32_t metric,
            int32_t precision, int32_t kprime, int32_t* knn_idx_dev, float* knn_dist_dev,
            int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream) {
  StageRangeGuard range_guard;
  Problem P;
  MSC_TRY(make_problem(P, n, d, k, metric, precision, kprime, nullptr, 1, MSC_MAX_K_KNN));
  if (bad_ptr(X_dev, "X") || bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  Carver c(workspace);
  KnnWs w = carve_knn(c, P);
  if (c.bytes() > workspace_bytes) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, c.bytes());
    return MSC_ERR_WORKSPACE;
  }
  cudaStream_t st = as_stream(stream);
  MSC_TRY(launch_single_segment(w.seg, n, st));
  MSC_TRY(run_knn(P, w, X_dev, knn_idx_dev, knn_dist_dev, 0, st));
  return copy_stats(w, stats_dev, st);
}

size_t msc_neighbors_workspace_bytes(int64_t n, int32_t d, int32_t k, int32_t metric,
                                     int32_t method, int32_t precision, int32_t kprime) {
  Problem P;
  if (make_problem(P, n, d, k, metric, precision, kprime, nullptr, 1) != MSC_OK) return 0;
  if (method != MSC_METHOD_UMAP && method != MSC_METHOD_GAUSS) return 0;
  Carver c(nullptr);
  carve_knn(c, P);
  carve_graph(c, n, k, method);
  return c.bytes();
}

int msc_neighbors(const float* X_dev, int64_t n, int32_t d, int32_t k, int32_t metric,
                  int32_t method, int32_t precision, int32_t kprime, int32_t* knn_idx_dev,
                  float* knn_dist_dev, int64_t* dist_indptr_dev, int32_t* dist_indices_dev,
                  float* dist_data_dev, int64_t* conn_indptr_dev, int32_t* conn_indices_dev,
                  float* conn_data_dev, int64_t* stats_dev, void* workspace,
                  size_t workspace_bytes, void* stream) {
  return msc_neighbors_ex(X_dev, n, d, k, metric, method, precision, kprime, knn_idx_dev,
                          knn_dist_dev, dist_indptr_dev, dist_indices_dev, dist_data_dev,
                          conn_indptr_dev, conn_indices_dev, conn_data_dev, stats_dev, workspace,
                          workspace_bytes, stream, nullptr);
}

int msc_neighbors_ex(const float* X_dev, int64_t n, int32_t d, int32_t k, int32_t metric,
                     int32_t method, int32_t precision, int32_t kprime, int32_t* knn_idx_dev,
                     float* knn_dist_dev, int64_t* dist_indptr_dev, int32_t* dist_indices_dev,
                     float* dist_data_dev, int64_t* conn_indptr_dev, int32_t* conn_indices_dev,
                     float* conn_data_dev, int64_t* stats_dev, void* workspace,
                     size_t workspace_bytes, void* stream, void* distances_ready_event) {
  StageRangeGuard range_guard;
  Problem P;
  MSC_TRY(make_problem(P, n, d, k, metric, precision, kprime, nullptr, 1));
  if (method != MSC_METHOD_UMAP && method != MSC_METHOD_GAUSS) {
    set_error("unknown method %d", method);
    return MSC_ERR_INVALID_ARG;
  }
  if (bad_ptr(X_dev, "X") || bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(dist_indptr_dev, "dist_indptr") || bad_ptr(dist_indices_dev, "dist_indices") ||
      bad_ptr(dist_data_dev, "dist_data") || bad_ptr(conn_indptr_dev, "conn_indptr") ||
      bad_ptr(conn_indices_dev, "conn_indices") || bad_ptr(conn_data_dev, "conn_data") ||
      bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  Carver c(workspace);
  KnnWs w = carve_knn(c, P);
  GraphWs g = carve_graph(c, n, k, method);
  if (c.bytes() > workspace_bytes) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, c.bytes());
    return MSC_ERR_WORKSPACE;
  }
  cudaStream_t st = as_stream(stream);
  MSC_TRY(launch_single_segment(w.seg, n, st));
  MSC_TRY(run_knn(P, w, X_dev, knn_idx_dev, knn_dist_dev, 0, st));
  MSC_TRY(launch_distances_csr(knn_idx_dev, knn_dist_dev, n, k, dist_indptr_dev, dist_indices_dev,
                               dist_data_dev, st));
  // the distances CSR (and the kNN lists) are final here: a caller can copy them out on another
  // stream while the connectivities are computed
  if (distances_ready_event)
    MSC_CUDA_TRY(cudaEventRecord(static_cast<cudaEvent_t>(distances_ready_event), st));
  if (method == MSC_METHOD_UMAP) {
    MSC_TRY(launch_smooth_knn(knn_dist_dev, n, k, 1.0f, g.sigma, g.rho, g.gsum, st));
    MSC_TRY(launch_membership(knn_idx_dev, knn_dist_dev, g.sigma, g.rho, n, k, g.w, st));
    stage_mark(st, 6);
    MSC_TRY(launch_union(0, knn_idx_dev, g.w, nullptr, n, k, conn_indptr_dev, conn_indices_dev,
                         conn_data_dev, nullptr, g.uws, g.uws_bytes, st));
  } else {
    MSC_TRY(launch_gauss_sigma(knn_dist_dev, n, k, g.sig2, st));
    stage_mark(st, 6);
    MSC_TRY(launch_union(1, knn_idx_dev, knn_dist_dev, g.sig2, n, k, conn_indptr_dev,
                         conn_indices_dev, conn_data_dev, nullptr, g.uws, g.uws_bytes, st));
  }
  store_nnz_kernel<<<1, 32, 0, st>>>(conn_indptr_dev, n, w.ctl);
  MSC_LAUNCH_CHECK();
  stage_mark(st, 7);
  return copy_stats(w, stats_dev, st);
}

size_t msc_batched_workspace_bytes(const int64_t* offsets_host, int32_t n_samples, int32_t d,
                                   int32_t k, int32_t metric, int32_t precision, int32_t kprime) {
  if (!offsets_host || n_samples < 1) return 0;
  Problem P;
  if (make_problem(P, offsets_host[n_samples], d, k, metric, precision, kprime, offsets_host,
                   n_samples) != MSC_OK)
    return 0;
  Carver c(nullptr);
  carve_knn(c, P);
  return c.bytes();
}

int msc_batched_prepare(const int64_t* offsets_host, int32_t n_samples, int32_t d, int32_t k,
                        int32_t metric, int32_t precision, int32_t kprime, void* workspace,
                        size_t workspace_bytes, void* stream) {
  if (!offsets_host || n_samples < 1) { set_error("offsets/n_samples invalid"); return MSC_ERR_INVALID_ARG; }
  Problem P;
  MSC_TRY(make_problem(P, offsets_host[n_samples], d, k, metric, precision, kprime, offsets_host,
                       n_samples));
  if (bad_ptr(workspace, "workspace")) return MSC_ERR_INVALID_ARG;
  Carver c(workspace);
  KnnWs w = carve_knn(c, P);
  if (c.bytes() > workspace_bytes) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, c.bytes());
    return MSC_ERR_WORKSPACE;
  }
  // samples packed largest first: the persistent kernels hand out query tiles round-robin, and
  // starting with the longest tiles balances the work across SMs
  std::vector<int> order(n_samples);
  for (int s = 0; s < n_samples; ++s) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return offsets_host[a + 1] - offsets_host[a] > offsets_host[b + 1] - offsets_host[b];
  });
  std::vector<SegDesc> segs(n_samples);
  int64_t poff = 0, tile = 0, ptile = 0;
  for (int r = 0; r < n_samples; ++r) {
    const int s = order[r];
    SegDesc sd{};
    sd.off = offsets_host[s];
    sd.n = offsets_host[s + 1] - offsets_host[s];
    sd.poff = poff;
    sd.padlen = round_up(sd.n, SEG_PAD);
    sd.tile0 = tile;
    sd.ptile0 = ptile;
    sd.ntiles = ceil_div(sd.n, QTILE);
    segs[r] = sd;
    poff += sd.padlen;
    tile += sd.ntiles;
    ptile += ceil_div(sd.n, 2 * QTILE);
  }
  cudaStream_t st = as_stream(stream);
  MSC_CUDA_TRY(cudaMemcpyAsync(w.seg, segs.data(), sizeof(SegDesc) * n_samples,
                               cudaMemcpyHostToDevice, st));
  MSC_CUDA_TRY(cudaStreamSynchronize(st));
  return MSC_OK;
}

int msc_batched_knn(const float* X_dev, const int64_t* offsets_host, int32_t n_samples, int32_t d,
                    int32_t k, int32_t metric, int32_t precision, int32_t kprime,
                    int32_t tile_config, int32_t* knn_idx_dev, float* knn_dist_dev,
                    int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream) {
  StageRangeGuard range_guard;
  if (!offsets_host || n_samples < 1) { set_error("offsets/n_samples invalid"); return MSC_ERR_INVALID_ARG; }
  Problem P;
  MSC_TRY(make_problem(P, offsets_host[n_samples], d, k, metric, precision, kprime, offsets_host,
                       n_samples));
  if (bad_ptr(X_dev, "X") || bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  Carver c(workspace);
  KnnWs w = carve_knn(c, P);
  if (c.bytes() > workspace_bytes) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, c.bytes());
    return MSC_ERR_WORKSPACE;
  }
  cudaStream_t st = as_stream(stream);
  MSC_TRY(run_knn(P, w, X_dev, knn_idx_dev, knn_dist_dev, tile_config, st));
  return copy_stats(w, stats_dev, st);
}

int msc_smooth_knn_dist(const float* knn_dist_dev, int64_t n, int32_t k,
                        float local_connectivity, float* sigma_dev, float* rho_dev,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 1 || k < 1 || k > MSC_MAX_K) { set_error("bad n/k"); return MSC_ERR_INVALID_ARG; }
  if (!(local_connectivity >= 0.f)) { set_error("local_connectivity must be >= 0"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(knn_dist_dev, "knn_dist") || bad_ptr(sigma_dev, "sigma") || bad_ptr(rho_dev, "rho") ||
      bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  if (workspace_bytes < sizeof(double) * 1025) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, sizeof(double) * 1025);
    return MSC_ERR_WORKSPACE;
  }
  return launch_smooth_knn(knn_dist_dev, n, k, local_connectivity, sigma_dev, rho_dev,
                           static_cast<double*>(workspace), as_stream(stream));
}

int msc_membership(const int32_t* knn_idx_dev, const float* knn_dist_dev, const float* sigma_dev,
                   const float* rho_dev, int64_t n, int32_t k, float* w_dev, void* stream) {
  if (n < 1 || k < 1 || k > MSC_MAX_K) { set_error("bad n/k"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(sigma_dev, "sigma") || bad_ptr(rho_dev, "rho") || bad_ptr(w_dev, "w"))
    return MSC_ERR_INVALID_ARG;
  return launch_membership(knn_idx_dev, knn_dist_dev, sigma_dev, rho_dev, n, k, w_dev,
                           as_stream(stream));
}

size_t msc_fuzzy_union_workspace_bytes(int64_t n, int32_t k) {
  if (n < 1 || k < 1) return 0;
  return union_workspace_bytes(n, k);
}

int msc_fuzzy_union(const int32_t* knn_idx_dev, const float* w_dev, int64_t n, int32_t k,
                    int64_t* indptr_dev, int32_t* indices_dev, float* data_dev, int64_t* nnz_dev,
                    void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 1 || k < 1 || k > MSC_MAX_K) { set_error("bad n/k"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(w_dev, "w") || bad_ptr(indptr_dev, "indptr") ||
      bad_ptr(indices_dev, "indices") || bad_ptr(data_dev, "data") || bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  return launch_union(0, knn_idx_dev, w_dev, nullptr, n, k, indptr_dev, indices_dev, data_dev,
                      nnz_dev, workspace, workspace_bytes, as_stream(stream));
}

size_t msc_gauss_workspace_bytes(int64_t n, int32_t k) {
  if (n < 1 || k < 1) return 0;
  Carver c(nullptr);
  c.take<double>(n);
  c.take<unsigned char>(union_workspace_bytes(n, k));
  return c.bytes();
}

int msc_gauss_connectivities(const int32_t* knn_idx_dev, const float* knn_dist_dev, int64_t n,
                             int32_t k, int64_t* indptr_dev, int32_t* indices_dev,
                             float* data_dev, int64_t* nnz_dev, void* workspace,
                             size_t workspace_bytes, void* stream) {
  if (n < 1 || k < 1 || k > MSC_MAX_K) { set_error("bad n/k"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(indptr_dev, "indptr") || bad_ptr(indices_dev, "indices") ||
      bad_ptr(data_dev, "data") || bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  if (workspace_bytes < msc_gauss_workspace_bytes(n, k)) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, msc_gauss_workspace_bytes(n, k));
    return MSC_ERR_WORKSPACE;
  }
  Carver c(workspace);
  double* sig2 = c.take<double>(n);
  const size_t ub = union_workspace_bytes(n, k);
  void* uws = c.take<unsigned char>(ub);
  cudaStream_t st = as_stream(stream);
  MSC_TRY(launch_gauss_sigma(knn_dist_dev, n, k, sig2, st));
  return launch_union(1, knn_idx_dev, knn_dist_dev, sig2, n, k, indptr_dev, indices_dev, data_dev,
                      nnz_dev, uws, ub, st);
}

int msc_distances_csr(const int32_t* knn_idx_dev, const float* knn_dist_dev, int64_t n,
                      int32_t k, int64_t* indptr_dev, int32_t* indices_dev, float* data_dev,
                      void* stream) {
  if (n < 1 || k < 1 || k > MSC_MAX_K) { set_error("bad n/k"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(indptr_dev, "indptr") || bad_ptr(indices_dev, "indices") || bad_ptr(data_dev, "data"))
    return MSC_ERR_INVALID_ARG;
  return launch_distances_csr(knn_idx_dev, knn_dist_dev, n, k, indptr_dev, indices_dev, data_dev,
                              as_stream(stream));
}

// ---- UMAP edge preparation on the device (embedding.py:115-137, 255-267) ----

size_t msc_umap_edges_workspace_bytes(int64_t n) { return n < 1 ? 0 : umap_edges_workspace_bytes(n); }

int msc_umap_edges(const int64_t* indptr_dev, const int32_t* indices_dev, const float* data_dev,
                   int64_t n, int32_t n_epochs, int64_t* out_indptr_dev, int32_t* rows_dev,
                   int32_t* cols_dev, float* weights_dev, double* epochs_per_sample_dev,
                   void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 1 || n >= (int64_t(1) << 31)) { set_error("n=%lld out of range", (long long)n); return MSC_ERR_INVALID_ARG; }
  if (n_epochs < 1) { set_error("n_epochs=%d must be >= 1", n_epochs); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(indptr_dev, "indptr") || bad_ptr(indices_dev, "indices") ||
      bad_ptr(data_dev, "data") || bad_ptr(out_indptr_dev, "out_indptr") ||
      bad_ptr(rows_dev, "rows") || bad_ptr(cols_dev, "cols") || bad_ptr(weights_dev, "weights") ||
      bad_ptr(epochs_per_sample_dev, "epochs_per_sample") || bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  if (workspace_bytes < umap_edges_workspace_bytes(n)) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, umap_edges_workspace_bytes(n));
    return MSC_ERR_WORKSPACE;
  }
  return launch_umap_edges(indptr_dev, indices_dev, data_dev, n, n_epochs, out_indptr_dev,
                           rows_dev, cols_dev, weights_dev, epochs_per_sample_dev, workspace,
                           as_stream(stream));
}

// ---- batch-balanced kNN (neighbors.py:491-559, 465-488) ----

static int bb_check(int64_t n, int32_t d, const int64_t* counts_host, int32_t n_batches,
                    int32_t kwb, int32_t precision) {
  if (n < 1 || d < 1 || d > MSC_MAX_D) {
    set_error("n=%lld must be >= 1 and d=%d in [1, %d]", (long long)n, d, MSC_MAX_D);
    return MSC_ERR_INVALID_ARG;
  }
  if (n_batches < 1 || !counts_host) {
    set_error("n_batches=%d must be >= 1 with a counts array", n_batches);
    return MSC_ERR_INVALID_ARG;
  }
  if (kwb < 1) { set_error("neighbors_within_batch=%d must be >= 1", kwb); return MSC_ERR_INVALID_ARG; }
  if (precision != MSC_PREC_FP32 && precision != MSC_PREC_BF16X3 && precision != MSC_PREC_FP16 &&
      precision != MSC_PREC_BF16) {
    set_error("unknown precision %d", precision);
    return MSC_ERR_INVALID_ARG;
  }
  int64_t tot = 0, keys = 0, width = 0;
  for (int32_t b = 0; b < n_batches; ++b) {
    if (counts_host[b] < 1) {
      set_error("batch %d has %lld cells (every batch needs one)", b, (long long)counts_host[b]);
      return MSC_ERR_INVALID_ARG;
    }
    tot += counts_host[b];
    keys += round_up(counts_host[b], SEG_PAD);
    width += std::min<int64_t>(kwb, counts_host[b]);
  }
  if (tot != n) {
    set_error("batch counts add up to %lld, not n=%lld", (long long)tot, (long long)n);
    return MSC_ERR_INVALID_ARG;
  }
  if (width > MSC_BBKNN_MAX_WIDTH) {
    set_error("neighbors_within_batch x batches = %lld entries per cell > %d", (long long)width,
              MSC_BBKNN_MAX_WIDTH);
    return MSC_ERR_INVALID_ARG;
  }
  if (keys + round_up(n, QTILE) >= (int64_t(1) << 31)) {
    set_error("n=%lld is too large for 32-bit packed rows", (long long)n);
    return MSC_ERR_INVALID_ARG;
  }
  return MSC_OK;
}

int32_t msc_bbknn_width(const int64_t* counts_host, int32_t n_batches, int32_t kwb) {
  if (!counts_host || n_batches < 1 || kwb < 1) return 0;
  int64_t width = 0;
  for (int32_t b = 0; b < n_batches; ++b) width += std::min<int64_t>(kwb, std::max<int64_t>(counts_host[b], 0));
  return int32_t(std::min<int64_t>(width, INT32_MAX));
}

size_t msc_bbknn_workspace_bytes(int64_t n, int32_t d, const int64_t* counts_host,
                                 int32_t n_batches, int32_t kwb, int32_t precision) {
  if (bb_check(n, d, counts_host, n_batches, kwb, precision) != MSC_OK) return 0;
  return bb_workspace_bytes(bb_plan(n, d, counts_host, n_batches, kwb, precision));
}

int msc_bbknn_knn(const float* X_dev, int64_t n, int32_t d, const int32_t* batch_dev,
                  const int64_t* counts_host, int32_t n_batches, int32_t kwb, int32_t precision,
                  int32_t* knn_idx_dev, float* knn_dist_dev, int64_t* stats_dev,
                  void* workspace, size_t workspace_bytes, void* stream) {
  MSC_TRY(bb_check(n, d, counts_host, n_batches, kwb, precision));
  if (bad_ptr(X_dev, "X") || bad_ptr(batch_dev, "batch") || bad_ptr(knn_idx_dev, "knn_idx") ||
      bad_ptr(knn_dist_dev, "knn_dist") || bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  const BbPlan P = bb_plan(n, d, counts_host, n_batches, kwb, precision);
  BbWs w;
  const size_t need = bb_carve(P, workspace, w);
  if (need > workspace_bytes) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, need);
    return MSC_ERR_WORKSPACE;
  }
  cudaStream_t st = as_stream(stream);
  MSC_TRY(run_bbknn(P, w, X_dev, batch_dev, counts_host, knn_idx_dev, knn_dist_dev, st));
  MSC_TRY(launch_set_stat(w.ctl, MSC_STAT_PRECISION, P.candidates ? P.prec : -1, st));
  if (stats_dev)
    MSC_CUDA_TRY(cudaMemcpyAsync(stats_dev, w.ctl->stats, sizeof(int64_t) * MSC_STATS_LEN,
                                 cudaMemcpyDeviceToDevice, st));
  return MSC_OK;
}

size_t msc_bbknn_distances_workspace_bytes(int64_t n) {
  return n < 1 ? 0 : bb_distances_workspace_bytes(n);
}

int msc_bbknn_distances_csr(const int32_t* knn_idx_dev, const float* knn_dist_dev, int64_t n,
                            int32_t K, int64_t* indptr_dev, int32_t* indices_dev, float* data_dev,
                            void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 1 || K < 1 || K > MSC_BBKNN_MAX_WIDTH) { set_error("bad n/K"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist") ||
      bad_ptr(indptr_dev, "indptr") || bad_ptr(indices_dev, "indices") ||
      bad_ptr(data_dev, "data") || bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  if (workspace_bytes < bb_distances_workspace_bytes(n)) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, bb_distances_workspace_bytes(n));
    return MSC_ERR_WORKSPACE;
  }
  return launch_bb_distances(knn_idx_dev, knn_dist_dev, n, K, indptr_dev, indices_dev, data_dev,
                             workspace, as_stream(stream));
}

size_t msc_trim_graph_workspace_bytes(int64_t n) { return n < 1 ? 0 : trim_workspace_bytes(n); }

int msc_trim_graph(const int64_t* indptr_dev, const int32_t* indices_dev, const float* data_dev,
                   int64_t n, int32_t trim, int64_t* out_indptr_dev, int32_t* out_indices_dev,
                   float* out_data_dev, void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 1 || trim < 1) { set_error("n=%lld and trim=%d must be >= 1", (long long)n, trim); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(indptr_dev, "indptr") || bad_ptr(indices_dev, "indices") ||
      bad_ptr(data_dev, "data") || bad_ptr(out_indptr_dev, "out_indptr") ||
      bad_ptr(out_indices_dev, "out_indices") || bad_ptr(out_data_dev, "out_data") ||
      bad_ptr(workspace, "workspace"))
    return MSC_ERR_INVALID_ARG;
  if (workspace_bytes < trim_workspace_bytes(n)) {
    set_error("workspace %zu < %zu bytes", workspace_bytes, trim_workspace_bytes(n));
    return MSC_ERR_WORKSPACE;
  }
  return launch_trim(indptr_dev, indices_dev, data_dev, n, trim, out_indptr_dev, out_indices_dev,
                     out_data_dev, workspace, as_stream(stream));
}

namespace {
int check_spatial(int64_t n, int32_t d, const void* coords, const void* stats, const void* ws,
                  size_t ws_bytes, size_t need) {
  if (n < 1 || n > MSC_SPATIAL_MAX_N) { set_error("n=%lld out of range", (long long)n); return MSC_ERR_INVALID_ARG; }
  if (d != 2 && d != 3) {
    set_error("spatial search expects 2-D or 3-D coordinates, got %d-D", d);
    return MSC_ERR_UNSUPPORTED;
  }
  if (bad_ptr(coords, "coords") || bad_ptr(stats, "stats") || bad_ptr(ws, "workspace"))
    return MSC_ERR_INVALID_ARG;
  if (ws_bytes < need) {
    set_error("workspace of %zu bytes, %zu needed", ws_bytes, need);
    return MSC_ERR_WORKSPACE;
  }
  return MSC_OK;
}
int check_radius(double radius, double min_radius) {
  if (!(radius >= 0) || !std::isfinite(radius) || !(min_radius >= 0) || !(min_radius <= radius)) {
    set_error("radius interval [%g, %g] is not a finite interval of non-negative values",
              min_radius, radius);
    return MSC_ERR_INVALID_ARG;
  }
  return MSC_OK;
}
}  // namespace

size_t msc_spatial_knn_workspace_bytes(int64_t n, int32_t d, int32_t k) {
  (void)d;
  (void)k;
  return n < 1 ? 0 : spatial_knn_workspace_bytes(n);
}

int msc_spatial_knn(const float* coords_dev, int64_t n, int32_t d, int32_t k, int32_t* knn_idx_dev,
                    float* knn_dist_dev, int64_t* stats_dev, void* workspace,
                    size_t workspace_bytes, void* stream) {
  MSC_TRY(check_spatial(n, d, coords_dev, stats_dev, workspace, workspace_bytes,
                        n < 1 ? 0 : spatial_knn_workspace_bytes(n)));
  if (k < 1 || k > MSC_SPATIAL_MAX_K || k > n) {
    set_error("k=%d must be in [1, min(n=%lld, %d)]", k, (long long)n, MSC_SPATIAL_MAX_K);
    return k > MSC_SPATIAL_MAX_K && k <= n ? MSC_ERR_UNSUPPORTED : MSC_ERR_INVALID_ARG;
  }
  if (bad_ptr(knn_idx_dev, "knn_idx") || bad_ptr(knn_dist_dev, "knn_dist")) return MSC_ERR_INVALID_ARG;
  return launch_spatial_knn(coords_dev, n, d, k, knn_idx_dev, knn_dist_dev, stats_dev, workspace,
                            as_stream(stream));
}

size_t msc_spatial_radius_workspace_bytes(int64_t n, int32_t d) {
  (void)d;
  return n < 1 ? 0 : spatial_radius_workspace_bytes(n);
}

int msc_spatial_radius_count(const float* coords_dev, int64_t n, int32_t d, double radius,
                             double min_radius, int64_t* indptr_dev, int64_t* stats_dev,
                             void* workspace, size_t workspace_bytes, void* stream) {
  MSC_TRY(check_spatial(n, d, coords_dev, stats_dev, workspace, workspace_bytes,
                        n < 1 ? 0 : spatial_radius_workspace_bytes(n)));
  MSC_TRY(check_radius(radius, min_radius));
  if (bad_ptr(indptr_dev, "indptr")) return MSC_ERR_INVALID_ARG;
  return launch_spatial_radius_count(coords_dev, n, d, radius, min_radius, indptr_dev, stats_dev,
                                     workspace, as_stream(stream));
}

size_t msc_spatial_radius_scratch_bytes(int64_t nnz) {
  return spatial_radius_fill_scratch_bytes(nnz < 0 ? 0 : nnz);
}

int msc_spatial_radius_fill(int64_t n, int32_t d, double radius, double min_radius,
                            const int64_t* indptr_dev, int64_t nnz, int32_t* indices_dev,
                            float* dist_dev, void* workspace, size_t workspace_bytes,
                            void* scratch, size_t scratch_bytes, void* stream) {
  MSC_TRY(check_spatial(n, d, indptr_dev, workspace, workspace, workspace_bytes,
                        n < 1 ? 0 : spatial_radius_workspace_bytes(n)));
  MSC_TRY(check_radius(radius, min_radius));
  if (nnz < 0) { set_error("nnz < 0"); return MSC_ERR_INVALID_ARG; }
  if (nnz > 0 && (bad_ptr(indices_dev, "indices") || bad_ptr(dist_dev, "dist") ||
                  bad_ptr(scratch, "scratch")))
    return MSC_ERR_INVALID_ARG;
  if (scratch_bytes < spatial_radius_fill_scratch_bytes(nnz)) {
    set_error("scratch of %zu bytes, %zu needed", scratch_bytes,
              spatial_radius_fill_scratch_bytes(nnz));
    return MSC_ERR_WORKSPACE;
  }
  return launch_spatial_radius_fill(n, d, radius, min_radius, indptr_dev, nnz, indices_dev,
                                    dist_dev, workspace, scratch, as_stream(stream));
}

int msc_spatial_edge_lengths(const double* coords64_dev, int64_t n, int32_t d,
                             const int64_t* indptr_dev, const int32_t* indices_dev,
                             double* out_dev, void* stream) {
  if (n < 1 || d < 1 || d > 3) { set_error("bad n/d"); return MSC_ERR_INVALID_ARG; }
  if (bad_ptr(coords64_dev, "coords64") || bad_ptr(indptr_dev, "indptr") ||
      bad_ptr(indices_dev, "indices") || bad_ptr(out_dev, "out"))
    return MSC_ERR_INVALID_ARG;
  return launch_spatial_edge_lengths(coords64_dev, n, d, indptr_dev, indices_dev, out_dev,
                                     as_stream(stream));
}

}  // extern "C"
