/*
 * msc_b200 — C ABI of the B200 neighbour-graph library (the `msc.pp.neighbors` hot path).
 *
 * Every entry point is stream-ordered: it enqueues work on `stream` (a cudaStream_t passed as
 * void*, NULL = legacy default stream) and returns without waiting.  Pointers named *_dev are
 * device pointers; nothing is allocated inside the library — scratch memory is the caller's
 * `workspace`, sized by the matching *_workspace_bytes() query.  Errors come back as an int status
 * (never as an exception across the ABI); msc_last_error() gives the message of the calling
 * thread's last failure.  Errors that can only be seen on the device (non-finite input, a timed-out
 * wait) are counted in the int64 `stats_dev` block (MSC_STAT_*) that the caller reads after the
 * stream completes.
 *
 * Conventions shared by all calls (the reference's, metalsinglecell `neighbors.py`):
 *   X          n×d float32, row-major, one cell per row (the PCA embedding).
 *   knn_idx    n×k int32, row i = [i, then the k-1 nearest other cells by (distance, index)].
 *   knn_dist   n×k float32, the matching distances (column 0 is 0).
 *   CSR        int64 indptr (n+1), int32 indices (column-sorted per row), float32 data.
 */
#ifndef MSC_B200_H
#define MSC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MSC_OK                  0
#define MSC_ERR_INVALID_ARG     1   /* bad shape, k, pointer or option (Python: ValueError)      */
#define MSC_ERR_WORKSPACE       2   /* workspace smaller than *_workspace_bytes() (MemoryError) */
#define MSC_ERR_TIMEOUT         3   /* a device-side wait hit its bound (RuntimeError)          */
#define MSC_ERR_CUDA            4   /* a CUDA runtime call failed (RuntimeError)                */
#define MSC_ERR_UNSUPPORTED     5   /* valid request the library does not handle (NotImplemented)*/

/* metric (the reference accepts only euclidean, pp.py:768-769) */
#define MSC_METRIC_EUCLIDEAN    0
#define MSC_METRIC_COSINE       1

/* candidate precision of the distance + top-k stage */
#define MSC_PREC_FP32           0   /* plain FP32 SIMT Gram form                                 */
#define MSC_PREC_BF16X3         1   /* tcgen05 BF16, 3-term split (hi·hi + hi·lo + lo·hi)        */
#define MSC_PREC_FP16           2   /* tcgen05 FP16, one term (the reference ranks on fp16)      */
#define MSC_PREC_BF16           3   /* tcgen05 BF16, one term                                    */

/* connectivity method */
#define MSC_METHOD_UMAP         0
#define MSC_METHOD_GAUSS        1

/* indices into the int64 stats block (MSC_STATS_LEN entries, zeroed by the call) */
#define MSC_STAT_NONFINITE      0   /* non-finite input values seen                              */
#define MSC_STAT_TIMEOUT        1   /* device waits that gave up                                 */
#define MSC_STAT_CERTIFIED      2   /* rows whose candidate set was proven to hold the exact kNN */
#define MSC_STAT_REFINED        3   /* rows re-run through the BF16x3 candidate stage            */
#define MSC_STAT_RESCANNED      4   /* rows finished by the exact FP64 full scan                 */
#define MSC_STAT_FP64_TIES      5   /* candidates re-ranked in FP64 at the k-th boundary         */
#define MSC_STAT_CONN_NNZ       6   /* nnz of the connectivities CSR                              */
#define MSC_STAT_PRECISION      7   /* candidate precision actually used (FP32 when the operand
                                       row is too wide for the tensor-core tile; -1: FP64 scan) */
#define MSC_STATS_LEN           8

#define MSC_MAX_K               129 /* largest n_neighbors (above 65 every row takes the FP64 scan) */
#define MSC_MAX_K_KNN           513 /* largest n_neighbors of msc_knn alone (FP64 scan above 65)  */
#define MSC_MAX_D               128 /* largest representation width                             */

int         msc_version(void);
const char* msc_last_error(void);

/* Instrumentation (no counterpart in the reference).
 *   msc_launch_count   kernels this library has launched in this process;
 *   msc_profile_enable process-wide switch: record CUDA events between pipeline stages
 *                      (prep | near pass | key-tile pruning plan | candidates | re-rank +
 *                      FP64 scan | CSR + rho/sigma + memberships | fuzzy union) of the following
 *                      calls — not for concurrent callers;
 *   msc_profile_read   waits for the last profiled call's events and writes its stage times in ms;
 *                      returns the number of stages written. */
long long msc_launch_count(void);
int       msc_profile_enable(int on);
int       msc_profile_read(float* ms_out, int max_stages);
/* pipeline counters of the tensor-core candidate kernel summed over CTAs since the last
 * msc_profile_enable(1) (cycles waiting / busy per role, hot chunks, compactions, candidate
 * insertions, CTAs), and in slots 10 and 11 the key tiles beyond the near ones that pruning
 * kept / could have kept; with max_counters >= 64, out[16 + 16·j + i] holds counter i of the
 * near pass (j = 0), the main scan (j = 1) and the refine pass (j = 2) alone; synchronizes the
 * device. */
int       msc_profile_counters(unsigned long long* out, int max_counters);

/* Self-test of the bounded device waits that every pipeline wait uses (no counterpart in the
 * reference): one kernel waits on a barrier that nothing arrives at, gives up after limit_ns
 * (1 us .. 10 s) and returns normally.  out_dev (int32[3]) = {1 if it gave up, abort flag,
 * elapsed ms}.  Nothing faults or hangs; the context stays usable. */
int       msc_selftest_wait_timeout(int64_t limit_ns, int32_t* out_dev, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Whole graph — replaces metalsinglecell `neighbors.neighbors` (neighbors.py:727-760), itself
 * called by `pp.neighbors` (pp.py:774).
 *   dist_*  : the distances CSR of neighbors.py:755-759 (k-1 entries per row, indptr i·(k-1)).
 *   conn_*  : the connectivities CSR (capacity 2·n·(k-1) entries); its nnz is written to
 *             stats_dev[MSC_STAT_CONN_NNZ] and conn_indptr[n].
 *   kprime  : candidates kept per row by the tensor-core stage (0 = automatic).
 * ------------------------------------------------------------------------------------------- */
size_t msc_neighbors_workspace_bytes(int64_t n, int32_t d, int32_t k, int32_t metric,
                                     int32_t method, int32_t precision, int32_t kprime);
int msc_neighbors(const float* X_dev, int64_t n, int32_t d, int32_t k, int32_t metric,
                  int32_t method, int32_t precision, int32_t kprime,
                  int32_t* knn_idx_dev, float* knn_dist_dev,
                  int64_t* dist_indptr_dev, int32_t* dist_indices_dev, float* dist_data_dev,
                  int64_t* conn_indptr_dev, int32_t* conn_indices_dev, float* conn_data_dev,
                  int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream);

/* msc_neighbors with one more argument: distances_ready_event (a cudaEvent_t, or NULL) is recorded
 * on the stream as soon as the kNN lists and the distances CSR are final, before the
 * connectivities are computed, so a caller can copy them to the host on another stream meanwhile.
 * No counterpart in the reference. */
int msc_neighbors_ex(const float* X_dev, int64_t n, int32_t d, int32_t k, int32_t metric,
                     int32_t method, int32_t precision, int32_t kprime,
                     int32_t* knn_idx_dev, float* knn_dist_dev,
                     int64_t* dist_indptr_dev, int32_t* dist_indices_dev, float* dist_data_dev,
                     int64_t* conn_indptr_dev, int32_t* conn_indices_dev, float* conn_data_dev,
                     int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream,
                     void* distances_ready_event);

/* ---------------------------------------------------------------------------------------------
 * Exact kNN — replaces `_knn` / `_knn_gpu` (neighbors.py:698-724, 82-132): the fp16 Gram
 * distance (neighbors.py:117-118), the register top-k kernel `topk_rows` (neighbors.py:25-79),
 * the fp32 recompute (neighbors.py:122-123) and the host sort (neighbors.py:129-131), as one fused
 * candidate kernel + exact re-rank.  Self first; ties by index.  n_neighbors up to MSC_MAX_K_KNN
 * (scrublet's k_adj + 1 over observed and simulated cells reaches several hundred); above 65
 * every row takes the exact FP64 scan.
 * ------------------------------------------------------------------------------------------- */
size_t msc_knn_workspace_bytes(int64_t n, int32_t d, int32_t k, int32_t metric, int32_t precision,
                               int32_t kprime);
int msc_knn(const float* X_dev, int64_t n, int32_t d, int32_t k, int32_t metric,
            int32_t precision, int32_t kprime, int32_t* knn_idx_dev, float* knn_dist_dev,
            int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream);

/* Many independent samples in one persistent launch: sample s is rows [offsets[s], offsets[s+1])
 * of X and its neighbours are searched only among its own rows.  `offsets_host` has n_samples+1
 * entries; every sample needs at least k cells.  New in this library (the reference loops in
 * Python over per-batch brute-force calls, neighbors.py:516-539).
 *   msc_batched_prepare  writes the sample table into the workspace and waits for that copy;
 *   msc_batched_knn      only enqueues kernels (capturable in a CUDA graph); call it with the
 *                        same offsets / shapes as the prepare call.
 * tile_config: 0 = automatic, else bn | stages<<12 | cb<<20 | epi8<<27 | pair<<28 | dual<<29
 * (key tile rows, pipeline depth in 64-element K atoms, selector buffer, eight instead of four
 * epilogue warps, two-CTA clusters on 256-row query tiles, two CTAs per SM with one accumulator
 * each) as chosen by the Python autotuner.  With 0, the environment variable
 * MSC_B200_TILE_CONFIG (same encoding) overrides the automatic choice for every entry point. */
size_t msc_batched_workspace_bytes(const int64_t* offsets_host, int32_t n_samples, int32_t d,
                                   int32_t k, int32_t metric, int32_t precision, int32_t kprime);
int msc_batched_prepare(const int64_t* offsets_host, int32_t n_samples, int32_t d, int32_t k,
                        int32_t metric, int32_t precision, int32_t kprime, void* workspace,
                        size_t workspace_bytes, void* stream);
int msc_batched_knn(const float* X_dev, const int64_t* offsets_host, int32_t n_samples, int32_t d,
                    int32_t k, int32_t metric, int32_t precision, int32_t kprime,
                    int32_t tile_config, int32_t* knn_idx_dev, float* knn_dist_dev,
                    int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------------------------------
 * UMAP fuzzy simplicial set pieces — replace umap-learn 0.5.12 `fuzzy_simplicial_set` as the
 * reference calls it (neighbors.py:742-753: set_op_mix_ratio=1, local_connectivity=1).
 * ------------------------------------------------------------------------------------------- */
/* per-row rho / sigma by bisection (umap-learn smooth_knn_dist); workspace >= 64 bytes */
int msc_smooth_knn_dist(const float* knn_dist_dev, int64_t n, int32_t k,
                        float local_connectivity, float* sigma_dev, float* rho_dev,
                        void* workspace, size_t workspace_bytes, void* stream);
/* memberships w_ij (umap-learn compute_membership_strengths); self -> 0 */
int msc_membership(const int32_t* knn_idx_dev, const float* knn_dist_dev, const float* sigma_dev,
                   const float* rho_dev, int64_t n, int32_t k, float* w_dev, void* stream);
/* P = A + A^T - A∘A^T as CSR (zeros of A eliminated first), bit-exact float32 arithmetic */
size_t msc_fuzzy_union_workspace_bytes(int64_t n, int32_t k);
int msc_fuzzy_union(const int32_t* knn_idx_dev, const float* w_dev, int64_t n, int32_t k,
                    int64_t* indptr_dev, int32_t* indices_dev, float* data_dev, int64_t* nnz_dev,
                    void* workspace, size_t workspace_bytes, void* stream);

/* The fuzzy union without caller-provided scratch.  No counterpart in the reference: it is for
 * callers that cannot give the library device memory — code under a memory manager that owns all
 * of the GPU's memory (a framework's caching allocator, a serving process that reserves its HBM
 * at start-up and offers plug-ins no allocator) or a hot loop where cudaMalloc/cudaFree, which may
 * synchronise the device, are not acceptable.  It allocates nothing: its scratch is a fixed 20 MiB
 * array in the library's own device memory (held on every GPU that loads the library until the
 * process exits), so it accepts only n <= MSC_NOALLOC_MAX_CELLS and n*k <= MSC_NOALLOC_MAX_ENTRIES
 * and answers MSC_ERR_INVALID_ARG beyond that.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that first call before any
 * stream capture.  The address is kept for the life of the process, so a cudaDeviceReset (or any
 * other teardown of the device's primary context) after that first call is not supported: the
 * kept address would no longer name the array.  All calls share the one array: calls that overlap
 * on the GPU (other streams, other host threads) race and corrupt each other's results —
 * serialise them. */
#define MSC_NOALLOC_MAX_CELLS   65536
#define MSC_NOALLOC_MAX_ENTRIES 1048576
int msc_fuzzy_union_noalloc(const int32_t* knn_idx_dev, const float* w_dev, int64_t n, int32_t k,
                            int64_t* indptr_dev, int32_t* indices_dev, float* data_dev,
                            int64_t* nnz_dev, void* stream);

/* method='gauss' connectivities (scanpy's locally scaled Gaussian kernel; not in the reference) */
size_t msc_gauss_workspace_bytes(int64_t n, int32_t k);
int msc_gauss_connectivities(const int32_t* knn_idx_dev, const float* knn_dist_dev, int64_t n,
                             int32_t k, int64_t* indptr_dev, int32_t* indices_dev,
                             float* data_dev, int64_t* nnz_dev, void* workspace,
                             size_t workspace_bytes, void* stream);

/* distances CSR exactly as neighbors.py:755-759 builds it (explicit zeros kept) */
int msc_distances_csr(const int32_t* knn_idx_dev, const float* knn_dist_dev, int64_t n,
                      int32_t k, int64_t* indptr_dev, int32_t* indices_dev, float* data_dev,
                      void* stream);

/* Edge preparation of the UMAP layout from a connectivities CSR already on the device (the graph
 * hand-off to its first consumer).  Replaces the host steps of metalsinglecell `embedding.umap`:
 * `_prune_weak_edges` (embedding.py:255-267: keep w >= fl32(max w / n_epochs)), the kept graph
 * as COO in CSR order (embedding.py:115) and `_make_epochs_per_sample` (embedding.py:123-137:
 * n_epochs / (n_epochs · (w / max w)) in FP64, -1 for an edge never sampled).
 *   input : CSR (indptr n+1 int64, indices int32, data float32), n_epochs >= 1
 *   output: the kept graph's indptr (n+1 int64; nnz = out_indptr[n]) and, per kept edge in CSR
 *           order, its row, column, weight and sampling period; capacity = the input's nnz */
size_t msc_umap_edges_workspace_bytes(int64_t n);
int msc_umap_edges(const int64_t* indptr_dev, const int32_t* indices_dev, const float* data_dev,
                   int64_t n, int32_t n_epochs, int64_t* out_indptr_dev, int32_t* rows_dev,
                   int32_t* cols_dev, float* weights_dev, double* epochs_per_sample_dev,
                   void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Batch-balanced kNN — replaces metalsinglecell `neighbors.bbknn` (neighbors.py:491-559), called
 * by `pp.bbknn` (pp.py:809-833).  Every cell gets its kk_b = min(neighbors_within_batch, n_b)
 * nearest cells of every batch b (exact; a cell of b finds itself at distance 0), K = Σ kk_b
 * entries per cell sorted by (distance, index).  The connectivities are the fuzzy set of these
 * lists (msc_smooth_knn_dist / msc_membership / msc_fuzzy_union with k = K).
 *   batch_dev   : batch code of every cell, 0 .. n_batches-1
 *   counts_host : cells per batch (n_batches entries, each >= 1, adding up to n); they must be
 *                 the histogram of batch_dev
 *   knn_*_dev   : n x K, K = msc_bbknn_width(counts_host, n_batches, neighbors_within_batch)
 * ------------------------------------------------------------------------------------------- */
#define MSC_BBKNN_MAX_WIDTH     128 /* largest K = Σ_b min(neighbors_within_batch, n_b)          */
int32_t msc_bbknn_width(const int64_t* counts_host, int32_t n_batches,
                        int32_t neighbors_within_batch);
size_t msc_bbknn_workspace_bytes(int64_t n, int32_t d, const int64_t* counts_host,
                                 int32_t n_batches, int32_t neighbors_within_batch,
                                 int32_t precision);
int msc_bbknn_knn(const float* X_dev, int64_t n, int32_t d, const int32_t* batch_dev,
                  const int64_t* counts_host, int32_t n_batches, int32_t neighbors_within_batch,
                  int32_t precision, int32_t* knn_idx_dev, float* knn_dist_dev,
                  int64_t* stats_dev, void* workspace, size_t workspace_bytes, void* stream);
/* the distances graph of the lists (neighbors.py:554-557): diagonal and zero distances dropped,
 * columns ascending; capacity n*K entries, nnz = indptr[n] */
size_t msc_bbknn_distances_workspace_bytes(int64_t n);
int msc_bbknn_distances_csr(const int32_t* knn_idx_dev, const float* knn_dist_dev, int64_t n,
                            int32_t K, int64_t* indptr_dev, int32_t* indices_dev,
                            float* data_dev, void* workspace, size_t workspace_bytes,
                            void* stream);
/* `_trim_graph` (neighbors.py:465-488): keep the stored entry (i, j, v) when v != 0, v >= θ_i and
 * v >= θ_j, θ_i = the trim-th largest stored value of row i when the row stores more than `trim`
 * entries, else 0.  Input: CSR without duplicate entries; output capacity = input nnz, in the
 * input's order within each row; nnz = out_indptr[n] */
size_t msc_trim_graph_workspace_bytes(int64_t n);
int msc_trim_graph(const int64_t* indptr_dev, const int32_t* indices_dev, const float* data_dev,
                   int64_t n, int32_t trim, int64_t* out_indptr_dev, int32_t* out_indices_dev,
                   float* out_data_dev, void* workspace, size_t workspace_bytes, void* stream);
/* ---- spatial (2-D / 3-D) uniform-grid search: replaces metalsinglecell
 *      neighbors._knn_grid (neighbors.py:333-417) and neighbors._radius_grid (neighbors.py:255-330),
 *      which gr.spatial_neighbors_knn / _radius (gr.py:186-255) and spatial.spatial_neighbors
 *      (spatial.py:13-44) call.  Coordinates are row-major float32 (n, d), d = 2 or 3.
 *      Arithmetic: d² = fl(fl(dx²) + fl(dy²)) [+ fl(dz²)], dx = fl(x_p - x_q), no fused
 *      multiply-add; distance = correctly rounded float32 sqrt(d²).  Exact for every row. ---- */
#define MSC_SPATIAL_MAX_K        65  /* largest k of msc_spatial_knn (self + 64 others)         */
#define MSC_SPATIAL_MAX_N        (1LL << 29)
#define MSC_SP_STAT_NONFINITE    0   /* non-finite coordinates (nothing is computed)             */
#define MSC_SP_STAT_STATUS       1   /* 0 ok, 1 non-finite input, 2 no cell plan                */
#define MSC_SP_STAT_CELLS        2   /* cells of the grid                                        */
#define MSC_SP_STAT_CHUNKS       3   /* query chunks (<= 32 points of one cell)                  */
#define MSC_SP_STAT_EVALS        4   /* candidate distances evaluated                            */
#define MSC_SP_STAT_EXPANDED     5   /* kNN rows that needed more than one ring of cells         */
#define MSC_SP_STAT_RING         6   /* radius search: rings of cells around the query's cell    */
#define MSC_SP_STAT_CELL_SIDE    7   /* cell side, the bits of a float64                         */
#define MSC_SP_STATS_LEN         8

/* k nearest points of every point (self first, then (distance, index) order): knn_idx (n, k)
 * int32 and knn_dist (n, k) float32, row-major.  1 <= k <= min(n, MSC_SPATIAL_MAX_K).
 * Replaces _knn_grid (neighbors.py:333-417), whose lists are self-inclusive and distance-sorted. */
size_t msc_spatial_knn_workspace_bytes(int64_t n, int32_t d, int32_t k);
int msc_spatial_knn(const float* coords_dev, int64_t n, int32_t d, int32_t k, int32_t* knn_idx_dev,
                    float* knn_dist_dev, int64_t* stats_dev, void* workspace,
                    size_t workspace_bytes, void* stream);

/* Every other point with min_radius² <= d² <= radius² (the two squares rounded to float32):
 * the two Metal passes of _radius_grid (neighbors.py:255-330).  The count call builds the grid
 * in the workspace and writes indptr (n + 1 int64); the fill call, given the same workspace
 * unchanged and indptr[n] = nnz, writes the columns (ascending in every row) and float32
 * distances. */
size_t msc_spatial_radius_workspace_bytes(int64_t n, int32_t d);
int msc_spatial_radius_count(const float* coords_dev, int64_t n, int32_t d, double radius,
                             double min_radius, int64_t* indptr_dev, int64_t* stats_dev,
                             void* workspace, size_t workspace_bytes, void* stream);
size_t msc_spatial_radius_scratch_bytes(int64_t nnz);
int msc_spatial_radius_fill(int64_t n, int32_t d, double radius, double min_radius,
                            const int64_t* indptr_dev, int64_t nnz, int32_t* indices_dev,
                            float* dist_dev, void* workspace, size_t workspace_bytes,
                            void* scratch, size_t scratch_bytes, void* stream);

/* Euclidean length of every edge of a CSR graph from float64 coordinates (n, d): squares summed
 * axis by axis in order, correctly rounded sqrt (gr._edge_lengths, gr.py:32-34). */
int msc_spatial_edge_lengths(const double* coords64_dev, int64_t n, int32_t d,
                             const int64_t* indptr_dev, const int32_t* indices_dev,
                             double* out_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MSC_B200_H */
