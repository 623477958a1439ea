// Fused pairwise-distance + per-row top-k' on the Blackwell tensor cores (sm_100a).
//
// Reference counterpart: metalsinglecell neighbors.py:114-119 — an fp16 Gram tile
// `sq_i + sq_j − 2·X_i·X_jᵀ` materialised as a block×n matrix in device memory, then the
// `topk_rows` register kernel (neighbors.py:25-79) scanning it.  Here the n×n matrix never leaves
// the SM: a 128-row query tile stays in shared memory, key tiles stream through a TMA pipeline,
// one thread issues tcgen05.mma into a double-buffered FP32 accumulator in tensor memory, and the
// epilogue warps read the accumulator (TMEM lane i = query row i) straight into the per-row
// selector while the next tile's MMAs run.  The key norms are folded into the key operand, so the
// accumulator already holds the ranking value v = |y|² − 2x·y.
//
// Roles (128 + 32·NEPI threads, one CTA per SM, persistent over query tiles):
//   warp 0  TMA producer      A tile once per query tile, then the key tiles of its sample
//   warp 1  MMA issuer        KSTEPS × tcgen05.mma (K=16) per key tile
//   warp 2  TMEM allocator    2·BN columns for two accumulators
//   warp 3  relay (pairs)     forwards the odd CTA's completed loads to the even CTA
//   warps 4.. epilogue        tcgen05.ld 32x32b → filter → selector; release the accumulator.
//                             NEPI = 4: one warp per TMEM lane quarter reads all BN columns;
//                             NEPI = 8: two warps per lane quarter read BN/2 columns each.
//
// CTA pairs (PAIR): a cluster of two CTAs computes a 256-row query tile against BN-key tiles with
// tcgen05.mma.cta_group::2 (M=256).  Each CTA stages its own 128 query rows and HALF of every key
// tile (BN/2 rows) in its own shared memory; the even CTA issues the MMAs, which read both halves,
// and each CTA's tensor memory receives its 128 rows × BN accumulator.  Key bytes per SM and per
// FLOP are halved, and the pipeline holds twice as many K-atom stages in the same shared memory.
// Every TMA load signals a barrier of the CTA that issued it, so each CTA can drain its own
// copies; the odd CTA's relay thread forwards those completions to the even CTA (remote mbarrier
// arrive), and the even CTA's commits reach both CTAs through tcgen05.commit's CTA mask.
//
// Every mbarrier wait is bounded (wall-clock, via %globaltimer); a wait that gives up raises an
// abort flag that every role polls, the kernel records MSC_STAT_TIMEOUT and all roles leave their
// loops, so a fault in the pipeline returns an error instead of hanging the GPU.
#include <cuda.h>
#include <cstdlib>

#include "kernels.cuh"
#include "msc_select.cuh"

namespace msc {

namespace {

constexpr int EPI_WARP0 = 4;
// Epilogue variants of the eight-epilogue-warp kernels, fixed at build time: the register split
// between warpgroup 0 and the epilogue warpgroups (setmaxnreg), and three TMEM chunk buffers with
// two chunks per wait (else two buffers, one chunk per wait).  Both are off: measured at
// 1.3M × 50 on one B200, the main scan took 74.0 ms with both, 81.1 ms with the three buffers
// alone and 64.1 ms with neither (the three-buffer epilogue spills under the 168-register launch
// budget; the split moves the spills, it does not remove them).
#ifndef MSC_TC_REGSPLIT
#define MSC_TC_REGSPLIT 0
#endif
#ifndef MSC_TC_TRIBUF
#define MSC_TC_TRIBUF 0
#endif
constexpr bool kRegSplit = MSC_TC_REGSPLIT != 0;
// The per-row candidate lists of the epilogue.  (A variant that buffered passing values per row
// and merged them into sorted lists with warp-wide bitonic networks measured slower: 81 ms
// against 57 ms for the 1.3M main scan, and 22 ms against 5 ms for the near pass, whose empty
// lists merge on almost every chunk.)
template <int KH>
struct SelectorOf {
  using type = RowTopK<KH, 128>;
};
constexpr bool kTriBuf = MSC_TC_TRIBUF != 0;
// register split of the eight-epilogue-warp kernels (see knn_tc_kernel)
constexpr int REG_LOW = 56, REG_HIGH = 224;
constexpr int REG_LAUNCH = (REG_LOW * 128 + REG_HIGH * 256) / 384;     // 168
static_assert(REG_LOW * 128 + REG_HIGH * 256 == REG_LAUNCH * 384, "split must fill the pool");
__device__ __forceinline__ void reg_dec() {
  asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(REG_LOW));
}
__device__ __forceinline__ void reg_inc() {
  asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(REG_HIGH));
}
constexpr int BM = 128;
constexpr int ITEM_RING = 4;                        // claimed work items in flight per CTA
constexpr uint64_t WAIT_LIMIT_NS = 4000000000ull;   // 4 s per wait
constexpr size_t SMEM_LIMIT = 232448;               // 227 KB opt-in per block
constexpr size_t SMEM_PER_SM = 233472;              // 228 KB per SM
constexpr size_t SMEM_BLOCK_RESERVE = 1024;         // reserved by the system per resident block

// ------------------------------------------------------------------------------------------------
// PTX wrappers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of `parity` to complete.  false = gave up (abort raised).
__device__ __noinline__ bool mbar_wait_slow(uint64_t* bar, uint32_t parity,
                                            volatile int* abort_flag,
                                            uint64_t limit_ns = WAIT_LIMIT_NS) {
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if (*abort_flag) return false;
    if ((it & 255) == 0 && globaltimer() - t0 > limit_ns) {
      *abort_flag = 1;
      return false;
    }
  }
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          volatile int* abort_flag) {
  if (mbar_test(bar, parity)) return true;
  return mbar_wait_slow(bar, parity, abort_flag);
}
// Teardown wait for work this thread itself started (copies, MMAs): ignores the abort flag
// because such work completes on its own, but is still bounded in time.
__device__ __noinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 0;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if ((it & 255) == 255 && globaltimer() - t0 > WAIT_LIMIT_NS) return false;
  }
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst)),
               "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
// tcgen05.ld of 32 columns of this warp's 32 lanes; completes at the next tmem_wait
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
// wait for this thread's outstanding tcgen05.ld; the registers of the load are operands so that
// no use of them can be scheduled before the wait
__device__ __forceinline__ void tmem_wait(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                 "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// --- CTA-pair forms ------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// address of the same shared-memory variable in cluster CTA `rank`
__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}
// try_wait with cluster-scope acquire, for barriers that the partner CTA arrives at
__device__ __forceinline__ bool mbar_test_cl(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __noinline__ bool mbar_wait_cl_slow(uint64_t* bar, uint32_t parity,
                                               volatile int* abort_flag) {
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_test_cl(bar, parity)) return true;
    if (*abort_flag) return false;
    if ((it & 255) == 0 && globaltimer() - t0 > WAIT_LIMIT_NS) {
      *abort_flag = 1;
      return false;
    }
  }
}
__device__ __forceinline__ bool mbar_wait_cl(uint64_t* bar, uint32_t parity,
                                             volatile int* abort_flag) {
  if (mbar_test_cl(bar, parity)) return true;
  return mbar_wait_cl_slow(bar, parity, abort_flag);
}
template <bool PAIR>
__device__ __forceinline__ void tmem_alloc_g(uint32_t* dst, uint32_t ncols) {
  if (PAIR)
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst)),
                 "r"(ncols));
  else
    tmem_alloc(dst, ncols);
}
template <bool PAIR>
__device__ __forceinline__ void tmem_relinquish_g() {
  if (PAIR) asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::);
  else tmem_relinquish();
}
template <bool PAIR>
__device__ __forceinline__ void tmem_dealloc_g(uint32_t taddr, uint32_t ncols) {
  if (PAIR)
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
  else
    tmem_dealloc(taddr, ncols);
}
template <bool PAIR>
__device__ __forceinline__ void umma_f16_g(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                           uint32_t idesc, uint32_t accumulate) {
  if (PAIR)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
  else
    umma_f16(tmem_d, adesc, bdesc, idesc, accumulate);
}
// commit: arrive at `bar` when the MMAs issued so far are complete — in a pair, at the barrier of
// the same offset in both CTAs
template <bool PAIR>
__device__ __forceinline__ void umma_commit_g(uint64_t* bar) {
  if (PAIR) {
    const uint16_t both = 3;
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
        " [%0], %1;" ::"r"(smem_u32(bar)),
        "h"(both)
        : "memory");
  } else {
    umma_commit(bar);
  }
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFFu) >> 4);       // start address
  d |= uint64_t(1) << 16;                        // leading byte offset (unused for SW128 K-major)
  d |= uint64_t(1024 >> 4) << 32;                // stride byte offset
  d |= uint64_t(1) << 46;                        // descriptor version (sm_100)
  d |= uint64_t(2) << 61;                        // SWIZZLE_128B
  return d;
}
// Instruction descriptor, kind::f16: F32 accumulate, A/B f16 or bf16, both K-major, M×N.
__host__ __device__ constexpr uint32_t idesc_f16(bool bf16, int m, int n) {
  return (1u << 4) | ((bf16 ? 1u : 0u) << 7) | ((bf16 ? 1u : 0u) << 10) |
         (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

struct TcParams {
  int kb;           // 64-element K atoms per row
  int ksteps;       // K=16 MMA steps per tile
  int bn;           // key tile rows
  int stages;       // key tile pipeline depth
  int na;           // query tile buffers
  int kprime;
  int cand_stride;
  int bf16;
  int n_items;
  uint32_t idesc;
  int prof;         // accumulate the pipeline counters below
  const int32_t* perm;   // packed position -> original row (-1: padding)
  const int32_t* qmap;   // query row -> packed position (refine pass over a row list), or null
  const int32_t* n_items_dev;   // work-item count in device memory (refine pass), or null
  int32_t* counter;             // next unclaimed work item (zero at launch; single CTAs only)
  const uint32_t* mask;         // per work item: key tiles to visit beyond the near tiles, or null
  int mask_words;               // mask words per work item
  int near_only;                // near pass: the near tiles only
  int reverse;                  // claim the work items from the last one down
  const int32_t* claim;         // else, when set: the claim order of the work items
  const float* seed;            // per packed query row: bound on its final k'-th value, or null
  int prof_slot;                // counter block of this launch (near / main / refine)
  // refine pass split over key ranges: *split_dev work items per refine item (1: no split), each
  // writing its rows' candidate lists to part / part_thr for refine_merge
  const int32_t* split_dev;
  int2* part;
  float* part_thr;
  float* cand_val;              // near pass: also write the values of the kept candidates
  // main pass after a near pass: load every row's list from the near pass's candidates (values,
  // original rows -> packed positions through iperm) and never offer its keys again (excl)
  const float* init_val;
  const int32_t* init_idx;
  const int32_t* iperm;
  const int4* excl;
  // main pass after a pruning plan: every work item's far tiles sorted by their distance bound
  // (VisitOrder in kernels.cuh), each row's fixed radius part roff, and the flag that the lists
  // were built; null: the mask walk
  const unsigned long long* vlist;
  const int64_t* voff;
  const double* roff;
  const int32_t* vok;
  // single CTAs: the producer alone walks the key tiles and hands each tile to the MMA thread and
  // the epilogue warps with the data (stage and accumulator tags); else every role walks
  int meta_walk;
};

// Key-tile order of a query tile whose own rows lie in key tile `diag`: first the NEAR tiles
// around it (diag, diag+1, diag-1, diag+2, diag-2, clipped to the sample), then all other tiles
// in plain order.  With the cells in locality order the near tiles hold most of the rows' true
// neighbours, so the thresholds fall close to their final values at once; the plain sweep after
// them is the same for every query tile, so the CTAs stream the keys through L2 together.
constexpr int NEAR_SIDE = 2;
__device__ __forceinline__ int key_tile_at(int j, int diag, int nkt) {
  const int lo = max(0, diag - NEAR_SIDE), hi = min(nkt - 1, diag + NEAR_SIDE);
  const int np = hi - lo + 1;
  if (j >= np) {
    const int t = j - np;
    return t < lo ? t : t + np;
  }
  const int left = diag - lo, right = hi - diag;
  const int m = min(left, right);
  if (j == 0) return diag;
  if (j <= 2 * m) return (j & 1) ? diag + ((j + 1) >> 1) : diag - (j >> 1);
  return right > left ? diag + (j - m) : diag - (j - m);
}

// The key tiles of one work item in the order every role walks them: the near tiles
// (key_tile_at), then all other tiles in plain order, or only those whose bit is set in the
// item's visit mask (the pruned scan), or none (the near pass).  Every role of the CTA walks the
// same sequence, so the tiles need no hand-off between them.
struct KeyTileWalk {
  int nkt, diag, np, j;
  const uint32_t* mask;
  int w, nw;
  uint32_t cur, nxt;
  bool near_only;
  int khi = 1 << 30;     // range walks stop before this tile
  bool range = false;
  __device__ __forceinline__ void init(const WorkItem& item, int qref, int bn,
                                       const uint32_t* m, int words, bool near) {
    nkt = (item.nkeys + bn - 1) / bn;
    diag = (qref - item.key0) / bn;
    const int lo = max(0, diag - NEAR_SIDE), hi = min(nkt - 1, diag + NEAR_SIDE);
    // the near pass only needs an upper bound on each row's k'-th value: the query tile's own
    // key tile gives one (measured: all five near tiles cost more in the near pass than they
    // save in the main scan)
    np = near ? 1 : hi - lo + 1;
    j = 0;
    near_only = near;
    mask = m;
    w = 0;
    nw = words;
    cur = m ? m[0] : 0u;
    nxt = (m && words > 1) ? m[1] : 0u;     // one word ahead: its load overlaps the near tiles
  }
  // A range walk (the refine pass): no near phase, only the tiles [lo, hi), in plain order or
  // as the mask's bits.
  __device__ __forceinline__ void set_range(int lo, int hi) {
    range = true;
    np = 0;
    j = lo;
    khi = hi;
    if (mask) {
      w = lo >> 5;
      cur = w < nw ? (mask[w] & (~0u << (lo & 31))) : 0u;
      nxt = w + 1 < nw ? mask[w + 1] : 0u;
    }
  }
  // the next key tile, or -1
  __device__ __forceinline__ int next() {
    if (j < np) return key_tile_at(j++, diag, nkt);
    if (near_only) return -1;
    if (!mask) {
      if (range) return j < khi ? j++ : -1;
      return j < nkt ? key_tile_at(j++, diag, nkt) : -1;
    }
    while (cur == 0u) {
      if (++w >= nw) return -1;
      cur = nxt;
      nxt = w + 1 < nw ? mask[w + 1] : 0u;
    }
    const int b = __ffs(cur) - 1;
    cur &= cur - 1u;
    const int kt = w * 32 + b;
    return kt < khi ? kt : -1;
  }
};

// Pipeline counters (cycles / events summed over CTAs), filled when profiling is enabled:
//   0 producer waiting for a free key stage     1 MMA waiting for a loaded key tile
//   2 MMA waiting for a free accumulator         3 epilogue waiting for an accumulator
//   4 epilogue cycles in its tile loops          5 kernel cycles (thread 0)
//   6 hot chunks (any row below its threshold)   7 compactions   8 appends   9 CTAs
// one block of 16 counters per launch kind: 0 near pass, 1 main scan, 2 refine pass
constexpr int PROF_SLOTS = 3;
__device__ unsigned long long g_tc_prof[PROF_SLOTS][16];

struct SmemPlan {
  size_t a_off, b_off, sel_off, pub_off, bar_off, total;
};
// brows = key rows this CTA stages per tile (BN, or BN/2 in a CTA pair);
// nh = column groups per TMEM lane quarter (1: four epilogue warps, 2: eight)
template <int KH>
__host__ __device__ inline SmemPlan smem_plan(int kb, int brows, int stages, int na, int nh) {
  SmemPlan p;
  p.a_off = 0;
  p.b_off = p.a_off + size_t(na) * kb * BM * 128;
  p.sel_off = p.b_off + size_t(stages) * brows * 128;
  p.pub_off = p.sel_off + size_t(nh) * SelectorOf<KH>::type::smem_bytes();
  p.bar_off = p.pub_off + (nh > 1 ? size_t(2) * BM * sizeof(float) : 0);
  p.total = p.bar_off + 512 + 1024;          // barriers + slack for 1024-byte alignment
  return p;
}

// NEPI epilogue warps: 4 (one per TMEM lane quarter, all columns of a tile) or 8 (two per lane
// quarter, each filtering half of the columns into its own list; the two lists of a row share
// their thresholds while filtering and are merged when the query tile is done).
// PAIR: two-CTA clusters, 256-row work items (see the file comment).
// DUAL: two CTAs per SM.  Each CTA holds 256 TMEM columns: every 256-key tile is computed as two
// N=128 halves into two 128-column accumulators, so the MMA of the next half runs while the
// epilogue filters the current one; the two CTAs' epilogue warps share each scheduler.  Needs
// one K atom per row (the halves read the same key stage) and the tagged walk.
template <int KH, int NEPI, bool PAIR, bool DUAL>
__global__ void __launch_bounds__((DUAL ? 64 : 128) + 32 * NEPI, DUAL ? 2 : 1)
knn_tc_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const TcParams P, const WorkItem* __restrict__ items, Ctl* __restrict__ ctl,
              int32_t* __restrict__ cand_idx, float* __restrict__ cand_thr) {
  static_assert(NEPI == 4 || NEPI == 8, "four or eight epilogue warps");
  static_assert(!DUAL || (NEPI == 4 && !PAIR), "two CTAs per SM: single CTAs, four epilogue warps");
  constexpr int NH = NEPI / 4;
  constexpr int NACC = 2;                               // accumulators in TMEM
  // warps: 0 producer, 1 MMA, then (single CTAs) 2 TMEM owner and 3 pair relay, then the
  // epilogue; DUAL has no warps 2 and 3 (the producer warp owns TMEM), so that two CTAs of six
  // warps get 168 registers per thread
  constexpr int EPI0 = DUAL ? 2 : EPI_WARP0;            // first epilogue warp
  constexpr int TMEM_WARP = DUAL ? 0 : 2;
  using Sel = typename SelectorOf<KH>::type;
  extern __shared__ unsigned char smem_dyn[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~uintptr_t(1023));
  const int brows = PAIR ? P.bn / 2 : P.bn;            // key rows this CTA stages per tile
  const SmemPlan sp = smem_plan<KH>(P.kb, brows, P.stages, P.na, NH);
  unsigned char* Asm = smem + sp.a_off;
  unsigned char* Bsm = smem + sp.b_off;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + sp.bar_off);
  uint64_t* a_full = bars;                 // [2] this CTA's query rows landed
  uint64_t* a_empty = bars + 2;            // [2]
  uint64_t* acc_full = bars + 4;           // [2]
  uint64_t* acc_empty = bars + 6;          // [2]
  uint64_t* done_bar = bars + 8;           // [1]
  uint64_t* b_full = bars + 9;             // [stages <= 8] this CTA's key rows landed
  uint64_t* b_empty = bars + 17;           // [stages <= 8]
  uint64_t* qbar = bars + 25;              // [4] the two epilogue warps of a lane quarter
  uint64_t* a_peer = bars + 29;            // [2] pair: the odd CTA's query rows landed
  uint64_t* b_peer = bars + 31;            // [stages <= 8] pair: the odd CTA's key rows landed
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 39);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 40);
  uint64_t* item_full = bars + 41;         // [ITEM_RING] a claimed work item is in item_ring
  uint64_t* item_empty = bars + 45;        // [ITEM_RING] every consumer has read it
  int* item_ring = reinterpret_cast<int*>(bars + 49);   // [ITEM_RING]
  // tagged walk: the key tile a stage / an accumulator holds (-1: the item's walk ends there);
  // ordered walk: per epilogue warp the largest radius R of its rows, tagged with the work item
  // (item << 32 | float bits); bytes 408..512 of the 512-byte block
  int* stage_meta = item_ring + ITEM_RING;                  // [stages <= 8]
  int* acc_meta = stage_meta + 8;                           // [2]
  unsigned long long* rq_pub = reinterpret_cast<unsigned long long*>(bars + 56);   // [NEPI]
  float* pub = reinterpret_cast<float*>(smem + sp.pub_off);

  const int warp = warp_id(), lane = lane_id();
  const uint32_t rank = PAIR ? cluster_ctarank() : 0u;
  const bool leader = rank == 0;
  const int unit = PAIR ? int(blockIdx.x >> 1) : int(blockIdx.x);
  const int nunits = PAIR ? int(gridDim.x >> 1) : int(gridDim.x);
  const size_t a_bytes = size_t(P.kb) * BM * 128;
  const size_t b_bytes = size_t(brows) * 128;           // one K atom of this CTA's key rows
  const int acc_cols = DUAL ? P.bn / 2 : P.bn;          // TMEM columns of one accumulator
  const uint32_t tmem_cols = uint32_t(NACC * acc_cols);
  const int n_items = P.n_items_dev ? *P.n_items_dev : P.n_items;
  // the producer drives the walk from the sorted list and ends it early (single CTAs only)
  const bool ordered = !PAIR && !P.near_only && P.qmap == nullptr && P.vlist != nullptr &&
                       *P.vok != 0;
  // the producer alone walks (from the list, or the mask) and tags stages and accumulators
  const bool meta = !PAIR && (DUAL || ordered || P.meta_walk != 0);

  if (threadIdx.x == 0) {
    for (int i = 0; i < NEPI; ++i) rq_pub[i] = ~0ull;       // no item yet
    for (int i = 0; i < 2; ++i) {
      mbar_init(&a_full[i], 1);
      mbar_init(&a_empty[i], 1);
      // tagged walk: the MMA commit and the MMA thread's own arrive (after it wrote acc_meta)
      mbar_init(&acc_full[i], meta ? 2 : 1);
      mbar_init(&acc_empty[i], PAIR ? 2 * NEPI : NEPI);
      mbar_init(&a_peer[i], 1);
    }
    mbar_init(done_bar, 1);
    for (int s = 0; s < P.stages; ++s) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
      mbar_init(&b_peer[s], 1);
    }
    for (int q = 0; q < 4; ++q) mbar_init(&qbar[q], 2);
    for (int r = 0; r < ITEM_RING; ++r) {
      mbar_init(&item_full[r], 1);
      mbar_init(&item_empty[r], 1 + NEPI);   // the MMA thread and every epilogue warp
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (NH > 1)
    for (int i = threadIdx.x; i < 2 * BM; i += blockDim.x) pub[i] = F_INF;
  if (warp == TMEM_WARP) {
    tmem_alloc_g<PAIR>(tmem_slot, tmem_cols);
    tmem_relinquish_g<PAIR>();
  }
  if (warp == 0 && lane == 0) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
  }
  tc_fence_before();
  __syncthreads();
  if (PAIR) cluster_sync();               // the partner's barriers exist before any remote arrive
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const long long t_kernel0 = clock64();
  // Register split (eight epilogue warps): warpgroup 0 (producer, MMA, TMEM owner, relay) gives
  // up registers and the two epilogue warpgroups take them, one setmaxnreg per warpgroup at the
  // head of its branch.  REG_LOW·128 + REG_HIGH·256 equals the block's pool at the launch
  // allocation REG_LAUNCH; the launcher checks that allocation first, since an increase beyond
  // the pool would wait forever.

  // Work distribution.  A single CTA claims work items dynamically: its producer thread takes the
  // next item from a global counter and hands it to the MMA thread and the epilogue warps through
  // a ring in shared memory, so query tiles of very different cost spread evenly over the SMs.
  // CTA pairs keep a static round-robin assignment (both CTAs of a pair take the same items).
  int r_slot = 0, s_next = unit;
  uint32_t r_phase = 0;
  // producer: claim the next item (-1: none left) and publish it; false = the kernel is aborting
  auto claim = [&](int& it) -> bool {
    if (PAIR) {
      it = s_next < n_items ? s_next : -1;
      s_next += nunits;
      return true;
    }
    if (!mbar_wait(&item_empty[r_slot], r_phase ^ 1, abort_flag)) return false;
    int v = atomicAdd(P.counter, 1);
    v = v < n_items ? (P.claim ? P.claim[v] : (P.reverse ? n_items - 1 - v : v)) : -1;
    item_ring[r_slot] = v;
    mbar_arrive(&item_full[r_slot]);         // release: the ring entry is visible to the waiters
    if (++r_slot == ITEM_RING) { r_slot = 0; r_phase ^= 1; }
    it = v;
    return true;
  };
  // Refine items split over key ranges: work item it = (refine item it / S, range it % S).
  const int S = P.split_dev ? max(1, *P.split_dev) : 1;
  auto item_of = [&](int it) { return S > 1 ? it / S : it; };
  auto walk_init = [&](KeyTileWalk& walk, const WorkItem& w, int it) {
    const int r = item_of(it);
    walk.init(w, P.qmap ? P.qmap[w.qrow0] : w.qrow0, P.bn,
              P.mask ? P.mask + int64_t(r) * P.mask_words : nullptr, P.mask_words,
              P.near_only != 0);
    if (P.qmap) {
      const int sidx = S > 1 ? it % S : 0;
      const int chunk = (walk.nkt + S - 1) / S;
      walk.set_range(sidx * chunk, min(walk.nkt, (sidx + 1) * chunk));
    }
  };
  // consumers: the next published item, by one thread or by a whole warp (warp_wide)
  auto receive = [&](int& it, bool warp_wide) -> bool {
    if (PAIR) {
      it = s_next < n_items ? s_next : -1;
      s_next += nunits;
      return true;
    }
    bool got = mbar_wait(&item_full[r_slot], r_phase, abort_flag);
    if (warp_wide) got = __all_sync(FULL, got);
    if (!got) return false;
    const int v = *reinterpret_cast<volatile int*>(&item_ring[r_slot]);
    if (warp_wide) __syncwarp();
    if (!warp_wide || lane_id() == 0) mbar_arrive(&item_empty[r_slot]);
    if (++r_slot == ITEM_RING) { r_slot = 0; r_phase ^= 1; }
    it = v;
    return true;
  };

  if (warp < EPI0) {
    // warpgroup 0: one register decrease for the whole warpgroup (the split needs one
    // setmaxnreg per warpgroup), then the roles; warp 2 (TMEM owner) waits for the teardown
    if constexpr (NEPI == 8 && kRegSplit) reg_dec();
    if (warp == 0) {
      // ------------------------------------------------------------------ TMA producer (each CTA)
      if (lane == 0) {
        int stage = 0, abuf = 0;
        uint32_t sphase = 0, aphase = 0;
        bool ok = true;
        long long c_wait = 0, n_far = 0, n_stop = 0;
        // ordered walk: the largest radius over the item's rows, from the epilogue warps' latest
        // figures for this item (+inf while a warp has none yet); a warp quarter's two column
        // groups both bound its rows' final thresholds, so the smaller of the two counts
        auto radius_bound = [&](int it) -> double {
          float rmax = -F_INF;
          for (int q = 0; q < 4; ++q) {
            float r = F_INF;
            for (int hh = 0; hh < NH; ++hh) {
              const unsigned long long v =
                  *reinterpret_cast<volatile unsigned long long*>(&rq_pub[hh * 4 + q]);
              if (int(uint32_t(v >> 32)) == it) r = fminf(r, __uint_as_float(uint32_t(v)));
            }
            rmax = fmaxf(rmax, r);
          }
          return double(rmax) * (1.0 + 1e-9);
        };
        for (;;) {
          int it;
          if (!claim(it)) { ok = false; break; }
          if (it < 0) break;
          const WorkItem w = items[item_of(it)];
          ok = mbar_wait(&a_empty[abuf], aphase ^ 1, abort_flag);
          if (!ok) break;
          mbar_expect_tx(&a_full[abuf], uint32_t(a_bytes));
          for (int kb = 0; kb < P.kb; ++kb)
            tma_load_2d(Asm + abuf * a_bytes + size_t(kb) * BM * 128, &tmA, &a_full[abuf], kb * 64,
                        w.qrow0 + int(rank) * BM);
          if (++abuf == P.na) { abuf = 0; aphase ^= 1; }
          KeyTileWalk walk;
          walk_init(walk, w, it);
          // ordered: the near tiles, then the sorted far tiles until one is provably beyond every
          // row's current radius (then so are all later ones)
          int64_t vo = 0, vn = 0;
          int jn = 0;
          if (ordered) { vo = P.voff[it]; vn = P.voff[it + 1] - vo; }
          auto next_tile = [&]() -> int {
            if (!ordered) return walk.next();
            if (jn < walk.np) return key_tile_at(jn++, walk.diag, walk.nkt);
            const int64_t jf = jn - walk.np;
            if (jf >= vn) return -1;
            const unsigned long long e = P.vlist[vo + jf];
            const float need = __uint_as_float(uint32_t(e >> 32));
            if (need > 0.f && double(need) > radius_bound(it)) { ++n_stop; return -1; }
            ++jn;
            ++n_far;
            return int(uint32_t(e));
          };
          for (int kt = next_tile(); kt >= 0 && ok; kt = next_tile()) {
            for (int kb = 0; kb < P.kb; ++kb) {           // one pipeline stage per K atom
              const long long tw = P.prof ? clock64() : 0;
              ok = mbar_wait(&b_empty[stage], sphase ^ 1, abort_flag);
              if (P.prof) c_wait += clock64() - tw;
              if (!ok) break;
              if (meta && kb == 0) *reinterpret_cast<volatile int*>(&stage_meta[stage]) = kt;
              mbar_expect_tx(&b_full[stage], uint32_t(b_bytes));
              tma_load_2d(Bsm + stage * b_bytes, &tmB, &b_full[stage], kb * 64,
                          w.key0 + kt * P.bn + int(rank) * brows);
              if (++stage == P.stages) { stage = 0; sphase ^= 1; }
            }
          }
          if (ok && meta) {
            // the end of the item's walk: a stage that carries no keys, tile -1
            ok = mbar_wait(&b_empty[stage], sphase ^ 1, abort_flag);
            if (ok) {
              *reinterpret_cast<volatile int*>(&stage_meta[stage]) = -1;
              mbar_arrive(&b_full[stage]);
              if (++stage == P.stages) { stage = 0; sphase ^= 1; }
            }
          }
          if (!ok) break;
        }
        if (P.prof) {
          atomicAdd(&g_tc_prof[P.prof_slot][0], (unsigned long long)c_wait);
          atomicAdd(&g_tc_prof[P.prof_slot][13], (unsigned long long)n_far);
          atomicAdd(&g_tc_prof[P.prof_slot][14], (unsigned long long)n_stop);
        }
        // drain: every load this thread armed completes on its own; wait for them (bounded)
        for (int s = 0; s < P.stages; ++s) {
          // stages armed in the current lap have parity sphase for indices < stage
          const uint32_t par = s < stage ? sphase : (sphase ^ 1);
          (void)mbar_drain(&b_full[s], par);
        }
        for (int a = 0; a < P.na; ++a) {
          const uint32_t par = a < abuf ? aphase : (aphase ^ 1);
          (void)mbar_drain(&a_full[a], par);
        }
      }
    } else if (warp == 3) {
      // ------------------------------------------------------------------ relay (odd CTA of a pair)
      if (PAIR && !leader && lane == 0) {
        int stage = 0, abuf = 0;
        uint32_t sphase = 0, aphase = 0;
        bool ok = true;
        for (int it = unit; it < n_items && ok; it += nunits) {
          const WorkItem w = items[item_of(it)];
          ok = mbar_wait(&a_full[abuf], aphase, abort_flag);
          if (!ok) break;
          mbar_arrive_remote(mapa_shared(smem_u32(&a_peer[abuf]), 0));
          if (++abuf == P.na) { abuf = 0; aphase ^= 1; }
          KeyTileWalk walk;
          walk_init(walk, w, it);
          for (int kt = walk.next(); kt >= 0 && ok; kt = walk.next()) {
            for (int kb = 0; kb < P.kb; ++kb) {
              ok = mbar_wait(&b_full[stage], sphase, abort_flag);
              if (!ok) break;
              mbar_arrive_remote(mapa_shared(smem_u32(&b_peer[stage]), 0));
              if (++stage == P.stages) { stage = 0; sphase ^= 1; }
            }
          }
        }
      }
    } else if (warp == 1) {
      // ------------------------------------------------------------------ MMA issuer (even CTA)
      if (leader && lane == 0) {
        int stage = 0, abuf = 0, acc = 0;
        uint32_t sphase = 0, aphase = 0, accphase = 0;
        bool ok = true, issued = false;
        long long c_b = 0, c_acc = 0;
        for (;;) {
          int it;
          if (!receive(it, false)) { ok = false; break; }
          if (it < 0) break;
          const WorkItem w = items[item_of(it)];
          ok = mbar_wait(&a_full[abuf], aphase, abort_flag);
          if (ok && PAIR) ok = mbar_wait_cl(&a_peer[abuf], aphase, abort_flag);
          if (!ok) break;
          const uint32_t a_base = smem_u32(Asm + abuf * a_bytes);
          KeyTileWalk walk;
          if (!meta) walk_init(walk, w, it);
          for (;;) {
            int kt_meta = 0;
            if (!meta) {
              if (walk.next() < 0) break;
            } else {
              // tagged walk: the next stage names the tile, or ends the item (a stage without keys)
              const long long t1 = P.prof ? clock64() : 0;
              ok = mbar_wait(&b_full[stage], sphase, abort_flag);
              if (P.prof) c_b += clock64() - t1;
              if (!ok) break;
              const int kt = *reinterpret_cast<volatile int*>(&stage_meta[stage]);
              if (kt < 0) {
                mbar_arrive(&b_empty[stage]);
                if (++stage == P.stages) { stage = 0; sphase ^= 1; }
                break;
              }
              kt_meta = kt;
            }
            if constexpr (DUAL) {
              // the tile's two N=128 halves, each into the next free accumulator (tagged 2·kt+half);
              // the key stage is released once both halves have read it
              const uint32_t b_base = smem_u32(Bsm + stage * b_bytes);
              for (int hf = 0; hf < 2; ++hf) {
                const long long t2 = P.prof ? clock64() : 0;
                ok = mbar_wait(&acc_empty[acc], accphase ^ 1, abort_flag);
                if (P.prof) c_acc += clock64() - t2;
                if (!ok) break;
                *reinterpret_cast<volatile int*>(&acc_meta[acc]) = 2 * kt_meta + hf;
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + uint32_t(acc * acc_cols);
                const uint32_t bh = b_base + uint32_t(hf * acc_cols * 128);
                for (int ks = 0; ks < P.ksteps; ++ks)
                  umma_f16_g<false>(d_tmem, sdesc(a_base + uint32_t((ks & 3) * 32)),
                                    sdesc(bh + uint32_t((ks & 3) * 32)), P.idesc, ks > 0 ? 1u : 0u);
                umma_commit_g<false>(&acc_full[acc]);
                mbar_arrive(&acc_full[acc]);              // releases acc_meta to the epilogue
                if (++acc == NACC) { acc = 0; accphase ^= 1; }
              }
              if (!ok) break;
              umma_commit_g<false>(&b_empty[stage]);
              if (++stage == P.stages) { stage = 0; sphase ^= 1; }
              issued = true;
              continue;
            }
            const long long t2 = P.prof ? clock64() : 0;
            ok = PAIR ? mbar_wait_cl(&acc_empty[acc], accphase ^ 1, abort_flag)
                      : mbar_wait(&acc_empty[acc], accphase ^ 1, abort_flag);
            if (P.prof) c_acc += clock64() - t2;
            if (!ok) break;
            // the epilogue read this accumulator's previous tile before it released it
            if (meta) *reinterpret_cast<volatile int*>(&acc_meta[acc]) = kt_meta;
            tc_fence_after();
            const uint32_t d_tmem = tmem_base + uint32_t(acc * P.bn);
            for (int kb = 0; kb < P.kb; ++kb) {
              if (!(meta && kb == 0)) {                    // tagged: the first stage is waited for
                const long long t1 = P.prof ? clock64() : 0;
                ok = mbar_wait(&b_full[stage], sphase, abort_flag);
                if (ok && PAIR) ok = mbar_wait_cl(&b_peer[stage], sphase, abort_flag);
                if (P.prof) c_b += clock64() - t1;
                if (!ok) break;
              }
              const uint32_t b_base = smem_u32(Bsm + stage * b_bytes);
              const int ks1 = min(P.ksteps, 4 * kb + 4);
              for (int ks = 4 * kb; ks < ks1; ++ks) {
                const uint32_t ao = uint32_t((ks >> 2) * BM * 128 + (ks & 3) * 32);
                umma_f16_g<PAIR>(d_tmem, sdesc(a_base + ao), sdesc(b_base + uint32_t((ks & 3) * 32)),
                                 P.idesc, ks > 0 ? 1u : 0u);
              }
              umma_commit_g<PAIR>(&b_empty[stage]);
              if (++stage == P.stages) { stage = 0; sphase ^= 1; }
            }
            if (!ok) break;
            issued = true;
            umma_commit_g<PAIR>(&acc_full[acc]);
            if (meta) mbar_arrive(&acc_full[acc]);        // releases acc_meta to the epilogue
            if (++acc == NACC) { acc = 0; accphase ^= 1; }
          }
          if (!ok) break;
          if (meta) {
            // the end of the item for the epilogue: an accumulator turn without a tile
            ok = mbar_wait(&acc_empty[acc], accphase ^ 1, abort_flag);
            if (!ok) break;
            *reinterpret_cast<volatile int*>(&acc_meta[acc]) = -1;
            mbar_arrive(&acc_full[acc]);
            mbar_arrive(&acc_full[acc]);
            if (++acc == NACC) { acc = 0; accphase ^= 1; }
          }
          umma_commit_g<PAIR>(&a_empty[abuf]);
          if (++abuf == P.na) { abuf = 0; aphase ^= 1; }
        }
        if (issued) {
          umma_commit_g<PAIR>(done_bar);
        } else {
          mbar_arrive(done_bar);
          if (PAIR) mbar_arrive_remote(mapa_shared(smem_u32(done_bar), 1));
        }
        if (P.prof) {
          atomicAdd(&g_tc_prof[P.prof_slot][1], (unsigned long long)c_b);
          atomicAdd(&g_tc_prof[P.prof_slot][2], (unsigned long long)c_acc);
        }
      }
    }
  } else {
    // ------------------------------------------------------------------ epilogue (each CTA)
    if constexpr (NEPI == 8 && kRegSplit) reg_inc();
    const int q = warp & 3;                        // TMEM lane quarter this warp may access
    const int h = (warp - EPI0) >> 2;              // column group
    const int row = q * 32 + lane;
    Sel sel;
    sel.bind(smem + sp.sel_off + size_t(h) * Sel::smem_bytes(), row, P.kprime);
    if (NH > 1) {
      sel.pub_own = pub + h * BM + row;
      sel.pub_other = pub + (1 - h) * BM + row;
    }
    sel.reset();
    sel.prof = P.prof != 0;
    const int gcols = acc_cols / NH;               // accumulator columns of this group
    const int nch = gcols / 32;
    int acc = 0;
    uint32_t accphase = 0, qphase = 0;
    bool ok = true;
    long long c_ew = 0, c_loop = 0;
    // the two warps of a lane quarter meet here (bounded, abort-aware)
    auto quarter_sync = [&]() -> bool {
      __syncwarp();
      if (lane == 0) mbar_arrive(&qbar[q]);
      const bool r = __all_sync(FULL, mbar_wait(&qbar[q], qphase, abort_flag));
      qphase ^= 1;
      return r;
    };
    for (;;) {
      int it;
      if (!receive(it, true)) { ok = false; break; }
      if (it < 0) break;
      const WorkItem w = items[item_of(it)];
      const long long tl = P.prof ? clock64() : 0;
      // neighbour ids are packed positions here; finish() maps them to original rows
      const int nq = min(BM, w.nq - int(rank) * BM);   // this CTA's valid query rows (may be <= 0)
      const int qrow = w.qrow0 + int(rank) * BM;
      const int self = P.qmap ? (row < nq ? P.qmap[qrow + row] : -1) : qrow + row;
      sel.set_seed((P.seed && row < nq) ? P.seed[qrow + row] : F_INF);
      if (P.init_val) {
        // both column halves start from the near pass's lists (merge_from skips the copies)
        const int nv = min(32, nq - q * 32);
        if (nv > 0)
          sel.load_warp(P.init_val, P.init_idx, P.iperm, P.perm, int64_t(qrow) + q * 32, nv,
                        P.cand_stride);
        if (row < nq) {
          const int4 ex = P.excl[qrow + row];
          sel.ex_r0 = ex.x; sel.ex_r1 = ex.y; sel.ex_o0 = ex.z; sel.ex_o1 = ex.w;
        }
      }
      const int limit = w.key0 + w.nkeys;
      KeyTileWalk walk;
      if (!meta) walk_init(walk, w, it);
      // ordered: R = threshold + roff of this row, published per warp after every tile
      const double roff_row = (ordered && row < nq) ? P.roff[qrow + row] : 0.0;
      for (;;) {
        int kt = 0;
        if (!meta) {
          kt = walk.next();
          if (kt < 0) break;
        }
        const long long te = P.prof ? clock64() : 0;
        ok = __all_sync(FULL, mbar_wait(&acc_full[acc], accphase, abort_flag));
        if (P.prof) c_ew += clock64() - te;
        if (!ok) break;
        int half = 0;                      // DUAL: which N=128 half of key tile kt
        if (meta) {
          kt = *reinterpret_cast<volatile int*>(&acc_meta[acc]);
          if (kt < 0) {                    // the item's walk ended: hand the turn back
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[acc]);
            if (++acc == NACC) { acc = 0; accphase ^= 1; }
            break;
          }
          if constexpr (DUAL) { half = kt & 1; kt >>= 1; }
        }
        tc_fence_after();
        sel.refresh();
        const uint32_t t0 =
            tmem_base + uint32_t(acc * acc_cols + h * gcols) + (uint32_t(q * 32) << 16);
        const int col_base = w.key0 + kt * P.bn + half * acc_cols + h * gcols;
        // two register buffers: the next chunk's TMEM load is in flight while the current chunk
        // is filtered; the accumulator is released right after its last load completes
        uint32_t ra[32], rb[32];
        auto release = [&]() {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) {
            if (PAIR && !leader) mbar_arrive_remote(mapa_shared(smem_u32(&acc_empty[acc]), 0));
            else mbar_arrive(&acc_empty[acc]);
          }
        };
        if constexpr (NEPI == 8 && kTriBuf) {
          // With the register split: three chunk buffers.  tcgen05.wait::ld waits for all of a
          // thread's loads, so chunks go two per wait: a cycle starts with chunks c, c+1 loaded
          // and a free third buffer, loads c+2 (free buffer) and c+3 (c's buffer, once c is
          // filtered) while it filters c and c+1, then waits.  Rotating the buffers over three
          // cycles keeps them in registers.  The accumulator is released once, right after the
          // wait that covers its last chunk.
          uint32_t rc[32];
          auto ld = [&](int c, uint32_t(&x)[32]) { tmem_ld32_async(t0 + uint32_t(c * 32), x); };
          auto push = [&](int c, uint32_t(&x)[32]) {
            sel.push32(reinterpret_cast<const float(&)[32]>(x), col_base + c * 32, self, limit);
          };
          auto cycle = [&](int c, uint32_t(&x)[32], uint32_t(&y)[32], uint32_t(&z)[32]) {
            const bool l2 = c + 2 < nch, l3 = c + 3 < nch;
            if (l2) ld(c + 2, z);
            push(c, x);
            if (c + 1 < nch) {
              if (l3) ld(c + 3, x);
              push(c + 1, y);
            }
            if (l2) {
              tmem_wait(z);
              if (l3) tmem_wait(x);
              if (c + 4 >= nch) release();
            }
            return l2;                             // chunk c+2 exists: another cycle follows
          };
          ld(0, ra);
          if (nch > 1) ld(1, rb);
          tmem_wait(ra);
          if (nch > 1) tmem_wait(rb);
          if (nch <= 2) release();
          for (int c = 0;; c += 6) {
            if (!cycle(c, ra, rb, rc)) break;
            if (!cycle(c + 2, rc, ra, rb)) break;
            if (!cycle(c + 4, rb, rc, ra)) break;
          }
        } else {
          tmem_ld32_async(t0, ra);
          tmem_wait(ra);
          if (nch == 1) release();
          for (int c = 0; c < nch; c += 2) {
            const bool more = c + 1 < nch;
            if (more) tmem_ld32_async(t0 + uint32_t((c + 1) * 32), rb);
            sel.push32(reinterpret_cast<const float(&)[32]>(ra), col_base + c * 32, self, limit);
            if (more) {
              tmem_wait(rb);
              if (c + 1 == nch - 1) release();
              const bool more2 = c + 2 < nch;
              if (more2) tmem_ld32_async(t0 + uint32_t((c + 2) * 32), ra);
              sel.push32(reinterpret_cast<const float(&)[32]>(rb), col_base + (c + 1) * 32,
                         self, limit);
              if (more2) {
                tmem_wait(ra);
                if (c + 2 == nch - 1) release();
              }
            }
          }
        }
        if (++acc == NACC) { acc = 0; accphase ^= 1; }
        if (ordered) {
          // an upper bound on R over this warp's rows: thr_f (the filter threshold) bounds the
          // row's final k'-th value, roff is the fixed part; rows past the tile's end do not count
          float rr = -F_INF;
          if (row < nq) rr = __double2float_ru(double(sel.thr_f) + roff_row);
          for (int o = 16; o > 0; o >>= 1) rr = fmaxf(rr, __shfl_xor_sync(FULL, rr, o));
          if (lane == 0)
            *reinterpret_cast<volatile unsigned long long*>(&rq_pub[warp - EPI0]) =
                (static_cast<unsigned long long>(uint32_t(it)) << 32) | __float_as_uint(rr);
        }
      }
      if (!ok) break;
      const int wrow0 = q * 32;
      const int nvalid = min(32, nq - wrow0);
      auto write_out = [&]() {
        if (S > 1)
          sel.finish_partial(P.part, P.part_thr, int64_t(it) * BM + wrow0, P.perm, nvalid,
                             P.kprime);
        else
          sel.finish(cand_idx, cand_thr, P.cand_stride, P.perm, P.qmap, int64_t(qrow) + wrow0,
                     nvalid, P.kprime, P.cand_val);
      };
      if (NH == 1) {
        if (nvalid > 0)
          write_out();
        else
          sel.flush();
      } else {
        // both lists final and both published thresholds back to +inf (the partner may still be
        // filtering this tile's columns; +inf only loosens its filter), then group 0 merges
        sel.flush();
        *reinterpret_cast<volatile float*>(sel.pub_own) = F_INF;
        ok = quarter_sync();
        if (!ok) break;
        if (h == 0) {
          sel.merge_from(smem + sp.sel_off + Sel::smem_bytes());
          if (nvalid > 0) write_out();
        }
        ok = quarter_sync();                       // the partner's list is read; reuse it
        if (!ok) break;
      }
      sel.reset();
      __syncwarp();
      if (P.prof) c_loop += clock64() - tl;
    }
    if (P.prof) {
      if (lane == 0) {
        atomicAdd(&g_tc_prof[P.prof_slot][3], (unsigned long long)c_ew);
        atomicAdd(&g_tc_prof[P.prof_slot][4], (unsigned long long)c_loop);
        atomicAdd(&g_tc_prof[P.prof_slot][6], (unsigned long long)sel.n_hot);
        atomicAdd(&g_tc_prof[P.prof_slot][11], (unsigned long long)sel.n_rounds);
        atomicAdd(&g_tc_prof[P.prof_slot][12], (unsigned long long)sel.c_hot);
      }
      atomicAdd(&g_tc_prof[P.prof_slot][7], (unsigned long long)sel.n_compact);
      atomicAdd(&g_tc_prof[P.prof_slot][8], (unsigned long long)sel.n_append);
    }
  }

  __syncthreads();
  if (warp == TMEM_WARP) {
    // the even CTA's last commit marks the end of every tensor-core write to TMEM (in a pair it
    // arrives at both CTAs)
    (void)mbar_drain(done_bar, 0);
    tc_fence_after();
  }
  // a pair leaves together: no remote arrive or MMA operand read can reach a CTA that has exited
  if (PAIR) cluster_sync();
  if (warp == TMEM_WARP) tmem_dealloc_g<PAIR>(tmem_base, tmem_cols);
  if (P.prof && threadIdx.x == 0) {
    atomicAdd(&g_tc_prof[P.prof_slot][5], (unsigned long long)(clock64() - t_kernel0));
    atomicAdd(&g_tc_prof[P.prof_slot][9], 1ull);
    atomicAdd(&g_tc_prof[P.prof_slot][10], (unsigned long long)NEPI);
  }
  if (threadIdx.x == 0 && *abort_flag) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->stats[MSC_STAT_TIMEOUT]), 1ull);
    atomicExch(&ctl->timeout_flag, 1);
  }
}

// Self-test of the bounded wait: an mbarrier that nothing ever arrives at.  The wait must give
// up after `limit_ns`, raise the abort flag and let the kernel return normally.
__global__ void wait_selftest_kernel(uint64_t limit_ns, int32_t* out) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint64_t t0 = globaltimer();
    const bool ok = mbar_wait_slow(&bar, 0, &abort_flag, limit_ns);
    out[0] = ok ? 0 : 1;                                  // 1 = gave up as designed
    out[1] = abort_flag;
    out[2] = int32_t((globaltimer() - t0) / 1000000ull);  // elapsed ms
  }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn get_encode() {
  // looked up once; the initialisation of a function-local static is thread-safe
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<EncodeTiledFn>(p);
    return nullptr;
  }();
  return fn;
}

int make_map(CUtensorMap* m, const void* base, int64_t rows, int kp, int box_rows, bool bf16) {
  EncodeTiledFn enc = get_encode();
  if (!enc) { set_error("cuTensorMapEncodeTiled unavailable"); return MSC_ERR_CUDA; }
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) {
    set_error("operand base not 16-byte aligned");
    return MSC_ERR_INVALID_ARG;
  }
  cuuint64_t dims[2] = {cuuint64_t(kp), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(kp) * 2};
  cuuint32_t box[2] = {64u, cuuint32_t(box_rows)};
  cuuint32_t estr[2] = {1u, 1u};
  CUresult r = enc(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                   const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", int(r));
    return MSC_ERR_CUDA;
  }
  return MSC_OK;
}

size_t config_smem(const TcConfig& c, int kb, int na) {
  const int nh = c.epi / 4;
  const int brows = c.pair ? c.bn / 2 : c.bn;
  if (c.kpl == 32) return smem_plan<32>(kb, brows, c.stages, na, nh).total;
  if (c.kpl == 48) return smem_plan<48>(kb, brows, c.stages, na, nh).total;
  if (c.kpl == 64) return smem_plan<64>(kb, brows, c.stages, na, nh).total;
  return SIZE_MAX;
}

int pick_na(const TcConfig& c, int kb) {
  if (c.ctas == 2) return 1;
  return config_smem(c, kb, 2) <= SMEM_LIMIT ? 2 : 1;
}

template <int KH, int NEPI, bool PAIR, bool DUAL>
int launch_tc_t(const TcParams& P, const CUtensorMap& ma, const CUtensorMap& mb,
                const WorkItem* items, Ctl* ctl, int32_t* cand_idx, float* cand_thr,
                cudaStream_t st) {
  const int brows = PAIR ? P.bn / 2 : P.bn;
  const size_t smem = smem_plan<KH>(P.kb, brows, P.stages, P.na, NEPI / 4).total;
  auto kern = knn_tc_kernel<KH, NEPI, PAIR, DUAL>;
  MSC_CUDA_TRY(raise_smem_cap(kern, smem));
  if (NEPI == 8 && kRegSplit) {
    // the register split needs the block's pool at REG_LAUNCH registers per thread
    cudaFuncAttributes fa{};
    MSC_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (((fa.numRegs + 7) / 8) * 8 < REG_LAUNCH) {
      set_error("candidate kernel compiled to %d registers; its register split needs %d",
                fa.numRegs, REG_LAUNCH);
      return MSC_ERR_UNSUPPORTED;
    }
  }
  if (!PAIR) {
    const int grid = std::max(1, std::min(P.n_items, (DUAL ? 2 : 1) * num_sms()));
    kern<<<grid, (DUAL ? 64 : 128) + 32 * NEPI, smem, st>>>(ma, mb, P, items, ctl, cand_idx,
                                                             cand_thr);
    MSC_LAUNCH_CHECK();
    return MSC_OK;
  }
  // one two-CTA cluster per pair of SMs, persistent over the 256-row work items
  const int pairs = std::max(1, std::min(P.n_items, num_sms() / 2));
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(unsigned(2 * pairs));
  lc.blockDim = dim3(unsigned(128 + 32 * NEPI));
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  MSC_CUDA_TRY(cudaLaunchKernelEx(&lc, kern, ma, mb, P, items, ctl, cand_idx, cand_thr));
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

template <int NEPI, bool PAIR, bool DUAL = false>
int launch_tc_epi(const TcConfig& cfg, const TcParams& P, const CUtensorMap& ma,
                  const CUtensorMap& mb, const WorkItem* items, Ctl* ctl, int32_t* cand_idx,
                  float* cand_thr, cudaStream_t st) {
  if (cfg.kpl == 32)
    return launch_tc_t<32, NEPI, PAIR, DUAL>(P, ma, mb, items, ctl, cand_idx, cand_thr, st);
  if (cfg.kpl == 48)
    return launch_tc_t<48, NEPI, PAIR, DUAL>(P, ma, mb, items, ctl, cand_idx, cand_thr, st);
  return launch_tc_t<64, NEPI, PAIR, DUAL>(P, ma, mb, items, ctl, cand_idx, cand_thr, st);
}

}  // namespace

// out[0..15]: all launches summed; out[16 + 16·slot + i]: launch kind `slot` alone
int tc_counters(unsigned long long* out, int max) {
  unsigned long long buf[PROF_SLOTS][16];
  MSC_CUDA_TRY(cudaMemcpyFromSymbol(buf, g_tc_prof, sizeof(buf)));
  for (int i = 0; i < max && i < 16; ++i) {
    out[i] = 0;
    for (int sl = 0; sl < PROF_SLOTS; ++sl) out[i] += buf[sl][i];
  }
  for (int sl = 0; sl < PROF_SLOTS; ++sl)
    for (int i = 0; i < 16 && 16 + 16 * sl + i < max; ++i) out[16 + 16 * sl + i] = buf[sl][i];
  return MSC_OK;
}
int tc_counters_clear() {
  unsigned long long z[PROF_SLOTS][16] = {};
  MSC_CUDA_TRY(cudaMemcpyToSymbol(g_tc_prof, z, sizeof(z)));
  return MSC_OK;
}

int launch_wait_selftest(uint64_t limit_ns, int32_t* out, cudaStream_t st) {
  wait_selftest_kernel<<<1, 32, 0, st>>>(limit_ns, out);
  MSC_LAUNCH_CHECK();
  return MSC_OK;
}

bool tc_config_ok(const TcConfig& c, int kp, int kprime) {
  if (c.bn != 32 && c.bn != 64 && c.bn != 128 && c.bn != 256) return false;
  if (c.ctas != 1 && c.ctas != 2) return false;
  if (c.ctas == 2) {
    // two CTAs per SM: single CTAs, four epilogue warps, 256-key tiles computed in two halves,
    // one K atom per row; both CTAs' shared memory (and the per-block reserve) within the SM's
    if (c.pair || c.epi != 4 || c.bn != 256 || kp != 64 || c.stages < 1 || c.stages > 8)
      return false;
    if (c.kpl < kprime || (c.kpl != 32 && c.kpl != 48 && c.kpl != 64)) return false;
    if (c.cb != 16 && c.cb != 32) return false;
    return 2 * (config_smem(c, kp / 64, 1) + SMEM_BLOCK_RESERVE) <= SMEM_PER_SM;
  }
  if (c.stages < 2 || c.stages > 8) return false;
  if (c.kpl < kprime || (c.kpl != 32 && c.kpl != 48 && c.kpl != 64)) return false;
  if (c.cb != 16 && c.cb != 32) return false;
  if (c.epi != 4 && c.epi != 8) return false;
  if (c.epi == 8 && c.bn < 64) return false;         // each column group takes >= 32 columns
  if (c.pair != 0 && c.pair != 1) return false;
  if (c.pair && c.bn < 64) return false;             // each CTA stages >= 32 key rows
  return config_smem(c, kp / 64, 1) <= SMEM_LIMIT;
}

// capacity of the per-row candidate list for a k' (32, 48 or 64 slots)
int list_slots(int kprime) { return kprime <= 32 ? 32 : (kprime <= 48 ? 48 : 64); }

TcConfig tc_default_config(int prec, int d, int kprime) {
  const OpLayout L = op_layout(prec, d);
  const int kpl = list_slots(kprime);
  // Single CTAs first: CTA pairs halve the key bytes per SM and double the K-atom stages that
  // fit, but measured slower at 1.3M × 50 (1057 vs 819 ms for the candidate stage), so they are
  // taken only when nothing else fits.  N=256 key tiles (one MMA costs the same ~186 cycles at
  // N = 64..256, so only N=256 reaches the tensor peak); four epilogue warps, one list per row
  // (measured at 1.3M × 50: main scan 55.1 ms and near pass 3.9 ms, against 56.9 and 5.0 with
  // eight warps whose two column halves each keep a list), else eight; then the deepest K-atom
  // pipeline that fits
  {
    // two CTAs per SM where they fit (one K atom per row): every scheduler runs two epilogue
    // warps of different rows.  MSC_B200_DUAL=0 turns this off.
    const char* env = std::getenv("MSC_B200_DUAL");
    if (!(env && *env == '0'))
      for (int stages = 8; stages >= 1; --stages) {
        TcConfig c{256, stages, kpl, 16, 4, 0, 2};
        if (tc_config_ok(c, L.kp, kprime)) return c;
      }
  }
  for (int pair : {0, 1})
    for (int bn : {256, 128, 64, 32})
      for (int epi : {4, 8})
        for (int stages = 8; stages >= 2; --stages) {
          TcConfig c{bn, stages, kpl, 16, epi, pair};
          if (tc_config_ok(c, L.kp, kprime)) return c;
        }
  return TcConfig{64, 2, kpl, 16, 4, 0};
}

int launch_knn_tc(int prec, const TcConfig& cfg, const void* Aop, const void* Bop,
                  int64_t a_rows, int64_t b_rows, int kp, int kmma, const WorkItem* items,
                  int64_t n_items, const int32_t* perm, const int32_t* qmap,
                  const int32_t* n_items_dev, int32_t* counter, Ctl* ctl, int kprime,
                  int32_t* cand_idx, float* cand_thr, int cand_stride, cudaStream_t st,
                  const uint32_t* mask, int mask_words, bool near_only, bool reverse,
                  const float* seed, const NearInit* init, const RefineSplit* split,
                  const VisitOrder* order, const int32_t* claim) {
  const int prof_slot = near_only ? 0 : (qmap ? 2 : 1);
  if (!tc_config_ok(cfg, kp, kprime)) {
    set_error("tensor-core tile config (bn=%d stages=%d kpl=%d cb=%d epi=%d pair=%d) does not fit",
              cfg.bn, cfg.stages, cfg.kpl, cfg.cb, cfg.epi, cfg.pair);
    return MSC_ERR_INVALID_ARG;
  }
  const bool bf16 = prec != PREC_FP16;
  CUtensorMap ma, mb;
  MSC_TRY(make_map(&ma, Aop, a_rows, kp, BM, bf16));
  MSC_TRY(make_map(&mb, Bop, b_rows, kp, cfg.pair ? cfg.bn / 2 : cfg.bn, bf16));
  TcParams P;
  P.ksteps = kmma / 16;
  P.kb = (P.ksteps + 3) / 4;                           // K atoms the MMAs read
  P.bn = cfg.bn;
  P.stages = cfg.stages;
  P.na = pick_na(cfg, P.kb);
  P.kprime = kprime;
  P.cand_stride = cand_stride;
  P.bf16 = bf16;
  P.n_items = int(n_items);
  P.idesc = idesc_f16(bf16, cfg.pair ? 2 * BM : BM, cfg.ctas == 2 ? cfg.bn / 2 : cfg.bn);
  P.prof = profiling_enabled() ? 1 : 0;
  P.perm = perm;
  P.qmap = qmap;
  P.n_items_dev = n_items_dev;
  P.counter = counter;
  P.mask = mask;
  P.mask_words = mask_words;
  P.near_only = near_only ? 1 : 0;
  P.reverse = reverse ? 1 : 0;
  P.claim = claim;
  P.seed = seed;
  P.prof_slot = prof_slot;
  P.split_dev = split ? split->split_dev : nullptr;
  P.part = split ? split->part : nullptr;
  P.part_thr = split ? split->part_thr : nullptr;
  P.cand_val = init && near_only ? init->val : nullptr;
  const bool load = init && !near_only;
  P.init_val = load ? init->val : nullptr;
  P.init_idx = load ? init->idx : nullptr;
  P.iperm = load ? init->iperm : nullptr;
  P.excl = load ? init->excl : nullptr;
  const bool ord = order && order->list && !near_only && !qmap && !cfg.pair;
  P.vlist = ord ? order->list : nullptr;
  P.voff = ord ? order->off : nullptr;
  P.roff = ord ? order->roff : nullptr;
  P.vok = ord ? order->ok : nullptr;
  {
    // measured 1.7 ms faster on the 1.3M main scan (the epilogue warps read no mask words);
    // MSC_B200_META_WALK=0 gives every role its own walk
    const char* env = std::getenv("MSC_B200_META_WALK");
    P.meta_walk = (env && *env == '0') ? 0 : 1;
  }
  if (cfg.pair && (mask || near_only)) {
    set_error("pruned scans run on single CTAs only");
    return MSC_ERR_INVALID_ARG;
  }
  if (cfg.pair) {
    if (cfg.epi == 8)
      return launch_tc_epi<8, true>(cfg, P, ma, mb, items, ctl, cand_idx, cand_thr, st);
    return launch_tc_epi<4, true>(cfg, P, ma, mb, items, ctl, cand_idx, cand_thr, st);
  }
  if (cfg.ctas == 2)
    return launch_tc_epi<4, false, true>(cfg, P, ma, mb, items, ctl, cand_idx, cand_thr, st);
  if (cfg.epi == 8)
    return launch_tc_epi<8, false>(cfg, P, ma, mb, items, ctl, cand_idx, cand_thr, st);
  return launch_tc_epi<4, false>(cfg, P, ma, mb, items, ctl, cand_idx, cand_thr, st);
}

}  // namespace msc
