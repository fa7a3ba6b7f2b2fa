// context.h -- the per-device context behind apspie_ctx.
//
// Owns the stream, a grow-only device workspace split into named slots, a
// pinned host staging word array, the last error message and a launch
// counter.  All algorithm entry points draw their scratch from here.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "apspie.h"

struct apspie_context {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  uint64_t launches = 0;

  struct Slot {
    void *ptr = nullptr;
    size_t bytes = 0;
  };
  std::vector<Slot> slots;

  // pinned host scratch for small device->host reads
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
  // ring of pinned host buffers for tables uploaded to the device (the
  // batched job table): a buffer is reused once the copy that last read it
  // has completed (its event), so a call need not wait for the stream's
  // earlier kernels.  The copy runs when the stream reaches it, so the ring
  // is as deep as the launches a caller may queue ahead of the GPU (a
  // server lane queues one batched launch per group: a ring of 4 made the
  // fifth group's launch wait for the first group's start)
  static constexpr int kUploadRing = 32;
  static constexpr size_t kUploadBytes = size_t(64) << 10;  // holds the largest job table
  void *up_pool = nullptr;  // kUploadRing buffers of kUploadBytes, allocated at first use
  void *up_host[kUploadRing] = {};
  size_t up_bytes[kUploadRing] = {};  // a buffer outside the pool when larger
  cudaEvent_t up_done[kUploadRing] = {};
  int up_next = 0;
  // test hook (apspie_debug_inject): the next workspace growth fails
  bool fail_next_alloc = false;

  // at most this many blocks per persistent launch (0: as many as fit), so
  // that two persistent kernels can share the GPU
  int max_grid = 0;
  // blocks per SM of the persistent BFS / SSSP / batched launches (0: as
  // many as fit); picked per graph by the autotuners
  int bfs_blocks_per_sm = 0;
  int sssp_blocks_per_sm = 0;
  int batch_blocks_per_sm = 0;
  // BFS tuning and the device block that holds the last run's statistics
  int bfs_alpha = 14;
  int bfs_beta = 24;
  int bfs_mode = 0;  // 0 auto, 1 push only, 2 pull only
  void *bfs_state = nullptr;  // device pointer into a workspace slot
  void *bfs_state_zeroed = nullptr;  // BFS state buffer zeroed once for the fused init
  int bfs_par = 0;                   // barrier counter set of the next BFS launch
  void *sort_err_zeroed = nullptr;   // radix sort give-up word, zeroed once when allocated
  void *sssp_state = nullptr;
  // SSSP near-far step (0: frontier Bellman-Ford)
  uint32_t sssp_delta_u32 = 0;
  float sssp_delta_f32 = 0.0f;
  int sssp_pull_alpha = 0;  // pull round when frontier out-edges * alpha > nnz (0: never)
  int sssp_pull_alpha_batch = 0;  // the same for the multi-source SSSP steps (off: measured slower)
  void *mis_state = nullptr;
  void *batch_state = nullptr;
  // SpMSpV: the bitmap path is taken when E * factor > m
  double spmspv_sort_factor = 4.0;
  // batched launches: the sources of jobs on deep graphs run as
  // single-source traversals on sub-contexts (own stream and workspace),
  // concurrently, with deep_blocks blocks in all (0: two thirds of the
  // resident ones when multi-source jobs run next to them); aux_done orders
  // their start after the context's stream
  int batch_deep_subs = 48;  // most concurrent single-source traversals (0: none)
  int deep_blocks = 0;
  cudaEvent_t aux_done = nullptr;
  std::vector<struct apspie_context *> subs;
  std::vector<cudaEvent_t> sub_done;
  int batch_subs_used = 0;  // sub-contexts the last batch ran sources on
  bool owns_stream = false;  // a sub-context's stream, destroyed with it
  // SpGEMM plan left by apspie_spgemm_symbolic for apspie_spgemm_numeric
  bool spgemm_plan_valid = false;
  const void *spgemm_plan_A = nullptr, *spgemm_plan_B = nullptr;
  int spgemm_plan_m = 0, spgemm_plan_n = 0;
  // row counts of the SpGEMM bins (symbolic and numeric) and, last, the
  // largest output row staged in global memory
  unsigned spgemm_plan_bins[16] = {};
  int spgemm_plan_words = 0;  // bitmap words per row (0: hash tables)
  long long spgemm_bitmap_max_cols = 1 << 18;
  // SpGEMM hash tables: every table holds at least table_load x its entries
  // (2 or 4; each row bin's limit is divided by table_load / 2, so rows move
  // to the next larger table); rows of at most warp_max_prod products (<= 256)
  // are one warp's work, longer ones a block's
  int spgemm_table_load = 2;
  int spgemm_warp_max_prod = 256;
  // the plan's table load, fixed by apspie_spgemm_symbolic for numeric
  int spgemm_plan_load = 2;
  // the symbolic pass's stored bitmaps (workspace slots), or null
  void *spgemm_plan_gbm = nullptr;
  void *spgemm_plan_bslot = nullptr;
  // autotuner results by graph fingerprint
  struct TuneEntry {
    uint64_t fp;
    int alpha, beta;
    float ms;
    int blocks_per_sm;
  };
  std::vector<TuneEntry> tune_cache;
  struct SsspTuneEntry {
    uint64_t fp;
    int blocks_per_sm, pull_alpha;
    float ms;
  };
  std::vector<SsspTuneEntry> sssp_tune_cache;
  struct SpgemmTuneEntry {
    uint64_t fp;
    int table_load, warp_max_prod;
    long long bitmap_max_cols;
    float ms;
  };
  std::vector<SpgemmTuneEntry> spgemm_tune_cache;
  struct BatchTuneEntry {
    uint64_t fp;
    int blocks_per_sm, deep_blocks;
    float ms;
  };
  std::vector<BatchTuneEntry> batch_tune_cache;
};

namespace apspie {

// Workspace slot ids (one buffer per id, grown on demand).
enum SlotId : int {
  kSlotBfsState = 0,
  kSlotBfsQueueA,
  kSlotBfsQueueB,
  kSlotBfsChunksA,
  kSlotBfsChunksB,
  kSlotBfsGroupMask,
  kSlotSsspState,
  kSlotSsspQueueA,
  kSlotSsspQueueB,
  kSlotSsspChunksA,
  kSlotSsspChunksB,
  kSlotSsspStamp,
  kSlotSsspNearFar,
  kSlotSsspHubs,
  kSlotSsspHubWord,
  kSlotMisState,
  kSlotMisQueueA,
  kSlotMisQueueB,
  kSlotSortKeysA,
  kSlotSortKeysB,
  kSlotSortValsA,
  kSlotSortValsB,
  kSlotSortHist,
  kSlotSortErr,  // radix sort: sticky give-up word of the look-back waits
  kSlotScan,
  kSlotDense,
  kSlotBitmap,
  kSlotMisc0,
  kSlotMisc1,
  kSlotMisc2,
  kSlotMisc3,
  kSlotMxvBuf,
  kSlotMxvFlags,
  kSlotSmall,
  kSlotBatch,
  kSlotFingerprint,
  // SpGEMM plan: kept from the symbolic phase for repeated numeric phases
  kSlotSpgProd,
  kSlotSpgLists,
  kSlotSpgCnt,
  kSlotSpgBins,
  kSlotSpgBits,
  kSlotSpgVals,
  kSlotSpgStoredBits,  // the symbolic pass's bitmaps of its bitmap rows
  kSlotSpgBitmapSlot,
  kSlotSpgSpillPos,    // numeric bitmap rows longer than one window: spilled products
  kSlotSpgSpillVal,
  kSlotCount
};

int set_error(apspie_context *ctx, int status, const char *fmt, ...);
// Returns a device buffer of at least `bytes` for slot `id` (contents
// undefined).  nullptr and an OOM error on failure.
void *workspace(apspie_context *ctx, int id, size_t bytes);
// Pinned host buffer of at least `bytes`.
void *pinned(apspie_context *ctx, size_t bytes);
// A pinned host buffer of at least `bytes` for a host-to-device upload and
// its slot: fill it, enqueue the copy, then upload_done(ctx, slot) records
// the copy's completion.  Waits only for the copy that used the buffer
// kUploadRing uploads ago.
void *upload_buffer(apspie_context *ctx, size_t bytes, int *slot);
int upload_done(apspie_context *ctx, int slot);
// Checks cudaGetLastError after launches; records the launch count.
int check_launch(apspie_context *ctx, const char *what, int nlaunches = 1);
int check_cuda(apspie_context *ctx, cudaError_t e, const char *what);

// Runs an entry point's body: a failure of its host bookkeeping
// (std::bad_alloc from a container, or another standard-library exception)
// becomes a status, so no C++ exception crosses the C ABI.
template <typename F>
int api_guard(F f) {
  try {
    return f();
  } catch (const std::bad_alloc &) {
    return APSPIE_ERR_OOM;
  } catch (const std::exception &) {
    return APSPIE_ERR_INVALID;
  }
}

}  // namespace apspie

#define APSPIE_CHECK_CTX(ctx)                                   \
  do {                                                          \
    if (!(ctx)) return APSPIE_ERR_INVALID;                      \
    cudaError_t _e = cudaSetDevice((ctx)->device);              \
    if (_e != cudaSuccess)                                      \
      return apspie::check_cuda((ctx), _e, "cudaSetDevice");    \
  } while (0)

namespace apspie {
// Fingerprint of a graph: m, nnz and its row offsets at 64 evenly spaced rows
// (synchronises the context's stream).
uint64_t graph_fingerprint(apspie_context *ctx, int m, int64_t nnz, const int *d_ptr);
// d_out[i] = d_ptr[m * i / 64] for i = 0..64 (one small launch)
int gather_offsets(apspie_context *ctx, const int *d_ptr, int m, int *d_out);

// Blocks of `kernel` (threads per block, no dynamic shared memory) that fit
// on the context's device at once: the occupancy times the SM count, cached
// per (kernel, device) under a lock (contexts may be used from several
// threads).  0 if the occupancy query fails.
int occupancy_grid(apspie_context *ctx, const void *kernel, int threads);

// Grid of a persistent launch: the occupancy-sized grid, capped by the
// context's max_grid.
inline int clamp_grid(const apspie_context *ctx, int grid) {
  return (ctx->max_grid > 0 && ctx->max_grid < grid) ? ctx->max_grid : grid;
}

// Grid of a persistent launch with a blocks-per-SM choice (0: the
// occupancy-sized grid), capped by the context's max_grid.
inline int persistent_grid(const apspie_context *ctx, int occ_grid, int blocks_per_sm) {
  int g = occ_grid;
  if (blocks_per_sm > 0 && g > blocks_per_sm * ctx->num_sms) g = blocks_per_sm * ctx->num_sms;
  return clamp_grid(ctx, g);
}
}  // namespace apspie
