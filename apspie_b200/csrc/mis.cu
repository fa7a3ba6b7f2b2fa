// mis.cu -- Luby-style maximal independent set with fixed priorities, and the
// neighbour-flag SpMSpV used to validate it.
//
// Replaces spmspvMis<V>() (src/spmspvMis.cuh:150-344).  The reference rounds
// are: candidates = undecided vertices with prio > minimum (buildVector :54,
// minimum -= delta per round), expand candidates to neighbours, radix sort,
// ReduceByKey(max) of candidate priorities per neighbour (:289), a candidate
// joins when its priority beats that maximum (updateMis :64), and the
// neighbours of joiners leave (updateNeighbor :71) -- with a full D->H copy of
// the candidate vector every round (:240).  Here one persistent kernel runs
// the rounds, one pass and one bounded grid barrier each: every undecided
// vertex v scans its neighbours' states (the max-priority SpMSpV with the
// comparison fused in) and
//   * leaves (OUT) when a neighbour is IN;
//   * else joins (IN), if it is a candidate of the round, when no
//     neighbour of larger key is still undecided, and at once marks its
//     undecided neighbours OUT (they would leave next round anyway; doing
//     it now lets their other neighbours decide a round earlier);
//   * else stays, and is compacted into the next round's queue (a queued
//     vertex marked OUT meanwhile is dropped next round).
// States change in place during the pass, so a neighbour's state may be
// read before or after its own update in the same pass; the stale value is
// always "undecided" (IN and OUT are final), which only delays a decision.
// v is IN exactly when no neighbour of larger key is IN, so the set is the
// greedy MIS in descending key order for any delta, whatever the timing.
// key(v) = (prio[v] << 32) | v, so ties in priority go to the larger id and
// every round decides at least the undecided vertex of largest key.
// Self-loops are ignored.  Work per round is spread over warps with the same scan-based
// edge dealing as the traversal kernels; a per-warp shared flag array
// collects the per-vertex OR of the edge predicates.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "context.h"

namespace apspie {
namespace {

constexpr int kMisThreads = 512;
constexpr int kUndecided = -1, kOut = 0, kIn = 1;

struct MisState {
  unsigned q[3];  // queue lengths, rotating
  alignas(8) unsigned bar[2];  // grid-barrier arrival counter (64-bit)
  int err;
  int rounds;
};

__device__ __forceinline__ unsigned long long mis_key(const uint32_t *prio, int v) {
  return ((unsigned long long)__ldg(prio + v) << 32) | (unsigned)v;
}

__global__ void mis_init(int m, int32_t *state, int *queue, MisState *st) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    state[v] = kUndecided;
    queue[v] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->q[0] = (unsigned)m;
    st->q[1] = st->q[2] = 0;
    st->bar[0] = st->bar[1] = 0;
    st->err = 0;
    st->rounds = 0;
  }
}

// Deals the edges of 32 queued vertices to the lanes of a warp.  code(v, u)
// is evaluated per edge (v = owner vertex, u = neighbour); lane j gets the
// OR of the codes over the edges of the warp's j-th vertex.
template <typename Code>
__device__ __forceinline__ unsigned warp_or_edges(int v, int s, int d, const int *__restrict__ ind,
                                                  unsigned *flags, Code code) {
  const int lane = lane_id();
  flags[lane] = 0u;
  __syncwarp();
  int incl = warp_incl_scan(d);
  int excl = incl - d;
  int total = __shfl_sync(kFull, incl, 31);
  for (int e0 = 0; e0 < total; e0 += 32) {
    int e = e0 + lane;
    int owner = warp_owner(excl, e);
    int so = __shfl_sync(kFull, s, owner);
    int eo = __shfl_sync(kFull, excl, owner);
    int vo = __shfl_sync(kFull, v, owner);
    if (e < total) {
      const unsigned c = code(vo, __ldg(ind + so + (e - eo)));
      if (c) atomicOr(flags + owner, c);
    }
  }
  __syncwarp();
  return flags[lane];
}

constexpr unsigned kHitIn = 1u, kHitLarger = 2u;

__global__ void __launch_bounds__(kMisThreads)
mis_persistent(int m, const int *__restrict__ ptr, const int *__restrict__ ind,
               const uint32_t *__restrict__ prio, int32_t *state, int *qa, int *qb, MisState *st,
               double delta, int max_rounds) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  __shared__ unsigned s_flags[kMisThreads];
  __shared__ unsigned s_q;
  unsigned *flags = s_flags + 32 * warp_in_block();
  int r = 0;
  for (;; ++r) {
    if (threadIdx.x == 0) {
      s_q = __ldcg(&st->q[r % 3]);
      if (blockIdx.x == 0) st->q[(r + 2) % 3] = 0;
    }
    __syncthreads();
    const unsigned nq = s_q;
    if (nq == 0 || (max_rounds > 0 && r >= max_rounds)) break;
    // candidates of this round: prio > threshold (the reference's minimum)
    double level = 1.0 - (double)(r + 1) * delta;
    unsigned long long thr = level <= 0.0 ? 0ull : (unsigned long long)(level * 4294967296.0);
    const int *qin = (r & 1) ? qb : qa;
    int *qout = (r & 1) ? qa : qb;
    for (unsigned base = (unsigned)gwarp * 32u; base < nq; base += (unsigned)nwarps * 32u) {
      const unsigned idx = base + lane;
      int v = -1, s = 0, d = 0;
      if (idx < nq) {
        v = __ldcg(qin + idx);
        if (__ldcg(state + v) == kUndecided) {
          s = __ldg(ptr + v);
          d = __ldg(ptr + v + 1) - s;
        } else {
          v = -1;  // marked OUT by a neighbour that joined after it was queued
        }
      }
      const unsigned hit = warp_or_edges(v, s, d, ind, flags, [&](int vo, int u) -> unsigned {
        if (u == vo) return 0u;
        const int su = __ldcg(state + u);
        if (su == kIn) return kHitIn;
        return (su == kUndecided && mis_key(prio, u) > mis_key(prio, vo)) ? kHitLarger : 0u;
      });
      bool survive = false, joined = false;
      if (v >= 0) {
        const bool cand = (thr == 0ull) || ((unsigned long long)__ldg(prio + v) >= thr);
        if (hit & kHitIn) {
          state[v] = kOut;
        } else if (cand && !(hit & kHitLarger)) {
          state[v] = kIn;
          joined = true;
        } else {
          survive = true;
        }
      }
      if (__ballot_sync(kFull, joined))
        warp_or_edges(v, s, joined ? d : 0, ind, flags, [&](int vo, int u) -> unsigned {
          if (u != vo && __ldcg(state + u) == kUndecided) state[u] = kOut;
          return 0u;
        });
      unsigned slot = warp_append(survive, &st->q[(r + 1) % 3]);
      if (survive) qout[slot] = v;
    }
    if (!grid_barrier(st->bar, &st->err)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->rounds = r;
}

__global__ void neighbor_flags_kernel(int m, const int *__restrict__ ptr,
                                      const int *__restrict__ ind, const int32_t *in,
                                      int32_t *out) {
  // one warp per flagged vertex, coalesced over its out-edges
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int base = gwarp * 32; base < m; base += nwarps * 32) {
    int v = base + lane;
    bool f = v < m && in[v] != 0;
    unsigned mask = __ballot_sync(kFull, f);
    while (mask) {
      int j = __ffs(mask) - 1;
      mask &= mask - 1;
      int vj = base + j;
      int s = __ldg(ptr + vj), e = __ldg(ptr + vj + 1);
      for (int k = s + lane; k < e; k += 32) out[__ldg(ind + k)] = 1;
    }
  }
}

__global__ void zero_i32(int n, int32_t *p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
}

int mis_grid(apspie_context *ctx) {
  return occupancy_grid(ctx, (const void *)mis_persistent, kMisThreads);
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_mis(apspie_ctx ctx, int64_t nnz, int m, const int *d_ptr, const int *d_ind,
               const uint32_t *d_prio, int32_t *d_mis, float delta) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || nnz < 0 || nnz >= (int64_t)INT32_MAX)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_mis: bad sizes m=%d nnz=%lld", m,
                     (long long)nnz);
  if (!d_ptr || !d_prio || !d_mis || (nnz > 0 && !d_ind))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_mis: null pointer");
  if (!(delta > 0.0f)) delta = 1.0f;
  auto *st = (MisState *)workspace(ctx, kSlotMisState, sizeof(MisState));
  auto *qa = (int *)workspace(ctx, kSlotMisQueueA, sizeof(int) * (size_t)m);
  auto *qb = (int *)workspace(ctx, kSlotMisQueueB, sizeof(int) * (size_t)m);
  if (!st || !qa || !qb) return APSPIE_ERR_OOM;
  ctx->mis_state = st;
  int grid = clamp_grid(ctx, mis_grid(ctx));
  if (grid <= 0) return set_error(ctx, APSPIE_ERR_CUDA, "apspie_mis: occupancy query failed");
  int init_grid = std::min((m + 255) / 256, ctx->num_sms * 8);
  mis_init<<<init_grid, 256, 0, ctx->stream>>>(m, d_mis, qa, st);
  int rc = check_launch(ctx, "mis_init");
  if (rc) return rc;
  double dd = (double)delta;
  // the round cap only guards against a stalled device loop: every round
  // decides at least one vertex, so m + 1 rounds always suffice
  int max_rounds = (int)std::min(2.0e9, (double)m + 1.0 + 1.0 / dd);
  void *args[] = {&m, (void *)&d_ptr, (void *)&d_ind, (void *)&d_prio, &d_mis, &qa, &qb, &st,
                  &dd, &max_rounds};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)mis_persistent, dim3(grid),
                                              dim3(kMisThreads), args, 0, ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "mis_persistent");
  ctx->launches += 1;
  return APSPIE_OK;
}

int apspie_mis_get_rounds(apspie_ctx ctx, int *rounds) {
  APSPIE_CHECK_CTX(ctx);
  if (!rounds || !ctx->mis_state)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_mis_get_rounds: no MIS has run");
  auto *h = (MisState *)pinned(ctx, sizeof(MisState));
  if (!h) return APSPIE_ERR_OOM;
  cudaError_t e = cudaMemcpyAsync(h, ctx->mis_state, sizeof(MisState), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "apspie_mis_get_rounds");
  *rounds = h->rounds;
  if (h->err) return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_mis: grid barrier timed out");
  return APSPIE_OK;
}

int apspie_neighbor_flags(apspie_ctx ctx, int64_t nnz, int m, const int *d_ptr,
                          const int *d_ind, const int32_t *d_in, int32_t *d_out) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || nnz < 0 || !d_ptr || !d_in || !d_out || (nnz > 0 && !d_ind))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_neighbor_flags: bad arguments");
  int grid = std::min((m + 255) / 256, ctx->num_sms * 8);
  zero_i32<<<grid, 256, 0, ctx->stream>>>(m, d_out);
  neighbor_flags_kernel<<<ctx->num_sms * 4, 512, 0, ctx->stream>>>(m, d_ptr, d_ind, d_in, d_out);
  return check_launch(ctx, "neighbor_flags", 2);
}

}  // extern "C"
