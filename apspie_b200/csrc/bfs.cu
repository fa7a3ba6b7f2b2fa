// bfs.cu -- direction-optimising BFS as one persistent kernel per traversal.
//
// Replaces the reference's level loop of mXv + addResult (src/bfs.cuh:87-110)
// and the keys-only spmspvBfs (src/spmspvBfs.cuh:150-224).  The reference does
// ~15 launches, 3 host syncs and a cudaMalloc per level; here one cooperative
// kernel runs every level, separated by a bounded software grid barrier.
//
// Per level L (frontier = vertices with depth L):
//   push (top-down): the frontier queue is expanded with a warp-level
//     scan-based gather (32 queued vertices per warp, edges dealt round-robin
//     to lanes, coalesced reads of the column segments); vertices of degree
//     > kBigDeg are split into kChunk-edge chunks shared by all warps.
//     Discovery is an atomicCAS on depth (the visited mask update fused into
//     the SpMSpV, replacing addResult, src/bfs.cuh:16-24).
//   pull (bottom-up): every unvisited vertex scans its neighbours, one warp
//     per vertex, until one has depth L (ballot early exit).
// The switch follows Beamer's rule: push->pull when the frontier's edges
// exceed (unexplored edges)/alpha, pull->push when the frontier has fewer
// than m/beta vertices.  Discovered vertices are appended to the next queue
// with one atomic per warp; the per-level counters rotate over three slots so
// no block reads a counter while another resets it.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "context.h"
#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kBfsThreads = 512;
constexpr int kProbe = 4;         // in-neighbours a lane probes alone in a pull level
constexpr int kTraceLevels = 64;  // levels recorded in the per-run trace

struct LevelTrace {
  int mode;  // 1 push, 2 pull
  int pad;
  unsigned long long nf, mf;
  unsigned long long t_end;  // %globaltimer at the end of the level (ns)
};

struct BfsState {
  LevelCounters c[3];
  unsigned bar[2];
  int err;
  int levels;
  int pull_levels;
  int pad;
  unsigned long long reached;
  unsigned long long edges;
  unsigned long long t_start;
  LevelTrace trace[kTraceLevels];
};

// Push visitor: an unvisited destination is claimed with one CAS.
struct BfsVisit {
  int next;
  int32_t *depth;
  __device__ __forceinline__ bool check(unsigned, int, int u, unsigned &) const {
    return __ldcg(depth + u) == -1;
  }
  __device__ __forceinline__ bool commit(unsigned, int, int u, unsigned) const {
    return atomicCAS(depth + u, -1, next) == -1;
  }
};

__global__ void bfs_init(int m, int src, int32_t *depth, const int *__restrict__ ptr,
                         int *queue, int2 *chunks, BfsState *st) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x)
    depth[v] = (v == src) ? 0 : -1;
  if (blockIdx.x == 0) {
    seed_frontier(src, ptr, queue, chunks, &st->c[0]);
    if (threadIdx.x == 0) {
      st->c[1] = LevelCounters{0, 0, 0, 0, 0ull};
      st->c[2] = LevelCounters{0, 0, 0, 0, 0ull};
      st->bar[0] = st->bar[1] = 0;
      st->err = 0;
      st->levels = 0;
      st->pull_levels = 0;
      st->reached = 0;
      st->edges = 0;
    }
  }
}

__global__ void __launch_bounds__(kBfsThreads, 3)
bfs_persistent(int m, long long nnz, const int *__restrict__ ptr, const int *__restrict__ ind,
               const int *__restrict__ tptr, const int *__restrict__ tind, int32_t *depth, int *qa, int *qb, int2 *ca, int2 *cb, BfsState *st,
               int max_levels, int alpha, int beta, int mode) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  __shared__ unsigned s_q, s_chunks, s_nbig;
  __shared__ unsigned long long s_edges;
  __shared__ unsigned s_found[kBfsThreads / 32];
  const int warp = warp_in_block();

  if (blockIdx.x == 0 && threadIdx.x == 0) st->t_start = globaltimer();
  bool pull = false;
  int pull_levels = 0;
  unsigned long long reached = 0, explored = 0;
  int L = 0;
  for (;; ++L) {
    LevelCounters *cur = &st->c[L % 3];
    LevelCounters *nxt = &st->c[(L + 1) % 3];
    LevelCounters *clr = &st->c[(L + 2) % 3];
    if (threadIdx.x == 0) {
      s_q = __ldcg(&cur->q);
      s_chunks = __ldcg(&cur->chunks);
      s_nbig = __ldcg(&cur->nbig);
      s_edges = __ldcg(&cur->edges);
      if (blockIdx.x == 0) {
        clr->q = 0;
        clr->chunks = 0;
        clr->nbig = 0;
        clr->edges = 0;
      }
    }
    __syncthreads();
    const unsigned nq = s_q, nch = s_chunks;
    const unsigned long long nf = (unsigned long long)nq + s_nbig;
    const unsigned long long mf = s_edges;
    if (nf == 0) break;
    reached += nf;
    explored += mf;
    if (max_levels > 0 && L + 1 >= max_levels) {
      ++L;
      break;
    }
    const long long unexplored = nnz - (long long)explored;
    if (mode == 1) {
      pull = false;
    } else if (mode == 2) {
      pull = true;
    } else if (!pull) {
      if ((long long)mf * alpha > unexplored) pull = true;
    } else if ((long long)nf * beta < (long long)m) {
      pull = false;
    }
    int *qin = (L & 1) ? qb : qa;
    int *qout = (L & 1) ? qa : qb;
    int2 *cin = (L & 1) ? cb : ca;
    int2 *cout = (L & 1) ? ca : cb;
    const int next = L + 1;

    if (!pull) {
      BfsVisit vis{next, depth};
      expand_push(ptr, ind, qin, nq, cin, nch, qout, cout, nxt, gwarp, nwarps,
                  [](int) { return 0u; }, vis);
    } else {
      ++pull_levels;
      // ---- pull: unvisited vertices look for a parent at depth L ----
      // Each lane first probes kProbe in-neighbours of its own vertex (all
      // index loads, then all depth loads).  The remaining in-neighbours of
      // the still-unresolved vertices of the warp are then laid out flat
      // (warp scan) and dealt 32 x kUnroll at a time, like a push gather; a
      // hit sets the owner's bit in a per-warp mask, slots of resolved owners
      // are skipped, and the warp stops once every owner is resolved.
      for (int base = gwarp * 32; base < m; base += nwarps * 32) {
        int v = base + lane;
        int s = 0, e = 0;
        bool found = false;
        if (v < m && __ldcg(depth + v) == -1) {
          s = __ldg(tptr + v);
          e = __ldg(tptr + v + 1);
        }
        if (s < e) {
          int nb[kProbe];
#pragma unroll
          for (int i = 0; i < kProbe; ++i) nb[i] = s + i < e ? __ldg(tind + s + i) : -1;
#pragma unroll
          for (int i = 0; i < kProbe; ++i) found |= nb[i] >= 0 && __ldcg(depth + nb[i]) == L;
          s = min(s + kProbe, e);
        }
        int d = found ? 0 : e - s;
        int incl = warp_incl_scan(d);
        int excl = incl - d;
        int total = __shfl_sync(kFull, incl, 31);
        if (total) {
          const unsigned want = __ballot_sync(kFull, d > 0);
          if (lane == 0) s_found[warp] = 0u;
          __syncwarp();
          for (int e0 = 0; e0 < total; e0 += 32 * kUnroll) {
            int nb[kUnroll], own[kUnroll];
            const unsigned done = *(volatile unsigned *)&s_found[warp];
#pragma unroll
            for (int r = 0; r < kUnroll; ++r) {
              int ee = e0 + r * 32 + lane;
              int owner = warp_owner(excl, ee);
              int so = __shfl_sync(kFull, s, owner);
              int eo = __shfl_sync(kFull, excl, owner);
              own[r] = owner;
              nb[r] = (ee < total && !((done >> owner) & 1u)) ? __ldg(tind + so + (ee - eo)) : -1;
            }
#pragma unroll
            for (int r = 0; r < kUnroll; ++r)
              if (nb[r] >= 0 && __ldcg(depth + nb[r]) == L) atomicOr(&s_found[warp], 1u << own[r]);
            __syncwarp();
            if ((*(volatile unsigned *)&s_found[warp] & want) == want) break;
          }
          found |= (*(volatile unsigned *)&s_found[warp] >> lane) & 1u;
          __syncwarp();
        }
        if (found) depth[v] = next;
        discover(found, v, ptr, qout, cout, nxt);
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && L < kTraceLevels) {
      st->trace[L].mode = pull ? 2 : 1;
      st->trace[L].nf = nf;
      st->trace[L].mf = mf;
    }
    if (!grid_barrier(st->bar, &st->err)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0 && L < kTraceLevels) st->trace[L].t_end = globaltimer();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->levels = L;
    st->pull_levels = pull_levels;
    st->reached = reached;
    st->edges = explored;
  }
}

int bfs_grid(apspie_context *ctx) {
  static int cached_dev = -1, cached_grid = 0;
  if (cached_dev == ctx->device && cached_grid > 0) return cached_grid;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bfs_persistent, kBfsThreads, 0) !=
          cudaSuccess ||
      occ < 1) {
    cudaGetLastError();
    return 0;
  }
  cached_dev = ctx->device;
  cached_grid = occ * ctx->num_sms;
  return cached_grid;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_bfs(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
               const int *d_ind, const int *d_tptr, const int *d_tind, int32_t *d_depth,
               int max_levels) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || src < 0 || src >= m)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_bfs: src %d outside [0,%d)", src, m);
  if (nnz < 0 || nnz >= (int64_t)INT32_MAX)
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "apspie_bfs: nnz %lld exceeds int32 offsets",
                     (long long)nnz);
  if (!d_ptr || !d_depth || (nnz > 0 && !d_ind) || (d_tptr && nnz > 0 && !d_tind))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_bfs: null pointer");
  size_t chunk_cap = chunk_capacity(nnz);
  auto *st = (BfsState *)workspace(ctx, kSlotBfsState, sizeof(BfsState));
  auto *qa = (int *)workspace(ctx, kSlotBfsQueueA, sizeof(int) * (size_t)m);
  auto *qb = (int *)workspace(ctx, kSlotBfsQueueB, sizeof(int) * (size_t)m);
  auto *ca = (int2 *)workspace(ctx, kSlotBfsChunksA, sizeof(int2) * chunk_cap);
  auto *cb = (int2 *)workspace(ctx, kSlotBfsChunksB, sizeof(int2) * chunk_cap);
  if (!st || !qa || !qb || !ca || !cb) return APSPIE_ERR_OOM;
  ctx->bfs_state = st;
  int grid = bfs_grid(ctx);
  if (grid <= 0) return set_error(ctx, APSPIE_ERR_CUDA, "apspie_bfs: occupancy query failed");

  int init_grid = std::min((m + 255) / 256, ctx->num_sms * 8);
  bfs_init<<<init_grid, 256, 0, ctx->stream>>>(m, src, d_depth, d_ptr, qa, ca, st);
  int rc = check_launch(ctx, "bfs_init");
  if (rc) return rc;
  long long nnz_ll = (long long)nnz;
  int alpha = ctx->bfs_alpha, beta = ctx->bfs_beta, mode = ctx->bfs_mode;
  if (!d_tptr) mode = 1;  // no in-adjacency: push only
  void *args[] = {&m,  &nnz_ll, (void *)&d_ptr, (void *)&d_ind, (void *)&d_tptr, (void *)&d_tind,
                  &d_depth, &qa, &qb, &ca, &cb, &st, &max_levels, &alpha, &beta, &mode};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)bfs_persistent, dim3(grid),
                                              dim3(kBfsThreads), args, 0, ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "bfs_persistent");
  ctx->launches += 1;
  return APSPIE_OK;
}

int apspie_bfs_get_stats(apspie_ctx ctx, apspie_bfs_stats *out) {
  APSPIE_CHECK_CTX(ctx);
  if (!out || !ctx->bfs_state)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_bfs_get_stats: no BFS has run");
  auto *h = (BfsState *)pinned(ctx, sizeof(BfsState));
  if (!h) return APSPIE_ERR_OOM;
  cudaError_t e = cudaMemcpyAsync(h, ctx->bfs_state, sizeof(BfsState), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "apspie_bfs_get_stats");
  out->levels = h->levels;
  out->pull_levels = h->pull_levels;
  out->vertices_reached = (int64_t)h->reached;
  out->edges_traversed = (int64_t)h->edges;
  if (h->err)
    return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_bfs: grid barrier timed out (status %d)",
                     h->err);
  return APSPIE_OK;
}

int apspie_bfs_set_params(apspie_ctx ctx, int alpha, int beta, int mode) {
  if (!ctx || alpha <= 0 || beta <= 0 || mode < 0 || mode > 2) return APSPIE_ERR_INVALID;
  ctx->bfs_alpha = alpha;
  ctx->bfs_beta = beta;
  ctx->bfs_mode = mode;
  return APSPIE_OK;
}

}  // extern "C"

extern "C" int apspie_bfs_get_trace(apspie_ctx ctx, int max_levels, int *n_out,
                                    int32_t *h_mode, int64_t *h_frontier,
                                    int64_t *h_frontier_edges, int64_t *h_ns) {
  APSPIE_CHECK_CTX(ctx);
  if (!ctx->bfs_state || max_levels < 0 || !n_out)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_bfs_get_trace: no BFS has run");
  auto *h = (BfsState *)pinned(ctx, sizeof(BfsState));
  if (!h) return APSPIE_ERR_OOM;
  cudaError_t e = cudaMemcpyAsync(h, ctx->bfs_state, sizeof(BfsState), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "apspie_bfs_get_trace");
  int n = std::min(std::min(max_levels, kTraceLevels), std::max(0, h->levels - 1));
  unsigned long long prev = h->t_start;
  for (int i = 0; i < n; ++i) {
    if (h_mode) h_mode[i] = h->trace[i].mode;
    if (h_frontier) h_frontier[i] = (int64_t)h->trace[i].nf;
    if (h_frontier_edges) h_frontier_edges[i] = (int64_t)h->trace[i].mf;
    if (h_ns) h_ns[i] = (int64_t)(h->trace[i].t_end - prev);
    prev = h->trace[i].t_end;
  }
  *n_out = n;
  return APSPIE_OK;
}
