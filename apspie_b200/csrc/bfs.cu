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
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kBfsThreads = 512;
constexpr int kProbe = 1;         // in-neighbours a lane probes per round in a pull level
constexpr int kTraceLevels = 64;  // levels recorded in the per-run trace

struct LevelTrace {
  int mode;  // 1 push, 2 pull
  int pad;
  unsigned long long nf, mf;
  unsigned long long t_end;      // %globaltimer at the end of the level (ns)
  unsigned long long queued;     // vertices queued from an implicit frontier (== nf when it ran)
  unsigned long long expanded;   // edges the push expansion walked (== mf)
  unsigned long long t_first;    // %globaltimer when the first block finished its share
  unsigned long long t_last;     // ... and when the last one did (the rest is barrier wait)
};

struct BfsState {
  LevelCounters c[3];
  // Queue counters of a frontier rebuilt from depth == L before a push level.
  // They must not be the level's own counters: slower blocks may still be
  // reading those to choose the direction while faster ones already append.
  // Two sets, by level parity; block 0 clears the other one each level.
  LevelCounters comp[2];
  alignas(128) unsigned bar[2];  // grid-barrier arrival counter (64-bit), separate init
  alignas(128) int err;
  int levels;
  int pull_levels;
  int par;  // counter set of the last launch with the initialisation fused in
  // Launches that clear the state themselves alternate between two barrier
  // counters and error words: a launch resets the set the next one will use
  // (the previous launch on the stream has finished, so nobody polls it).
  alignas(128) unsigned barp[2][2];
  alignas(128) int errp[2];
  // test hook (apspie_debug_inject): set, the next launch's last block leaves
  // before its first grid barrier; never cleared by the initialisation
  int inject;
  unsigned long long reached;
  unsigned long long edges;
  unsigned long long t_start;
  LevelTrace trace[kTraceLevels];
};

// Push visitor: an unvisited destination is claimed with one CAS.
struct BfsVisit {
  static constexpr bool kTwoWay = false;
  int next;
  int32_t *depth;
  __device__ __forceinline__ bool two_way() const { return false; }
  __device__ __forceinline__ bool check(unsigned, int, int u, unsigned &) const {
    return __ldcg(depth + u) == -1;
  }
  template <int N>
  __device__ __forceinline__ void commit_n(const unsigned (&)[N], const int (&)[N],
                                           const int (&u)[N], const unsigned (&)[N],
                                           const bool (&ok)[N], int (&cls)[N]) const {
    int old[N];
#pragma unroll
    for (int r = 0; r < N; ++r) old[r] = ok[r] ? atomicCAS(depth + u[r], -1, next) : 0;
#pragma unroll
    for (int r = 0; r < N; ++r) cls[r] = (ok[r] && old[r] == -1) ? 1 : 0;
  }
};

// Clears the depths (the source at 0) and, in block 0, seeds the level-0
// frontier and resets the counters and the trace.  With reset_bar the
// separate barrier counter and error word too (bfs_init only: a fused
// launch polls its own counter set, see BfsState::barp).
__device__ __forceinline__ void bfs_clear(int m, int src, int32_t *depth,
                                          const int *__restrict__ ptr, int *queue, int2 *chunks,
                                          BfsState *st, bool reset_bar) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x)
    depth[v] = (v == src) ? 0 : -1;
  if (blockIdx.x == 0) {
    seed_frontier(src, ptr, queue, chunks, &st->c[0]);
    if (threadIdx.x == 0) {
      st->c[1] = LevelCounters{0ull, 0, 0, 0ull};
      st->c[2] = LevelCounters{0ull, 0, 0, 0ull};
      st->comp[0] = LevelCounters{0ull, 0, 0, 0ull};
      st->comp[1] = LevelCounters{0ull, 0, 0, 0ull};
      if (reset_bar) st->bar[0] = st->bar[1] = 0;
      st->err = 0;
      st->levels = 0;
      st->pull_levels = 0;
      st->reached = 0;
      st->edges = 0;
    }
    for (int i = threadIdx.x; i < kTraceLevels; i += blockDim.x) {
      st->trace[i].queued = 0;
      st->trace[i].expanded = 0;
      st->trace[i].t_first = ~0ull;
      st->trace[i].t_last = 0;
    }
  }
}

__global__ void bfs_init(int m, int src, int32_t *depth, const int *__restrict__ ptr,
                         int *queue, int2 *chunks, BfsState *st) {
  bfs_clear(m, src, depth, ptr, queue, chunks, st, true);
  if (blockIdx.x == 0 && threadIdx.x == 0) st->par = -1;
}

__global__ void __launch_bounds__(kBfsThreads, 3)
bfs_persistent(int m, long long nnz, const int *__restrict__ ptr, const int *__restrict__ ind,
               const int *__restrict__ tptr, const int *__restrict__ tind, int32_t *depth,
               int *qa, int *qb, int2 *ca, int2 *cb, BfsState *st, int max_levels, int alpha,
               int beta, int mode, unsigned *gmask, int src, int init_par) {
  const int lane = lane_id();
  const int warp = warp_in_block();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  __shared__ unsigned s_q, s_chunks, s_nbig, s_nimpl;
  __shared__ unsigned long long s_edges;
  __shared__ unsigned s_found[kBfsThreads / 32];
  __shared__ int s_rank[kBfsThreads / 32][32];
  __shared__ unsigned s_bcnt;
  __shared__ unsigned long long s_bedg;
  __shared__ unsigned s_next;  // per-block group counter of pull / compaction sweeps

  // test hook: the last block leaves at once (one-shot), so the others'
  // first grid barrier waits out its bound and reports APSPIE_ERR_TIMEOUT
  __shared__ int s_leave;
  if (threadIdx.x == 0)
    s_leave = (gridDim.x > 1 && blockIdx.x == gridDim.x - 1) ? atomicExch(&st->inject, 0) : 0;
  __syncthreads();
  if (s_leave) return;
  // init_par >= 0: the launch clears the state itself (no bfs_init before
  // it) and uses barrier counter set init_par
  unsigned *bar = init_par < 0 ? st->bar : st->barp[init_par];
  int *err = init_par < 0 ? &st->err : &st->errp[init_par];
  if (init_par >= 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      *reinterpret_cast<unsigned long long *>(st->barp[init_par ^ 1]) = 0ull;
      st->errp[init_par ^ 1] = 0;
      st->par = init_par;
    }
    bfs_clear(m, src, depth, ptr, qa, ca, st, false);
    if (!grid_barrier(bar, err)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->t_start = globaltimer();
  bool pull = false;
  int pull_levels = 0;
  unsigned long long prev_nf = 0;
  unsigned long long reached = 0, explored = 0;
  int L = 0;
  for (;; ++L) {
    LevelCounters *cur = &st->c[L % 3];
    LevelCounters *nxt = &st->c[(L + 1) % 3];
    LevelCounters *clr = &st->c[(L + 2) % 3];
    if (threadIdx.x == 0) {
      const unsigned long long bc = __ldcg(&cur->bc);
      s_q = __ldcg(&cur->q);
      s_chunks = bc_chunks(bc);
      s_nbig = bc_big(bc);
      s_nimpl = __ldcg(&cur->nimpl);
      s_edges = __ldcg(&cur->edges);
      s_bcnt = 0;
      s_bedg = 0;
      s_next = 0;
      if (blockIdx.x == 0) {
        *clr = LevelCounters{0ull, 0, 0, 0ull};
        st->comp[(L + 1) & 1] = LevelCounters{0ull, 0, 0, 0ull};
      }
    }
    __syncthreads();
    unsigned nq = s_q, nch = s_chunks;
    const unsigned nimpl = s_nimpl;
    const unsigned long long nf = (unsigned long long)nq + s_nbig + nimpl;
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
      if (nimpl) {
        // the frontier came from a pull level and exists only implicitly:
        // queue it (and chunk its hubs) before expanding.  That pull level
        // left one found-mask word per 32-vertex group (gmask), so this reads
        // m / 8 bytes rather than the depth array.  Each block takes its own
        // range of groups, 32 groups per warp batch from a shared counter;
        // each round every lane with bits left hands one vertex to the
        // warp's append.
        const unsigned ngroups = (unsigned)((m + 31) / 32);
        const unsigned per_block = (ngroups + gridDim.x - 1) / gridDim.x;
        const unsigned gbeg = blockIdx.x * per_block;
        const unsigned gend = min(gbeg + per_block, ngroups);
        DiscoverAcc acc;
        for (;;) {
          unsigned g0 = 0;
          if (lane == 0) g0 = atomicAdd(&s_next, 32u);
          g0 = __shfl_sync(kFull, g0, 0);
          if (gbeg + g0 >= gend) break;
          const unsigned gw = gbeg + g0 + lane;
          unsigned bits = gw < gend ? __ldcg(gmask + gw) : 0u;
          unsigned fm;
          while ((fm = __ballot_sync(kFull, bits != 0u)) != 0u) {
            bool f[1] = {bits != 0u};
            int u[1] = {f[0] ? (int)(gw * 32u) + __ffs(bits) - 1 : 0};
            bits &= bits - 1u;
            discover_n<1, false>(f, u, ptr, qin, cin, &st->comp[L & 1], acc);
            if (lane == 0 && L < kTraceLevels)
              atomicAdd(&st->trace[L].queued, (unsigned long long)__popc(fm));
          }
        }
        flush_acc(acc, &st->comp[L & 1]);
        if (!grid_barrier(bar, err)) return;
        if (threadIdx.x == 0) {
          const unsigned long long bc = __ldcg(&st->comp[L & 1].bc);
          s_q = __ldcg(&st->comp[L & 1].q);
          s_chunks = bc_chunks(bc);
          s_nbig = bc_big(bc);
        }
        __syncthreads();
        nq = s_q;
        nch = s_chunks;
      }
      BfsVisit vis{next, depth};
      expand_push_direct(ptr, ind, qin, nq, cin, s_nbig, nch, qout, cout, nxt, cur, gwarp,
                         nwarps, [](int, bool, bool &) { return 0u; }, vis,
                         L < kTraceLevels ? &st->trace[L].expanded : nullptr);
    } else {
      ++pull_levels;
      // ---- pull: unvisited vertices look for a parent at depth L ----
      // While the frontier grows the next level will pull again, and its
      // frontier stays implicit (depth == L + 1, counted only).  Once it
      // shrinks the next level may push: each group's found-mask is then
      // kept (gmask) and, when the block has finished its range, the block
      // appends its discoveries to the next queue, so that level need not
      // rebuild the queue from the depth array behind a grid barrier.
      const bool append = nf < prev_nf;
      // The unresolved vertices of a warp share its lanes round-robin: with k
      // of them unresolved, vertex of rank j gets lanes j, j+k, j+2k, ... and
      // each of those lanes probes kProbe in-neighbours (all index loads, then
      // all depth loads), so every round keeps 32 x kProbe probes in flight and
      // a vertex leaves as soon as one probe hits.  Discoveries are counted,
      // not queued: the next frontier is depth == L + 1.
      unsigned cnt = 0;
      unsigned long long edg = 0;
      // Each block owns a contiguous range of 32-vertex groups; its warps
      // take groups from a shared counter (no warp waits at the level end on
      // a statically assigned slow group), and the depth word and in-offsets
      // of the next group are loaded while the current one is probed.
      const unsigned ngroups = (unsigned)((m + 31) / 32);
      const unsigned per_block = (ngroups + gridDim.x - 1) / gridDim.x;
      const unsigned gbeg = blockIdx.x * per_block;
      const unsigned gend = min(gbeg + per_block, ngroups);
      auto grab = [&]() {
        unsigned g = 0;
        if (lane == 0) g = atomicAdd(&s_next, 1u);
        return gbeg + __shfl_sync(kFull, g, 0);
      };
      unsigned g = grab();
      int pv = -2, ps = 0, pe = 0;  // prefetched depth and in-range of the next group
      if (g < gend) {
        int v = (int)(g * 32u) + lane;
        if (v < m) {
          pv = __ldcg(depth + v);
          ps = __ldg(tptr + v);
          pe = __ldg(tptr + v + 1);
        }
      }
      while (g < gend) {
        const int v = (int)(g * 32u) + lane;
        int s = 0, e = 0;
        if (pv == -1) {
          s = ps;
          e = pe;
        }
        const unsigned gn = grab();
        if (gn < gend) {
          int vn = (int)(gn * 32u) + lane;
          pv = -2;
          if (vn < m) {
            pv = __ldcg(depth + vn);
            ps = __ldg(tptr + vn);
            pe = __ldg(tptr + vn + 1);
          }
        }
        bool found = false;
        unsigned U = __ballot_sync(kFull, s < e);
        if (U) {
          if (lane == 0) s_found[warp] = 0u;
          __syncwarp();
        }
        while (U) {
          const int k = __popc(U);
          const bool mine = (U >> lane) & 1u;
          const int myrank = __popc(U & ((1u << lane) - 1u));
          if (mine) s_rank[warp][myrank] = lane;
          __syncwarp();
          const int per = 32 / k, extra = 32 % k;
          const int j = lane % k, slot = lane / k;
          const int nl = per + (j < extra ? 1 : 0);
          const int owner = s_rank[warp][j];
          const int so = __shfl_sync(kFull, s, owner);
          const int eo = __shfl_sync(kFull, e, owner);
          int nb[kProbe];
#pragma unroll
          for (int i = 0; i < kProbe; ++i) {
            int idx = so + slot + i * nl;
            nb[i] = idx < eo ? __ldg(tind + idx) : -1;
          }
          bool hit = false;
#pragma unroll
          for (int i = 0; i < kProbe; ++i) hit |= nb[i] >= 0 && __ldcg(depth + nb[i]) == L;
          if (hit) atomicOr(&s_found[warp], 1u << owner);
          __syncwarp();
          const unsigned fm = *(volatile unsigned *)&s_found[warp];
          if (mine) s += (per + (myrank < extra ? 1 : 0)) * kProbe;
          found = (fm >> lane) & 1u;
          U = __ballot_sync(kFull, mine && !found && s < e);
        }
        if (found) depth[v] = next;
        // the found-mask of every group, also when the discoveries are only
        // counted: a push level after this one rebuilds its queue from it
        const unsigned fw = __ballot_sync(kFull, found);
        if (lane == 0) gmask[g] = fw;
        if (!append && found) {
          ++cnt;
          edg += (unsigned long long)(__ldg(ptr + v + 1) - __ldg(ptr + v));
        }
        g = gn;
      }
      if (append) {
        // block-local append of the discoveries of [gbeg, gend): 32 groups
        // per warp batch, each round every lane with bits left hands one
        // vertex to the warp's append
        __syncthreads();
        if (threadIdx.x == 0) s_next = 0;
        __syncthreads();
        DiscoverAcc pacc;
        for (;;) {
          unsigned g0 = 0;
          if (lane == 0) g0 = atomicAdd(&s_next, 32u);
          g0 = __shfl_sync(kFull, g0, 0);
          if (gbeg + g0 >= gend) break;
          const unsigned gw = gbeg + g0 + lane;
          unsigned bits = gw < gend ? gmask[gw] : 0u;
          while (__ballot_sync(kFull, bits != 0u)) {
            bool f1[1] = {bits != 0u};
            int u1[1] = {f1[0] ? (int)(gw * 32u) + __ffs(bits) - 1 : 0};
            bits &= bits - 1u;
            discover_n<1>(f1, u1, ptr, qout, cout, nxt, pacc);
          }
        }
        flush_acc(pacc, nxt);
      }
      cnt = warp_sum(cnt);
      edg = warp_sum(edg);
      if (lane == 0 && cnt) {
        atomicAdd(&s_bcnt, cnt);
        atomicAdd(&s_bedg, edg);
      }
      __syncthreads();
      if (threadIdx.x == 0 && s_bcnt) {
        atomicAdd(&nxt->nimpl, s_bcnt);
        atomicAdd(&nxt->edges, s_bedg);
      }
    }
    prev_nf = nf;
    if (L < kTraceLevels) {
      __syncthreads();
      if (threadIdx.x == 0) {
        const unsigned long long t = globaltimer();
        atomicMin(&st->trace[L].t_first, t);
        atomicMax(&st->trace[L].t_last, t);
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && L < kTraceLevels) {
      st->trace[L].mode = pull ? 2 : 1;
      st->trace[L].nf = nf;
      st->trace[L].mf = mf;
    }
    if (!grid_barrier(bar, err)) return;
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
  return occupancy_grid(ctx, (const void *)bfs_persistent, kBfsThreads);
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
  auto *gmask = (unsigned *)workspace(ctx, kSlotBfsGroupMask, sizeof(unsigned) * ((size_t)m / 32 + 1));
  if (!st || !qa || !qb || !ca || !cb || !gmask) return APSPIE_ERR_OOM;
  ctx->bfs_state = st;
  int grid = persistent_grid(ctx, bfs_grid(ctx), ctx->bfs_blocks_per_sm);
  if (grid <= 0) return set_error(ctx, APSPIE_ERR_CUDA, "apspie_bfs: occupancy query failed");

  // the kernel clears the depths and its state itself (one grid barrier
  // instead of a separate launch); a state buffer it has not seen yet is
  // zeroed once, so both barrier counter sets start at 0
  if (ctx->bfs_state_zeroed != st) {
    cudaError_t ez = cudaMemsetAsync(st, 0, sizeof(BfsState), ctx->stream);
    if (ez != cudaSuccess) return check_cuda(ctx, ez, "apspie_bfs: state");
    ctx->bfs_state_zeroed = st;
    ctx->bfs_par = 0;
  }
  long long nnz_ll = (long long)nnz;
  int alpha = ctx->bfs_alpha, beta = ctx->bfs_beta, mode = ctx->bfs_mode;
  if (!d_tptr) mode = 1;  // no in-adjacency: push only
  int par = ctx->bfs_par;
  void *args[] = {&m,  &nnz_ll, (void *)&d_ptr, (void *)&d_ind, (void *)&d_tptr, (void *)&d_tind,
                  &d_depth, &qa, &qb, &ca, &cb, &st, &max_levels, &alpha, &beta, &mode,
                  &gmask, &src, &par};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)bfs_persistent, dim3(grid),
                                              dim3(kBfsThreads), args, 0, ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "bfs_persistent");
  ctx->bfs_par ^= 1;
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
  const int kerr = h->err ? h->err : (h->par >= 0 && h->par < 2 ? h->errp[h->par] : 0);
  if (kerr)
    return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_bfs: grid barrier timed out (status %d)",
                     kerr);
  return APSPIE_OK;
}

int apspie_bfs_set_params(apspie_ctx ctx, int alpha, int beta, int mode) {
  if (!ctx || alpha < 0 || beta < 0 || mode < 0 || mode > 2) return APSPIE_ERR_INVALID;
  ctx->bfs_alpha = alpha;
  ctx->bfs_beta = beta;
  ctx->bfs_mode = mode;
  return APSPIE_OK;
}

}  // extern "C"

extern "C" int apspie_bfs_get_trace(apspie_ctx ctx, int max_levels, int *n_out,
                                    int32_t *h_mode, int64_t *h_frontier,
                                    int64_t *h_frontier_edges, int64_t *h_ns,
                                    int64_t *h_queued, int64_t *h_expanded,
                                    int64_t *h_work_first_ns, int64_t *h_work_last_ns) {
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
    if (h_queued) h_queued[i] = (int64_t)h->trace[i].queued;
    if (h_expanded) h_expanded[i] = (int64_t)h->trace[i].expanded;
    if (h_work_first_ns) h_work_first_ns[i] = (int64_t)(h->trace[i].t_first - prev);
    if (h_work_last_ns) h_work_last_ns[i] = (int64_t)(h->trace[i].t_last - prev);
    prev = h->trace[i].t_end;
  }
  *n_out = n;
  return APSPIE_OK;
}

// ---------------------------------------------------------------------------
// BFS that allocates nothing.
//
// Some callers cannot call cudaMalloc: code running while a stream is being
// captured into a CUDA graph, real-time or embedded hosts whose device memory
// is reserved up front by a fixed budget, and plugins loaded into a process
// whose allocator they do not own.  apspie_bfs_noalloc serves them with the
// same kernels as apspie_bfs, but its scratch (the level counters, the two
// frontier queues and the two chunk lists) lives in the fixed-size device
// array below instead of a context workspace.  The array is sized for graphs
// of at most kNoAllocMaxVertices vertices and kNoAllocMaxEdges edges (about
// 14 MiB); every GPU that loads this library holds it until the process
// exits.
namespace apspie {
namespace {

constexpr int kNoAllocMaxVertices = 1 << 20;
constexpr long long kNoAllocMaxEdges = 1ll << 24;
constexpr size_t kNoAllocChunkCap = (size_t)(kNoAllocMaxEdges / kChunk + kNoAllocMaxEdges / kBigDeg + 2);

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kNaOffQa = align256(sizeof(BfsState));
constexpr size_t kNaOffQb = kNaOffQa + align256(sizeof(int) * (size_t)kNoAllocMaxVertices);
constexpr size_t kNaOffCa = kNaOffQb + align256(sizeof(int) * (size_t)kNoAllocMaxVertices);
constexpr size_t kNaOffCb = kNaOffCa + align256(sizeof(int2) * kNoAllocChunkCap);
constexpr size_t kNaOffGm = kNaOffCb + align256(sizeof(int2) * kNoAllocChunkCap);
constexpr size_t kNaBytes = kNaOffGm + align256(sizeof(unsigned) * (kNoAllocMaxVertices / 32 + 1));

static __device__ __align__(256) unsigned char g_bfs_noalloc_scratch[kNaBytes];

// Device address of the scratch array, looked up once per CUDA context (a
// __device__ array has an address per context: the device's primary
// context, or one a caller made with the driver API; after cudaDeviceReset
// the primary context is new).  In host code g_bfs_noalloc_scratch names a
// host-side stand-in, never the device memory, so it must not be passed to
// a kernel.
struct NaEntry {
  int dev;
  void *cu_ctx;  // the CUcontext current at set-up
  unsigned char *ptr;
  int grid;
};
std::mutex g_na_mutex;
std::vector<NaEntry> g_na_cache;

// The current driver context (cuCtxGetCurrent through the runtime's
// driver entry point, so the library needs no libcuda link); nullptr if
// the entry point is unavailable.
void *current_cu_ctx() {
  using CtxGetCurrent = int (*)(void **);
  static CtxGetCurrent fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (CtxGetCurrent)f;
    cudaGetLastError();
  });
  void *c = nullptr;
  if (fn && fn(&c) != 0) c = nullptr;
  return c;
}

int noalloc_setup(int dev, unsigned char **ptr, int *grid) {
  void *cu = current_cu_ctx();
  std::lock_guard<std::mutex> lock(g_na_mutex);
  for (const NaEntry &e : g_na_cache)
    if (e.dev == dev && e.cu_ctx == cu) {
      *ptr = e.ptr;
      *grid = e.grid;
      return APSPIE_OK;
    }
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_bfs_noalloc_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return APSPIE_ERR_CUDA;
  }
  int occ = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bfs_persistent, kBfsThreads, 0) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      occ < 1) {
    cudaGetLastError();
    return APSPIE_ERR_CUDA;
  }
  g_na_cache.push_back(NaEntry{dev, cu, (unsigned char *)p, occ * sms});
  *ptr = (unsigned char *)p;
  *grid = occ * sms;
  return APSPIE_OK;
}

// Copies the run's status word (0 or APSPIE_ERR_TIMEOUT) to the caller.
__global__ void bfs_write_status(const BfsState *st, int32_t *out) {
  *out = *(const volatile int *)&st->err;
}

__global__ void set_word(int *p, int v) { *p = v; }

}  // namespace
}  // namespace apspie

extern "C" int apspie_bfs_noalloc(void *stream, int src, int64_t nnz, int m, const int *d_ptr,
                                  const int *d_ind, const int *d_tptr, const int *d_tind,
                                  int32_t *d_depth, int max_levels) {
  using namespace apspie;
  if (m <= 0 || src < 0 || src >= m || nnz < 0) return APSPIE_ERR_INVALID;
  if (m > kNoAllocMaxVertices || nnz > kNoAllocMaxEdges) return APSPIE_ERR_TOO_LARGE;
  if (!d_ptr || !d_depth || (nnz > 0 && !d_ind) || (d_tptr && nnz > 0 && !d_tind))
    return APSPIE_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return APSPIE_ERR_CUDA;
  }
  unsigned char *base = nullptr;
  int grid = 0;
  int rc = noalloc_setup(dev, &base, &grid);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  auto *state = (BfsState *)base;
  auto *qa = (int *)(base + kNaOffQa);
  auto *qb = (int *)(base + kNaOffQb);
  auto *ca = (int2 *)(base + kNaOffCa);
  auto *cb = (int2 *)(base + kNaOffCb);
  auto *gmask = (unsigned *)(base + kNaOffGm);
  // bfs_init clears every counter and status word the kernel reads, so the
  // contents left by the previous call do not matter
  int init_grid = std::min((m + 255) / 256, grid * 2);
  bfs_init<<<init_grid, 256, 0, st>>>(m, src, d_depth, d_ptr, qa, ca, state);
  if (cudaGetLastError() != cudaSuccess) return APSPIE_ERR_CUDA;
  long long nnz_ll = (long long)nnz;
  int alpha = 14, beta = 24, mode = d_tptr ? 0 : 1;
  int no_fused = -1;
  void *args[] = {&m,  &nnz_ll, (void *)&d_ptr, (void *)&d_ind, (void *)&d_tptr, (void *)&d_tind,
                  &d_depth, &qa, &qb, &ca, &cb, &state, &max_levels, &alpha, &beta, &mode,
                  &gmask, &src, &no_fused};
  if (cudaLaunchCooperativeKernel((const void *)bfs_persistent, dim3(grid), dim3(kBfsThreads), args,
                                  0, st) != cudaSuccess) {
    cudaGetLastError();
    return APSPIE_ERR_CUDA;
  }
  return APSPIE_OK;
}

extern "C" int apspie_bfs_noalloc_status(void *stream, int32_t *d_status) {
  using namespace apspie;
  if (!d_status) return APSPIE_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return APSPIE_ERR_CUDA;
  }
  unsigned char *base = nullptr;
  int grid = 0;
  int rc = noalloc_setup(dev, &base, &grid);
  if (rc) return rc;
  // the status word of the one scratch array's BfsState, read after the
  // traversals queued before it on this stream
  bfs_write_status<<<1, 1, 0, (cudaStream_t)stream>>>((const BfsState *)base, d_status);
  if (cudaGetLastError() != cudaSuccess) return APSPIE_ERR_CUDA;
  return APSPIE_OK;
}

namespace apspie {

// Test hook of apspie_debug_inject for the BFS kernel: the next launch on
// ctx (ctx NULL: the next apspie_bfs_noalloc on the current device) loses
// its last block before the first grid barrier.
int bfs_inject(apspie_context *ctx) {
  BfsState *st = nullptr;
  cudaStream_t stream = nullptr;
  if (ctx) {
    st = (BfsState *)workspace(ctx, kSlotBfsState, sizeof(BfsState));
    if (!st) return APSPIE_ERR_OOM;
    if (ctx->bfs_state_zeroed != st) {
      cudaError_t ez = cudaMemsetAsync(st, 0, sizeof(BfsState), ctx->stream);
      if (ez != cudaSuccess) return check_cuda(ctx, ez, "apspie_debug_inject");
      ctx->bfs_state_zeroed = st;
      ctx->bfs_par = 0;
    }
    stream = ctx->stream;
  } else {
    int dev = 0, grid = 0;
    unsigned char *base = nullptr;
    if (cudaGetDevice(&dev) != cudaSuccess) return APSPIE_ERR_CUDA;
    int rc = noalloc_setup(dev, &base, &grid);
    if (rc) return rc;
    st = (BfsState *)base;
  }
  set_word<<<1, 1, 0, stream>>>(&st->inject, 1);
  if (cudaGetLastError() != cudaSuccess) return APSPIE_ERR_CUDA;
  return ctx ? APSPIE_OK : (cudaStreamSynchronize(stream) == cudaSuccess ? APSPIE_OK : APSPIE_ERR_CUDA);
}

}  // namespace apspie
