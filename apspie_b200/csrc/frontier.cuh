// frontier.cuh -- load-balanced push expansion of a sparse frontier, shared by
// the BFS, SSSP and batched traversal kernels.
//
// This is the SpMSpV gather of the reference (IntervalGather/IntervalExpand
// of the frontier's column segments, src/mXv.cuh:159-176) done in registers:
//   * queued vertices (degree <= kBigDeg): 32 per warp; an inclusive warp scan
//     of their degrees lays the warp's edges out flat, each round deals 32
//     consecutive edges to the lanes (coalesced reads of ind[]), and a 5-step
//     shuffle search maps an edge back to its owner lane;
//   * vertices of degree > kBigDeg are split into kChunk-edge chunks that
//     every warp of the grid takes a share of, so a small frontier of hubs
//     still spreads over the whole GPU.  They are listed once each, as
//     (vertex, first chunk index) in a "big list" whose chunk indices grow
//     with the list position; a warp finds the vertex of its first chunk by
//     a 32-way search of that list and walks on from there.  (Writing one
//     entry per chunk at discovery cost more than the expansion of small
//     levels, and is wasted when the next level pulls.)
// Rounds are issued kUnroll at a time: all index loads of the batch, then all
// visitor checks (the random loads), then the atomic commits, so each lane
// keeps several independent loads in flight.  A visitor provides
//   check(payload, k, u, &aux) -> bool   (plain loads only)
//   commit_n<N>(payload[], k[], u[], aux[], ok[], cls[])   (the atomics of
//     the N candidates for which ok[r], issued together -- each class of
//     atomic for all N before the next class -- so a batch waits for one or
//     two atomic round trips, not N dependent ones; cls[r] = 1 when u joins
//     the next frontier)
// discover_n() appends joiners (warp-aggregated) to the next queue or the
// next big list: one atomic per warp for the queue slots, one for the big
// list, whose length and chunk total share a 64-bit word so that list order
// and chunk order agree; the next frontier's edge count is summed in
// registers and added once per warp per level (flush_acc).
// expand_push() instead stages a warp's joiners in shared memory
// (WarpStage) and reserves their global slots once per kStageQ queue entries
// or kStageB big-list entries, and sums the edge tally per block: every one of
// those reservations is an atomic on a single address, and same-address
// atomics complete at about 1.1 - 1.5 G/s on a B200 against 10 - 13 G/s when
// spread over 32 or more lines (measured), so a large level that reserved per
// warp batch waited on its counters.  For the same reason each counter of a
// level sits on its own 128-byte line.
#pragma once
#include "common.cuh"

namespace apspie {

constexpr int kBigDeg = 32;   // out-degree above which a vertex is chunked
constexpr int kChunk = 128;   // edges per chunk (one unrolled batch of a warp)
constexpr int kUnroll = 4;    // rounds of 32 edges issued together

// One level's counters, each on its own 128-byte line (an L2 slice
// serialises atomics on one address; separate lines keep the queue, big-list,
// tally and hand-out atomics of a level from queueing behind each other).
struct LevelCounters {
  alignas(128) unsigned long long bc;  // low 32 bits: vertices in the big list (degree >
                                       // kBigDeg); high 32 bits: their chunks
  alignas(128) unsigned q;  // vertices in the queue (degree <= kBigDeg)
  unsigned nimpl;  // vertices of an implicit frontier (BFS pull: depth == level), not queued
  alignas(128) unsigned long long edges;  // sum of out-degrees of the frontier
  alignas(128) unsigned grab;             // queue units handed out so far while this level expands
  alignas(128) unsigned cgrab;            // chunks handed out so far
};

__device__ __forceinline__ unsigned bc_big(unsigned long long bc) { return (unsigned)bc; }
__device__ __forceinline__ unsigned bc_chunks(unsigned long long bc) { return (unsigned)(bc >> 32); }

// Per-lane tally of a warp's appends during one level, flushed once.
struct DiscoverAcc {
  unsigned long long edges = 0;
};

__device__ __forceinline__ void flush_acc(DiscoverAcc &acc, LevelCounters *nxt) {
  const unsigned long long e = warp_sum(acc.edges);
  if (lane_id() == 0 && e) atomicAdd(&nxt->edges, e);
  acc = DiscoverAcc{};
}

// Position in the big list (entries (vertex, first chunk), first chunks
// increasing) of the vertex that owns chunk c: the largest i with
// big[i].y <= c.  Warp-collective: 32 pivots per step, so a list of n
// entries takes ceil(log32 n) dependent loads.
__device__ __forceinline__ int big_search(const int2 *big, int nbig, unsigned c) {
  const int lane = lane_id();
  int lo = 0, hi = nbig;  // big[lo].y <= c < big[hi].y (big[nbig].y = infinity)
  while (hi - lo > 1) {
    const long long span = hi - lo;
    const int piv = lo + (int)(span * lane / 32);
    const bool le = (unsigned)__ldcg(&big[piv].y) <= c;
    const unsigned b = __ballot_sync(kFull, le);  // lane 0 (piv == lo) is always set
    const int last = 31 - __clz(b);
    const int nlo = lo + (int)(span * last / 32);
    const int nhi = last == 31 ? hi : lo + (int)(span * (last + 1) / 32);
    lo = nlo;
    hi = max(nhi, nlo + 1);
  }
  return lo;
}

// Capacity of a chunk list for a graph with nnz edges: every big vertex has
// more than kBigDeg edges, so there are fewer than nnz / kBigDeg of them.
inline size_t chunk_capacity(long long nnz) {
  return (size_t)(nnz / kChunk + nnz / kBigDeg + 2);
}

// Called by all 32 lanes with N candidates per lane; candidate r of a lane
// joins the next frontier when found[r].  One atomic per warp reserves the
// queue slots of all N x 32 candidates, one the big-list entries and their
// chunks; the edge tally goes to acc (kCountEdges = false leaves it alone).
template <int N, bool kCountEdges = true>
__device__ __forceinline__ void discover_n(const bool (&found)[N], const int (&u)[N],
                                           const int *__restrict__ ptr, int *qout, int2 *bout,
                                           LevelCounters *nxt, DiscoverAcc &acc) {
  const int lane = lane_id();
  int deg[N];
#pragma unroll
  for (int r = 0; r < N; ++r) deg[r] = found[r] ? __ldg(ptr + u[r] + 1) - __ldg(ptr + u[r]) : 0;
  int nsmall = 0, nbig = 0, nchunk = 0;
  unsigned long long edges = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    bool big = found[r] && deg[r] > kBigDeg;
    nsmall += (found[r] && !big) ? 1 : 0;
    nbig += big ? 1 : 0;
    nchunk += big ? (deg[r] + kChunk - 1) / kChunk : 0;
    edges += (unsigned long long)deg[r];
  }
  if (kCountEdges) acc.edges += edges;
  const int qincl = warp_incl_scan(nsmall);
  const unsigned qtot = (unsigned)__shfl_sync(kFull, qincl, 31);
  const unsigned bany = __ballot_sync(kFull, nbig > 0);
  int bincl = 0, cincl = 0;
  unsigned btot = 0, ctot = 0;
  if (bany) {
    bincl = warp_incl_scan(nbig);
    cincl = warp_incl_scan(nchunk);
    btot = (unsigned)__shfl_sync(kFull, bincl, 31);
    ctot = (unsigned)__shfl_sync(kFull, cincl, 31);
  }
  unsigned qbase = 0;
  unsigned long long bbase = 0;
  if (lane == 31) {
    if (qtot) qbase = atomicAdd(&nxt->q, qtot);
    if (btot) bbase = atomicAdd(&nxt->bc, ((unsigned long long)ctot << 32) | btot);
  }
  if (qtot) {
    unsigned qb = __shfl_sync(kFull, qbase, 31) + (unsigned)(qincl - nsmall);
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (found[r] && deg[r] <= kBigDeg) qout[qb++] = u[r];
  }
  if (bany) {
    bbase = __shfl_sync(kFull, bbase, 31);
    unsigned bi = bc_big(bbase) + (unsigned)(bincl - nbig);
    unsigned ci = bc_chunks(bbase) + (unsigned)(cincl - nchunk);
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (found[r] && deg[r] > kBigDeg) {
        bout[bi++] = make_int2(u[r], (int)ci);
        ci += (unsigned)((deg[r] + kChunk - 1) / kChunk);
      }
  }
}

// Appends up to N candidates per lane to a plain vertex list (no chunking),
// one atomic per warp.
template <int N>
__device__ __forceinline__ void append_plain(const bool (&f)[N], const int (&u)[N], int *list,
                                             unsigned *count) {
  const int lane = lane_id();
  int n = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) n += f[r] ? 1 : 0;
  const int incl = warp_incl_scan(n);
  const unsigned tot = (unsigned)__shfl_sync(kFull, incl, 31);
  if (tot == 0u) return;
  unsigned base = 0;
  if (lane == 31) base = atomicAdd(count, tot);
  base = __shfl_sync(kFull, base, 31) + (unsigned)(incl - n);
#pragma unroll
  for (int r = 0; r < N; ++r)
    if (f[r]) list[base++] = u[r];
}

// Shared-memory staging of one warp's joiners during expand_push: queue
// vertices and (vertex, chunk count) big-list entries collect here and get
// their global slots with one atomic per flush.  Warp-collective.
constexpr int kStageWarps = 16;  // warps per block of the kernels that call expand_push
constexpr int kStageQ = 256;     // queue entries per warp (>= kUnroll * 32)
constexpr int kStageB = 128;     // big-list entries per warp (>= kUnroll * 32)
static_assert(kStageQ >= kUnroll * 32 && kStageB >= kUnroll * 32,
              "a batch of joiners must fit a flushed stage");

struct WarpStage {
  int *q;
  int2 *b;  // (vertex, its chunk count)
  int nq, nb;
};

__device__ __forceinline__ void stage_flush_q(WarpStage &s, int *qout, LevelCounters *nxt) {
  if (s.nq == 0) return;
  __syncwarp();
  unsigned base = 0;
  if (lane_id() == 0) base = atomicAdd(&nxt->q, (unsigned)s.nq);
  base = __shfl_sync(kFull, base, 0);
  for (int i = lane_id(); i < s.nq; i += 32) qout[base + i] = s.q[i];
  __syncwarp();
  s.nq = 0;
}

// Reserves the staged big-list entries and their chunks with one 64-bit
// atomic (list order = chunk order) and writes (vertex, first chunk).
__device__ __forceinline__ void stage_flush_b(WarpStage &s, int2 *bout, LevelCounters *nxt) {
  if (s.nb == 0) return;
  __syncwarp();
  const int lane = lane_id();
  int cnt[kStageB / 32], excl[kStageB / 32];
  unsigned carry = 0;
#pragma unroll
  for (int i = 0; i < kStageB / 32; ++i) {
    const int j = i * 32 + lane;
    cnt[i] = j < s.nb ? s.b[j].y : 0;
    const int inc = warp_incl_scan(cnt[i]);
    excl[i] = (int)carry + inc - cnt[i];
    carry += (unsigned)__shfl_sync(kFull, inc, 31);
  }
  unsigned long long base = 0;
  if (lane == 0)
    base = atomicAdd(&nxt->bc, ((unsigned long long)carry << 32) | (unsigned)s.nb);
  base = __shfl_sync(kFull, base, 0);
  const unsigned bi = bc_big(base), ci = bc_chunks(base);
#pragma unroll
  for (int i = 0; i < kStageB / 32; ++i) {
    const int j = i * 32 + lane;
    if (j < s.nb) bout[bi + j] = make_int2(s.b[j].x, (int)(ci + (unsigned)excl[i]));
  }
  __syncwarp();
  s.nb = 0;
}

// discover_n into the warp's stage: candidate r of a lane joins when
// found[r]; the stage is flushed first when the batch would not fit.
template <int N>
__device__ __forceinline__ void stage_n(const bool (&found)[N], const int (&u)[N],
                                        const int *__restrict__ ptr, WarpStage &s, int *qout,
                                        int2 *bout, LevelCounters *nxt, DiscoverAcc &acc) {
  const unsigned any = __ballot_sync(kFull, [&] {
    bool a = false;
#pragma unroll
    for (int r = 0; r < N; ++r) a |= found[r];
    return a;
  }());
  if (!any) return;
  int deg[N];
#pragma unroll
  for (int r = 0; r < N; ++r) deg[r] = found[r] ? __ldg(ptr + u[r] + 1) - __ldg(ptr + u[r]) : 0;
  int nsmall = 0, nbig = 0;
  unsigned long long edges = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const bool big = found[r] && deg[r] > kBigDeg;
    nsmall += (found[r] && !big) ? 1 : 0;
    nbig += big ? 1 : 0;
    edges += (unsigned long long)deg[r];
  }
  acc.edges += edges;
  const int qincl = warp_incl_scan(nsmall);
  const int qtot = __shfl_sync(kFull, qincl, 31);
  if (qtot) {
    if (s.nq + qtot > kStageQ) stage_flush_q(s, qout, nxt);
    int at = s.nq + qincl - nsmall;
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (found[r] && deg[r] <= kBigDeg) s.q[at++] = u[r];
    s.nq += qtot;
  }
  if (__ballot_sync(kFull, nbig > 0)) {
    const int bincl = warp_incl_scan(nbig);
    const int btot = __shfl_sync(kFull, bincl, 31);
    if (s.nb + btot > kStageB) stage_flush_b(s, bout, nxt);
    int at = s.nb + bincl - nbig;
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (found[r] && deg[r] > kBigDeg) s.b[at++] = make_int2(u[r], (deg[r] + kChunk - 1) / kChunk);
    s.nb += btot;
  }
  __syncwarp();
}

// Seeds a frontier of one vertex (used by the init kernels; block-wide).
__device__ __forceinline__ void seed_frontier(int src, const int *__restrict__ ptr, int *queue,
                                              int2 *big, LevelCounters *c) {
  if (threadIdx.x == 0) {
    const int deg = __ldg(ptr + src + 1) - __ldg(ptr + src);
    *c = LevelCounters{0ull, 0, 0, 0ull};
    if (deg > kBigDeg) {
      big[0] = make_int2(src, 0);
      c->bc = ((unsigned long long)((deg + kChunk - 1) / kChunk) << 32) | 1ull;
    } else {
      queue[0] = src;
      c->q = 1;
    }
    c->edges = (unsigned long long)deg;
  }
}

// Chunks of the big vertices, in runs of consecutive chunks: the warp finds
// the vertex of a run's first chunk and walks on; when load() skips the
// vertex, the rest of its chunks in the run are passed over.  With at most two chunks
// per warp every warp takes its own run (no counter traffic); larger levels
// hand runs of about a quarter of a warp's share (at least two chunks) out
// on demand from the level's counter, because equal chunk counts are not
// equal work (a chunk whose targets improve appends and chunks others).
template <typename Load, typename Visit>
__device__ __forceinline__ void expand_chunks(const int *__restrict__ ptr,
                                              const int *__restrict__ ind, const int2 *bin,
                                              unsigned nbig, unsigned nch, int *qout, int2 *bout,
                                              LevelCounters *nxt, int gwarp, int nwarps, Load load,
                                              Visit &visit, DiscoverAcc &acc,
                                              unsigned long long &nwalk, unsigned *cgrab,
                                              WarpStage &stg) {
  const int lane = lane_id();
  const bool dynamic = nch > 2u * (unsigned)nwarps;
  const unsigned run = dynamic ? max(2u, nch / ((unsigned)nwarps * 4u))
                               : (nch + (unsigned)nwarps - 1) / (unsigned)nwarps;
  const bool two_way = visit.two_way();
  for (int turn = 0;; ++turn) {
    unsigned c_beg;
    if (dynamic) {
      c_beg = 0;
      if (lane == 0) c_beg = atomicAdd(cgrab, run);
      c_beg = __shfl_sync(kFull, c_beg, 0);
    } else {
      c_beg = turn == 0 ? (unsigned)gwarp * run : nch;
    }
    if (c_beg >= nch) break;
    const unsigned c_end = min(c_beg + run, nch);
    int bi = big_search(bin, (int)nbig, c_beg);
    int2 bcur = __ldcg(bin + bi);
    unsigned bnext = bi + 1 < (int)nbig ? (unsigned)__ldcg(&bin[bi + 1].y) : 0xffffffffu;
    for (unsigned c = c_beg; c < c_end; ++c) {
      while (c >= bnext) {
        ++bi;
        bcur = __ldcg(bin + bi);
        bnext = bi + 1 < (int)nbig ? (unsigned)__ldcg(&bin[bi + 1].y) : 0xffffffffu;
      }
      const int v = bcur.x;
      bool skip = false;
      const unsigned pay = load(v, false, skip);
      if (skip) {
        // the loader skips the vertex: none of its chunks in this run
        c = min(bnext, c_end) - 1u;
        continue;
      }
      const int s = __ldg(ptr + v) + (int)(c - (unsigned)bcur.y) * kChunk;
      const int e = min(s + kChunk, __ldg(ptr + v + 1));
      nwalk += (unsigned long long)(e - s);
      for (int k0 = s; k0 < e; k0 += 32 * kUnroll) {
        int uu[kUnroll];
        unsigned aux[kUnroll];
        bool ok[kUnroll];
#pragma unroll
        for (int r = 0; r < kUnroll; ++r) {
          int k = k0 + r * 32 + lane;
          uu[r] = k < e ? __ldg(ind + k) : -1;
        }
#pragma unroll
        for (int r = 0; r < kUnroll; ++r)
          ok[r] = uu[r] >= 0 && visit.check(pay, k0 + r * 32 + lane, uu[r], aux[r]);
        bool f[kUnroll], g[kUnroll];
        int cls[kUnroll], kk[kUnroll];
        unsigned pp[kUnroll];
#pragma unroll
        for (int r = 0; r < kUnroll; ++r) {
          kk[r] = k0 + r * 32 + lane;
          pp[r] = pay;
        }
        visit.template commit_n<kUnroll>(pp, kk, uu, aux, ok, cls);
#pragma unroll
        for (int r = 0; r < kUnroll; ++r) {
          f[r] = cls[r] == 1;
          g[r] = cls[r] == 2;
        }
        stage_n<kUnroll>(f, uu, ptr, stg, qout, bout, nxt, acc);
        if constexpr (Visit::kTwoWay) {
          if (two_way) {
            append_plain<kUnroll>(g, uu, visit.far_list, visit.far_count);
            visit.note_far(cls, aux);
          }
        }
      }
    }
  }
}

// Push expansion of (qin[0..nq), cin[0..nch)); every thread of every block
// calls it (it synchronises the block).  `load(v, whole, skip)` gives the
// 32-bit payload of a source vertex (e.g. its distance), broadcast to its
// edges; whole is true when the call covers all of v's edges (a queued
// vertex) and false for one chunk of a big vertex; the loader may set skip
// to leave v (or this chunk and the rest of the vertex's chunks in the run)
// unexpanded, e.g. when v was already expanded with the same distance.  visit.commit returns a
// class: 0 = nothing, 1 = joins the next frontier, 2 (visitors with kTwoWay,
// when visit.two_way()) = goes to the visitor's secondary list
// (visit.far_list / visit.far_count, appended without chunking), 3 = a
// secondary-list member already listed; visit.note_far sees the classes and
// the visitor's aux values of each batch.  Queue units come first and hub
// chunks (finer grained) after them, so the chunks even out the end of the
// level.  *walked (may be NULL) gets the edges walked.
template <typename Load, typename Visit>
__device__ __forceinline__ void expand_push(const int *__restrict__ ptr,
                                            const int *__restrict__ ind, const int *qin,
                                            unsigned nq, const int2 *bin, unsigned nbig,
                                            unsigned nch, int *qout, int2 *bout,
                                            LevelCounters *nxt, LevelCounters *cur, int gwarp,
                                            int nwarps, Load load, Visit &visit,
                                            unsigned long long *walked = nullptr) {
  __shared__ int s_stq[kStageWarps][kStageQ];
  __shared__ int2 s_stb[kStageWarps][kStageB];
  __shared__ unsigned long long s_blk_edges, s_blk_walk;
  const int lane = lane_id();
  if (threadIdx.x == 0) {
    s_blk_edges = 0;
    s_blk_walk = 0;
  }
  __syncthreads();
  WarpStage stg{s_stq[warp_in_block()], s_stb[warp_in_block()], 0, 0};
  unsigned long long nwalk = 0;
  DiscoverAcc acc;
  const bool two_way = visit.two_way();
  // queue units of 32 vertices (at most 32 x kBigDeg edges): one per warp in
  // turn when there are few, else handed out on demand from the level's
  // counter, so a warp that drew heavy units takes fewer of them
  const unsigned nunits = (nq + 31u) / 32u;
  const bool dynamic = nunits > (unsigned)nwarps;
  for (unsigned turn = 0;; ++turn) {
    unsigned unit;
    if (dynamic) {
      unit = 0;
      if (lane == 0) unit = atomicAdd(&cur->grab, 1u);
      unit = __shfl_sync(kFull, unit, 0);
    } else {
      unit = (unsigned)gwarp + turn * (unsigned)nwarps;
    }
    const unsigned base = unit * 32u;
    if (base >= nq) break;
    unsigned idx = base + lane;
    int v = idx < nq ? __ldcg(qin + idx) : -1;
    int s = 0, d = 0;
    unsigned pay = 0;
    if (v >= 0) {
      s = __ldg(ptr + v);
      d = __ldg(ptr + v + 1) - s;
      bool skip = false;
      pay = load(v, true, skip);
      if (skip) d = 0;
    }
    int incl = warp_incl_scan(d);
    int excl = incl - d;
    int total = __shfl_sync(kFull, incl, 31);
    nwalk += (unsigned long long)(lane == 0 ? total : 0);
    for (int e0 = 0; e0 < total; e0 += 32 * kUnroll) {
      int kk[kUnroll], uu[kUnroll];
      unsigned pp[kUnroll], aux[kUnroll];
      bool ok[kUnroll];
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) {
        int e = e0 + r * 32 + lane;
        int owner = warp_owner(excl, e);
        int so = __shfl_sync(kFull, s, owner);
        int eo = __shfl_sync(kFull, excl, owner);
        pp[r] = __shfl_sync(kFull, pay, owner);
        kk[r] = e < total ? so + (e - eo) : -1;
      }
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) uu[r] = kk[r] >= 0 ? __ldg(ind + kk[r]) : -1;
#pragma unroll
      for (int r = 0; r < kUnroll; ++r)
        ok[r] = uu[r] >= 0 && visit.check(pp[r], kk[r], uu[r], aux[r]);
      bool f[kUnroll], g[kUnroll];
      int cls[kUnroll];
      visit.template commit_n<kUnroll>(pp, kk, uu, aux, ok, cls);
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) {
        f[r] = cls[r] == 1;
        g[r] = cls[r] == 2;
      }
      stage_n<kUnroll>(f, uu, ptr, stg, qout, bout, nxt, acc);
      if constexpr (Visit::kTwoWay) {
        if (two_way) {
          append_plain<kUnroll>(g, uu, visit.far_list, visit.far_count);
          visit.note_far(cls, aux);
        }
      }
    }
  }
  unsigned long long cwalk = 0;
  expand_chunks(ptr, ind, bin, nbig, nch, qout, bout, nxt, gwarp, nwarps, load, visit, acc, cwalk,
                &cur->cgrab, stg);
  stage_flush_q(stg, qout, nxt);
  stage_flush_b(stg, bout, nxt);
  // per-block sums of the next frontier's edges and of the edges walked
  const unsigned long long e = warp_sum(acc.edges);
  nwalk += lane == 0 ? cwalk : 0;
  const unsigned long long wk = warp_sum(nwalk);
  if (lane == 0) {
    if (e) atomicAdd(&s_blk_edges, e);
    if (wk) atomicAdd(&s_blk_walk, wk);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_blk_edges) atomicAdd(&nxt->edges, s_blk_edges);
    if (walked && s_blk_walk) atomicAdd(walked, s_blk_walk);
  }
}

// ---- direct form (BFS): joiners reserve their slots per warp batch ----
// The frontier expansion without staging: no block-wide synchronisation, so
// a level with a handful of vertices costs less (BFS push levels are small;
// its large levels pull).  Chunks of the big vertices, in runs of
// consecutive chunks: the warp finds the vertex of a run's first chunk and
// walks on.  With at most two chunks
// per warp every warp takes its own run (no counter traffic: a level's
// worth of same-address atomics from every warp costs microseconds); larger
// levels hand runs of about an eighth of a warp's share out on demand from
// the level's counter, because equal chunk counts are not equal work (a
// chunk whose targets improve appends and chunks others).
template <typename Load, typename Visit>
__device__ __forceinline__ void expand_chunks_direct(const int *__restrict__ ptr,
                                              const int *__restrict__ ind, const int2 *bin,
                                              unsigned nbig, unsigned nch, int *qout, int2 *bout,
                                              LevelCounters *nxt, int gwarp, int nwarps, Load load,
                                              Visit &visit, DiscoverAcc &acc,
                                              unsigned long long &nwalk, unsigned *cgrab) {
  const int lane = lane_id();
  const bool dynamic = nch > 2u * (unsigned)nwarps;
  const unsigned run = dynamic ? max(1u, nch / ((unsigned)nwarps * 8u))
                               : (nch + (unsigned)nwarps - 1) / (unsigned)nwarps;
  for (int turn = 0;; ++turn) {
    unsigned c_beg;
    if (dynamic) {
      c_beg = 0;
      if (lane == 0) c_beg = atomicAdd(cgrab, run);
      c_beg = __shfl_sync(kFull, c_beg, 0);
    } else {
      c_beg = turn == 0 ? (unsigned)gwarp * run : nch;
    }
    if (c_beg >= nch) break;
    const unsigned c_end = min(c_beg + run, nch);
    int bi = big_search(bin, (int)nbig, c_beg);
    int2 bcur = __ldcg(bin + bi);
    unsigned bnext = bi + 1 < (int)nbig ? (unsigned)__ldcg(&bin[bi + 1].y) : 0xffffffffu;
    for (unsigned c = c_beg; c < c_end; ++c) {
      while (c >= bnext) {
        ++bi;
        bcur = __ldcg(bin + bi);
        bnext = bi + 1 < (int)nbig ? (unsigned)__ldcg(&bin[bi + 1].y) : 0xffffffffu;
      }
      const int v = bcur.x;
      const int s = __ldg(ptr + v) + (int)(c - (unsigned)bcur.y) * kChunk;
      const int e = min(s + kChunk, __ldg(ptr + v + 1));
      nwalk += (unsigned long long)(e - s);
      bool skip = false;
      const unsigned pay = load(v, false, skip);
      for (int k0 = s; k0 < e; k0 += 32 * kUnroll) {
        int uu[kUnroll];
        unsigned aux[kUnroll];
        bool ok[kUnroll];
#pragma unroll
        for (int r = 0; r < kUnroll; ++r) {
          int k = k0 + r * 32 + lane;
          uu[r] = k < e ? __ldg(ind + k) : -1;
        }
#pragma unroll
        for (int r = 0; r < kUnroll; ++r)
          ok[r] = uu[r] >= 0 && visit.check(pay, k0 + r * 32 + lane, uu[r], aux[r]);
        bool f[kUnroll], g[kUnroll];
        int cls[kUnroll], kk[kUnroll];
        unsigned pp[kUnroll];
#pragma unroll
        for (int r = 0; r < kUnroll; ++r) {
          kk[r] = k0 + r * 32 + lane;
          pp[r] = pay;
        }
        visit.template commit_n<kUnroll>(pp, kk, uu, aux, ok, cls);
#pragma unroll
        for (int r = 0; r < kUnroll; ++r) {
          f[r] = cls[r] == 1;
          g[r] = cls[r] == 2;
        }
        discover_n<kUnroll>(f, uu, ptr, qout, bout, nxt, acc);
        if constexpr (Visit::kTwoWay) {
          append_plain<kUnroll>(g, uu, visit.far_list, visit.far_count);
          visit.note_far(cls, aux);
        }
      }
    }
  }
}

// Push expansion of (qin[0..nq), cin[0..nch)) without staging.  `load(v,
// whole, skip)` gives the 32-bit payload of a source vertex, broadcast to
// its edges (skip is ignored on this path).
// visit.commit returns a class: 0 = nothing, 1 = joins the next frontier,
// 2 (visitors with kTwoWay) = goes to the visitor's secondary list
// (visit.far_list / visit.far_count, appended without chunking), 3 = a
// secondary-list member already listed; visit.note_far sees the classes
// and the visitor's aux values of each batch.
template <typename Load, typename Visit>
__device__ __forceinline__ void expand_push_direct(const int *__restrict__ ptr,
                                            const int *__restrict__ ind, const int *qin,
                                            unsigned nq, const int2 *bin, unsigned nbig,
                                            unsigned nch, int *qout, int2 *bout,
                                            LevelCounters *nxt, LevelCounters *cur, int gwarp,
                                            int nwarps, Load load, Visit &visit,
                                            unsigned long long *walked = nullptr) {
  const int lane = lane_id();
  unsigned long long nwalk = 0;
  DiscoverAcc acc;
  expand_chunks_direct(ptr, ind, bin, nbig, nch, qout, bout, nxt, gwarp, nwarps, load, visit, acc, nwalk,
                &cur->cgrab);
  // queue units of 32 vertices (at most 32 x kBigDeg edges): one per warp in
  // turn on small levels, handed out on demand from the level's counter on
  // large ones, so a warp that drew heavy units takes fewer of them
  const unsigned nunits = (nq + 31u) / 32u;
  const bool dynamic = nunits > 2u * (unsigned)nwarps;
  for (unsigned turn = 0;; ++turn) {
    unsigned unit;
    if (dynamic) {
      unit = 0;
      if (lane == 0) unit = atomicAdd(&cur->grab, 1u);
      unit = __shfl_sync(kFull, unit, 0);
    } else {
      unit = (unsigned)gwarp + turn * (unsigned)nwarps;
    }
    const unsigned base = unit * 32u;
    if (base >= nq) break;
    unsigned idx = base + lane;
    int v = idx < nq ? __ldcg(qin + idx) : -1;
    int s = 0, d = 0;
    unsigned pay = 0;
    if (v >= 0) {
      s = __ldg(ptr + v);
      d = __ldg(ptr + v + 1) - s;
      bool skip = false;
      pay = load(v, false, skip);
    }
    int incl = warp_incl_scan(d);
    int excl = incl - d;
    int total = __shfl_sync(kFull, incl, 31);
    nwalk += (unsigned long long)total;
    for (int e0 = 0; e0 < total; e0 += 32 * kUnroll) {
      int kk[kUnroll], uu[kUnroll];
      unsigned pp[kUnroll], aux[kUnroll];
      bool ok[kUnroll];
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) {
        int e = e0 + r * 32 + lane;
        int owner = warp_owner(excl, e);
        int so = __shfl_sync(kFull, s, owner);
        int eo = __shfl_sync(kFull, excl, owner);
        pp[r] = __shfl_sync(kFull, pay, owner);
        kk[r] = e < total ? so + (e - eo) : -1;
      }
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) uu[r] = kk[r] >= 0 ? __ldg(ind + kk[r]) : -1;
#pragma unroll
      for (int r = 0; r < kUnroll; ++r)
        ok[r] = uu[r] >= 0 && visit.check(pp[r], kk[r], uu[r], aux[r]);
      bool f[kUnroll], g[kUnroll];
      int cls[kUnroll];
      visit.template commit_n<kUnroll>(pp, kk, uu, aux, ok, cls);
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) {
        f[r] = cls[r] == 1;
        g[r] = cls[r] == 2;
      }
      discover_n<kUnroll>(f, uu, ptr, qout, bout, nxt, acc);
      if constexpr (Visit::kTwoWay) {
        append_plain<kUnroll>(g, uu, visit.far_list, visit.far_count);
        visit.note_far(cls, aux);
      }
    }
  }
  flush_acc(acc, nxt);
  if (walked && lane == 0 && nwalk) atomicAdd(walked, nwalk);
}

}  // namespace apspie
