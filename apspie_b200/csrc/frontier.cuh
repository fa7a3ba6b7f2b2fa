// frontier.cuh -- load-balanced push expansion of a sparse frontier, shared by
// the BFS, SSSP and batched traversal kernels.
//
// This is the SpMSpV gather of the reference (IntervalGather/IntervalExpand
// of the frontier's column segments, src/mXv.cuh:159-176) done in registers:
//   * queued vertices (degree <= kBigDeg): 32 per warp; an inclusive warp scan
//     of their degrees lays the warp's edges out flat, each round deals 32
//     consecutive edges to the lanes (coalesced reads of ind[]), and a 5-step
//     shuffle search maps an edge back to its owner lane;
//   * vertices of degree > kBigDeg are split into kChunk-edge chunks, listed
//     as (vertex, chunk) pairs that every warp of the grid pulls from, so a
//     small frontier of hubs still spreads over the whole GPU.
// Rounds are issued kUnroll at a time: all index loads of the batch, then all
// visitor checks (the random loads), then the atomic commits, so each lane
// keeps several independent loads in flight.  A visitor provides
//   check(payload, k, u, &aux) -> bool   (plain loads only)
//   commit(payload, k, u, aux) -> bool   (atomics; true = u joins the next frontier)
// discover_n() appends joiners (warp-aggregated) to the next queue or, for
// big vertices, writes their chunk entries cooperatively.  Every warp of the
// grid appends to the same counters, and same-address atomics serialise in
// L2, so an append costs ONE returning atomic: queue and chunk-list lengths
// share a 64-bit word and are reserved together, while the big-vertex count
// and the next frontier's edge count are summed in registers and added once
// per warp per level (flush_acc).
#pragma once
#include "common.cuh"

namespace apspie {

constexpr int kBigDeg = 64;   // out-degree above which a vertex is chunked
constexpr int kChunk = 128;   // edges per chunk (one unrolled batch of a warp)
constexpr int kUnroll = 4;    // rounds of 32 edges issued together

struct LevelCounters {
  unsigned long long qc;  // low 32 bits: vertices in the queue (degree <= kBigDeg);
                          // high 32 bits: entries in the chunk list
  unsigned nbig;          // vertices in the chunk list
  unsigned nimpl;         // vertices of an implicit frontier (BFS pull: depth == level), not queued
  unsigned long long edges;  // sum of out-degrees of the frontier
};

__device__ __forceinline__ unsigned qc_queue(unsigned long long qc) { return (unsigned)qc; }
__device__ __forceinline__ unsigned qc_chunks(unsigned long long qc) { return (unsigned)(qc >> 32); }

// Per-lane tallies of a warp's appends during one level, flushed once.
struct DiscoverAcc {
  unsigned nbig = 0;
  unsigned long long edges = 0;
};

__device__ __forceinline__ void flush_acc(DiscoverAcc &acc, LevelCounters *nxt) {
  const unsigned b = warp_sum(acc.nbig);
  const unsigned long long e = warp_sum(acc.edges);
  if (lane_id() == 0) {
    if (b) atomicAdd(&nxt->nbig, b);
    if (e) atomicAdd(&nxt->edges, e);
  }
  acc = DiscoverAcc{};
}

// Capacity of a chunk list for a graph with nnz edges: every big vertex has
// more than kBigDeg edges, so there are fewer than nnz / kBigDeg of them.
inline size_t chunk_capacity(long long nnz) {
  return (size_t)(nnz / kChunk + nnz / kBigDeg + 2);
}

// Called by all 32 lanes with N candidates per lane; candidate r of a lane
// joins the next frontier when found[r].  One atomic per warp reserves the
// queue slots and chunk entries of all N x 32 candidates; the big-vertex and
// edge tallies go to acc (kCountEdges = false leaves the edge tally alone).
template <int N, bool kCountEdges = true>
__device__ __forceinline__ void discover_n(const bool (&found)[N], const int (&u)[N],
                                           const int *__restrict__ ptr, int *qout, int2 *cout,
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
  acc.nbig += (unsigned)nbig;
  if (kCountEdges) acc.edges += edges;
  const int qincl = warp_incl_scan(nsmall);
  const int cincl = warp_incl_scan(nchunk);
  const unsigned qtot = (unsigned)__shfl_sync(kFull, qincl, 31);
  const unsigned ctot = (unsigned)__shfl_sync(kFull, cincl, 31);
  if ((qtot | ctot) == 0u) return;
  unsigned long long base = 0;
  if (lane == 31) base = atomicAdd(&nxt->qc, ((unsigned long long)ctot << 32) | qtot);
  base = __shfl_sync(kFull, base, 31);
  // queue slots
  if (qtot) {
    unsigned qbase = qc_queue(base) + (unsigned)(qincl - nsmall);
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (found[r] && deg[r] <= kBigDeg) qout[qbase++] = u[r];
  }
  // chunk entries of big vertices, written cooperatively
  if (ctot) {
    unsigned cbase = qc_chunks(base) + (unsigned)(cincl - nchunk);
#pragma unroll
    for (int r = 0; r < N; ++r) {
      bool big = found[r] && deg[r] > kBigDeg;
      int nch = big ? (deg[r] + kChunk - 1) / kChunk : 0;
      unsigned rm = __ballot_sync(kFull, big);
      while (rm) {
        int j = __ffs(rm) - 1;
        rm &= rm - 1;
        int uj = __shfl_sync(kFull, u[r], j);
        unsigned bj = __shfl_sync(kFull, cbase, j);
        int nj = __shfl_sync(kFull, nch, j);
        for (int c = lane; c < nj; c += 32) cout[bj + c] = make_int2(uj, c);
      }
      cbase += (unsigned)nch;
    }
  }
}

// Seeds a frontier of one vertex (used by the init kernels; block-wide).
__device__ __forceinline__ void seed_frontier(int src, const int *__restrict__ ptr, int *queue,
                                              int2 *chunks, LevelCounters *c) {
  int deg = __ldg(ptr + src + 1) - __ldg(ptr + src);
  int nch = deg > kBigDeg ? (deg + kChunk - 1) / kChunk : 0;
  for (int j = threadIdx.x; j < nch; j += blockDim.x) chunks[j] = make_int2(src, j);
  if (threadIdx.x == 0) {
    *c = LevelCounters{0ull, 0, 0, 0ull};
    if (nch) {
      c->qc = (unsigned long long)nch << 32;
      c->nbig = 1;
    } else {
      queue[0] = src;
      c->qc = 1ull;
    }
    c->edges = (unsigned long long)deg;
  }
}

// Push expansion of (qin[0..nq), cin[0..nch)).  `load(v)` gives the 32-bit
// payload of a source vertex (e.g. its distance), broadcast to its edges.
template <typename Load, typename Visit>
__device__ __forceinline__ void expand_push(const int *__restrict__ ptr,
                                            const int *__restrict__ ind, const int *qin,
                                            unsigned nq, const int2 *cin, unsigned nch,
                                            int *qout, int2 *cout, LevelCounters *nxt,
                                            int gwarp, int nwarps, Load load, Visit &visit,
                                            unsigned long long *walked = nullptr) {
  const int lane = lane_id();
  unsigned long long nwalk = 0;
  DiscoverAcc acc;
  for (unsigned base = (unsigned)gwarp * 32u; base < nq; base += (unsigned)nwarps * 32u) {
    unsigned idx = base + lane;
    int v = idx < nq ? __ldcg(qin + idx) : -1;
    int s = 0, d = 0;
    unsigned pay = 0;
    if (v >= 0) {
      s = __ldg(ptr + v);
      d = __ldg(ptr + v + 1) - s;
      pay = load(v);
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
      bool f[kUnroll];
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) f[r] = ok[r] && visit.commit(pp[r], kk[r], uu[r], aux[r]);
      discover_n<kUnroll>(f, uu, ptr, qout, cout, nxt, acc);
    }
  }
  for (unsigned c = (unsigned)gwarp; c < nch; c += (unsigned)nwarps) {
    int2 ch = __ldcg(cin + c);
    int s = __ldg(ptr + ch.x) + ch.y * kChunk;
    int e = min(s + kChunk, __ldg(ptr + ch.x + 1));
    nwalk += (unsigned long long)(e - s);
    unsigned pay = load(ch.x);
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
      bool f[kUnroll];
#pragma unroll
      for (int r = 0; r < kUnroll; ++r)
        f[r] = ok[r] && visit.commit(pay, k0 + r * 32 + lane, uu[r], aux[r]);
      discover_n<kUnroll>(f, uu, ptr, qout, cout, nxt, acc);
    }
  }
  flush_acc(acc, nxt);
  if (walked && lane == 0 && nwalk) atomicAdd(walked, nwalk);
}

}  // namespace apspie
