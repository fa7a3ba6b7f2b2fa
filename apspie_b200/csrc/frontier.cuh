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
// discover() appends joiners (warp-aggregated) to the next queue or, for big
// vertices, writes their chunk entries cooperatively, and accumulates the
// next frontier's edge count.
#pragma once
#include "common.cuh"

namespace apspie {

constexpr int kBigDeg = 64;   // out-degree above which a vertex is chunked
constexpr int kChunk = 256;   // edges per chunk
constexpr int kUnroll = 4;    // rounds of 32 edges issued together

struct LevelCounters {
  unsigned q;       // vertices in the queue (degree <= kBigDeg)
  unsigned chunks;  // entries in the chunk list
  unsigned nbig;    // vertices in the chunk list
  unsigned pad;
  unsigned long long edges;  // sum of out-degrees of those vertices
};

// Capacity of a chunk list for a graph with nnz edges: every big vertex has
// more than kBigDeg edges, so there are fewer than nnz / kBigDeg of them.
inline size_t chunk_capacity(long long nnz) {
  return (size_t)(nnz / kChunk + nnz / kBigDeg + 2);
}

// Called by all 32 lanes; lanes with found == true append vertex u.
__device__ __forceinline__ void discover(bool found, int u, const int *__restrict__ ptr,
                                         int *qout, int2 *cout, LevelCounters *nxt) {
  const int lane = lane_id();
  int deg = 0;
  if (found) deg = __ldg(ptr + u + 1) - __ldg(ptr + u);
  bool big = found && deg > kBigDeg;
  bool small = found && !big;
  unsigned slot = warp_append(small, &nxt->q);
  if (small) qout[slot] = u;
  unsigned bmask = __ballot_sync(kFull, big);
  if (bmask) {
    int nch = big ? (deg + kChunk - 1) / kChunk : 0;
    int incl = warp_incl_scan(nch);
    int total = __shfl_sync(kFull, incl, 31);
    unsigned base = 0;
    if (lane == 0) {
      base = atomicAdd(&nxt->chunks, (unsigned)total);
      atomicAdd(&nxt->nbig, (unsigned)__popc(bmask));
    }
    base = __shfl_sync(kFull, base, 0) + (unsigned)(incl - nch);
    while (bmask) {
      int j = __ffs(bmask) - 1;
      bmask &= bmask - 1;
      int uj = __shfl_sync(kFull, u, j);
      unsigned bj = __shfl_sync(kFull, base, j);
      int nj = __shfl_sync(kFull, nch, j);
      for (int c = lane; c < nj; c += 32) cout[bj + c] = make_int2(uj, c);
    }
  }
  unsigned long long e = warp_sum((unsigned long long)deg);
  if (lane == 0 && e) atomicAdd(&nxt->edges, e);
}

// Seeds a frontier of one vertex (used by the init kernels; block-wide).
__device__ __forceinline__ void seed_frontier(int src, const int *__restrict__ ptr, int *queue,
                                              int2 *chunks, LevelCounters *c) {
  int deg = __ldg(ptr + src + 1) - __ldg(ptr + src);
  int nch = deg > kBigDeg ? (deg + kChunk - 1) / kChunk : 0;
  for (int j = threadIdx.x; j < nch; j += blockDim.x) chunks[j] = make_int2(src, j);
  if (threadIdx.x == 0) {
    *c = LevelCounters{0, 0, 0, 0, 0ull};
    if (nch) {
      c->chunks = (unsigned)nch;
      c->nbig = 1;
    } else {
      queue[0] = src;
      c->q = 1;
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
                                            int gwarp, int nwarps, Load load, Visit &visit) {
  const int lane = lane_id();
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
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) {
        bool f = ok[r] && visit.commit(pp[r], kk[r], uu[r], aux[r]);
        discover(f, uu[r], ptr, qout, cout, nxt);
      }
    }
  }
  for (unsigned c = (unsigned)gwarp; c < nch; c += (unsigned)nwarps) {
    int2 ch = __ldcg(cin + c);
    int s = __ldg(ptr + ch.x) + ch.y * kChunk;
    int e = min(s + kChunk, __ldg(ptr + ch.x + 1));
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
#pragma unroll
      for (int r = 0; r < kUnroll; ++r) {
        bool f = ok[r] && visit.commit(pay, k0 + r * 32 + lane, uu[r], aux[r]);
        discover(f, uu[r], ptr, qout, cout, nxt);
      }
    }
  }
}

}  // namespace apspie
