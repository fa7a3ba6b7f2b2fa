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
//     as (vertex, chunk) pairs that every warp of the grid pulls from.
// A visitor decides per edge whether the destination enters the next
// frontier; discover() appends it (warp-aggregated) to the next queue or, if
// it is a big vertex, to the next chunk list, and accumulates the next
// frontier's edge count.
#pragma once
#include "common.cuh"

namespace apspie {

constexpr int kBigDeg = 1024;  // out-degree above which a vertex is chunked
constexpr int kChunk = 1024;   // edges per chunk

struct LevelCounters {
  unsigned q;       // vertices in the queue (degree <= kBigDeg)
  unsigned chunks;  // entries in the chunk list
  unsigned nbig;    // vertices in the chunk list
  unsigned pad;
  unsigned long long edges;  // sum of out-degrees of those vertices
};

// Capacity of a chunk list for a graph with nnz edges.
inline size_t chunk_capacity(long long nnz) {
  return (size_t)(nnz / kChunk + nnz / kBigDeg + 2);
}

// Called by all 32 lanes; lanes with found == true append vertex u.
__device__ __forceinline__ void discover(bool found, int u, const int *__restrict__ ptr,
                                         int *qout, int2 *cout, LevelCounters *nxt) {
  int deg = 0;
  if (found) deg = __ldg(ptr + u + 1) - __ldg(ptr + u);
  bool big = found && deg > kBigDeg;
  bool small = found && !big;
  unsigned slot = warp_append(small, &nxt->q);
  if (small) qout[slot] = u;
  if (big) {
    int nch = (deg + kChunk - 1) / kChunk;
    unsigned base = atomicAdd(&nxt->chunks, (unsigned)nch);
    atomicAdd(&nxt->nbig, 1u);
    for (int j = 0; j < nch; ++j) cout[base + j] = make_int2(u, j);
  }
  unsigned long long e = warp_sum((unsigned long long)deg);
  if (lane_id() == 0 && e) atomicAdd(&nxt->edges, e);
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

// Push expansion of (qin[0..nq), cin[0..nch)).  Per source vertex v the
// functor `load(v)` returns a 32-bit payload (e.g. its distance) that is
// broadcast to its edges; `visit(payload, edge_index, dst)` returns true when
// dst must join the next frontier.  Warp-uniform control flow throughout.
template <typename Load, typename Visit>
__device__ __forceinline__ void expand_push(const int *__restrict__ ptr,
                                            const int *__restrict__ ind, const int *qin,
                                            unsigned nq, const int2 *cin, unsigned nch,
                                            int *qout, int2 *cout, LevelCounters *nxt,
                                            int gwarp, int nwarps, Load load, Visit visit) {
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
    for (int e0 = 0; e0 < total; e0 += 32) {
      int e = e0 + lane;
      int owner = warp_owner(excl, e);
      int so = __shfl_sync(kFull, s, owner);
      int eo = __shfl_sync(kFull, excl, owner);
      unsigned po = __shfl_sync(kFull, pay, owner);
      bool found = false;
      int u = -1;
      if (e < total) {
        int k = so + (e - eo);
        u = __ldg(ind + k);
        found = visit(po, k, u);
      }
      discover(found, u, ptr, qout, cout, nxt);
    }
  }
  for (unsigned c = (unsigned)gwarp; c < nch; c += (unsigned)nwarps) {
    int2 ch = __ldcg(cin + c);
    int s = __ldg(ptr + ch.x) + ch.y * kChunk;
    int e = min(s + kChunk, __ldg(ptr + ch.x + 1));
    unsigned pay = load(ch.x);
    for (int k0 = s; k0 < e; k0 += 32) {
      int k = k0 + lane;
      bool found = false;
      int u = -1;
      if (k < e) {
        u = __ldg(ind + k);
        found = visit(pay, k, u);
      }
      discover(found, u, ptr, qout, cout, nxt);
    }
  }
}

}  // namespace apspie
