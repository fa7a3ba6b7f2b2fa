// sssp.cu -- single-source shortest paths as a frontier-driven min-plus
// SpMSpV in one persistent kernel.
//
// Replaces sssp<V>() (src/sssp.cuh:28-115) and its per-iteration
// spmspvSssp<V>() (src/spmspvSssp.cuh:92-291: bitify every finite vertex,
// gather, "+" per edge, radix sort, ReduceByKey(min), scatter, fmin).
// Here each round expands only the vertices whose distance dropped in the
// previous round (the reference re-expands every finite vertex), the (+)
// is fused into the gather and the (min) reduction is an atomicMin on the
// distance word, so no (row, value) pairs are materialised or sorted.  A
// vertex enters the next frontier once per round (stamp array).
//
// Near-far scheduling (Davidson, Baxter, Garland & Owens, "Work-Efficient
// Parallel GPU Methods for Single-Source Shortest Paths", IPDPS 2014): with a
// threshold T, only vertices whose new distance is below T join the next
// frontier ("near"); the others go to a far list.  When the near frontier
// runs dry T grows by delta and the far list is split again.  Vertices are
// then mostly expanded once, with their final distance, instead of once per
// improvement.  delta = 0 disables it (T = infinity: plain frontier
// Bellman-Ford, fewer rounds, more relaxations -- better on high-diameter
// graphs).  The schedule only changes the order of relaxations.
//
// Pull rounds (apspie_sssp_*_pull, given the in-adjacency with its weights,
// near-far off): a round whose frontier's out-edges exceed nnz / alpha
// scans every in-edge instead -- each vertex takes the minimum of
// d[u] + w(u,v) over its in-neighbours u in the frontier (stamp of the
// previous round or this one) and writes its own distance, with no
// atomics; vertices of more than kHubIn in-edges are split into chunks of
// kPullChunk edges whose minima go through atomicMin.  Improved vertices
// are queued as in a push round, so either direction may follow.  The
// relaxations are the same min-plus steps, so the fixpoint is the same.
//
// Push rounds stage their appends per warp in shared memory (one global
// reservation per 256 queued vertices or 128 hub entries, frontier.cuh), and
// skip re-expansions that relax nothing new: a queued vertex whose distance
// equals the one it was last expanded with was queued again by an
// improvement that the same expansion already used; a hub of
// kHubSkipMinDeg+ edges, expanded chunk by chunk, decides the same by one
// CAS per round on a (round, skip, distance) word.
//
// Distances are kept as 32-bit words: uint32 sums for integer weights, and
// the IEEE bit pattern for float weights -- non-negative floats order like
// their bit patterns, so atomicMin on the word is min on the value.  Each
// float relaxation is one round-to-nearest single add, and chaotic
// relaxation converges to the unique fixpoint of
// d[v] = min(d[v], min_u fl(d[u] + w(u,v))), so the result is bit-identical
// to the reference's label-correcting CPU SSSP (src/testSssp.cpp:33-115).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "context.h"
#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kSsspThreads = 512;
constexpr int kHubIn = 1024;      // in-degree above which a pull round splits a vertex
constexpr int kPullChunk = 1024;  // in-edges per chunk of such a vertex

constexpr int kSsspTraceRounds = 64;  // rounds recorded in the per-run trace
// out-degree from which a hub's chunks may skip a re-expansion with an
// unchanged distance (CAS-decided per round; measured on R-MAT 20 / 22 / 23:
// 4 % faster on the symmetric graphs at 256 - 1024, 1 - 2 % slower on the
// directed one when every hub takes part)
constexpr int kHubSkipMinDeg = 512;


struct RoundTrace {
  unsigned frontier;          // queued vertices + big-list vertices
  unsigned phase;
  unsigned long long edges;   // their out-edges
  unsigned long long t_last;  // %globaltimer when the last block finished its share
  unsigned long long t_end;   // ... and when the round's barrier released
};

struct SsspState {
  LevelCounters c[3];
  unsigned far_count[3];  // far lists rotate by phase
  unsigned far_min[3];    // least distance sent to each far list
  alignas(128) unsigned bar[2];  // grid-barrier arrival counter (64-bit), its own line
  alignas(128) int err;
  int rounds;
  int phases;
  unsigned nhc;  // chunks of the high in-degree vertices (pull rounds)
  unsigned long long relaxations;  // edges walked over all rounds (pull rounds: nnz each)
  unsigned long long reached;
  unsigned long long edges;        // sum of out-degrees of reached vertices
  unsigned long long t_start;
  RoundTrace trace[kSsspTraceRounds];
};

template <typename W>
struct Arith;

template <>
struct Arith<uint32_t> {
  static constexpr unsigned kInf = 0xffffffffu;
  __device__ __forceinline__ static unsigned add(unsigned d, uint32_t w) {
    unsigned s = d + w;
    return (s < d || s == kInf) ? kInf - 1u : s;  // saturate below "unreached"
  }
  // threshold + delta (delta given as the weight type's bits), saturating at kInf
  __device__ __forceinline__ static unsigned step(unsigned t, unsigned delta) {
    unsigned s = t + delta;
    return s < t ? kInf : s;
  }
};

template <>
struct Arith<float> {
  static constexpr unsigned kInf = 0x7f800000u;  // +inf
  __device__ __forceinline__ static unsigned add(unsigned d, float w) {
    return __float_as_uint(__fadd_rn(__uint_as_float(d), w));
  }
  __device__ __forceinline__ static unsigned step(unsigned t, unsigned delta) {
    return __float_as_uint(__fadd_rn(__uint_as_float(t), __uint_as_float(delta)));
  }
};

// Push visitor: relax (u, w[k]) with the tail's distance du as payload.  An
// improved target below the threshold joins the next frontier (class 1,
// once per round by the stamp); one at or above it goes to the far list
// (class 2, once per phase by the far stamp).
template <typename W>
struct SsspVisit {
  static constexpr bool kTwoWay = true;
  const W *__restrict__ w;
  unsigned *dist;
  int *stamp;
  int *fstamp;
  int round, phase;
  unsigned thresh;
  int *far_list;
  unsigned *far_count;
  unsigned *far_min;
  // far lists only exist under a finite threshold (near-far schedule)
  __device__ __forceinline__ bool two_way() const { return thresh != Arith<W>::kInf; }
  __device__ __forceinline__ bool check(unsigned du, int k, int u, unsigned &nd) const {
    nd = Arith<W>::add(du, __ldg(w + k));
    return nd < __ldcg(dist + u);
  }
  template <int N>
  __device__ __forceinline__ void commit_n(const unsigned (&)[N], const int (&)[N],
                                           const int (&u)[N], const unsigned (&nd)[N],
                                           const bool (&ok)[N], int (&cls)[N]) const {
    // The distance minimum and the stamp exchange are issued together, not
    // one after the other: a target that passed check() (nd below the
    // distance read this round) is improved this round, by this minimum or
    // by another that got in between, so it belongs in the next frontier
    // either way, and the first exchange of the round queues it.  A vertex
    // queued with a distance it was already expanded with is skipped at
    // expansion.  (Waiting for the minimum's old value first cost 4 - 6 %:
    // R-MAT 20 u32 0.556 against 0.533 ms, R-MAT 22 3.13 against 2.93 ms.)
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (ok[r]) atomicMin(dist + u[r], nd[r]);
    int prev[N];
#pragma unroll
    for (int r = 0; r < N; ++r) {
      prev[r] = 0;
      if (ok[r])
        prev[r] = nd[r] < thresh ? atomicExch(stamp + u[r], round) : atomicExch(fstamp + u[r], phase);
    }
#pragma unroll
    for (int r = 0; r < N; ++r) {
      cls[r] = 0;
      if (ok[r]) cls[r] = nd[r] < thresh ? (prev[r] != round ? 1 : 0)
                                         : (prev[r] != phase ? 2 : 3);  // 3: far, already listed
    }
  }
  // least distance sent far by this warp's batch (classes 2 and 3), one atomic
  template <int N>
  __device__ __forceinline__ void note_far(const int (&cls)[N], const unsigned (&nd)[N]) const {
    unsigned lo = Arith<W>::kInf;
#pragma unroll
    for (int r = 0; r < N; ++r)
      if (cls[r] >= 2) lo = min(lo, nd[r]);
    lo = __reduce_min_sync(kFull, lo);
    if (lo != Arith<W>::kInf && lane_id() == 0) atomicMin(far_min, lo);
  }
};

template <typename W>
__global__ void sssp_init(int m, int src, unsigned *dist, int *stamp, int *fstamp, unsigned *xd,
                          unsigned long long *xw, const int *__restrict__ ptr, int *queue,
                          int2 *chunks, SsspState *st) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    dist[v] = (v == src) ? 0u : Arith<W>::kInf;
    stamp[v] = -1;
    fstamp[v] = -1;
    xd[v] = Arith<W>::kInf;
    // no round yet (tag all ones), no distance recorded
    xw[v] = (0x7fffffffull << 33) | Arith<W>::kInf;
  }
  if (blockIdx.x == 0) {
    seed_frontier(src, ptr, queue, chunks, &st->c[0]);
    if (threadIdx.x == 0) {
      st->c[1] = LevelCounters{0ull, 0, 0, 0ull};
      st->c[2] = LevelCounters{0ull, 0, 0, 0ull};
      st->far_count[0] = st->far_count[1] = st->far_count[2] = 0;
      st->far_min[0] = st->far_min[1] = st->far_min[2] = Arith<W>::kInf;
      st->bar[0] = st->bar[1] = 0;
      st->err = 0;
      st->rounds = 0;
      st->phases = 0;
      st->nhc = 0;
      for (int i = 0; i < kSsspTraceRounds; ++i) st->trace[i] = RoundTrace{0, 0, 0ull, 0ull, 0ull};
      st->relaxations = 0;
      st->reached = 0;
      st->edges = 0;
    }
  }
}

// Lists the (vertex, chunk) units of the vertices with more than kHubIn
// in-edges for the pull rounds (runs after sssp_init, which zeroes nhc).
__global__ void sssp_hub_chunks(int m, const int *__restrict__ tptr, int2 *hubc, SsspState *st) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    const int d = __ldg(tptr + v + 1) - __ldg(tptr + v);
    if (d > kHubIn) {
      const unsigned nc = (unsigned)((d + kPullChunk - 1) / kPullChunk);
      const unsigned at = atomicAdd(&st->nhc, nc);
      for (unsigned c = 0; c < nc; ++c) hubc[at + c] = make_int2(v, (int)c);
    }
  }
}

// MINB blocks per SM: 2 for the push-only entry points; 3 when pull rounds
// are possible (their loops carry no atomics and gain from the extra warps:
// R-MAT 22 push/pull 4.0 vs 4.7 ms per source, while push-only ran 12 %
// slower at 3 blocks, which costs spills at 40 registers; measured).
template <typename W, int MINB>
__global__ void __launch_bounds__(kSsspThreads, MINB)
sssp_persistent(int m, const int *__restrict__ ptr, const int *__restrict__ ind,
                const W *__restrict__ w, unsigned *dist, int *stamp, int *qa, int *qb, int2 *ca,
                int2 *cb, SsspState *st, int max_rounds, int *fstamp, unsigned *xd, int *far0,
                int *far1, int *far2, unsigned delta, long long nnz, const int *__restrict__ tptr,
                const int *__restrict__ tind, const W *__restrict__ tw, const int2 *hubc,
                int alpha, unsigned long long *xw) {
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const int lane = lane_id();
  __shared__ unsigned s_q, s_chunks, s_nbig, s_far;
  __shared__ unsigned long long s_edges;
  __shared__ unsigned s_best[kSsspThreads / 32][32];
  // T = infinity without near-far; else the first phase covers [0, delta)
  if (blockIdx.x == 0 && threadIdx.x == 0) st->t_start = globaltimer();
  unsigned thresh = delta ? delta : Arith<W>::kInf;
  int phase = 0;
  int r = 0;
  for (;; ++r) {
    LevelCounters *cur = &st->c[r % 3];
    LevelCounters *nxt = &st->c[(r + 1) % 3];
    LevelCounters *clr = &st->c[(r + 2) % 3];
    if (threadIdx.x == 0) {
      const unsigned long long bc = __ldcg(&cur->bc);
      s_q = __ldcg(&cur->q);
      s_chunks = bc_chunks(bc);
      s_nbig = bc_big(bc);
      s_edges = __ldcg(&cur->edges);
      s_far = __ldcg(&st->far_count[phase % 3]);
      if (blockIdx.x == 0) *clr = LevelCounters{0ull, 0, 0, 0ull};
    }
    __syncthreads();
    const unsigned nq = s_q, nch = s_chunks;
    if (max_rounds > 0 && r >= max_rounds) break;
    int *qout = (r & 1) ? qa : qb;
    int2 *cout = (r & 1) ? ca : cb;
    if (nq == 0 && nch == 0) {
      // near frontier empty: done, or open the next phase by splitting the
      // far list of this one into the next near frontier and the next far list
      const unsigned nfar = s_far;
      if (nfar == 0) break;
      int *fin = phase % 3 == 0 ? far0 : (phase % 3 == 1 ? far1 : far2);
      // the next threshold: one step up, or one step above the least far
      // distance when that is higher (skips empty ranges); it always grows
      const unsigned fmin = __ldcg(&st->far_min[phase % 3]);
      unsigned nt = Arith<W>::step(thresh, delta);
      const unsigned nf = Arith<W>::step(fmin, delta);
      nt = nf > nt ? nf : nt;
      thresh = nt > thresh ? nt : Arith<W>::kInf;
      ++phase;
      int *fout = phase % 3 == 0 ? far0 : (phase % 3 == 1 ? far1 : far2);
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->far_count[(phase + 1) % 3] = 0;
        st->far_min[(phase + 1) % 3] = Arith<W>::kInf;
      }
      DiscoverAcc acc;
      for (unsigned base = (unsigned)gwarp * 32u; base < nfar; base += (unsigned)nwarps * 32u) {
        const unsigned idx = base + lane;
        const int u = idx < nfar ? __ldcg(fin + idx) : 0;
        bool to_near[1] = {false}, keep[1] = {false};
        if (idx < nfar) {
          const unsigned d = __ldcg(dist + u);
          // below the new threshold and not yet expanded with this distance
          if (d < thresh) {
            to_near[0] = d != __ldcg(xd + u) && atomicExch(stamp + u, r) != r;
          } else {
            keep[0] = atomicExch(fstamp + u, phase) != phase;
            if (keep[0]) atomicMin(&st->far_min[phase % 3], d);
          }
        }
        int uu[1] = {u};
        discover_n<1>(to_near, uu, ptr, qout, cout, nxt, acc);
        append_plain<1>(keep, uu, fout, &st->far_count[phase % 3]);
      }
      flush_acc(acc, nxt);
      if (!grid_barrier(st->bar, &st->err)) return;
      continue;
    }
    if (tptr && delta == 0u && r > 0 && alpha > 0 &&
        (long long)s_edges * alpha > nnz) {
      // ---- pull round: every vertex takes the least d[u] + w over its
      // in-neighbours in the frontier; hub chunks and 32-vertex groups are
      // handed out by the round's counter ----
      if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(&st->relaxations, (unsigned long long)nnz);
      LevelCounters *nx = nxt;
      DiscoverAcc acc;
      const int warp = warp_in_block();
      const unsigned ngroups = (unsigned)((m + 31) / 32);
      const unsigned nhc = __ldcg(&st->nhc);
      for (;;) {
        unsigned unit = 0;
        if (lane == 0) unit = atomicAdd(&cur->grab, 1u);
        unit = __shfl_sync(kFull, unit, 0);
        if (unit >= nhc + ngroups) break;
        if (unit < nhc) {
          const int2 hc = hubc[unit];
          const int v = hc.x;
          const int a0 = __ldg(tptr + v) + hc.y * kPullChunk;
          const int a1 = min(__ldg(tptr + v + 1), a0 + kPullChunk);
          unsigned best = Arith<W>::kInf;
          for (int k = a0 + lane; k < a1; k += 32) {
            const int u = __ldg(tind + k);
            if (__ldcg(stamp + u) >= r - 1) {
              const unsigned du = __ldcg(dist + u);
              if (du != Arith<W>::kInf) best = min(best, Arith<W>::add(du, __ldg(tw + k)));
            }
          }
          best = __reduce_min_sync(kFull, best);
          bool f[1] = {false};
          if (lane == 0 && best < __ldcg(dist + v)) {
            const unsigned old = atomicMin(dist + v, best);
            if (best < old) f[0] = atomicExch(stamp + v, r) != r;
          }
          int uu[1] = {v};
          discover_n<1>(f, uu, ptr, qout, cout, nx, acc);
        } else {
          const int v = (int)((unit - nhc) * 32u) + lane;
          int s = 0, d = 0;
          if (v < m) {
            s = __ldg(tptr + v);
            d = __ldg(tptr + v + 1) - s;
            if (d > kHubIn) d = 0;  // its chunks are separate units
          }
          s_best[warp][lane] = Arith<W>::kInf;
          __syncwarp();
          const int incl = warp_incl_scan(d);
          const int excl = incl - d;
          const int total = __shfl_sync(kFull, incl, 31);
          for (int e0 = 0; e0 < total; e0 += 32) {
            const int e = e0 + lane;
            const int owner = warp_owner(excl, e);
            const int so = __shfl_sync(kFull, s, owner);
            const int eo = __shfl_sync(kFull, excl, owner);
            if (e < total) {
              const int k = so + (e - eo);
              const int u = __ldg(tind + k);
              if (__ldcg(stamp + u) >= r - 1) {
                const unsigned du = __ldcg(dist + u);
                if (du != Arith<W>::kInf)
                  atomicMin(&s_best[warp][owner], Arith<W>::add(du, __ldg(tw + k)));
              }
            }
          }
          __syncwarp();
          const unsigned best = s_best[warp][lane];
          bool f[1] = {false};
          if (v < m && d > 0 && best < __ldcg(dist + v)) {
            // only this lane writes v in a pull round (hubs are the chunk units)
            dist[v] = best;
            stamp[v] = r;
            f[0] = true;
          }
          int uu[1] = {v < m ? v : 0};
          discover_n<1>(f, uu, ptr, qout, cout, nx, acc);
        }
      }
      flush_acc(acc, nx);
      if (r < kSsspTraceRounds) {
        __syncthreads();
        if (threadIdx.x == 0) atomicMax(&st->trace[r].t_last, globaltimer());
        if (blockIdx.x == 0 && threadIdx.x == 0) {
          st->trace[r].frontier = nq + s_nbig;
          st->trace[r].phase = 0xffffffffu;  // marks a pull round
          st->trace[r].edges = s_edges;
        }
      }
      if (!grid_barrier(st->bar, &st->err)) return;
      if (r < kSsspTraceRounds && blockIdx.x == 0 && threadIdx.x == 0)
        st->trace[r].t_end = globaltimer();
      continue;
    }
    int *qin = (r & 1) ? qb : qa;
    int2 *cin = (r & 1) ? cb : ca;
    int *fout = phase % 3 == 0 ? far0 : (phase % 3 == 1 ? far1 : far2);
    SsspVisit<W> vis{w,    dist,   stamp, fstamp, r, phase, thresh, fout, &st->far_count[phase % 3],
                     &st->far_min[phase % 3]};
    // A queued vertex whose distance still equals the one it was last
    // expanded with (it improved again in the round that expanded it, so it
    // was queued once more) has nothing new to relax: skipped.  A hub's
    // chunks are expanded by several warps with the distance each reads; the
    // first chunk of the hub to run in a round decides for all of them, by
    // one CAS on the hub's word xw = (round, skip, distance): skip when the
    // recorded distance equals the current one, else record the current one.
    // Every chunk of the round relaxes with at most the recorded distance
    // (its own read, or the recorded value when its read is older), so a
    // later round that finds the distance unchanged knows every chunk
    // relaxed with it.
    expand_push(ptr, ind, qin, nq, cin, s_nbig, nch, qout, cout, nxt, cur, gwarp, nwarps,
                [&](int v, bool whole, bool &skip) {
                  const unsigned d = __ldcg(dist + v);
                  if (!whole && __ldg(ptr + v + 1) - __ldg(ptr + v) < kHubSkipMinDeg) {
                    // a hub of a few chunks: the decision's CAS would cost
                    // more than the skip saves; expanded, and its recorded
                    // distance voided
                    xd[v] = Arith<W>::kInf;
                    return d;
                  }
                  if (!whole) {
                    unsigned long long xv = __ldcg(xw + v);
                    if ((unsigned)(xv >> 33) != (unsigned)r) {
                      const unsigned rec = (unsigned)xv;
                      const bool sk = rec == d;
                      const unsigned long long nv = ((unsigned long long)(unsigned)r << 33) |
                                                    ((unsigned long long)sk << 32) | d;
                      const unsigned long long pv = atomicCAS(xw + v, xv, nv);
                      xv = pv == xv ? nv : pv;  // lost the race: follow the winner
                    }
                    skip = (xv >> 32) & 1ull;
                    // this read may predate the recorded one: relax with at
                    // most the recorded distance, so that it stays the
                    // largest distance any chunk of the round used
                    return min(d, (unsigned)xv);
                  }
                  if (__ldcg(xd + v) == d) {
                    skip = true;
                    return d;
                  }
                  xd[v] = d;  // the distance v is expanded with
                  return d;
                },
                vis, &st->relaxations);
    if (r < kSsspTraceRounds) {
      __syncthreads();
      if (threadIdx.x == 0) atomicMax(&st->trace[r].t_last, globaltimer());
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->trace[r].frontier = nq + s_nbig;
        st->trace[r].phase = (unsigned)phase;
        st->trace[r].edges = s_edges;
      }
    }
    if (!grid_barrier(st->bar, &st->err)) return;
    if (r < kSsspTraceRounds && blockIdx.x == 0 && threadIdx.x == 0)
      st->trace[r].t_end = globaltimer();
  }
  // reached vertices and their out-degrees (E_R)
  unsigned long long cnt = 0, edg = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x)
    if (__ldcg(dist + v) != Arith<W>::kInf) {
      ++cnt;
      edg += (unsigned long long)(__ldg(ptr + v + 1) - __ldg(ptr + v));
    }
  cnt = warp_sum(cnt);
  edg = warp_sum(edg);
  if (lane_id() == 0 && cnt) {
    atomicAdd(&st->reached, cnt);
    atomicAdd(&st->edges, edg);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rounds = r;
    st->phases = phase;
  }
}

template <typename W, int MINB>
int sssp_grid(apspie_context *ctx) {
  return occupancy_grid(ctx, (const void *)sssp_persistent<W, MINB>, kSsspThreads);
}

template <typename W>
int sssp_run(apspie_context *ctx, int src, int64_t nnz, int m, const int *d_ptr, const int *d_ind,
             const W *d_w, unsigned *d_dist, int max_rounds, unsigned delta,
             const int *d_tptr = nullptr, const int *d_tind = nullptr, const W *d_tw = nullptr) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || src < 0 || src >= m)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp: src %d outside [0,%d)", src, m);
  if (nnz < 0 || nnz >= (int64_t)INT32_MAX)
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "apspie_sssp: nnz exceeds int32 offsets");
  if (!d_ptr || !d_dist || (nnz > 0 && (!d_ind || !d_w)) ||
      (d_tptr && nnz > 0 && (!d_tind || !d_tw)))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp: null pointer");
  // without a pull switch no round pulls: the in-adjacency is not needed
  // and the push-only kernel (two blocks per SM, more registers) runs
  if (ctx->sssp_pull_alpha == 0) {
    d_tptr = nullptr;
    d_tind = nullptr;
    d_tw = nullptr;
  }
  size_t cap = chunk_capacity(nnz);
  auto *st = (SsspState *)workspace(ctx, kSlotSsspState, sizeof(SsspState));
  auto *qa = (int *)workspace(ctx, kSlotSsspQueueA, sizeof(int) * (size_t)m);
  auto *qb = (int *)workspace(ctx, kSlotSsspQueueB, sizeof(int) * (size_t)m);
  auto *ca = (int2 *)workspace(ctx, kSlotSsspChunksA, sizeof(int2) * cap);
  auto *cb = (int2 *)workspace(ctx, kSlotSsspChunksB, sizeof(int2) * cap);
  auto *stamp = (int *)workspace(ctx, kSlotSsspStamp, sizeof(int) * (size_t)m);
  // far stamps, expanded distances and three far lists of m entries
  const size_t mm = ((size_t)m + 63) & ~size_t(63);
  auto *nf = (int *)workspace(ctx, kSlotSsspNearFar, sizeof(int) * mm * 5);
  // per-vertex (round, skip, distance) words of the hubs' chunked expansions
  auto *xw = (unsigned long long *)workspace(ctx, kSlotSsspHubWord,
                                             sizeof(unsigned long long) * (size_t)m);
  if (!st || !qa || !qb || !ca || !cb || !stamp || !nf || !xw) return APSPIE_ERR_OOM;
  int *fstamp = nf, *far0 = nf + 2 * mm, *far1 = nf + 3 * mm, *far2 = nf + 4 * mm;
  unsigned *xd = (unsigned *)(nf + mm);
  ctx->sssp_state = st;
  const bool pull3 = d_tptr != nullptr;
  int grid = persistent_grid(ctx, pull3 ? sssp_grid<W, 3>(ctx) : sssp_grid<W, 2>(ctx),
                             ctx->sssp_blocks_per_sm);
  if (grid <= 0) return set_error(ctx, APSPIE_ERR_CUDA, "apspie_sssp: occupancy query failed");
  int init_grid = std::min((m + 255) / 256, ctx->num_sms * 8);
  sssp_init<W><<<init_grid, 256, 0, ctx->stream>>>(m, src, d_dist, stamp, fstamp, xd, xw, d_ptr,
                                                   qa, ca, st);
  int rc = check_launch(ctx, "sssp_init");
  if (rc) return rc;
  int2 *hubc = nullptr;
  if (d_tptr) {
    hubc = (int2 *)workspace(ctx, kSlotSsspHubs,
                             sizeof(int2) * ((size_t)nnz / kPullChunk + (size_t)nnz / kHubIn + 1));
    if (!hubc) return APSPIE_ERR_OOM;
    sssp_hub_chunks<<<init_grid, 256, 0, ctx->stream>>>(m, d_tptr, hubc, st);
    rc = check_launch(ctx, "sssp_hub_chunks");
    if (rc) return rc;
  }
  long long nnz_ll = nnz;
  int alpha = d_tptr ? ctx->sssp_pull_alpha : 0;
  void *args[] = {&m,  (void *)&d_ptr, (void *)&d_ind, (void *)&d_w, &d_dist, &stamp,
                  &qa, &qb,            &ca,            &cb,           &st,     &max_rounds,
                  &fstamp, &xd, &far0, &far1, &far2, &delta, &nnz_ll, (void *)&d_tptr,
                  (void *)&d_tind, (void *)&d_tw, &hubc, &alpha, &xw};
  const void *kern =
      pull3 ? (const void *)sssp_persistent<W, 3> : (const void *)sssp_persistent<W, 2>;
  cudaError_t e = cudaLaunchCooperativeKernel(kern, dim3(grid),
                                              dim3(kSsspThreads), args, 0, ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "sssp_persistent");
  ctx->launches += 1;
  return APSPIE_OK;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_sssp_u32(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
                    const int *d_ind, const uint32_t *d_w, uint32_t *d_dist, int max_rounds) {
  return sssp_run<uint32_t>(ctx, src, nnz, m, d_ptr, d_ind, d_w, d_dist, max_rounds,
                            ctx->sssp_delta_u32);
}

int apspie_sssp_f32(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
                    const int *d_ind, const float *d_w, float *d_dist, int max_rounds) {
  float df = ctx->sssp_delta_f32;
  unsigned bits = 0;
  std::memcpy(&bits, &df, sizeof(bits));
  return sssp_run<float>(ctx, src, nnz, m, d_ptr, d_ind, d_w, (unsigned *)d_dist, max_rounds,
                         df > 0.0f ? bits : 0u);
}

int apspie_sssp_u32_pull(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
                         const int *d_ind, const uint32_t *d_w, const int *d_tptr,
                         const int *d_tind, const uint32_t *d_tw, uint32_t *d_dist,
                         int max_rounds) {
  if (!d_tptr) return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp_u32_pull: no in-adjacency");
  return sssp_run<uint32_t>(ctx, src, nnz, m, d_ptr, d_ind, d_w, d_dist, max_rounds,
                            ctx->sssp_delta_u32, d_tptr, d_tind, d_tw);
}

int apspie_sssp_f32_pull(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
                         const int *d_ind, const float *d_w, const int *d_tptr,
                         const int *d_tind, const float *d_tw, float *d_dist, int max_rounds) {
  if (!d_tptr) return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp_f32_pull: no in-adjacency");
  float df = ctx->sssp_delta_f32;
  unsigned bits = 0;
  std::memcpy(&bits, &df, sizeof(bits));
  return sssp_run<float>(ctx, src, nnz, m, d_ptr, d_ind, d_w, (unsigned *)d_dist, max_rounds,
                         df > 0.0f ? bits : 0u, d_tptr, d_tind, d_tw);
}

int apspie_sssp_set_pull(apspie_ctx ctx, int alpha) {
  APSPIE_CHECK_CTX(ctx);
  if (alpha < 0) return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp_set_pull: alpha < 0");
  ctx->sssp_pull_alpha = alpha;
  return APSPIE_OK;
}

int apspie_sssp_set_params(apspie_ctx ctx, uint32_t delta_u32, float delta_f32) {
  APSPIE_CHECK_CTX(ctx);
  if (!(delta_f32 >= 0.0f) || delta_f32 > 3.0e38f)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp_set_params: bad float delta");
  ctx->sssp_delta_u32 = delta_u32;
  ctx->sssp_delta_f32 = delta_f32;
  return APSPIE_OK;
}

int apspie_sssp_get_trace(apspie_ctx ctx, int max_rounds, int *n_out, int64_t *h_frontier,
                          int64_t *h_frontier_edges, int64_t *h_ns, int64_t *h_work_last_ns) {
  APSPIE_CHECK_CTX(ctx);
  if (!ctx->sssp_state || max_rounds < 0 || !n_out)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp_get_trace: no SSSP has run");
  auto *h = (SsspState *)pinned(ctx, sizeof(SsspState));
  if (!h) return APSPIE_ERR_OOM;
  cudaError_t e = cudaMemcpyAsync(h, ctx->sssp_state, sizeof(SsspState), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "apspie_sssp_get_trace");
  const int n = std::min(std::min(max_rounds, kSsspTraceRounds), h->rounds);
  unsigned long long prev = h->t_start;
  int k = 0;
  for (int i = 0; i < n; ++i) {
    if (h->trace[i].t_end == 0) continue;  // a phase change round (no expansion)
    if (h_frontier) h_frontier[k] = h->trace[i].frontier;
    if (h_frontier_edges) h_frontier_edges[k] = (int64_t)h->trace[i].edges;
    if (h_ns) h_ns[k] = (int64_t)(h->trace[i].t_end - prev);
    if (h_work_last_ns) h_work_last_ns[k] = (int64_t)(h->trace[i].t_last - prev);
    prev = h->trace[i].t_end;
    ++k;
  }
  *n_out = k;
  return APSPIE_OK;
}

int apspie_sssp_get_stats(apspie_ctx ctx, apspie_sssp_stats *out) {
  APSPIE_CHECK_CTX(ctx);
  if (!out || !ctx->sssp_state)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp_get_stats: no SSSP has run");
  auto *h = (SsspState *)pinned(ctx, sizeof(SsspState));
  if (!h) return APSPIE_ERR_OOM;
  cudaError_t e = cudaMemcpyAsync(h, ctx->sssp_state, sizeof(SsspState), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return check_cuda(ctx, e, "apspie_sssp_get_stats");
  out->rounds = h->rounds;
  out->phases = h->phases;
  out->vertices_reached = (int64_t)h->reached;
  out->edges_traversed = (int64_t)h->edges;
  out->relaxations = (int64_t)h->relaxations;
  if (h->err)
    return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_sssp: grid barrier timed out");
  return APSPIE_OK;
}

}  // extern "C"
