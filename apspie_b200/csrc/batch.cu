// batch.cu -- many traversals on graphs of uneven size in one launch.
//
// A persistent work-queue kernel runs a set of jobs together.  A job is
//   * a multi-source BFS over up to 64 sources of one graph: every vertex
//     carries 64-bit masks (visited, and the frontier of three consecutive
//     levels), bit s standing for source s -- the "frontier matrix" of
//     MS-BFS -- and the depths are vertex-major, one row per vertex of the
//     sources rounded up to a power of two; or
//   * a multi-source uint32 SSSP over up to 32 sources of one graph: the
//     distances are vertex-major, dist[v][0..sw) one row of sw = 1, 2, 4, 8,
//     16 or 32 words (the sources rounded up to a power of two), and every
//     vertex carries a mask of the sources whose distance at it dropped in
//     the last round.  A warp relaxes 32 / sw edges (v -> u, w) at a time, sw
//     lanes per edge, one per source (lane s: atomicMin(dist[u][s],
//     dist[v][s] + w) when s is active at v), so an edge is read once per
//     round for all sources and a row is one coalesced access; the improved
//     lanes' bits are OR-ed into u's next mask, and the edge whose OR found
//     the mask empty appends u to the next frontier.
// Each super-step advances every unfinished job by one level / round.  The
// work of a super-step is cut into units (BFS: 32 frontier vertices or one
// 128-edge chunk of a hub; SSSP: 8 frontier vertices or one 64-edge chunk;
// 32 vertices of a pull sweep; 32 stale frontier words to clear) and the units of all jobs are dealt round-robin over the warps of
// the grid, so a large graph and a small one share the GPU in the same
// launch.  Super-steps are separated by the bounded grid barrier; per-job
// direction switches (push / pull, Beamer's rule with per-job thresholds from
// the autotuner) are decided identically by every block from counters that
// nobody writes during the step in which they are read.
//
// A unit's joiners (vertices that enter a job's next frontier) are staged
// per warp and job in shared memory and appended with one reservation per
// flush; the next step's hub and edge tallies are summed per block.  Jobs on
// deep graphs (a probe BFS of more than 64 levels) run their sources as
// single-source traversals on sub-contexts beside the launch instead.
//
// Per source, the results are exactly those of the single-source kernels:
// BFS levels are set once per (source, vertex) by the thread whose atomicOr
// on the visited mask first sets the bit; SSSP converges to the same
// min-plus fixpoint (the fixpoint is unique, whatever the relaxation order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "context.h"
#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kBatchThreads = 512;
constexpr int kMaxJobs = 64;
constexpr int kJobBfs = 0, kJobSssp = 1;
constexpr int kMsbfsWidth = 64;   // sources per BFS device job (one 64-bit mask)
constexpr int kMssspWidth = 32;   // most sources per SSSP device job (one lane each)
// SSSP jobs relax a whole distance row per edge, so their units are smaller:
// 4 queued vertices of degree <= kSsspBigDeg, or kSsspChunk edges of a hub
constexpr int kSsspBigDeg = 32;
constexpr int kSsspChunk = 64;
constexpr int kSsspPerUnit = 8;  // queued vertices per SSSP unit (4: the batched config 1.4 % slower)
constexpr int kSsspSlots = 4;     // rounds of 32 / sw edges a warp relaxes together
// SSSP pull steps: in-degree above which a vertex is split into chunks of
// kMsPullChunk in-edges, and vertices per pull unit
constexpr int kMsHubIn = 1024;
constexpr int kMsPullChunk = 1024;
constexpr int kMsPullVerts = 8;

// A level's counters, on a 128-byte line of their own (away from the job's
// read-mostly fields and from the other levels' counters).
struct alignas(128) JobCounters {
  unsigned long long qc;  // queue length (low 32 bits) | chunk-list length (high 32 bits)
  unsigned nbig, pad;
  unsigned long long edges;
};

struct BatchJob {
  int type, m, nsrc, alpha;
  int beta, pad0;
  long long nnz;
  const int *ptr, *ind, *tptr, *tind;
  const uint32_t *w;
  const int *src;
  int32_t *out;  // vertex-major results: BFS depth [m][64]; SSSP distance [m][32]
  unsigned long long *visited, *F0, *F1, *F2;
  int *q0, *q1, *q2;
  int2 *c0, *c1, *c2;
  int big_deg, chunk;  // degree above which a vertex is chunked, edges per chunk
  int sw, salpha;      // result row width (power of two >= nsrc); SSSP pull switch
  // SSSP pull steps: in-adjacency with its weights, and the chunks of the
  // vertices of more than kMsHubIn in-edges
  const int *stptr, *stind;
  const uint32_t *stw;
  int2 *hubc;
  unsigned nhc, pad2;
  JobCounters c[3];
};

struct BatchState {
  alignas(8) unsigned bar[2];  // grid-barrier arrival counter (64-bit)
  int err;
  int steps;
  unsigned long long edges;  // sum over jobs of frontier edges walked
};

__device__ __forceinline__ unsigned long long *jobF(BatchJob *j, int i) {
  return i == 0 ? j->F0 : (i == 1 ? j->F1 : j->F2);
}
__device__ __forceinline__ int *jobQ(BatchJob *j, int i) {
  return i == 0 ? j->q0 : (i == 1 ? j->q1 : j->q2);
}
__device__ __forceinline__ int2 *jobC(BatchJob *j, int i) {
  return i == 0 ? j->c0 : (i == 1 ? j->c1 : j->c2);
}

__device__ __forceinline__ unsigned long long srcmask(int nsrc) {
  return nsrc >= 64 ? ~0ull : ((1ull << nsrc) - 1ull);
}

// ------------------------------------------------------------------ init ---
// Queues the distinct sources of job j as its level-0 frontier (one thread).
__device__ void seed_queue(BatchJob *j) {
  for (int i = 0; i < 3; ++i) j->c[i] = JobCounters{0ull, 0, 0, 0ull};
  unsigned q = 0, nch_total = 0;
  for (int s = 0; s < j->nsrc; ++s) {
    int v = j->src[s];
    bool first = true;
    for (int t = 0; t < s; ++t)
      if (j->src[t] == v) first = false;
    if (!first) continue;
    int deg = __ldg(j->ptr + v + 1) - __ldg(j->ptr + v);
    if (deg > j->big_deg) {
      int nch = (deg + j->chunk - 1) / j->chunk;
      for (int c = 0; c < nch; ++c) j->c0[nch_total + c] = make_int2(v, c);
      nch_total += (unsigned)nch;
      j->c[0].nbig += 1;
    } else {
      j->q0[q++] = v;
    }
    j->c[0].edges += (unsigned long long)deg;
  }
  j->c[0].qc = ((unsigned long long)nch_total << 32) | q;
}

__global__ void batch_init_bfs(BatchJob *jobs, int jid) {
  BatchJob *j = jobs + jid;
  const int m = j->m;
  const size_t n64 = (size_t)m * j->sw;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n64;
       i += (size_t)gridDim.x * blockDim.x)
    j->out[i] = -1;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    j->visited[v] = 0ull;
    j->F0[v] = 0ull;
    j->F1[v] = 0ull;
    j->F2[v] = 0ull;
  }
}

// sources: set visited / frontier bits and depth 0, queue each distinct source
__global__ void batch_seed_bfs(BatchJob *jobs, int jid) {
  BatchJob *j = jobs + jid;
  if (blockIdx.x != 0) return;
  for (int s = threadIdx.x; s < j->nsrc; s += blockDim.x) {
    int v = j->src[s];
    atomicOr(j->visited + v, 1ull << s);
    atomicOr(j->F0 + v, 1ull << s);
    j->out[(size_t)v * j->sw + s] = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    seed_queue(j);
  }
}

__global__ void batch_init_sssp(BatchJob *jobs, int jid) {
  BatchJob *j = jobs + jid;
  const size_t n = (size_t)j->m * j->sw;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    j->out[i] = -1;  // 0xFFFFFFFF: unreached
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < j->m; v += gridDim.x * blockDim.x) {
    j->F0[v] = 0ull;
    j->F1[v] = 0ull;
    j->F2[v] = 0ull;
  }
}

__global__ void batch_seed_sssp(BatchJob *jobs, int jid) {
  BatchJob *j = jobs + jid;
  if (blockIdx.x != 0) return;
  for (int s = threadIdx.x; s < j->nsrc; s += blockDim.x) {
    int v = j->src[s];
    j->out[(size_t)v * j->sw + s] = 0;
    atomicOr(j->F0 + v, 1ull << s);
  }
  __syncthreads();
  if (threadIdx.x == 0) seed_queue(j);
}

// --------------------------------------------------------- append helper ---
// A warp's joiners are staged in shared memory (JobStage) and get their
// slots in the job's next queue / chunk list with one packed atomic per
// flush, instead of one per warp batch: a reservation is an atomic on a
// single address, and same-address atomics run at about 1.1 - 1.5 G/s on a
// B200 (measured), so a pull step that appended per 32-vertex unit waited on
// them.  The stage holds the entries of one job and one step; it is flushed
// when the warp moves to a unit of another job and at the end of the step.
// The next frontier's big-vertex count and edge total are summed per block
// in shared memory and added once per block and job after the step.
constexpr int kJStageQ = 256;  // queue entries per warp
constexpr int kJStageB = 128;  // (vertex, degree) big entries per warp
// one append call adds at most N x 32 entries of either kind, N <= 4
// (kMsbfsUnroll): each stage must hold a whole call after a flush
static_assert(kJStageQ >= 4 * 32 && kJStageB >= 4 * 32, "stage smaller than one append");
constexpr int kStageWarpsB = kBatchThreads / 32;

struct JobStage {
  int *q;
  int2 *b;  // (vertex, degree)
  int nq, nb;
  BatchJob *job;  // job of the staged entries, or nullptr
  int level;      // the step: entries go to the level-(step + 1) lists
};

// Writes the staged entries of stg.job into its next queue / chunk list.
// Warp-collective.
__device__ __noinline__ void stage_flush(JobStage &stg) {
  if (stg.nq == 0 && stg.nb == 0) return;
  __syncwarp();
  const int lane = lane_id();
  BatchJob *j = stg.job;
  const int L = stg.level;
  const int ck = j->chunk;
  int *qout = jobQ(j, (L + 1) % 3);
  int2 *cout = jobC(j, (L + 1) % 3);
  JobCounters *nxt = &j->c[(L + 1) % 3];
  // chunk counts of the big entries and their exclusive prefix
  int nch[kJStageB / 32], excl[kJStageB / 32];
  unsigned ctot = 0;
#pragma unroll
  for (int i = 0; i < kJStageB / 32; ++i) {
    const int e = i * 32 + lane;
    nch[i] = e < stg.nb ? (stg.b[e].y + ck - 1) / ck : 0;
    const int inc = warp_incl_scan(nch[i]);
    excl[i] = (int)ctot + inc - nch[i];
    ctot += (unsigned)__shfl_sync(kFull, inc, 31);
  }
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(&nxt->qc, ((unsigned long long)ctot << 32) | (unsigned)stg.nq);
  base = __shfl_sync(kFull, base, 0);
  const unsigned qb = (unsigned)base, cb = (unsigned)(base >> 32);
  for (int i = lane; i < stg.nq; i += 32) qout[qb + (unsigned)i] = stg.q[i];
  // chunk entries (vertex, chunk index), 32 at a time over the flat list
#pragma unroll
  for (int i = 0; i < kJStageB / 32; ++i) {
    const int tot = __shfl_sync(kFull, excl[i] + nch[i], 31) - __shfl_sync(kFull, excl[i], 0);
    const int first = __shfl_sync(kFull, excl[i], 0);
    const int rel = excl[i] - first;
    for (int c0 = 0; c0 < tot; c0 += 32) {
      const int e = c0 + lane;
      const int owner = warp_owner(rel, min(e, tot - 1));
      const int uo = __shfl_sync(kFull, i * 32 + lane < stg.nb ? stg.b[i * 32 + lane].x : 0,
                                 owner);
      const int ro = __shfl_sync(kFull, rel, owner);
      if (e < tot) cout[cb + (unsigned)(first + e)] = make_int2(uo, e - ro);
    }
  }
  __syncwarp();
  stg.nq = 0;
  stg.nb = 0;
}

// Stages up to N joiners per lane (vertex u[r] of degree deg[r] where
// found[r]) of job j; the next frontier's big count and edges go to the
// block's tallies.  Warp-collective.
template <int N>
__device__ __forceinline__ void append_n(BatchJob *j, const bool (&found)[N], const int (&u)[N],
                                         const int (&deg)[N], JobStage &stg, unsigned *blk_nbig,
                                         unsigned long long *blk_edges, int jid) {
  const int lane = lane_id();
  const int bd = j->big_deg;
  int nsmall = 0, nbig = 0;
  unsigned long long edges = 0;
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const bool big = found[r] && deg[r] > bd;
    nsmall += (found[r] && !big) ? 1 : 0;
    nbig += big ? 1 : 0;
    edges += found[r] ? (unsigned long long)deg[r] : 0ull;
  }
  const int qincl = warp_incl_scan(nsmall);
  const int bincl = warp_incl_scan(nbig);
  const int qtot = __shfl_sync(kFull, qincl, 31);
  const int btot = __shfl_sync(kFull, bincl, 31);
  if ((qtot | btot) == 0) return;
  if (stg.job != j) {
    stage_flush(stg);
    stg.job = j;
  }
  if (stg.nq + qtot > kJStageQ || stg.nb + btot > kJStageB) stage_flush(stg);
  int qa = stg.nq + qincl - nsmall, ba = stg.nb + bincl - nbig;
#pragma unroll
  for (int r = 0; r < N; ++r)
    if (found[r]) {
      if (deg[r] > bd)
        stg.b[ba++] = make_int2(u[r], deg[r]);
      else
        stg.q[qa++] = u[r];
    }
  stg.nq += qtot;
  stg.nb += btot;
  __syncwarp();
  const unsigned b = warp_sum((unsigned)nbig);
  edges = warp_sum(edges);
  if (lane == 0) {
    if (b) atomicAdd(blk_nbig + jid, b);
    if (edges) atomicAdd(blk_edges + jid, edges);
  }
}

// What a unit needs to append: the warp's stage and the block's tallies.
struct AppendCtx {
  JobStage *stg;
  unsigned *blk_nbig;
  unsigned long long *blk_edges;
  int jid;
};

template <int N>
__device__ __forceinline__ void append_n(BatchJob *j, const bool (&found)[N], const int (&u)[N],
                                         const int (&deg)[N], const AppendCtx &ac) {
  append_n<N>(j, found, u, deg, *ac.stg, ac.blk_nbig, ac.blk_edges, ac.jid);
}

// ------------------------------------------------------------ MS-BFS ---
// Push relaxation of K edges per lane (v -> u[r]) carrying the tail's
// frontier mask f[r] at level L: claims the bits of f that u has not seen
// (found[r]: u enters the next frontier for the first time in this level).
// The visited ORs of all K edges are issued together, then the frontier ORs.
template <int K>
__device__ __forceinline__ void msbfs_relax_n(BatchJob *j, const unsigned long long (&f)[K],
                                              const int (&u)[K], int next,
                                              unsigned long long *Fn, bool (&found)[K]) {
  unsigned long long nb[K], old[K];
#pragma unroll
  for (int r = 0; r < K; ++r) nb[r] = u[r] >= 0 ? f[r] & ~__ldcg(j->visited + u[r]) : 0ull;
#pragma unroll
  for (int r = 0; r < K; ++r) old[r] = nb[r] ? atomicOr(j->visited + u[r], nb[r]) : ~0ull;
  unsigned long long mine[K], fo[K];
#pragma unroll
  for (int r = 0; r < K; ++r) {
    mine[r] = nb[r] & ~old[r];
    if (mine[r]) {
      int32_t *row = j->out + (size_t)u[r] * j->sw;
      for (unsigned long long b = mine[r]; b; b &= b - 1) row[__ffsll((long long)b) - 1] = next;
    }
  }
#pragma unroll
  for (int r = 0; r < K; ++r) fo[r] = mine[r] ? atomicOr(Fn + u[r], mine[r]) : 1ull;
#pragma unroll
  for (int r = 0; r < K; ++r) found[r] = mine[r] != 0ull && fo[r] == 0ull;
}

constexpr int kMsbfsUnroll = 4;  // edges per lane per batch
static_assert(kMsbfsUnroll * 32 <= kJStageB && kMsbfsUnroll * 32 <= kJStageQ,
              "an MS-BFS batch must fit a flushed stage");

// 32 queued frontier vertices, edges dealt flat over the warp, 4 x 32 a batch
__device__ void msbfs_push_queue(BatchJob *j, int L, int unit, unsigned nq, const AppendCtx &ac) {
  const int lane = lane_id();
  int *qin = jobQ(j, L % 3);
  unsigned long long *Fc = jobF(j, L % 3), *Fn = jobF(j, (L + 1) % 3);
  unsigned idx = (unsigned)unit * 32u + lane;
  int v = idx < nq ? __ldcg(qin + idx) : -1;
  int s = 0, d = 0;
  unsigned long long f = 0;
  if (v >= 0) {
    s = __ldg(j->ptr + v);
    d = __ldg(j->ptr + v + 1) - s;
    f = __ldcg(Fc + v);
  }
  int incl = warp_incl_scan(d);
  int excl = incl - d;
  int total = __shfl_sync(kFull, incl, 31);
  for (int e0 = 0; e0 < total; e0 += 32 * kMsbfsUnroll) {
    unsigned long long fo[kMsbfsUnroll];
    int u[kMsbfsUnroll], dg[kMsbfsUnroll];
    bool found[kMsbfsUnroll];
#pragma unroll
    for (int r = 0; r < kMsbfsUnroll; ++r) {
      const int e = e0 + r * 32 + lane;
      const int owner = warp_owner(excl, min(e, total - 1));
      const int so = __shfl_sync(kFull, s, owner);
      const int eo = __shfl_sync(kFull, excl, owner);
      fo[r] = __shfl_sync(kFull, f, owner);
      u[r] = e < total ? __ldg(j->ind + so + (e - eo)) : -1;
    }
    msbfs_relax_n<kMsbfsUnroll>(j, fo, u, L + 1, Fn, found);
#pragma unroll
    for (int r = 0; r < kMsbfsUnroll; ++r)
      dg[r] = found[r] ? __ldg(j->ptr + u[r] + 1) - __ldg(j->ptr + u[r]) : 0;
    append_n<kMsbfsUnroll>(j, found, u, dg, ac);
  }
}

// one kChunk-edge chunk of a hub, 4 x 32 edges a batch
__device__ void msbfs_push_chunk(BatchJob *j, int L, int unit, const AppendCtx &ac) {
  const int lane = lane_id();
  int2 *cin = jobC(j, L % 3);
  unsigned long long *Fc = jobF(j, L % 3), *Fn = jobF(j, (L + 1) % 3);
  int2 ch = __ldcg(cin + unit);
  int s = __ldg(j->ptr + ch.x) + ch.y * kChunk;
  int e = min(s + kChunk, __ldg(j->ptr + ch.x + 1));
  unsigned long long f = __ldcg(Fc + ch.x);
  for (int k0 = s; k0 < e; k0 += 32 * kMsbfsUnroll) {
    unsigned long long fo[kMsbfsUnroll];
    int u[kMsbfsUnroll], dg[kMsbfsUnroll];
    bool found[kMsbfsUnroll];
#pragma unroll
    for (int r = 0; r < kMsbfsUnroll; ++r) {
      const int k = k0 + r * 32 + lane;
      fo[r] = f;
      u[r] = k < e ? __ldg(j->ind + k) : -1;
    }
    msbfs_relax_n<kMsbfsUnroll>(j, fo, u, L + 1, Fn, found);
#pragma unroll
    for (int r = 0; r < kMsbfsUnroll; ++r)
      dg[r] = found[r] ? __ldg(j->ptr + u[r] + 1) - __ldg(j->ptr + u[r]) : 0;
    append_n<kMsbfsUnroll>(j, found, u, dg, ac);
  }
}

// pull: vertices [32*unit, 32*unit+32) OR the frontier masks of their
// in-neighbours (round-robin over the warp) until every source still missing
// at the vertex is covered or the list ends
__device__ void msbfs_pull(BatchJob *j, int L, int unit, unsigned long long *s_acc,
                           int *s_rank, const AppendCtx &ac) {
  const int lane = lane_id();
  const int m = j->m;
  const unsigned long long all = srcmask(j->nsrc);
  unsigned long long *Fc = jobF(j, L % 3), *Fn = jobF(j, (L + 1) % 3);
  int v = unit * 32 + lane;
  int s = 0, e = 0;
  unsigned long long want = 0;
  if (v < m) {
    want = all & ~__ldcg(j->visited + v);
    if (want) {
      s = __ldg(j->tptr + v);
      e = __ldg(j->tptr + v + 1);
    }
  }
  s_acc[lane] = 0ull;
  __syncwarp();
  unsigned U = __ballot_sync(kFull, want != 0 && s < e);
  while (U) {
    const int k = __popc(U);
    const bool mine = (U >> lane) & 1u;
    const int myrank = __popc(U & ((1u << lane) - 1u));
    if (mine) s_rank[myrank] = lane;
    __syncwarp();
    const int per = 32 / k, extra = 32 % k;
    const int jr = lane % k, slot = lane / k;
    const int nl = per + (jr < extra ? 1 : 0);
    const int owner = s_rank[jr];
    const int so = __shfl_sync(kFull, s, owner);
    const int eo = __shfl_sync(kFull, e, owner);
    unsigned long long acc = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int idx = so + slot + i * nl;
      if (idx < eo) acc |= __ldcg(Fc + __ldg(j->tind + idx));
    }
    if (acc) atomicOr(s_acc + owner, acc);
    __syncwarp();
    if (mine) s += (per + (myrank < extra ? 1 : 0)) * 4;
    unsigned long long got = *(volatile unsigned long long *)(s_acc + lane);
    U = __ballot_sync(kFull, mine && (want & ~got) != 0ull && s < e);
  }
  unsigned long long nb = want & *(volatile unsigned long long *)(s_acc + lane);
  bool found[1] = {nb != 0ull};
  int u[1] = {v}, dg[1] = {0};
  if (found[0]) {
    j->visited[v] |= nb;  // only this lane touches v's masks in a pull step
    Fn[v] = nb;
    int32_t *row = j->out + (size_t)v * j->sw;
    for (unsigned long long b = nb; b; b &= b - 1) row[__ffsll((long long)b) - 1] = L + 1;
    dg[0] = __ldg(j->ptr + v + 1) - __ldg(j->ptr + v);
  }
  append_n<1>(j, found, u, dg, ac);
  __syncwarp();
}

// clear the frontier words of the level before last (they become the next
// level's frontier buffer)
__device__ void msbfs_clear(BatchJob *j, int L, int unit, unsigned prevq, bool chunks) {
  const int lane = lane_id();
  const int slot = (L + 2) % 3;
  unsigned long long *F = jobF(j, slot);
  unsigned idx = (unsigned)unit * 32u + lane;
  if (idx >= prevq) return;
  if (chunks) {
    int2 c = __ldcg(jobC(j, slot) + idx);
    if (c.y == 0) F[c.x] = 0ull;
  } else {
    F[__ldcg(jobQ(j, slot) + idx)] = 0ull;
  }
}

// ---------------------------------------------------- multi-source SSSP ---
__device__ __forceinline__ unsigned sat_add(unsigned d, unsigned w) {
  unsigned t = d + w;
  return (t < d || t == 0xffffffffu) ? 0xfffffffeu : t;  // saturate below "unreached"
}

// Edges per batch of a job with row width sw: kSsspSlots rounds of 32 / sw
// edges, at most 32 (one per loading lane).
__device__ __forceinline__ int mssp_batch(int sw) { return min(32, kSsspSlots * (32 / sw)); }

// Relaxes the batch of edges held by lanes 0..nb-1 (ue: target, we: weight,
// ve: tail, me: the tail's active-source mask; me == 0 for no edge), for every
// active source.  Lane l of a round works on edge (round * 32/sw + l / sw)
// and source l % sw.  Returns, on the loading lanes, whether that edge's
// target entered the next frontier.
__device__ __forceinline__ bool mssp_relax(BatchJob *j, int ue, unsigned we, int ve, unsigned me,
                                           unsigned long long *Fn) {
  const int lane = lane_id();
  const int sw = j->sw;
  const int per = 32 / sw;                 // edges per round
  const int src = lane & (sw - 1), eo = lane / sw;
  const unsigned grp = sw == 32 ? 0xffffffffu : ((1u << sw) - 1u);
  unsigned *dist = reinterpret_cast<unsigned *>(j->out);
  unsigned nd[kSsspSlots], cur[kSsspSlots];
  int uu[kSsspSlots];
  bool act[kSsspSlots];
#pragma unroll
  for (int i = 0; i < kSsspSlots; ++i) {
    const int el = i * per + eo;           // the edge's loading lane
    const bool in = el < 32;
    const unsigned mi = __shfl_sync(kFull, me, el & 31);
    const int vi = __shfl_sync(kFull, ve, el & 31);
    const unsigned wi = __shfl_sync(kFull, we, el & 31);
    uu[i] = __shfl_sync(kFull, ue, el & 31);
    act[i] = in && ((mi >> src) & 1u);
    // the tail's distance is read from L2 (it dropped in the last round)
    nd[i] = act[i] ? sat_add(__ldcg(dist + (size_t)vi * sw + src), wi) : 0u;
    cur[i] = act[i] ? __ldcg(dist + (size_t)uu[i] * sw + src) : 0u;
  }
  // the slots' minima, issued without waiting for their old values: a
  // (target, source) whose distance read this step is above nd drops this
  // step, by this minimum or by one that got in between (whose lane sets the
  // same frontier bit), so the bits set are the same as with the old values
  // and the ballots need not wait for the atomics
#pragma unroll
  for (int i = 0; i < kSsspSlots; ++i)
    if (act[i] && nd[i] < cur[i]) atomicMin(dist + (size_t)uu[i] * sw + src, nd[i]);
  unsigned mybal = 0;
#pragma unroll
  for (int i = 0; i < kSsspSlots; ++i) {
    const bool imp = act[i] && nd[i] < cur[i];
    const unsigned b = __ballot_sync(kFull, imp);
    // loading lane i * per + g takes the bits of its edge's group g
    const int g = lane - i * per;
    if (g >= 0 && g < per) mybal = (b >> (g * sw)) & grp;
  }
  bool first = false;
  if (mybal) first = atomicOr(Fn + ue, (unsigned long long)mybal) == 0ull;
  return first;
}

// kSsspPerUnit queued vertices: their edges laid out flat, a batch at a time
__device__ void mssp_queue(BatchJob *j, int L, int unit, unsigned nq, const AppendCtx &ac) {
  const int lane = lane_id();
  int *qin = jobQ(j, L % 3);
  unsigned long long *Fc = jobF(j, L % 3), *Fn = jobF(j, (L + 1) % 3);
  const int nb = mssp_batch(j->sw);
  const unsigned idx = (unsigned)unit * kSsspPerUnit + (unsigned)lane;
  int v = -1, s = 0, d = 0;
  if (lane < kSsspPerUnit && idx < nq) {
    v = __ldcg(qin + idx);
    s = __ldg(j->ptr + v);
    d = __ldg(j->ptr + v + 1) - s;
  }
  const int incl = warp_incl_scan(d);
  const int excl = incl - d;
  const int total = __shfl_sync(kFull, incl, 31);
  for (int e0 = 0; e0 < total; e0 += nb) {
    const int e = e0 + lane;
    const int owner = warp_owner(excl, min(e, total - 1));
    const int so = __shfl_sync(kFull, s, owner);
    const int eo = __shfl_sync(kFull, excl, owner);
    const int vo = __shfl_sync(kFull, v, owner);
    int ue = 0, ve = 0;
    unsigned we = 0, me = 0;
    if (lane < nb && e < total) {
      const int k = so + (e - eo);
      ue = __ldg(j->ind + k);
      we = __ldg(j->w + k);
      ve = vo;
      me = (unsigned)__ldcg(Fc + vo);
    }
    bool f[1] = {mssp_relax(j, ue, we, ve, me, Fn)};
    int u1[1] = {ue}, dg[1] = {0};
    if (f[0]) dg[0] = __ldg(j->ptr + ue + 1) - __ldg(j->ptr + ue);
    append_n<1>(j, f, u1, dg, ac);
  }
}

// one kSsspChunk-edge chunk of a hub
__device__ void mssp_chunk(BatchJob *j, int L, int unit, const AppendCtx &ac) {
  const int lane = lane_id();
  int2 *cin = jobC(j, L % 3);
  unsigned long long *Fc = jobF(j, L % 3), *Fn = jobF(j, (L + 1) % 3);
  const int2 ch = __ldcg(cin + unit);
  const int v = ch.x;
  const int s = __ldg(j->ptr + v) + ch.y * kSsspChunk;
  const int e = min(s + kSsspChunk, __ldg(j->ptr + v + 1));
  const unsigned mv = (unsigned)__ldcg(Fc + v);
  const int nb = mssp_batch(j->sw);
  for (int k0 = s; k0 < e; k0 += nb) {
    const int k = k0 + lane;
    int ue = 0;
    unsigned we = 0, me = 0;
    if (lane < nb && k < e) {
      ue = __ldg(j->ind + k);
      we = __ldg(j->w + k);
      me = mv;
    }
    bool f[1] = {mssp_relax(j, ue, we, v, me, Fn)};
    int u1[1] = {ue}, dg[1] = {0};
    if (f[0]) dg[0] = __ldg(j->ptr + ue + 1) - __ldg(j->ptr + ue);
    append_n<1>(j, f, u1, dg, ac);
  }
}

// ------------------------------------------------------- SSSP pull steps ---
// Lists the (vertex, chunk) pull units of an SSSP job's vertices with more
// than kMsHubIn in-edges (after the job table upload, which zeroes nhc).
__global__ void batch_hub_chunks(BatchJob *jobs, int jid) {
  BatchJob *j = jobs + jid;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < j->m; v += gridDim.x * blockDim.x) {
    const int d = __ldg(j->stptr + v + 1) - __ldg(j->stptr + v);
    if (d > kMsHubIn) {
      const unsigned nc = (unsigned)((d + kMsPullChunk - 1) / kMsPullChunk);
      const unsigned at = atomicAdd(&j->nhc, nc);
      for (unsigned c = 0; c < nc; ++c) j->hubc[at + c] = make_int2(v, (int)c);
    }
  }
}

// Least d[u][s] + w(u, v) over in-edges [a0, a1) of v whose tail u changed
// for source s in the last step, for every source s at once: lane =
// (edge slot, source) with 32 / sw edge slots, the slots' minima combined
// by xor shuffles; lanes 0 .. sw-1 return the source's minimum.
__device__ __forceinline__ unsigned mssp_pull_min(const BatchJob *j, int a0, int a1,
                                                  const unsigned long long *Fc) {
  const int lane = lane_id();
  const int sw = j->sw, per = 32 / sw;
  const int src = lane & (sw - 1), eo = lane / sw;
  const unsigned *dist = reinterpret_cast<const unsigned *>(j->out);
  unsigned best = 0xffffffffu;
  // four in-edges per lane in flight: their indices, then their frontier
  // words, then the distances (each lane's k stays below a1: the loops
  // may run different counts per lane and meet again before the shuffles)
  int k = a0 + eo;
  if (src < j->nsrc) {
    for (; k + 3 * per < a1; k += 4 * per) {
      int u[4];
      unsigned fm[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) u[q] = __ldg(j->stind + k + q * per);
#pragma unroll
      for (int q = 0; q < 4; ++q) fm[q] = (unsigned)__ldcg(Fc + u[q]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if ((fm[q] >> src) & 1u)
          best = min(best, sat_add(__ldcg(dist + (size_t)u[q] * sw + src),
                                   __ldg(j->stw + k + q * per)));
    }
    for (; k < a1; k += per) {
      const int u = __ldg(j->stind + k);
      const unsigned fm = (unsigned)__ldcg(Fc + u);
      if ((fm >> src) & 1u) best = min(best, sat_add(__ldcg(dist + (size_t)u * sw + src),
                                                     __ldg(j->stw + k)));
    }
  }
  for (int o = sw; o < 32; o <<= 1) best = min(best, __shfl_xor_sync(kFull, best, o));
  return best;
}

// One pull unit of an SSSP job: a hub chunk (minima through atomicMin, the
// hub's other chunks run elsewhere) or kMsPullVerts vertices, each taken
// by the whole warp and written by it alone (no atomics).  Improved
// vertices get their next-frontier bits and are queued, as in a push step.
__device__ void mssp_pull(BatchJob *j, int L, int unit, const AppendCtx &ac) {
  const int lane = lane_id();
  const int sw = j->sw;
  unsigned *dist = reinterpret_cast<unsigned *>(j->out);
  const unsigned long long *Fc = jobF(j, L % 3);
  unsigned long long *Fn = jobF(j, (L + 1) % 3);
  const unsigned low = sw == 32 ? 0xffffffffu : ((1u << sw) - 1u);
  const bool mine = lane < sw && lane < j->nsrc;  // this lane's source after the reduction
  if ((unsigned)unit < j->nhc) {
    const int2 hc = j->hubc[unit];
    const int v = hc.x;
    const int a0 = __ldg(j->stptr + v) + hc.y * kMsPullChunk;
    const int a1 = min(__ldg(j->stptr + v + 1), a0 + kMsPullChunk);
    const unsigned best = mssp_pull_min(j, a0, a1, Fc);
    bool imp = false;
    if (mine && best < __ldcg(dist + (size_t)v * sw + lane)) {
      const unsigned old = atomicMin(dist + (size_t)v * sw + lane, best);
      imp = best < old;
    }
    const unsigned b = __ballot_sync(kFull, imp) & low;
    bool f[1] = {false};
    if (lane == 0 && b) f[0] = atomicOr(Fn + v, (unsigned long long)b) == 0ull;
    int u1[1] = {v}, dg[1] = {0};
    if (f[0]) dg[0] = __ldg(j->ptr + v + 1) - __ldg(j->ptr + v);
    append_n<1>(j, f, u1, dg, ac);
    return;
  }
  const int v0 = (unit - (int)j->nhc) * kMsPullVerts;
  for (int i = 0; i < kMsPullVerts; ++i) {
    const int v = v0 + i;
    if (v >= j->m) break;
    const int a0 = __ldg(j->stptr + v), a1 = __ldg(j->stptr + v + 1);
    if (a1 - a0 > kMsHubIn || a1 == a0) continue;  // a hub's chunks are units of their own
    const unsigned best = mssp_pull_min(j, a0, a1, Fc);
    bool imp = false;
    if (mine && best < __ldcg(dist + (size_t)v * sw + lane)) {
      dist[(size_t)v * sw + lane] = best;  // only this warp writes v in a pull step
      imp = true;
    }
    const unsigned b = __ballot_sync(kFull, imp) & low;
    bool f[1] = {lane == 0 && b != 0u};
    if (f[0]) Fn[v] = (unsigned long long)b;
    int u1[1] = {v}, dg[1] = {0};
    if (f[0]) dg[0] = __ldg(j->ptr + v + 1) - __ldg(j->ptr + v);
    append_n<1>(j, f, u1, dg, ac);
  }
}

// ---------------------------------------------------------------- kernel ---
__global__ void __launch_bounds__(kBatchThreads, 2)
batch_persistent(BatchJob *jobs, int njobs, BatchState *st, int max_steps) {
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const int warp = warp_in_block();
  __shared__ unsigned s_q[kMaxJobs], s_ch[kMaxJobs];
  __shared__ unsigned long long s_edges[kMaxJobs], s_explored[kMaxJobs];
  __shared__ unsigned s_prevq[kMaxJobs], s_prevch[kMaxJobs];
  __shared__ int s_pull[kMaxJobs], s_done[kMaxJobs];
  // unit layout per job: [clear queue][clear chunks][work: queue or pull][work chunks]
  __shared__ unsigned s_u0[kMaxJobs], s_u1[kMaxJobs], s_u2[kMaxJobs], s_u3[kMaxJobs];
  __shared__ unsigned s_pre[kMaxJobs + 1];
  __shared__ unsigned long long s_acc[kBatchThreads / 32][32];
  __shared__ int s_rank[kBatchThreads / 32][32];
  // appends: per-warp stages, per-block tallies of the next frontiers
  __shared__ int s_stq[kStageWarpsB][kJStageQ];
  __shared__ int2 s_stb[kStageWarpsB][kJStageB];
  __shared__ unsigned s_nbig_next[kMaxJobs];
  __shared__ unsigned long long s_edges_next[kMaxJobs];
  JobStage stg{s_stq[warp], s_stb[warp], 0, 0, nullptr, 0};

  for (int jj = threadIdx.x; jj < njobs; jj += blockDim.x) {
    s_explored[jj] = 0;
    s_pull[jj] = 0;
    s_done[jj] = 0;
    s_prevq[jj] = 0;
    s_prevch[jj] = 0;
  }
  __syncthreads();
  int step = 0;
  for (;; ++step) {
    // Step set-up, one thread per job (all blocks compute the same values
    // from counters nobody writes during this step): the job's frontier,
    // direction and units.
    if (threadIdx.x < njobs) {
      const int jj = threadIdx.x;
      BatchJob *j = jobs + jj;
      JobCounters *cur = &j->c[step % 3];
      const unsigned long long qc = __ldcg(&cur->qc);
      const unsigned q = (unsigned)qc, ch = (unsigned)(qc >> 32), nb = __ldcg(&cur->nbig);
      const unsigned long long ed = __ldcg(&cur->edges);
      s_q[jj] = q;
      s_ch[jj] = ch;
      s_edges[jj] = ed;
      if (blockIdx.x == 0) j->c[(step + 2) % 3] = JobCounters{0ull, 0, 0, 0ull};
      const unsigned long long nf = (unsigned long long)q + nb;
      const bool active = !s_done[jj] && nf > 0 && (max_steps <= 0 || step < max_steps);
      if (!active) s_done[jj] = 1;
      // clear the frontier words of level step-1 (they are reused at step+1)
      unsigned u0 = (s_prevq[jj] + 31) / 32, u1 = (s_prevch[jj] + 31) / 32, u2 = 0, u3 = 0;
      if (active) {
        s_explored[jj] += ed;
        if (j->type == kJobBfs) {
          long long unexplored = j->nnz - (long long)s_explored[jj];
          if (!s_pull[jj]) {
            if ((long long)ed * j->alpha > unexplored) s_pull[jj] = 1;
          } else if ((long long)nf * j->beta < (long long)j->m) {
            s_pull[jj] = 0;
          }
          if (s_pull[jj]) {
            u2 = (unsigned)((j->m + 31) / 32);
          } else {
            u2 = (q + 31) / 32;
            u3 = ch;
          }
        } else if (j->stptr && j->salpha > 0 && (long long)ed * j->salpha > j->nnz) {
          // pull step: hub chunks, then units of kMsPullVerts vertices
          s_pull[jj] = 1;
          u2 = j->nhc + (unsigned)((j->m + kMsPullVerts - 1) / kMsPullVerts);
        } else {
          s_pull[jj] = 0;
          u2 = (q + kSsspPerUnit - 1) / kSsspPerUnit;
          u3 = ch;
        }
      }
      s_u0[jj] = u0;
      s_u1[jj] = u1;
      s_u2[jj] = u2;
      s_u3[jj] = u3;
      s_nbig_next[jj] = 0;
      s_edges_next[jj] = 0;
    }
    __syncthreads();
    stg.level = step;
    stg.job = nullptr;
    // exclusive prefix of the jobs' unit counts (warp 0; at most 64 jobs)
    if (warp == 0) {
      const int lane = lane_id();
      unsigned carry = 0;
      for (int b = 0; b < njobs; b += 32) {
        const int jj = b + lane;
        const unsigned cnt = jj < njobs ? s_u0[jj] + s_u1[jj] + s_u2[jj] + s_u3[jj] : 0u;
        const unsigned incl = warp_incl_scan(cnt);
        if (jj < njobs) s_pre[jj] = carry + incl - cnt;
        carry += __shfl_sync(kFull, incl, 31);
      }
      if (lane == 0) s_pre[njobs] = carry;
    }
    const bool any_active = __syncthreads_or(threadIdx.x < njobs && !s_done[threadIdx.x]) != 0;
    const unsigned total = s_pre[njobs];
    if (!any_active) break;
    for (unsigned g = (unsigned)gwarp; g < total; g += (unsigned)nwarps) {
      int lo = 0, hi = njobs - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (s_pre[mid] <= g) lo = mid; else hi = mid - 1;
      }
      // skip empty jobs that share the same prefix
      while (lo + 1 < njobs && s_pre[lo + 1] <= g) ++lo;
      BatchJob *j = jobs + lo;
      const AppendCtx ac{&stg, s_nbig_next, s_edges_next, lo};
      unsigned loc = g - s_pre[lo];
      if (loc < s_u0[lo]) {
        msbfs_clear(j, step, (int)loc, s_prevq[lo], false);
        continue;
      }
      loc -= s_u0[lo];
      if (loc < s_u1[lo]) {
        msbfs_clear(j, step, (int)loc, s_prevch[lo], true);
        continue;
      }
      loc -= s_u1[lo];
      if (j->type == kJobBfs) {
        if (s_pull[lo]) {
          msbfs_pull(j, step, (int)loc, s_acc[warp], s_rank[warp], ac);
        } else if (loc < s_u2[lo]) {
          msbfs_push_queue(j, step, (int)loc, s_q[lo], ac);
        } else {
          msbfs_push_chunk(j, step, (int)(loc - s_u2[lo]), ac);
        }
      } else if (s_pull[lo]) {
        mssp_pull(j, step, (int)loc, ac);
      } else {
        if (loc < s_u2[lo])
          mssp_queue(j, step, (int)loc, s_q[lo], ac);
        else
          mssp_chunk(j, step, (int)(loc - s_u2[lo]), ac);
      }
    }
    stage_flush(stg);
    __syncthreads();
    if (threadIdx.x < njobs) {
      const int jj = threadIdx.x;
      JobCounters *nx = &jobs[jj].c[(step + 1) % 3];
      if (s_nbig_next[jj]) atomicAdd(&nx->nbig, s_nbig_next[jj]);
      if (s_edges_next[jj]) atomicAdd(&nx->edges, s_edges_next[jj]);
      // the frontier of this step is cleared two steps later
      const bool was_active = s_u2[jj] + s_u3[jj] > 0;
      s_prevq[jj] = was_active ? s_q[jj] : 0;
      s_prevch[jj] = was_active ? s_ch[jj] : 0;
      if (blockIdx.x == 0 && was_active && s_edges[jj]) atomicAdd(&st->edges, s_edges[jj]);
    }
    if (!grid_barrier(st->bar, &st->err)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->steps = step;
}

// vertex-major results [m][width] -> source-major out[s][m] for s < nsrc
// (width 64 or 32)
__global__ void batch_transpose(const int32_t *vm, int m, int width, int nsrc, int32_t *out) {
  __shared__ int32_t tile[32][65];
  const int v0 = blockIdx.x * 32;
  for (int t = threadIdx.x; t < 32 * width; t += blockDim.x) {
    int vv = t / width, s = t % width;
    tile[vv][s] = (v0 + vv < m) ? vm[(size_t)(v0 + vv) * width + s] : -1;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 32 * width; t += blockDim.x) {
    int s = t / 32, vv = t % 32;
    if (s < nsrc && v0 + vv < m) out[(size_t)s * m + v0 + vv] = tile[vv][s];
  }
}

int batch_grid(apspie_context *ctx) {
  return occupancy_grid(ctx, (const void *)batch_persistent, kBatchThreads);
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Jobs whose graphs take more levels than this run in their own launch with
// a small grid next to the others (a grid graph's ~2,000 levels of a few
// thousand vertices each would otherwise set the step count of the whole
// batch while the rest of the GPU idles).
constexpr int kDeepLevels = 64;

// BFS levels of graph J from its first vertex with edges (one probe BFS per
// graph), cached for the whole process by (device, row-offset pointer, m,
// nnz): every context and sub-context reads the same entry without touching
// the device.  The depth only routes a job (multi-source launch or
// concurrent single-source traversals); either route gives the same
// results, so a stale entry (a graph freed and another of the same size
// built at the same address) can only cost time.
struct DepthEntry {
  int dev;
  const int *ptr;
  int m;
  long long nnz;
  int levels;
};
std::mutex g_depth_mu;
std::vector<DepthEntry> g_depth_cache;

int graph_levels(apspie_context *ctx, const apspie_job &J, int *levels) {
  *levels = 0;
  if (J.nnz == 0) return APSPIE_OK;
  {
    std::lock_guard<std::mutex> lock(g_depth_mu);
    for (const auto &e : g_depth_cache)
      if (e.dev == ctx->device && e.ptr == J.d_ptr && e.m == J.m && e.nnz == J.nnz) {
        *levels = e.levels;
        return APSPIE_OK;
      }
  }
  const int nh = std::min(J.m, 4096);
  int *h = (int *)pinned(ctx, sizeof(int) * (nh + 1));
  if (!h) return APSPIE_ERR_OOM;
  cudaMemcpyAsync(h, J.d_ptr, sizeof(int) * (nh + 1), cudaMemcpyDeviceToHost, ctx->stream);
  int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "graph_levels");
  if (rc) return rc;
  int src = -1;
  for (int u = 0; u < nh && src < 0; ++u)
    if (h[u + 1] > h[u]) src = u;
  int lv = 0;
  if (src >= 0) {
    auto *depth = (int32_t *)workspace(ctx, kSlotDense, sizeof(int32_t) * (size_t)J.m);
    if (!depth) return APSPIE_ERR_OOM;
    const int *tp = J.d_tptr ? J.d_tptr : (J.symmetric ? J.d_ptr : nullptr);
    const int *ti = J.d_tptr ? J.d_tind : (J.symmetric ? J.d_ind : nullptr);
    rc = apspie_bfs(ctx, src, J.nnz, J.m, J.d_ptr, J.d_ind, tp, ti, depth, 0);
    apspie_bfs_stats bs;
    if (!rc) rc = apspie_bfs_get_stats(ctx, &bs);
    if (rc) return rc;
    lv = bs.levels;
  }
  std::lock_guard<std::mutex> lock(g_depth_mu);
  g_depth_cache.push_back(DepthEntry{ctx->device, J.d_ptr, J.m, (long long)J.nnz, lv});
  *levels = lv;
  return APSPIE_OK;
}

// Distance-row width of an SSSP job: the sources rounded up to a power of two.
int row_width(int nsrc) {
  int w = 1;
  while (w < nsrc) w <<= 1;
  return w;
}

// Chunk-list capacity of a job: its big vertices have more than big_deg edges.
size_t job_chunk_capacity(long long nnz, bool bfs) {
  const long long bd = bfs ? kBigDeg : kSsspBigDeg, ck = bfs ? kChunk : kSsspChunk;
  return (size_t)(nnz / ck + nnz / bd + 2);
}

// The deep jobs' sources as single-source traversals, spread over up to
// batch_deep_subs sub-contexts (each its own stream and workspace) and run
// concurrently next to whatever is already queued on the context's stream
// (which waits for them at the end).  Sources go to the least loaded
// sub-context, SSSP first; each traversal gets budget / K blocks.  SSSP
// runs near-far (the context's step, else kDeepDelta): on a deep weighted
// graph frontier Bellman-Ford re-relaxes every edge dozens of times (211 M
// relaxations for 4.2 M edges on the 1024 x 1024 grid, weights 1..255),
// which needs a large grid per source, while near-far does 7 M over 40 %
// more rounds and runs on a few blocks.  Results are written straight into
// the caller's rows.
constexpr unsigned kDeepDelta = 1024;
int ensure_subs(apspie_context *ctx, int k) {
  while ((int)ctx->subs.size() < k) {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      if (s) cudaStreamDestroy(s);
      return check_cuda(ctx, cudaGetLastError(), "apspie_batch_run: sub-context stream");
    }
    apspie_ctx sub = nullptr;
    int rc = apspie_ctx_create(ctx->device, s, &sub);
    if (rc) {
      cudaStreamDestroy(s);
      cudaEventDestroy(ev);
      return set_error(ctx, rc, "apspie_batch_run: sub-context");
    }
    sub->owns_stream = true;
    ctx->subs.push_back(sub);
    ctx->sub_done.push_back(ev);
  }
  return APSPIE_OK;
}

int run_deep_sources(apspie_context *ctx, int njobs, const apspie_job *jobs,
                     const std::vector<char> &deep_job, int budget) {
  int nsrc = 0;
  for (int i = 0; i < njobs; ++i)
    if (deep_job[i]) nsrc += jobs[i].nsrc;
  const int K = std::max(1, std::min(nsrc, ctx->batch_deep_subs));
  int rc = ensure_subs(ctx, K);
  if (rc) return rc;
  if (!ctx->aux_done &&
      cudaEventCreateWithFlags(&ctx->aux_done, cudaEventDisableTiming) != cudaSuccess)
    return check_cuda(ctx, cudaGetLastError(), "apspie_batch_run: event");
  // the sub-streams start after everything queued so far (inputs, uploads)
  cudaEventRecord(ctx->aux_done, ctx->stream);
  const int grid = std::max(1, budget / K);
  for (int k = 0; k < K; ++k) {
    apspie_context *sub = ctx->subs[k];
    cudaStreamWaitEvent(sub->stream, ctx->aux_done, 0);
    sub->max_grid = grid;
    sub->bfs_alpha = ctx->bfs_alpha;
    sub->bfs_beta = ctx->bfs_beta;
    sub->bfs_mode = ctx->bfs_mode;
    sub->sssp_delta_u32 = ctx->sssp_delta_u32 ? ctx->sssp_delta_u32 : kDeepDelta;
  }
  std::vector<double> load(K, 0.0);
  for (int pass = 0; pass < 2; ++pass)  // SSSP sources first, then BFS
    for (int i = 0; i < njobs; ++i) {
      const apspie_job &J = jobs[i];
      const bool bfs = J.type == APSPIE_JOB_BFS;
      if (!deep_job[i] || bfs != (pass == 1)) continue;
      const int *tp = J.d_tptr ? J.d_tptr : (J.symmetric ? J.d_ptr : nullptr);
      const int *ti = J.d_tptr ? J.d_tind : (J.symmetric ? J.d_ind : nullptr);
      for (int s = 0; s < J.nsrc; ++s) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[k] += 1.0;
        apspie_context *sub = ctx->subs[k];
        int32_t *out = J.d_out + (size_t)s * J.m;
        rc = bfs ? apspie_bfs(sub, J.h_src[s], J.nnz, J.m, J.d_ptr, J.d_ind, tp, ti, out, 0)
                 : apspie_sssp_u32(sub, J.h_src[s], J.nnz, J.m, J.d_ptr, J.d_ind, J.d_w,
                                   reinterpret_cast<uint32_t *>(out), 0);
        if (rc) return set_error(ctx, rc, "apspie_batch_run: deep source: %s",
                                 sub->last_error.c_str());
      }
    }
  for (int k = 0; k < K; ++k) {
    ctx->launches += ctx->subs[k]->launches;
    ctx->subs[k]->launches = 0;
    cudaEventRecord(ctx->sub_done[k], ctx->subs[k]->stream);
    cudaStreamWaitEvent(ctx->stream, ctx->sub_done[k], 0);
  }
  ctx->batch_subs_used = K;
  return check_cuda(ctx, cudaGetLastError(), "apspie_batch_run: deep sources");
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_batch_run(apspie_ctx ctx, int njobs, const apspie_job *jobs, int max_steps) {
  return api_guard([&]() -> int {
    APSPIE_CHECK_CTX(ctx);
    if (njobs <= 0 || !jobs)
      return set_error(ctx, APSPIE_ERR_INVALID, "apspie_batch_run: no jobs");
    for (int i = 0; i < njobs; ++i) {
      const apspie_job &J = jobs[i];
      if ((J.type != APSPIE_JOB_BFS && J.type != APSPIE_JOB_SSSP_U32) || J.m <= 0 || J.nnz < 0 ||
          J.nnz >= (int64_t)INT32_MAX || J.nsrc <= 0 || !J.h_src || !J.d_ptr || !J.d_out ||
          (J.nnz > 0 && !J.d_ind) || (J.type == APSPIE_JOB_SSSP_U32 && J.nnz > 0 && !J.d_w) ||
          (J.d_stptr && J.nnz > 0 && (!J.d_stind || !J.d_stw)))
        return set_error(ctx, APSPIE_ERR_INVALID, "apspie_batch_run: bad job %d", i);
      for (int s = 0; s < J.nsrc; ++s)
        if (J.h_src[s] < 0 || J.h_src[s] >= J.m)
          return set_error(ctx, APSPIE_ERR_INVALID, "apspie_batch_run: job %d source %d out of range",
                           i, J.h_src[s]);
    }
    // Jobs on deep graphs (a BFS of more than kDeepLevels levels, probed once
    // per graph) are latency bound per level and gain little from sharing
    // their levels: their sources run as independent single-source traversals,
    // concurrently on sub-contexts with small grids.  The others are split
    // into device jobs of at most 64 (BFS) / 32 (SSSP) sources for one
    // multi-source launch.
    std::vector<char> deep_job(njobs, 0);
    if (max_steps <= 0 && ctx->batch_deep_subs > 0)
      for (int i = 0; i < njobs; ++i) {
        int lv = 0;
        int rc0 = graph_levels(ctx, jobs[i], &lv);
        if (rc0) return rc0;
        deep_job[i] = lv > kDeepLevels;
      }
    struct Part {
      int job, first, n;
    };
    std::vector<Part> parts;
    int ndeep_src = 0;
    for (int i = 0; i < njobs; ++i) {
      const apspie_job &J = jobs[i];
      if (deep_job[i]) {
        ndeep_src += J.nsrc;
        continue;
      }
      const int width = J.type == APSPIE_JOB_BFS ? kMsbfsWidth : kMssspWidth;
      for (int f = 0; f < J.nsrc; f += width)
        parts.push_back(Part{i, f, std::min(width, J.nsrc - f)});
    }
    const int nparts = (int)parts.size();
    if (nparts > kMaxJobs)
      return set_error(ctx, APSPIE_ERR_INVALID, "apspie_batch_run: %d device jobs > %d", nparts,
                       kMaxJobs);
    const int full = persistent_grid(ctx, batch_grid(ctx), ctx->batch_blocks_per_sm);
    if (full <= 0) return set_error(ctx, APSPIE_ERR_CUDA, "apspie_batch_run: occupancy query failed");
    // the deep sources get deep_blocks in all (default half the resident
    // blocks: their traversals are latency bound, a grid filled to the last
    // block slowed them down, and the multi-source launch beside them needs
    // the rest; measured on the batched benchmark)
    const int deep_budget =
        ndeep_src == 0 ? 0
                       : std::max(1, std::min(full - (nparts > 0 ? 1 : 0),
                                              ctx->deep_blocks > 0 ? ctx->deep_blocks : full / 2));
    const int grid1 = std::max(1, full - (nparts > 0 ? deep_budget : 0));
    cudaStream_t st = ctx->stream;
    int rc = APSPIE_OK;
    ctx->batch_state = nullptr;
    ctx->batch_subs_used = 0;
    if (nparts > 0) {
      // workspace layout per device job
      std::vector<size_t> off(nparts + 1, 0);
      size_t total = align_up(sizeof(BatchJob) * kMaxJobs) + align_up(sizeof(BatchState)) +
                     align_up(sizeof(int) * 64 * kMaxJobs);
      for (int p = 0; p < nparts; ++p) {
        const apspie_job &J = jobs[parts[p].job];
        const bool bfs = J.type == APSPIE_JOB_BFS;
        const size_t m = (size_t)J.m, cap = job_chunk_capacity(J.nnz, bfs);
        size_t b = 0;
        b += align_up(8 * m) * (bfs ? 4 : 3);  // (BFS: visited +) 3 frontier masks
        b += align_up(4 * m) * 3;              // queues
        b += align_up(8 * cap) * 3;            // chunk lists
        b += align_up(4 * m * row_width(parts[p].n));  // vertex-major results
        if (!bfs && J.d_stptr)  // hub chunks of the SSSP pull steps
          b += align_up(8 * ((size_t)J.nnz / kMsPullChunk + (size_t)J.nnz / kMsHubIn + 1));
        off[p] = total;
        total += b;
      }
      unsigned char *ws = (unsigned char *)workspace(ctx, kSlotBatch, total);
      if (!ws) return APSPIE_ERR_OOM;
      auto *djobs = (BatchJob *)ws;
      auto *dstate = (BatchState *)(ws + align_up(sizeof(BatchJob) * kMaxJobs));
      int *dsrc = (int *)(ws + align_up(sizeof(BatchJob) * kMaxJobs) + align_up(sizeof(BatchState)));
      // host image of the job table (pinned, copied in one transfer), in a
      // ring of upload buffers: no wait for the stream's earlier kernels
      size_t host_bytes = sizeof(BatchJob) * nparts + sizeof(int) * 64 * nparts;
      int up_slot = 0;
      auto *hjobs = (BatchJob *)upload_buffer(ctx, host_bytes, &up_slot);
      if (!hjobs) return APSPIE_ERR_OOM;
      int *hsrc = (int *)(hjobs + nparts);
      for (int p = 0; p < nparts; ++p) {
        const apspie_job &J = jobs[parts[p].job];
        BatchJob &B = hjobs[p];
        std::memset(&B, 0, sizeof(B));
        B.type = J.type == APSPIE_JOB_BFS ? kJobBfs : kJobSssp;
        B.m = J.m;
        B.nnz = J.nnz;
        B.nsrc = parts[p].n;
        B.ptr = J.d_ptr;
        B.ind = J.d_ind;
        B.tptr = J.d_tptr ? J.d_tptr : J.d_ptr;
        B.tind = J.d_tptr ? J.d_tind : J.d_ind;
        B.w = J.d_w;
        B.alpha = J.alpha >= 0 ? J.alpha : ctx->bfs_alpha;
        B.beta = J.beta >= 0 ? J.beta : ctx->bfs_beta;
        // no in-adjacency for a directed graph: never pull (alpha 0)
        if (!J.d_tptr && !J.symmetric) B.alpha = 0;
        for (int s = 0; s < parts[p].n; ++s) hsrc[p * 64 + s] = J.h_src[parts[p].first + s];
        B.src = dsrc + p * 64;
        unsigned char *b = ws + off[p];
        const bool bfs = B.type == kJobBfs;
        const size_t m = (size_t)J.m, cap = job_chunk_capacity(J.nnz, bfs);
        B.big_deg = bfs ? kBigDeg : kSsspBigDeg;
        B.sw = row_width(B.nsrc);  // result row: the sources rounded up to a power of two
        B.chunk = bfs ? kChunk : kSsspChunk;
        if (bfs) {
          B.visited = (unsigned long long *)b;
          b += align_up(8 * m);
        }
        B.F0 = (unsigned long long *)b; b += align_up(8 * m);
        B.F1 = (unsigned long long *)b; b += align_up(8 * m);
        B.F2 = (unsigned long long *)b; b += align_up(8 * m);
        B.q0 = (int *)b; b += align_up(4 * m);
        B.q1 = (int *)b; b += align_up(4 * m);
        B.q2 = (int *)b; b += align_up(4 * m);
        B.c0 = (int2 *)b; b += align_up(8 * cap);
        B.c1 = (int2 *)b; b += align_up(8 * cap);
        B.c2 = (int2 *)b; b += align_up(8 * cap);
        B.out = (int32_t *)b;  // vertex-major; transposed into the caller's array after
        b += align_up(4 * m * B.sw);
        if (!bfs && J.d_stptr) {
          B.stptr = J.d_stptr;
          B.stind = J.d_stind;
          B.stw = J.d_stw;
          B.salpha = ctx->sssp_pull_alpha_batch;
          B.hubc = (int2 *)b;
        }
      }
      cudaMemcpyAsync(djobs, hjobs, host_bytes, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(dsrc, hsrc, sizeof(int) * 64 * nparts, cudaMemcpyHostToDevice, st);
      rc = upload_done(ctx, up_slot);
      if (rc) return rc;
      cudaMemsetAsync(dstate, 0, align_up(sizeof(BatchState)), st);
      rc = check_cuda(ctx, cudaGetLastError(), "apspie_batch_run upload");
      if (rc) return rc;
      int nhub_launches = 0;
      for (int p = 0; p < nparts; ++p) {
        const long long m = jobs[parts[p].job].m;
        int g = (int)std::max(1ll, std::min((m * hjobs[p].sw + 255) / 256, (long long)ctx->num_sms * 8));
        if (hjobs[p].type == kJobBfs) {
          batch_init_bfs<<<g, 256, 0, st>>>(djobs, p);
          batch_seed_bfs<<<1, 64, 0, st>>>(djobs, p);
        } else {
          batch_init_sssp<<<g, 256, 0, st>>>(djobs, p);
          batch_seed_sssp<<<1, 32, 0, st>>>(djobs, p);
          if (hjobs[p].stptr) {
            batch_hub_chunks<<<std::min(g, ctx->num_sms * 4), 256, 0, st>>>(djobs, p);
            ++nhub_launches;
          }
        }
      }
      rc = check_launch(ctx, "batch init", 2 * nparts + nhub_launches);
      if (rc) return rc;
      int n1 = nparts;
      void *args1[] = {&djobs, &n1, &dstate, &max_steps};
      cudaError_t e = cudaLaunchCooperativeKernel((const void *)batch_persistent, dim3(grid1),
                                                  dim3(kBatchThreads), args1, 0, st);
      if (e != cudaSuccess) return check_cuda(ctx, e, "batch_persistent");
      ctx->launches += 1;
      for (int p = 0; p < nparts; ++p) {
        const apspie_job &J = jobs[parts[p].job];
        batch_transpose<<<(J.m + 31) / 32, 256, 0, st>>>(
            hjobs[p].out, J.m, hjobs[p].sw, parts[p].n, J.d_out + (size_t)parts[p].first * J.m);
      }
      rc = check_launch(ctx, "batch_transpose", nparts);
      if (rc) return rc;
      ctx->batch_state = dstate;
    }
    if (ndeep_src > 0) {
      rc = run_deep_sources(ctx, njobs, jobs, deep_job, deep_budget);
      if (rc) return rc;
    }
    return APSPIE_OK;
  });
}

int apspie_batch_get_stats(apspie_ctx ctx, apspie_batch_stats *out) {
  APSPIE_CHECK_CTX(ctx);
  if (!out || (!ctx->batch_state && ctx->batch_subs_used == 0))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_batch_get_stats: no batch has run");
  out->super_steps = 0;
  out->frontier_edges = 0;
  int err = 0;
  if (ctx->batch_state) {
    auto *h = (BatchState *)pinned(ctx, sizeof(BatchState));
    if (!h) return APSPIE_ERR_OOM;
    cudaMemcpyAsync(h, ctx->batch_state, sizeof(BatchState), cudaMemcpyDeviceToHost, ctx->stream);
    int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "apspie_batch_get_stats");
    if (rc) return rc;
    out->super_steps = h->steps;
    out->frontier_edges = (int64_t)h->edges;
    err = h->err;
  }
  // deep sources: each sub-context's last traversal of each kind (a barrier
  // timeout leaves its device stuck, so the later runs on it time out too);
  // super_steps counts their levels / rounds as well
  for (int k = 0; k < ctx->batch_subs_used; ++k) {
    apspie_context *sub = ctx->subs[k];
    if (sub->bfs_state) {
      apspie_bfs_stats b;
      if (apspie_bfs_get_stats(sub, &b) == APSPIE_ERR_TIMEOUT) err = 1;
      else out->super_steps = std::max(out->super_steps, b.levels);
    }
    if (sub->sssp_state) {
      apspie_sssp_stats q;
      if (apspie_sssp_get_stats(sub, &q) == APSPIE_ERR_TIMEOUT) err = 1;
      else out->super_steps = std::max(out->super_steps, q.rounds);
    }
  }
  if (err) return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_batch_run: grid barrier timed out");
  return APSPIE_OK;
}

}  // extern "C"
