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
// Distances are kept as 32-bit words: uint32 sums for integer weights, and
// the IEEE bit pattern for float weights -- non-negative floats order like
// their bit patterns, so atomicMin on the word is min on the value.  Each
// float relaxation is one round-to-nearest single add, and chaotic
// relaxation converges to the unique fixpoint of
// d[v] = min(d[v], min_u fl(d[u] + w(u,v))), so the result is bit-identical
// to the reference's label-correcting CPU SSSP (src/testSssp.cpp:33-115).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "context.h"
#include "frontier.cuh"

namespace apspie {
namespace {

constexpr int kSsspThreads = 512;

struct SsspState {
  LevelCounters c[3];
  unsigned bar[2];
  int err;
  int rounds;
  unsigned long long relaxations;  // edges scanned over all rounds
  unsigned long long reached;
  unsigned long long edges;        // sum of out-degrees of reached vertices
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
};

template <>
struct Arith<float> {
  static constexpr unsigned kInf = 0x7f800000u;  // +inf
  __device__ __forceinline__ static unsigned add(unsigned d, float w) {
    return __float_as_uint(__fadd_rn(__uint_as_float(d), w));
  }
};

// Push visitor: relax (u, w[k]) with the source's distance du as payload.
template <typename W>
struct SsspVisit {
  const W *__restrict__ w;
  unsigned *dist;
  int *stamp;
  int round;
  __device__ __forceinline__ bool check(unsigned du, int k, int u, unsigned &nd) const {
    nd = Arith<W>::add(du, __ldg(w + k));
    return nd < __ldcg(dist + u);
  }
  __device__ __forceinline__ bool commit(unsigned, int, int u, unsigned nd) const {
    if (nd >= atomicMin(dist + u, nd)) return false;
    return atomicExch(stamp + u, round) != round;
  }
};

template <typename W>
__global__ void sssp_init(int m, int src, unsigned *dist, int *stamp, const int *__restrict__ ptr,
                          int *queue, int2 *chunks, SsspState *st) {
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    dist[v] = (v == src) ? 0u : Arith<W>::kInf;
    stamp[v] = -1;
  }
  if (blockIdx.x == 0) {
    seed_frontier(src, ptr, queue, chunks, &st->c[0]);
    if (threadIdx.x == 0) {
      st->c[1] = LevelCounters{0ull, 0, 0, 0ull};
      st->c[2] = LevelCounters{0ull, 0, 0, 0ull};
      st->bar[0] = st->bar[1] = 0;
      st->err = 0;
      st->rounds = 0;
      st->relaxations = 0;
      st->reached = 0;
      st->edges = 0;
    }
  }
}

template <typename W>
__global__ void __launch_bounds__(kSsspThreads, 3)
sssp_persistent(int m, const int *__restrict__ ptr, const int *__restrict__ ind,
                const W *__restrict__ w, unsigned *dist, int *stamp, int *qa, int *qb, int2 *ca,
                int2 *cb, SsspState *st, int max_rounds) {
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  __shared__ unsigned s_q, s_chunks;
  __shared__ unsigned long long s_edges;
  unsigned long long relax = 0;
  int r = 0;
  for (;; ++r) {
    LevelCounters *cur = &st->c[r % 3];
    LevelCounters *nxt = &st->c[(r + 1) % 3];
    LevelCounters *clr = &st->c[(r + 2) % 3];
    if (threadIdx.x == 0) {
      const unsigned long long qc = __ldcg(&cur->qc);
      s_q = qc_queue(qc);
      s_chunks = qc_chunks(qc);
      s_edges = __ldcg(&cur->edges);
      if (blockIdx.x == 0) *clr = LevelCounters{0ull, 0, 0, 0ull};
    }
    __syncthreads();
    const unsigned nq = s_q, nch = s_chunks;
    if (nq == 0 && nch == 0) break;
    if (max_rounds > 0 && r >= max_rounds) break;
    relax += s_edges;
    int *qin = (r & 1) ? qb : qa;
    int *qout = (r & 1) ? qa : qb;
    int2 *cin = (r & 1) ? cb : ca;
    int2 *cout = (r & 1) ? ca : cb;
    SsspVisit<W> vis{w, dist, stamp, r};
    expand_push(ptr, ind, qin, nq, cin, nch, qout, cout, nxt, gwarp, nwarps,
                [&](int v) { return __ldcg(dist + v); }, vis);
    if (!grid_barrier(st->bar, &st->err)) return;
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
    st->relaxations = relax;
  }
}

template <typename W>
int sssp_grid(apspie_context *ctx) {
  static int cached_dev = -1, cached_grid = 0;
  if (cached_dev == ctx->device && cached_grid > 0) return cached_grid;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sssp_persistent<W>, kSsspThreads, 0) !=
          cudaSuccess ||
      occ < 1) {
    cudaGetLastError();
    return 0;
  }
  cached_dev = ctx->device;
  cached_grid = occ * ctx->num_sms;
  return cached_grid;
}

template <typename W>
int sssp_run(apspie_context *ctx, int src, int64_t nnz, int m, const int *d_ptr, const int *d_ind,
             const W *d_w, unsigned *d_dist, int max_rounds) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || src < 0 || src >= m)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp: src %d outside [0,%d)", src, m);
  if (nnz < 0 || nnz >= (int64_t)INT32_MAX)
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "apspie_sssp: nnz exceeds int32 offsets");
  if (!d_ptr || !d_dist || (nnz > 0 && (!d_ind || !d_w)))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_sssp: null pointer");
  size_t cap = chunk_capacity(nnz);
  auto *st = (SsspState *)workspace(ctx, kSlotSsspState, sizeof(SsspState));
  auto *qa = (int *)workspace(ctx, kSlotSsspQueueA, sizeof(int) * (size_t)m);
  auto *qb = (int *)workspace(ctx, kSlotSsspQueueB, sizeof(int) * (size_t)m);
  auto *ca = (int2 *)workspace(ctx, kSlotSsspChunksA, sizeof(int2) * cap);
  auto *cb = (int2 *)workspace(ctx, kSlotSsspChunksB, sizeof(int2) * cap);
  auto *stamp = (int *)workspace(ctx, kSlotSsspStamp, sizeof(int) * (size_t)m);
  if (!st || !qa || !qb || !ca || !cb || !stamp) return APSPIE_ERR_OOM;
  ctx->sssp_state = st;
  int grid = sssp_grid<W>(ctx);
  if (grid <= 0) return set_error(ctx, APSPIE_ERR_CUDA, "apspie_sssp: occupancy query failed");
  int init_grid = std::min((m + 255) / 256, ctx->num_sms * 8);
  sssp_init<W><<<init_grid, 256, 0, ctx->stream>>>(m, src, d_dist, stamp, d_ptr, qa, ca, st);
  int rc = check_launch(ctx, "sssp_init");
  if (rc) return rc;
  void *args[] = {&m,  (void *)&d_ptr, (void *)&d_ind, (void *)&d_w, &d_dist, &stamp,
                  &qa, &qb,            &ca,            &cb,           &st,     &max_rounds};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)sssp_persistent<W>, dim3(grid),
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
  return sssp_run<uint32_t>(ctx, src, nnz, m, d_ptr, d_ind, d_w, d_dist, max_rounds);
}

int apspie_sssp_f32(apspie_ctx ctx, int src, int64_t nnz, int m, const int *d_ptr,
                    const int *d_ind, const float *d_w, float *d_dist, int max_rounds) {
  return sssp_run<float>(ctx, src, nnz, m, d_ptr, d_ind, d_w, (unsigned *)d_dist, max_rounds);
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
  out->vertices_reached = (int64_t)h->reached;
  out->edges_traversed = (int64_t)h->edges;
  out->relaxations = (int64_t)h->relaxations;
  if (h->err)
    return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_sssp: grid barrier timed out");
  return APSPIE_OK;
}

}  // extern "C"
