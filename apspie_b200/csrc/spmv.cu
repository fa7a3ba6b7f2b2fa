// spmv.cu -- dense SpMV y = A (x) x over every row of a CSR matrix, under the
// four semirings of the library: the fully dense end of the push/pull
// continuum, where every vertex is in the frontier.
//
// Replaces the reference's dense SpMV calls: mgpu::SpmvCsrBinary behind
// spmv() (src/bfs.cuh:12-14) and cusparseScsrmv behind cuspmv()
// (src/tc.cuh:18-59).  Rows of at most kLongRow entries go one warp per row
// (lanes stride the row, indices and values read coalesced, x gathered);
// longer rows (hubs) are listed during that pass and reduced by a whole block
// each.  Each row is reduced in a fixed order (per-lane partials, then a
// fixed butterfly / tree), so the result does not depend on scheduling.
// PLUS_TIMES accumulates in double and rounds once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "context.h"

namespace apspie {
namespace {

constexpr int kSr_PlusTimes = 0, kSr_MinPlus = 1, kSr_MaxTimes = 2, kSr_OrAnd = 3;
constexpr int kLongRow = 4096;
constexpr int kLongThreads = 512;

struct SpmvSmall {
  unsigned nlong;
  unsigned pad;
};

// the semiring's (+) identity and one (x) term, as float (double for plus)
__device__ __forceinline__ double sr_identity(int sr) {
  switch (sr) {
    case kSr_MinPlus: return (double)FLT_MAX;
    case kSr_MaxTimes: return -(double)FLT_MAX;
    default: return 0.0;  // PLUS_TIMES, OR_AND
  }
}

__device__ __forceinline__ double sr_term(int sr, float a, float x) {
  switch (sr) {
    case kSr_MinPlus: return (double)__fadd_rn(a, x);
    case kSr_MaxTimes: return (double)__fmul_rn(a, x);
    case kSr_OrAnd: return (a != 0.0f && x != 0.0f) ? 1.0 : 0.0;
    default: return (double)a * (double)x;  // PLUS_TIMES: exact product in double
  }
}

__device__ __forceinline__ double sr_add(int sr, double p, double q) {
  switch (sr) {
    case kSr_MinPlus: return fmin(p, q);
    case kSr_MaxTimes: return fmax(p, q);
    case kSr_OrAnd: return (p != 0.0 || q != 0.0) ? 1.0 : 0.0;
    default: return p + q;
  }
}

__device__ __forceinline__ float sr_out(int sr, double v) {
  // MIN_PLUS / MAX_TIMES terms are floats already; PLUS_TIMES rounds once
  return (float)v;
}

__global__ void spmv_warp_rows(int sr, int m, const int *__restrict__ ptr,
                               const int *__restrict__ ind, const float *__restrict__ val,
                               const float *__restrict__ x, float *y, unsigned *nlong,
                               int *long_rows) {
  const int lane = lane_id();
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m;
       r += (gridDim.x * blockDim.x) >> 5) {
    const int s = __ldg(ptr + r), e = __ldg(ptr + r + 1);
    if (e - s > kLongRow) {
      if (lane == 0) long_rows[atomicAdd(nlong, 1u)] = r;
      continue;
    }
    double acc = sr_identity(sr);
    for (int k = s + lane; k < e; k += 32) {
      const float a = val ? __ldg(val + k) : 1.0f;
      acc = sr_add(sr, acc, sr_term(sr, a, __ldg(x + __ldg(ind + k))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = sr_add(sr, acc, __shfl_xor_sync(kFull, acc, o));
    if (lane == 0) y[r] = sr_out(sr, acc);
  }
}

__global__ void __launch_bounds__(kLongThreads)
spmv_long_rows(int sr, const int *__restrict__ ptr, const int *__restrict__ ind,
               const float *__restrict__ val, const float *__restrict__ x, float *y,
               const unsigned *nlong, const int *long_rows) {
  __shared__ double part[kLongThreads / 32];
  const int lane = lane_id(), w = warp_in_block();
  const unsigned n = *nlong;
  for (unsigned i = blockIdx.x; i < n; i += gridDim.x) {
    const int r = long_rows[i];
    const int s = __ldg(ptr + r), e = __ldg(ptr + r + 1);
    double acc = sr_identity(sr);
    for (int k = s + (int)threadIdx.x; k < e; k += kLongThreads) {
      const float a = val ? __ldg(val + k) : 1.0f;
      acc = sr_add(sr, acc, sr_term(sr, a, __ldg(x + __ldg(ind + k))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = sr_add(sr, acc, __shfl_xor_sync(kFull, acc, o));
    if (lane == 0) part[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = part[0];
      for (int j = 1; j < kLongThreads / 32; ++j) t = sr_add(sr, t, part[j]);
      y[r] = sr_out(sr, t);
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" int apspie_spmv(apspie_ctx ctx, int semiring, int m, int64_t nnz, const int *d_ptr,
                           const int *d_ind, const float *d_val, const float *d_x, float *d_y) {
  APSPIE_CHECK_CTX(ctx);
  if (semiring < 0 || semiring > 3 || m <= 0 || nnz < 0 || nnz >= (int64_t)INT32_MAX || !d_ptr ||
      (nnz > 0 && !d_ind) || !d_x || !d_y)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_spmv: bad arguments");
  auto *sm = (SpmvSmall *)workspace(ctx, kSlotSmall, sizeof(SpmvSmall));
  auto *rows = (int *)workspace(ctx, kSlotMisc0, sizeof(int) * ((size_t)nnz / kLongRow + 1));
  if (!sm || !rows) return APSPIE_ERR_OOM;
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(&sm->nlong, 0, sizeof(unsigned), st);
  const long long warps = std::min((long long)m, (long long)ctx->num_sms * 64);
  spmv_warp_rows<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(
      semiring, m, d_ptr, d_ind, d_val, d_x, d_y, &sm->nlong, rows);
  spmv_long_rows<<<ctx->num_sms * 2, kLongThreads, 0, st>>>(semiring, d_ptr, d_ind, d_val, d_x,
                                                           d_y, &sm->nlong, rows);
  return check_launch(ctx, "apspie_spmv", 2);
}
