// spmv.cu -- dense SpMV y = A (x) x over every row of a CSR matrix, under the
// four semirings of the library: the fully dense end of the push/pull
// continuum, where every vertex is in the frontier.
//
// Replaces the reference's dense SpMV calls: mgpu::SpmvCsrBinary behind
// spmv() (src/bfs.cuh:12-14) and cusparseScsrmv behind cuspmv()
// (src/tc.cuh:18-59).  Three tiers: rows of at most kMidRow entries go to
// groups of L lanes (L = 4 .. 32 from the mean row length, 32 / L rows per
// warp in flight, so that short rows do not leave a warp with one chain of
// dependent loads); rows of at most kLongRow entries are listed and go one
// warp per row; longer rows (hubs) are listed and split into chunks that
// are spread over all blocks.  Each row is reduced in a fixed
// order (per-lane partials, then a fixed butterfly / tree, then the chunks
// in order), so the result does not depend on scheduling.
// PLUS_TIMES accumulates in double and rounds once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "context.h"

namespace apspie {
namespace {

constexpr int kSr_PlusTimes = 0, kSr_MinPlus = 1, kSr_MaxTimes = 2, kSr_OrAnd = 3;
constexpr int kMidRow = 256;
constexpr int kLongRow = 4096;
constexpr int kLongThreads = 512;

struct SpmvSmall {
  unsigned nlong;
  unsigned nmid;
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

// Sum of the terms of entries k0, k0 + stride, ... < k1 in a fixed order:
// four index loads, then four x loads, in flight per step (the loads of a
// lane's entries are independent; a plain loop would wait for each x
// before issuing the next index load).
__device__ __forceinline__ double row_part(int sr, int k0, int k1, int stride,
                                           const int *__restrict__ ind,
                                           const float *__restrict__ val,
                                           const float *__restrict__ x) {
  double acc = sr_identity(sr);
  int k = k0;
  for (; k + 3 * stride < k1; k += 4 * stride) {
    int c[4];
    float a[4], xv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      c[q] = __ldg(ind + k + q * stride);
      a[q] = val ? __ldg(val + k + q * stride) : 1.0f;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) xv[q] = __ldg(x + c[q]);
#pragma unroll
    for (int q = 0; q < 4; ++q) acc = sr_add(sr, acc, sr_term(sr, a[q], xv[q]));
  }
  for (; k < k1; k += stride) {
    const float a = val ? __ldg(val + k) : 1.0f;
    acc = sr_add(sr, acc, sr_term(sr, a, __ldg(x + __ldg(ind + k))));
  }
  return acc;
}

// Groups of L lanes, one row each; rows longer than kMidRow are listed for
// spmv_warp_rows.  The row loop is warp-uniform (every lane runs the same
// number of batches), so the group reductions stay converged.
template <int L>
__global__ void spmv_group_rows(int sr, int m, const int *__restrict__ ptr,
                                const int *__restrict__ ind, const float *__restrict__ val,
                                const float *__restrict__ x, float *y, unsigned *nmid,
                                int *mid_rows) {
  constexpr int G = 32 / L;
  const int lane = lane_id(), sub = lane & (L - 1), grp = lane / L;
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int base = gwarp * G; base < m; base += nwarps * G) {
    const int r = base + grp;
    int s = 0, e = 0;
    if (r < m) {
      s = __ldg(ptr + r);
      e = __ldg(ptr + r + 1);
    }
    const bool mid = e - s > kMidRow;
    if (mid && sub == 0) mid_rows[atomicAdd(nmid, 1u)] = r;
    double acc = mid ? sr_identity(sr) : row_part(sr, s + sub, e, L, ind, val, x);
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) acc = sr_add(sr, acc, __shfl_xor_sync(kFull, acc, o));
    if (sub == 0 && r < m && !mid) y[r] = sr_out(sr, acc);
  }
}

// One warp per row, over every row (list == nullptr) or the listed ones;
// rows longer than kLongRow are listed for the hub chunks (spmv_long_plan,
// spmv_long_chunks, spmv_long_finish).
__global__ void spmv_warp_rows(int sr, int m, const int *__restrict__ ptr,
                               const int *__restrict__ ind, const float *__restrict__ val,
                               const float *__restrict__ x, float *y, unsigned *nlong,
                               int *long_rows, const unsigned *nlist, const int *list) {
  const int lane = lane_id();
  const int n = list ? (int)*nlist : m;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
       i += (gridDim.x * blockDim.x) >> 5) {
    const int r = list ? list[i] : i;
    const int s = __ldg(ptr + r), e = __ldg(ptr + r + 1);
    if (e - s > kLongRow) {
      if (lane == 0) long_rows[atomicAdd(nlong, 1u)] = r;
      continue;
    }
    double acc = row_part(sr, s + lane, e, 32, ind, val, x);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = sr_add(sr, acc, __shfl_xor_sync(kFull, acc, o));
    if (lane == 0) y[r] = sr_out(sr, acc);
  }
}

// Rows longer than kLongRow (hubs) in chunks of kLongChunk entries spread
// over all blocks.  spmv_long_plan (one block) numbers the listed rows'
// chunks in list order (first_chunk, an exclusive scan; the total after the
// last row); chunk g goes to block g mod gridDim.x, which finds its row by
// binary search and reduces it in a fixed order into partial[g];
// spmv_long_finish adds each row's partials in chunk order, so the result
// does not depend on scheduling.
constexpr int kLongChunk = 8192;

__global__ void __launch_bounds__(1024)
spmv_long_plan(const int *__restrict__ ptr, const unsigned *nlong, const int *long_rows,
               unsigned *first_chunk) {
  __shared__ unsigned sw[33];
  const unsigned n = *nlong;
  unsigned carry = 0;
  for (unsigned b = 0; b < n; b += blockDim.x) {
    const unsigned i = b + threadIdx.x;
    unsigned nc = 0;
    if (i < n) {
      const int r = long_rows[i];
      nc = (unsigned)((__ldg(ptr + r + 1) - __ldg(ptr + r) + kLongChunk - 1) / kLongChunk);
    }
    const unsigned lane = lane_id(), w = warp_in_block(), nw = blockDim.x >> 5;
    const unsigned incl = warp_incl_scan(nc);
    if (lane == 31) sw[w] = incl;
    __syncthreads();
    if (w == 0) {
      const unsigned v = lane < nw ? sw[lane] : 0u;
      const unsigned vi = warp_incl_scan(v);
      if (lane < nw) sw[lane] = vi - v;
      if (lane == nw - 1) sw[32] = vi;
    }
    __syncthreads();
    if (i < n) first_chunk[i] = carry + sw[w] + incl - nc;
    carry += sw[32];
    __syncthreads();
  }
  if (threadIdx.x == 0) first_chunk[n] = carry;
}

__global__ void __launch_bounds__(kLongThreads)
spmv_long_chunks(int sr, const int *__restrict__ ptr, const int *__restrict__ ind,
                 const float *__restrict__ val, const float *__restrict__ x,
                 const unsigned *nlong, const int *long_rows, const unsigned *first_chunk,
                 double *partial) {
  __shared__ double part[kLongThreads / 32];
  const int lane = lane_id(), w = warp_in_block();
  const unsigned n = *nlong;
  const unsigned total = n ? first_chunk[n] : 0u;
  for (unsigned g = blockIdx.x; g < total; g += gridDim.x) {
    unsigned lo = 0, hi = n - 1;
    while (lo < hi) {
      const unsigned mid = (lo + hi + 1) >> 1;
      if (first_chunk[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const int r = long_rows[lo];
    const int s = __ldg(ptr + r), e = __ldg(ptr + r + 1);
    const int k0 = s + (int)(g - first_chunk[lo]) * kLongChunk, k1 = min(e, k0 + kLongChunk);
    double acc = row_part(sr, k0 + (int)threadIdx.x, k1, kLongThreads, ind, val, x);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = sr_add(sr, acc, __shfl_xor_sync(kFull, acc, o));
    if (lane == 0) part[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = part[0];
      for (int j = 1; j < kLongThreads / 32; ++j) t = sr_add(sr, t, part[j]);
      partial[g] = t;
    }
    __syncthreads();
  }
}

__global__ void spmv_long_finish(int sr, const unsigned *nlong, const int *long_rows,
                                 const double *partial, const unsigned *first_chunk, float *y) {
  const unsigned n = *nlong;
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned c0 = first_chunk[i], c1 = first_chunk[i + 1];
    double t = partial[c0];
    for (unsigned c = c0 + 1; c < c1; ++c) t = sr_add(sr, t, partial[c]);
    y[long_rows[i]] = sr_out(sr, t);
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
  auto *mid = (int *)workspace(ctx, kSlotMisc1, sizeof(int) * ((size_t)nnz / kMidRow + 1));
  // chunks of the long rows: at most nnz / kLongChunk full ones plus one
  // partial per row; each row's first chunk number
  const size_t max_long = (size_t)nnz / kLongRow + 1;
  auto *partial = (double *)workspace(ctx, kSlotMisc2,
                                      sizeof(double) * ((size_t)nnz / kLongChunk + max_long + 1));
  auto *first = (unsigned *)workspace(ctx, kSlotMisc3, sizeof(unsigned) * (max_long + 1));
  if (!sm || !rows || !mid || !partial || !first) return APSPIE_ERR_OOM;
  cudaStream_t st = ctx->stream;
  cudaMemsetAsync(sm, 0, sizeof(SpmvSmall), st);
  // lanes per short row from the mean row length
  const double mean = (double)nnz / m;
  const int L = mean <= 6 ? 4 : (mean <= 20 ? 8 : (mean <= 48 ? 16 : 32));
  const long long warps = std::min((long long)m, (long long)ctx->num_sms * 64);
  const unsigned blocks = (unsigned)((warps * 32 + 255) / 256);
  int launches = 2;
  if (L == 32) {
    spmv_warp_rows<<<blocks, 256, 0, st>>>(semiring, m, d_ptr, d_ind, d_val, d_x, d_y, &sm->nlong,
                                           rows, nullptr, nullptr);
  } else {
    if (L == 4)
      spmv_group_rows<4><<<blocks, 256, 0, st>>>(semiring, m, d_ptr, d_ind, d_val, d_x, d_y,
                                                 &sm->nmid, mid);
    else if (L == 8)
      spmv_group_rows<8><<<blocks, 256, 0, st>>>(semiring, m, d_ptr, d_ind, d_val, d_x, d_y,
                                                 &sm->nmid, mid);
    else
      spmv_group_rows<16><<<blocks, 256, 0, st>>>(semiring, m, d_ptr, d_ind, d_val, d_x, d_y,
                                                  &sm->nmid, mid);
    spmv_warp_rows<<<ctx->num_sms * 8, 256, 0, st>>>(semiring, m, d_ptr, d_ind, d_val, d_x, d_y,
                                                    &sm->nlong, rows, &sm->nmid, mid);
    ++launches;
  }
  spmv_long_plan<<<1, 1024, 0, st>>>(d_ptr, &sm->nlong, rows, first);
  spmv_long_chunks<<<ctx->num_sms * 2, kLongThreads, 0, st>>>(
      semiring, d_ptr, d_ind, d_val, d_x, &sm->nlong, rows, first, partial);
  spmv_long_finish<<<4, 256, 0, st>>>(semiring, &sm->nlong, rows, partial, first, d_y);
  return check_launch(ctx, "apspie_spmv", launches + 2);
}
