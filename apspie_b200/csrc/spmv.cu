// spmv.cu -- dense SpMV y = A (x) x over every row of a CSR matrix, under the
// four semirings of the library: the fully dense end of the push/pull
// continuum, where every vertex is in the frontier.
//
// Replaces the reference's dense SpMV calls: mgpu::SpmvCsrBinary behind
// spmv() (src/bfs.cuh:12-14) and cusparseScsrmv behind cuspmv()
// (src/tc.cuh:18-59).  Merge-path partition (Merrill & Garland, "Merge-based
// parallel sparse matrix-vector multiplication", SC'16): the row ends
// (ptr[1..m]) and the nonzeros form one merged list of m + nnz items, cut
// into tiles of kMpTile items, so a tile's work is fixed whatever the row
// lengths (hubs, empty rows).  A block stages its tile's terms and row
// offsets in shared memory (coalesced loads of ind / val, gathers of x),
// then reduces each row's segment: short segments a thread each, long ones
// a warp each.  Rows that end in the tile are written; a row that runs on
// past the tile leaves its partial (carry) and the tile where it ends its
// head partial, which spmv_merge_fixup adds in tile order.  Every sum is
// taken in a fixed order, so the result does not depend on scheduling.
// PLUS_TIMES accumulates in double and rounds once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <type_traits>

#include "common.cuh"
#include "context.h"

namespace apspie {
namespace {

constexpr int kSr_PlusTimes = 0, kSr_MinPlus = 1, kSr_MaxTimes = 2, kSr_OrAnd = 3;
constexpr int kMpThreads = 256;
constexpr int kMpItems = 8;                     // merged items per thread
constexpr int kMpTile = kMpThreads * kMpItems;  // row ends + nonzeros per tile
constexpr int kMpWarpSeg = 32;                  // longer segments are reduced by a warp

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

// coordinates of the ntiles + 1 tile boundaries, a warp each: a 32-way
// search (each round probes 32 evenly spaced rows and keeps the interval
// between the last probe that precedes the diagonal and the first that
// does not), then one round over the last <= 32 candidates
__global__ void spmv_merge_plan(int m, int nnz, int ntiles, const int *__restrict__ ptr,
                                int2 *coord) {
  const long long total = (long long)m + nnz;
  const int lane = lane_id();
  for (int b = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); b <= ntiles;
       b += (int)((gridDim.x * blockDim.x) >> 5)) {
    const long long d = min((long long)b * kMpTile, total);
    // C(i): row end i precedes the diagonal's nonzero, true below the answer
    auto before = [&](long long i) { return (long long)__ldg(ptr + i + 1) <= d - i - 1; };
    long long lo = max(0ll, d - nnz), hi = min(d, (long long)m);
    while (hi - lo > 32) {
      const long long step = (hi - lo + 31) / 32;
      const long long p = lo + lane * step;
      const int k = __popc(__ballot_sync(kFull, p < hi && before(p)));
      const long long nlo = k == 0 ? lo : lo + (k - 1) * step + 1;
      hi = k < 32 ? min(hi, lo + k * step) : hi;
      lo = nlo;
    }
    const int k = __popc(__ballot_sync(kFull, lo + lane < hi && before(lo + lane)));
    if (lane == 0) coord[b] = make_int2((int)(lo + k), (int)(d - lo - k));
  }
}

// One tile per block.  Tile b holds the row ends [i0, i1) and the nonzeros
// [j0, j1); it touches rows i0 .. min(i1, m - 1).  Row i1 (when < m) is
// open at the tile's end: its partial goes to carry_val[b].  Row i0, when
// it has nonzeros before j0 and ends in this tile, goes to head_val[b].
template <int SR>
__global__ void __launch_bounds__(kMpThreads)
spmv_merge_tiles(int m, const int *__restrict__ ptr, const int *__restrict__ ind,
                 const float *__restrict__ val, const float *__restrict__ x, float *y,
                 const int2 *__restrict__ coord, int *carry_row, double *carry_val,
                 int *head_row, double *head_val) {
  __shared__ double s_term[kMpTile];
  __shared__ int s_ptr[kMpTile + 2];
  __shared__ int s_long[kMpTile / (kMpWarpSeg + 1) + 1];
  __shared__ unsigned s_nlong;
  constexpr int sr = SR;  // the semiring, fixed per instantiation
  const int b = blockIdx.x, t = threadIdx.x;
  const int2 c0 = coord[b], c1 = coord[b + 1];
  const int i0 = c0.x, j0 = c0.y, i1 = c1.x, j1 = c1.y;
  const int nr = min(i1, m - 1) - i0 + 1;  // rows touched (i0 < m in every tile)
  const int nz = j1 - j0;
  if (t == 0) s_nlong = 0;
  for (int q = t; q <= nr; q += kMpThreads) s_ptr[q] = __ldg(ptr + i0 + q);
  // the tile's terms: all index / value loads, then all x loads, in flight
  {
    int c[kMpItems];
    float a[kMpItems], xv[kMpItems];
#pragma unroll
    for (int u = 0; u < kMpItems; ++u) {
      const int q = t + u * kMpThreads;
      c[u] = q < nz ? __ldg(ind + j0 + q) : 0;
      a[u] = q < nz ? (val ? __ldg(val + j0 + q) : 1.0f) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < kMpItems; ++u) xv[u] = t + u * kMpThreads < nz ? __ldg(x + c[u]) : 0.0f;
#pragma unroll
    for (int u = 0; u < kMpItems; ++u) {
      const int q = t + u * kMpThreads;
      if (q < nz) s_term[q] = sr_term(sr, a[u], xv[u]);
    }
  }
  if (t == 0) {
    carry_row[b] = i1 < m ? i1 : -1;
    head_row[b] = (i0 < i1 && s_ptr[0] < j0) ? i0 : -1;
  }
  __syncthreads();
  auto emit = [&](int q, double acc) {
    const int i = i0 + q;
    if (i == i1) carry_val[b] = acc;                     // open at the tile's end
    else if (q == 0 && s_ptr[0] < j0) head_val[b] = acc;  // began in an earlier tile
    else y[i] = sr_out(sr, acc);
  };
  // short segments a thread each; long ones listed for the warps
  for (int q = t; q < nr; q += kMpThreads) {
    const int s = max(s_ptr[q], j0) - j0, e = min(s_ptr[q + 1], j1) - j0;
    if (e - s > kMpWarpSeg) {
      s_long[atomicAdd(&s_nlong, 1u)] = q;
      continue;
    }
    // four partial sums, combined in a fixed order
    double a0 = sr_identity(sr), a1 = a0, a2 = a0, a3 = a0;
    int k = s;
    for (; k + 3 < e; k += 4) {
      a0 = sr_add(sr, a0, s_term[k]);
      a1 = sr_add(sr, a1, s_term[k + 1]);
      a2 = sr_add(sr, a2, s_term[k + 2]);
      a3 = sr_add(sr, a3, s_term[k + 3]);
    }
    for (; k < e; ++k) a0 = sr_add(sr, a0, s_term[k]);
    emit(q, sr_add(sr, sr_add(sr, a0, a1), sr_add(sr, a2, a3)));
  }
  __syncthreads();
  const int lane = lane_id(), w = warp_in_block();
  for (unsigned l = w; l < s_nlong; l += kMpThreads / 32) {
    const int q = s_long[l];
    const int s = max(s_ptr[q], j0) - j0, e = min(s_ptr[q + 1], j1) - j0;
    double acc = sr_identity(sr);
    for (int k = s + lane; k < e; k += 32) acc = sr_add(sr, acc, s_term[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc = sr_add(sr, acc, __shfl_xor_sync(kFull, acc, o));
    if (lane == 0) emit(q, acc);
  }
}

// Rows that span tiles: the tile where row r ends (head_row[b] == r) adds,
// in tile order, the carries of the tiles before it that were open on r,
// then its own head partial.
template <int SR>
__global__ void spmv_merge_fixup(int ntiles, const int *__restrict__ carry_row,
                                 const double *__restrict__ carry_val,
                                 const int *__restrict__ head_row,
                                 const double *__restrict__ head_val, float *y) {
  constexpr int sr = SR;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < ntiles; b += gridDim.x * blockDim.x) {
    const int r = head_row[b];
    if (r < 0) continue;
    int first = b - 1;  // carry_row[b - 1] == r: row r is i0 of tile b
    while (first > 0 && carry_row[first - 1] == r) --first;
    double acc = carry_val[first];
    for (int u = first + 1; u < b; ++u) acc = sr_add(sr, acc, carry_val[u]);
    y[r] = sr_out(sr, sr_add(sr, acc, head_val[b]));
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
  const long long items = (long long)m + nnz;
  const int ntiles = (int)((items + kMpTile - 1) / kMpTile);
  auto *coord = (int2 *)workspace(ctx, kSlotMisc0, sizeof(int2) * ((size_t)ntiles + 1));
  auto *rows = (int *)workspace(ctx, kSlotMisc1, sizeof(int) * 2 * (size_t)ntiles);
  auto *vals = (double *)workspace(ctx, kSlotMisc2, sizeof(double) * 2 * (size_t)ntiles);
  if (!coord || !rows || !vals) return APSPIE_ERR_OOM;
  cudaStream_t st = ctx->stream;
  const int pgrid = (int)std::min<long long>((32ll * (ntiles + 1) + 255) / 256, ctx->num_sms * 16ll);
  spmv_merge_plan<<<pgrid, 256, 0, st>>>(m, (int)nnz, ntiles, d_ptr, coord);
  const unsigned fgrid = (unsigned)((ntiles + 255) / 256);
  auto launch = [&](auto sr_tag) {
    constexpr int SR = decltype(sr_tag)::value;
    spmv_merge_tiles<SR><<<ntiles, kMpThreads, 0, st>>>(m, d_ptr, d_ind, d_val, d_x, d_y, coord,
                                                        rows, vals, rows + ntiles, vals + ntiles);
    spmv_merge_fixup<SR><<<fgrid, 256, 0, st>>>(ntiles, rows, vals, rows + ntiles, vals + ntiles,
                                                d_y);
  };
  switch (semiring) {
    case kSr_MinPlus: launch(std::integral_constant<int, kSr_MinPlus>{}); break;
    case kSr_MaxTimes: launch(std::integral_constant<int, kSr_MaxTimes>{}); break;
    case kSr_OrAnd: launch(std::integral_constant<int, kSr_OrAnd>{}); break;
    default: launch(std::integral_constant<int, kSr_PlusTimes>{}); break;
  }
  return check_launch(ctx, "apspie_spmv", 3);
}
