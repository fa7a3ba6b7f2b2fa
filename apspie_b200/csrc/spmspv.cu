// spmspv.cu -- generic semiring SpMSpV: sparse x times A (column lists),
// sparse sorted y, plus the dense-in/dense-out form.
//
// Replaces both mXv<T>() overloads (src/mXv.cuh:111-247 dense, :250-389
// sparse) and the min-plus spmspvSssp (src/spmspvSssp.cuh:92-291).  The
// reference gathers column segments with four IntervalGathers and an
// IntervalExpand, multiplies, cub-radix-sorts all (row, value) pairs on 32
// key bits and reduces by key.  Here:
//   * sort path (sparse output): one expand kernel writes (row, x (x) a)
//     pairs at their scanned offsets (warp scan-based gather, big columns in a
//     block-strided second kernel), the pairs are radix-sorted on only
//     ceil(log2 m) key bits, and a segmented reduce emits sorted y;
//   * bitmap path (dense frontier): products are combined with atomics into a
//     dense accumulator and a touched bitmap, and y is compacted from the
//     bitmap in index order -- no sort at all.
// The path is chosen from the expanded size E against m (threshold settable,
// picked by the autotuner).  Both give y sorted by row with one entry per
// touched row; PLUS_TIMES accumulates in double and rounds once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "common.cuh"
#include "context.h"
#include "frontier.cuh"
#include "primitives.cuh"

namespace apspie {
namespace {

constexpr int kPlusTimes = 0, kMinPlus = 1, kMaxTimes = 2, kOrAnd = 3;

struct SpmspvSmall {  // device-side scalars of one call
  long long total;    // expanded size E
  unsigned nbig;      // columns of more than kBigDeg edges (a warp each)
  int ynnz;           // nnz(y)
  unsigned cnt;       // frontier size of the dense form
  unsigned nhub;      // chunks of the columns of more than kHubDeg edges
};

// Columns longer than this are cut into kHubChunk-edge chunks, a warp each;
// between kBigDeg and this a warp takes one column
constexpr int kHubDeg = 1024;
constexpr int kHubChunk = 2048;
constexpr int kExpandThreads = 256;

__device__ __forceinline__ float sr_term(int sr, float a, float x) {
  switch (sr) {
    case kMinPlus: return __fadd_rn(a, x);
    case kOrAnd: return 1.0f;
    default: return __fmul_rn(a, x);  // PLUS_TIMES, MAX_TIMES
  }
}

// ---- expansion into (row, term) pairs at scanned offsets ----
__global__ void frontier_degrees(int xnnz, const int *__restrict__ xind, const int *__restrict__ ptr,
                                 long long *deg) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < xnnz; j += gridDim.x * blockDim.x) {
    int c = xind[j];
    deg[j] = (long long)(__ldg(ptr + c + 1) - __ldg(ptr + c));
  }
}

__global__ void __launch_bounds__(kExpandThreads)
expand_pairs(int sr, int xnnz, const int *__restrict__ xind, const float *__restrict__ xval,
             const int *__restrict__ ptr, const int *__restrict__ ind,
             const float *__restrict__ val, const long long *__restrict__ offs, int *keys,
             float *vals, int *big, unsigned *nbig, int2 *hub, unsigned *nhub) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int base = gwarp * 32; base < xnnz; base += nwarps * 32) {
    int j = base + lane;
    int s = 0, d = 0;
    float xv = 0.f;
    bool isbig = false;
    if (j < xnnz) {
      int c = xind[j];
      s = __ldg(ptr + c);
      d = __ldg(ptr + c + 1) - s;
      xv = xval ? xval[j] : 1.0f;
      if (d > kBigDeg) isbig = true;
    }
    const bool ishub = isbig && d > kHubDeg;
    const bool ismid = isbig && !ishub;
    unsigned slot = warp_append(ismid, nbig);
    if (ismid) big[slot] = j;
    if (ishub) {
      const int nc = (d + kHubChunk - 1) / kHubChunk;
      const unsigned at = atomicAdd(nhub, (unsigned)nc);
      for (int c = 0; c < nc; ++c) hub[at + c] = make_int2(j, c);
    }
    if (isbig) d = 0;
    int incl = warp_incl_scan(d);
    int excl = incl - d;
    int total = __shfl_sync(kFull, incl, 31);
    for (int e0 = 0; e0 < total; e0 += 32) {
      int e = e0 + lane;
      int owner = warp_owner(excl, e);
      int so = __shfl_sync(kFull, s, owner);
      int eo = __shfl_sync(kFull, excl, owner);
      float xo = __shfl_sync(kFull, xv, owner);
      int jo = __shfl_sync(kFull, j, owner);
      if (e < total) {
        int k = so + (e - eo);
        long long pos = offs[jo] + (e - eo);
        keys[pos] = __ldg(ind + k);
        vals[pos] = sr_term(sr, val ? __ldg(val + k) : 1.0f, xo);
      }
    }
  }
}

// The listed columns: a warp per column of the medium list, then a warp per
// hub chunk (a hub's edges spread over all SMs).
__global__ void expand_big(int sr, const int *__restrict__ xind, const float *__restrict__ xval,
                           const int *__restrict__ ptr, const int *__restrict__ ind,
                           const float *__restrict__ val, const long long *__restrict__ offs,
                           const int *big, const unsigned *nbig, const int2 *hub,
                           const unsigned *nhub, int *keys, float *vals) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const unsigned nb = *nbig;
  for (unsigned b = gwarp; b < nb; b += nwarps) {
    const int j = big[b];
    const int c = xind[j];
    const int s = __ldg(ptr + c), e = __ldg(ptr + c + 1);
    const float xv = xval ? xval[j] : 1.0f;
    const long long o = offs[j] - s;
    for (int k = s + lane; k < e; k += 32) {
      keys[o + k] = __ldg(ind + k);
      vals[o + k] = sr_term(sr, val ? __ldg(val + k) : 1.0f, xv);
    }
  }
  const unsigned nh = *nhub;
  for (unsigned b = gwarp; b < nh; b += nwarps) {
    const int2 hc = hub[b];
    const int j = hc.x;
    const int c = xind[j];
    const int s0 = __ldg(ptr + c);
    const int s = s0 + hc.y * kHubChunk, e = min(__ldg(ptr + c + 1), s + kHubChunk);
    const float xv = xval ? xval[j] : 1.0f;
    const long long o = offs[j] - s0;
    for (int k = s + lane; k < e; k += 32) {
      keys[o + k] = __ldg(ind + k);
      vals[o + k] = sr_term(sr, val ? __ldg(val + k) : 1.0f, xv);
    }
  }
}

// ---- segmented reduce of sorted pairs ----
__global__ void head_flags(const int *keys, long long n, unsigned *flags) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void reduce_segments(int sr, const int *keys, const float *vals, long long n,
                                const unsigned *segid, int *yind, float *yval, int ycap) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int k = keys[i];
    if (i > 0 && keys[i - 1] == k) continue;
    double accd = 0.0;
    float accf = vals[i];
    long long j = i;
    for (; j < n && keys[j] == k; ++j) {
      float t = vals[j];
      switch (sr) {
        case kPlusTimes: accd += (double)t; break;
        case kMinPlus: accf = fminf(accf, t); break;
        case kMaxTimes: accf = fmaxf(accf, t); break;
        default: accf = 1.0f; break;
      }
    }
    // at most m distinct rows from a sorted run; more only from a sort that
    // gave up (reported by the caller), whose extra segments are dropped
    unsigned s = segid[i];
    if (s >= (unsigned)ycap) continue;
    yind[s] = k;
    yval[s] = sr == kPlusTimes ? (float)accd : accf;
  }
}

// ---- bitmap path ----
__global__ void acc_init(int sr, int m, double *acc, unsigned *bits) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    double idv = 0.0;
    if (sr == kMinPlus) idv = (double)FLT_MAX * 2.0;  // above any float
    if (sr == kMaxTimes) idv = -(double)FLT_MAX * 2.0;
    acc[i] = idv;
    if ((i & 31) == 0) bits[i >> 5] = 0u;
  }
}

__device__ __forceinline__ void atomic_min_double(double *p, double v) {
  unsigned long long *a = (unsigned long long *)p;
  unsigned long long old = *a;
  while (__longlong_as_double(old) > v) {
    unsigned long long prev = atomicCAS(a, old, __double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}
__device__ __forceinline__ void atomic_max_double(double *p, double v) {
  unsigned long long *a = (unsigned long long *)p;
  unsigned long long old = *a;
  while (__longlong_as_double(old) < v) {
    unsigned long long prev = atomicCAS(a, old, __double_as_longlong(v));
    if (prev == old) break;
    old = prev;
  }
}

// Bitmap path expansion.  32 consecutive frontier entries per warp: their
// edges are dealt over the lanes by an inclusive warp scan of the degrees
// (coalesced over each column, no lane idles on a short column).  Columns
// of more than kBigDeg edges are listed instead: up to kHubDeg edges a warp
// takes one in expand_accumulate_big, longer ones (hubs) are cut into
// kHubChunk-edge chunks that warps take one by one.  Each product is folded into acc[row] with the
// semiring's atomic and marks the row's bit.
__device__ __forceinline__ void accumulate_one(int sr, int r, float t, double *acc,
                                               unsigned *bits) {
  switch (sr) {
    case kPlusTimes: atomicAdd(acc + r, (double)t); break;
    case kMinPlus: atomic_min_double(acc + r, (double)t); break;
    case kMaxTimes: atomic_max_double(acc + r, (double)t); break;
    default: break;
  }
  const unsigned bit = 1u << (r & 31);
  if (!(__ldcg(bits + (r >> 5)) & bit)) atomicOr(bits + (r >> 5), bit);
}

__global__ void __launch_bounds__(kExpandThreads)
expand_accumulate(int sr, int xnnz, const int *__restrict__ xind, const float *__restrict__ xval,
                  const int *__restrict__ ptr, const int *__restrict__ ind,
                  const float *__restrict__ val, double *acc, unsigned *bits, int *big,
                  unsigned *nbig, int2 *hub, unsigned *nhub) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int base = gwarp * 32; base < xnnz; base += nwarps * 32) {
    const int j = base + lane;
    int s = 0, d = 0;
    float xv = 0.f;
    bool isbig = false;
    if (j < xnnz) {
      const int c = xind[j];
      s = __ldg(ptr + c);
      d = __ldg(ptr + c + 1) - s;
      xv = xval ? xval[j] : 1.0f;
      if (d > kBigDeg) isbig = true;
    }
    const bool ishub = isbig && d > kHubDeg;
    const bool ismid = isbig && !ishub;
    unsigned slot = warp_append(ismid, nbig);
    if (ismid) big[slot] = j;
    if (ishub) {
      const int nc = (d + kHubChunk - 1) / kHubChunk;
      const unsigned at = atomicAdd(nhub, (unsigned)nc);
      for (int c = 0; c < nc; ++c) hub[at + c] = make_int2(j, c);
    }
    if (isbig) d = 0;
    const int incl = warp_incl_scan(d);
    const int excl = incl - d;
    const int total = __shfl_sync(kFull, incl, 31);
    for (int e0 = 0; e0 < total; e0 += 32) {
      const int e = e0 + lane;
      const int owner = warp_owner(excl, e);
      const int so = __shfl_sync(kFull, s, owner);
      const int eo = __shfl_sync(kFull, excl, owner);
      const float xo = __shfl_sync(kFull, xv, owner);
      if (e < total) {
        const int k = so + (e - eo);
        accumulate_one(sr, __ldg(ind + k), sr_term(sr, val ? __ldg(val + k) : 1.0f, xo), acc,
                       bits);
      }
    }
  }
}

// The listed long columns: a warp per column of the medium list, then a warp
// per hub chunk (a hub's edges spread over all SMs).
__global__ void __launch_bounds__(kExpandThreads)
expand_accumulate_big(int sr, const int *__restrict__ xind, const float *__restrict__ xval,
                      const int *__restrict__ ptr, const int *__restrict__ ind,
                      const float *__restrict__ val, const int *big, const unsigned *nbig,
                      const int2 *hub, const unsigned *nhub, double *acc, unsigned *bits) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  const unsigned nb = *nbig;
  for (unsigned b = gwarp; b < nb; b += nwarps) {
    const int j = big[b];
    const int c = xind[j];
    const int s = __ldg(ptr + c), e = __ldg(ptr + c + 1);
    const float xv = xval ? xval[j] : 1.0f;
    // four index / value loads in flight per lane before their atomics
    int k = s + lane;
    for (; k + 96 < e; k += 128) {
      int r[4];
      float a[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        r[q] = __ldg(ind + k + 32 * q);
        a[q] = val ? __ldg(val + k + 32 * q) : 1.0f;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) accumulate_one(sr, r[q], sr_term(sr, a[q], xv), acc, bits);
    }
    for (; k < e; k += 32)
      accumulate_one(sr, __ldg(ind + k), sr_term(sr, val ? __ldg(val + k) : 1.0f, xv), acc,
                     bits);
  }
  const unsigned nh = *nhub;
  for (unsigned b = gwarp; b < nh; b += nwarps) {
    const int2 hc = hub[b];
    const int j = hc.x;
    const int c = xind[j];
    const int s = __ldg(ptr + c) + hc.y * kHubChunk;
    const int e = min(__ldg(ptr + c + 1), s + kHubChunk);
    const float xv = xval ? xval[j] : 1.0f;
    int k = s + lane;
    for (; k + 96 < e; k += 128) {
      int r[4];
      float a[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        r[q] = __ldg(ind + k + 32 * q);
        a[q] = val ? __ldg(val + k + 32 * q) : 1.0f;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) accumulate_one(sr, r[q], sr_term(sr, a[q], xv), acc, bits);
    }
    for (; k < e; k += 32)
      accumulate_one(sr, __ldg(ind + k), sr_term(sr, val ? __ldg(val + k) : 1.0f, xv), acc,
                     bits);
  }
}

__global__ void bitmap_counts(const unsigned *bits, int words, unsigned *cnt) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x)
    cnt[w] = __popc(bits[w]);
}

__global__ void bitmap_emit(int sr, const unsigned *bits, int words, const unsigned *offs,
                            const double *acc, int *yind, float *yval) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    unsigned b = bits[w];
    unsigned o = offs[w];
    while (b) {
      int t = __ffs(b) - 1;
      b &= b - 1;
      int r = w * 32 + t;
      yind[o] = r;
      yval[o] = sr == kOrAnd ? 1.0f : (float)acc[r];
      ++o;
    }
  }
}

// ---- dense in / dense out helpers (mXv dense form) ----
__global__ void dense_frontier_flags(int sr, int m, const float *x, unsigned *flags) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    float v = x[i];
    bool in;
    if (sr == kMinPlus)
      in = v > -1.0f && v < 1e38f;  // finite distance (src/spmspvSssp.cuh:31-36)
    else if (sr == kPlusTimes)
      in = v > 0.5f;  // bitify (src/mXv.cuh:50-55)
    else
      in = v != 0.0f;
    flags[i] = in ? 1u : 0u;
  }
}

__global__ void dense_compact(int m, const float *x, const unsigned *flags, const unsigned *offs,
                              int *xind, float *xval) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    if (flags[i]) {
      xind[offs[i]] = i;
      xval[offs[i]] = x[i];
    }
}

__global__ void dense_fill(int m, float v, float *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) y[i] = v;
}

__global__ void dense_scatter(const int *nnz, const int *yind, const float *yval, float *y) {
  int n = *nnz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[yind[i]] = yval[i];
}

int grid_for(apspie_context *ctx, long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  return (int)std::max(1ll, std::min(g, (long long)ctx->num_sms * 16));
}

// Core sparse SpMSpV.  On return *d_ynnz (device) holds nnz(y); *h_total
// the expanded size E (host, after a sync).
int spmspv_core(apspie_context *ctx, int sr, int m, const int *ptr, const int *ind,
                const float *val, int xnnz, const int *xind, const float *xval, int *yind,
                float *yval, int *d_ynnz, long long *h_total) {
  cudaStream_t st = ctx->stream;
  long long *offs = (long long *)workspace(ctx, kSlotMisc0, sizeof(long long) * (size_t)(xnnz + 1));
  auto *sm = (SpmspvSmall *)workspace(ctx, kSlotSmall, sizeof(SpmspvSmall));
  if (!offs || !sm) return APSPIE_ERR_OOM;
  long long *d_tot = &sm->total;
  long long E = 0;
  if (xnnz > 0) {
    frontier_degrees<<<grid_for(ctx, xnnz, 256), 256, 0, st>>>(xnnz, xind, ptr, offs);
    int rc = check_launch(ctx, "frontier_degrees");
    if (rc) return rc;
    rc = device_exclusive_scan<long long>(ctx, offs, offs, xnnz, d_tot);
    if (rc) return rc;
    long long *h = (long long *)pinned(ctx, sizeof(long long));
    if (!h) return APSPIE_ERR_OOM;
    rc = check_cuda(ctx, cudaMemcpyAsync(h, d_tot, sizeof(long long), cudaMemcpyDeviceToHost, st),
                    "spmspv total");
    if (rc) return rc;
    rc = check_cuda(ctx, cudaStreamSynchronize(st), "spmspv total");
    if (rc) return rc;
    E = *h;
  }
  if (h_total) *h_total = E;
  if (E == 0) {
    return check_cuda(ctx, cudaMemsetAsync(d_ynnz, 0, sizeof(int), st), "spmspv empty");
  }
  if (E >= (long long)INT32_MAX)
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "spmspv: %lld expanded pairs", E);
  bool bitmap = (double)E * ctx->spmspv_sort_factor > (double)m;
  if (bitmap) {
    int words = (m + 31) / 32;
    double *acc = (double *)workspace(ctx, kSlotDense, sizeof(double) * (size_t)m);
    unsigned *bits = (unsigned *)workspace(ctx, kSlotBitmap, sizeof(unsigned) * (size_t)(2 * words + 2));
    if (!acc || !bits) return APSPIE_ERR_OOM;
    unsigned *woffs = bits + words + 1;
    const size_t nbig_cap = ((size_t)xnnz + 2) & ~size_t(1);  // keeps the chunk list 8-aligned
    int *big = (int *)workspace(ctx, kSlotMisc2,
                                sizeof(int) * nbig_cap +
                                    sizeof(int2) * ((size_t)E / kHubChunk + (size_t)xnnz + 1));
    if (!big) return APSPIE_ERR_OOM;
    int2 *hub = (int2 *)(big + nbig_cap);
    int rc = check_cuda(ctx, cudaMemsetAsync(&sm->nbig, 0, sizeof(unsigned), st), "spmspv nbig");
    if (rc) return rc;
    rc = check_cuda(ctx, cudaMemsetAsync(&sm->nhub, 0, sizeof(unsigned), st), "spmspv nhub");
    if (rc) return rc;
    acc_init<<<grid_for(ctx, m, 256), 256, 0, st>>>(sr, m, acc, bits);
    expand_accumulate<<<grid_for(ctx, (long long)xnnz * 32, kExpandThreads), kExpandThreads, 0,
                        st>>>(sr, xnnz, xind, xval, ptr, ind, val, acc, bits, big, &sm->nbig,
                              hub, &sm->nhub);
    expand_accumulate_big<<<ctx->num_sms * 4, kExpandThreads, 0, st>>>(
        sr, xind, xval, ptr, ind, val, big, &sm->nbig, hub, &sm->nhub, acc, bits);
    bitmap_counts<<<grid_for(ctx, words, 256), 256, 0, st>>>(bits, words, woffs);
    rc = check_launch(ctx, "spmspv bitmap", 4);
    if (rc) return rc;
    rc = device_exclusive_scan<unsigned>(ctx, woffs, woffs, words, (unsigned *)d_ynnz);
    if (rc) return rc;
    bitmap_emit<<<grid_for(ctx, words, 256), 256, 0, st>>>(sr, bits, words, woffs, acc, yind, yval);
    return check_launch(ctx, "bitmap_emit");
  }
  // sort path
  int *ka = (int *)workspace(ctx, kSlotSortKeysA, sizeof(int) * (size_t)E);
  int *kb = (int *)workspace(ctx, kSlotSortKeysB, sizeof(int) * (size_t)E);
  float *va = (float *)workspace(ctx, kSlotSortValsA, sizeof(float) * (size_t)E);
  float *vb = (float *)workspace(ctx, kSlotSortValsB, sizeof(float) * (size_t)E);
  const size_t nbig_cap = ((size_t)xnnz + 2) & ~size_t(1);  // keeps the chunk list 8-aligned
  int *big = (int *)workspace(ctx, kSlotMisc2,
                              sizeof(int) * nbig_cap +
                                  sizeof(int2) * ((size_t)E / kHubChunk + (size_t)xnnz + 1));
  unsigned *nbig = &sm->nbig;
  if (!ka || !kb || !va || !vb || !big) return APSPIE_ERR_OOM;
  int2 *hub = (int2 *)(big + nbig_cap);
  int rc = check_cuda(ctx, cudaMemsetAsync(nbig, 0, sizeof(unsigned), st), "spmspv nbig");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaMemsetAsync(&sm->nhub, 0, sizeof(unsigned), st), "spmspv nhub");
  if (rc) return rc;
  expand_pairs<<<grid_for(ctx, (long long)xnnz * 32, kExpandThreads), kExpandThreads, 0, st>>>(
      sr, xnnz, xind, xval, ptr, ind, val, offs, ka, va, big, nbig, hub, &sm->nhub);
  expand_big<<<ctx->num_sms * 4, kExpandThreads, 0, st>>>(sr, xind, xval, ptr, ind, val, offs,
                                                          big, nbig, hub, &sm->nhub, ka, va);
  rc = check_launch(ctx, "expand_pairs", 2);
  if (rc) return rc;
  bool in_b = false;
  rc = device_radix_sort<int, float>(ctx, ka, va, kb, vb, E, bits_for(m), &in_b);
  if (rc) return rc;
  int *ks = in_b ? kb : ka;
  float *vs = in_b ? vb : va;
  unsigned *flags = (unsigned *)workspace(ctx, kSlotMisc3, sizeof(unsigned) * (size_t)E);
  if (!flags) return APSPIE_ERR_OOM;
  head_flags<<<grid_for(ctx, E, 256), 256, 0, st>>>(ks, E, flags);
  rc = check_launch(ctx, "head_flags");
  if (rc) return rc;
  rc = device_exclusive_scan<unsigned>(ctx, flags, flags, E, (unsigned *)d_ynnz);
  if (rc) return rc;
  reduce_segments<<<grid_for(ctx, E, 256), 256, 0, st>>>(sr, ks, vs, E, flags, yind, yval, m);
  return check_launch(ctx, "reduce_segments");
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_spmspv(apspie_ctx ctx, int semiring, int m, int64_t nnz, const int *d_ptr,
                  const int *d_ind, const float *d_val, int xnnz, const int *d_xind,
                  const float *d_xval, int *d_yind, float *d_yval, int *h_ynnz,
                  int64_t *h_expanded) {
  APSPIE_CHECK_CTX(ctx);
  if (semiring < 0 || semiring > 3 || m <= 0 || nnz < 0 || xnnz < 0 || xnnz > m || !d_ptr ||
      (nnz > 0 && !d_ind) || (xnnz > 0 && !d_xind) || !d_yind || !d_yval || !h_ynnz)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_spmspv: bad arguments");
  auto *sm = (SpmspvSmall *)workspace(ctx, kSlotSmall, sizeof(SpmspvSmall));
  if (!sm) return APSPIE_ERR_OOM;
  int *d_ynnz = &sm->ynnz;
  long long E = 0;
  int rc = spmspv_core(ctx, semiring, m, d_ptr, d_ind, d_val, xnnz, d_xind, d_xval, d_yind, d_yval,
                       d_ynnz, &E);
  if (rc) return rc;
  int *h = (int *)pinned(ctx, sizeof(long long));
  int *sort_err = radix_sort_err(ctx);
  if (!h || !sort_err) return APSPIE_ERR_OOM;
  rc = check_cuda(ctx, cudaMemcpyAsync(h, d_ynnz, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream),
                  "apspie_spmspv");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaMemcpyAsync(h + 1, sort_err, sizeof(int), cudaMemcpyDeviceToHost,
                                       ctx->stream), "apspie_spmspv");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "apspie_spmspv");
  if (rc) return rc;
  if (h[1]) {  // the sort path's look-back gave up: the output is not sorted
    rc = check_cuda(ctx, cudaMemsetAsync(sort_err, 0, sizeof(int), ctx->stream), "apspie_spmspv");
    if (rc) return rc;
    return set_error(ctx, APSPIE_ERR_TIMEOUT, "apspie_spmspv: radix sort look-back gave up");
  }
  *h_ynnz = *h;
  if (h_expanded) *h_expanded = E;
  return APSPIE_OK;
}

int apspie_mxv_dense(apspie_ctx ctx, int semiring, int m, int64_t nnz, const int *d_ptr,
                     const int *d_ind, const float *d_val, const float *d_x, float *d_y,
                     int64_t *h_expanded) {
  APSPIE_CHECK_CTX(ctx);
  if (semiring < 0 || semiring > 3 || m <= 0 || nnz < 0 || !d_ptr || (nnz > 0 && !d_ind) ||
      !d_x || !d_y)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_mxv_dense: bad arguments");
  cudaStream_t st = ctx->stream;
  unsigned *flags = (unsigned *)workspace(ctx, kSlotMxvFlags, sizeof(unsigned) * ((size_t)m + 1));
  // frontier (xind, xval) and the sparse result share one buffer of 4m words
  int *buf = (int *)workspace(ctx, kSlotMxvBuf, sizeof(int) * 4 * ((size_t)m + 1));
  if (!flags || !buf) return APSPIE_ERR_OOM;
  int *fx = buf;
  float *fv = (float *)(buf + (m + 1));
  int *yi = buf + 2 * (m + 1);
  float *yv = (float *)(buf + 3 * (m + 1));
  auto *sm = (SpmspvSmall *)workspace(ctx, kSlotSmall, sizeof(SpmspvSmall));
  if (!sm) return APSPIE_ERR_OOM;
  unsigned *d_cnt = &sm->cnt;
  dense_frontier_flags<<<grid_for(ctx, m, 256), 256, 0, st>>>(semiring, m, d_x, flags);
  int rc = check_launch(ctx, "dense_frontier_flags");
  if (rc) return rc;
  rc = device_exclusive_scan<unsigned>(ctx, flags + 0, flags + 0, m, d_cnt);
  if (rc) return rc;
  // flags were overwritten by their scan; recompute membership in the compaction
  dense_frontier_flags<<<grid_for(ctx, m, 256), 256, 0, st>>>(semiring, m, d_x,
                                                              (unsigned *)yi);
  dense_compact<<<grid_for(ctx, m, 256), 256, 0, st>>>(m, d_x, (unsigned *)yi, flags, fx, fv);
  rc = check_launch(ctx, "dense_compact", 2);
  if (rc) return rc;
  unsigned *h = (unsigned *)pinned(ctx, sizeof(long long));
  if (!h) return APSPIE_ERR_OOM;
  cudaMemcpyAsync(h, d_cnt, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  rc = check_cuda(ctx, cudaStreamSynchronize(st), "apspie_mxv_dense");
  if (rc) return rc;
  int xnnz = (int)*h;
  // y reset to the semiring's empty value, as preprocessFlag does
  // (0 for mXv, src/mXv.cuh:45; 1.70141e38 for SSSP, src/spmspvSssp.cuh:26)
  float empty = semiring == kMinPlus ? 1.70141e+38f : 0.0f;
  int *d_ynnz = &sm->ynnz;
  long long E = 0;
  rc = spmspv_core(ctx, semiring, m, d_ptr, d_ind, d_val, xnnz, fx, fv, yi, yv, d_ynnz, &E);
  if (rc) return rc;
  dense_fill<<<grid_for(ctx, m, 256), 256, 0, st>>>(m, empty, d_y);
  dense_scatter<<<grid_for(ctx, m, 256), 256, 0, st>>>(d_ynnz, yi, yv, d_y);
  rc = check_launch(ctx, "dense_scatter", 2);
  if (rc) return rc;
  if (h_expanded) *h_expanded = E;
  return APSPIE_OK;
}

int apspie_spmspv_set_params(apspie_ctx ctx, double sort_factor) {
  if (!ctx || !(sort_factor >= 0.0)) return APSPIE_ERR_INVALID;
  ctx->spmspv_sort_factor = sort_factor;
  return APSPIE_OK;
}

}  // extern "C"
