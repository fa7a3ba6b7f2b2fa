// spgemm.cu -- row-wise (Gustavson) hash SpGEMM C = A * B with per-row hash
// tables in shared memory, rows binned by their product count.
//
// Replaces spgemm(d_matrix *C, A, B, partSize, partNum) (src/spgemm.cuh:132-
// 342, KernelInsert src/spgemmKernel.cuh:210-343): the reference tiles A and B
// into partNum x partNum DCSC blocks, intersects k-sets per tile pair on the
// host, inserts every product into a global-memory open-addressing table of
// TABLE_SIZE slots per tile (atomicCAS key (row<<16|col), atomicAdd float,
// entries DROPPED after 25 probes), then radix-sorts the whole tables and
// converts COO to CSR.  Here:
//   0. prod[i] = sum over A(i,k) of nnz(B(k,:)) (an upper bound of nnz(C(i,:)));
//   1. rows are binned: prod <= 256 -> one warp per row, table of
//      next_pow2(2*prod) slots in shared memory; prod <= 8192 -> one block per
//      row, table up to 16384 slots; larger -> one block per row with a dense
//      accumulator (bitmap + values) in global memory;
//   2. symbolic pass counts distinct columns per row (keys only), a scan gives
//      C's row offsets, C is allocated exactly;
//   3. numeric pass accumulates the products in double (so the float result is
//      the correctly rounded exact sum up to double error) and writes the row
//      into C in column order: warp rows bitonic-sort their small table; block
//      rows scatter the occupied entries into C by column bucket (512 buckets
//      over the column range: counts, a scan, atomic slots) and each thread
//      insertion-sorts one bucket in place -- linear work instead of sorting
//      the whole table (a row whose fullest bucket holds more than 128
//      entries falls back to the bitonic sort).
// Tables are at most half full, probing is linear and every insert succeeds
// (nothing is dropped).  Explicit zeros (cancellation) stay in the structure,
// as the reference's insert keeps every touched key.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "common.cuh"
#include "context.h"
#include "primitives.cuh"

namespace apspie {
namespace {

constexpr int kWarpRowMaxProd = 256;
constexpr int kWarpTable = 512;
constexpr int kBlockRowMaxProd = 8192;
constexpr int kBlockTable = 16384;
constexpr int kSpgThreads = 512;
constexpr int kWarpsPerBlockSmall = 4;
constexpr int kEmpty = INT_MAX;

__device__ __forceinline__ unsigned hash_col(int j) { return (unsigned)j * 0x9E3779B1u; }

__device__ __forceinline__ int table_bits(long long prod, int cap_bits) {
  int b = 5;
  while ((1ll << b) < 2 * prod && b < cap_bits) ++b;
  return b;
}

// insert key j into keys[0..T); returns the slot; *fresh = true when new
__device__ __forceinline__ int table_insert(int *keys, int bits, int j, bool *fresh) {
  unsigned mask = (1u << bits) - 1u;
  unsigned h = hash_col(j) >> (32 - bits);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    int old = atomicCAS(keys + h, kEmpty, j);
    if (old == kEmpty) {
      *fresh = true;
      return (int)h;
    }
    if (old == j) {
      *fresh = false;
      return (int)h;
    }
    h = (h + 1) & mask;
  }
  *fresh = false;  // unreachable: the table is at most half full
  return -1;
}

// ---------------------------------------------------------- row products ---
__global__ void row_products(int m, const int *__restrict__ Aptr, const int *__restrict__ Aind,
                             const int *__restrict__ Bptr, long long *prod) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int i = gwarp; i < m; i += nwarps) {
    long long acc = 0;
    for (int a = __ldg(Aptr + i) + lane; a < __ldg(Aptr + i + 1); a += 32) {
      int k = __ldg(Aind + a);
      acc += __ldg(Bptr + k + 1) - __ldg(Bptr + k);
    }
    acc = warp_sum(acc);
    if (lane == 0) prod[i] = acc;
  }
}

struct Bins {
  unsigned n[3];
  unsigned pad;
};

__global__ void bin_rows(int m, const long long *prod, int *lists, Bins *bins, int *cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    long long p = prod[i];
    if (p == 0) {
      cnt[i] = 0;
      continue;
    }
    int b = p <= kWarpRowMaxProd ? 0 : (p <= kBlockRowMaxProd ? 1 : 2);
    unsigned s = atomicAdd(&bins->n[b], 1u);
    lists[(size_t)b * m + s] = i;
  }
}

// Deals the products of row i over `nthreads` threads of a group (a warp or
// a block): f(j, value) is called once per product.  Group-level scan-based
// gather over the row's A entries, up to `width` A entries per step.
template <bool WARP, typename F>
__device__ __forceinline__ void for_each_product(int i, const int *__restrict__ Aptr,
                                                 const int *__restrict__ Aind,
                                                 const float *__restrict__ Aval,
                                                 const int *__restrict__ Bptr,
                                                 const int *__restrict__ Bind,
                                                 const float *__restrict__ Bval, int *s_off,
                                                 int *s_bs, float *s_av, F f) {
  const int a0 = __ldg(Aptr + i), a1 = __ldg(Aptr + i + 1);
  const int width = WARP ? 32 : (int)blockDim.x;
  const int tid = WARP ? lane_id() : (int)threadIdx.x;
  for (int c0 = a0; c0 < a1; c0 += width) {
    int a = c0 + tid;
    int bs = 0, d = 0;
    float av = 0.f;
    if (a < a1) {
      int k = __ldg(Aind + a);
      bs = __ldg(Bptr + k);
      d = __ldg(Bptr + k + 1) - bs;
      av = Aval ? __ldg(Aval + a) : 1.0f;
    }
    int excl, total;
    if (WARP) {
      int incl = warp_incl_scan(d);
      excl = incl - d;
      total = __shfl_sync(kFull, incl, 31);
    } else {
      __shared__ int sw[33];
      excl = block_excl_scan(d, sw, &total);
    }
    s_off[tid] = excl;
    s_bs[tid] = bs;
    s_av[tid] = av;
    if (WARP) __syncwarp(); else __syncthreads();
    const int n_a = min(width, a1 - c0);
    // owner of product p: the largest t < n_a with s_off[t] <= p.  A thread's
    // p grows by `width` per step, so its owner only moves forward: gallop
    // from the previous one
    int lo = 0;
    for (int p = tid; p < total; p += width) {
      if (lo + 1 < n_a && s_off[lo + 1] <= p) {
        int step = 1, hi = lo + 1;
        while (hi + step < n_a && s_off[hi + step] <= p) {
          hi += step;
          step <<= 1;
        }
        int l2 = hi, h2 = min(hi + step, n_a) - 1;
        while (l2 < h2) {
          int mid = (l2 + h2 + 1) >> 1;
          if (s_off[mid] <= p) l2 = mid; else h2 = mid - 1;
        }
        lo = l2;
      }
      int b = s_bs[lo] + (p - s_off[lo]);
      f(__ldg(Bind + b), (double)s_av[lo] * (double)(Bval ? __ldg(Bval + b) : 1.0f));
    }
    if (WARP) __syncwarp(); else __syncthreads();
  }
}

// In-place bitonic sort of (keys, vals)[0..n), n a power of two, ascending.
template <bool WARP>
__device__ __forceinline__ void bitonic_sort(int *keys, double *vals, int n) {
  const int width = WARP ? 32 : (int)blockDim.x;
  const int tid = WARP ? lane_id() : (int)threadIdx.x;
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < n / 2; t += width) {
        int lo = 2 * t - (t & (j - 1));
        int hi = lo + j;
        bool up = ((lo & k) == 0);
        int kl = keys[lo], kh = keys[hi];
        if ((kl > kh) == up) {
          keys[lo] = kh;
          keys[hi] = kl;
          if (vals) {
            double t2 = vals[lo];
            vals[lo] = vals[hi];
            vals[hi] = t2;
          }
        }
      }
      if (WARP) __syncwarp(); else __syncthreads();
    }
  }
}

// ------------------------------------------------------------ warp rows ---
template <bool NUMERIC>
__global__ void __launch_bounds__(32 * kWarpsPerBlockSmall)
spgemm_warp_rows(const int *list, const Bins *bins, const long long *prod,
                 const int *__restrict__ Aptr, const int *__restrict__ Aind,
                 const float *__restrict__ Aval, const int *__restrict__ Bptr,
                 const int *__restrict__ Bind, const float *__restrict__ Bval, int *cnt,
                 const int *Cptr, int *Cind, float *Cval) {
  __shared__ int s_keys[kWarpsPerBlockSmall][kWarpTable];
  __shared__ double s_vals[NUMERIC ? kWarpsPerBlockSmall : 1][NUMERIC ? kWarpTable : 1];
  __shared__ int s_off[kWarpsPerBlockSmall][32], s_bs[kWarpsPerBlockSmall][32];
  __shared__ float s_av[kWarpsPerBlockSmall][32];
  const int w = warp_in_block(), lane = lane_id();
  int *keys = s_keys[w];
  double *vals = NUMERIC ? s_vals[w] : nullptr;
  const unsigned nrows = bins->n[0];
  for (unsigned r = blockIdx.x * kWarpsPerBlockSmall + w; r < nrows;
       r += gridDim.x * kWarpsPerBlockSmall) {
    int i = list[r];
    int bits = table_bits(prod[i], 9);
    int T = 1 << bits;
    for (int t = lane; t < T; t += 32) {
      keys[t] = kEmpty;
      if (NUMERIC) vals[t] = 0.0;
    }
    __syncwarp();
    int fresh_count = 0;
    for_each_product<true>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off[w], s_bs[w], s_av[w],
                           [&](int j, double v) {
                             bool fresh;
                             int h = table_insert(keys, bits, j, &fresh);
                             fresh_count += fresh;
                             if (NUMERIC) atomicAdd(vals + h, v);
                           });
    __syncwarp();
    if (!NUMERIC) {
      int c = warp_sum(fresh_count);
      if (lane == 0) cnt[i] = c;
    } else {
      bitonic_sort<true>(keys, vals, T);
      int base = Cptr[i], n = Cptr[i + 1] - base;
      for (int t = lane; t < n; t += 32) {
        Cind[base + t] = keys[t];
        Cval[base + t] = (float)vals[t];
      }
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------- block rows ---
constexpr int kBuckets = kSpgThreads;  // one per thread of the block
constexpr int kBucketMax = 128;        // fuller buckets: bitonic sort instead

template <bool NUMERIC>
__global__ void __launch_bounds__(kSpgThreads)
spgemm_block_rows(const int *list, const Bins *bins, const long long *prod,
                  const int *__restrict__ Aptr, const int *__restrict__ Aind,
                  const float *__restrict__ Aval, const int *__restrict__ Bptr,
                  const int *__restrict__ Bind, const float *__restrict__ Bval, int *cnt,
                  const int *Cptr, int *Cind, float *Cval, int ncols) {
  extern __shared__ __align__(16) unsigned char dyn[];
  double *vals = NUMERIC ? (double *)dyn : nullptr;
  int *keys = (int *)(dyn + (NUMERIC ? sizeof(double) * kBlockTable : 0));
  __shared__ int s_off[kSpgThreads], s_bs[kSpgThreads];
  __shared__ float s_av[kSpgThreads];
  __shared__ int s_cnt;
  const unsigned nrows = bins->n[1];
  for (unsigned r = blockIdx.x; r < nrows; r += gridDim.x) {
    int i = list[r];
    int bits = table_bits(prod[i], 14);
    int T = 1 << bits;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
      keys[t] = kEmpty;
      if (NUMERIC) vals[t] = 0.0;
    }
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    int fresh_count = 0;
    for_each_product<false>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off, s_bs, s_av,
                            [&](int j, double v) {
                              bool fresh;
                              int h = table_insert(keys, bits, j, &fresh);
                              fresh_count += fresh;
                              if (NUMERIC) atomicAdd(vals + h, v);
                            });
    if (!NUMERIC) {
      int c = warp_sum(fresh_count);
      if (lane_id() == 0 && c) atomicAdd(&s_cnt, c);
      __syncthreads();
      if (threadIdx.x == 0) cnt[i] = s_cnt;
    } else {
      __syncthreads();
      const int base = Cptr[i], n = Cptr[i + 1] - base;
      // bucket b holds columns [b * ncols / kBuckets, (b + 1) * ncols / kBuckets)
      __shared__ int s_bcnt[kBuckets], s_bfill[kBuckets], sw2[33];
      s_bcnt[threadIdx.x] = 0;
      s_bfill[threadIdx.x] = 0;
      __syncthreads();
      for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const int j = keys[t];
        if (j != kEmpty) atomicAdd(&s_bcnt[(int)(((long long)j * kBuckets) / ncols)], 1);
      }
      __syncthreads();
      const int mine = s_bcnt[threadIdx.x];
      int total;
      const int start = block_excl_scan(mine, sw2, &total);
      const int fullest = __syncthreads_or(mine > kBucketMax);
      if (!fullest) {
        // the buckets' starts replace their counts, then the scatter
        s_bcnt[threadIdx.x] = start;
        __syncthreads();
        for (int t = threadIdx.x; t < T; t += blockDim.x) {
          const int j = keys[t];
          if (j == kEmpty) continue;
          const int b = (int)(((long long)j * kBuckets) / ncols);
          const int pos = base + s_bcnt[b] + atomicAdd(&s_bfill[b], 1);
          Cind[pos] = j;
          Cval[pos] = (float)vals[t];
        }
        __syncthreads();
        // each thread insertion-sorts its bucket in C (columns are distinct)
        int *ci = Cind + base + start;
        float *cv = Cval + base + start;
        for (int a = 1; a < mine; ++a) {
          const int kj = ci[a];
          const float kv = cv[a];
          int b = a - 1;
          while (b >= 0 && ci[b] > kj) {
            ci[b + 1] = ci[b];
            cv[b + 1] = cv[b];
            --b;
          }
          ci[b + 1] = kj;
          cv[b + 1] = kv;
        }
      } else {
        bitonic_sort<false>(keys, vals, T);
        for (int t = threadIdx.x; t < n; t += blockDim.x) {
          Cind[base + t] = keys[t];
          Cval[base + t] = (float)vals[t];
        }
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------- dense accumulator ---
// One block per row; each resident block owns a bitmap of n bits and n
// doubles in global memory, cleared as the row is emitted.
template <bool NUMERIC>
__global__ void __launch_bounds__(kSpgThreads)
spgemm_dense_rows(const int *list, const Bins *bins, int n,
                  const int *__restrict__ Aptr, const int *__restrict__ Aind,
                  const float *__restrict__ Aval, const int *__restrict__ Bptr,
                  const int *__restrict__ Bind, const float *__restrict__ Bval,
                  unsigned *gbits, double *gvals, int *cnt, const int *Cptr, int *Cind,
                  float *Cval) {
  __shared__ int s_off[kSpgThreads], s_bs[kSpgThreads];
  __shared__ float s_av[kSpgThreads];
  __shared__ int sw[33];
  const int words = (n + 31) / 32;
  unsigned *bits = gbits + (size_t)blockIdx.x * words;
  double *vals = NUMERIC ? gvals + (size_t)blockIdx.x * n : nullptr;
  const unsigned nrows = bins->n[2];
  for (unsigned r = blockIdx.x; r < nrows; r += gridDim.x) {
    int i = list[r];
    for_each_product<false>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off, s_bs, s_av,
                            [&](int j, double v) {
                              unsigned bit = 1u << (j & 31);
                              if (!(__ldcg(bits + (j >> 5)) & bit)) atomicOr(bits + (j >> 5), bit);
                              if (NUMERIC) atomicAdd(vals + j, v);
                            });
    __syncthreads();
    // emit in column order: scan of popcounts over the bitmap, chunk by chunk
    int run = NUMERIC ? Cptr[i] : 0;
    for (int w0 = 0; w0 < words; w0 += blockDim.x) {
      int w = w0 + threadIdx.x;
      unsigned b = w < words ? __ldcg(bits + w) : 0u;
      int total;
      int o = block_excl_scan((int)__popc(b), sw, &total) + run;
      if (NUMERIC) {
        while (b) {
          int t = __ffs(b) - 1;
          b &= b - 1;
          int j = w * 32 + t;
          Cind[o] = j;
          Cval[o] = (float)__ldcg(vals + j);
          vals[j] = 0.0;
          ++o;
        }
      }
      if (w < words) bits[w] = 0u;
      run += total;
    }
    if (!NUMERIC && threadIdx.x == 0) cnt[i] = run;
    __syncthreads();
  }
}

__global__ void to_int32_offsets(int m, const long long *in, int *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += gridDim.x * blockDim.x)
    out[i] = (int)in[i];
}

__global__ void widen_counts(int m, const int *cnt, long long *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    out[i] = cnt[i];
}

__global__ void zero_words(size_t n, unsigned *p) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = 0u;
}
__global__ void zero_doubles(size_t n, double *p) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

int gridsz(apspie_context *ctx, long long n, int threads, int per_sm = 16) {
  long long g = (n + threads - 1) / threads;
  return (int)std::max(1ll, std::min(g, (long long)ctx->num_sms * per_sm));
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_spgemm_symbolic(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B,
                           int *d_Cptr, int64_t *h_nnz) {
  APSPIE_CHECK_CTX(ctx);
  if (!A || !B || !d_Cptr || !h_nnz || A->m < 0 || A->n < 0 || B->m != A->n || B->n < 0 ||
      !A->d_ptr || !B->d_ptr || (A->nnz > 0 && !A->d_ind) || (B->nnz > 0 && !B->d_ind))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_spgemm_symbolic: bad matrices");
  ctx->spgemm_plan_valid = false;
  const int m = A->m, n = B->n;
  cudaStream_t st = ctx->stream;
  auto *prod = (long long *)workspace(ctx, kSlotSpgProd, sizeof(long long) * ((size_t)m + 1));
  auto *lists = (int *)workspace(ctx, kSlotSpgLists, sizeof(int) * 3 * ((size_t)m + 1));
  auto *cnt = (int *)workspace(ctx, kSlotSpgCnt, sizeof(int) * ((size_t)m + 1));
  auto *offs = (long long *)workspace(ctx, kSlotMisc3, sizeof(long long) * ((size_t)m + 2));
  auto *bins = (Bins *)workspace(ctx, kSlotSpgBins, sizeof(Bins) + 64);
  if (!prod || !lists || !cnt || !offs || !bins) return APSPIE_ERR_OOM;
  long long *d_total = (long long *)(bins + 1);
  cudaMemsetAsync(bins, 0, sizeof(Bins), st);
  if (m > 0) {
    row_products<<<gridsz(ctx, (long long)m * 32, 256), 256, 0, st>>>(m, A->d_ptr, A->d_ind,
                                                                      B->d_ptr, prod);
    bin_rows<<<gridsz(ctx, m, 256), 256, 0, st>>>(m, prod, lists, bins, cnt);
    int rc = check_launch(ctx, "spgemm bin", 2);
    if (rc) return rc;
  }
  Bins hb;
  {
    auto *h = (Bins *)pinned(ctx, sizeof(Bins));
    if (!h) return APSPIE_ERR_OOM;
    cudaMemcpyAsync(h, bins, sizeof(Bins), cudaMemcpyDeviceToHost, st);
    int rc = check_cuda(ctx, cudaStreamSynchronize(st), "spgemm bins");
    if (rc) return rc;
    hb = *h;
  }
  const size_t dyn_num = sizeof(double) * kBlockTable + sizeof(int) * kBlockTable;
  const size_t dyn_sym = sizeof(int) * kBlockTable;
  cudaFuncSetAttribute(spgemm_block_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)dyn_num);
  cudaFuncSetAttribute(spgemm_block_rows<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)dyn_sym);
  const int dense_blocks = (int)std::min<unsigned>(hb.n[2], (unsigned)ctx->num_sms * 2);
  const int words = (n + 31) / 32;
  unsigned *gbits = nullptr;
  double *gvals = nullptr;
  if (dense_blocks > 0) {
    gbits = (unsigned *)workspace(ctx, kSlotSpgBits, sizeof(unsigned) * (size_t)words * dense_blocks);
    gvals = (double *)workspace(ctx, kSlotSpgVals, sizeof(double) * (size_t)n * dense_blocks);
    if (!gbits || !gvals) return APSPIE_ERR_OOM;
    zero_words<<<gridsz(ctx, (long long)words * dense_blocks, 256), 256, 0, st>>>(
        (size_t)words * dense_blocks, gbits);
    zero_doubles<<<gridsz(ctx, (long long)n * dense_blocks, 256), 256, 0, st>>>(
        (size_t)n * dense_blocks, gvals);
  }
  // bin b's rows are lists[b * m ...] (bin_rows)
  const int *l0 = lists, *l1 = lists + (size_t)m, *l2 = lists + 2 * (size_t)m;
  // ---- symbolic ----
  if (hb.n[0])
    spgemm_warp_rows<false><<<gridsz(ctx, hb.n[0], kWarpsPerBlockSmall, 64),
                              32 * kWarpsPerBlockSmall, 0, st>>>(
        l0, bins, prod, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind, nullptr, cnt, nullptr,
        nullptr, nullptr);
  if (hb.n[1])
    spgemm_block_rows<false><<<gridsz(ctx, hb.n[1], 1, 4), kSpgThreads, dyn_sym, st>>>(
        l1, bins, prod, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind, nullptr, cnt, nullptr,
        nullptr, nullptr, n);
  if (hb.n[2])
    spgemm_dense_rows<false><<<dense_blocks, kSpgThreads, 0, st>>>(
        l2, bins, n, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind, nullptr, gbits, gvals, cnt,
        nullptr, nullptr, nullptr);
  int rc = check_launch(ctx, "spgemm symbolic", 3);
  if (rc) return rc;
  // ---- row offsets ----
  if (m > 0) {
    widen_counts<<<gridsz(ctx, m, 256), 256, 0, st>>>(m, cnt, offs);
    rc = check_launch(ctx, "widen_counts");
    if (rc) return rc;
    rc = device_exclusive_scan<long long>(ctx, offs, offs, m, d_total);
    if (rc) return rc;
  }
  long long nnzC = 0;
  {
    auto *h = (long long *)pinned(ctx, sizeof(long long));
    if (!h) return APSPIE_ERR_OOM;
    if (m > 0) {
      cudaMemcpyAsync(h, d_total, sizeof(long long), cudaMemcpyDeviceToHost, st);
      rc = check_cuda(ctx, cudaStreamSynchronize(st), "spgemm nnz");
      if (rc) return rc;
      nnzC = *h;
    }
  }
  if (nnzC >= (long long)INT32_MAX)
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "apspie_spgemm: nnz(C) = %lld exceeds int32",
                     nnzC);
  if (m > 0) {
    // offs[m] = total after the scan wrote offs[0..m); set the last entry
    cudaMemcpyAsync(offs + m, d_total, sizeof(long long), cudaMemcpyDeviceToDevice, st);
    to_int32_offsets<<<gridsz(ctx, m + 1, 256), 256, 0, st>>>(m, offs, d_Cptr);
  } else {
    cudaMemsetAsync(d_Cptr, 0, sizeof(int), st);
  }
  rc = check_launch(ctx, "to_int32_offsets");
  if (rc) return rc;
  // the bins, lists, counts and dense accumulators stay in the workspace for
  // the numeric phase
  ctx->spgemm_plan_valid = true;
  ctx->spgemm_plan_A = A->d_ptr;
  ctx->spgemm_plan_B = B->d_ptr;
  ctx->spgemm_plan_m = m;
  ctx->spgemm_plan_n = n;
  for (int b = 0; b < 3; ++b) ctx->spgemm_plan_bins[b] = hb.n[b];
  *h_nnz = nnzC;
  return APSPIE_OK;
}

int apspie_spgemm_numeric(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B,
                          const int *d_Cptr, int *d_Cind, float *d_Cval) {
  APSPIE_CHECK_CTX(ctx);
  if (!A || !B || !d_Cptr || !ctx->spgemm_plan_valid || ctx->spgemm_plan_A != A->d_ptr ||
      ctx->spgemm_plan_B != B->d_ptr || ctx->spgemm_plan_m != A->m || ctx->spgemm_plan_n != B->n)
    return set_error(ctx, APSPIE_ERR_INVALID,
                     "apspie_spgemm_numeric: no matching apspie_spgemm_symbolic before it");
  const int m = A->m, n = B->n;
  cudaStream_t st = ctx->stream;
  Bins hb;
  for (int b = 0; b < 3; ++b) hb.n[b] = ctx->spgemm_plan_bins[b];
  // the symbolic phase's buffers (own slots, same sizes: no reallocation;
  // the dense accumulators are left cleared by every dense-row pass)
  auto *prod = (long long *)workspace(ctx, kSlotSpgProd, sizeof(long long) * ((size_t)m + 1));
  auto *lists = (int *)workspace(ctx, kSlotSpgLists, sizeof(int) * 3 * ((size_t)m + 1));
  auto *cnt = (int *)workspace(ctx, kSlotSpgCnt, sizeof(int) * ((size_t)m + 1));
  auto *bins = (Bins *)workspace(ctx, kSlotSpgBins, sizeof(Bins) + 64);
  if (!prod || !lists || !cnt || !bins) return APSPIE_ERR_OOM;
  const size_t dyn_num = sizeof(double) * kBlockTable + sizeof(int) * kBlockTable;
  const int dense_blocks = (int)std::min<unsigned>(hb.n[2], (unsigned)ctx->num_sms * 2);
  const int words = (n + 31) / 32;
  unsigned *gbits = nullptr;
  double *gvals = nullptr;
  if (dense_blocks > 0) {
    gbits = (unsigned *)workspace(ctx, kSlotSpgBits, sizeof(unsigned) * (size_t)words * dense_blocks);
    gvals = (double *)workspace(ctx, kSlotSpgVals, sizeof(double) * (size_t)n * dense_blocks);
    if (!gbits || !gvals) return APSPIE_ERR_OOM;
  }
  const int *l0 = lists, *l1 = lists + (size_t)m, *l2 = lists + 2 * (size_t)m;
  const int *Cptr = d_Cptr;
  int *Cind = d_Cind;
  float *Cval = d_Cval;
  int rc;
  // ---- numeric ----
  if (hb.n[0])
    spgemm_warp_rows<true><<<gridsz(ctx, hb.n[0], kWarpsPerBlockSmall, 32),
                             32 * kWarpsPerBlockSmall, 0, st>>>(
        l0, bins, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind, B->d_val, cnt, Cptr,
        Cind, Cval);
  if (hb.n[1])
    spgemm_block_rows<true><<<gridsz(ctx, hb.n[1], 1, 1), kSpgThreads, dyn_num, st>>>(
        l1, bins, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind, B->d_val, cnt, Cptr,
        Cind, Cval, n);
  if (hb.n[2])
    spgemm_dense_rows<true><<<dense_blocks, kSpgThreads, 0, st>>>(
        l2, bins, n, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind, B->d_val, gbits, gvals,
        cnt, Cptr, Cind, Cval);
  return check_launch(ctx, "spgemm numeric", 3);
}

int apspie_spgemm(apspie_ctx ctx, const apspie_csr *A, const apspie_csr *B, apspie_csr *C) {
  APSPIE_CHECK_CTX(ctx);
  if (!C) return set_error(ctx, APSPIE_ERR_INVALID, "apspie_spgemm: bad matrices");
  C->m = A ? A->m : 0;
  C->n = B ? B->n : 0;
  C->nnz = 0;
  C->d_ptr = nullptr;
  C->d_ind = nullptr;
  C->d_val = nullptr;
  if (!A || !B || A->m < 0)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_spgemm: bad matrices");
  // C is allocated by the library, as the reference's spgemm does
  // (src/spgemmKernel.cuh:669-681); release it with apspie_csr_free.
  int *Cptr = nullptr, *Cind = nullptr;
  float *Cval = nullptr;
  cudaError_t e = cudaMalloc(&Cptr, sizeof(int) * ((size_t)A->m + 1));
  if (e != cudaSuccess) return check_cuda(ctx, e, "apspie_spgemm: allocating C");
  int64_t nnzC = 0;
  int rc = apspie_spgemm_symbolic(ctx, A, B, Cptr, &nnzC);
  if (rc) {
    cudaFree(Cptr);
    return rc;
  }
  e = cudaMalloc(&Cind, sizeof(int) * (size_t)std::max<int64_t>(1, nnzC));
  if (e == cudaSuccess) e = cudaMalloc(&Cval, sizeof(float) * (size_t)std::max<int64_t>(1, nnzC));
  if (e != cudaSuccess) {
    cudaFree(Cptr);
    cudaFree(Cind);
    cudaFree(Cval);
    return check_cuda(ctx, e, "apspie_spgemm: allocating C");
  }
  rc = apspie_spgemm_numeric(ctx, A, B, Cptr, Cind, Cval);
  if (rc) {
    cudaFree(Cptr);
    cudaFree(Cind);
    cudaFree(Cval);
    return rc;
  }
  C->nnz = nnzC;
  C->d_ptr = Cptr;
  C->d_ind = Cind;
  C->d_val = Cval;
  return APSPIE_OK;
}

int apspie_csr_copy_out(apspie_ctx ctx, const apspie_csr *C, int *d_ptr, int *d_ind,
                        float *d_val) {
  APSPIE_CHECK_CTX(ctx);
  if (!C || !C->d_ptr || !d_ptr)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_csr_copy_out: bad arguments");
  cudaStream_t st = ctx->stream;
  cudaMemcpyAsync(d_ptr, C->d_ptr, sizeof(int) * ((size_t)C->m + 1), cudaMemcpyDeviceToDevice, st);
  if (C->nnz > 0 && d_ind)
    cudaMemcpyAsync(d_ind, C->d_ind, sizeof(int) * (size_t)C->nnz, cudaMemcpyDeviceToDevice, st);
  if (C->nnz > 0 && d_val && C->d_val)
    cudaMemcpyAsync(d_val, C->d_val, sizeof(float) * (size_t)C->nnz, cudaMemcpyDeviceToDevice, st);
  return check_cuda(ctx, cudaGetLastError(), "apspie_csr_copy_out");
}

int apspie_csr_free(apspie_ctx ctx, apspie_csr *C) {
  if (!C) return APSPIE_ERR_INVALID;
  if (ctx) cudaSetDevice(ctx->device);
  if (ctx) cudaStreamSynchronize(ctx->stream);
  cudaFree(C->d_ptr);
  cudaFree(C->d_ind);
  cudaFree(C->d_val);
  C->d_ptr = nullptr;
  C->d_ind = nullptr;
  C->d_val = nullptr;
  C->nnz = 0;
  return APSPIE_OK;
}

}  // extern "C"
