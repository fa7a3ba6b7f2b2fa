// spgemm.cu -- row-wise (Gustavson) hash SpGEMM C = A * B with per-row hash
// tables in shared memory, rows binned by their product count.
//
// Replaces spgemm(d_matrix *C, A, B, partSize, partNum) (src/spgemm.cuh:132-
// 342, KernelInsert src/spgemmKernel.cuh:210-343): the reference tiles A and B
// into partNum x partNum DCSC blocks, intersects k-sets per tile pair on the
// host, inserts every product into a global-memory open-addressing table of
// TABLE_SIZE slots per tile (atomicCAS key (row<<16|col), atomicAdd float,
// entries DROPPED after 25 probes), then radix-sorts the whole tables and
// converts COO to CSR.  Here, in two phases (apspie_spgemm_symbolic /
// apspie_spgemm_numeric, the plan kept in the context between them):
//   0. prod[i] = sum over A(i,k) of nnz(B(k,:)) (an upper bound of nnz(C(i,:)));
//   1. symbolic rows are binned by prod: <= 256 one warp per row (shared hash
//      table); <= 1024 / <= 4096 one block per row on a 2048 / 8192-key
//      shared table (spgemm_mid_rows); longer rows over a shared-memory
//      bitmap of C's columns when B has at most bitmap_max_cols columns
//      (spgemm_bitmap_rows<0>), else a 16384-key table (<= 8192 products) or
//      a dense accumulator in global memory; the distinct columns per row
//      give nnz(C(i,:)), a scan gives C's row offsets;
//   2. the block-row bins are re-binned by that exact output size
//      (rebin_rows): <= 512 / 1024 / 2048 outputs on mid tables of 1024 /
//      2048 / 4096 slots whose entries are put in column order by an
//      in-shared bucket sort; longer rows (bitmap case) on the column bitmap,
//      where a product's position in the column-ordered row is the prefix
//      popcount of the bitmap up to its column (no sort), values staged in
//      shared memory (rows of up to 4096 outputs at 512 threads, windows of
//      16384 positions at 1024 threads for longer ones);
//   3. the numeric pass accumulates in double (so the float result is the
//      correctly rounded exact sum up to double error); warp rows compact
//      their table and emit by rank in column order.
// The bin limits above are those of table load 2 (every table at most half
// full); at load 4 (apspie_ctx_set_tuning, picked per matrix pair by
// apspie_autotune_spgemm) each limit is halved and tables are sized to four
// times their entries, and the warp bin's limit can be lowered so that more
// rows get a 128-thread block.  Probing is linear and every insert succeeds
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
constexpr int kLbsPer = 4;  // products per thread per step of for_each_product_lbs

// The smallest s with (ncols - 1) >> s < nb: buckets of 2^s consecutive
// columns, at most nb of them, in column order.
__device__ __forceinline__ int bucket_shift(int ncols, int nb) {
  int s = 0;
  while (s < 31 && ((ncols - 1) >> s) >= nb) ++s;
  return s;
}

__device__ __forceinline__ unsigned hash_col(int j) { return (unsigned)j * 0x9E3779B1u; }

// log2 of a table of at least load x n slots (load 2 or 4), at most 2^cap_bits
__device__ __forceinline__ int table_bits(long long n, int cap_bits, int load) {
  int b = 5;
  while ((1ll << b) < load * n && b < cap_bits) ++b;
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
  // unreachable while the tables are sized from this product count (at most
  // half full); a numeric call after A or B changed structure can fill one,
  // and the caller then skips the product instead of indexing slot -1
  *fresh = false;
  return -1;
}

// ---------------------------------------------------------- row products ---
// Eight lanes per row (four rows per warp in flight): most rows of A are
// short, so a whole warp per row would leave most lanes idle.
__global__ void row_products(int m, const int *__restrict__ Aptr, const int *__restrict__ Aind,
                             const int *__restrict__ Bptr, long long *prod) {
  const int sub = threadIdx.x & 7;
  const int g = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 3);
  const int ng = (int)((gridDim.x * blockDim.x) >> 3);
  const int rounds = (m + ng - 1) / ng;  // the same for every lane: shuffles stay converged
  for (int rr = 0; rr < rounds; ++rr) {
    const int i = g + rr * ng;
    long long acc = 0;
    if (i < m) {
      const int a1 = __ldg(Aptr + i + 1);
      for (int a = __ldg(Aptr + i) + sub; a < a1; a += 8) {
        const int k = __ldg(Aind + a);
        acc += __ldg(Bptr + k + 1) - __ldg(Bptr + k);
      }
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (i < m && sub == 0) prod[i] = acc;
  }
}

// Row bins.  Symbolic phase, by products: warp rows, two sizes of
// mid rows (hash tables of 2048 / 8192 keys), block rows (bitmap or a
// 16384-key table), dense rows (hash mode only).  Numeric phase, by the
// exact output size of the non-warp rows: three mid sizes (tables of
// 1024 / 2048 / 4096 entries), block rows, bitmap rows staged in global
// memory.  Bin b's rows are lists[b * m ...].
enum {
  kBinWarp = 0,
  kBinMid1,
  kBinMid2,
  kBinBlock,
  kBinDense,
  kBinN1,
  kBinN2,
  kBinN3,
  kBinN4,
  kBinN5,
  kNumBins
};
constexpr int kMid1MaxProd = 1024;
constexpr int kMid2MaxProd = 4096;
constexpr int kN1MaxNnz = 512, kN2MaxNnz = 1024, kN3MaxNnz = 2048;

// Row-bin limits of one SpGEMM.  At table load 2 they are the constants
// above (every table at most half full); at load 4 each is halved, so a row
// goes to the next larger table and every table is at most a quarter full.
// The warp bin's limit may be lowered further (rows then go to the 128-thread
// mid tables).
struct BinLimits {
  int warp, mid1, mid2, block;  // symbolic: products per row
  int n1, n2, n3;               // numeric: outputs per row
};

BinLimits bin_limits(int load, int warp_max_prod) {
  const int d = load >= 4 ? 2 : 1;
  return BinLimits{std::min(warp_max_prod, kWarpRowMaxProd / d), kMid1MaxProd / d,
                   kMid2MaxProd / d, kBlockRowMaxProd / d, kN1MaxNnz / d, kN2MaxNnz / d,
                   kN3MaxNnz / d};
}

// Device-side counters of one SpGEMM, read back by the host in one copy.
struct SpgState {
  unsigned n[kNumBins];
  unsigned maxc;  // largest output row of bin kBinN5
  unsigned maxp;  // most products of a kBinN5 row longer than one staging window
  long long total;  // nnz(C)
};

// Slot of this lane's row in bin b: one atomic per distinct bin of the
// active lanes (the bins' counters are few and hot).
__device__ __forceinline__ unsigned warp_bin_slot(unsigned *counters, int b) {
  const unsigned peers = __match_any_sync(__activemask(), b);
  const int leader = __ffs(peers) - 1;
  unsigned base = 0;
  if (lane_id() == leader) base = atomicAdd(counters + b, (unsigned)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane_id()) - 1u));
}

__global__ void bin_rows(int m, const long long *prod, int *lists, SpgState *st, int *cnt,
                         bool bitmap, BinLimits lim) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    long long p = prod[i];
    if (p == 0) {
      cnt[i] = 0;
      continue;
    }
    int b = p <= lim.warp ? kBinWarp
            : p <= lim.mid1 ? kBinMid1
            : p <= lim.mid2 ? kBinMid2
            : (bitmap || p <= lim.block) ? kBinBlock
                                         : kBinDense;
    lists[(size_t)b * m + warp_bin_slot(st->n, b)] = i;
  }
}

// Deals the products of row i over `nthreads` threads of a group (a warp or
// a block): f(j, value) is called once per product.  Group-level scan-based
// gather over the row's A entries, up to `width` A entries per step.  RUNS
// (blocks only): each thread takes runs of consecutive products (one owner
// search per run; measured faster for the symbolic passes), otherwise the
// threads stride the products (coalesced loads of B; measured faster for
// the numeric passes, which load two arrays of B per product).
template <bool WARP, bool RUNS = false, typename F>
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
    if (!WARP && RUNS) {
      // block: each thread takes runs of vt consecutive products (vt grows
      // with the chunk's products, up to 8): one binary search for a run's
      // first owner (the largest t with s_off[t] <= p), then a linear walk
      const int vt = max(1, min(8, total / width));
      for (int p0 = tid * vt; p0 < total; p0 += width * vt) {
        int lo = 0, hi = n_a - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_off[mid] <= p0) lo = mid; else hi = mid - 1;
        }
        int nxt = lo + 1 < n_a ? s_off[lo + 1] : INT_MAX;
        const int pend = min(p0 + vt, total);
        // the run's product positions first, then all its loads, then the
        // calls: up to 8 independent loads in flight per thread
        int pos[8];
        float av[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int p = p0 + q;
          pos[q] = -1;
          av[q] = 0.f;
          if (p < pend) {
            while (p >= nxt) {
              ++lo;
              nxt = lo + 1 < n_a ? s_off[lo + 1] : INT_MAX;
            }
            pos[q] = s_bs[lo] + (p - s_off[lo]);
            av[q] = s_av[lo];
          }
        }
        int jb[8];
        float bv[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          jb[q] = pos[q] >= 0 ? __ldg(Bind + pos[q]) : -1;
          bv[q] = (pos[q] >= 0 && Bval) ? __ldg(Bval + pos[q]) : 1.0f;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (jb[q] >= 0) f(jb[q], (double)av[q] * (double)bv[q]);
      }
      __syncthreads();
      continue;
    }
    // strided: owner of product p, the largest t < n_a with s_off[t] <= p.
    // A thread's p grows by `width` per step, so its owner only moves
    // forward: gallop from the previous one
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

// Block-wide exclusive max-scan of one int per thread (identity -1).
template <int TPB>
__device__ __forceinline__ int block_excl_max(int v, int *sw) {
  const int lane = lane_id(), w = warp_in_block();
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl = max(incl, y);
  }
  if (lane == 31) sw[w] = incl;
  __syncthreads();
  if (w == 0) {
    int x = lane < TPB / 32 ? sw[lane] : -1;
    int xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, xi, o);
      if (lane >= o) xi = max(xi, y);
    }
    const int prev = __shfl_up_sync(kFull, xi, 1);
    if (lane < TPB / 32) sw[lane] = lane ? prev : -1;
  }
  __syncthreads();
  const int before = sw[w];
  const int ex = __shfl_up_sync(kFull, incl, 1);
  const int res = max(before, lane ? ex : -1);
  __syncthreads();
  return res;
}

// Block version of for_each_product by load-balanced search: the chunk's
// products are taken in windows of 2 * TPB; each A entry marks the window
// position of its first product with its index (the entry running into the
// window marks position 0), an inclusive max-scan turns the marks into the
// owner of every position, and thread t handles positions t and t + TPB --
// one shared-memory read for the owner, and the loads of B's rows coalesced.
template <int TPB, int PER = kLbsPer, typename F>
__device__ __forceinline__ void for_each_product_lbs(int i, const int *__restrict__ Aptr,
                                                     const int *__restrict__ Aind,
                                                     const float *__restrict__ Aval,
                                                     const int *__restrict__ Bptr,
                                                     const int *__restrict__ Bind,
                                                     const float *__restrict__ Bval, int *s_off,
                                                     int *s_bs, float *s_av, F f) {
  // PER products per thread per step: the owner map and its max-scan
  // (five block barriers) are paid once per PER * TPB products
  constexpr int CAP = PER * TPB;
  __shared__ int s_om[CAP];
  __shared__ int sw[33];
  const int a0 = __ldg(Aptr + i), a1 = __ldg(Aptr + i + 1);
  const int tid = threadIdx.x;
  int pb = 0;  // products of the row before this chunk of A entries
  for (int c0 = a0; c0 < a1; c0 += TPB) {
    const int a = c0 + tid;
    int bs = 0, d = 0;
    float av = 0.f;
    if (a < a1) {
      const int k = __ldg(Aind + a);
      bs = __ldg(Bptr + k);
      d = __ldg(Bptr + k + 1) - bs;
      av = Aval ? __ldg(Aval + a) : 1.0f;
    }
    int total;
    const int excl = block_excl_scan(d, sw, &total);
    s_off[tid] = excl;
    s_bs[tid] = bs;
    s_av[tid] = av;
    for (int w0 = 0; w0 < total; w0 += CAP) {
      const int wn = min(CAP, total - w0);
#pragma unroll
      for (int h = 0; h < PER; ++h) s_om[tid + h * TPB] = -1;
      __syncthreads();
      if (d > 0) {
        if (excl >= w0 && excl < w0 + wn) s_om[excl - w0] = tid;
        else if (excl < w0 && excl + d > w0) s_om[0] = tid;
      }
      __syncthreads();
      int run[PER];
#pragma unroll
      for (int h = 0; h < PER; ++h) {
        run[h] = s_om[PER * tid + h];
        if (h) run[h] = max(run[h], run[h - 1]);
      }
      const int pre = block_excl_max<TPB>(run[PER - 1], sw);
#pragma unroll
      for (int h = 0; h < PER; ++h) s_om[PER * tid + h] = max(pre, run[h]);
      __syncthreads();
#pragma unroll
      for (int h = 0; h < PER; ++h) {
        const int q = tid + h * TPB;
        if (q < wn) {
          const int o = s_om[q];
          const int b = s_bs[o] + (w0 + q - s_off[o]);
          f(__ldg(Bind + b), (double)s_av[o] * (double)(Bval ? __ldg(Bval + b) : 1.0f),
            pb + w0 + q);
        }
      }
      __syncthreads();
    }
    pb += total;
    __syncthreads();
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
// Writes the warp's compacted row (keys[0..fill) distinct, keys[fill..fill4)
// padded with kEmpty) to C in column order: lane l holds entries l, l + 32,
// ..., (P of them) and counts, over the whole row read four keys at a time
// (broadcast loads), the keys below each; that count is the entry's place.
template <int P>
__device__ __forceinline__ void rank_emit(const int *keys, const double *vals, int fill,
                                          int fill4, int n, int *ci, float *cv) {
  const int lane = lane_id();
  int myk[P], rk[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int e = lane + 32 * q;
    myk[q] = e < fill ? keys[e] : kEmpty;
    rk[q] = 0;
  }
  const int4 *k4 = reinterpret_cast<const int4 *>(keys);
  for (int f = 0; f < (fill4 >> 2); ++f) {
    const int4 x = k4[f];
#pragma unroll
    for (int q = 0; q < P; ++q)
      rk[q] += (x.x < myk[q]) + (x.y < myk[q]) + (x.z < myk[q]) + (x.w < myk[q]);
  }
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const int e = lane + 32 * q;
    if (e < fill && rk[q] < n) {
      ci[rk[q]] = myk[q];
      cv[rk[q]] = (float)vals[e];
    }
  }
}

template <bool NUMERIC>
__global__ void __launch_bounds__(32 * kWarpsPerBlockSmall)
spgemm_warp_rows(const int *list, const unsigned *nlist, const long long *prod,
                 const int *__restrict__ Aptr, const int *__restrict__ Aind,
                 const float *__restrict__ Aval, const int *__restrict__ Bptr,
                 const int *__restrict__ Bind, const float *__restrict__ Bval, int *cnt,
                 const int *Cptr, int *Cind, float *Cval, int load) {
  __shared__ int s_keys[kWarpsPerBlockSmall][kWarpTable];
  __shared__ double s_vals[NUMERIC ? kWarpsPerBlockSmall : 1][NUMERIC ? kWarpTable : 1];
  __shared__ int s_off[kWarpsPerBlockSmall][32], s_bs[kWarpsPerBlockSmall][32];
  __shared__ float s_av[kWarpsPerBlockSmall][32];
  const int w = warp_in_block(), lane = lane_id();
  int *keys = s_keys[w];
  double *vals = NUMERIC ? s_vals[w] : nullptr;
  const unsigned nrows = *nlist;
  for (unsigned r = blockIdx.x * kWarpsPerBlockSmall + w; r < nrows;
       r += gridDim.x * kWarpsPerBlockSmall) {
    int i = list[r];
    int bits = table_bits(prod[i], 9, load);
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
                             if (NUMERIC && h >= 0) atomicAdd(vals + h, v);
                           });
    __syncwarp();
    if (!NUMERIC) {
      int c = warp_sum(fresh_count);
      if (lane == 0) cnt[i] = c;
    } else {
      // compact the occupied slots to the front (in place: a slot moves
      // only left, and each chunk of 32 is read before it is written), pad
      // to a power of two and sort that instead of the whole table
      int base = Cptr[i], n = Cptr[i + 1] - base;
      int fill = 0;
      for (int t0 = 0; t0 < T; t0 += 32) {
        const int k = keys[t0 + lane];
        const double v = vals[t0 + lane];
        const unsigned occ = __ballot_sync(kFull, k != kEmpty);
        __syncwarp();
        if (k != kEmpty) {
          const int d = fill + __popc(occ & ((1u << lane) - 1u));
          keys[d] = k;
          vals[d] = v;
        }
        fill += __popc(occ);
        __syncwarp();
      }
      // pad to a multiple of four with keys that compare above every column
      const int fill4 = (fill + 3) & ~3;
      if (fill + lane < fill4) keys[fill + lane] = kEmpty;
      __syncwarp();
      // each entry's rank among the row's (distinct) columns is its place in C
      const int per = (fill + 31) >> 5;
      if (per <= 1) rank_emit<1>(keys, vals, fill, fill4, n, Cind + base, Cval + base);
      else if (per <= 2) rank_emit<2>(keys, vals, fill, fill4, n, Cind + base, Cval + base);
      else if (per <= 4) rank_emit<4>(keys, vals, fill, fill4, n, Cind + base, Cval + base);
      else rank_emit<8>(keys, vals, fill, fill4, n, Cind + base, Cval + base);
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------- block rows ---
constexpr int kBuckets = kSpgThreads;  // one per thread of the block
constexpr int kBucketMax = 128;        // fuller buckets: bitonic sort instead

template <bool NUMERIC>
__global__ void __launch_bounds__(kSpgThreads)
spgemm_block_rows(const int *list, const unsigned *nlist, const long long *prod,
                  const int *__restrict__ Aptr, const int *__restrict__ Aind,
                  const float *__restrict__ Aval, const int *__restrict__ Bptr,
                  const int *__restrict__ Bind, const float *__restrict__ Bval, int *cnt,
                  const int *Cptr, int *Cind, float *Cval, int ncols, int load) {
  extern __shared__ __align__(16) unsigned char dyn[];
  double *vals = NUMERIC ? (double *)dyn : nullptr;
  int *keys = (int *)(dyn + (NUMERIC ? sizeof(double) * kBlockTable : 0));
  __shared__ int s_off[kSpgThreads], s_bs[kSpgThreads];
  __shared__ float s_av[kSpgThreads];
  __shared__ int s_cnt;
  const unsigned nrows = *nlist;
  // column buckets of 2^bshift columns, at most kBuckets of them
  const int bshift = bucket_shift(ncols, kBuckets);
  for (unsigned r = blockIdx.x; r < nrows; r += gridDim.x) {
    int i = list[r];
    int bits = table_bits(prod[i], 14, load);
    int T = 1 << bits;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
      keys[t] = kEmpty;
      if (NUMERIC) vals[t] = 0.0;
    }
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    int fresh_count = 0;
    for_each_product_lbs<kSpgThreads>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off, s_bs, s_av,
                            [&](int j, double v, int) {
                              bool fresh;
                              int h = table_insert(keys, bits, j, &fresh);
                              fresh_count += fresh;
                              if (NUMERIC && h >= 0) atomicAdd(vals + h, v);
                            });
    if (!NUMERIC) {
      int c = warp_sum(fresh_count);
      if (lane_id() == 0 && c) atomicAdd(&s_cnt, c);
      __syncthreads();
      if (threadIdx.x == 0) cnt[i] = s_cnt;
    } else {
      __syncthreads();
      const int base = Cptr[i], n = Cptr[i + 1] - base;
      // bucket b holds columns [b << bshift, (b + 1) << bshift)
      __shared__ int s_bcnt[kBuckets], s_bfill[kBuckets], sw2[33];
      s_bcnt[threadIdx.x] = 0;
      s_bfill[threadIdx.x] = 0;
      __syncthreads();
      for (int t = threadIdx.x; t < T; t += blockDim.x) {
        const int j = keys[t];
        if (j != kEmpty) atomicAdd(&s_bcnt[j >> bshift], 1);
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
          const int b = j >> bshift;
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

// ------------------------------------------------------------- mid rows ---
// One block of TPB threads per row, a hash table of up to 2^TBITS slots in
// dynamic shared memory sized to the row (products for the symbolic pass,
// the exact output size for the numeric pass, so at most half full).  The
// numeric pass then sorts the row in shared memory: the occupied entries are
// scattered by column range into TPB buckets (counts, a scan, atomic slots),
// each thread insertion-sorts one bucket, and the row is written to C
// coalesced.  A row whose fullest bucket holds more than kMidBucketMax
// entries bitonic-sorts its table instead.  Several rows per SM are in
// flight, which is what hides the L2 latency of gathering B's rows.
constexpr int kMidBucketMax = 64;

template <int TPB, int TBITS, bool NUMERIC>
constexpr size_t mid_smem() {
  return NUMERIC ? (size_t)16 << TBITS : (size_t)4 << TBITS;
}

template <bool NUMERIC, int TPB, int TBITS>
__global__ void __launch_bounds__(TPB)
spgemm_mid_rows(const int *list, const unsigned *nlist, const long long *prod,
                const int *__restrict__ Aptr, const int *__restrict__ Aind,
                const float *__restrict__ Aval, const int *__restrict__ Bptr,
                const int *__restrict__ Bind, const float *__restrict__ Bval, int *cnt,
                const int *Cptr, int *Cind, float *Cval, int ncols, int load) {
  constexpr int T = 1 << TBITS;
  extern __shared__ __align__(16) unsigned char dyn[];
  // numeric: vals double[T] | keys int[T] | skeys int[T/2] | svals float[T/2]
  double *vals = NUMERIC ? (double *)dyn : nullptr;
  int *keys = (int *)(dyn + (NUMERIC ? sizeof(double) * T : 0));
  int *skeys = keys + T;
  float *svals = (float *)(skeys + T / 2);
  __shared__ int s_off[TPB], s_bs[TPB];
  __shared__ float s_av[TPB];
  __shared__ int s_bstart[TPB], s_bfill[TPB], sw[33];
  __shared__ int s_cnt;
  const int tid = threadIdx.x;
  const unsigned nrows = *nlist;
  // column buckets of 2^bshift columns, at most TPB of them (a shift per
  // key instead of a 64-bit division)
  const int bshift = bucket_shift(ncols, TPB);
  for (unsigned r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = list[r];
    const int base = NUMERIC ? Cptr[i] : 0;
    const int n = NUMERIC ? Cptr[i + 1] - base : 0;
    const int bits = table_bits(NUMERIC ? (long long)n : prod[i], TBITS, load);
    const int Tn = 1 << bits;
    for (int t = tid; t < Tn; t += TPB) {
      keys[t] = kEmpty;
      if (NUMERIC) vals[t] = 0.0;
    }
    s_bstart[tid] = 0;
    s_bfill[tid] = 0;
    if (tid == 0) s_cnt = 0;
    __syncthreads();
    int fresh_count = 0;
    for_each_product_lbs<TPB>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off, s_bs, s_av,
                            [&](int j, double v, int) {
                              bool fresh;
                              const int h = table_insert(keys, bits, j, &fresh);
                              fresh_count += fresh;
                              if (NUMERIC && h >= 0) atomicAdd(vals + h, v);
                            });
    if (!NUMERIC) {
      const int c = warp_sum(fresh_count);
      if (lane_id() == 0 && c) atomicAdd(&s_cnt, c);
      __syncthreads();
      if (tid == 0) cnt[i] = s_cnt;
      __syncthreads();
      continue;
    }
    // bucket b holds columns [b << bshift, (b + 1) << bshift)
    for (int t = tid; t < Tn; t += TPB) {
      const int j = keys[t];
      if (j != kEmpty) atomicAdd(&s_bstart[j >> bshift], 1);
    }
    __syncthreads();
    const int mine = s_bstart[tid];
    int total;
    const int start = block_excl_scan(mine, sw, &total);
    if (!__syncthreads_or(mine > kMidBucketMax)) {
      s_bstart[tid] = start;
      __syncthreads();
      for (int t = tid; t < Tn; t += TPB) {
        const int j = keys[t];
        if (j == kEmpty) continue;
        const int b = j >> bshift;
        const int pos = s_bstart[b] + atomicAdd(&s_bfill[b], 1);
        if (pos < T / 2) {
          skeys[pos] = j;
          svals[pos] = (float)vals[t];
        }
      }
      __syncthreads();
      int *ck = skeys + start;
      float *cv = svals + start;
      const int len = min(mine, T / 2 - start);
      for (int a = 1; a < len; ++a) {
        const int kj = ck[a];
        const float kv = cv[a];
        int b = a - 1;
        while (b >= 0 && ck[b] > kj) {
          ck[b + 1] = ck[b];
          cv[b + 1] = cv[b];
          --b;
        }
        ck[b + 1] = kj;
        cv[b + 1] = kv;
      }
      __syncthreads();
      const int nw = min(n, T / 2);
      for (int t = tid; t < nw; t += TPB) {
        Cind[base + t] = skeys[t];
        Cval[base + t] = svals[t];
      }
    } else {
      bitonic_sort<false>(keys, vals, Tn);
      for (int t = tid; t < n && t < Tn; t += TPB) {
        Cind[base + t] = keys[t];
        Cval[base + t] = (float)vals[t];
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
spgemm_dense_rows(const int *list, const unsigned *nlist, int n,
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
  const unsigned nrows = *nlist;
  for (unsigned r = blockIdx.x; r < nrows; r += gridDim.x) {
    int i = list[r];
    for_each_product_lbs<kSpgThreads>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off, s_bs, s_av,
                            [&](int j, double v, int) {
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

// ---------------------------------------------------------- bitmap rows ---
// One block per row over a bitmap of the W = ceil(ncols / 32) words of C's
// columns in shared memory.  MODE 0 (symbolic): set a bit per product, the
// row's size is the popcount.  MODE 1 (numeric): set the bits, then
// woff[w] = popcount of words [0, w) (a scan over the words), so the product
// in column j lands at woff[j / 32] + popcount(word & bits below j) of the
// column-ordered row; its value is added there in a double staging row of
// scap entries in shared memory and the row is emitted word by word.  A row
// longer than scap is done in windows of scap positions, one pass over its
// products per window (products outside the window are skipped), so no
// value ever goes through a global atomic.  Staging values are cleared as
// they are emitted and the bits after the last window, so each row starts
// clean.
// With gbm (symbolic: store; numeric: load), the symbolic pass keeps each
// row's finished bitmap in global memory at slot r of its bin (bslot[i] = r)
// and the numeric pass of a row of more than kStageSmem outputs (always a
// bitmap row of the symbolic phase) loads it instead of setting the bits
// again.  With sp_pos / sp_val (numeric, rows longer than one window), the
// first window's pass also records every product's position and value in
// the block's spill region of sp_cap entries, and the later windows stream
// that list instead of gathering the products again.
constexpr int kStageSmem = 4096;     // 512-thread numeric rows: nnz(C(i,:)) <= this
constexpr int kStageBig = 16384;     // 1024-thread numeric rows: window of this many
constexpr int kBitmapMaxWords = 8192;
// device memory the symbolic pass may keep its bitmap rows' bitmaps in, and
// the numeric pass its spilled products in (above: recomputed / re-gathered)
constexpr size_t kStoredBitmapBudget = size_t(1) << 30;
constexpr size_t kSpillBudget = size_t(1) << 30;

template <int MODE, int TPB>
__global__ void __launch_bounds__(TPB, TPB <= 512 ? 2 : 1)
spgemm_bitmap_rows(const int *list, const unsigned *nlist, int W,
                   const int *__restrict__ Aptr, const int *__restrict__ Aind,
                   const float *__restrict__ Aval, const int *__restrict__ Bptr,
                   const int *__restrict__ Bind, const float *__restrict__ Bval, int *cnt,
                   const int *Cptr, int *Cind, float *Cval, int scap, unsigned *gbm,
                   int *bslot, const long long *prod, int *sp_pos, double *sp_val, int sp_cap) {
  extern __shared__ __align__(16) unsigned char dyn[];
  unsigned *bits = (unsigned *)dyn;
  int *woff = (int *)(bits + W);
  double *stage = (double *)(dyn + (size_t)8 * ((W + 1) & ~1));
  __shared__ int s_off[TPB], s_bs[TPB];
  __shared__ float s_av[TPB];
  __shared__ int s_wt[33];
  const int tid = threadIdx.x, lane = lane_id(), wi = warp_in_block();
  constexpr int nw = TPB / 32;
  for (int t = tid; t < W; t += TPB) bits[t] = 0u;
  if (MODE == 1)
    for (int t = tid; t < scap; t += TPB) stage[t] = 0.0;
  __syncthreads();
  // warp wi scans words [ws, we)
  const int seg = ((W + nw - 1) / nw + 31) & ~31;
  const int ws = min(W, wi * seg), we = min(W, ws + seg);
  const unsigned nrows = *nlist;
  for (unsigned r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = list[r];
    if (MODE == 1 && gbm) {
      // the symbolic pass's bitmap of this row
      const unsigned *src = gbm + (size_t)bslot[i] * W;
      for (int w = tid; w < W; w += TPB) bits[w] = __ldcg(src + w);
    } else {
      // bits only: runs of consecutive products per thread measured faster
      // here than the load-balanced search (one array of B per product)
      for_each_product<false, true>(i, Aptr, Aind, nullptr, Bptr, Bind, nullptr, s_off, s_bs,
                                    s_av, [&](int j, double) {
                                      const unsigned bit = 1u << (j & 31);
                                      if (!(bits[j >> 5] & bit)) atomicOr(bits + (j >> 5), bit);
                                    });
    }
    __syncthreads();
    if (MODE == 0) {
      int c = 0;
      unsigned *dst = gbm ? gbm + (size_t)r * W : nullptr;
      for (int w = tid; w < W; w += TPB) {
        c += __popc(bits[w]);
        if (dst) __stcg(dst + w, bits[w]);
        bits[w] = 0u;
      }
      if (gbm && tid == 0) bslot[i] = (int)r;
      c = warp_sum(c);
      if (lane == 0) s_wt[wi] = c;
      __syncthreads();
      if (tid == 0) {
        int tot = 0;
        for (int k = 0; k < nw; ++k) tot += s_wt[k];
        cnt[i] = tot;
      }
      __syncthreads();
      continue;
    }
    int carry = 0;
    for (int w0 = ws; w0 < we; w0 += 32) {
      const int w = w0 + lane;
      const int c = w < we ? __popc(bits[w]) : 0;
      const int incl = warp_incl_scan(c);
      if (w < we) woff[w] = carry + incl - c;
      carry += __shfl_sync(kFull, incl, 31);
    }
    if (lane == 0) s_wt[wi] = carry;
    __syncthreads();
    if (wi == 0) {
      const int x = lane < nw ? s_wt[lane] : 0;
      const int xi = warp_incl_scan(x);
      if (lane < nw) s_wt[lane] = xi - x;
    }
    __syncthreads();
    const int add = s_wt[wi];
    for (int w = ws + lane; w < we; w += 32) woff[w] += add;
    __syncthreads();
    // the row's length from the symbolic phase bounds every position (it
    // equals the popcount unless A or B changed structure in between)
    const int base = Cptr[i];
    const int len = Cptr[i + 1] - base;
    const int np = (int)prod[i];
    // later windows stream the first window's spilled (position, value) list
    const bool spill = sp_pos != nullptr && len > scap && np <= sp_cap;
    int *my_pos = spill ? sp_pos + (size_t)blockIdx.x * sp_cap : nullptr;
    double *my_val = spill ? sp_val + (size_t)blockIdx.x * sp_cap : nullptr;
    for (int p0 = 0; p0 < len; p0 += scap) {
      const int p1 = min(len, p0 + scap);
      if (p0 == 0 || !spill) {
        for_each_product_lbs<TPB>(i, Aptr, Aind, Aval, Bptr, Bind, Bval, s_off, s_bs, s_av,
                                  [&](int j, double v, int q) {
                                    const int w = j >> 5;
                                    const int pos =
                                        woff[w] + __popc(bits[w] & ((1u << (j & 31)) - 1u));
                                    if (spill && q < np) {
                                      __stcg(my_pos + q, pos);
                                      __stcg(my_val + q, v);
                                    }
                                    if (pos >= p0 && pos < p1) atomicAdd(stage + (pos - p0), v);
                                  });
      } else {
        for (int q = tid; q < np; q += TPB) {
          const int pos = __ldcg(my_pos + q);
          if (pos >= p0 && pos < p1) atomicAdd(stage + (pos - p0), __ldcg(my_val + q));
        }
      }
      __syncthreads();
      for (int w = tid; w < W; w += TPB) {
        unsigned b = bits[w];
        int k = woff[w];
        if (!b || k >= p1 || k + __popc(b) <= p0) continue;
        while (b && k < p1) {
          const int t = __ffs(b) - 1;
          b &= b - 1;
          if (k >= p0) {
            Cind[base + k] = w * 32 + t;
            Cval[base + k] = (float)stage[k - p0];
            stage[k - p0] = 0.0;
          }
          ++k;
        }
      }
      __syncthreads();
    }
    for (int w = tid; w < W; w += TPB) bits[w] = 0u;
    __syncthreads();
  }
}

// Re-bins the rows of the mid and block bins for the numeric phase by
// their exact output size (cnt, from the symbolic phase).
__global__ void rebin_rows(int m, int *lists, SpgState *st, const int *cnt, bool bitmap,
                           BinLimits lim, const long long *prod) {
  const unsigned n1 = st->n[kBinMid1], n2 = st->n[kBinMid2], n3 = st->n[kBinBlock];
  const unsigned n = n1 + n2 + n3;
  for (unsigned r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int src = r < n1 ? kBinMid1 : (r < n1 + n2 ? kBinMid2 : kBinBlock);
    const unsigned k = r < n1 ? r : (r < n1 + n2 ? r - n1 : r - n1 - n2);
    const int i = lists[(size_t)src * m + k];
    const int c = cnt[i];
    const int b = c <= lim.n1   ? kBinN1
                  : c <= lim.n2 ? kBinN2
                  : c <= lim.n3 ? kBinN3
                  : (!bitmap || c <= kStageSmem) ? kBinN4
                                                 : kBinN5;
    lists[(size_t)b * m + warp_bin_slot(st->n, b)] = i;
    if (b == kBinN5) {
      atomicMax(&st->maxc, (unsigned)c);
      if (c > kStageBig) atomicMax(&st->maxp, (unsigned)prod[i]);
    }
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
  auto *lists = (int *)workspace(ctx, kSlotSpgLists, sizeof(int) * kNumBins * ((size_t)m + 1));
  auto *cnt = (int *)workspace(ctx, kSlotSpgCnt, sizeof(int) * ((size_t)m + 1));
  auto *offs = (long long *)workspace(ctx, kSlotMisc3, sizeof(long long) * ((size_t)m + 2));
  auto *sst = (SpgState *)workspace(ctx, kSlotSpgBins, sizeof(SpgState));
  if (!prod || !lists || !cnt || !offs || !sst) return APSPIE_ERR_OOM;
  long long *d_total = &sst->total;
  // block rows over a column bitmap when C's columns fit shared memory
  const int bwords = (n + 31) / 32;
  const bool bitmap = n > 0 && (long long)n <= ctx->spgemm_bitmap_max_cols &&
                      bwords <= kBitmapMaxWords;
  auto L = [&](int b) { return lists + (size_t)b * m; };
  const int load = ctx->spgemm_table_load;
  const BinLimits lim = bin_limits(load, ctx->spgemm_warp_max_prod);
  int rc0 = check_cuda(ctx, cudaMemsetAsync(sst, 0, sizeof(SpgState), st), "spgemm bins");
  if (rc0) return rc0;
  if (m > 0) {
    row_products<<<gridsz(ctx, (long long)m * 32, 256), 256, 0, st>>>(m, A->d_ptr, A->d_ind,
                                                                      B->d_ptr, prod);
    bin_rows<<<gridsz(ctx, m, 256), 256, 0, st>>>(m, prod, lists, sst, cnt, bitmap, lim);
    int rc = check_launch(ctx, "spgemm bin", 2);
    if (rc) return rc;
  }
  SpgState hb{};
  {
    auto *h = (SpgState *)pinned(ctx, sizeof(SpgState));
    if (!h) return APSPIE_ERR_OOM;
    cudaMemcpyAsync(h, sst, sizeof(SpgState), cudaMemcpyDeviceToHost, st);
    int rc = check_cuda(ctx, cudaStreamSynchronize(st), "spgemm bins");
    if (rc) return rc;
    hb = *h;
  }
  const size_t dyn_sym = sizeof(int) * kBlockTable;
  cudaFuncSetAttribute(spgemm_block_rows<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)dyn_sym);
  cudaFuncSetAttribute(spgemm_bitmap_rows<0, kSpgThreads>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(4 * kBitmapMaxWords));
  cudaFuncSetAttribute(spgemm_mid_rows<false, 256, 13>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mid_smem<256, 13, false>());
  const unsigned nd = hb.n[kBinDense];
  const int dense_blocks = (int)std::min<unsigned>(nd, (unsigned)ctx->num_sms * 2);
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
  // the bitmap rows keep their bitmaps for the numeric phase when they fit
  unsigned *gbm = nullptr;
  int *bslot = nullptr;
  if (bitmap && hb.n[kBinBlock] > 0 &&
      (size_t)hb.n[kBinBlock] * bwords * sizeof(unsigned) <= kStoredBitmapBudget) {
    gbm = (unsigned *)workspace(ctx, kSlotSpgStoredBits,
                                (size_t)hb.n[kBinBlock] * bwords * sizeof(unsigned));
    bslot = (int *)workspace(ctx, kSlotSpgBitmapSlot, sizeof(int) * ((size_t)m + 1));
    if (!gbm || !bslot) {  // not kept: the numeric phase sets the bits again
      gbm = nullptr;
      bslot = nullptr;
    }
  }
  // ---- symbolic ----
  const unsigned *nb = sst->n;
  int launches = 0;
  if (hb.n[kBinWarp]) {
    spgemm_warp_rows<false><<<gridsz(ctx, hb.n[kBinWarp], kWarpsPerBlockSmall, 64),
                              32 * kWarpsPerBlockSmall, 0, st>>>(
        L(kBinWarp), nb + kBinWarp, prod, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind,
        nullptr, cnt, nullptr, nullptr, nullptr, load);
    ++launches;
  }
  if (hb.n[kBinMid1]) {
    spgemm_mid_rows<false, 128, 11><<<gridsz(ctx, hb.n[kBinMid1], 1, 16), 128,
                                      mid_smem<128, 11, false>(), st>>>(
        L(kBinMid1), nb + kBinMid1, prod, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind,
        nullptr, cnt, nullptr, nullptr, nullptr, n, load);
    ++launches;
  }
  if (hb.n[kBinMid2]) {
    spgemm_mid_rows<false, 256, 13><<<gridsz(ctx, hb.n[kBinMid2], 1, 6), 256,
                                      mid_smem<256, 13, false>(), st>>>(
        L(kBinMid2), nb + kBinMid2, prod, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind,
        nullptr, cnt, nullptr, nullptr, nullptr, n, load);
    ++launches;
  }
  if (hb.n[kBinBlock] && bitmap) {
    spgemm_bitmap_rows<0, kSpgThreads><<<gridsz(ctx, hb.n[kBinBlock], 1, 4), kSpgThreads,
                                         (size_t)4 * bwords, st>>>(
        L(kBinBlock), nb + kBinBlock, bwords, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind,
        nullptr, cnt, nullptr, nullptr, nullptr, 0, gbm, bslot, prod, nullptr, nullptr, 0);
    ++launches;
  } else if (hb.n[kBinBlock]) {
    spgemm_block_rows<false><<<gridsz(ctx, hb.n[kBinBlock], 1, 4), kSpgThreads, dyn_sym, st>>>(
        L(kBinBlock), nb + kBinBlock, prod, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind,
        nullptr, cnt, nullptr, nullptr, nullptr, n, load);
    ++launches;
  }
  if (nd) {
    spgemm_dense_rows<false><<<dense_blocks, kSpgThreads, 0, st>>>(
        L(kBinDense), nb + kBinDense, n, A->d_ptr, A->d_ind, nullptr, B->d_ptr, B->d_ind, nullptr,
        gbits, gvals, cnt, nullptr, nullptr, nullptr);
    ++launches;
  }
  int rc = check_launch(ctx, "spgemm symbolic", launches);
  if (rc) return rc;
  // ---- row offsets ----
  if (m > 0) {
    widen_counts<<<gridsz(ctx, m, 256), 256, 0, st>>>(m, cnt, offs);
    rc = check_launch(ctx, "widen_counts");
    if (rc) return rc;
    rc = device_exclusive_scan<long long>(ctx, offs, offs, m, d_total);
    if (rc) return rc;
  }
  const unsigned nre = hb.n[kBinMid1] + hb.n[kBinMid2] + hb.n[kBinBlock];
  if (nre) {
    rebin_rows<<<gridsz(ctx, nre, 256), 256, 0, st>>>(m, lists, sst, cnt, bitmap, lim, prod);
    rc = check_launch(ctx, "rebin_rows");
    if (rc) return rc;
  }
  long long nnzC = 0;
  SpgState hs{};
  if (m > 0) {
    auto *h = (SpgState *)pinned(ctx, sizeof(SpgState));
    if (!h) return APSPIE_ERR_OOM;
    cudaMemcpyAsync(h, sst, sizeof(SpgState), cudaMemcpyDeviceToHost, st);
    rc = check_cuda(ctx, cudaStreamSynchronize(st), "spgemm nnz");
    if (rc) return rc;
    hs = *h;
    nnzC = hs.total;
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
  // the lists, counts and dense accumulators stay in the workspace for the
  // numeric phase
  ctx->spgemm_plan_valid = true;
  ctx->spgemm_plan_A = A->d_ptr;
  ctx->spgemm_plan_B = B->d_ptr;
  ctx->spgemm_plan_m = m;
  ctx->spgemm_plan_n = n;
  for (int b = 0; b < kNumBins; ++b) ctx->spgemm_plan_bins[b] = hs.n[b];
  ctx->spgemm_plan_bins[kNumBins] = hs.maxc;
  ctx->spgemm_plan_bins[kNumBins + 1] = hs.maxp;
  ctx->spgemm_plan_gbm = gbm;
  ctx->spgemm_plan_bslot = bslot;
  ctx->spgemm_plan_words = bitmap ? bwords : 0;
  ctx->spgemm_plan_load = load;
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
  const unsigned *hn = ctx->spgemm_plan_bins;
  const int maxc = (int)hn[kNumBins];
  const int bwords = ctx->spgemm_plan_words;
  const int load = ctx->spgemm_plan_load;
  // the symbolic phase's buffers (own slots, same sizes: no reallocation;
  // the dense accumulators are left cleared by every dense-row pass)
  auto *prod = (long long *)workspace(ctx, kSlotSpgProd, sizeof(long long) * ((size_t)m + 1));
  auto *lists = (int *)workspace(ctx, kSlotSpgLists, sizeof(int) * kNumBins * ((size_t)m + 1));
  auto *cnt = (int *)workspace(ctx, kSlotSpgCnt, sizeof(int) * ((size_t)m + 1));
  auto *sst = (SpgState *)workspace(ctx, kSlotSpgBins, sizeof(SpgState));
  if (!prod || !lists || !cnt || !sst) return APSPIE_ERR_OOM;
  auto L = [&](int b) { return lists + (size_t)b * m; };
  const unsigned *nb = sst->n;
  const size_t dyn_num = sizeof(double) * kBlockTable + sizeof(int) * kBlockTable;
  cudaFuncSetAttribute(spgemm_block_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)dyn_num);
  cudaFuncSetAttribute(spgemm_bitmap_rows<1, kSpgThreads>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(8 * kBitmapMaxWords + 8 * kStageSmem + 16));
  cudaFuncSetAttribute(spgemm_bitmap_rows<1, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)(8 * kBitmapMaxWords + 8 * kStageBig + 16));
  cudaFuncSetAttribute(spgemm_mid_rows<true, 256, 12>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mid_smem<256, 12, true>());
  const unsigned nd = hn[kBinDense];
  const int dense_blocks = (int)std::min<unsigned>(nd, (unsigned)ctx->num_sms * 2);
  const int words = (n + 31) / 32;
  unsigned *gbits = nullptr;
  double *gvals = nullptr;
  if (dense_blocks > 0) {
    gbits = (unsigned *)workspace(ctx, kSlotSpgBits, sizeof(unsigned) * (size_t)words * dense_blocks);
    gvals = (double *)workspace(ctx, kSlotSpgVals, sizeof(double) * (size_t)n * dense_blocks);
    if (!gbits || !gvals) return APSPIE_ERR_OOM;
  }
  const int *Cptr = d_Cptr;
  int *Cind = d_Cind;
  float *Cval = d_Cval;
  int launches = 0;
  // ---- numeric ----
  if (hn[kBinWarp]) {
    spgemm_warp_rows<true><<<gridsz(ctx, hn[kBinWarp], kWarpsPerBlockSmall, 32),
                             32 * kWarpsPerBlockSmall, 0, st>>>(
        L(kBinWarp), nb + kBinWarp, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, load);
    ++launches;
  }
  if (hn[kBinN1]) {
    spgemm_mid_rows<true, 128, 10><<<gridsz(ctx, hn[kBinN1], 1, 12), 128,
                                     mid_smem<128, 10, true>(), st>>>(
        L(kBinN1), nb + kBinN1, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, n, load);
    ++launches;
  }
  if (hn[kBinN2]) {
    spgemm_mid_rows<true, 128, 11><<<gridsz(ctx, hn[kBinN2], 1, 6), 128,
                                     mid_smem<128, 11, true>(), st>>>(
        L(kBinN2), nb + kBinN2, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, n, load);
    ++launches;
  }
  if (hn[kBinN3]) {
    spgemm_mid_rows<true, 256, 12><<<gridsz(ctx, hn[kBinN3], 1, 3), 256,
                                     mid_smem<256, 12, true>(), st>>>(
        L(kBinN3), nb + kBinN3, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, n, load);
    ++launches;
  }
  if (hn[kBinN4] && bwords) {
    spgemm_bitmap_rows<1, kSpgThreads><<<gridsz(ctx, hn[kBinN4], 1, 2), kSpgThreads,
                                         (size_t)8 * ((bwords + 1) & ~1) + 8 * kStageSmem, st>>>(
        L(kBinN4), nb + kBinN4, bwords, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, kStageSmem, nullptr, nullptr, prod, nullptr, nullptr,
        0);
    ++launches;
  } else if (hn[kBinN4]) {
    spgemm_block_rows<true><<<gridsz(ctx, hn[kBinN4], 1, 1), kSpgThreads, dyn_num, st>>>(
        L(kBinN4), nb + kBinN4, prod, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, n, load);
    ++launches;
  }
  if (hn[kBinN5]) {
    // rows longer than kStageSmem: 1024 threads, windows of kStageBig, the
    // symbolic pass's bitmaps when it kept them; rows longer than one window
    // spill their products' positions and values in the first window's pass
    const int scap = std::min(kStageBig, std::max(maxc, 1));
    const int g5 = gridsz(ctx, hn[kBinN5], 1, 1);
    const unsigned maxp = hn[kNumBins + 1];
    int *sp_pos = nullptr;
    double *sp_val = nullptr;
    int sp_cap = 0;
    if (maxp > 0 && (size_t)g5 * maxp * (sizeof(int) + sizeof(double)) <= kSpillBudget) {
      sp_pos = (int *)workspace(ctx, kSlotSpgSpillPos, sizeof(int) * (size_t)g5 * maxp);
      sp_val = (double *)workspace(ctx, kSlotSpgSpillVal, sizeof(double) * (size_t)g5 * maxp);
      if (sp_pos && sp_val) {
        sp_cap = (int)maxp;
      } else {  // not spilled: every window gathers the products again
        sp_pos = nullptr;
        sp_val = nullptr;
      }
    }
    spgemm_bitmap_rows<1, 1024><<<g5, 1024,
                                  (size_t)8 * ((bwords + 1) & ~1) + 8 * (size_t)scap, st>>>(
        L(kBinN5), nb + kBinN5, bwords, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, cnt, Cptr, Cind, Cval, scap, (unsigned *)ctx->spgemm_plan_gbm,
        (int *)ctx->spgemm_plan_bslot, prod, sp_pos, sp_val, sp_cap);
    ++launches;
  }
  if (nd) {
    spgemm_dense_rows<true><<<dense_blocks, kSpgThreads, 0, st>>>(
        L(kBinDense), nb + kBinDense, n, A->d_ptr, A->d_ind, A->d_val, B->d_ptr, B->d_ind,
        B->d_val, gbits, gvals, cnt, Cptr, Cind, Cval);
    ++launches;
  }
  return check_launch(ctx, "spgemm numeric", launches);
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
