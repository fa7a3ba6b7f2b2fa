// tc.cu -- triangle counting as an L-masked hash SpGEMM with an int64 count,
// and the device-side degree relabelling that builds L.
//
// Replaces the reference's TC path (test/tc/main.cu:139-261): host buildLower
// of the strict lower / upper triangles, cuSPARSE csrgemm U * L materialising
// every wedge (src/tc.cuh:63-165), the ewiseMultTc merge-intersect
// (src/tc.cuh:169-199) and a float mgpu::Reduce.  Here nothing but the count
// is produced: for each row i of L, L(i,:) goes into a shared-memory hash
// set, and every wedge j in L(k,:) for k in L(i,:) probes it; a hit is a
// triangle (i > k > j).  Rows of up to 256 entries go one warp per row
// (table 512).  Longer rows are cut into units of 512 of their k's, one
// block per unit, so a hub row's wedges spread over many blocks; the unit's
// set of L(i,:) is a bitmap over all vertex ids in shared memory when the
// graph has at most kTcBitmapMaxVerts vertices (one bit probe per wedge),
// else a hash table (rows up to 8192) or a binary search of the sorted row.
// Per-warp partial counts are summed in 64-bit and added with one atomic per
// warp.
//
// tc_prepare relabels vertices by ascending (degree, id) with the stable
// radix sort, keeps the edges with new(col) < new(row), sorts them by
// (row, col) with one radix sort on the packed key and builds L's offsets.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>

#include "common.cuh"
#include "context.h"
#include "gen_common.h"
#include "primitives.cuh"

namespace apspie {
namespace {

// rows of L up to kTcWarpMax entries are one warp's (R-MAT 18, timed side
// by side: 256 -> 2.55 ms, 128 -> 2.26 ms, 64 -> 2.26 ms, 512 -> 17.9 ms);
// longer ones are cut into units
constexpr int kTcWarpMax = 128, kTcWarpTable = 512;
constexpr int kTcBlockMax = 4096, kTcBlockTable = 8192;
constexpr int kTcThreads = 256;
constexpr int kTcWarps = 4;
constexpr int kNone = INT_MAX;

__device__ __forceinline__ unsigned tc_hash(int j) { return (unsigned)j * 0x9E3779B1u; }

__device__ __forceinline__ void set_insert(int *keys, int bits, int j) {
  unsigned mask = (1u << bits) - 1u, h = tc_hash(j) >> (32 - bits);
  for (unsigned p = 0; p <= mask; ++p) {
    int old = atomicCAS(keys + h, kNone, j);
    if (old == kNone || old == j) return;
    h = (h + 1) & mask;
  }
}

__device__ __forceinline__ bool set_has(const int *keys, int bits, int j) {
  unsigned mask = (1u << bits) - 1u, h = tc_hash(j) >> (32 - bits);
  for (unsigned p = 0; p <= mask; ++p) {
    int k = keys[h];
    if (k == j) return true;
    if (k == kNone) return false;
    h = (h + 1) & mask;
  }
  return false;
}

__device__ __forceinline__ int tbits(int n, int cap) {
  int b = 5;
  while ((1 << b) < 2 * n && b < cap) ++b;
  return b;
}

struct TcBins {
  unsigned n[3];
  unsigned pad;
  unsigned long long count;
};

// k's of a long row per block unit: smaller units balance the blocks better
// than the row's column set (rebuilt per unit) costs (R-MAT 18, timed
// side by side: 512 -> 3.2 ms, 256 -> 2.8 ms, 128 -> 2.6 ms, 64 -> 2.55 ms)
constexpr int kTcUnitK = 64;
constexpr int kTcBitmapMaxVerts = 1 << 20;    // 128 KiB of shared bitmap

// warp rows -> lists[0..); long rows -> units (i, piece) in units[0..)
__global__ void tc_bin(int m, const int *__restrict__ Lp, int *lists, int2 *units, TcBins *bins) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    int d = Lp[i + 1] - Lp[i];
    if (d < 2) continue;  // a triangle needs two lower neighbours
    if (d <= kTcWarpMax) {
      lists[atomicAdd(&bins->n[0], 1u)] = i;
    } else {
      const int pieces = (d + kTcUnitK - 1) / kTcUnitK;
      const unsigned s = atomicAdd(&bins->n[1], (unsigned)pieces);
      for (int p = 0; p < pieces; ++p) units[s + p] = make_int2(i, p);
    }
  }
}

// Wedges (k, j) for the k's at positions [a0, a1) of Li, dealt over a group
// (warp or block): visit(j) per wedge.
template <bool WARP, typename F>
__device__ __forceinline__ void for_each_wedge_in(int a0, int a1, const int *__restrict__ Lp,
                                                  const int *__restrict__ Li, int *s_off,
                                                  int *s_bs, F visit) {
  const int width = WARP ? 32 : (int)blockDim.x;
  const int tid = WARP ? lane_id() : (int)threadIdx.x;
  for (int c0 = a0; c0 < a1; c0 += width) {
    int a = c0 + tid, bs = 0, d = 0;
    if (a < a1) {
      int k = __ldg(Li + a);
      bs = __ldg(Lp + k);
      d = __ldg(Lp + k + 1) - bs;
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
    if (WARP) __syncwarp(); else __syncthreads();
    const int n_a = min(width, a1 - c0);
    if (!WARP) {
      // block: runs of vt consecutive wedges per thread (vt grows with the
      // chunk's wedges, up to 8): one binary search for the run's first
      // owner (the largest t with s_off[t] <= p), then a linear walk
      const int vt = max(1, min(8, total / width));
      for (int p0 = tid * vt; p0 < total; p0 += width * vt) {
        int lo = 0, hi = n_a - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_off[mid] <= p0) lo = mid; else hi = mid - 1;
        }
        int nxt = lo + 1 < n_a ? s_off[lo + 1] : INT_MAX;
        const int pend = min(p0 + vt, total);
        // the run's wedge positions first, then all its loads, then the
        // visits: up to 8 independent loads in flight per thread
        int pos[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int p = p0 + q;
          pos[q] = -1;
          if (p < pend) {
            while (p >= nxt) {
              ++lo;
              nxt = lo + 1 < n_a ? s_off[lo + 1] : INT_MAX;
            }
            pos[q] = s_bs[lo] + (p - s_off[lo]);
          }
        }
        int jv[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) jv[q] = pos[q] >= 0 ? __ldg(Li + pos[q]) : -1;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (jv[q] >= 0) visit(jv[q]);
      }
      __syncthreads();
      continue;
    }
    // warp: the k owning wedge p; a lane's p grows by 32 per step, so its
    // owner only moves forward -- gallop from the previous one
    int lo = 0;
    for (int p = tid; p < total; p += width) {
      if (lo + 1 < n_a && s_off[lo + 1] <= p) {
        int step = 1, hi = lo + 1;
        while (hi + step < n_a && s_off[hi + step] <= p) {
          hi += step;
          step <<= 1;
        }
        // owner in [hi, min(hi + step, n_a) - 1]
        int l2 = hi, h2 = min(hi + step, n_a) - 1;
        while (l2 < h2) {
          int mid = (l2 + h2 + 1) >> 1;
          if (s_off[mid] <= p) l2 = mid; else h2 = mid - 1;
        }
        lo = l2;
      }
      visit(__ldg(Li + s_bs[lo] + (p - s_off[lo])));
    }
    if (WARP) __syncwarp(); else __syncthreads();
  }
}

// Wedges of row i.
template <bool WARP, typename F>
__device__ __forceinline__ void for_each_wedge(int i, const int *__restrict__ Lp,
                                               const int *__restrict__ Li, int *s_off, int *s_bs,
                                               F visit) {
  for_each_wedge_in<WARP>(__ldg(Lp + i), __ldg(Lp + i + 1), Lp, Li, s_off, s_bs, visit);
}

__global__ void __launch_bounds__(32 * kTcWarps)
tc_warp_rows(const int *list, TcBins *bins, const int *__restrict__ Lp, const int *__restrict__ Li) {
  __shared__ int s_keys[kTcWarps][kTcWarpTable];
  __shared__ int s_off[kTcWarps][32], s_bs[kTcWarps][32];
  const int w = warp_in_block(), lane = lane_id();
  int *keys = s_keys[w];
  unsigned long long cnt = 0;
  const unsigned nrows = bins->n[0];
  for (unsigned r = blockIdx.x * kTcWarps + w; r < nrows; r += gridDim.x * kTcWarps) {
    int i = list[r];
    int a0 = __ldg(Lp + i), d = __ldg(Lp + i + 1) - a0;
    int bits = tbits(d, 9);
    for (int t = lane; t < (1 << bits); t += 32) keys[t] = kNone;
    __syncwarp();
    for (int t = lane; t < d; t += 32) set_insert(keys, bits, __ldg(Li + a0 + t));
    __syncwarp();
    for_each_wedge<true>(i, Lp, Li, s_off[w], s_bs[w],
                         [&](int j) { cnt += set_has(keys, bits, j) ? 1 : 0; });
    __syncwarp();
  }
  cnt = warp_sum(cnt);
  if (lane == 0 && cnt) atomicAdd(&bins->count, cnt);
}

// One unit = the k's [piece * kTcUnitK, +kTcUnitK) of a long row i, one
// block per unit.  MODE 0: L(i,:) as a bitmap over all vertex ids (dynamic
// shared memory, zero between units: set bits are cleared again); MODE 1:
// hash table (rows up to kTcBlockMax); MODE 2: binary search in the row.
template <int MODE>
__global__ void __launch_bounds__(kTcThreads)
tc_units(const int2 *units, TcBins *bins, int m, const int *__restrict__ Lp,
         const int *__restrict__ Li) {
  extern __shared__ unsigned tc_smem[];
  __shared__ int s_off[kTcThreads], s_bs[kTcThreads];
  unsigned long long cnt = 0;
  const unsigned nunits = bins->n[1];
  if (MODE != 2) {
    const int words = MODE == 0 ? (m + 31) / 32 : kTcBlockTable;
    for (int t = threadIdx.x; t < words; t += blockDim.x) tc_smem[t] = MODE == 0 ? 0u : (unsigned)kNone;
    __syncthreads();
  }
  for (unsigned u = blockIdx.x; u < nunits; u += gridDim.x) {
    const int2 un = units[u];
    const int i = un.x;
    const int a0 = __ldg(Lp + i), a1 = __ldg(Lp + i + 1), d = a1 - a0;
    const int k0 = a0 + un.y * kTcUnitK, k1 = min(k0 + kTcUnitK, a1);
    if (MODE == 0) {
      for (int t = threadIdx.x; t < d; t += blockDim.x) {
        const int j = __ldg(Li + a0 + t);
        atomicOr(tc_smem + (j >> 5), 1u << (j & 31));
      }
      __syncthreads();
      for_each_wedge_in<false>(k0, k1, Lp, Li, s_off, s_bs,
                               [&](int j) { cnt += (tc_smem[j >> 5] >> (j & 31)) & 1u; });
      __syncthreads();
      for (int t = threadIdx.x; t < d; t += blockDim.x) tc_smem[__ldg(Li + a0 + t) >> 5] = 0u;
      __syncthreads();
    } else if (MODE == 1 && d <= kTcBlockMax) {
      int *keys = reinterpret_cast<int *>(tc_smem);
      const int bits = tbits(d, 13);
      for (int t = threadIdx.x; t < (1 << bits); t += blockDim.x) keys[t] = kNone;
      __syncthreads();
      for (int t = threadIdx.x; t < d; t += blockDim.x) set_insert(keys, bits, __ldg(Li + a0 + t));
      __syncthreads();
      for_each_wedge_in<false>(k0, k1, Lp, Li, s_off, s_bs,
                               [&](int j) { cnt += set_has(keys, bits, j) ? 1 : 0; });
      __syncthreads();
    } else {
      for_each_wedge_in<false>(k0, k1, Lp, Li, s_off, s_bs, [&](int j) {
        int lo = a0, hi = a1;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (__ldg(Li + mid) < j) lo = mid + 1; else hi = mid;
        }
        cnt += (lo < a1 && __ldg(Li + lo) == j) ? 1 : 0;
      });
    }
  }
  cnt = warp_sum(cnt);
  if (lane_id() == 0 && cnt) atomicAdd(&bins->count, cnt);
}

// ------------------------------------------------------------- prepare ---
__global__ void degree_keys(int m, const int *__restrict__ ptr, unsigned *keys, int *ids,
                            unsigned *maxdeg) {
  unsigned mx = 0;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < m; v += gridDim.x * blockDim.x) {
    unsigned d = (unsigned)(__ldg(ptr + v + 1) - __ldg(ptr + v));
    keys[v] = d;
    ids[v] = v;
    mx = max(mx, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
  if (lane_id() == 0) atomicMax(maxdeg, mx);
}

__global__ void rank_to_perm(int m, const int *order, int *perm) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x)
    perm[order[r]] = r;
}

// Per vertex v of new id r: how many neighbours rank below r (the length
// of L's row r) and how many above (v's entries in L's columns).  A warp
// per vertex, both counts from one read of the row.  The same pass sums a
// 64-bit hash of every edge (v, u) and of its reverse (u, v) into hsum[0] and
// hsum[1] (wrapping): the edge multiset equals its transpose -- the graph is
// symmetric -- exactly when the multisets of hashed pairs agree, which the two
// sums confirm up to a 2^-64 chance.
__global__ void split_counts(int m, const int *__restrict__ ptr, const int *__restrict__ ind,
                            const int *__restrict__ perm, int *lcnt, int *ucnt,
                            unsigned long long *hsum) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  unsigned long long h_fwd = 0, h_rev = 0;
  for (int v = gwarp; v < m; v += nwarps) {
    const int r = __ldg(perm + v);
    const int s = __ldg(ptr + v), e = __ldg(ptr + v + 1);
    int lo = 0, hi = 0;
    for (int k = s + lane; k < e; k += 32) {
      const int u = __ldg(ind + k);
      const int pu = __ldg(perm + u);
      lo += pu < r;
      hi += pu > r;
      h_fwd += apspie_gen::mix64(((unsigned long long)(unsigned)v << 32) | (unsigned)u);
      h_rev += apspie_gen::mix64(((unsigned long long)(unsigned)u << 32) | (unsigned)v);
    }
    lo = warp_sum(lo);
    hi = warp_sum(hi);
    if (lane == 0) {
      lcnt[r] = lo;
      ucnt[r] = hi;
    }
  }
  h_fwd = warp_sum(h_fwd);
  h_rev = warp_sum(h_rev);
  if (lane == 0 && (h_fwd | h_rev)) {
    atomicAdd(hsum, h_fwd);
    atomicAdd(hsum + 1, h_rev);
  }
}

// L's entries as (row new(u), column r) pairs, grouped by column r in
// ascending order (segment uoff[r]): a stable sort by row then leaves each
// row's columns ascending.  A warp per vertex, lanes compacted by ballot.
__global__ void upper_pairs(int m, const int *__restrict__ ptr, const int *__restrict__ ind,
                            const int *__restrict__ perm, const int *__restrict__ uoff,
                            unsigned *rows, int *cols) {
  const int lane = lane_id();
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int v = gwarp; v < m; v += nwarps) {
    const int r = __ldg(perm + v);
    const int s = __ldg(ptr + v), e = __ldg(ptr + v + 1);
    int out = __ldg(uoff + r);
    for (int k0 = s; k0 < e; k0 += 32) {
      const int k = k0 + lane;
      const int pu = k < e ? __ldg(perm + __ldg(ind + k)) : -1;
      const bool keep = pu > r;
      const unsigned mask = __ballot_sync(kFull, keep);
      if (keep) {
        const int at = out + __popc(mask & ((1u << lane) - 1u));
        rows[at] = (unsigned)pu;
        cols[at] = r;
      }
      out += __popc(mask);
    }
  }
}

int tgrid(apspie_context *ctx, long long n, int threads, int per_sm = 16) {
  long long g = (n + threads - 1) / threads;
  return (int)std::max(1ll, std::min(g, (long long)ctx->num_sms * per_sm));
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_tc_prepare(apspie_ctx ctx, int64_t nnz, int m, const int *d_ptr, const int *d_ind,
                      int *d_perm, int *d_Lptr, int *d_Lind, int64_t *h_lnnz) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || nnz < 0 || nnz >= (int64_t)INT32_MAX || !d_ptr || !d_perm || !d_Lptr ||
      (nnz > 0 && (!d_ind || !d_Lind)) || !h_lnnz)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_tc_prepare: bad arguments");
  cudaStream_t st = ctx->stream;
  const int cbits = bits_for(m);
  if (2 * cbits > 62) return set_error(ctx, APSPIE_ERR_OVERFLOW, "apspie_tc_prepare: m too large");
  // 1. order by (degree, id): stable radix sort of degree keys over ids
  auto *dk = (unsigned *)workspace(ctx, kSlotSortKeysA, sizeof(unsigned) * (size_t)m);
  auto *dk2 = (unsigned *)workspace(ctx, kSlotSortKeysB, sizeof(unsigned) * (size_t)m);
  auto *ids = (int *)workspace(ctx, kSlotSortValsA, sizeof(int) * (size_t)m);
  auto *ids2 = (int *)workspace(ctx, kSlotSortValsB, sizeof(int) * (size_t)m);
  auto *small = (unsigned *)workspace(ctx, kSlotSmall, 64);
  if (!dk || !dk2 || !ids || !ids2 || !small) return APSPIE_ERR_OOM;
  cudaMemsetAsync(small, 0, 64, st);
  degree_keys<<<tgrid(ctx, m, 256), 256, 0, st>>>(m, d_ptr, dk, ids, small);
  int rc = check_launch(ctx, "degree_keys");
  if (rc) return rc;
  unsigned *hs = (unsigned *)pinned(ctx, 64);
  if (!hs) return APSPIE_ERR_OOM;
  cudaMemcpyAsync(hs, small, 8, cudaMemcpyDeviceToHost, st);
  rc = check_cuda(ctx, cudaStreamSynchronize(st), "tc_prepare maxdeg");
  if (rc) return rc;
  const int dbits = std::max(1, bits_for((long long)hs[0] + 1));
  bool in_b = false;
  rc = device_radix_sort<unsigned, int>(ctx, dk, ids, dk2, ids2, m, dbits, &in_b);
  if (rc) return rc;
  rc = radix_sort_check(ctx);  // before the sorted ids index anything
  if (rc) return rc;
  rank_to_perm<<<tgrid(ctx, m, 256), 256, 0, st>>>(m, in_b ? ids2 : ids, d_perm);
  // 2. row lengths of L (indexed by new id) and each vertex's count above it
  auto *lcnt = d_Lptr;
  auto *uoff = (int *)workspace(ctx, kSlotMisc0, sizeof(int) * ((size_t)m + 1));
  if (!uoff) return APSPIE_ERR_OOM;
  cudaMemsetAsync(lcnt + m, 0, sizeof(int), st);
  cudaMemsetAsync(uoff + m, 0, sizeof(int), st);
  // small[0]: the largest degree; small + 8 bytes .. + 24: the two edge hashes
  auto *hsum = reinterpret_cast<unsigned long long *>(small) + 1;
  split_counts<<<tgrid(ctx, (long long)m * 32, 256), 256, 0, st>>>(m, d_ptr, d_ind, d_perm, lcnt,
                                                                   uoff, hsum);
  rc = check_launch(ctx, "split_counts");
  if (rc) return rc;
  // exclusive scans of the m + 1 entries (entry m is 0): offsets + totals
  rc = device_exclusive_scan<int>(ctx, lcnt, d_Lptr, (long long)m + 1, nullptr);
  if (rc) return rc;
  rc = device_exclusive_scan<int>(ctx, uoff, uoff, (long long)m + 1, nullptr);
  if (rc) return rc;
  rc = check_cuda(ctx, cudaMemcpyAsync(hs, d_Lptr + m, 4, cudaMemcpyDeviceToHost, st),
                  "tc_prepare counts");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaMemcpyAsync(hs + 1, uoff + m, 4, cudaMemcpyDeviceToHost, st),
                  "tc_prepare counts");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaMemcpyAsync(hs + 2, hsum, 16, cudaMemcpyDeviceToHost, st),
                  "tc_prepare counts");
  if (rc) return rc;
  rc = check_cuda(ctx, cudaStreamSynchronize(st), "tc_prepare counts");
  if (rc) return rc;
  const long long lnnz = hs[0];
  unsigned long long hh[2];
  std::memcpy(hh, hs + 2, sizeof(hh));
  // L is read from both ends of every edge: the graph must be symmetric
  if (hh[0] != hh[1] || hs[1] != hs[0] || lnnz > nnz / 2)
    return set_error(ctx, APSPIE_ERR_INVALID,
                     "apspie_tc_prepare: the graph is not symmetric (%u entries below, %u above, "
                     "edge hashes %s)",
                     hs[0], hs[1], hh[0] == hh[1] ? "equal" : "differ");
  if (lnnz > 0) {
    // 3. (row, column) pairs grouped by ascending column, stable-sorted by row:
    //    the columns come out in d_Lind (or in the other buffer, then copied)
    auto *ka = (unsigned *)workspace(ctx, kSlotMisc1, sizeof(unsigned) * (size_t)lnnz);
    auto *kb = (unsigned *)workspace(ctx, kSlotMisc2, sizeof(unsigned) * (size_t)lnnz);
    auto *va = (int *)workspace(ctx, kSlotMisc3, sizeof(int) * (size_t)lnnz);
    if (!ka || !kb || !va) return APSPIE_ERR_OOM;
    upper_pairs<<<tgrid(ctx, (long long)m * 32, 256), 256, 0, st>>>(m, d_ptr, d_ind, d_perm,
                                                                    uoff, ka, va);
    rc = check_launch(ctx, "upper_pairs");
    if (rc) return rc;
    in_b = false;
    rc = device_radix_sort<unsigned, int>(ctx, ka, va, kb, d_Lind, lnnz, cbits, &in_b);
    if (rc) return rc;
    rc = radix_sort_check(ctx);
    if (rc) return rc;
    if (!in_b) {
      rc = check_cuda(ctx, cudaMemcpyAsync(d_Lind, va, sizeof(int) * (size_t)lnnz,
                                           cudaMemcpyDeviceToDevice, st),
                      "tc_prepare copy");
      if (rc) return rc;
    }
  }
  *h_lnnz = lnnz;
  return APSPIE_OK;
}

int apspie_tc(apspie_ctx ctx, int m, int64_t lnnz, const int *d_Lptr, const int *d_Lind,
              int64_t *h_count) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || lnnz < 0 || !d_Lptr || (lnnz > 0 && !d_Lind) || !h_count)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_tc: bad arguments");
  cudaStream_t st = ctx->stream;
  auto *lists = (int *)workspace(ctx, kSlotMisc0, sizeof(int) * (size_t)m);
  // units: at most lnnz / kTcUnitK + (rows longer than kTcWarpMax) pieces
  auto *units = (int2 *)workspace(
      ctx, kSlotMisc1, sizeof(int2) * ((size_t)lnnz / kTcUnitK + (size_t)lnnz / kTcWarpMax + 2));
  auto *bins = (TcBins *)workspace(ctx, kSlotSmall, sizeof(TcBins));
  if (!lists || !units || !bins) return APSPIE_ERR_OOM;
  cudaMemsetAsync(bins, 0, sizeof(TcBins), st);
  tc_bin<<<tgrid(ctx, m, 256), 256, 0, st>>>(m, d_Lptr, lists, units, bins);
  tc_warp_rows<<<ctx->num_sms * 16, 32 * kTcWarps, 0, st>>>(lists, bins, d_Lptr, d_Lind);
  // every resident block: the units are L2-latency bound, so occupancy is
  // what hides the latency (the bitmap's shared memory sets the limit)
  if (m <= kTcBitmapMaxVerts) {
    const int smem = (int)(sizeof(unsigned) * (size_t)((m + 31) / 32));
    cudaFuncSetAttribute(tc_units<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc_units<0>, kTcThreads, smem);
    tc_units<0><<<ctx->num_sms * std::max(1, per_sm), kTcThreads, smem, st>>>(units, bins, m,
                                                                              d_Lptr, d_Lind);
  } else {
    const int smem = (int)(sizeof(int) * kTcBlockTable);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc_units<1>, kTcThreads, smem);
    tc_units<1><<<ctx->num_sms * std::max(1, per_sm), kTcThreads, smem, st>>>(units, bins, m,
                                                                              d_Lptr, d_Lind);
  }
  int rc = check_launch(ctx, "apspie_tc", 3);
  if (rc) return rc;
  auto *h = (TcBins *)pinned(ctx, sizeof(TcBins));
  if (!h) return APSPIE_ERR_OOM;
  cudaMemcpyAsync(h, bins, sizeof(TcBins), cudaMemcpyDeviceToHost, st);
  rc = check_cuda(ctx, cudaStreamSynchronize(st), "apspie_tc");
  if (rc) return rc;
  *h_count = (int64_t)h->count;
  return APSPIE_OK;
}

}  // extern "C"
