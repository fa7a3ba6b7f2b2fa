// primitives.cuh -- device-wide scan and a stable LSD radix sort of
// (key, value) pairs, written for this library (the reference uses moderngpu
// Scan and cub::DeviceRadixSort, src/mXv.cuh:142,191-193).
//
// Scan: reduce-then-scan in three launches (tile sums, scan of tile sums in
// one block, tile scans seeded by the scanned sums).  No inter-block waits.
//
// Radix sort: 8-bit digits, only as many passes as the key's significant
// bits need (ceil(log2 m) bits for row indices).  Each pass is
//   1. per-tile digit counts, stored digit-major (counts[d * ntiles + t]);
//   2. one exclusive scan of that array = global base of (digit, tile);
//   3. tile scatter with stable ranks: inside a warp, __match_any_sync groups
//      lanes with the same digit and a per-warp shared histogram carries the
//      running count across rounds; per-digit prefix over the warps of the
//      tile orders the warps.
// Tiles are 256 threads x 16 keys; every key keeps its input order among
// equal digits, so the LSD passes sort stably.
#pragma once
#include <cstdint>

#include "common.cuh"
#include "context.h"

namespace apspie {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread; returns the prefix and
// writes the block total to *total (all threads).
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *smem_warp, T *total) {
  const int lane = lane_id(), w = warp_in_block(), nw = blockDim.x >> 5;
  T incl = warp_incl_scan(v);
  if (lane == 31) smem_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    T x = lane < nw ? smem_warp[lane] : T(0);
    T xi = warp_incl_scan(x);
    if (lane < nw) smem_warp[lane] = xi - x;
    if (lane == nw - 1) smem_warp[32] = xi;
  }
  __syncthreads();
  T res = smem_warp[w] + incl - v;
  *total = smem_warp[32];
  __syncthreads();
  return res;
}

template <typename T>
__global__ void scan_tile_sums(const T *in, long long n, T *sums) {
  __shared__ T sw[33];
  long long base = (long long)blockIdx.x * kScanTile;
  T acc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    long long idx = base + (long long)i * kScanThreads + threadIdx.x;
    if (idx < n) acc += in[idx];
  }
  T tot;
  block_excl_scan(acc, sw, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Exclusive scan of sums[0..n) in one block, blockDim.x values per pass;
// writes the grand total to *total.
template <typename T>
__global__ void scan_single_block(T *sums, int n, T *total) {
  __shared__ T sw[33];
  __shared__ T carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    T v = i < n ? sums[i] : T(0);
    T tot;
    T ex = block_excl_scan(v, sw, &tot);
    if (i < n) sums[i] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

template <typename T>
__global__ void scan_tiles(const T *in, long long n, const T *sums, T *out) {
  __shared__ T sw[33];
  long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  T v[kScanItems];
  T acc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    long long idx = base + i;
    v[i] = idx < n ? in[idx] : T(0);
    acc += v[i];
  }
  T tot;
  T run = block_excl_scan(acc, sw, &tot) + sums[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    long long idx = base + i;
    if (idx < n) out[idx] = run;
    run += v[i];
  }
}

// Exclusive scan in[0..n) -> out[0..n) (may alias); *d_total gets the sum.
// Scratch: slot kSlotScan.  Returns a status.
template <typename T>
int device_exclusive_scan(apspie_context *ctx, const T *in, T *out, long long n, T *d_total) {
  long long tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles < 1) tiles = 1;
  // the tile sums are scanned by one block in a loop: fine up to 2^20 tiles
  // (2^32 elements); T must hold the total
  if (tiles > (1ll << 20))
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "device scan: %lld elements too many", n);
  T *sums = (T *)workspace(ctx, kSlotScan, sizeof(T) * (size_t)(tiles + 1));
  if (!sums) return APSPIE_ERR_OOM;
  // tile sums are computed from `in` before `out` is written, so in == out works
  scan_tile_sums<T><<<(unsigned)tiles, kScanThreads, 0, ctx->stream>>>(in, n, sums);
  scan_single_block<T><<<1, kScanThreads, 0, ctx->stream>>>(sums, (int)tiles, d_total);
  scan_tiles<T><<<(unsigned)tiles, kScanThreads, 0, ctx->stream>>>(in, n, sums, out);
  return check_launch(ctx, "device_exclusive_scan", 3);
}

// ------------------------------------------------------------ radix sort ---
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

template <typename K>
__global__ void radix_count(const K *keys, long long n, int shift, unsigned *counts,
                            unsigned ntiles) {
  __shared__ unsigned hist[kRadix];
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[d] = 0;
  __syncthreads();
  long long base = (long long)blockIdx.x * kSortTile;
  for (int i = threadIdx.x; i < kSortTile; i += blockDim.x) {
    long long idx = base + i;
    if (idx < n) atomicAdd(&hist[(unsigned)(keys[idx] >> shift) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x)
    counts[(size_t)d * ntiles + blockIdx.x] = hist[d];
}

template <typename K, typename V>
__global__ void __launch_bounds__(kSortThreads)
radix_scatter(const K *keys_in, const V *vals_in, K *keys_out, V *vals_out, long long n, int shift,
              const unsigned *offsets, unsigned ntiles) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ unsigned whist[kWarps][kRadix];
  const int lane = lane_id(), w = warp_in_block();
  for (int d = lane; d < kRadix; d += 32) whist[w][d] = 0;
  __syncwarp();
  // this warp's slice: kSortItems rounds of 32 consecutive keys
  long long wbase = (long long)blockIdx.x * kSortTile + (long long)w * 32 * kSortItems;
  unsigned rank[kSortItems];
  unsigned dig[kSortItems];
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    long long idx = wbase + i * 32 + lane;
    bool valid = idx < n;
    unsigned d = valid ? (unsigned)(keys_in[idx] >> shift) & (kRadix - 1) : (unsigned)kRadix;
    unsigned peers = __match_any_sync(kFull, d);
    unsigned lower = peers & ((1u << lane) - 1u);
    int leader = __ffs(peers) - 1;
    unsigned prev = 0;
    if (valid && lane == leader) {
      prev = whist[w][d];
      whist[w][d] = prev + __popc(peers);
    }
    prev = __shfl_sync(kFull, prev, leader);
    rank[i] = prev + __popc(lower);
    dig[i] = d;
    __syncwarp();
  }
  __syncthreads();
  // exclusive prefix over warps per digit, plus the tile's global base
  for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
    unsigned run = offsets[(size_t)d * ntiles + blockIdx.x];
    for (int ww = 0; ww < kWarps; ++ww) {
      unsigned c = whist[ww][d];
      whist[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    long long idx = wbase + i * 32 + lane;
    if (idx < n) {
      unsigned pos = whist[w][dig[i]] + rank[i];
      keys_out[pos] = keys_in[idx];
      if (vals_in) vals_out[pos] = vals_in[idx];  // keys-only sorts pass no values
    }
  }
}

// Stable sort of n (key, value) pairs on the low `bits` bits of the key
// (va == vb == nullptr sorts keys only).  Ping-pongs between (ka, va) and
// (kb, vb); *result_in_b tells where the sorted data ended up.  Scratch: slots kSlotSortHist (+ kSlotScan).
template <typename K, typename V>
int device_radix_sort(apspie_context *ctx, K *ka, V *va, K *kb, V *vb, long long n, int bits,
                      bool *result_in_b) {
  *result_in_b = false;
  if (n <= 1 || bits <= 0) return APSPIE_OK;
  long long tiles = (n + kSortTile - 1) / kSortTile;
  if (tiles * kRadix >= (1ll << 31))
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "radix sort: %lld keys too many", n);
  unsigned nt = (unsigned)tiles;
  auto *counts = (unsigned *)workspace(ctx, kSlotSortHist, sizeof(unsigned) * (size_t)nt * kRadix);
  if (!counts) return APSPIE_ERR_OOM;
  K *kin = ka, *kout = kb;
  V *vin = va, *vout = vb;
  for (int shift = 0; shift < bits; shift += kRadixBits) {
    radix_count<K><<<nt, kSortThreads, 0, ctx->stream>>>(kin, n, shift, counts, nt);
    int rc = check_launch(ctx, "radix_count");
    if (rc) return rc;
    rc = device_exclusive_scan<unsigned>(ctx, counts, counts, (long long)nt * kRadix, nullptr);
    if (rc) return rc;
    radix_scatter<K, V><<<nt, kSortThreads, 0, ctx->stream>>>(kin, vin, kout, vout, n, shift,
                                                              counts, nt);
    rc = check_launch(ctx, "radix_scatter");
    if (rc) return rc;
    std::swap(kin, kout);
    std::swap(vin, vout);
    *result_in_b = !*result_in_b;
  }
  return APSPIE_OK;
}

inline int bits_for(long long m) {
  int b = 0;
  while ((1ll << b) < m) ++b;
  return b;
}

}  // namespace apspie
