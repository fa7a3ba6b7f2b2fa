// primitives.cuh -- device-wide scan and a stable LSD radix sort of
// (key, value) pairs, written for this library (the reference uses moderngpu
// Scan and cub::DeviceRadixSort, src/mXv.cuh:142,191-193).
//
// Scan: reduce-then-scan in three launches (tile sums, scan of tile sums in
// one block, tile scans seeded by the scanned sums).  No inter-block waits.
//
// Radix sort: 8-bit digits, only as many passes as the key's significant
// bits need (ceil(log2 m) bits for row indices), in the onesweep form: one
// read of the keys counts every pass's digits (radix_histograms), then one
// kernel per pass (radix_onesweep) whose tiles of 256 threads x 16 keys
//   * rank their keys: inside a warp, __match_any_sync groups lanes with the
//     same digit, and a per-warp shared histogram carries the running count
//     across rounds; a per-digit prefix over the warps of the tile orders
//     the warps;
//   * find each digit's output offset by decoupled look-back over the tiles
//     before them (bounded waits);
//   * write each digit's run contiguously from a shared-memory copy of the
//     tile, the values copied in by cp.async while the keys were ranked.
// Every key keeps its input order among equal digits, so the LSD passes
// sort stably.
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
// Onesweep LSD radix sort (Adinets & Merrill, "Onesweep: A Faster Least
// Significant Digit Radix Sort for GPUs", 2022): one read of the keys
// counts every pass's digits, then one kernel per 8-bit pass.  A pass's
// tiles take ids from a counter (so a tile only waits on tiles that are
// already running), rank their keys locally (match_any per warp, a prefix
// over the warps), publish their per-digit counts, and find their digit
// offsets by decoupled look-back over the tiles before them: each status
// word holds a flag (aggregate of this tile / inclusive of all before and
// this one), the pass's tag and the count.  Stable.
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxPasses = 8;
constexpr unsigned long long kStAgg = 1ull << 62, kStIncl = 2ull << 62;
constexpr unsigned long long kStCountMask = (1ull << 40) - 1;

// all passes' digit counts in one read of the keys
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
radix_histograms(const K *keys, long long n, int npass, unsigned long long *ghist) {
  __shared__ unsigned hist[kMaxPasses][kRadix];
  for (int t = threadIdx.x; t < kMaxPasses * kRadix; t += blockDim.x) hist[t / kRadix][t % kRadix] = 0;
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const K k = keys[i];
    for (int p = 0; p < npass; ++p)
      atomicAdd(&hist[p][(unsigned)(k >> (p * kRadixBits)) & (kRadix - 1)], 1u);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < npass * kRadix; t += blockDim.x) {
    const unsigned c = hist[t / kRadix][t % kRadix];
    if (c) atomicAdd(ghist + t, (unsigned long long)c);
  }
}

// per pass, exclusive prefix of the digit counts (one block of kRadix)
template <int R = kRadix>
__global__ void radix_digit_offsets(unsigned long long *ghist, int npass) {
  __shared__ unsigned long long sw[33];
  for (int p = 0; p < npass; ++p) {
    const unsigned long long c = ghist[p * R + threadIdx.x];
    unsigned long long total;
    const unsigned long long ex = block_excl_scan(c, sw, &total);
    ghist[p * R + threadIdx.x] = ex;
    __syncthreads();
  }
}

// Polls of a look-back wait before it gives up (a predecessor normally
// publishes within microseconds; about half a second with the back-off).
constexpr unsigned kLookbackSpinLimit = 1u << 20;
constexpr int kLookbackWindow = 4;  // predecessors whose status words are loaded at once

template <typename K, typename V>
__global__ void __launch_bounds__(kSortThreads, 3)
radix_onesweep(const K *keys_in, const V *vals_in, K *keys_out, V *vals_out, long long n,
               int pass, const unsigned long long *goff, unsigned long long *status,
               unsigned *tile_counter, int *err, int *gaveup) {
  constexpr int kWarps = kSortThreads / 32;
  static_assert(sizeof(V) <= sizeof(K), "values are staged in the keys' shared array");
  // the tile in digit order (keys, then values), each key's digit, per-warp
  // digit counts, and per digit the output position of the tile's run minus
  // its start within the tile
  __shared__ __align__(16) K skeys[kSortTile];
  __shared__ unsigned char sdig[kSortTile];
  __shared__ unsigned whist[kWarps][kRadix];
  __shared__ unsigned long long gbase[kRadix];
  __shared__ unsigned long long s_scan[33];
  __shared__ unsigned s_tile;
  __shared__ int s_withhold;
  // the tile's values, copied in by cp.async while the keys are ranked
  // (dynamic: kSortTile values when the sort has values, else none)
  extern __shared__ __align__(16) unsigned char sort_dyn[];
  V *svin = reinterpret_cast<V *>(sort_dyn);
  const int lane = lane_id(), w = warp_in_block();
  const int shift = pass * kRadixBits;
  const unsigned long long tag = (unsigned long long)(pass + 1) << 40;
  if (threadIdx.x == 0) {
    s_tile = atomicAdd(tile_counter, 1u);
    // test hook (apspie_debug_inject): err[1] set makes tile 0 of the next
    // pass withhold its status, so that its successors' bounded look-back
    // waits run out; one-shot
    s_withhold = (s_tile == 0u && n > kSortTile) ? atomicExch(err + 1, 0) : 0;
  }
  for (int d = lane; d < kRadix; d += 32) whist[w][d] = 0;
  __syncthreads();
  const unsigned tile = s_tile;
  const long long tbase = (long long)tile * kSortTile;
  const int tlen = (int)min((long long)kSortTile, n - tbase);
  // Values [0, vdone) of the tile are copied to shared memory in the
  // background, 16 bytes a copy, when they start on a 16-byte boundary; the
  // rest (a ragged end, or an unaligned array) are loaded when placed.
  int vdone = 0;
  if (vals_in && (reinterpret_cast<uintptr_t>(vals_in + tbase) & 15u) == 0) {
    constexpr int kPer = 16 / (int)sizeof(V);
    const int nchunk = tlen / kPer;
    vdone = nchunk * kPer;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(svin);
    for (int c = threadIdx.x; c < nchunk; c += kSortThreads)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sbase + 16u * c),
                   "l"(vals_in + tbase + (long long)c * kPer)
                   : "memory");
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  // this warp's slice of the tile: kSortItems rounds of 32 consecutive keys
  const int wofs = w * 32 * kSortItems;
  // per key its rank (then its tile position); its digit is recomputed
  // from the key where needed (registers for three blocks per SM)
  unsigned pos[kSortItems];
  K kv[kSortItems];
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const int t = wofs + i * 32 + lane;
    kv[i] = t < tlen ? keys_in[tbase + t] : K(0);
  }
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const bool valid = wofs + i * 32 + lane < tlen;
    const unsigned d = valid ? (unsigned)(kv[i] >> shift) & (kRadix - 1) : (unsigned)kRadix;
    const unsigned peers = __match_any_sync(kFull, d);
    const int leader = __ffs(peers) - 1;
    unsigned prev = 0;
    if (valid && lane == leader) {
      prev = whist[w][d];
      whist[w][d] = prev + __popc(peers);
    }
    prev = __shfl_sync(kFull, prev, leader);
    pos[i] = prev + __popc(peers & ((1u << lane) - 1u));
    __syncwarp();
  }
  __syncthreads();
  // per digit (one per thread): prefix over the warps, the tile's count,
  // its start within the tile, then the look-back for its output offset
  const int d = threadIdx.x;
  unsigned run = 0;
  for (int ww = 0; ww < kWarps; ++ww) {
    const unsigned c = whist[ww][d];
    whist[ww][d] = run;
    run += c;
  }
  unsigned long long tot;
  const unsigned long long loc = block_excl_scan((unsigned long long)run, s_scan, &tot);
  unsigned long long *mine = status + (size_t)tile * kRadix + d;
  unsigned long long excl = 0;
  if (tile == 0) {
    if (!s_withhold) __stcg(mine, kStIncl | tag | (unsigned long long)run);
  } else {
    __stcg(mine, kStAgg | tag | (unsigned long long)run);
    // Look back kLookbackWindow predecessors at a time (their status words
    // loaded together, relaxed: a word's count is all that is read), adding
    // counts from the nearest one back until an inclusive word; a word not
    // yet published stops the window and is polled again.
    long long t = (long long)tile - 1;
    unsigned spins = 0;
    while (t >= 0) {
      unsigned long long sv[kLookbackWindow];
#pragma unroll
      for (int k = 0; k < kLookbackWindow; ++k)
        sv[k] = t - k >= 0 ? ld_relaxed64(status + (size_t)(t - k) * kRadix + d) : 0ull;
      bool done = false, stalled = false;
#pragma unroll
      for (int k = 0; k < kLookbackWindow; ++k) {
        if (done || stalled || t < 0) continue;
        const unsigned long long w = sv[k];
        if ((w & (0x3FFFFFull << 40)) != tag || (w >> 62) == 0ull) {
          stalled = true;
          continue;
        }
        excl += w & kStCountMask;
        if ((w >> 62) == 2ull) done = true;  // inclusive: everything before is in it
        else --t;
      }
      if (done) break;
      if (stalled) {
        // a predecessor has not published: give up after kLookbackSpinLimit
        // polls, or at once when another tile of this sort already gave up
        // (checked every 256; *gaveup is zeroed with the sort's status words)
        if (++spins > kLookbackSpinLimit ||
            ((spins & 255u) == 0u && *(volatile int *)gaveup != 0)) {
          atomicExch(err, 1);
          atomicExch(gaveup, 1);
          break;
        }
        if ((spins & 15u) == 0u) __nanosleep(64);
      }
    }
    __stcg(mine, kStIncl | tag | (excl + run));
  }
  gbase[d] = goff[pass * kRadix + d] + excl - loc;
  for (int ww = 0; ww < kWarps; ++ww) whist[ww][d] += (unsigned)loc;
  __syncthreads();
  // tile position of every key: its digit's start + the warps before it + its rank
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    if (wofs + i * 32 + lane < tlen) {
      const unsigned dd = (unsigned)(kv[i] >> shift) & (kRadix - 1);
      pos[i] += whist[w][dd];
      skeys[pos[i]] = kv[i];
      sdig[pos[i]] = (unsigned char)dd;
    }
  }
  __syncthreads();
  // the bound holds for every sorted pass; it guards a pass after a
  // look-back give-up, whose input then holds keys the histograms did not
  // count
  for (int t = threadIdx.x; t < tlen; t += kSortThreads) {
    const unsigned long long at = gbase[sdig[t]] + t;
    if (at < (unsigned long long)n) keys_out[at] = skeys[t];
  }
  if (vals_in) {  // keys-only sorts pass no values
    if (vdone > 0) asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    V *svals = reinterpret_cast<V *>(skeys);
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
      const int t = wofs + i * 32 + lane;
      if (t < tlen) svals[pos[i]] = t < vdone ? svin[t] : vals_in[tbase + t];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < tlen; t += kSortThreads) {
      const unsigned long long at = gbase[sdig[t]] + t;
      if (at < (unsigned long long)n) vals_out[at] = svals[t];
    }
  }
}

// The context's radix-sort give-up word: set by a tile whose look-back
// waited kLookbackSpinLimit polls for a predecessor (the output is then in
// bounds but neither sorted nor a permutation of the input: some slots keep
// stale contents).  A caller that uses sorted keys or values as indices must
// therefore check it (radix_sort_check) before doing so; apspie_spmspv,
// which only bounds-checks its segment writes, checks it at its end.  Sticky: zeroed when first allocated and by
// radix_sort_check, not by each sort, so a caller that synchronises only
// at its end still sees a give-up of any sort it ran.  Stream-ordered
// callers that never synchronise (apspie_bfs_prepare, apspie_csr_transpose)
// leave it to the next call on the context that reads it back (the device
// graph build, apspie_tc_prepare, apspie_spmspv).
inline int *radix_sort_err(apspie_context *ctx) {
  auto *e = (int *)workspace(ctx, kSlotSortErr, 16);
  if (e && ctx->sort_err_zeroed != e) {
    cudaMemsetAsync(e, 0, 16, ctx->stream);
    ctx->sort_err_zeroed = e;
  }
  return e;
}

// Reads the give-up word back (synchronises the stream): APSPIE_ERR_TIMEOUT
// when a sort since the last check gave up, clearing the word.
inline int radix_sort_check(apspie_context *ctx) {
  int *e = radix_sort_err(ctx);
  int *h = (int *)pinned(ctx, sizeof(int));
  if (!e || !h) return APSPIE_ERR_OOM;
  cudaMemcpyAsync(h, e, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  const cudaError_t ce = cudaStreamSynchronize(ctx->stream);
  if (ce != cudaSuccess) return check_cuda(ctx, ce, "radix sort check");
  if (*h == 0) return APSPIE_OK;
  cudaMemsetAsync(e, 0, sizeof(int), ctx->stream);
  return set_error(ctx, APSPIE_ERR_TIMEOUT, "radix sort: a look-back wait gave up");
}

// Stable sort of n (key, value) pairs on the low `bits` bits of the key
// (va == vb == nullptr sorts keys only).  Ping-pongs between (ka, va) and
// (kb, vb); *result_in_b tells where the sorted data ended up.  Scratch:
// slot kSlotSortHist (histograms, tile counters, status words).
template <typename K, typename V>
int device_radix_sort(apspie_context *ctx, K *ka, V *va, K *kb, V *vb, long long n, int bits,
                      bool *result_in_b) {
  *result_in_b = false;
  if (n <= 1 || bits <= 0) return APSPIE_OK;
  const int npass = (bits + kRadixBits - 1) / kRadixBits;
  if (npass > kMaxPasses || n >= (1ll << 40))
    return set_error(ctx, APSPIE_ERR_OVERFLOW, "radix sort: %lld keys of %d bits", n, bits);
  const long long tiles = (n + kSortTile - 1) / kSortTile;
  // [histograms: npass x 256 u64][tile counters: 8 x u32, padded; the
  // sort's give-up word at u32 15][status: tiles x 256 u64]
  const size_t hist_bytes = sizeof(unsigned long long) * kMaxPasses * kRadix;
  const size_t head = hist_bytes + 64;
  const size_t bytes = head + sizeof(unsigned long long) * (size_t)tiles * kRadix;
  int *err = radix_sort_err(ctx);
  auto *ws = (unsigned char *)workspace(ctx, kSlotSortHist, bytes);
  if (!ws || !err) return APSPIE_ERR_OOM;
  auto *ghist = (unsigned long long *)ws;
  auto *counters = (unsigned *)(ws + hist_bytes);
  auto *status = (unsigned long long *)(ws + head);
  cudaStream_t st = ctx->stream;
  // zero the histograms, counters and every status word
  cudaMemsetAsync(ws, 0, bytes, st);
  const int hgrid = (int)std::max(1ll, std::min((n + kSortThreads * 8 - 1) / (kSortThreads * 8),
                                                (long long)ctx->num_sms * 4));
  radix_histograms<K><<<hgrid, kSortThreads, 0, st>>>(ka, n, npass, ghist);
  radix_digit_offsets<kRadix><<<1, kRadix, 0, st>>>(ghist, npass);
  int rc = check_launch(ctx, "radix_histograms", 2);
  if (rc) return rc;
  K *kin = ka, *kout = kb;
  V *vin = va, *vout = vb;
  const size_t vdyn = va ? sizeof(V) * kSortTile : 0;
  if (vdyn)
    cudaFuncSetAttribute(radix_onesweep<K, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)vdyn);
  for (int p = 0; p < npass; ++p) {
    radix_onesweep<K, V><<<(unsigned)tiles, kSortThreads, vdyn, st>>>(kin, vin, kout, vout, n, p,
                                                                      ghist, status, counters + p,
                                                                      err, (int *)(counters + 15));
    rc = check_launch(ctx, "radix_onesweep");
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
