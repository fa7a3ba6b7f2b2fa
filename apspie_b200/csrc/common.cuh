// common.cuh -- shared device primitives for the apspie_b200 kernels (sm_100a).
//
// Warp-level scan / compaction, warp-aggregated queue append and a bounded
// software grid barrier for the persistent traversal kernels.  Every spin in
// this library has an iteration cap: on timeout it records APSPIE_ERR_TIMEOUT
// in the kernel's status word and the kernel returns.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "apspie.h"

namespace apspie {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_in_block() { return threadIdx.x >> 5; }

// Inclusive warp scan (Kogge-Stone over shuffles).
template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T n = __shfl_up_sync(kFull, v, o);
    if (lane_id() >= o) v += n;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Largest lane j with excl[j] <= e, for a non-decreasing per-lane excl.
// Used to map a flat edge index back to its owner vertex inside a warp.
__device__ __forceinline__ int warp_owner(int excl, int e) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    int probe = lo + step;
    int val = __shfl_sync(kFull, excl, probe & 31);
    if (probe <= 31 && val <= e) lo = probe;
  }
  return lo;
}

// Warp-aggregated append of the lanes with pred set: one atomicAdd per warp.
// Returns this lane's slot (undefined where pred is false).
__device__ __forceinline__ unsigned warp_append(bool pred, unsigned *counter) {
  unsigned mask = __ballot_sync(kFull, pred);
  unsigned base = 0;
  int leader = __ffs(mask) - 1;
  if (mask && lane_id() == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
  base = __shfl_sync(kFull, base, leader < 0 ? 0 : leader);
  return base + __popc(mask & ((1u << lane_id()) - 1u));
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Relaxed 64-bit load at gpu scope: several can be in flight at once (an
// acquire load orders the loads after it), for a word whose value is all
// the reader needs.
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier for cooperatively launched kernels, on one 64-bit arrival
// counter that only grows (bar must be 8-byte aligned and zero at launch):
// the k-th barrier of every block waits until the counter reaches
// k * nblocks, so the last block to arrive has nothing left to do and the
// others see the release as soon as its arrival lands.  Returns false (and
// sets *err = APSPIE_ERR_TIMEOUT) if the other blocks do not arrive within
// kSpinLimit polls; the caller must then leave the kernel.
constexpr unsigned kSpinLimit = 1u << 24;

// Grid-wide barrier of a co-resident (cooperative) grid on a monotonic
// 64-bit arrival counter: after the block's barrier, thread 0 arrives with
// a release add (cumulative over the block's writes, ordered before it by
// the block barrier) and polls with acquire loads until the generation's
// last block has arrived; the block barrier after it publishes that to
// the block.  Release/acquire instead of two full fences measured about
// 0.25 us less per barrier (1.35 vs 1.6 us, 444 blocks on a B200).  The
// poll gives up after kSpinLimit rounds, or when another block has flagged
// an error (checked every 256 rounds), and reports APSPIE_ERR_TIMEOUT.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long *ctr = reinterpret_cast<unsigned long long *>(bar);
    const unsigned long long nblocks = gridDim.x * gridDim.y * gridDim.z;
    unsigned long long arrived;
    asm volatile("atom.add.release.gpu.global.u64 %0, [%1], 1;"
                 : "=l"(arrived) : "l"(ctr) : "memory");
    const unsigned long long target = (arrived / nblocks + 1) * nblocks;
    int ok = 1;
    unsigned spins = 0;
    while (ld_acquire64(ctr) < target) {
      if (++spins > kSpinLimit || ((spins & 255u) == 0u && *(volatile int *)err != 0)) {
        atomicCAS(err, 0, (int)APSPIE_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace apspie
