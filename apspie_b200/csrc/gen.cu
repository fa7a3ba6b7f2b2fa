// gen.cu -- device builder for the synthetic graphs: R-MAT and Erdos-Renyi
// edges drawn on the GPU with the same counter-based hash as the host builder
// (gen_common.h), packed as (row << bits | col), sorted with the library's
// radix sort, deduplicated and turned into CSR -- the same arrays as
// apspie_gen_*_host, bit for bit, in a fraction of the time.
//
// The reference builds its CSR on the host (makeSymmetric's qsort and
// buildMatrix's counting sort, src/util.cuh:573-643, src/matrix.cpp:56-111).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "context.h"
#include "gen_common.h"
#include "primitives.cuh"

namespace apspie {
namespace {

using namespace apspie_gen;

__global__ void rmat_keys(RmatParams P, long long samples, int symmetric, int bits,
                          unsigned long long *keys) {
  const unsigned long long pad = 1ull << (2 * bits);
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < samples;
       s += (long long)gridDim.x * blockDim.x) {
    uint32_t u, v;
    rmat_sample(P, (uint64_t)s, &u, &v);
    unsigned long long k0 = pad, k1 = pad;
    if (u != v) {
      k0 = ((unsigned long long)u << bits) | v;
      k1 = ((unsigned long long)v << bits) | u;
    }
    if (symmetric) {
      keys[2 * s] = k0;
      keys[2 * s + 1] = k1;
    } else {
      keys[s] = k0;
    }
  }
}

__global__ void er_keys(uint64_t seed, long long samples, uint32_t n, int bits,
                        unsigned long long *keys) {
  const unsigned long long pad = 1ull << (2 * bits);
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < samples;
       s += (long long)gridDim.x * blockDim.x) {
    uint32_t u, v;
    er_sample(seed, (uint64_t)s, n, &u, &v);
    unsigned long long k0 = pad, k1 = pad;
    if (u != v) {
      k0 = ((unsigned long long)u << bits) | v;
      k1 = ((unsigned long long)v << bits) | u;
    }
    keys[2 * s] = k0;
    keys[2 * s + 1] = k1;
  }
}

// keep[i] = 1 for the first of each run of equal real keys
__global__ void unique_flags(const unsigned long long *k, long long n, int bits, unsigned *flag) {
  const unsigned long long pad = 1ull << (2 * bits);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    flag[i] = (k[i] != pad && (i == 0 || k[i] != k[i - 1])) ? 1u : 0u;
}

// scatter unique keys to their rank as column indices and count each row;
// keys are sorted, so lanes of a warp mostly share a row: one atomic per
// (warp, row) group
__global__ void keys_to_csr(const unsigned long long *k, long long n, int bits, const unsigned *flag,
                            const unsigned *rank, int *row_count, int *ind) {
  const unsigned long long mask = (1ull << bits) - 1ull;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long long i = base + (threadIdx.x & 31);
    unsigned f = 0;
    unsigned row = 0xffffffffu;
    if (i < n && flag[i]) {
      unsigned long long key = k[i];
      ind[rank[i]] = (int)(key & mask);
      f = 1;
      row = (unsigned)(key >> bits);
    }
    unsigned peers = __match_any_sync(kFull, row);
    unsigned flagged = __ballot_sync(kFull, f) & peers;
    if (f && (threadIdx.x & 31) == __ffs(flagged) - 1) atomicAdd(&row_count[row], __popc(flagged));
  }
}

// edge weights as functions of (row, col, seed): one warp per row
__global__ void weights_u32_kernel(int m, const int *ptr, const int *ind, uint64_t seed,
                                   uint32_t lo, uint32_t hi, uint32_t *w) {
  const int lane = threadIdx.x & 31;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < m;
       u += (gridDim.x * blockDim.x) >> 5)
    for (int k = ptr[u] + lane; k < ptr[u + 1]; k += 32)
      w[k] = weight_u32(seed, (uint32_t)u, (uint32_t)ind[k], lo, hi);
}

__global__ void weights_f32_kernel(int m, const int *ptr, const int *ind, uint64_t seed,
                                   float *w) {
  const int lane = threadIdx.x & 31;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < m;
       u += (gridDim.x * blockDim.x) >> 5)
    for (int k = ptr[u] + lane; k < ptr[u + 1]; k += 32)
      w[k] = weight_f32(seed, (uint32_t)u, (uint32_t)ind[k]);
}

// key of edge (u -> v) for the pull-ordered in-adjacency: row v, then u's
// out-degree descending (clamped to dbits bits); value u
__global__ void pull_keys(int m, const int *ptr, const int *ind, int dbits,
                          unsigned long long *keys, int *vals) {
  const int lane = threadIdx.x & 31;
  const unsigned long long dmax = (1ull << dbits) - 1ull;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < m;
       u += (gridDim.x * blockDim.x) >> 5) {
    const int s = ptr[u], e = ptr[u + 1];
    const unsigned long long d = min((unsigned long long)(e - s), dmax);
    for (int k = s + lane; k < e; k += 32) {
      keys[k] = ((unsigned long long)ind[k] << dbits) | (dmax - d);
      vals[k] = u;
    }
  }
}

// row lengths of the sorted keys (row = key >> dbits), one atomic per run
__global__ void key_rows(const unsigned long long *k, long long n, int dbits, int *row_count) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long long i = base + (threadIdx.x & 31);
    const unsigned row = i < n ? (unsigned)(k[i] >> dbits) : 0xffffffffu;
    const unsigned peers = __match_any_sync(kFull, row);
    if (i < n && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&row_count[row], __popc(peers));
  }
}

// key of edge k = (row u -> col ind[k]) for the transpose: (col, row); value k
__global__ void transpose_keys(int m, const int *ptr, const int *ind, int rbits,
                               unsigned long long *keys, int *vals) {
  const int lane = threadIdx.x & 31;
  for (int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < m;
       u += (gridDim.x * blockDim.x) >> 5)
    for (int k = ptr[u] + lane; k < ptr[u + 1]; k += 32) {
      keys[k] = ((unsigned long long)ind[k] << rbits) | (unsigned)u;
      vals[k] = k;
    }
}

__global__ void transpose_emit(long long n, int rbits, const unsigned long long *keys,
                               const int *vals, const float *val, int *tind, float *tval) {
  const unsigned long long mask = (1ull << rbits) - 1ull;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    tind[i] = (int)(keys[i] & mask);
    if (tval) tval[i] = val ? val[vals[i]] : 1.0f;
  }
}

__global__ void copy_int(long long n, const int *in, int *out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i];
}

__global__ void fill_int(int n, int v, int *p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

int gg(apspie_context *ctx, long long n, int threads = 256) {
  long long g = (n + threads - 1) / threads;
  return (int)std::max(1ll, std::min(g, (long long)ctx->num_sms * 16));
}

// sort + dedup + CSR for n packed keys in ka (kb scratch)
int keys_to_graph(apspie_context *ctx, unsigned long long *ka, unsigned long long *kb, long long n,
                  int bits, int m, apspie_csr *out) {
  cudaStream_t st = ctx->stream;
  bool in_b = false;
  int rc = device_radix_sort<unsigned long long, int>(ctx, ka, nullptr, kb, nullptr, n,
                                                      2 * bits + 1, &in_b);
  if (rc) return rc;
  rc = radix_sort_check(ctx);
  if (rc) return rc;
  unsigned long long *k = in_b ? kb : ka;
  unsigned *flag = (unsigned *)workspace(ctx, kSlotMisc2, sizeof(unsigned) * (size_t)n);
  unsigned *rank = (unsigned *)workspace(ctx, kSlotMisc3, sizeof(unsigned) * (size_t)n);
  unsigned *d_tot = (unsigned *)workspace(ctx, kSlotSmall, 64);
  if (!flag || !rank || !d_tot) return APSPIE_ERR_OOM;
  unique_flags<<<gg(ctx, n), 256, 0, st>>>(k, n, bits, flag);
  rc = check_launch(ctx, "unique_flags");
  if (rc) return rc;
  rc = device_exclusive_scan<unsigned>(ctx, flag, rank, n, d_tot);
  if (rc) return rc;
  unsigned *h = (unsigned *)pinned(ctx, 64);
  if (!h) return APSPIE_ERR_OOM;
  cudaMemcpyAsync(h, d_tot, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  rc = check_cuda(ctx, cudaStreamSynchronize(st), "keys_to_graph");
  if (rc) return rc;
  const long long nnz = h[0];
  int *ptr = nullptr, *ind = nullptr;
  cudaError_t e = cudaMalloc(&ptr, sizeof(int) * ((size_t)m + 1));
  if (e == cudaSuccess) e = cudaMalloc(&ind, sizeof(int) * (size_t)std::max(1ll, nnz));
  if (e != cudaSuccess) {
    cudaFree(ptr);
    cudaFree(ind);
    return check_cuda(ctx, e, "keys_to_graph: allocating the CSR");
  }
  fill_int<<<gg(ctx, m + 1), 256, 0, st>>>(m + 1, 0, ptr);
  if (nnz > 0) keys_to_csr<<<gg(ctx, n), 256, 0, st>>>(k, n, bits, flag, rank, ptr, ind);
  rc = check_launch(ctx, "keys_to_csr");
  // row counts -> offsets (the scan total lands in ptr[m])
  if (!rc) rc = device_exclusive_scan<int>(ctx, ptr, ptr, (long long)m + 1, nullptr);
  if (rc) {
    cudaFree(ptr);
    cudaFree(ind);
    return rc;
  }
  out->m = m;
  out->n = m;
  out->nnz = nnz;
  out->d_ptr = ptr;
  out->d_ind = ind;
  out->d_val = nullptr;
  return APSPIE_OK;
}

}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" {

int apspie_gen_rmat_device(apspie_ctx ctx, int scale, int edge_factor, uint64_t seed,
                           int symmetric, int scramble, apspie_csr *out) {
  APSPIE_CHECK_CTX(ctx);
  if (scale < 1 || scale > 30 || edge_factor < 1 || !out)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_gen_rmat_device: bad arguments");
  const long long samples = (long long)edge_factor << scale;
  const long long n = samples * (symmetric ? 2 : 1);
  auto *ka = (unsigned long long *)workspace(ctx, kSlotSortKeysA, sizeof(unsigned long long) * (size_t)n);
  auto *kb = (unsigned long long *)workspace(ctx, kSlotSortKeysB, sizeof(unsigned long long) * (size_t)n);
  if (!ka || !kb) return APSPIE_ERR_OOM;
  RmatParams P = rmat_params(scale, seed, scramble != 0);
  rmat_keys<<<gg(ctx, samples), 256, 0, ctx->stream>>>(P, samples, symmetric, scale, ka);
  int rc = check_launch(ctx, "rmat_keys");
  if (rc) return rc;
  return keys_to_graph(ctx, ka, kb, n, scale, 1 << scale, out);
}

int apspie_gen_er_device(apspie_ctx ctx, int n, int mean_degree, uint64_t seed, apspie_csr *out) {
  APSPIE_CHECK_CTX(ctx);
  if (n < 2 || mean_degree < 1 || !out)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_gen_er_device: bad arguments");
  const long long samples = (long long)n * mean_degree / 2;
  const long long nk = 2 * samples;
  int bits = bits_for(n);
  auto *ka = (unsigned long long *)workspace(ctx, kSlotSortKeysA, sizeof(unsigned long long) * (size_t)nk);
  auto *kb = (unsigned long long *)workspace(ctx, kSlotSortKeysB, sizeof(unsigned long long) * (size_t)nk);
  if (!ka || !kb) return APSPIE_ERR_OOM;
  er_keys<<<gg(ctx, samples), 256, 0, ctx->stream>>>(mix64(seed ^ 0x45524552ull), samples,
                                                      (uint32_t)n, bits, ka);
  int rc = check_launch(ctx, "er_keys");
  if (rc) return rc;
  return keys_to_graph(ctx, ka, kb, nk, bits, n, out);
}

int apspie_bfs_prepare(apspie_ctx ctx, int m, int64_t nnz, const int *d_ptr, const int *d_ind,
                       int *d_tptr, int *d_tind) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || nnz < 0 || nnz >= (int64_t)INT32_MAX || !d_ptr || !d_tptr ||
      (nnz > 0 && (!d_ind || !d_tind)))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_bfs_prepare: bad arguments");
  cudaStream_t st = ctx->stream;
  fill_int<<<gg(ctx, m + 1), 256, 0, st>>>(m + 1, 0, d_tptr);
  int rc = check_launch(ctx, "fill_int");
  if (rc || nnz == 0) return rc;
  const int vbits = bits_for(m);
  const int dbits = std::min(24, 63 - vbits);
  auto *ka = (unsigned long long *)workspace(ctx, kSlotSortKeysA, 8 * (size_t)nnz);
  auto *kb = (unsigned long long *)workspace(ctx, kSlotSortKeysB, 8 * (size_t)nnz);
  auto *va = (int *)workspace(ctx, kSlotSortValsA, 4 * (size_t)nnz);
  auto *vb = (int *)workspace(ctx, kSlotSortValsB, 4 * (size_t)nnz);
  if (!ka || !kb || !va || !vb) return APSPIE_ERR_OOM;
  pull_keys<<<gg(ctx, (long long)m * 32), 256, 0, st>>>(m, d_ptr, d_ind, dbits, ka, va);
  rc = check_launch(ctx, "pull_keys");
  if (rc) return rc;
  bool in_b = false;
  rc = device_radix_sort<unsigned long long, int>(ctx, ka, va, kb, vb, nnz, vbits + dbits, &in_b);
  if (rc) return rc;
  rc = radix_sort_check(ctx);  // before the sorted keys index anything
  if (rc) return rc;
  const unsigned long long *k = in_b ? kb : ka;
  const int *v = in_b ? vb : va;
  key_rows<<<gg(ctx, nnz), 256, 0, st>>>(k, nnz, dbits, d_tptr);
  copy_int<<<gg(ctx, nnz), 256, 0, st>>>(nnz, v, d_tind);
  rc = check_launch(ctx, "key_rows", 2);
  if (rc) return rc;
  return device_exclusive_scan<int>(ctx, d_tptr, d_tptr, (long long)m + 1, nullptr);
}

int apspie_csr_transpose(apspie_ctx ctx, int m, int n, int64_t nnz, const int *d_ptr,
                         const int *d_ind, const float *d_val, int *d_tptr, int *d_tind,
                         float *d_tval) {
  APSPIE_CHECK_CTX(ctx);
  if (m <= 0 || n <= 0 || nnz < 0 || nnz >= (int64_t)INT32_MAX || !d_ptr || !d_tptr ||
      (nnz > 0 && (!d_ind || !d_tind)))
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_csr_transpose: bad arguments");
  cudaStream_t st = ctx->stream;
  fill_int<<<gg(ctx, (long long)n + 1), 256, 0, st>>>(n + 1, 0, d_tptr);
  int rc = check_launch(ctx, "fill_int");
  if (rc || nnz == 0) return rc;
  const int rbits = std::max(1, bits_for(m)), cbits = std::max(1, bits_for(n));
  auto *ka = (unsigned long long *)workspace(ctx, kSlotSortKeysA, 8 * (size_t)nnz);
  auto *kb = (unsigned long long *)workspace(ctx, kSlotSortKeysB, 8 * (size_t)nnz);
  auto *va = (int *)workspace(ctx, kSlotSortValsA, 4 * (size_t)nnz);
  auto *vb = (int *)workspace(ctx, kSlotSortValsB, 4 * (size_t)nnz);
  if (!ka || !kb || !va || !vb) return APSPIE_ERR_OOM;
  transpose_keys<<<gg(ctx, (long long)m * 32), 256, 0, st>>>(m, d_ptr, d_ind, rbits, ka, va);
  rc = check_launch(ctx, "transpose_keys");
  if (rc) return rc;
  // rows within a column come out ascending: the keys hold them, and the
  // sort only needs the column bits above them (stable LSD on all bits)
  bool in_b = false;
  rc = device_radix_sort<unsigned long long, int>(ctx, ka, va, kb, vb, nnz, rbits + cbits, &in_b);
  if (rc) return rc;
  rc = radix_sort_check(ctx);  // before the sorted keys index anything
  if (rc) return rc;
  const unsigned long long *k = in_b ? kb : ka;
  const int *v = in_b ? vb : va;
  key_rows<<<gg(ctx, nnz), 256, 0, st>>>(k, nnz, rbits, d_tptr);
  transpose_emit<<<gg(ctx, nnz), 256, 0, st>>>(nnz, rbits, k, v, d_val, d_tind, d_tval);
  rc = check_launch(ctx, "transpose_emit", 2);
  if (rc) return rc;
  return device_exclusive_scan<int>(ctx, d_tptr, d_tptr, (long long)n + 1, nullptr);
}

int apspie_gen_weights_u32_device(apspie_ctx ctx, int m, const int *d_ptr, const int *d_ind,
                                  uint64_t seed, uint32_t lo, uint32_t hi, uint32_t *d_w) {
  APSPIE_CHECK_CTX(ctx);
  if (m < 0 || !d_ptr || !d_w || hi < lo)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_gen_weights_u32_device: bad arguments");
  if (m == 0) return APSPIE_OK;
  weights_u32_kernel<<<gg(ctx, (long long)m * 32), 256, 0, ctx->stream>>>(m, d_ptr, d_ind, seed, lo,
                                                                         hi, d_w);
  return check_launch(ctx, "weights_u32_kernel");
}

int apspie_gen_weights_f32_device(apspie_ctx ctx, int m, const int *d_ptr, const int *d_ind,
                                  uint64_t seed, float *d_w) {
  APSPIE_CHECK_CTX(ctx);
  if (m < 0 || !d_ptr || !d_w)
    return set_error(ctx, APSPIE_ERR_INVALID, "apspie_gen_weights_f32_device: bad arguments");
  if (m == 0) return APSPIE_OK;
  weights_f32_kernel<<<gg(ctx, (long long)m * 32), 256, 0, ctx->stream>>>(m, d_ptr, d_ind, seed,
                                                                         d_w);
  return check_launch(ctx, "weights_f32_kernel");
}

}  // extern "C"

namespace apspie {
namespace {
__global__ void gather_offsets_kernel(const int *__restrict__ ptr, int m, int *out) {
  const int i = threadIdx.x;
  if (i <= 64) out[i] = ptr[(size_t)((int64_t)m * i / 64)];
}
}  // namespace

int gather_offsets(apspie_context *ctx, const int *d_ptr, int m, int *d_out) {
  gather_offsets_kernel<<<1, 96, 0, ctx->stream>>>(d_ptr, m, d_out);
  return check_launch(ctx, "gather_offsets");
}
}  // namespace apspie
