// context.cpp -- apspie_ctx lifetime, workspace slots and error reporting.
#include "context.h"

#include <cstdarg>
#include <cstdlib>
#include <map>
#include <mutex>

namespace apspie {

int set_error(apspie_context *ctx, int status, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->last_error = buf;
  }
  return status;
}

int check_cuda(apspie_context *ctx, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return APSPIE_OK;
  int st = (e == cudaErrorMemoryAllocation) ? APSPIE_ERR_OOM : APSPIE_ERR_CUDA;
  return set_error(ctx, st, "%s: %s", what, cudaGetErrorString(e));
}

int check_launch(apspie_context *ctx, const char *what, int nlaunches) {
  ctx->launches += (uint64_t)nlaunches;
  return check_cuda(ctx, cudaGetLastError(), what);
}

void *workspace(apspie_context *ctx, int id, size_t bytes) {
  if (id < 0) return nullptr;
  if ((size_t)id >= ctx->slots.size()) ctx->slots.resize(id + 1);
  auto &s = ctx->slots[id];
  if (bytes == 0) bytes = 16;
  if (s.bytes >= bytes) return s.ptr;
  if (ctx->fail_next_alloc) {
    // test hook: this growth fails as a cudaMalloc that ran out of memory
    ctx->fail_next_alloc = false;
    set_error(ctx, APSPIE_ERR_OOM, "workspace slot %d: allocation failure injected", id);
    return nullptr;
  }
  if (s.ptr) {
    // the stream may still use the old buffer
    cudaStreamSynchronize(ctx->stream);
    cudaFree(s.ptr);
    s.ptr = nullptr;
    s.bytes = 0;
  }
  size_t want = (bytes + 255) & ~size_t(255);
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(ctx, APSPIE_ERR_OOM, "workspace slot %d: cudaMalloc(%zu) failed: %s",
              id, want, cudaGetErrorString(e));
    return nullptr;
  }
  s.ptr = p;
  s.bytes = want;
  return p;
}

void *pinned(apspie_context *ctx, size_t bytes) {
  if (ctx->pinned_bytes >= bytes) return ctx->pinned;
  if (ctx->pinned) {
    cudaStreamSynchronize(ctx->stream);  // copies may still read the old buffer
    cudaFreeHost(ctx->pinned);
  }
  ctx->pinned = nullptr;
  ctx->pinned_bytes = 0;
  size_t want = bytes < 4096 ? 4096 : bytes;
  if (cudaMallocHost(&ctx->pinned, want) != cudaSuccess) {
    cudaGetLastError();
    ctx->pinned = nullptr;
    set_error(ctx, APSPIE_ERR_OOM, "cudaMallocHost(%zu) failed", want);
    return nullptr;
  }
  ctx->pinned_bytes = want;
  return ctx->pinned;
}

}  // namespace apspie

using namespace apspie;

namespace apspie {

uint64_t graph_fingerprint(apspie_context *ctx, int m, int64_t nnz, const int *d_ptr) {
  // offsets sampled at 64 evenly spaced rows (plus the last), gathered on
  // the device and read back in one copy
  uint64_t f = 1469598103934665603ull ^ ((uint64_t)m << 32) ^ (uint64_t)nnz;
  int *h = (int *)pinned(ctx, sizeof(int) * 65);
  int *d = (int *)workspace(ctx, kSlotFingerprint, sizeof(int) * 65);
  if (!h || !d || gather_offsets(ctx, d_ptr, m, d) != APSPIE_OK) {
    cudaGetLastError();
    return f;
  }
  cudaMemcpyAsync(h, d, sizeof(int) * 65, cudaMemcpyDeviceToHost, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  for (int i = 0; i <= 64; ++i) f = (f ^ (uint64_t)(uint32_t)h[i]) * 1099511628211ull;
  return f;
}

int occupancy_grid(apspie_context *ctx, const void *kernel, int threads) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kernel, ctx->device);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, 0) != cudaSuccess ||
      occ < 1) {
    cudaGetLastError();
    return 0;
  }
  return cache[key] = occ * ctx->num_sms;
}

void *upload_buffer(apspie_context *ctx, size_t bytes, int *slot) {
  const int k = ctx->up_next;
  ctx->up_next = (k + 1) % apspie_context::kUploadRing;
  if (ctx->up_done[k]) {
    // the copy that last read this buffer
    cudaError_t e = cudaEventSynchronize(ctx->up_done[k]);
    if (e != cudaSuccess) {
      check_cuda(ctx, e, "upload buffer");
      return nullptr;
    }
  } else if (cudaEventCreateWithFlags(&ctx->up_done[k], cudaEventDisableTiming) != cudaSuccess) {
    check_cuda(ctx, cudaGetLastError(), "upload buffer event");
    return nullptr;
  }
  // the ring's buffers come from one pinned pool, allocated at first use
  // (pinned allocations are slow: none happens on a later call)
  if (!ctx->up_pool) {
    if (cudaMallocHost(&ctx->up_pool, apspie_context::kUploadBytes *
                                          apspie_context::kUploadRing) != cudaSuccess) {
      cudaGetLastError();
      ctx->up_pool = nullptr;
      set_error(ctx, APSPIE_ERR_OOM, "cudaMallocHost of the upload ring failed");
      return nullptr;
    }
  }
  *slot = k;
  if (bytes <= apspie_context::kUploadBytes)
    return (char *)ctx->up_pool + (size_t)k * apspie_context::kUploadBytes;
  if (ctx->up_bytes[k] < bytes) {  // larger than a pool buffer: its own
    if (ctx->up_host[k]) cudaFreeHost(ctx->up_host[k]);
    ctx->up_host[k] = nullptr;
    ctx->up_bytes[k] = 0;
    if (cudaMallocHost(&ctx->up_host[k], bytes) != cudaSuccess) {
      cudaGetLastError();
      ctx->up_host[k] = nullptr;
      set_error(ctx, APSPIE_ERR_OOM, "cudaMallocHost(%zu) failed", bytes);
      return nullptr;
    }
    ctx->up_bytes[k] = bytes;
  }
  return ctx->up_host[k];
}

int upload_done(apspie_context *ctx, int slot) {
  return check_cuda(ctx, cudaEventRecord(ctx->up_done[slot], ctx->stream), "upload event");
}

}  // namespace apspie

extern "C" {

int apspie_ctx_create(int device, void *stream, apspie_ctx *out) {
  return api_guard([&]() -> int {
    if (!out) return APSPIE_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
      cudaGetLastError();
      return APSPIE_ERR_INVALID;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
      cudaGetLastError();
      return APSPIE_ERR_CUDA;
    }
    auto *ctx = new (std::nothrow) apspie_context();
    if (!ctx) return APSPIE_ERR_OOM;
    ctx->device = device;
    ctx->stream = (cudaStream_t)stream;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    ctx->slots.resize(kSlotCount);
    *out = ctx;
    return APSPIE_OK;
  });
}

int apspie_ctx_destroy(apspie_ctx ctx) {
  if (!ctx) return APSPIE_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (apspie_context *sub : ctx->subs) apspie_ctx_destroy(sub);
  for (cudaEvent_t ev : ctx->sub_done) cudaEventDestroy(ev);
  if (ctx->aux_done) cudaEventDestroy(ctx->aux_done);
  for (auto &s : ctx->slots)
    if (s.ptr) cudaFree(s.ptr);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  for (int k = 0; k < apspie_context::kUploadRing; ++k) {
    if (ctx->up_host[k]) cudaFreeHost(ctx->up_host[k]);
    if (ctx->up_done[k]) cudaEventDestroy(ctx->up_done[k]);
  }
  if (ctx->up_pool) cudaFreeHost(ctx->up_pool);
  if (ctx->owns_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return APSPIE_OK;
}

int apspie_ctx_set_max_grid(apspie_ctx ctx, int blocks) {
  if (!ctx || blocks < 0) return APSPIE_ERR_INVALID;
  ctx->max_grid = blocks;
  return APSPIE_OK;
}

int apspie_batch_set_params(apspie_ctx ctx, int deep_blocks) {
  if (!ctx || deep_blocks < 0) return APSPIE_ERR_INVALID;
  ctx->deep_blocks = deep_blocks;
  return APSPIE_OK;
}

int apspie_batch_set_sssp_pull(apspie_ctx ctx, int alpha) {
  if (!ctx || alpha < 0) return APSPIE_ERR_INVALID;
  ctx->sssp_pull_alpha_batch = alpha;
  return APSPIE_OK;
}

int apspie_batch_set_deep_mode(apspie_ctx ctx, int max_concurrent) {
  if (!ctx || max_concurrent < 0 || max_concurrent > 64) return APSPIE_ERR_INVALID;
  ctx->batch_deep_subs = max_concurrent;
  return APSPIE_OK;
}

int apspie_spgemm_set_params(apspie_ctx ctx, int64_t bitmap_max_cols) {
  if (!ctx || bitmap_max_cols < 0) return APSPIE_ERR_INVALID;
  ctx->spgemm_bitmap_max_cols = bitmap_max_cols;
  return APSPIE_OK;
}

int apspie_ctx_resident_blocks(apspie_ctx ctx, int *blocks) {
  if (!ctx || !blocks) return APSPIE_ERR_INVALID;
  *blocks = 2 * ctx->num_sms;  // 512-thread persistent blocks: two per SM fit every kernel
  return APSPIE_OK;
}

int apspie_ctx_set_stream(apspie_ctx ctx, void *stream) {
  if (!ctx) return APSPIE_ERR_INVALID;
  ctx->stream = (cudaStream_t)stream;
  return APSPIE_OK;
}

int apspie_ctx_sync(apspie_ctx ctx) {
  APSPIE_CHECK_CTX(ctx);
  return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
}

int apspie_ctx_launch_count(apspie_ctx ctx, uint64_t *out) {
  if (!ctx || !out) return APSPIE_ERR_INVALID;
  *out = ctx->launches;
  return APSPIE_OK;
}

int apspie_ctx_workspace_bytes(apspie_ctx ctx, size_t *out) {
  if (!ctx || !out) return APSPIE_ERR_INVALID;
  size_t t = 0;
  for (auto &s : ctx->slots) t += s.bytes;
  for (apspie_context *sub : ctx->subs)
    if (sub)
      for (auto &s : sub->slots) t += s.bytes;
  *out = t;
  return APSPIE_OK;
}

const char *apspie_last_error(apspie_ctx ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

const char *apspie_status_string(int status) {
  switch (status) {
    case APSPIE_OK: return "ok";
    case APSPIE_ERR_INVALID: return "invalid argument";
    case APSPIE_ERR_OOM: return "out of memory";
    case APSPIE_ERR_CUDA: return "CUDA error";
    case APSPIE_ERR_TIMEOUT: return "device-side wait timed out";
    case APSPIE_ERR_OVERFLOW: return "result exceeds int32 layout";
    case APSPIE_ERR_UNSUPPORTED: return "unsupported";
    case APSPIE_ERR_BUSY: return "busy";
    case APSPIE_ERR_TOO_LARGE: return "input exceeds the fixed scratch size";
    default: return "unknown status";
  }
}

}  // extern "C"
