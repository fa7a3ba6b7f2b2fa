// debug.cu -- test hooks for the failure paths of the bounded device waits.
//
// Every device-side wait in the library (the persistent kernels' grid
// barrier, the radix sort's look-back) gives up after a bounded number of
// polls and reports APSPIE_ERR_TIMEOUT.  These hooks make such a wait run
// out on purpose, without a fault, a trap or an unbounded wait: a block
// that leaves a persistent launch before its first grid barrier (the other
// blocks' arrival count never completes), or the first tile of a radix sort
// that withholds its look-back status (its successors never see it).  A
// third hook fails the next workspace allocation on the host, for the
// out-of-memory path.  Each hook is one-shot.  They exist for the tests of
// the failure paths.
#include <cuda_runtime.h>

#include "context.h"
#include "primitives.cuh"

namespace apspie {
int bfs_inject(apspie_context *ctx);
namespace {
__global__ void debug_set_word(int *p, int v) { *p = v; }
}  // namespace
}  // namespace apspie

using namespace apspie;

extern "C" int apspie_debug_inject(apspie_ctx ctx, int what) {
  switch (what) {
    case APSPIE_INJECT_BFS_BARRIER:
      if (ctx) APSPIE_CHECK_CTX(ctx);
      return bfs_inject(ctx);
    case APSPIE_INJECT_SORT_LOOKBACK: {
      if (!ctx) return APSPIE_ERR_INVALID;
      APSPIE_CHECK_CTX(ctx);
      int *err = radix_sort_err(ctx);
      if (!err) return APSPIE_ERR_OOM;
      debug_set_word<<<1, 1, 0, ctx->stream>>>(err + 1, 1);
      return check_launch(ctx, "apspie_debug_inject");
    }
    case APSPIE_INJECT_ALLOC_FAIL:
      if (!ctx) return APSPIE_ERR_INVALID;
      ctx->fail_next_alloc = true;
      return APSPIE_OK;
    default:
      return ctx ? set_error(ctx, APSPIE_ERR_INVALID, "apspie_debug_inject: unknown hook %d", what)
                 : APSPIE_ERR_INVALID;
  }
}
