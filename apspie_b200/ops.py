"""Device entry points: thin wrappers that pass torch tensors' device
pointers to the C ABI.  Argument meaning follows the reference's functions
(cited on each wrapper)."""
from __future__ import annotations

import ctypes as C

from ._native import BfsStats, check, lib


class Context:
    """An apspie context on one device and stream (mgpu::CudaContext
    stand-in, test/bfs/main.cu:27).  stream=None uses torch's current stream
    at construction time."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream(device)
        handle = stream if isinstance(stream, int) else stream.cuda_stream
        self.device = device
        self._h = C.c_void_p()
        check(lib.apspie_ctx_create(device, C.c_void_p(handle), C.byref(self._h)),
              what="apspie_ctx_create")

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise RuntimeError("context closed")
        return self._h

    def set_stream(self, stream) -> None:
        handle = stream if isinstance(stream, int) else stream.cuda_stream
        check(lib.apspie_ctx_set_stream(self.handle, C.c_void_p(handle)), self.handle)

    def sync(self) -> None:
        check(lib.apspie_ctx_sync(self.handle), self.handle, "sync")

    @property
    def launches(self) -> int:
        v = C.c_uint64()
        check(lib.apspie_ctx_launch_count(self.handle, C.byref(v)), self.handle)
        return int(v.value)

    @property
    def workspace_bytes(self) -> int:
        v = C.c_size_t()
        check(lib.apspie_ctx_workspace_bytes(self.handle, C.byref(v)), self.handle)
        return int(v.value)

    def close(self) -> None:
        if self._h is not None:
            lib.apspie_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _p(t) -> C.c_void_p:
    return C.c_void_p(0 if t is None else t.data_ptr())


def bfs(ctx: Context, g, src: int, depth=None, max_levels: int = 0):
    """bfs<T>() (src/bfs.cuh:33): int32 depth per vertex, -1 unreached."""
    import torch
    if depth is None:
        depth = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
    check(lib.apspie_bfs(ctx.handle, int(src), int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind),
                         _p(depth), int(max_levels)), ctx.handle, "apspie_bfs")
    return depth


def bfs_stats(ctx: Context) -> dict:
    s = BfsStats()
    check(lib.apspie_bfs_get_stats(ctx.handle, C.byref(s)), ctx.handle, "apspie_bfs_get_stats")
    return {"levels": s.levels, "pull_levels": s.pull_levels,
            "vertices_reached": s.vertices_reached, "edges_traversed": s.edges_traversed}


def bfs_set_params(ctx: Context, alpha: int = 14, beta: int = 24, mode: int = 0) -> None:
    """Direction-switch thresholds; mode 0 auto, 1 push only, 2 pull only."""
    check(lib.apspie_bfs_set_params(ctx.handle, alpha, beta, mode), ctx.handle,
          "apspie_bfs_set_params")
