"""Device entry points: thin wrappers that pass torch tensors' device
pointers to the C ABI.  Argument meaning follows the reference's functions
(cited on each wrapper)."""
from __future__ import annotations

import ctypes as C

from ._native import BatchStats, BfsStats, Csr, Job, SsspStats, Tuning, check, lib


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
    """Device pointer of a tensor for the C ABI (0 for None).  The kernels
    read a tensor's storage as one dense array in device memory, so a host
    tensor or a strided view is refused here, before anything is launched."""
    if t is None:
        return C.c_void_p(0)
    if not t.is_cuda:
        raise ValueError(f"apspie_b200: expected a CUDA tensor, got one on {t.device}")
    if not t.is_contiguous():
        raise ValueError("apspie_b200: expected a contiguous tensor, got a strided view")
    return C.c_void_p(t.data_ptr())


def _row(t, n: int, what: str):
    """A caller's per-vertex tensor: at least n entries of 32 bits (the
    kernels read or write n of them)."""
    if t is not None and (t.numel() < n or t.element_size() != 4):
        raise ValueError(f"{what}: needs {n} 32-bit entries, got {t.numel()} of "
                         f"{t.element_size()} bytes")
    return t


def _graph(g):
    """A device graph's arrays hold what m and nnz promise (m + 1 offsets,
    nnz indices, 32-bit entries)."""
    _row(g.ptr, g.m + 1, "graph row offsets")
    if g.nnz > 0:
        _row(g.ind, g.nnz, "graph column indices")
    return g


def bfs(ctx: Context, g, src: int, depth=None, max_levels: int = 0):
    """bfs<T>() (src/bfs.cuh:33): int32 depth per vertex, -1 unreached.
    The pull direction uses g.tptr / g.tind (in-adjacency): the same arrays
    for a symmetric graph; a directed graph without them is traversed by
    push only."""
    import torch
    _graph(g)
    if depth is None:
        depth = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
    _row(depth, g.m, "depth")
    if getattr(g, "tptr", None) is not None:
        tptr, tind = g.tptr, g.tind
    else:
        tptr, tind = (g.ptr, g.ind) if g.symmetric else (None, None)
    check(lib.apspie_bfs(ctx.handle, int(src), int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind),
                         _p(tptr), _p(tind), _p(depth), int(max_levels)), ctx.handle,
          "apspie_bfs")
    return depth


def csr_transpose(ctx: Context, m: int, n: int, ptr, ind, val=None):
    """CSC of an m x n CSR on the device (apspie_csr_transpose): returns
    (tptr, tind, tval) tensors, row ids ascending within each column."""
    import torch
    dev = ptr.device
    nnz = int(ind.numel())
    _row(ptr, m + 1, "row offsets")
    _row(val, nnz, "values")
    tptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    tind = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    tval = torch.empty(max(nnz, 1), dtype=torch.float32, device=dev)
    check(lib.apspie_csr_transpose(ctx.handle, int(m), int(n), nnz, _p(ptr), _p(ind), _p(val),
                                   _p(tptr), _p(tind), _p(tval)), ctx.handle,
          "apspie_csr_transpose")
    return tptr, tind[:nnz], tval[:nnz]


def bfs_prepare(ctx: Context, g):
    """Pull-ordered in-adjacency of g (apspie_bfs_prepare): sets g.tptr /
    g.tind, which bfs() then pulls over."""
    import torch
    _graph(g)
    dev = g.ptr.device
    tptr = torch.empty(g.m + 1, dtype=torch.int32, device=dev)
    tind = torch.empty(max(g.nnz, 1), dtype=torch.int32, device=dev)
    check(lib.apspie_bfs_prepare(ctx.handle, int(g.m), int(g.nnz), _p(g.ptr), _p(g.ind),
                                 _p(tptr), _p(tind)), ctx.handle, "apspie_bfs_prepare")
    g.tptr, g.tind = tptr, tind[:g.nnz]
    return g


def bfs_trace(ctx: Context, max_levels: int = 64) -> list[dict]:
    """Per-level direction, frontier size / edges and device ns of the last BFS."""
    import numpy as np
    mode = np.zeros(max_levels, np.int32)
    nf = np.zeros(max_levels, np.int64)
    mf = np.zeros(max_levels, np.int64)
    ns = np.zeros(max_levels, np.int64)
    qd = np.zeros(max_levels, np.int64)
    ex = np.zeros(max_levels, np.int64)
    wf = np.zeros(max_levels, np.int64)
    wl = np.zeros(max_levels, np.int64)
    cnt = C.c_int()
    check(lib.apspie_bfs_get_trace(ctx.handle, max_levels, C.byref(cnt), mode.ctypes.data,
                                   nf.ctypes.data, mf.ctypes.data, ns.ctypes.data,
                                   qd.ctypes.data, ex.ctypes.data, wf.ctypes.data,
                                   wl.ctypes.data), ctx.handle, "apspie_bfs_get_trace")
    n = cnt.value
    return [{"level": i, "dir": "pull" if mode[i] == 2 else "push", "frontier": int(nf[i]),
             "frontier_edges": int(mf[i]), "us": ns[i] / 1e3, "queued": int(qd[i]),
             "expanded": int(ex[i]), "work_first_us": wf[i] / 1e3, "work_last_us": wl[i] / 1e3}
            for i in range(n)]


def bfs_stats(ctx: Context) -> dict:
    s = BfsStats()
    check(lib.apspie_bfs_get_stats(ctx.handle, C.byref(s)), ctx.handle, "apspie_bfs_get_stats")
    return {"levels": s.levels, "pull_levels": s.pull_levels,
            "vertices_reached": s.vertices_reached, "edges_traversed": s.edges_traversed}


def bfs_set_params(ctx: Context, alpha: int = 14, beta: int = 24, mode: int = 0) -> None:
    """Direction-switch thresholds; mode 0 auto, 1 push only, 2 pull only."""
    check(lib.apspie_bfs_set_params(ctx.handle, alpha, beta, mode), ctx.handle,
          "apspie_bfs_set_params")


def sssp(ctx: Context, g, src: int, dist=None, weights: str = "u32", max_rounds: int = 0):
    """sssp<V>() (src/sssp.cuh:28): min-plus SpMSpV to convergence.
    weights "u32" uses g.w_u32 and returns int32-viewed uint32 distances
    (0xFFFFFFFF unreached); "f32" uses g.w_f32 and returns float32 (+inf)."""
    import torch
    if weights == "u32":
        if dist is None:
            dist = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
        fn, w = lib.apspie_sssp_u32, g.w_u32
    elif weights == "f32":
        if dist is None:
            dist = torch.empty(g.m, dtype=torch.float32, device=g.ptr.device)
        fn, w = lib.apspie_sssp_f32, g.w_f32
    else:
        raise ValueError(weights)
    if w is None:
        raise ValueError(f"graph has no {weights} weights")
    _graph(g)
    _row(dist, g.m, "dist")
    _row(w, g.nnz, f"{weights} weights")
    tin = g.extra.get("sssp_in", {}).get(weights)
    if tin is not None:
        # in-adjacency with its weights from sssp_prepare: push/pull rounds
        tptr, tind, tw = tin
        pfn = lib.apspie_sssp_u32_pull if weights == "u32" else lib.apspie_sssp_f32_pull
        check(pfn(ctx.handle, int(src), int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind), _p(w),
                  _p(tptr), _p(tind), _p(tw), _p(dist), int(max_rounds)), ctx.handle,
              "apspie_sssp_pull")
        return dist
    check(fn(ctx.handle, int(src), int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind), _p(w), _p(dist),
             int(max_rounds)), ctx.handle, "apspie_sssp")
    return dist


def sssp_prepare(ctx: Context, g):
    """In-adjacency of g with its edge weights (apspie_csr_transpose, one sort
    per weight array present), kept on g; sssp() then runs push/pull rounds
    over it (apspie_sssp_*_pull)."""
    import torch
    _graph(g)
    g.extra["sssp_in"] = {}
    for kind, w in (("u32", g.w_u32), ("f32", g.w_f32)):
        if w is None:
            continue
        # the transpose moves 32-bit words: uint32 weights travel as float bits
        tptr, tind, tw = csr_transpose(ctx, g.m, g.m, g.ptr, g.ind, w.view(torch.float32))
        g.extra["sssp_in"][kind] = (tptr, tind, tw.view(torch.int32) if kind == "u32" else tw)
    return g


def sssp_set_pull(ctx: Context, alpha: int = 0) -> None:
    """Pull rounds when the frontier's out-edges * alpha exceed nnz (0: never,
    the default)."""
    check(lib.apspie_sssp_set_pull(ctx.handle, int(alpha)), ctx.handle, "apspie_sssp_set_pull")


def sssp_stats(ctx: Context) -> dict:
    s = SsspStats()
    check(lib.apspie_sssp_get_stats(ctx.handle, C.byref(s)), ctx.handle, "apspie_sssp_get_stats")
    return {"rounds": s.rounds, "phases": s.phases, "vertices_reached": s.vertices_reached,
            "edges_traversed": s.edges_traversed, "relaxations": s.relaxations}


def sssp_trace(ctx: Context, max_rounds: int = 64) -> list[dict]:
    """Per-round frontier, out-edges and device us of the last SSSP."""
    import numpy as np
    nf, mf, ns, wl = (np.zeros(max_rounds, np.int64) for _ in range(4))
    cnt = C.c_int()
    check(lib.apspie_sssp_get_trace(ctx.handle, max_rounds, C.byref(cnt), nf.ctypes.data,
                                    mf.ctypes.data, ns.ctypes.data, wl.ctypes.data), ctx.handle,
          "apspie_sssp_get_trace")
    return [{"round": i, "frontier": int(nf[i]), "frontier_edges": int(mf[i]),
             "us": ns[i] / 1e3, "work_last_us": wl[i] / 1e3} for i in range(cnt.value)]


def sssp_set_params(ctx: Context, delta_u32: int = 0, delta_f32: float = 0.0) -> None:
    """Near-far step of SSSP (0 = frontier Bellman-Ford); see
    apspie_sssp_set_params."""
    check(lib.apspie_sssp_set_params(ctx.handle, int(delta_u32), float(delta_f32)), ctx.handle,
          "apspie_sssp_set_params")


def mis(ctx: Context, g, prio, out=None, delta: float = 1.0):
    """spmspvMis<V>() (src/spmspvMis.cuh:150): int32 membership (1 / 0).
    prio: device tensor of uint32 priorities (int32 view)."""
    import torch
    _graph(g)
    _row(prio, g.m, "prio")
    if out is None:
        out = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
    _row(out, g.m, "out")
    check(lib.apspie_mis(ctx.handle, int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind), _p(prio),
                         _p(out), float(delta)), ctx.handle, "apspie_mis")
    return out


def mis_rounds(ctx: Context) -> int:
    r = C.c_int()
    check(lib.apspie_mis_get_rounds(ctx.handle, C.byref(r)), ctx.handle, "apspie_mis_get_rounds")
    return int(r.value)


def neighbor_flags(ctx: Context, g, flags, out=None):
    """spmspvCsr() (src/spmspvMis.cuh:81): 1 for out-neighbours of flagged vertices."""
    import torch
    _graph(g)
    _row(flags, g.m, "flags")
    if out is None:
        out = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
    _row(out, g.m, "out")
    check(lib.apspie_neighbor_flags(ctx.handle, int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind),
                                    _p(flags), _p(out)), ctx.handle, "apspie_neighbor_flags")
    return out


PLUS_TIMES, MIN_PLUS, MAX_TIMES, OR_AND = 0, 1, 2, 3


def spmspv(ctx: Context, semiring: int, g, xind, xval=None, val=None):
    """Sparse mXv<T>() (src/mXv.cuh:250): returns (yind, yval, expanded).
    g.ptr / g.ind list the columns of A; val (float32 tensor, nnz) or None."""
    import torch
    _graph(g)
    _row(val, g.nnz, "val")
    _row(xval, xind.numel(), "xval")
    dev = g.ptr.device
    yind = torch.empty(max(g.m, 1), dtype=torch.int32, device=dev)
    yval = torch.empty(max(g.m, 1), dtype=torch.float32, device=dev)
    n = C.c_int()
    e = C.c_int64()
    check(lib.apspie_spmspv(ctx.handle, int(semiring), int(g.m), int(g.nnz), _p(g.ptr), _p(g.ind),
                            _p(val), int(xind.numel()), _p(xind), _p(xval), _p(yind), _p(yval),
                            C.byref(n), C.byref(e)), ctx.handle, "apspie_spmspv")
    return yind[:n.value], yval[:n.value], int(e.value)


def mxv_dense(ctx: Context, semiring: int, g, x, val=None, y=None):
    """Dense mXv<T>() (src/mXv.cuh:111): returns (y, total)."""
    import torch
    _graph(g)
    _row(val, g.nnz, "val")
    _row(x, g.m, "x")
    if y is None:
        y = torch.empty(g.m, dtype=torch.float32, device=g.ptr.device)
    _row(y, g.m, "y")
    e = C.c_int64()
    check(lib.apspie_mxv_dense(ctx.handle, int(semiring), int(g.m), int(g.nnz), _p(g.ptr),
                               _p(g.ind), _p(val), _p(x), _p(y), C.byref(e)), ctx.handle,
          "apspie_mxv_dense")
    return y, int(e.value)


def spmspv_set_params(ctx: Context, sort_factor: float = 4.0) -> None:
    check(lib.apspie_spmspv_set_params(ctx.handle, float(sort_factor)), ctx.handle)


def _csr(m, n, ptr, ind, val) -> Csr:
    nnz = int(ind.numel()) if ind is not None else 0
    _row(ptr, int(m) + 1, "row offsets")
    _row(val, nnz, "values")
    return Csr(int(m), int(n), nnz, _p(ptr), _p(ind), _p(val))


def spmv(ctx: Context, m: int, ptr, ind, val, x, semiring: int = 0, y=None):
    """Dense SpMV over every row (apspie_spmv; the reference's spmv() /
    cuspmv()): y[r] = (+)_k A(r, ind[k]) (x) x[ind[k]].  val may be None
    (ones)."""
    import torch
    if y is None:
        y = torch.empty(m, dtype=torch.float32, device=ptr.device)
    nnz = int(ind.numel()) if ind is not None else 0
    _row(ptr, m + 1, "row offsets")
    _row(val, nnz, "values")
    _row(y, m, "y")
    check(lib.apspie_spmv(ctx.handle, int(semiring), int(m), nnz, _p(ptr), _p(ind), _p(val),
                          _p(x), _p(y)), ctx.handle, "apspie_spmv")
    return y


def spgemm_symbolic(ctx: Context, A, B):
    """Symbolic phase of C = A * B: returns (ptr, nnz) with ptr C's m + 1
    row offsets on the device.  The numeric phase (spgemm_numeric) must
    follow on the same context with the same A and B."""
    import torch
    a, b = _csr(*A), _csr(*B)
    ptr = torch.empty(a.m + 1, dtype=torch.int32, device=A[2].device)
    nnz = C.c_int64(0)
    check(lib.apspie_spgemm_symbolic(ctx.handle, C.byref(a), C.byref(b), _p(ptr), C.byref(nnz)),
          ctx.handle, "apspie_spgemm_symbolic")
    return ptr, int(nnz.value)


def spgemm_set_params(ctx: Context, bitmap_max_cols: int = 1 << 18):
    """Rows with more than 4096 products (2048 at table load 4) use a
    shared-memory column bitmap when B has at most bitmap_max_cols columns
    (0: always hash tables)."""
    check(lib.apspie_spgemm_set_params(ctx.handle, int(bitmap_max_cols)), ctx.handle,
          "apspie_spgemm_set_params")


def spgemm_numeric(ctx: Context, A, B, ptr, ind, val):
    """Numeric phase of C = A * B into caller buffers ind / val (nnz(C)
    entries each), stream-ordered, no synchronisation."""
    a, b = _csr(*A), _csr(*B)
    _row(ptr, a.m + 1, "C row offsets")
    check(lib.apspie_spgemm_numeric(ctx.handle, C.byref(a), C.byref(b), _p(ptr), _p(ind),
                                    _p(val)), ctx.handle, "apspie_spgemm_numeric")


def spgemm(ctx: Context, A, B):
    """C = A * B (spgemm(d_matrix*...), src/spgemm.cuh:132).  A and B are
    (m, n, ptr, ind, val) tuples of device tensors (val may be None = ones);
    returns (ptr, ind, val) tensors of C (columns ascending per row)."""
    import torch
    ptr, nnz = spgemm_symbolic(ctx, A, B)
    ind = torch.empty(max(nnz, 1), dtype=torch.int32, device=ptr.device)
    val = torch.empty(max(nnz, 1), dtype=torch.float32, device=ptr.device)
    spgemm_numeric(ctx, A, B, ptr, ind, val)
    return ptr, ind[:nnz], val[:nnz]


def _take_csr(ctx: Context, c: Csr, with_val: bool):
    """Copy a library-owned CSR into torch tensors on the context's device,
    then release it."""
    import torch
    nnz = int(c.nnz)
    try:
        dev = torch.device("cuda", ctx.device)
        ptr = torch.empty(c.m + 1, dtype=torch.int32, device=dev)
        ind = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
        val = torch.empty(max(nnz, 1), dtype=torch.float32, device=dev) if with_val else None
        check(lib.apspie_csr_copy_out(ctx.handle, C.byref(c), _p(ptr),
                                      _p(ind),
                                      _p(val if with_val else None)),
              ctx.handle, "apspie_csr_copy_out")
        ctx.sync()
    finally:
        lib.apspie_csr_free(ctx.handle, C.byref(c))
    return ptr, ind[:nnz], (val[:nnz] if with_val else None)


def gen_rmat_device(ctx: Context, scale: int, edge_factor: int = 16, seed: int = 1,
                    symmetric: bool = True, scramble: bool = True):
    """The graph of graph.gen_rmat with the same arguments, built on the
    device (apspie_gen_rmat_device); returns a DeviceGraph."""
    from .graph import DeviceGraph
    c = Csr()
    check(lib.apspie_gen_rmat_device(ctx.handle, scale, edge_factor, seed, int(symmetric),
                                     int(scramble), C.byref(c)), ctx.handle,
          "apspie_gen_rmat_device")
    ptr, ind, _ = _take_csr(ctx, c, False)
    return DeviceGraph(1 << scale, int(ind.numel()), ptr, ind,
                       name=f"rmat{scale}{'s' if symmetric else 'd'}", symmetric=symmetric)


def gen_er_device(ctx: Context, n: int, mean_degree: int = 8, seed: int = 1):
    """graph.gen_er built on the device (apspie_gen_er_device)."""
    from .graph import DeviceGraph
    c = Csr()
    check(lib.apspie_gen_er_device(ctx.handle, n, mean_degree, seed, C.byref(c)), ctx.handle,
          "apspie_gen_er_device")
    ptr, ind, _ = _take_csr(ctx, c, False)
    return DeviceGraph(n, int(ind.numel()), ptr, ind, name=f"er{n}", symmetric=True)


def weights_device(ctx: Context, g, seed: int = 7, lo: int = 1, hi: int = 255):
    """graph.weights_u32 / weights_f32 computed on the device for a
    DeviceGraph: sets g.w_u32 (uint32 bits in an int32 tensor) and g.w_f32."""
    import torch
    _graph(g)
    w = torch.empty(max(g.nnz, 1), dtype=torch.int32, device=g.ptr.device)
    wf = torch.empty(max(g.nnz, 1), dtype=torch.float32, device=g.ptr.device)
    check(lib.apspie_gen_weights_u32_device(ctx.handle, int(g.m), _p(g.ptr), _p(g.ind), seed, lo,
                                            hi, _p(w)), ctx.handle, "weights_u32_device")
    check(lib.apspie_gen_weights_f32_device(ctx.handle, int(g.m), _p(g.ptr), _p(g.ind), seed,
                                            _p(wf)), ctx.handle, "weights_f32_device")
    g.w_u32, g.w_f32 = w[:g.nnz], wf[:g.nnz]
    return g


def tc_prepare(ctx: Context, g):
    """Degree-ordered strict lower triangle of a symmetric graph:
    returns (perm, Lptr, Lind) device tensors."""
    import torch
    _graph(g)
    dev = g.ptr.device
    perm = torch.empty(g.m, dtype=torch.int32, device=dev)
    lp = torch.empty(g.m + 1, dtype=torch.int32, device=dev)
    li = torch.empty(max(1, g.nnz // 2 + 1), dtype=torch.int32, device=dev)
    n = C.c_int64()
    check(lib.apspie_tc_prepare(ctx.handle, int(g.nnz), int(g.m), _p(g.ptr), _p(g.ind), _p(perm),
                                _p(lp), _p(li), C.byref(n)), ctx.handle, "apspie_tc_prepare")
    return perm, lp, li[:n.value]


def triangle_count(ctx: Context, m: int, lptr, lind) -> int:
    """Masked hash SpGEMM (L*L).*L summed in int64 (test/tc/main.cu:243-261)."""
    _row(lptr, int(m) + 1, "L row offsets")
    out = C.c_int64()
    check(lib.apspie_tc(ctx.handle, int(m), int(lind.numel()), _p(lptr), _p(lind),
                        C.byref(out)), ctx.handle, "apspie_tc")
    return int(out.value)


JOB_BFS, JOB_SSSP_U32 = 0, 1


def batch_run(ctx: Context, jobs: list[dict], max_steps: int = 0):
    """Run many BFS / SSSP traversals on several graphs in one persistent
    launch.  Each job: {"type": "bfs" | "sssp", "graph": DeviceGraph,
    "sources": [...], optional "alpha", "beta"}.  Returns one int32 tensor of
    shape (len(sources), m) per job (SSSP: uint32 bits, 0xFFFFFFFF
    unreached)."""
    arr, outs, _keep = _job_array(jobs)
    check(lib.apspie_batch_run(ctx.handle, len(jobs), arr, int(max_steps)), ctx.handle,
          "apspie_batch_run")
    return outs


def _job_array(jobs: list[dict]):
    """The apspie_job array of a job list, the output tensors, and the host
    source arrays the array points into (kept alive by the caller)."""
    import torch
    outs, keep = [], []
    arr = (Job * len(jobs))()
    for i, jd in enumerate(jobs):
        g = _graph(jd["graph"])
        if jd["type"] == "sssp":
            _row(g.w_u32, g.nnz, "u32 weights")
        src = (C.c_int * len(jd["sources"]))(*[int(s) for s in jd["sources"]])
        keep.append(src)
        out = torch.empty((len(jd["sources"]), g.m), dtype=torch.int32, device=g.ptr.device)
        outs.append(out)
        sym = bool(getattr(g, "symmetric", False))
        tptr = None if sym else getattr(g, "tptr", None)
        tind = None if sym else getattr(g, "tind", None)
        arr[i] = Job(JOB_BFS if jd["type"] == "bfs" else JOB_SSSP_U32, int(g.m), int(g.nnz),
                     _p(g.ptr), _p(g.ind),
                     _p(tptr),
                     _p(tind),
                     _p(g.w_u32), int(sym),
                     len(jd["sources"]), src, _p(out),
                     int(jd.get("alpha", -1)), int(jd.get("beta", -1)))
        sin = g.extra.get("sssp_in", {}).get("u32") if jd["type"] == "sssp" else None
        if sin is not None:
            # in-adjacency with weights from sssp_prepare: pull steps
            arr[i].d_stptr = _p(sin[0])
            arr[i].d_stind = _p(sin[1])
            arr[i].d_stw = _p(sin[2])
    return arr, outs, keep


def batch_set_params(ctx: Context, deep_blocks: int = 0, deep_concurrent: int = 48):
    """Sources of jobs on deep graphs (BFS of more than 64 levels) run as
    single-source traversals, up to deep_concurrent at a time on
    sub-contexts, with deep_blocks blocks in all (0: the default share);
    deep_concurrent=0 keeps them in the multi-source launch."""
    check(lib.apspie_batch_set_params(ctx.handle, int(deep_blocks)), ctx.handle,
          "apspie_batch_set_params")
    check(lib.apspie_batch_set_deep_mode(ctx.handle, int(deep_concurrent)), ctx.handle,
          "apspie_batch_set_deep_mode")


def batch_set_sssp_pull(ctx: Context, alpha: int = 0) -> None:
    """Pull switch of the multi-source SSSP steps (0 = never pull, the default)."""
    check(lib.apspie_batch_set_sssp_pull(ctx.handle, int(alpha)), ctx.handle,
          "apspie_batch_set_sssp_pull")


def batch_stats(ctx: Context) -> dict:
    s = BatchStats()
    check(lib.apspie_batch_get_stats(ctx.handle, C.byref(s)), ctx.handle, "apspie_batch_get_stats")
    return {"super_steps": s.super_steps, "frontier_edges": s.frontier_edges}


TUNING_FIELDS = [f for f, _ in Tuning._fields_]


def get_tuning(ctx: Context) -> dict:
    """The context's per-graph choices (apspie_ctx_get_tuning)."""
    t = Tuning()
    check(lib.apspie_ctx_get_tuning(ctx.handle, C.byref(t)), ctx.handle, "apspie_ctx_get_tuning")
    return {f: getattr(t, f) for f in TUNING_FIELDS}


def set_tuning(ctx: Context, **kw) -> dict:
    """Set some of the context's per-graph choices (the others keep their
    values); returns the whole set."""
    cur = get_tuning(ctx)
    bad = set(kw) - set(cur)
    if bad:
        raise KeyError(f"unknown tuning fields: {sorted(bad)}")
    cur.update(kw)
    t = Tuning(**cur)
    check(lib.apspie_ctx_set_tuning(ctx.handle, C.byref(t)), ctx.handle, "apspie_ctx_set_tuning")
    return cur


def reset_tuning(ctx: Context) -> dict:
    """Back to the library defaults."""
    return set_tuning(ctx, **DEFAULT_TUNING)


DEFAULT_TUNING = {"bfs_alpha": 14, "bfs_beta": 24, "bfs_blocks_per_sm": 0,
                  "sssp_blocks_per_sm": 0, "sssp_pull_alpha": 0, "batch_blocks_per_sm": 0,
                  "batch_deep_blocks": 0, "spgemm_table_load": 2, "spgemm_warp_max_prod": 256,
                  "spgemm_bitmap_max_cols": 1 << 18, "spmspv_sort_factor": 4.0}


def autotune_sssp(ctx: Context, g, sources) -> dict:
    """Pick and cache the persistent SSSP launch's blocks per SM and, when g
    carries its weighted in-adjacency (sssp_prepare), the pull switch, on
    uint32 weights."""
    import torch
    if g.w_u32 is None:
        raise ValueError("graph has no u32 weights")
    _graph(g)
    _row(g.w_u32, g.nnz, "u32 weights")
    dist = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
    src = (C.c_int * len(sources))(*[int(s) for s in sources])
    tin = g.extra.get("sssp_in", {}).get("u32")
    tptr, tind, tw = tin if tin is not None else (None, None, None)
    ms, cached = C.c_float(), C.c_int()
    check(lib.apspie_autotune_sssp(ctx.handle, len(sources), src, int(g.nnz), int(g.m), _p(g.ptr),
                                   _p(g.ind), _p(g.w_u32), _p(tptr), _p(tind), _p(tw), _p(dist),
                                   C.byref(ms), C.byref(cached)), ctx.handle,
          "apspie_autotune_sssp")
    t = get_tuning(ctx)
    return {"blocks_per_sm": t["sssp_blocks_per_sm"], "pull_alpha": t["sssp_pull_alpha"],
            "ms_per_sssp": ms.value, "cached": bool(cached.value)}


def autotune_spgemm(ctx: Context, A, B) -> dict:
    """Pick and cache the SpGEMM table load, warp-row limit and long-row
    accumulator for A * B ((m, n, ptr, ind, val) tuples as in spgemm)."""
    a, b = _csr(*A), _csr(*B)
    ms, cached = C.c_float(), C.c_int()
    check(lib.apspie_autotune_spgemm(ctx.handle, C.byref(a), C.byref(b), C.byref(ms),
                                     C.byref(cached)), ctx.handle, "apspie_autotune_spgemm")
    t = get_tuning(ctx)
    return {"table_load": t["spgemm_table_load"], "warp_max_prod": t["spgemm_warp_max_prod"],
            "bitmap_max_cols": t["spgemm_bitmap_max_cols"], "ms": ms.value,
            "cached": bool(cached.value)}


def autotune_batch(ctx: Context, jobs: list[dict]) -> dict:
    """Pick and cache the batched launch's blocks per SM and the deep-graph
    sources' block share for this job list (runs batch_run on it)."""
    arr, _outs, _keep = _job_array(jobs)
    ms, cached = C.c_float(), C.c_int()
    check(lib.apspie_autotune_batch(ctx.handle, len(jobs), arr, C.byref(ms), C.byref(cached)),
          ctx.handle, "apspie_autotune_batch")
    t = get_tuning(ctx)
    return {"blocks_per_sm": t["batch_blocks_per_sm"], "deep_blocks": t["batch_deep_blocks"],
            "ms": ms.value, "cached": bool(cached.value)}


def autotune_bfs(ctx: Context, g, sources) -> dict:
    """Pick and cache the BFS direction thresholds and the persistent
    launch's blocks per SM for graph g."""
    import torch
    _graph(g)
    depth = torch.empty(g.m, dtype=torch.int32, device=g.ptr.device)
    src = (C.c_int * len(sources))(*[int(s) for s in sources])
    sym = bool(getattr(g, "symmetric", False))
    tptr, tind = (g.ptr, g.ind) if sym else (g.tptr, g.tind)
    a, b, ms = C.c_int(), C.c_int(), C.c_float()
    check(lib.apspie_autotune_bfs(ctx.handle, len(sources), src, int(g.nnz), int(g.m), _p(g.ptr),
                                  _p(g.ind), _p(tptr), _p(tind), _p(depth), C.byref(a),
                                  C.byref(b), C.byref(ms)), ctx.handle, "apspie_autotune_bfs")
    return {"alpha": a.value, "beta": b.value, "ms_per_bfs": ms.value,
            "blocks_per_sm": get_tuning(ctx)["bfs_blocks_per_sm"]}


def autotune_spmspv(ctx: Context, g, val=None) -> float:
    import torch
    _graph(g)
    _row(val, g.nnz, "val")
    dev = g.ptr.device
    xi = torch.empty(g.m, dtype=torch.int32, device=dev)
    xv = torch.empty(g.m, dtype=torch.float32, device=dev)
    yi = torch.empty(g.m, dtype=torch.int32, device=dev)
    yv = torch.empty(g.m, dtype=torch.float32, device=dev)
    f = C.c_double()
    check(lib.apspie_autotune_spmspv(ctx.handle, int(g.m), int(g.nnz), _p(g.ptr), _p(g.ind),
                                     _p(val), _p(xi), _p(xv), _p(yi), _p(yv), C.byref(f)),
          ctx.handle, "apspie_autotune_spmspv")
    return f.value
