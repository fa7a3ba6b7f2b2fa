"""Graph containers and the synthetic graph builders of the benchmark configs.

HostGraph holds a CSR (int32 row offsets, int32 column indices) in numpy;
DeviceGraph holds the same arrays resident in device memory as torch
tensors (torch is used only as the device allocator).  The CSR row of u
lists u's out-neighbours, which is what the reference drivers pass to its
SpMSpV as "CSC" (test/bfs/main.cu:140).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._native import check, lib


def _take_int_array(p: C.c_void_p, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.int32)
    if n:
        C.memmove(out.ctypes.data, p.value, 4 * n)
    lib.apspie_host_free(p)
    return out


@dataclass
class HostGraph:
    m: int
    ptr: np.ndarray
    ind: np.ndarray
    name: str = ""
    w_u32: np.ndarray | None = None
    w_f32: np.ndarray | None = None
    symmetric: bool = False

    @property
    def nnz(self) -> int:
        return int(self.ind.shape[0])

    def degrees(self) -> np.ndarray:
        return np.diff(self.ptr)

    def transpose(self) -> "HostGraph":
        """CSR of the transpose (in-adjacency), rows sorted by source id."""
        src = np.repeat(np.arange(self.m, dtype=np.int32), np.diff(self.ptr))
        order = np.argsort(self.ind, kind="stable")
        ptr = np.zeros(self.m + 1, dtype=np.int64)
        np.add.at(ptr, self.ind.astype(np.int64) + 1, 1)
        return HostGraph(self.m, np.cumsum(ptr).astype(np.int32), src[order].copy(),
                         name=self.name + "^T")

    def to_device(self, device: int | str = 0, with_transpose: bool = True) -> "DeviceGraph":
        import torch
        dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)

        def t(a):
            if a is None:
                return None
            if a.size == 0:
                return torch.zeros(1, dtype=torch.from_numpy(a[:0]).dtype, device=dev)
            return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

        w_u32 = None if self.w_u32 is None else t(self.w_u32.view(np.int32))
        g = DeviceGraph(self.m, self.nnz, t(self.ptr), t(self.ind), w_u32=w_u32,
                        w_f32=t(self.w_f32), name=self.name, symmetric=self.symmetric)
        if with_transpose and not self.symmetric:
            tr = self.transpose()
            g.tptr, g.tind = t(tr.ptr), t(tr.ind)
        return g


@dataclass
class DeviceGraph:
    m: int
    nnz: int
    ptr: "object"
    ind: "object"
    w_u32: "object" = None   # stored as int32 tensor holding uint32 bits
    w_f32: "object" = None
    name: str = ""
    symmetric: bool = False
    tptr: "object" = None    # in-adjacency (transpose CSR) for pull traversal
    tind: "object" = None
    extra: dict = field(default_factory=dict)


def gen_rmat(scale: int, edge_factor: int = 16, seed: int = 1, symmetric: bool = True,
             scramble: bool = True) -> HostGraph:
    """R-MAT (0.57, 0.19, 0.19, 0.05), self-loops and duplicates removed."""
    m = C.c_int()
    nnz = C.c_int64()
    p, i = C.c_void_p(), C.c_void_p()
    check(lib.apspie_gen_rmat_host(scale, edge_factor, seed, int(symmetric), int(scramble),
                                   C.byref(m), C.byref(nnz), C.byref(p), C.byref(i)),
          what="gen_rmat")
    name = f"rmat{scale}{'s' if symmetric else 'd'}"
    return HostGraph(m.value, _take_int_array(p, m.value + 1), _take_int_array(i, nnz.value),
                     name=name, symmetric=symmetric)


def gen_er(n: int, mean_degree: int = 8, seed: int = 1) -> HostGraph:
    nnz = C.c_int64()
    p, i = C.c_void_p(), C.c_void_p()
    check(lib.apspie_gen_er_host(n, mean_degree, seed, C.byref(nnz), C.byref(p), C.byref(i)),
          what="gen_er")
    return HostGraph(n, _take_int_array(p, n + 1), _take_int_array(i, nnz.value), name=f"er{n}",
                     symmetric=True)


def gen_grid(rows: int, cols: int) -> HostGraph:
    nnz = C.c_int64()
    p, i = C.c_void_p(), C.c_void_p()
    check(lib.apspie_gen_grid_host(rows, cols, C.byref(nnz), C.byref(p), C.byref(i)),
          what="gen_grid")
    m = rows * cols
    return HostGraph(m, _take_int_array(p, m + 1), _take_int_array(i, nnz.value),
                     name=f"grid{rows}x{cols}", symmetric=True)


def weights_u32(g: HostGraph, seed: int = 7, lo: int = 1, hi: int = 255) -> np.ndarray:
    w = np.empty(g.nnz, dtype=np.uint32)
    check(lib.apspie_gen_weights_u32_host(g.m, g.ptr.ctypes.data, g.ind.ctypes.data, seed, lo,
                                          hi, w.ctypes.data), what="weights_u32")
    g.w_u32 = w
    return w


def weights_f32(g: HostGraph, seed: int = 7) -> np.ndarray:
    w = np.empty(g.nnz, dtype=np.float32)
    check(lib.apspie_gen_weights_f32_host(g.m, g.ptr.ctypes.data, g.ind.ctypes.data, seed,
                                          w.ctypes.data), what="weights_f32")
    g.w_f32 = w
    return w


def gen_powerlaw(m: int = 1 << 18, n: int | None = None, alpha: float = 2.1, mean: float = 16.0,
                 max_deg: int = 4096, seed: int = 1) -> HostGraph:
    """Power-law-row matrix of the SpGEMM benchmark; values in w_f32,
    the solved x_min in .name."""
    n = m if n is None else n
    xmin = C.c_double()
    nnz = C.c_int64()
    p, i, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(lib.apspie_gen_powerlaw_host(m, n, alpha, mean, max_deg, seed, C.byref(xmin),
                                       C.byref(nnz), C.byref(p), C.byref(i), C.byref(v)),
          what="gen_powerlaw")
    vals = np.empty(nnz.value, dtype=np.float32)
    if nnz.value:
        C.memmove(vals.ctypes.data, v.value, 4 * nnz.value)
    lib.apspie_host_free(v)
    g = HostGraph(m, _take_int_array(p, m + 1), _take_int_array(i, nnz.value),
                  name=f"powerlaw{m}x{n}(xmin={xmin.value:.4f})")
    g.w_f32 = vals
    g.ncols = n
    g.xmin = xmin.value
    return g


def mt19937(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    check(lib.apspie_mt19937_fill_host(seed, n, out.ctypes.data), what="mt19937")
    return out


def read_mtx(path: str, undirected: bool = False) -> HostGraph:
    """Matrix Market file -> CSR with the reference's orientation (row = the
    second index of a line, column = the first; src/util.cuh:371-430)."""
    m = C.c_int()
    nnz = C.c_int64()
    p, i, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    weighted = C.c_int()
    check(lib.apspie_read_mtx_host(str(path).encode(), int(undirected), C.byref(m), C.byref(nnz),
                                   C.byref(p), C.byref(i), C.byref(v), C.byref(weighted)),
          what=f"read_mtx({path})")
    vals = np.empty(nnz.value, dtype=np.float32)
    if nnz.value:
        C.memmove(vals.ctypes.data, v.value, 4 * nnz.value)
    lib.apspie_host_free(v)
    g = HostGraph(m.value, _take_int_array(p, m.value + 1), _take_int_array(i, nnz.value),
                  name=str(path).rsplit("/", 1)[-1], symmetric=bool(undirected))
    if weighted.value:
        g.w_f32 = vals
    return g


def from_edges(m: int, rows: np.ndarray, cols: np.ndarray, name: str = "") -> HostGraph:
    """CSR from an edge list (kept in the given order within each row,
    duplicates kept), as the reference's buildMatrix (src/matrix.cpp:56-111)."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int32)
    order = np.argsort(rows, kind="stable")
    ptr = np.zeros(m + 1, dtype=np.int64)
    np.add.at(ptr, rows + 1, 1)
    return HostGraph(m, np.cumsum(ptr).astype(np.int32), cols[order].copy(), name=name)


def largest_cc_vertex(g: HostGraph, seed: int = 0) -> int:
    """A seed-chosen vertex of the largest (weakly) connected component."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    a = sp.csr_matrix((np.ones(g.nnz, dtype=np.int8), g.ind, g.ptr), shape=(g.m, g.m))
    _, label = connected_components(a, directed=True, connection="weak")
    counts = np.bincount(label)
    members = np.flatnonzero(label == int(np.argmax(counts)))
    rng = np.random.default_rng(seed)
    return int(members[int(rng.integers(len(members)))])


def seeded_sources(g: HostGraph, k: int, seed: int = 0) -> list[int]:
    """k seed-chosen vertices of the largest connected component."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    a = sp.csr_matrix((np.ones(g.nnz, dtype=np.int8), g.ind, g.ptr), shape=(g.m, g.m))
    _, label = connected_components(a, directed=True, connection="weak")
    members = np.flatnonzero(label == int(np.argmax(np.bincount(label))))
    rng = np.random.default_rng(seed)
    return [int(x) for x in members[rng.integers(len(members), size=k)]]
