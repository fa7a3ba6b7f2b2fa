"""The Python entry points refuse, before anything reaches the library, the
tensors a kernel would misread: host tensors, strided views, per-vertex
rows shorter than the graph or wider than 32 bits, graphs whose arrays are
shorter than m and nnz promise.  A stand-in context is enough: every check
runs before the context's handle is used."""
import ctypes as C

import numpy as np
import pytest
import torch

import apspie_b200 as ap
from apspie_b200 import ops


class _Ctx:
    handle = C.c_void_p(0)  # never passed on: the checks raise first


class _Graph:
    def __init__(self, m=8, nnz=12, ptr_len=None, ind_len=None, dtype=torch.int32):
        self.m, self.nnz, self.symmetric = m, nnz, True
        self.ptr = torch.zeros(m + 1 if ptr_len is None else ptr_len, dtype=dtype)
        self.ind = torch.zeros(nnz if ind_len is None else ind_len, dtype=dtype)
        self.w_u32 = torch.zeros(nnz, dtype=torch.int32)
        self.w_f32 = torch.zeros(nnz, dtype=torch.float32)
        self.extra = {}


class _FakeCuda:
    """Looks like a CUDA tensor but is strided."""
    is_cuda = True

    def is_contiguous(self):
        return False


def test_pointer_helper_refuses_host_and_strided_tensors():
    assert ops._p(None).value is None
    with pytest.raises(ValueError, match="CUDA tensor"):
        ops._p(torch.zeros(4, dtype=torch.int32))
    with pytest.raises(ValueError, match="contiguous"):
        ops._p(_FakeCuda())


def test_rows_must_cover_the_graph_with_32_bit_entries():
    ops._row(torch.zeros(8, dtype=torch.int32), 8, "x")
    ops._row(torch.zeros(9, dtype=torch.float32), 8, "x")
    ops._row(None, 8, "x")
    with pytest.raises(ValueError, match="needs 8"):
        ops._row(torch.zeros(7, dtype=torch.int32), 8, "x")
    with pytest.raises(ValueError, match="needs 8"):
        ops._row(torch.zeros(8, dtype=torch.int64), 8, "x")


@pytest.mark.parametrize("bad", [dict(ptr_len=8), dict(ind_len=11), dict(dtype=torch.int64)])
def test_graph_arrays_must_hold_m_and_nnz(bad):
    g = _Graph(**bad)
    with pytest.raises(ValueError, match="graph"):
        ap.bfs(_Ctx(), g, 0)
    with pytest.raises(ValueError, match="graph"):
        ap.mis(_Ctx(), g, torch.zeros(g.m, dtype=torch.int32))


def test_entry_points_refuse_short_outputs_and_host_tensors():
    g = _Graph()
    with pytest.raises(ValueError, match="depth"):
        ap.bfs(_Ctx(), g, 0, depth=torch.zeros(g.m - 1, dtype=torch.int32))
    with pytest.raises(ValueError, match="dist"):
        ap.sssp(_Ctx(), g, 0, dist=torch.zeros(g.m, dtype=torch.int64))
    with pytest.raises(ValueError, match="prio"):
        ap.mis(_Ctx(), g, torch.zeros(g.m - 1, dtype=torch.int32))
    with pytest.raises(ValueError, match="flags"):
        ap.neighbor_flags(_Ctx(), g, torch.zeros(2, dtype=torch.int32))
    with pytest.raises(ValueError, match="x"):
        ap.mxv_dense(_Ctx(), 0, g, torch.zeros(g.m - 1, dtype=torch.float32))
    with pytest.raises(ValueError, match="val"):
        ap.spmspv(_Ctx(), 0, g, torch.zeros(1, dtype=torch.int32),
                  val=torch.zeros(g.nnz - 1, dtype=torch.float32))
    # well-sized host tensors pass the size checks and stop at the pointer check
    with pytest.raises(ValueError, match="CUDA tensor"):
        ap.bfs(_Ctx(), g, 0)
    with pytest.raises(ValueError, match="CUDA tensor"):
        ap.sssp(_Ctx(), g, 0, weights="f32")
    with pytest.raises(ValueError, match="CUDA tensor"):
        ap.mis(_Ctx(), g, torch.zeros(g.m, dtype=torch.int32))


def test_matrix_entry_points_check_offsets_and_values():
    z = lambda n, dt=torch.int32: torch.zeros(n, dtype=dt)
    ctx = _Ctx()
    # (m, n, ptr, ind, val): offsets must cover m + 1 rows, values every index
    with pytest.raises(ValueError, match="row offsets"):
        ap.spgemm(ctx, (4, 4, z(4), z(6), None), (4, 4, z(5), z(6), None))
    with pytest.raises(ValueError, match="values"):
        ap.spgemm(ctx, (4, 4, z(5), z(6), z(5, torch.float32)), (4, 4, z(5), z(6), None))
    with pytest.raises(ValueError, match="row offsets"):
        ap.csr_transpose(ctx, 4, 4, z(3), z(6))
    with pytest.raises(ValueError, match="values"):
        ap.spmv(ctx, 4, z(5), z(6), z(6, torch.float64), z(4, torch.float32))
    with pytest.raises(ValueError, match="L row offsets"):
        ap.triangle_count(ctx, 8, z(8), z(3))
    # graph-taking builders and tuners check the graph first
    bad = _Graph(ptr_len=3)
    for call in (lambda: ap.bfs_prepare(ctx, bad), lambda: ap.tc_prepare(ctx, bad),
                 lambda: ap.weights_device(ctx, bad), lambda: ap.autotune_bfs(ctx, bad, [0]),
                 lambda: ap.autotune_sssp(ctx, bad, [0]),
                 lambda: ap.batch_run(ctx, [{"type": "bfs", "graph": bad, "sources": [0]}])):
        with pytest.raises(ValueError, match="graph row offsets"):
            call()
    g = _Graph()
    g.w_u32 = z(g.nnz - 1)
    with pytest.raises(ValueError, match="u32 weights"):
        ap.batch_run(ctx, [{"type": "sssp", "graph": g, "sources": [0]}])
