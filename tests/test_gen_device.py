"""Device graph builder against the host builder: the same arrays, bit for
bit (both follow the counter-based R-MAT / ER draws of gen_common.h)."""
import numpy as np
import pytest

import apspie_b200 as ap


@pytest.mark.gpu
@pytest.mark.parametrize("scale,ef,sym,scr", [(8, 4, True, True), (12, 16, True, True),
                                              (12, 16, False, True), (14, 8, True, False),
                                              (16, 16, True, True)])
def test_rmat_device_matches_host(ctx, scale, ef, sym, scr):
    h = ap.gen_rmat(scale, ef, seed=3, symmetric=sym, scramble=scr)
    d = ap.gen_rmat_device(ctx, scale, ef, seed=3, symmetric=sym, scramble=scr)
    assert d.m == h.m and d.nnz == h.nnz
    np.testing.assert_array_equal(d.ptr.cpu().numpy(), h.ptr)
    np.testing.assert_array_equal(d.ind.cpu().numpy(), h.ind)


@pytest.mark.gpu
@pytest.mark.parametrize("n,deg", [(2, 1), (1000, 8), (1 << 16, 16)])
def test_er_device_matches_host(ctx, n, deg):
    h = ap.gen_er(n, deg, seed=5)
    d = ap.gen_er_device(ctx, n, deg, seed=5)
    assert d.nnz == h.nnz
    np.testing.assert_array_equal(d.ptr.cpu().numpy(), h.ptr)
    np.testing.assert_array_equal(d.ind.cpu().numpy(), h.ind)


@pytest.mark.gpu
def test_rmat22_device_properties(ctx):
    """At the benchmark size: rows sorted and strictly increasing, no
    self-loops, symmetric (checked by the transpose having the same nnz and
    a checksum of (row, col) pairs equal in both orientations)."""
    import torch
    d = ap.gen_rmat_device(ctx, 22, 16, seed=1)
    ptr, ind = d.ptr.long(), d.ind.long()
    rows = torch.repeat_interleave(torch.arange(d.m, device=ptr.device), ptr[1:] - ptr[:-1])
    assert int(ptr[-1]) == d.nnz
    assert not bool((rows == ind).any())
    key = rows * d.m + ind
    assert bool((key[1:] > key[:-1]).all())
    tkey = ind * d.m + rows
    assert int((key * 2654435761 % (1 << 61)).sum()) == int((tkey * 2654435761 % (1 << 61)).sum())


@pytest.mark.gpu
def test_weights_device_match_host(ctx):
    h = ap.gen_rmat(12, 16, seed=3)
    wu = ap.weights_u32(h, seed=9)
    wf = ap.weights_f32(h, seed=9)
    d = ap.weights_device(ctx, h.to_device(), seed=9)
    np.testing.assert_array_equal(d.w_u32.cpu().numpy().view(np.uint32), wu)
    np.testing.assert_array_equal(d.w_f32.cpu().numpy(), wf)


@pytest.mark.gpu
@pytest.mark.parametrize("m,n", [(1000, 1000), (700, 1500), (3000, 40)])
def test_csr_transpose_matches_host(ctx, m, n):
    """apspie_csr_transpose = the CSC: offsets, row ids ascending within a
    column, values carried along (scipy's csr -> csc as the reference)."""
    import scipy.sparse as sp
    import torch
    rng = np.random.default_rng(m + n)
    a = sp.random(m, n, density=0.01, format="csr", random_state=rng, dtype=np.float32)
    a.sort_indices()
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    tp, ti, tv = ap.csr_transpose(ctx, m, n, t(a.indptr.astype(np.int32)),
                                  t(a.indices.astype(np.int32)), t(a.data))
    c = a.tocsc()
    c.sort_indices()
    np.testing.assert_array_equal(tp.cpu().numpy(), c.indptr)
    np.testing.assert_array_equal(ti.cpu().numpy(), c.indices)
    np.testing.assert_array_equal(tv.cpu().numpy(), c.data)
