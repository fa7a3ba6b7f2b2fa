"""Generic SpMSpV parity (both mXv forms, every semiring, both the radix-sort
and the bitmap path) against the oracle's restatement of src/mXv.cuh."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

SEMIRINGS = [0, 1, 2, 3]   # PLUS_TIMES, MIN_PLUS, MAX_TIMES, OR_AND
PLUS_REL_TOL = 1e-5        # float sums vs the FP64 oracle, relative to sum |terms|


def _graph(scale=12, seed=3, positive=False):
    import apspie_b200 as ap
    h = ap.gen_rmat(scale, 16, seed=seed, symmetric=False)
    rng = np.random.default_rng(seed)
    vals = rng.uniform(0.01, 1.0, h.nnz) if positive else rng.uniform(-1, 1, h.nnz)
    return h, vals.astype(np.float32)


def _compare(sr, got_i, got_v, ref_i, ref_v, h, vals, xind, xval):
    np.testing.assert_array_equal(got_i, ref_i)
    if sr == 0:
        # bound on the rounding of a float sum: relative to the sum of |terms|
        absref = oracle.spmspv(0, h.m, h.ptr, h.ind, np.abs(vals), xind, np.abs(xval))[1]
        assert np.all(np.abs(got_v - ref_v) <= PLUS_REL_TOL * absref + 1e-30)
    else:
        np.testing.assert_array_equal(got_v.astype(np.float32), ref_v.astype(np.float32))


@pytest.mark.parametrize("sr", SEMIRINGS)
@pytest.mark.parametrize("path", ["sort", "bitmap"])
@pytest.mark.parametrize("density", [0.001, 0.05])
def test_spmspv_vs_oracle(ctx, sr, path, density):
    import torch
    import apspie_b200 as ap
    h, vals = _graph(positive=(sr == 1))
    g = h.to_device(with_transpose=False)
    rng = np.random.default_rng(int(density * 1000) + sr)
    xind = np.flatnonzero(rng.random(h.m) < density).astype(np.int32)
    xval = rng.uniform(0.1, 2.0, xind.size).astype(np.float32)
    ap.spmspv_set_params(ctx, 0.0 if path == "sort" else 1e12)
    try:
        yi, yv, e = ap.spmspv(ctx, sr, g, torch.from_numpy(xind).cuda(),
                              torch.from_numpy(xval).cuda(), torch.from_numpy(vals).cuda())
    finally:
        ap.spmspv_set_params(ctx)
    ri, rv = oracle.spmspv(sr, h.m, h.ptr, h.ind, vals, xind, xval)
    assert e == int(h.degrees()[xind].sum())
    _compare(sr, yi.cpu().numpy(), yv.cpu().numpy().astype(np.float64), ri, rv, h, vals, xind,
             xval)


def test_spmspv_hub_columns_and_empty(ctx):
    import torch
    import apspie_b200 as ap
    h, vals = _graph(scale=14, seed=5)
    g = h.to_device(with_transpose=False)
    deg = h.degrees()
    hubs = np.sort(np.argsort(deg)[-20:]).astype(np.int32)  # columns far above the chunk size
    assert deg[hubs].max() > 256
    xval = np.ones(hubs.size, np.float32)
    for path in (0.0, 1e12):
        ap.spmspv_set_params(ctx, path)
        yi, yv, _ = ap.spmspv(ctx, 0, g, torch.from_numpy(hubs).cuda(),
                              torch.from_numpy(xval).cuda(), torch.from_numpy(vals).cuda())
        ri, rv = oracle.spmspv(0, h.m, h.ptr, h.ind, vals, hubs, xval)
        _compare(0, yi.cpu().numpy(), yv.cpu().numpy().astype(np.float64), ri, rv, h, vals, hubs,
                 xval)
    ap.spmspv_set_params(ctx)
    yi, yv, e = ap.spmspv(ctx, 0, g, torch.zeros(0, dtype=torch.int32, device="cuda"))
    assert yi.numel() == 0 and e == 0


@pytest.mark.parametrize("sr", [0, 1])
def test_mxv_dense_reference_semantics(ctx, sr):
    """Dense in / dense out: frontier by bitify (> 0.5) or finite (< 1e38),
    untouched rows 0 (or 1.70141e38), return value = expanded size."""
    import torch
    import apspie_b200 as ap
    h, vals = _graph(positive=True)
    g = h.to_device(with_transpose=False)
    rng = np.random.default_rng(7)
    if sr == 0:
        x = np.where(rng.random(h.m) < 0.01, 1.0, 0.0).astype(np.float32)
        front = np.flatnonzero(x > 0.5)
    else:
        x = np.where(rng.random(h.m) < 0.01, rng.uniform(0, 5, h.m),
                     np.float32(1.70141e38)).astype(np.float32)
        front = np.flatnonzero((x > -1) & (x < 1e38))
    y, total = ap.mxv_dense(ctx, sr, g, torch.from_numpy(x).cuda(), torch.from_numpy(vals).cuda())
    y = y.cpu().numpy()
    ri, rv = oracle.spmspv(sr, h.m, h.ptr, h.ind, vals, front, x[front])
    assert total == int(h.degrees()[front].sum())
    empty = np.float32(0.0) if sr == 0 else np.float32(1.70141e38)
    expect = np.full(h.m, empty, np.float32)
    expect[ri] = rv.astype(np.float32)
    untouched = np.ones(h.m, bool)
    untouched[ri] = False
    np.testing.assert_array_equal(y[untouched], expect[untouched])
    np.testing.assert_allclose(y[ri], expect[ri], rtol=1e-5)


def test_spmspv_bfs_step_matches_bfs(ctx):
    """One OR_AND SpMSpV from a source = the source's out-neighbours."""
    import torch
    import apspie_b200 as ap
    h, _ = _graph()
    g = h.to_device(with_transpose=False)
    s = int(np.argmax(h.degrees()))
    yi, _, _ = ap.spmspv(ctx, 3, g, torch.tensor([s], dtype=torch.int32, device="cuda"))
    np.testing.assert_array_equal(yi.cpu().numpy(), np.unique(h.ind[h.ptr[s]:h.ptr[s + 1]]))


@pytest.mark.gpu
@pytest.mark.parametrize("semiring", [0, 1, 2, 3])
def test_dense_spmv_all_rows(ctx, semiring):
    """apspie_spmv against an FP64 / exact restatement: power-law rows with
    a few hubs above the block threshold (4096) and empty rows."""
    import torch
    import apspie_b200 as ap
    rng = np.random.default_rng(semiring)
    m = 6000
    lens = rng.integers(0, 20, m)
    lens[::997] = 0
    lens[[5, 1234, 4321]] = [5000, 9000, 4097]
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ind = rng.integers(0, m, int(ptr[-1])).astype(np.int32)
    val = rng.uniform(-1, 1, int(ptr[-1])).astype(np.float32)
    x = rng.uniform(-1, 1, m).astype(np.float32)
    x[::5] = 0
    t = lambda a: torch.from_numpy(a).cuda()
    y = ap.spmv(ctx, m, t(ptr), t(ind), t(val), t(x), semiring).cpu().numpy()
    for r in range(m):
        a, xs = val[ptr[r]:ptr[r + 1]], x[ind[ptr[r]:ptr[r + 1]]]
        if semiring == 0:
            ref = float(np.sum(a.astype(np.float64) * xs.astype(np.float64)))
            tol = 1e-6 * max(1.0, float(np.sum(np.abs(a.astype(np.float64) * xs))))
            assert abs(y[r] - ref) <= tol, (r, y[r], ref)
        elif semiring == 1:
            ref = np.float32(np.min(a + xs)) if len(a) else np.finfo(np.float32).max
            assert y[r] == ref, (r, y[r], ref)
        elif semiring == 2:
            ref = np.float32(np.max(a * xs)) if len(a) else -np.finfo(np.float32).max
            assert y[r] == ref, (r, y[r], ref)
        else:
            ref = 1.0 if np.any((a != 0) & (xs != 0)) else 0.0
            assert y[r] == ref, (r, y[r], ref)
