"""Hash SpGEMM and triangle counting parity against the oracle (FP64
Gustavson; int64 sorted-merge triangle count): SpGEMM structure exact,
values within 1e-5 relative (plus a double-rounding floor relative to the
sum of |products|); triangle counts exact."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

VAL_RTOL = 1e-5


def _dev_csr(h):
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ind = t(h.ind) if h.nnz else torch.zeros(1, dtype=torch.int32, device="cuda")
    val = t(h.w_f32) if h.w_f32 is not None and h.nnz else None
    return (h.m, getattr(h, "ncols", h.m), t(h.ptr), ind if h.nnz else ind[:0], val)


def _check_product(ctx, A, B):
    import apspie_b200 as ap
    cp, ci, cv = ap.spgemm(ctx, _dev_csr(A), _dev_csr(B))
    cp, ci, cv = cp.cpu().numpy(), ci.cpu().numpy(), cv.cpu().numpy()
    n = getattr(B, "ncols", B.m)
    rp, ri, rv = oracle.spgemm(A.m, n, A.ptr, A.ind, A.w_f32, B.ptr, B.ind, B.w_f32)
    np.testing.assert_array_equal(cp, rp.astype(np.int32))
    np.testing.assert_array_equal(ci, ri)
    absA = None if A.w_f32 is None else np.abs(A.w_f32)
    absB = None if B.w_f32 is None else np.abs(B.w_f32)
    _, _, mag = oracle.spgemm(A.m, n, A.ptr, A.ind, absA, B.ptr, B.ind, absB)
    err = np.abs(cv.astype(np.float64) - rv)
    assert np.all(err <= VAL_RTOL * np.abs(rv) + 1e-12 * mag + 1e-30), err.max()
    return cp[-1]


def test_spgemm_fixture_and_small(ctx, golden):
    import apspie_b200 as ap
    h = ap.HostGraph(4, golden["mtx/test_spgemm/dir_ptr"], golden["mtx/test_spgemm/dir_ind"])
    h.w_f32 = np.arange(1, h.nnz + 1, dtype=np.float32)
    _check_product(ctx, h, h)
    rng = np.random.default_rng(0)
    for m in (1, 7, 300):
        rows = rng.integers(0, m, 5 * m)
        cols = rng.integers(0, m, 5 * m)
        key = np.unique(rows * m + cols)
        g = ap.from_edges(m, key // m, key % m)
        g.w_f32 = rng.uniform(-1, 1, g.nnz).astype(np.float32)
        _check_product(ctx, g, g)


def test_spgemm_keeps_cancellation(ctx):
    import apspie_b200 as ap
    A = ap.HostGraph(1, np.array([0, 2], np.int32), np.array([0, 1], np.int32))
    A.w_f32 = np.array([1.0, -1.0], np.float32)
    A.ncols = 2
    B = ap.HostGraph(2, np.array([0, 1, 2], np.int32), np.array([0, 0], np.int32))
    B.w_f32 = np.array([1.0, 1.0], np.float32)
    B.ncols = 1
    import torch
    cp, ci, cv = ap.spgemm(ctx, _dev_csr(A), _dev_csr(B))
    assert cp.tolist() == [0, 1] and ci.tolist() == [0] and cv.tolist() == [0.0]


@pytest.mark.parametrize("bitmap", [True, False])
def test_spgemm_all_bins_rectangular(ctx, bitmap):
    """Power-law rows reach the warp, block and dense-accumulator bins (hash
    tables) or the warp and both bitmap bins (output rows up to 4096 staged
    in shared memory, larger ones in global memory)."""
    import apspie_b200 as ap
    A = ap.gen_powerlaw(1 << 12, 1 << 11, max_deg=1024, seed=2)
    B = ap.gen_powerlaw(1 << 11, 1 << 14, max_deg=1024, seed=3)
    prod = np.array([B.degrees()[A.ind[A.ptr[i]:A.ptr[i + 1]]].sum() for i in range(A.m)])
    assert (prod <= 256).any() and ((prod > 256) & (prod <= 8192)).any() and (prod > 8192).any()
    ap.spgemm_set_params(ctx, 1 << 18 if bitmap else 0)
    try:
        nnz_rows = np.diff(oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, None, B.ptr, B.ind, None)[0])
        assert (nnz_rows > 4096).any()
        _check_product(ctx, A, B)
    finally:
        ap.spgemm_set_params(ctx)


def test_spgemm_two_phase_reuse(ctx):
    """Symbolic once, numeric into caller buffers; the numeric phase repeats
    for new values on the same structure; a numeric call for other matrices
    is refused."""
    import torch
    import apspie_b200 as ap
    A = ap.gen_powerlaw(1 << 12, 1 << 11, max_deg=1024, seed=2)
    B = ap.gen_powerlaw(1 << 11, 1 << 12, max_deg=1024, seed=3)
    dA, dB = _dev_csr(A), _dev_csr(B)
    ptr, nnz = ap.spgemm_symbolic(ctx, dA, dB)
    ind = torch.empty(nnz, dtype=torch.int32, device="cuda")
    val = torch.empty(nnz, dtype=torch.float32, device="cuda")
    rp, ri, _ = oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, A.w_f32, B.ptr, B.ind, B.w_f32)
    np.testing.assert_array_equal(ptr.cpu().numpy(), rp.astype(np.int32))
    for scale in (1.0, -2.5):
        dA[4].copy_(torch.from_numpy(A.w_f32 * np.float32(scale)))
        ap.spgemm_numeric(ctx, dA, dB, ptr, ind, val)
        _, _, rv = oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, A.w_f32 * np.float32(scale),
                                 B.ptr, B.ind, B.w_f32)
        np.testing.assert_array_equal(ind.cpu().numpy(), ri)
        absA = np.abs(A.w_f32 * np.float32(scale))
        _, _, mag = oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, absA, B.ptr, B.ind, np.abs(B.w_f32))
        err = np.abs(val.cpu().numpy().astype(np.float64) - rv)
        assert np.all(err <= VAL_RTOL * np.abs(rv) + 1e-12 * mag + 1e-30), err.max()
    with pytest.raises(ap.ApspieError):
        ap.spgemm_numeric(ctx, dB, dA, ptr, ind, val)


def test_spgemm_powerlaw_full_config(ctx):
    """2^18 x 2^18, row nnz power law (alpha 2.1, mean 16, max 4096): A * A."""
    import apspie_b200 as ap
    A = ap.gen_powerlaw(1 << 18, seed=1)
    nnz_c = _check_product(ctx, A, A)
    assert nnz_c > 6e7


def _tc(ctx, h):
    import apspie_b200 as ap
    g = h.to_device(with_transpose=False)
    perm, lp, li = ap.tc_prepare(ctx, g)
    operm, olp, oli = oracle.tc_build_lower(h.m, h.ptr, h.ind)
    np.testing.assert_array_equal(perm.cpu().numpy(), operm)
    np.testing.assert_array_equal(lp.cpu().numpy(), olp)
    np.testing.assert_array_equal(li.cpu().numpy(), oli)
    got = ap.triangle_count(ctx, h.m, lp, li)
    assert got == oracle.tc_lower(h.m, olp, oli)
    return got


def test_tc_known_answers(ctx):
    import apspie_b200 as ap
    k4 = ap.HostGraph(4, np.array([0, 3, 6, 9, 12], np.int32),
                      np.array([1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2], np.int32))
    assert _tc(ctx, k4) == 4
    assert _tc(ctx, ap.gen_grid(32, 32)) == 0


def test_tc_fixtures(ctx, golden, fixture_names):
    import apspie_b200 as ap
    for name in fixture_names:
        ptr, ind = golden[f"mtx/{name}/und_ptr"], golden[f"mtx/{name}/und_ind"]
        src = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
        keep = src != ind   # self-loops carry no triangles
        h = ap.from_edges(len(ptr) - 1, src[keep], ind[keep])
        _tc(ctx, h)


def test_tc_matches_reference_kernel_goldens(ctx, golden, fixture_names):
    """apspie_tc against the counts of the reference's own intersection
    kernel (ewiseMultTc, src/tc.cuh:168-199, run host-side on U*L) stored in
    the goldens: every undirected fixture and R-MAT 10 / 12."""
    import apspie_b200 as ap
    graphs = {}
    for name in fixture_names:
        ptr, ind = golden[f"mtx/{name}/und_ptr"], golden[f"mtx/{name}/und_ind"]
        src = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
        keep = src != ind
        graphs[name] = ap.from_edges(len(ptr) - 1, src[keep], ind[keep])
    for sc in (10, 12):
        graphs[f"rmat{sc}"] = ap.gen_rmat(sc, 16, seed=3, symmetric=True)
    for name, h in graphs.items():
        g = h.to_device(with_transpose=False)
        _, lp, li = ap.tc_prepare(ctx, g)
        assert ap.triangle_count(ctx, h.m, lp, li) == int(golden[f"tc/{name}"][0]), name


def test_tc_prepare_rejects_a_directed_graph(ctx):
    """L is read from both ends of every edge, so the input must be
    symmetric: a directed R-MAT graph is refused, not miscounted."""
    import apspie_b200 as ap
    g = ap.gen_rmat(12, 16, seed=1, symmetric=False).to_device(with_transpose=False)
    with pytest.raises(ap.ApspieError, match="not symmetric"):
        ap.tc_prepare(ctx, g)


def test_tc_prepare_rejects_a_directed_graph_with_balanced_counts(ctx):
    """A directed graph whose entries below and above the degree order are
    equal in number (3 and 3: 0->1, 3->1, 3->2 below; 1->0, 0->3, 2->3
    above) is still refused: the hashes of its edges and of their reverses
    differ."""
    import apspie_b200 as ap
    rows = np.array([0, 0, 1, 2, 3, 3])
    cols = np.array([1, 3, 0, 3, 1, 2])
    g = ap.from_edges(4, rows, cols).to_device(with_transpose=False)
    with pytest.raises(ap.ApspieError, match="not symmetric"):
        ap.tc_prepare(ctx, g)


@pytest.mark.parametrize("scale", [12, 18])
def test_tc_rmat(ctx, scale):
    """R-MAT scale 18, edge factor 16, symmetrised: the TC configuration."""
    import apspie_b200 as ap
    count = _tc(ctx, ap.gen_rmat(scale, 16, seed=1))
    assert count > 0


def _sym(m, pairs):
    import apspie_b200 as ap
    e = np.asarray(pairs, dtype=np.int64)
    rows = np.concatenate([e[:, 0], e[:, 1]])
    cols = np.concatenate([e[:, 1], e[:, 0]])
    order = np.lexsort((cols, rows))
    return ap.from_edges(m, rows[order], cols[order])


@pytest.mark.parametrize("m", [6000, 1_200_000])
def test_tc_long_rows_both_set_forms(ctx, m):
    """A hub whose lower row has 5,000 entries (more than the hash-table bound
    of 4,096) and R-MAT 12 edges, spread over m vertex ids: m = 6,000 uses
    the shared-memory bitmap, m = 1.2 M (more than 2^20) the hash table and
    the binary search; the count matches the oracle either way."""
    import apspie_b200 as ap
    stride = (m - 1) // 5200
    hub, path = 0, [stride * (t + 1) for t in range(5000)]
    pairs = [(hub, p) for p in path] + [(path[t], path[t + 1]) for t in range(4999)]
    assert _tc(ctx, _sym(m, pairs)) == 4999
    r = ap.gen_rmat(12, 16, seed=3)
    src = np.repeat(np.arange(r.m), np.diff(r.ptr))
    keep = src < r.ind
    spread = lambda v: v.astype(np.int64) * ((m - 1) // r.m)
    _tc(ctx, _sym(m, np.stack([spread(src[keep]), spread(r.ind[keep])], axis=1)))
