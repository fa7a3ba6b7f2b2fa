"""The oracle against independent code (SciPy), on CPU: for the routines no
reference code can run here (SpGEMM, whose reference arithmetic lives in
absent moderngpu / cuSPARSE code; the SpMSpV semirings) and as a second pin
for the rest (u32 / f64 SSSP against Dijkstra, BFS against an unweighted
shortest path, triangle counts against trace(A^3) / 6, the MIS against
Luby's rounds run in NumPy).  SpGEMM and
plus-times SpMSpV sum in a different order here, so their values agree to
1e-12 relative; everything else is exact."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse import csgraph

import apspie_b200 as ap
import oracle

RTOL = 1e-12


def _csr(h, vals=None):
    v = np.ones(h.nnz) if vals is None else np.asarray(vals, np.float64)
    return sp.csr_matrix((v, h.ind, h.ptr), shape=(h.m, getattr(h, "ncols", h.m)))


@pytest.mark.parametrize("seed", [1, 2])
def test_spgemm_oracle_against_scipy(seed):
    A = ap.gen_powerlaw(1 << 10, 1 << 9, max_deg=256, seed=seed)
    B = ap.gen_powerlaw(1 << 9, 1 << 11, max_deg=256, seed=seed + 10)
    cp, ci, cv = oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, A.w_f32, B.ptr, B.ind, B.w_f32)
    # structure: the pattern product (no cancellation possible)
    pat = (_csr(A) @ _csr(B)).tocsr()
    pat.sort_indices()
    np.testing.assert_array_equal(cp, pat.indptr)
    np.testing.assert_array_equal(ci, pat.indices)
    # values: the FP64 product of the same float32 inputs
    ref = (_csr(A, A.w_f32) @ _csr(B, B.w_f32)).tocsr()
    dense_ref = np.asarray(ref[np.repeat(np.arange(A.m), np.diff(cp)), ci]).ravel()
    mag = np.asarray((abs(_csr(A, A.w_f32)) @ abs(_csr(B, B.w_f32)))
                     [np.repeat(np.arange(A.m), np.diff(cp)), ci]).ravel()
    assert np.all(np.abs(cv - dense_ref) <= RTOL * mag)


@pytest.mark.parametrize("semiring", [0, 1, 2, 3])
def test_spmspv_oracle_against_scipy(semiring):
    h = ap.gen_rmat(11, 16, seed=5, symmetric=False)
    rng = np.random.default_rng(semiring)
    val = rng.uniform(0.1, 2.0, h.nnz).astype(np.float32)
    xind = np.flatnonzero(rng.random(h.m) < 0.05).astype(np.int32)
    xval = rng.uniform(0.1, 2.0, xind.size).astype(np.float32)
    yi, yv = oracle.spmspv(semiring, h.m, h.ptr, h.ind, val, xind, xval)
    # rows reached: out-neighbours of the frontier (row j of the CSR lists j's targets)
    frontier = np.zeros(h.m)
    frontier[xind] = 1.0
    reach = _csr(h).T @ frontier
    np.testing.assert_array_equal(yi, np.flatnonzero(reach > 0))
    # values, per semiring, from the edge list
    rows = np.repeat(np.arange(h.m), np.diff(h.ptr))
    xfull = np.zeros(h.m, np.float32)
    xfull[xind] = xval
    on = np.isin(rows, xind)
    tgt, a, xv = h.ind[on], val[on], xfull[rows[on]]
    if semiring == 0:
        y = _csr(h, val).T @ xfull.astype(np.float64)
        mag = _csr(h, np.abs(val)).T @ np.abs(xfull).astype(np.float64)
        assert np.all(np.abs(yv - y[yi]) <= RTOL * mag[yi])
    else:
        if semiring == 1:
            term, init, red = (a + xv).astype(np.float32), np.inf, np.minimum
        elif semiring == 2:
            term, init, red = (a * xv).astype(np.float32), -np.inf, np.maximum
        else:
            term, init, red = np.ones(tgt.size), -np.inf, np.maximum
        y = np.full(h.m, init)
        red.at(y, tgt, term.astype(np.float64))
        np.testing.assert_array_equal(yv, y[yi])


def test_sssp_oracles_against_dijkstra():
    h = ap.gen_rmat(11, 16, seed=3, symmetric=False)
    wu = ap.weights_u32(h, seed=3)
    wf = ap.weights_f32(h, seed=3)
    src = ap.seeded_sources(h, 1, seed=1)[0]
    du = oracle.sssp_u32(h.m, h.ptr, h.ind, wu, src)
    ref = csgraph.dijkstra(_csr(h, wu.astype(np.float64)), directed=True, indices=src)
    exp = np.where(np.isinf(ref), 0xFFFFFFFF, ref).astype(np.uint64)
    np.testing.assert_array_equal(du.astype(np.uint64), exp)
    df = oracle.sssp_f64(h.m, h.ptr, h.ind, wf, src)
    reff = csgraph.dijkstra(_csr(h, wf.astype(np.float64)), directed=True, indices=src)
    fin = np.isfinite(reff)
    np.testing.assert_array_equal(np.isfinite(df), fin)
    np.testing.assert_allclose(df[fin], reff[fin], rtol=RTOL, atol=0)


def test_bfs_oracle_against_unweighted_shortest_paths():
    h = ap.gen_rmat(11, 16, seed=4, symmetric=False)
    src = ap.seeded_sources(h, 1, seed=2)[0]
    d, _ = oracle.bfs(h.m, h.ptr, h.ind, src)
    ref = csgraph.shortest_path(_csr(h), directed=True, unweighted=True, indices=src)
    np.testing.assert_array_equal(d, np.where(np.isinf(ref), -1, ref).astype(np.int32))


@pytest.mark.parametrize("scale", [9, 11])
def test_tc_oracle_against_trace_of_a_cubed(scale):
    h = ap.gen_rmat(scale, 16, seed=scale)
    A = _csr(h)
    A.setdiag(0)
    A.eliminate_zeros()
    ref = int(round((A @ A).multiply(A).sum() / 6))
    _, lp, li = oracle.tc_build_lower(h.m, h.ptr, h.ind)
    assert oracle.tc_lower(h.m, lp, li) == ref


def _luby_rounds(m, ptr, ind, prio):
    """Luby's rounds, vectorised: every undecided vertex whose key (priority,
    then id) beats all its undecided neighbours joins; their undecided
    neighbours leave; repeat.  The reference's round loop
    (src/spmspvMis.cuh:232-318) in plain NumPy, independent of the oracle's
    one-pass greedy form."""
    key = (prio.astype(np.uint64) << np.uint64(32)) | np.arange(m, dtype=np.uint64)
    rows = np.repeat(np.arange(m), np.diff(ptr))
    cols = ind.astype(np.int64)
    off = rows != cols
    state = np.full(m, -1)
    for _ in range(m + 1):
        und = state == -1
        if not und.any():
            break
        live = off & und[rows] & und[cols]
        nbmax = np.zeros(m, np.uint64)
        np.maximum.at(nbmax, rows[live], key[cols[live]])
        has_nb = np.zeros(m, bool)
        has_nb[rows[live]] = True
        join = und & (~has_nb | (key > nbmax))
        state[join] = 1
        drop = off & join[rows] & (state[cols] == -1)
        state[cols[drop]] = 0
    return state


@pytest.mark.parametrize("which", ["rmat", "er", "grid"])
def test_mis_oracle_against_luby_rounds(which):
    g = {"rmat": lambda: ap.gen_rmat(11, 16, seed=6),
         "er": lambda: ap.gen_er(1 << 11, 8, seed=6),
         "grid": lambda: ap.gen_grid(40, 50)}[which]()
    prio = ap.mt19937(5489, g.m)
    ref = _luby_rounds(g.m, g.ptr, g.ind, prio)
    assert np.all(ref >= 0)
    np.testing.assert_array_equal(oracle.mis(g.m, g.ptr, g.ind, prio), ref)
