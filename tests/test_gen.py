"""Host graph builders: sizes of the benchmark configurations, structural
invariants, determinism, and the .mtx ingest orientation."""
import numpy as np
import pytest

import apspie_b200 as ap

REF_SMALL = ["test_cc", "test_bc", "test_pr", "test_spgemm", "test_mis", "test_mesh", "chesapeake"]


def _check_simple(g, symmetric):
    src = np.repeat(np.arange(g.m), np.diff(g.ptr))
    assert np.all(src != g.ind), "self-loop"
    key = src.astype(np.int64) * g.m + g.ind
    assert np.all(np.diff(key) > 0), "rows must be sorted, no duplicates"
    if symmetric:
        rev = np.sort(g.ind.astype(np.int64) * g.m + src)
        np.testing.assert_array_equal(rev, key)


def test_rmat14_config_sizes_and_invariants():
    g = ap.gen_rmat(14, 16, seed=1)
    assert g.m == 16384
    assert 400_000 < g.nnz < 450_000
    _check_simple(g, True)
    again = ap.gen_rmat(14, 16, seed=1)
    np.testing.assert_array_equal(g.ind, again.ind)
    other = ap.gen_rmat(14, 16, seed=2)
    assert not np.array_equal(g.ind[:1000], other.ind[:1000])


def test_rmat_directed_and_unscrambled():
    g = ap.gen_rmat(12, 16, seed=4, symmetric=False, scramble=False)
    _check_simple(g, False)
    deg = g.degrees()
    # without the scramble vertex 0 is the (0,0)-quadrant hub
    assert deg[0] == deg.max()


def test_er_and_grid_sizes():
    g = ap.gen_er(1 << 14, 8, seed=1)
    _check_simple(g, True)
    assert abs(g.nnz - (1 << 14) * 8) < 200
    grid = ap.gen_grid(1024, 1024)
    assert grid.nnz == 4_190_208
    _check_simple(grid, True)
    small = ap.gen_grid(2, 3)
    np.testing.assert_array_equal(small.degrees(), [2, 3, 2, 2, 3, 2])


def test_weights_ranges_and_order_independence():
    g = ap.gen_rmat(10, 16, seed=1, symmetric=False)
    wu = ap.weights_u32(g, seed=3)
    wf = ap.weights_f32(g, seed=3)
    assert wu.min() >= 1 and wu.max() <= 255 and len(np.unique(wu)) > 200
    assert wf.min() > 0 and wf.max() <= 1
    assert np.all((wf * (1 << 24)) == np.round(wf * (1 << 24)))
    # weight is a function of (row, col): a reversed-row CSR gets the same weights per edge
    src = np.repeat(np.arange(g.m), np.diff(g.ptr))
    perm = np.lexsort((-g.ind, src))
    g2 = ap.HostGraph(g.m, g.ptr, g.ind[perm].copy())
    np.testing.assert_array_equal(ap.weights_u32(g2, seed=3), wu[perm])


def test_mt19937_known_answer():
    assert int(ap.mt19937(5489, 1)[0]) == 3499211612


def test_generator_pinned_by_golden_hash(golden):
    import hashlib

    def sha(*arrays):
        h = hashlib.sha256()
        for a in arrays:
            h.update(np.ascontiguousarray(a).tobytes())
        return h.hexdigest().encode()

    g = ap.gen_rmat(10, 16, seed=3, symmetric=True)
    assert sha(g.ptr, g.ind) == golden["rmat10/sym_sha"].tobytes()
    gd = ap.gen_rmat(10, 16, seed=3, symmetric=False)
    assert sha(gd.ptr, gd.ind, ap.weights_u32(gd, seed=11),
               ap.weights_f32(gd, seed=11)) == golden["rmat10/dir_sha"].tobytes()


def test_mtx_ingest_matches_reference_orientation(golden, tmp_path):
    """read_mtx parses as readMtx + buildMatrix / makeSymmetric: the goldens
    hold the CSR the golden script derived from the reference's .mtx files.
    The files themselves are regenerated here from the golden CSR."""
    for name in REF_SMALL:
        ptr = golden[f"mtx/{name}/dir_ptr"]
        ind = golden[f"mtx/{name}/dir_ind"]
        m = len(ptr) - 1
        rows = np.repeat(np.arange(m), np.diff(ptr))
        path = tmp_path / f"{name}.mtx"
        with open(path, "w") as f:
            f.write("%%MatrixMarket matrix coordinate pattern general\n% comment\n")
            f.write(f"{m} {m} {len(ind)}\n")
            for r, c in zip(rows, ind):
                f.write(f"{c + 1} {r + 1}\n")   # first index = column
        g = ap.read_mtx(path)
        np.testing.assert_array_equal(g.ptr, ptr)
        np.testing.assert_array_equal(g.ind, ind)
        gu = ap.read_mtx(path, undirected=True)
        np.testing.assert_array_equal(gu.ptr, golden[f"mtx/{name}/und_ptr"])
        np.testing.assert_array_equal(gu.ind, golden[f"mtx/{name}/und_ind"])


def test_mtx_weighted_and_malformed(tmp_path):
    p = tmp_path / "w.mtx"
    p.write_text("3 3 2\n2 1 0.5\n3 2 2.5\n")
    g = ap.read_mtx(p)
    np.testing.assert_array_equal(g.ptr, [0, 1, 2, 2])
    np.testing.assert_array_equal(g.ind, [1, 2])
    np.testing.assert_array_equal(g.w_f32, [0.5, 2.5])
    bad = tmp_path / "bad.mtx"
    bad.write_text("3 3 1\n7 1\n")
    with pytest.raises(ap.ApspieError):
        ap.read_mtx(bad)
    # a header that promises far more entries than the file holds: the count
    # is a hint (nothing of its size is allocated); the entries present are read
    short = tmp_path / "short.mtx"
    short.write_text("4 4 2000000000\n2 1\n4 3\n")
    g = ap.read_mtx(short, undirected=True)
    np.testing.assert_array_equal(g.ptr, [0, 1, 2, 3, 4])
    np.testing.assert_array_equal(g.ind, [1, 0, 3, 2])
    missing = tmp_path / "none.mtx"
    with pytest.raises(ap.ApspieError):
        ap.read_mtx(missing)


def test_transpose_host():
    g = ap.gen_rmat(10, 8, seed=2, symmetric=False)
    t = g.transpose()
    tt = t.transpose()
    np.testing.assert_array_equal(tt.ptr, g.ptr)
    np.testing.assert_array_equal(tt.ind, g.ind)
    assert t.nnz == g.nnz
    sym = ap.gen_rmat(10, 8, seed=2)
    st = sym.transpose()
    np.testing.assert_array_equal(st.ind, sym.ind)


def test_numpy_rmat_restatement_equals_builder(golden):
    """oracle.inputs (the reference arm's input builder, which loads none of
    the library) gives the library's R-MAT graphs and sources bit for bit,
    and the golden hash of R-MAT 10."""
    import hashlib
    import oracle.inputs as oi
    for scale, sym, seed in ((10, True, 3), (11, False, 5), (13, True, 1)):
        m, ptr, ind = oi.gen_rmat(scale, 16, seed=seed, symmetric=sym, chunk=1 << 10)
        g = ap.gen_rmat(scale, 16, seed=seed, symmetric=sym)
        np.testing.assert_array_equal(ptr, g.ptr)
        np.testing.assert_array_equal(ind, g.ind)
        assert oi.seeded_sources(m, ptr, ind, 6, seed=2) == ap.seeded_sources(g, 6, seed=2)
    m, ptr, ind = oi.gen_rmat(10, 16, seed=3, symmetric=True)
    h = hashlib.sha256()
    for a in (ptr, ind):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest().encode() == golden["rmat10/sym_sha"].tobytes()
