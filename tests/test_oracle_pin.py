"""Pins the oracle to the reference's own CPU code.

The golden vectors in tests/golden/golden.npz were produced by the reference's
bfsCPU / ssspCPU / genrand_int32 compiled from its sources
(tests/golden/make_golden.py).  When oracle/_ref is present the oracle is also
compared live against the reference routines on synthetic graphs."""
import numpy as np
import pytest

import oracle


def _graph(golden, name, kind):
    return golden[f"mtx/{name}/{kind}_ptr"], golden[f"mtx/{name}/{kind}_ind"]


@pytest.mark.parametrize("kind", ["dir", "und"])
def test_oracle_bfs_matches_reference_goldens(golden, fixture_names, kind):
    for name in fixture_names:
        ptr, ind = _graph(golden, name, kind)
        m = len(ptr) - 1
        ref = golden[f"mtx/{name}/{kind}_bfs"]
        for s in range(m):
            d, _ = oracle.bfs(m, ptr, ind, s)
            np.testing.assert_array_equal(d, ref[s], err_msg=f"{name}/{kind} src {s}")


def test_oracle_sssp_matches_reference_goldens(golden, fixture_names):
    for name in fixture_names:
        ptr, ind = _graph(golden, name, "und")
        m = len(ptr) - 1
        w = golden[f"mtx/{name}/und_w"]
        ref = golden[f"mtx/{name}/und_sssp"]
        for s in range(m):
            d = oracle.sssp_f32(m, ptr, ind, w, s)
            # bit-exact: same float additions, same fixpoint
            np.testing.assert_array_equal(d.view(np.uint32), ref[s].view(np.uint32),
                                          err_msg=f"{name} src {s}")
            d64 = oracle.sssp_f64(m, ptr, ind, w, s)
            reach = ref[s] >= 0
            assert np.all(np.isinf(d64[~reach]))
            np.testing.assert_allclose(d64[reach], ref[s][reach], rtol=1e-6)


def test_oracle_mt19937_matches_reference(golden):
    for seed in (5489, 42):
        np.testing.assert_array_equal(oracle.mt_fill(seed, 2000), golden[f"mt/{seed}"])
    assert int(golden["mt/5489"][0]) == 3499211612  # known answer of genrand_int32


def test_oracle_on_rmat10_goldens(golden):
    import apspie_b200 as ap
    g = ap.gen_rmat(10, 16, seed=3, symmetric=True)
    for s, ref in zip(golden["rmat10/sym_src"], golden["rmat10/sym_bfs"]):
        np.testing.assert_array_equal(oracle.bfs(g.m, g.ptr, g.ind, int(s))[0], ref)
    gd = ap.gen_rmat(10, 16, seed=3, symmetric=False)
    wu = ap.weights_u32(gd, seed=11)
    wf = ap.weights_f32(gd, seed=11)
    for s, ru, rf in zip(golden["rmat10/sym_src"], golden["rmat10/dir_sssp_u32"],
                         golden["rmat10/dir_sssp_f32"]):
        du = oracle.sssp_u32(gd.m, gd.ptr, gd.ind, wu, int(s))
        expect = np.where(ru < 0, np.uint32(0xFFFFFFFF), ru.astype(np.uint32))
        np.testing.assert_array_equal(du, expect)
        df = oracle.sssp_f32(gd.m, gd.ptr, gd.ind, wf, int(s))
        np.testing.assert_array_equal(df.view(np.uint32), rf.view(np.uint32))


@pytest.mark.skipif(not oracle.have_reference(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_live_against_reference(seed):
    import apspie_b200 as ap
    g = ap.gen_rmat(12, 16, seed=seed, symmetric=True)
    for s in ap.seeded_sources(g, 2, seed=seed):
        np.testing.assert_array_equal(oracle.bfs(g.m, g.ptr, g.ind, s)[0],
                                      oracle.ref_bfs(g.m, g.ptr, g.ind, s)[0])
    gd = ap.gen_rmat(12, 16, seed=seed, symmetric=False)
    wf = ap.weights_f32(gd, seed=seed)
    s = ap.seeded_sources(gd, 1, seed=seed)[0]
    np.testing.assert_array_equal(oracle.sssp_f32(gd.m, gd.ptr, gd.ind, wf, s).view(np.uint32),
                                  oracle.ref_sssp(gd.m, gd.ptr, gd.ind, wf, s).view(np.uint32))
    np.testing.assert_array_equal(oracle.mt_fill(seed, 5000), oracle.ref_mt_fill(seed, 5000))


def test_oracle_mis_is_valid_greedy():
    import apspie_b200 as ap
    g = ap.gen_er(2000, 8, seed=5)
    prio = oracle.mt_fill(7, g.m)
    mis = oracle.mis(g.m, g.ptr, g.ind, prio)
    assert oracle.mis_check(g.m, g.ptr, g.ind, mis) == 0
    # the highest-priority vertex is always in the set
    assert mis[int(np.argmax(prio))] == 1
    # a planted mistake is caught: flip one member out
    bad = mis.copy()
    bad[int(np.flatnonzero(mis == 1)[0])] = 0
    assert oracle.mis_check(g.m, g.ptr, g.ind, bad) > 0


def test_oracle_tc_known_answers():
    import apspie_b200 as ap
    # K4 has 4 triangles; a 3x3 grid has none
    ptr = np.array([0, 3, 6, 9, 12], np.int32)
    ind = np.array([1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2], np.int32)
    _, lp, li = oracle.tc_build_lower(4, ptr, ind)
    assert oracle.tc_lower(4, lp, li) == 4
    g = ap.gen_grid(3, 3)
    _, lp, li = oracle.tc_build_lower(g.m, g.ptr, g.ind)
    assert oracle.tc_lower(g.m, lp, li) == 0


def test_oracle_spgemm_structure_keeps_cancellation():
    # A = [[1, -1]], B = [[1],[1]] -> C = [[0]] must stay as an explicit entry
    cp, ci, cv = oracle.spgemm(1, 1, [0, 2], [0, 1], [1.0, -1.0], [0, 1, 2], [0, 0], [1.0, 1.0])
    assert list(cp) == [0, 1] and list(ci) == [0] and cv[0] == 0.0


def test_oracle_tc_matches_reference_kernel_goldens(golden, fixture_names):
    """Triangle counts of the reference's own intersection kernel
    (ewiseMultTc, src/tc.cuh:168-199, run host-side on the U*L product as
    test/tc/main.cu:241-247 runs it) pin the oracle's L-masked count."""
    import apspie_b200 as ap
    graphs = {n: (golden[f"mtx/{n}/und_ptr"], golden[f"mtx/{n}/und_ind"]) for n in fixture_names}
    for sc in (10, 12):
        g = ap.gen_rmat(sc, 16, seed=3, symmetric=True)
        graphs[f"rmat{sc}"] = (g.ptr, g.ind)
    for name, (ptr, ind) in graphs.items():
        m = len(ptr) - 1
        _, lp, li = oracle.tc_build_lower(m, ptr, ind)
        assert oracle.tc_lower(m, lp, li) == int(golden[f"tc/{name}"][0]), name


def test_oracle_mis_matches_reference_kernel_goldens(golden):
    """MIS of the reference's own round kernels and loop (src/spmspvMis.cuh:
    10-78, 232-318) at two step sizes pins the oracle's greedy MIS: with
    distinct priorities both are the greedy set in descending priority."""
    names = sorted({k.split("/")[1] for k in golden if k.startswith("mis/")})
    assert len(names) >= 9
    for name in names:
        ptr, ind = golden[f"mis/{name}/ptr"], golden[f"mis/{name}/ind"]
        m = len(ptr) - 1
        got = oracle.mis(m, ptr, ind, oracle.mt_fill(5489, m))
        for delta in (0.1, 1.0):
            np.testing.assert_array_equal(got, golden[f"mis/{name}/d{delta}"].astype(np.int32),
                                          err_msg=f"{name} delta {delta}")


@pytest.mark.skipif(not oracle.have_reference(), reason="oracle/_ref not built")
def test_oracle_tc_live_against_reference_kernel():
    import apspie_b200 as ap
    for g in (ap.gen_rmat(12, 16, seed=1), ap.gen_rmat(11, 16, seed=2), ap.gen_er(3000, 12, seed=4),
              ap.gen_grid(20, 30)):
        _, lp, li = oracle.tc_build_lower(g.m, g.ptr, g.ind)
        assert oracle.ref_tc(g.m, g.ptr, g.ind) == oracle.tc_lower(g.m, lp, li)


@pytest.mark.skipif(not oracle.have_reference(), reason="oracle/_ref not built")
@pytest.mark.parametrize("delta", [0.05, 0.1, 1.0])
def test_oracle_mis_live_against_reference_kernels(delta):
    import apspie_b200 as ap
    for seed, g in ((5489, ap.gen_rmat(12, 16, seed=2)), (42, ap.gen_er(1 << 12, 8, seed=4)),
                    (7, ap.gen_grid(48, 48))):
        prio = oracle.mt_fill(seed, g.m)
        ref, rounds = oracle.ref_mis(g.m, g.ptr, g.ind, prio, delta)
        assert rounds > 0 and np.all(ref >= 0)
        np.testing.assert_array_equal(oracle.mis(g.m, g.ptr, g.ind, prio), ref)
    # a planted mistake in the oracle's answer is seen by the comparison
    bad = oracle.mis(g.m, g.ptr, g.ind, prio)
    bad[int(np.flatnonzero(bad == 1)[0])] = 0
    assert not np.array_equal(bad, ref)
