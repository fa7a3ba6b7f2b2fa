"""SSSP parity: apspie_sssp_{u32,f32} against the reference's CPU SSSP
(golden vectors and the compiled routine through the oracle): uint32
distances bit-exact, float distances bit-exact with the reference's float
label-correcting SSSP and within 1e-6 relative of FP64 Dijkstra."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

F32_REL_TOL = 1e-6   # tolerance of float SSSP against the FP64 oracle


def _unreached_f32(x):
    return np.isinf(x)


def test_sssp_fixtures_every_source(ctx, golden, fixture_names):
    import apspie_b200 as ap
    for name in fixture_names:
        ptr, ind = golden[f"mtx/{name}/und_ptr"], golden[f"mtx/{name}/und_ind"]
        h = ap.HostGraph(len(ptr) - 1, ptr, ind)
        h.w_f32 = golden[f"mtx/{name}/und_w"]
        g = h.to_device()
        ref = golden[f"mtx/{name}/und_sssp"]
        for s in range(h.m):
            d = ap.sssp(ctx, g, s, weights="f32").cpu().numpy()
            r = ref[s]
            assert np.array_equal(_unreached_f32(d), r == -1), f"{name} src {s}"
            np.testing.assert_array_equal(d[r >= 0].view(np.uint32), r[r >= 0].view(np.uint32))


def test_sssp_rmat10_goldens(ctx, golden):
    import apspie_b200 as ap
    h = ap.gen_rmat(10, 16, seed=3, symmetric=False)
    ap.weights_u32(h, seed=11)
    ap.weights_f32(h, seed=11)
    g = h.to_device()
    for s, ru, rf in zip(golden["rmat10/sym_src"], golden["rmat10/dir_sssp_u32"],
                         golden["rmat10/dir_sssp_f32"]):
        du = ap.sssp(ctx, g, int(s), weights="u32").cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(du, np.where(ru < 0, np.uint32(0xFFFFFFFF),
                                                   ru.astype(np.uint32)))
        df = ap.sssp(ctx, g, int(s), weights="f32").cpu().numpy()
        assert np.array_equal(np.isinf(df), rf == -1)
        np.testing.assert_array_equal(df[rf >= 0].view(np.uint32), rf[rf >= 0].view(np.uint32))


def _check_against_oracle(ctx, h, g, s):
    import apspie_b200 as ap
    du = ap.sssp(ctx, g, s, weights="u32").cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(du, oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, s))
    st = ap.sssp_stats(ctx)
    reach = du != 0xFFFFFFFF
    assert st["vertices_reached"] == int(reach.sum())
    assert st["edges_traversed"] == int(h.degrees()[reach].sum())
    assert st["relaxations"] >= st["edges_traversed"]
    df = ap.sssp(ctx, g, s, weights="f32").cpu().numpy()
    ref32 = oracle.sssp_f32(h.m, h.ptr, h.ind, h.w_f32, s)
    ref64 = oracle.sssp_f64(h.m, h.ptr, h.ind, h.w_f32, s)
    assert np.array_equal(np.isinf(df), ref32 == -1)
    fin = ~np.isinf(df)
    np.testing.assert_array_equal(df[fin].view(np.uint32), ref32[fin].view(np.uint32))
    rel = np.abs(df[fin] - ref64[fin]) / np.maximum(ref64[fin], 1e-30)
    rel[ref64[fin] == 0] = 0
    assert rel.max(initial=0) <= F32_REL_TOL, rel.max()
    return rel.max(initial=0)


@pytest.mark.parametrize("scale,symmetric", [(12, False), (14, False), (14, True)])
def test_sssp_rmat_vs_oracle(ctx, scale, symmetric):
    import apspie_b200 as ap
    h = ap.gen_rmat(scale, 16, seed=scale + 1, symmetric=symmetric)
    ap.weights_u32(h, seed=5)
    ap.weights_f32(h, seed=5)
    g = h.to_device()
    for s in ap.seeded_sources(h, 3, seed=2) + [int(np.argmax(h.degrees()))]:
        _check_against_oracle(ctx, h, g, s)


@pytest.mark.parametrize("scale,symmetric", [(12, False), (14, True)])
@pytest.mark.parametrize("alpha", [3, 1 << 20])
def test_sssp_pull_rounds_same_fixpoint(ctx, scale, symmetric, alpha):
    """Push/pull SSSP over the in-adjacency (default switch point, and pull
    in every round after the first): same distances as the oracle, and the
    pull rounds did run (each scans all nnz in-edges)."""
    import apspie_b200 as ap
    h = ap.gen_rmat(scale, 16, seed=scale + 7, symmetric=symmetric)
    ap.weights_u32(h, seed=6)
    ap.weights_f32(h, seed=6)
    g = ap.sssp_prepare(ctx, h.to_device())
    ap.sssp_set_pull(ctx, alpha)
    try:
        for s in ap.seeded_sources(h, 3, seed=4) + [int(np.argmax(h.degrees()))]:
            _check_against_oracle(ctx, h, g, s)
            if alpha > 3:
                assert ap.sssp_stats(ctx)["relaxations"] >= h.nnz
    finally:
        ap.sssp_set_pull(ctx)


def test_sssp_edge_cases(ctx):
    import apspie_b200 as ap
    h = ap.HostGraph(4, np.array([0, 2, 2, 3, 3], np.int32), np.array([1, 2, 1], np.int32))
    h.w_u32 = np.array([5, 1, 1], np.uint32)
    h.w_f32 = np.array([5, 1, 1], np.float32)
    g = h.to_device()
    # 0->1 (5), 0->2 (1), 2->1 (1), 3 unreachable: the reference's own probe graph
    np.testing.assert_array_equal(ap.sssp(ctx, g, 0).cpu().numpy().view(np.uint32),
                                  [0, 2, 1, 0xFFFFFFFF])
    np.testing.assert_array_equal(ap.sssp(ctx, g, 0, weights="f32").cpu().numpy(),
                                  [0, 2, 1, np.inf])
    np.testing.assert_array_equal(ap.sssp(ctx, g, 3).cpu().numpy().view(np.uint32),
                                  [0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0])
    # one round only reaches the out-neighbours of the source
    np.testing.assert_array_equal(ap.sssp(ctx, g, 0, max_rounds=1).cpu().numpy().view(np.uint32),
                                  [0, 5, 1, 0xFFFFFFFF])
    with pytest.raises(ap.ApspieError):
        ap.sssp(ctx, g, -1)


def test_sssp_rmat20_full_size(ctx):
    """The SSSP benchmark graph (R-MAT 20 directed), both weight variants."""
    import apspie_b200 as ap
    h = ap.gen_rmat(20, 16, seed=1, symmetric=False)
    ap.weights_u32(h, seed=1)
    ap.weights_f32(h, seed=1)
    g = h.to_device()
    s = ap.seeded_sources(h, 1, seed=0)[0]
    rel = _check_against_oracle(ctx, h, g, s)
    assert rel <= F32_REL_TOL


@pytest.mark.parametrize("delta_u32,delta_f32", [(16, 0.05), (256, 0.5), (1 << 31, 1e30)])
def test_sssp_near_far_same_fixpoint(ctx, delta_u32, delta_f32):
    """Near-far schedules give exactly the delta-0 distances (u32 against the
    oracle's Dijkstra, f32 against the reference's float SSSP), on a directed
    R-MAT and on a grid, whose many phases exercise the far lists."""
    import apspie_b200 as ap
    cases = [ap.gen_rmat(13, 16, seed=31, symmetric=False), ap.gen_grid(40, 60)]
    try:
        for h in cases:
            ap.weights_u32(h, seed=4)
            ap.weights_f32(h, seed=4)
            g = h.to_device()
            ap.sssp_set_params(ctx, delta_u32, delta_f32)
            for s in ap.seeded_sources(h, 3, seed=5):
                du = ap.sssp(ctx, g, s, weights="u32").cpu().numpy().view(np.uint32)
                np.testing.assert_array_equal(du, oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, s))
                st = ap.sssp_stats(ctx)
                if delta_u32 < 1 << 20 and h.m == 2400:
                    assert st["phases"] > 0
                df = ap.sssp(ctx, g, s, weights="f32").cpu().numpy()
                ref = oracle.sssp_f32(h.m, h.ptr, h.ind, h.w_f32, s)
                assert np.array_equal(np.isinf(df), ref == -1)
                fin = ~np.isinf(df)
                np.testing.assert_array_equal(df[fin].view(np.uint32), ref[fin].view(np.uint32))
    finally:
        ap.sssp_set_params(ctx, 0, 0.0)


def test_sssp_trace_accounts_for_every_round(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(14, 16, seed=32, symmetric=False)
    ap.weights_u32(h, seed=6)
    g = h.to_device()
    ap.sssp(ctx, g, ap.seeded_sources(h, 1, seed=7)[0], weights="u32")
    st, tr = ap.sssp_stats(ctx), ap.sssp_trace(ctx)
    assert len(tr) == st["rounds"]
    # relaxations count the edges walked: every reached vertex's edges at
    # least once (with its final distance), at most every frontier's edges
    # (a queued vertex already expanded with its current distance is skipped)
    assert st["edges_traversed"] <= st["relaxations"] <= sum(t["frontier_edges"] for t in tr)
    assert tr[0]["frontier"] == 1 and all(t["us"] > 0 for t in tr)


def test_persistent_kernels_with_a_capped_grid(ctx):
    """A context whose persistent launches are capped to a few blocks (the
    server's small-grid lane) gives the same BFS depths and SSSP distances."""
    import apspie_b200 as ap
    from apspie_b200._native import lib
    h = ap.gen_rmat(13, 16, seed=33)
    ap.weights_u32(h, seed=8)
    g = h.to_device()
    srcs = ap.seeded_sources(h, 3, seed=9)
    full = [(ap.bfs(ctx, g, s).cpu().numpy(), ap.sssp(ctx, g, s, weights="u32").cpu().numpy())
            for s in srcs]
    assert lib.apspie_ctx_set_max_grid(ctx.handle, 4) == 0
    try:
        for s, (d0, w0) in zip(srcs, full):
            np.testing.assert_array_equal(ap.bfs(ctx, g, s).cpu().numpy(), d0)
            np.testing.assert_array_equal(ap.sssp(ctx, g, s, weights="u32").cpu().numpy(), w0)
    finally:
        lib.apspie_ctx_set_max_grid(ctx.handle, 0)
