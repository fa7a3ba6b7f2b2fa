"""BFS parity: apspie_bfs (sm_100a, through the C ABI) against the reference's
CPU BFS (golden vectors) and the oracle, bit-exact, including the fixed
iteration count of the reference driver and both traversal directions."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _dev(ptr, ind):
    import apspie_b200 as ap
    return ap.HostGraph(len(ptr) - 1, np.asarray(ptr, np.int32), np.asarray(ind, np.int32)).to_device()


@pytest.mark.parametrize("kind", ["dir", "und"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_bfs_fixtures_every_source(ctx, golden, fixture_names, kind, mode):
    import apspie_b200 as ap
    ap.bfs_set_params(ctx, mode=mode)
    try:
        for name in fixture_names:
            ptr, ind = golden[f"mtx/{name}/{kind}_ptr"], golden[f"mtx/{name}/{kind}_ind"]
            g = _dev(ptr, ind)
            ref = golden[f"mtx/{name}/{kind}_bfs"]
            for s in range(g.m):
                d = ap.bfs(ctx, g, s).cpu().numpy()
                np.testing.assert_array_equal(d, ref[s], err_msg=f"{name}/{kind} src {s}")
                st = ap.bfs_stats(ctx)
                assert st["levels"] == int(ref[s].max()) + 1
                assert st["vertices_reached"] == int((ref[s] >= 0).sum())
    finally:
        ap.bfs_set_params(ctx)


@pytest.mark.parametrize("scale,symmetric", [(14, True), (16, True), (14, False)])
def test_bfs_rmat_vs_oracle(ctx, scale, symmetric):
    import apspie_b200 as ap
    h = ap.gen_rmat(scale, 16, seed=scale, symmetric=symmetric)
    g = h.to_device()
    deg = h.degrees()
    for s in ap.seeded_sources(h, 6, seed=1) + [int(np.argmax(deg))]:
        d = ap.bfs(ctx, g, s).cpu().numpy()
        ref, depth = oracle.bfs(h.m, h.ptr, h.ind, s)
        np.testing.assert_array_equal(d, ref)
        st = ap.bfs_stats(ctx)
        assert st["levels"] == depth
        assert st["edges_traversed"] == int(deg[ref >= 0].sum())


def test_bfs_directions_agree(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(15, 16, seed=9)
    g = h.to_device()
    s = ap.seeded_sources(h, 1, seed=2)[0]
    ref, _ = oracle.bfs(h.m, h.ptr, h.ind, s)
    pulls = []
    try:
        for mode in (0, 1, 2):
            ap.bfs_set_params(ctx, mode=mode)
            np.testing.assert_array_equal(ap.bfs(ctx, g, s).cpu().numpy(), ref)
            pulls.append(ap.bfs_stats(ctx)["pull_levels"])
    finally:
        ap.bfs_set_params(ctx)
    assert pulls[1] == 0 and pulls[2] > 0 and pulls[0] > 0


def test_bfs_fixed_iteration_count(ctx):
    """max_levels = the reference driver's `depth` argument (src/bfs.cuh:87)."""
    import apspie_b200 as ap
    h = ap.gen_rmat(13, 16, seed=4)
    g = h.to_device()
    s = ap.seeded_sources(h, 1, seed=3)[0]
    full, depth = oracle.bfs(h.m, h.ptr, h.ind, s)
    for k in (1, 2, 3, depth, depth + 5):
        d = ap.bfs(ctx, g, s, max_levels=k).cpu().numpy()
        expect = np.where(full < k, full, -1) if k < depth else full
        np.testing.assert_array_equal(d, expect, err_msg=f"max_levels={k}")


def test_bfs_edge_cases(ctx):
    import apspie_b200 as ap
    # isolated source, single vertex, edgeless graph
    g = _dev([0, 0, 1, 2], [2, 1])
    np.testing.assert_array_equal(ap.bfs(ctx, g, 0).cpu().numpy(), [0, -1, -1])
    np.testing.assert_array_equal(ap.bfs(ctx, g, 1).cpu().numpy(), [-1, 0, 1])
    g1 = _dev([0, 0], [])
    np.testing.assert_array_equal(ap.bfs(ctx, g1, 0).cpu().numpy(), [0])
    # a hub above the chunking threshold and a long path (many levels)
    n = 5000
    rows = np.concatenate([np.zeros(n - 1, np.int64), np.arange(1, n)])
    cols = np.concatenate([np.arange(1, n), np.zeros(n - 1, np.int64)])
    star = ap.from_edges(n, rows, cols)
    ref, _ = oracle.bfs(n, star.ptr, star.ind, 7)
    np.testing.assert_array_equal(ap.bfs(ctx, star.to_device(), 7).cpu().numpy(), ref)
    grid = ap.gen_grid(256, 256)
    ref, depth = oracle.bfs(grid.m, grid.ptr, grid.ind, 0)
    np.testing.assert_array_equal(ap.bfs(ctx, grid.to_device(), 0).cpu().numpy(), ref)
    assert ap.bfs_stats(ctx)["levels"] == depth == 511
    with pytest.raises(ap.ApspieError):
        ap.bfs(ctx, grid.to_device(), grid.m)


def test_bfs_rmat22_full_size(ctx):
    """The benchmark graph: bit-exact against the oracle at full size."""
    import apspie_b200 as ap
    h = ap.gen_rmat(22, 16, seed=1)
    g = h.to_device()
    s = ap.seeded_sources(h, 1, seed=0)[0]
    d = ap.bfs(ctx, g, s).cpu().numpy()
    ref, depth = oracle.bfs(h.m, h.ptr, h.ind, s)
    np.testing.assert_array_equal(d, ref)
    st = ap.bfs_stats(ctx)
    assert st["levels"] == depth and st["pull_levels"] > 0
    assert st["edges_traversed"] == int(h.degrees()[ref >= 0].sum())


def test_bfs_repeated_runs_with_direction_switches(ctx):
    """Repeated traversals that switch push -> pull -> push are all exact.
    (A frontier rebuilt for a push level once shared its counters with the
    level's direction decision; slower blocks then chose a different
    direction in a few percent of the runs.)"""
    import apspie_b200 as ap
    h = ap.gen_rmat(16, 16, seed=16)
    g = h.to_device()
    for s in (2300, 30945):
        ref, _ = oracle.bfs(h.m, h.ptr, h.ind, s)
        dirs = None
        for _ in range(40):
            np.testing.assert_array_equal(ap.bfs(ctx, g, s).cpu().numpy(), ref)
            tr = ap.bfs_trace(ctx)
            dirs = [t["dir"] for t in tr]
            for t in tr:
                if t["dir"] == "push":
                    assert t["expanded"] == t["frontier_edges"]
                    if t["queued"]:
                        assert t["queued"] == t["frontier"]
        assert "pull" in dirs and dirs[-1] == "push"


@pytest.mark.parametrize("symmetric", [True, False])
@pytest.mark.parametrize("mode", [0, 2])
def test_bfs_prepared_in_adjacency(ctx, symmetric, mode):
    """apspie_bfs_prepare: each in-row is the set of in-neighbours ordered by
    out-degree (highest first, ties by id), and BFS over it gives the same
    depths as the oracle."""
    import apspie_b200 as ap
    h = ap.gen_rmat(14, 16, seed=21, symmetric=symmetric)
    g = ap.bfs_prepare(ctx, h.to_device(with_transpose=False))
    tptr, tind = g.tptr.cpu().numpy(), g.tind.cpu().numpy()
    tr = h.transpose()
    deg = np.diff(h.ptr)
    np.testing.assert_array_equal(tptr, tr.ptr)
    for v in range(0, h.m, 97):
        row = tind[tptr[v]:tptr[v + 1]]
        exp = sorted(tr.ind[tr.ptr[v]:tr.ptr[v + 1]], key=lambda u: (-deg[u], u))
        np.testing.assert_array_equal(row, exp, err_msg=f"row {v}")
    ap.bfs_set_params(ctx, mode=mode)
    try:
        for s in ap.seeded_sources(h, 6, seed=2):
            ref, _ = oracle.bfs(h.m, h.ptr, h.ind, s)
            np.testing.assert_array_equal(ap.bfs(ctx, g, s).cpu().numpy(), ref)
    finally:
        ap.bfs_set_params(ctx, mode=0)
