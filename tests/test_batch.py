"""Batched traversal (many BFS / SSSP sources on uneven graphs in one
persistent launch): every source's result equals the plain single-source
path and the oracle, bit for bit."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _graphs():
    import apspie_b200 as ap
    a = ap.gen_rmat(12, 16, seed=5)
    b = ap.gen_rmat(14, 16, seed=6)
    c = ap.gen_grid(64, 64)
    d = ap.gen_rmat(12, 16, seed=7, symmetric=False)
    ap.weights_u32(d, seed=2)
    ap.weights_u32(a, seed=3)
    return a, b, c, d


@pytest.fixture(params=[48, 3, 0], ids=["deep-single-source", "deep-3-streams", "deep-multi-source"])
def deep_mode(ctx, request):
    """Jobs on the deep grids as concurrent single-source traversals (the
    default; or fewer sub-contexts than sources) or inside the multi-source
    launch."""
    import apspie_b200 as ap
    ap.batch_set_params(ctx, 0, request.param)
    yield request.param
    ap.batch_set_params(ctx)


def test_batch_bfs_and_sssp_mixed(ctx, deep_mode):
    import apspie_b200 as ap
    a, b, c, d = _graphs()
    ga, gb, gc, gd = (x.to_device() for x in (a, b, c, d))
    rng = np.random.default_rng(0)
    jobs = [
        {"type": "bfs", "graph": ga, "sources": ap.seeded_sources(a, 40, seed=1)},
        {"type": "bfs", "graph": gb, "sources": ap.seeded_sources(b, 100, seed=2)},  # 2 device jobs
        {"type": "bfs", "graph": gc, "sources": [0, 4095, 2080, 2080]},              # duplicate
        {"type": "bfs", "graph": gd, "sources": [int(x) for x in rng.integers(0, d.m, 9)]},
        {"type": "sssp", "graph": gd, "sources": ap.seeded_sources(d, 20, seed=3)},
        {"type": "sssp", "graph": ga, "sources": ap.seeded_sources(a, 5, seed=4)},
    ]
    outs = ap.batch_run(ctx, jobs)
    st = ap.batch_stats(ctx)
    assert st["super_steps"] >= 127  # the 64 x 64 grid from a corner has 127 levels
    for jd, out, h in zip(jobs, outs, (a, b, c, d, d, a)):
        out = out.cpu().numpy()
        for i, s in enumerate(jd["sources"]):
            if jd["type"] == "bfs":
                ref, _ = oracle.bfs(h.m, h.ptr, h.ind, s)
                np.testing.assert_array_equal(out[i], ref, err_msg=f"bfs {h.name} src {s}")
            else:
                ref = oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, s)
                np.testing.assert_array_equal(out[i].view(np.uint32), ref,
                                              err_msg=f"sssp {h.name} src {s}")


def test_batch_equals_single_source_path(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(16, 16, seed=9)
    g = h.to_device()
    srcs = ap.seeded_sources(h, 64, seed=5)
    out = ap.batch_run(ctx, [{"type": "bfs", "graph": g, "sources": srcs}])[0].cpu().numpy()
    for i, s in enumerate(srcs):
        np.testing.assert_array_equal(out[i], ap.bfs(ctx, g, s).cpu().numpy())


def test_batch_forced_push_and_pull(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(13, 16, seed=11)
    g = h.to_device()
    srcs = ap.seeded_sources(h, 30, seed=6)
    refs = [oracle.bfs(h.m, h.ptr, h.ind, s)[0] for s in srcs]
    for alpha, beta in ((0, 24), (1 << 20, 1 << 30)):   # never pull / pull early and stay
        out = ap.batch_run(ctx, [{"type": "bfs", "graph": g, "sources": srcs, "alpha": alpha,
                                  "beta": beta}])[0].cpu().numpy()
        for i in range(len(srcs)):
            np.testing.assert_array_equal(out[i], refs[i])


@pytest.mark.parametrize("alpha", [2, 1 << 20])
def test_batch_sssp_pull_steps(ctx, alpha):
    """Multi-source SSSP with the in-adjacency and weights: pull steps when the
    frontier's out-edges pass nnz / 2 and in every step after the first, on a symmetric
    R-MAT with hubs of more than 1024 in-edges (chunked) and on a directed
    one; every row equals the oracle's Dijkstra."""
    import apspie_b200 as ap
    r = ap.gen_rmat(15, 16, seed=21)
    ap.weights_u32(r, seed=8)
    assert (r.degrees() > 1024).any()
    dd = ap.gen_rmat(12, 8, seed=22, symmetric=False)
    ap.weights_u32(dd, seed=9)
    gr = ap.sssp_prepare(ctx, r.to_device())
    gd = ap.sssp_prepare(ctx, dd.to_device())
    jobs = [{"type": "sssp", "graph": gr, "sources": ap.seeded_sources(r, 40, seed=3)},
            {"type": "sssp", "graph": gd, "sources": list(range(0, 4096, 500))},
            {"type": "sssp", "graph": gr, "sources": [int(np.argmax(r.degrees()))]}]
    ap.batch_set_sssp_pull(ctx, alpha)
    try:
        outs = ap.batch_run(ctx, jobs)
    finally:
        ap.batch_set_sssp_pull(ctx)
    for jd, out, h in zip(jobs, outs, (r, dd, r)):
        out = out.cpu().numpy().view(np.uint32)
        for i, s in enumerate(jd["sources"]):
            ref = oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, s)
            np.testing.assert_array_equal(out[i], ref, err_msg=f"sssp {h.name} src {s}")


def test_batch_rejects_bad_jobs(ctx):
    import apspie_b200 as ap
    a, *_ = _graphs()
    ga = a.to_device()
    with pytest.raises(ap.ApspieError):
        ap.batch_run(ctx, [{"type": "bfs", "graph": ga, "sources": [a.m]}])


def test_autotuner_picks_and_caches(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(16, 16, seed=12)
    g = h.to_device()
    srcs = ap.seeded_sources(h, 4, seed=1)
    first = ap.autotune_bfs(ctx, g, srcs)
    again = ap.autotune_bfs(ctx, g, srcs)   # cached: same answer
    assert first == again and first["ms_per_bfs"] > 0
    ref, _ = oracle.bfs(h.m, h.ptr, h.ind, srcs[0])
    np.testing.assert_array_equal(ap.bfs(ctx, g, srcs[0]).cpu().numpy(), ref)
    f = ap.autotune_spmspv(ctx, g)
    assert f >= 0
    ap.reset_tuning(ctx)  # restore defaults for the other tests


def test_batch_sssp_multi_source_parts(ctx, deep_mode):
    """Multi-source SSSP rows: more than 32 sources (two device jobs), a
    duplicated source, hubs split into chunks, a directed graph and a
    grid with heavy weights; every row equals the oracle's Dijkstra."""
    import apspie_b200 as ap
    r = ap.gen_rmat(13, 16, seed=11)          # hubs of degree >> 32
    ap.weights_u32(r, seed=5)
    g = ap.gen_grid(48, 48)
    ap.weights_u32(g, seed=6, lo=200, hi=255)
    dd = ap.gen_rmat(12, 8, seed=12, symmetric=False)
    ap.weights_u32(dd, seed=7)
    srcs = ap.seeded_sources(r, 45, seed=8)
    srcs[7] = srcs[3]
    jobs = [{"type": "sssp", "graph": r.to_device(), "sources": srcs},
            {"type": "sssp", "graph": g.to_device(), "sources": [0, 2303, 1200]},
            {"type": "sssp", "graph": dd.to_device(), "sources": list(range(0, 4096, 300))},
            {"type": "sssp", "graph": r.to_device(), "sources": [srcs[0]]},          # row width 1
            {"type": "sssp", "graph": g.to_device(), "sources": [5, 77]}]            # row width 2
    outs = ap.batch_run(ctx, jobs)
    for jd, out, h in zip(jobs, outs, (r, g, dd, r, g)):
        out = out.cpu().numpy().view(np.uint32)
        for i, s in enumerate(jd["sources"]):
            ref = oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, s)
            np.testing.assert_array_equal(out[i], ref, err_msg=f"sssp {h.name} src {s}")
