"""Query server: every answer equals the single-query path, alone and in a
mix of concurrent BFS / SSSP / MIS queries on several resident graphs; the
state budget gates admission; latencies are reported."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graphs():
    import apspie_b200 as ap
    gs = [ap.gen_rmat(12, 16, seed=1), ap.gen_rmat(14, 16, seed=2), ap.gen_grid(64, 64),
          ap.gen_rmat(11, 16, seed=3, symmetric=False)]
    for i, g in enumerate(gs):
        ap.weights_u32(g, seed=10 + i)
    return gs


def _alone(ctx, g, dg, kind, src, seed):
    import torch
    import apspie_b200 as ap
    if kind == 0:
        return ap.bfs(ctx, dg, src).cpu().numpy()
    if kind == 1:
        return ap.sssp(ctx, dg, src, weights="u32").cpu().numpy()
    prio = torch.from_numpy(ap.mt19937(seed, g.m).view(np.int32)).cuda()
    return ap.mis(ctx, dg, prio).cpu().numpy()


def test_server_mix_equals_alone(ctx):
    import apspie_b200 as ap
    hs = _graphs()
    ds = [h.to_device() for h in hs]
    rng = np.random.default_rng(0)
    with ap.Server(budget_bytes=8 << 30, max_batch=128) as srv:
        gids = [srv.add_graph(d) for d in ds]
        queries = []
        for _ in range(300):
            gi = int(rng.integers(len(hs)))
            kind = int(rng.choice([0, 1, 2], p=[0.6, 0.3, 0.1]))
            if kind == 2 and not hs[gi].symmetric:
                kind = 0
            src = int(rng.integers(hs[gi].m))
            seed = int(rng.integers(1 << 31))
            queries.append((gi, kind, src, seed, srv.submit(kind, gids[gi], src, seed)))
        results = [srv.wait(rid) for *_, rid in queries]
        st = srv.stats()
    assert st["completed"] == len(queries)
    assert st["batches"] < len(queries)          # queries were coalesced
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (gi, kind, src, seed, _), (out, lat) in zip(queries, results):
        ref = _alone(ctx, hs[gi], ds[gi], kind, src, seed)
        np.testing.assert_array_equal(out, ref.view(np.int32), err_msg=f"{kind} {gi} {src}")
        assert lat > 0


def test_server_push_pull_sssp_large_graph(ctx):
    """A graph above the batched-SSSP size limit with its in-adjacency and
    weights registered: SSSP queries, alone and in a group (run one by one
    through the push/pull kernel), equal the push-only single-query path."""
    import torch
    import apspie_b200 as ap
    g = ap.gen_rmat_device(ctx, 22, 16, seed=5)
    ap.weights_device(ctx, g, seed=5)
    srcs = [int(x) for x in torch.nonzero(g.ptr[1:] - g.ptr[:-1]).flatten()[:4:1].cpu()]
    refs = [ap.sssp(ctx, g, s, weights="u32").cpu().numpy() for s in srcs]   # push rounds only
    ap.sssp_prepare(ctx, g)
    with ap.Server(budget_bytes=16 << 30, max_batch=64) as srv:
        gid = srv.add_graph(g)
        rids = [srv.submit(1, gid, s) for s in srcs]
        outs = [srv.wait(r)[0] for r in rids]
    for s, out, ref in zip(srcs, outs, refs):
        np.testing.assert_array_equal(out, ref.view(np.int32), err_msg=f"sssp src {s}")


def test_server_budget_admits_one_at_a_time(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(12, 16, seed=4)
    ap.weights_u32(h, seed=1)
    d = h.to_device()
    with ap.Server(budget_bytes=1, max_batch=64) as srv:   # below any query's state
        gid = srv.add_graph(d)
        rids = [srv.submit(0, gid, s) for s in range(0, 400, 40)]
        outs = [srv.wait(r)[0] for r in rids]
        st = srv.stats()
    assert st["batches"] == len(rids)   # each query admitted alone
    for s, out in zip(range(0, 400, 40), outs):
        np.testing.assert_array_equal(out, ap.bfs(ctx, d, s).cpu().numpy())


def test_server_poisson_arrivals(ctx):
    """Queries arriving over time while earlier ones run are admitted and
    answered; latency percentiles are reported."""
    import apspie_b200 as ap
    hs = _graphs()
    ds = [h.to_device() for h in hs]
    rng = np.random.default_rng(1)
    with ap.Server(budget_bytes=8 << 30) as srv:
        gids = [srv.add_graph(d) for d in ds]
        rids = []
        t = time.perf_counter()
        for _ in range(200):
            t += rng.exponential(1 / 5000.0)   # 5,000 queries / s
            while time.perf_counter() < t:
                pass
            gi = int(rng.integers(3))
            rids.append(srv.submit(int(rng.choice([0, 1])), gids[gi], int(rng.integers(hs[gi].m))))
        for r in rids:
            srv.wait(r)
        st = srv.stats()
    assert st["completed"] == 200 and st["p99_ms"] > 0


def test_server_rejects_bad_queries():
    import apspie_b200 as ap
    h = ap.gen_rmat(10, 8, seed=1)
    d = h.to_device()
    with ap.Server(budget_bytes=1 << 30) as srv:
        gid = srv.add_graph(d)
        with pytest.raises(ap.ApspieError):
            srv.submit(0, gid, h.m)          # source out of range
        with pytest.raises(ap.ApspieError):
            srv.submit(1, gid, 0)            # SSSP on an unweighted graph
        with pytest.raises(ap.ApspieError):
            srv.submit(0, gid + 5, 0)        # unknown graph


def test_server_device_results_and_replay(ctx):
    """Results delivered into device buffers equal the single-query path;
    the open-loop replay and the plain one-at-a-time replay both finish a
    timed stream and report one latency per query."""
    import torch
    import apspie_b200 as ap
    from apspie_b200.serving import QUERY_DTYPE
    hs = _graphs()
    ds = [h.to_device() for h in hs]
    rng = np.random.default_rng(2)
    with ap.Server(budget_bytes=8 << 30) as srv:
        gids = [srv.add_graph(d) for d in ds]
        outs, rids, qs = [], [], []
        for _ in range(40):
            gi = int(rng.integers(3))
            kind = int(rng.choice([0, 1, 2]))
            src, seed = int(rng.integers(hs[gi].m)), int(rng.integers(1 << 31))
            out = torch.empty(hs[gi].m, dtype=torch.int32, device="cuda")
            outs.append(out)
            qs.append((gi, kind, src, seed))
            rids.append(srv.submit_device(kind, gids[gi], src, seed, out))
        for r in rids:
            srv.wait(r)
        for (gi, kind, src, seed), out in zip(qs, outs):
            ref = _alone(ctx, hs[gi], ds[gi], kind, src, seed)
            np.testing.assert_array_equal(out.cpu().numpy(), ref.view(np.int32))
        n = 120
        q = np.zeros(n, dtype=QUERY_DTYPE)
        q["type"] = rng.choice([0, 1, 2], size=n, p=[0.6, 0.3, 0.1])
        q["graph"] = rng.integers(0, 3, size=n)
        q["source"] = [int(rng.integers(hs[g].m)) for g in q["graph"]]
        q["seed"] = 5
        q["t_us"] = np.cumsum(rng.exponential(1e6 / 2000.0, size=n))   # 2,000 queries / s
        lat, wall = srv.replay(q)
        lat_p, wall_p = srv.replay(q, plain=True)
    assert (lat > 0).all() and (lat_p > 0).all()
    assert wall >= q["t_us"][-1] / 1e3 and wall_p >= q["t_us"][-1] / 1e3
