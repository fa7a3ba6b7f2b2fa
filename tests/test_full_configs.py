"""Every answer of the two full-size multi-query workloads.

Batched: 256 BFS + 64 SSSP sources over R-MAT 12 / 16 / 20 / 22
(symmetrised) and the 1024 x 1024 grid in one apspie_batch_run; every one of
the 320 result rows must equal the plain single-source path bit for bit, and
the R-MAT 12 / 16 rows also the oracle (the reference's BFS and the uint32
Dijkstra restatement).

Serving: the 8 resident graphs (R-MAT 12 ... 23 symmetrised + the grid) and
a Poisson stream replayed through the server, every (graph, kind) pair
present; every served answer, kept on the device during the timed replay,
must equal the single-query path.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_batched_config_every_source(ctx):
    import torch
    import apspie_b200 as ap
    from apspie_b200 import workloads as wl
    hosts = wl.batched_graphs()
    devs = {k: h.to_device() for k, h in hosts.items()}
    jobs = wl.batched_jobs(hosts, devs)
    assert sum(len(j["sources"]) for j in jobs if j["type"] == "bfs") == 256
    assert sum(len(j["sources"]) for j in jobs if j["type"] == "sssp") == 64
    outs = ap.batch_run(ctx, jobs)
    checked = against_oracle = 0
    for j, out in zip(jobs, outs):
        h = hosts[j["key"]]
        for i, s in enumerate(j["sources"]):
            if j["type"] == "bfs":
                ref = ap.bfs(ctx, j["graph"], s)
            else:
                ref = ap.sssp(ctx, j["graph"], s, weights="u32")
            assert torch.equal(out[i], ref), f"{j['type']} on {j['key']} source {s}"
            checked += 1
            if j["key"] in (12, 16):
                row = out[i].cpu().numpy()
                if j["type"] == "bfs":
                    exp = oracle.bfs(h.m, h.ptr, h.ind, s)[0]
                else:
                    exp = oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, s).view(np.int32)
                np.testing.assert_array_equal(row, exp, err_msg=f"oracle {j['key']} {s}")
                against_oracle += 1
    assert checked == 320 and against_oracle == 32 + 16 + 64 + 16


def test_serving_config_every_answer(ctx):
    import torch
    import apspie_b200 as ap
    from apspie_b200 import workloads as wl
    graphs = wl.serving_graphs(ctx)
    with ap.Server(budget_bytes=120 << 30, max_batch=256) as srv:
        gids = [srv.add_graph(g) for g in graphs]
        q, gi = wl.poisson_stream(graphs, gids, 240, 100_000.0, seed=11, cover=True,
                                  mis_seed=None)
        pairs = {(int(g), int(k)) for g, k in zip(gi, q["type"])}
        assert len(pairs) == 3 * len(graphs)
        keep = {i: torch.empty(graphs[int(gi[i])].m, dtype=torch.int32, device="cuda")
                for i in range(len(q))}
        lat, wall = srv.replay(q, keep=keep)
        st = srv.stats()
    assert (lat > 0).all() and st["batches"] < len(q)   # queries were coalesced
    for i in range(len(q)):
        g = graphs[int(gi[i])]
        ref = wl.plain_answer(ctx, g, int(q["type"][i]), int(q["source"][i]), int(q["seed"][i]))
        assert torch.equal(keep[i], ref), (
            f"query {i}: kind {q['type'][i]} on {wl.serving_names()[gi[i]]} source {q['source'][i]}")
