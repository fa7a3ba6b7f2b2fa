"""The batched and serving workloads' host logic, on CPU: the batched
configuration's source counts (256 BFS + 64 SSSP over R-MAT 12/16/20/22 and
the grid, spread unevenly) and the serving stream's shape (60 / 30 / 10 %
BFS / SSSP / MIS, graph chosen in proportion to its vertex count, sources
among the vertices with edges, Poisson arrivals at the given rate, every
(graph, kind) pair covered on request).  Small stand-in graphs replace the
full-size ones, which only the GPU tests build."""
import numpy as np
import pytest
import torch

import apspie_b200 as ap
from apspie_b200 import workloads as wl


def test_batched_workload_has_the_configured_source_counts():
    assert sum(wl.BATCH_BFS.values()) == 256
    assert sum(wl.BATCH_SSSP.values()) == 64
    assert set(wl.BATCH_BFS) == set(wl.BATCH_SSSP) == {12, 16, 20, 22, "grid"}
    # uneven: the graphs do not all get the same number of sources
    assert len(set(wl.BATCH_BFS.values())) > 1 and len(set(wl.BATCH_SSSP.values())) > 1


def test_batched_jobs_split_each_graphs_sources_between_bfs_and_sssp():
    hosts = {k: ap.gen_rmat(12, 16, seed=1) for k in (12, 16, 20, 22)}
    hosts["grid"] = ap.gen_grid(64, 64)
    jobs = wl.batched_jobs(hosts, dict(hosts))
    assert len(jobs) == 10
    by = {(j["key"], j["type"]): j["sources"] for j in jobs}
    for k in hosts:
        assert len(by[(k, "bfs")]) == wl.BATCH_BFS[k]
        assert len(by[(k, "sssp")]) == wl.BATCH_SSSP[k]
        assert all(0 <= s < hosts[k].m for s in by[(k, "bfs")] + by[(k, "sssp")])
    assert sum(len(j["sources"]) for j in jobs if j["type"] == "bfs") == 256
    assert sum(len(j["sources"]) for j in jobs if j["type"] == "sssp") == 64
    # grid sources: every m/64-th vertex, the first 32 for BFS
    g = hosts["grid"]
    assert by[("grid", "bfs")] == list(range(0, g.m, g.m // 64))[:32]


class _Graph:
    """A stand-in for a device graph: row offsets as a CPU tensor."""

    def __init__(self, degrees):
        self.m = len(degrees)
        self.ptr = torch.from_numpy(np.concatenate([[0], np.cumsum(degrees)]).astype(np.int32))


def _graphs():
    rng = np.random.default_rng(3)
    out = []
    for m in (64, 256, 1024, 4096):
        d = rng.integers(0, 5, size=m)
        d[0] = 1
        out.append(_Graph(d))
    return out


def test_poisson_stream_mix_graph_choice_sources_and_arrivals():
    graphs = _graphs()
    gids = [10, 11, 12, 13]
    n, rate = 40000, 5000.0
    q, gi = wl.poisson_stream(graphs, gids, n, rate, seed=5)
    assert len(q) == n and len(gi) == n
    # kinds 60 / 30 / 10 %
    frac = np.bincount(q["type"], minlength=3) / n
    np.testing.assert_allclose(frac, wl.SERVE_MIX, atol=0.01)
    # graph in proportion to its vertex count; ids mapped through gids
    ms = np.array([g.m for g in graphs], dtype=np.float64)
    np.testing.assert_allclose(np.bincount(gi, minlength=4) / n, ms / ms.sum(), atol=0.01)
    assert np.array_equal(q["graph"], np.array(gids)[gi])
    # every source is a vertex with out-edges of its graph
    for i in range(0, n, 97):
        deg = graphs[gi[i]].ptr.numpy()
        s = int(q["source"][i])
        assert 0 <= s < graphs[gi[i]].m and deg[s + 1] > deg[s]
    # arrivals: increasing, mean gap 1/rate
    t = q["t_us"]
    assert np.all(np.diff(t) > 0)
    assert abs(t[-1] / n - 1e6 / rate) < 0.03 * (1e6 / rate)
    # MIS seed: fixed by default
    assert np.all(q["seed"] == 1)


def test_poisson_stream_cover_puts_every_pair_first_and_is_seeded():
    graphs = _graphs()
    gids = list(range(4))
    q, gi = wl.poisson_stream(graphs, gids, 50, 100.0, seed=9, cover=True, mis_seed=None)
    pairs = {(int(gi[i]), int(q["type"][i])) for i in range(12)}
    assert pairs == {(g, k) for g in range(4) for k in (0, 1, 2)}
    assert len(set(q["seed"].tolist())) > 1  # a seed per query
    q2, gi2 = wl.poisson_stream(graphs, gids, 50, 100.0, seed=9, cover=True, mis_seed=None)
    assert np.array_equal(q, q2) and np.array_equal(gi, gi2)
    q3, _ = wl.poisson_stream(graphs, gids, 50, 100.0, seed=10, cover=True, mis_seed=None)
    assert not np.array_equal(q, q3)


@pytest.mark.parametrize("n", [0, 1, 5])
def test_poisson_stream_short_streams(n):
    q, gi = wl.poisson_stream(_graphs(), [0, 1, 2, 3], n, 1000.0, seed=1, cover=True)
    assert len(q) == n and len(gi) == n
