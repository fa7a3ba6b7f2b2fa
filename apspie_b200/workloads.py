"""The batched and serving workloads on their full-size graphs, built the same
way for the benchmark and for the tests that check every answer.

Batched: 256 BFS + 64 SSSP (uint32 weights in [1, 255]) sources spread
unevenly over R-MAT scales 12, 16, 20 and 22 (edge factor 16, symmetrised)
and the 1024 x 1024 grid.  Serving: 8 device-resident graphs (R-MAT 12, 14,
16, 18, 20, 22, 23 symmetrised and the grid, uint32 weights) and a Poisson
stream of 60 % BFS / 30 % SSSP / 10 % MIS queries, graph chosen in
proportion to its vertex count, sources among the vertices with edges.
"""
from __future__ import annotations

import numpy as np

from .graph import gen_grid, gen_rmat, seeded_sources, weights_u32
from .ops import bfs, gen_rmat_device, mis, sssp, weights_device

EDGE_FACTOR = 16
BATCH_BFS = {22: 64, 20: 64, 16: 64, 12: 32, "grid": 32}
BATCH_SSSP = {22: 8, 20: 16, 16: 16, 12: 16, "grid": 8}
SERVE_SCALES = (12, 14, 16, 18, 20, 22, 23)
SERVE_MIX = (0.6, 0.3, 0.1)


def batched_graphs(seed: int = 1, big=None) -> dict:
    """Host graphs of the batched workload (u32 weights added); `big` may
    pass an already built R-MAT 22 host graph."""
    gs = {12: gen_rmat(12, EDGE_FACTOR, seed=seed), 16: gen_rmat(16, EDGE_FACTOR, seed=seed),
          20: gen_rmat(20, EDGE_FACTOR, seed=seed),
          22: big if big is not None else gen_rmat(22, EDGE_FACTOR, seed=seed),
          "grid": gen_grid(1024, 1024)}
    for h in gs.values():
        if h.w_u32 is None:
            weights_u32(h, seed=seed)
    return gs


def batched_jobs(hosts: dict, devs: dict) -> list:
    """The 10 jobs (a BFS and an SSSP job per graph) with their sources:
    R-MAT sources seed-chosen in the largest component, grid sources every
    m/64-th vertex."""
    jobs = []
    for k, h in hosts.items():
        if k == "grid":
            srcs = list(range(0, h.m, h.m // 64))
        else:
            srcs = seeded_sources(h, BATCH_BFS[k] + BATCH_SSSP[k], seed=7)
        jobs.append({"type": "bfs", "graph": devs[k], "sources": srcs[:BATCH_BFS[k]], "key": k})
        jobs.append({"type": "sssp", "graph": devs[k],
                     "sources": srcs[BATCH_BFS[k]:][:BATCH_SSSP[k]], "key": k})
    return jobs


def serving_graphs(ctx, seed: int = 1) -> list:
    """The 8 serving graphs built on the device, with uint32 weights."""
    graphs = [gen_rmat_device(ctx, sc, EDGE_FACTOR, seed=seed) for sc in SERVE_SCALES]
    graphs.append(gen_grid(1024, 1024).to_device())
    for g in graphs:
        weights_device(ctx, g, seed=seed)
    return graphs


def serving_names() -> list:
    return [f"rmat{sc}" for sc in SERVE_SCALES] + ["grid1024"]


def poisson_stream(graphs: list, gids: list, n: int, rate: float, seed: int,
                   cover: bool = False, mis_seed: int | None = 1):
    """A Poisson stream of n queries at `rate` queries/s (QUERY_DTYPE).
    With cover, every (graph, kind) pair is made to occur at least once (the
    first 24 queries are one of each, in a seeded order).  MIS queries use
    mt19937(mis_seed) priorities, or a seeded random seed per query when
    mis_seed is None."""
    from .serving import QUERY_DTYPE
    rng = np.random.default_rng(seed)
    ms = np.array([g.m for g in graphs], dtype=np.float64)
    nonzero = [np.flatnonzero((g.ptr[1:] - g.ptr[:-1]).cpu().numpy() > 0) for g in graphs]
    q = np.zeros(n, dtype=QUERY_DTYPE)
    kinds = rng.choice([0, 1, 2], size=n, p=list(SERVE_MIX))
    gi = rng.choice(len(graphs), size=n, p=ms / ms.sum())
    if cover:
        pairs = [(g, k) for g in range(len(graphs)) for k in (0, 1, 2)]
        order = rng.permutation(len(pairs))
        for i, p in enumerate(order[:n]):
            gi[i], kinds[i] = pairs[p]
    q["type"] = kinds
    q["graph"] = [gids[i] for i in gi]
    q["source"] = [int(nonzero[i][rng.integers(len(nonzero[i]))]) for i in gi]
    q["seed"] = rng.integers(1, 1 << 31, size=n) if mis_seed is None else mis_seed
    q["t_us"] = np.cumsum(rng.exponential(1e6 / rate, size=n))
    return q, gi


def plain_answer(ctx, g, kind: int, source: int, seed: int):
    """The single-query answer of one query, as an int32 device tensor."""
    import torch
    from .graph import mt19937
    if kind == 0:
        return bfs(ctx, g, int(source))
    if kind == 1:
        return sssp(ctx, g, int(source), weights="u32")
    prio = torch.from_numpy(mt19937(int(seed), g.m).view(np.int32)).to(g.ptr.device)
    return mis(ctx, g, prio)
