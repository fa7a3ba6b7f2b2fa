"""Benchmark: single-source BFS GTEPS on R-MAT scale 22 (one B200), with the
HBM roofline of the traversal kernel, the end-to-end figure through the C ABI
with host buffers, and the reference's CPU BFS timed on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one BFS traversal from one seed-chosen source of the largest
connected component.  Inputs are resident in HBM before timing; the CSR
(~530 MB) is larger than the 126 MB L2, so no flush is needed between steps.
Multi-GPU runs are independent replicas (queries shard with no data-path
collective): value = all ranks' traversed edges / max-over-ranks time.
Prints exactly one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SCALE = 22
EDGE_FACTOR = 16
SEED = 1
WORKLOAD = (f"bfs_rmat{SCALE}: R-MAT scale {SCALE} (2^{SCALE} vertices), edge factor "
            f"{EDGE_FACTOR}, (0.57,0.19,0.19,0.05), symmetrised, self-loops/duplicates removed, "
            f"int32 CSR, single source per step from the largest connected component")
METRIC = "BFS GTEPS (R-MAT scale 22, single source, 1 B200)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=SCALE)
    p.add_argument("--profile-case", default=None,
                   choices=["mis_er", "mis_grid", "tc", "spgemm", "batch", "spmspv", "spmv",
                            "sssp_pull", "sort"],
                   help="run one workload three times for an ncu capture, print nothing else")
    p.add_argument("--no-prepare", action="store_true",
                   help="pull over the CSR as given instead of the degree-ordered in-adjacency")
    p.add_argument("--no-tune", action="store_true",
                   help="keep the default push/pull switch points (alpha 14, beta 24)")
    p.add_argument("--switch", default=None,
                   help="ALPHA,BETA: use these push/pull switch points instead of tuning "
                        "(for profiling the tuned configuration without the tuning launches)")
    p.add_argument("--workload", default="bfs", choices=["bfs", "serving"],
                   help="serving: only the serving sweep (rates 100 .. 100,000 queries/s), "
                        "one JSON line")
    p.add_argument("--profile-run", action="store_true",
                   help="only the timed traversals (for ncu captures): no clock extension, "
                        "no end-to-end leg, no CPU baseline")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


def profile_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summaries, if
    any: the last figure a summary gives (summaries append re-captures)."""
    found = None
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for line in f.read_text().splitlines():
            if line.startswith(f"traffic_bytes_per_launch[{kernel}]:"):
                try:
                    found = float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    pass
    return found


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_graph(scale):
    import apspie_b200 as ap
    h = ap.gen_rmat(scale, EDGE_FACTOR, seed=SEED, symmetric=True)
    return h


def cpu_reference_bfs(h, sources, budget_s):
    """The reference's SimpleReferenceBfs (oracle/_ref) on one host thread,
    one source after another until the sources or the time budget run out.
    Returns (edges, seconds, traversals)."""
    import oracle
    deg = h.degrees()
    edges, n = 0, 0
    with quiet_stdout():
        t0 = time.perf_counter()
        for s in sources:
            if time.perf_counter() - t0 > budget_s:
                break
            d = np.empty(h.m, np.int32)
            oracle._r.ref_bfs_cpu(int(s), h.m, h.ptr.ctypes.data, h.ind.ctypes.data,
                                  d.ctypes.data, 1 << 30)
            edges += int(deg[d >= 0].sum())
            n += 1
        wall = time.perf_counter() - t0
    return edges, wall, n


class quiet_stdout:
    """The reference routines print timings to stdout; keep them off the
    single JSON line this script prints."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        ctypes.CDLL(None).fflush(None)
        self.saved = os.dup(1)
        self.devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.devnull, 1)
        return self

    def __exit__(self, *exc):
        import ctypes
        ctypes.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.devnull)


def shared_config(scale, m, nnz, world):
    """The `config` object both arms print (same workload, same graph)."""
    return {"workload": WORKLOAD, "scale": scale, "m": int(m), "nnz": int(nnz),
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (CSR %.0f MB), no flush" % ((4 * (m + 1) + 4 * nnz) / 1e6)}


def run_reference(args):
    """The reference's own CPU BFS (SimpleReferenceBfs, src/testBfs.cpp:7-72,
    compiled into oracle/_ref) on all host threads: a step is one round of
    concurrent single-threaded traversals, one per host thread, each from its
    own source.  The graph and sources come from oracle.inputs (a NumPy
    restatement of the library's builder), so this arm loads none of the
    product's code."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    import oracle.inputs as oi
    kind = "reference" if oracle.have_reference() else "port"
    m, ptr, ind = oi.gen_rmat(args.scale, EDGE_FACTOR, seed=SEED, symmetric=True)
    threads = os.cpu_count() or 1
    K, W = max(args.steps, 1), max(args.warmup, 0)
    sources = oi.seeded_sources(m, ptr, ind, (K + W) * threads, seed=0)
    deg = np.diff(ptr).astype(np.int64)

    def one_round(srcs):
        edges = [0] * len(srcs)

        def work(i):
            d = np.empty(m, np.int32)
            oracle._r.ref_bfs_cpu(int(srcs[i]), m, ptr.ctypes.data, ind.ctypes.data,
                                  d.ctypes.data, 1 << 30)
            edges[i] = int(deg[d >= 0].sum())
        th = [threading.Thread(target=work, args=(i,)) for i in range(len(srcs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        return sum(edges)

    with quiet_stdout():
        for st in range(W):
            one_round(sources[st * threads:(st + 1) * threads])
        t0 = time.perf_counter()
        edges = 0
        for st in range(W, W + K):
            edges += one_round(sources[st * threads:(st + 1) * threads])
        wall = time.perf_counter() - t0
    gteps = edges / wall / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gteps, "unit": "GTEPS",
        "n_gpus": args.gpus, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * wall / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": shared_config(args.scale, m, len(ind), world),
        "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": threads, "kind": kind,
                         "sample": f"{K} steps of {threads} concurrent single-threaded "
                                   f"SimpleReferenceBfs (src/testBfs.cpp:7-72, -O3) traversals "
                                   f"of R-MAT {args.scale}, one source each ({K * threads} "
                                   f"traversals), after {W} untimed steps"},
        "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _sssp_block(ctx, g, srcs, kind, m):
    """Mean device ms per SSSP over srcs (CUDA events), GTEPS, algorithmic
    GB/s (8 E_R + 8 |R| + 4 m per traversal), edges walked per reached edge."""
    import torch
    import apspie_b200 as ap
    st = []
    for s in srcs:
        ap.sssp(ctx, g, s, weights=kind)
        st.append(ap.sssp_stats(ctx))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(torch.cuda.current_stream())
    for s in srcs:
        ap.sssp(ctx, g, s, weights=kind)
    b.record(torch.cuda.current_stream())
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / len(srcs)
    edges = sum(x["edges_traversed"] for x in st) / len(st)
    reached = sum(x["vertices_reached"] for x in st) / len(st)
    b_alg = 8.0 * edges + 8.0 * reached + 4.0 * m
    return {"ms_per_sssp": ms, "gteps": edges / (ms * 1e-3) / 1e9,
            "hbm_gbs_alg": b_alg / (ms * 1e-3) / 1e9,
            "relaxations_per_edge": sum(x["relaxations"] for x in st) / max(1.0, edges * len(st)),
            "rounds": st[-1]["rounds"], "sources": len(srcs)}


def sssp_leg(ctx, big, steps=20):
    """SSSP on R-MAT 20 (directed, dedup) with uint32 weights in [1, 255]
    and float weights in (0, 1], and on the symmetrised R-MAT 22 / 23 of the
    serving workload with uint32 weights (push rounds, one source at a time):
    device time per traversal, inputs resident."""
    import apspie_b200 as ap
    h = ap.gen_rmat(20, EDGE_FACTOR, seed=SEED, symmetric=False)
    ap.weights_u32(h, seed=SEED)
    ap.weights_f32(h, seed=SEED)
    g = h.to_device()
    # the weighted in-adjacency (built once, outside the timing) lets the
    # tuner weigh pull rounds against push-only
    ap.sssp_prepare(ctx, g)
    srcs = ap.seeded_sources(h, steps, seed=3)
    out = {"graph": f"R-MAT 20 directed, m={h.m}, nnz={h.nnz}",
           "tuning": "per graph by apspie_autotune_sssp on 8 untimed sources (u32 weights; "
                     "blocks per SM, and the pull switch over the weighted in-adjacency "
                     "built by sssp_prepare outside the timed region)"}
    tuned = _sssp_tune(ctx, g, ap.seeded_sources(h, 8, seed=77))
    for kind in ("u32", "f32"):
        for s in srcs[:3]:
            ap.sssp(ctx, g, s, weights=kind)
        out[kind] = _sssp_block(ctx, g, srcs, kind, h.m)
        out[kind]["tuned"] = tuned
    del g
    if big.w_u32 is None:
        ap.weights_u32(big, seed=SEED)
    g22 = ap.sssp_prepare(ctx, big.to_device())
    tuned = _sssp_tune(ctx, g22, ap.seeded_sources(big, 8, seed=77))
    out["rmat22_sym_u32"] = _sssp_block(ctx, g22, ap.seeded_sources(big, 8, seed=3), "u32", big.m)
    out["rmat22_sym_u32"]["tuned"] = tuned
    del g22
    g23 = ap.gen_rmat_device(ctx, 23, EDGE_FACTOR, seed=SEED)
    ap.weights_device(ctx, g23, seed=SEED)
    ap.sssp_prepare(ctx, g23)
    deg = (g23.ptr[1:] - g23.ptr[:-1]).cpu().numpy()
    cand = np.flatnonzero(deg > 0)
    rng = np.random.default_rng(3)
    s23 = [int(x) for x in cand[rng.integers(len(cand), size=6)]]
    tuned = _sssp_tune(ctx, g23, [int(x) for x in cand[rng.integers(len(cand), size=6)]])
    ap.sssp(ctx, g23, s23[0], weights="u32")
    out["rmat23_sym_u32"] = _sssp_block(ctx, g23, s23, "u32", g23.m)
    out["rmat23_sym_u32"]["tuned"] = tuned
    ap.set_tuning(ctx, sssp_blocks_per_sm=0, sssp_pull_alpha=0)
    return out


def _sssp_tune(ctx, g, srcs):
    import apspie_b200 as ap
    t = ap.autotune_sssp(ctx, g, srcs)
    return {"blocks_per_sm": t["blocks_per_sm"], "pull_alpha": t["pull_alpha"]}


def _ev_ms(fn, reps=5):
    """Mean device ms of fn() over reps calls (CUDA events on the current stream)."""
    import torch
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def mis_tc_spgemm_leg(ctx):
    """Luby MIS (ER n = 2^20 mean degree 8; grid 1024 x 1024; mt19937
    priorities), triangle counting (R-MAT 18 symmetrised) and hash SpGEMM
    A*A (2^18 x 2^18 power-law rows): device time, inputs resident, and the
    algorithmic bytes of each over the measured HBM peak."""
    import torch
    import apspie_b200 as ap
    pk, _ = peaks()
    hbm = pk["hbm_gbs"]
    out = {}
    for name, h in (("mis_er20_deg8", ap.gen_er(1 << 20, 8, seed=SEED)),
                    ("mis_grid1024", ap.gen_grid(1024, 1024))):
        g = h.to_device()
        prio = torch.from_numpy(ap.mt19937(5489, h.m).view(np.int32)).cuda()
        res = torch.empty(h.m, dtype=torch.int32, device="cuda")
        ms = _ev_ms(lambda: ap.mis(ctx, g, prio, res))
        rounds = ap.mis_rounds(ctx)
        b_alg = 4.0 * h.nnz + 12.0 * h.m  # column indices once, priority + state + result
        out[name] = {"ms": ms, "rounds": rounds, "members": int(res.sum().item()),
                     "hbm_gbs_alg": b_alg / (ms * 1e-3) / 1e9, "frac": b_alg / (ms * 1e-3) / 1e9 / hbm}
    h = ap.gen_rmat(18, EDGE_FACTOR, seed=SEED)
    g = h.to_device()
    prep_ms = _ev_ms(lambda: ap.tc_prepare(ctx, g), reps=2)
    _, lp, li = ap.tc_prepare(ctx, g)
    count = ap.triangle_count(ctx, h.m, lp, li)
    ms = _ev_ms(lambda: ap.triangle_count(ctx, h.m, lp, li))
    lpn, lin = lp.cpu().numpy().astype(np.int64), li.cpu().numpy().astype(np.int64)
    prods = int(np.sum(np.diff(lpn)[lin]))  # P = sum over (i, k) in L of nnz(L(k,:))
    b_alg = 4.0 * prods + 8.0 * len(lin) + 4.0 * h.m
    out["tc_rmat18"] = {"ms": ms, "prepare_ms": prep_ms, "triangles": count, "nnz_L": int(len(lin)),
                        "products": prods, "hbm_gbs_alg": b_alg / (ms * 1e-3) / 1e9,
                        "frac": b_alg / (ms * 1e-3) / 1e9 / hbm}
    a = ap.gen_powerlaw(1 << 18, seed=SEED)
    t = lambda x: torch.from_numpy(x).cuda()
    A = (a.m, a.ncols, t(a.ptr), t(a.ind), t(a.w_f32))
    tuned = ap.autotune_spgemm(ctx, A, A)
    cp, ci, cv = ap.spgemm(ctx, A, A)
    ms_call = _ev_ms(lambda: ap.spgemm(ctx, A, A), reps=3)
    # the two phases into preallocated C (no allocation inside the timing):
    # symbolic (row sizes, offsets, one read of nnz(C)) then numeric
    ms = _ev_ms(lambda: (ap.spgemm_symbolic(ctx, A, A),
                         ap.spgemm_numeric(ctx, A, A, cp, ci, cv)), reps=3)
    ap.spgemm_symbolic(ctx, A, A)
    ms_num = _ev_ms(lambda: (ap.spgemm_numeric(ctx, A, A, cp, ci, cv)), reps=1)
    deg = np.diff(a.ptr).astype(np.int64)
    prods = int(np.sum(deg[a.ind]))
    b_alg = 8.0 * a.nnz + 8.0 * prods + 8.0 * int(ci.numel()) + 8.0 * (a.m + 1)
    out["spgemm_powerlaw18"] = {"ms": ms, "ms_numeric": ms_num, "ms_call": ms_call,
                                "nnz_A": int(a.nnz), "products": prods,
                                "nnz_C": int(ci.numel()), "xmin": a.xmin,
                                "hbm_gbs_alg": b_alg / (ms * 1e-3) / 1e9,
                                "frac": b_alg / (ms * 1e-3) / 1e9 / hbm,
                                "tuned": {k: tuned[k] for k in ("table_load", "warp_max_prod",
                                                                "bitmap_max_cols")},
                                "note": "ms = symbolic + numeric into preallocated C; "
                                        "ms_call = ap.spgemm with C allocated per call; "
                                        "tuned = apspie_autotune_spgemm's pick for A * A"}
    ap.set_tuning(ctx, spgemm_table_load=2, spgemm_warp_max_prod=256,
                  spgemm_bitmap_max_cols=1 << 18)
    return out


def batched_leg(ctx, big):
    """256 BFS + 64 SSSP (uint32 weights) sources over R-MAT 12/16/20/22
    (symmetrised) and the 1024x1024 grid, in one batched launch, against the
    same queries one at a time through the single-source kernels.  Every one
    of the 320 batched rows is compared with its single-source result (bit
    for bit; a mismatch raises).  Per graph: its sources one at a time and
    its two jobs in a batched launch of their own."""
    import torch
    import apspie_b200 as ap
    from apspie_b200 import workloads as wl
    hosts = wl.batched_graphs(seed=SEED, big=big)
    devs = {k: h.to_device() for k, h in hosts.items()}
    jobs = wl.batched_jobs(hosts, devs)
    stream = torch.cuda.current_stream()

    def plain_run(js, keep=None):
        edges = 0
        for j in js:
            for s in j["sources"]:
                if j["type"] == "bfs":
                    r = ap.bfs(ctx, j["graph"], s)
                else:
                    r = ap.sssp(ctx, j["graph"], s, weights="u32")
                if keep is not None:
                    edges += (ap.bfs_stats(ctx) if j["type"] == "bfs"
                              else ap.sssp_stats(ctx))["edges_traversed"]
                    keep.append(r)
        return edges

    def timed(fn):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        out = fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]), out

    # warm-up (workspaces, autotuner / depth caches) and the reference rows
    refs = []
    edges = plain_run(jobs, refs)
    ap.batch_run(ctx, jobs)
    tuned = ap.autotune_batch(ctx, jobs)
    plain_ms, _ = timed(lambda: plain_run(jobs))
    batch_ms, outs = timed(lambda: ap.batch_run(ctx, jobs))
    st = ap.batch_stats(ctx)
    verified = 0
    it = iter(refs)
    for j, o in zip(jobs, outs):
        for i, s in enumerate(j["sources"]):
            if not torch.equal(o[i], next(it)):
                raise RuntimeError(f"batched {j['type']} row of source {s} on {j['key']} "
                                   "differs from the single-source path")
            verified += 1
    per_graph = {}
    for k in hosts:
        js = [j for j in jobs if j["key"] == k]
        pm, _ = timed(lambda: plain_run(js))
        ap.batch_run(ctx, js)
        bm, _ = timed(lambda: ap.batch_run(ctx, js))
        per_graph["grid1024" if k == "grid" else f"rmat{k}"] = {
            "bfs": len(js[0]["sources"]), "sssp": len(js[1]["sources"]),
            "plain_ms": pm, "batched_alone_ms": bm, "speedup": pm / bm}
    nq = sum(len(j["sources"]) for j in jobs)
    return {"queries": nq, "bfs": 256, "sssp": 64,
            "graphs": "R-MAT 12/16/20/22 symmetrised + grid 1024x1024",
            "batched_gteps": edges / (batch_ms * 1e-3) / 1e9,
            "plain_gteps": edges / (plain_ms * 1e-3) / 1e9,
            "speedup_vs_plain": plain_ms / batch_ms, "batched_ms": batch_ms,
            "plain_ms": plain_ms, "super_steps": st["super_steps"], "verified": verified,
            "per_graph": per_graph,
            "tuned": {"blocks_per_sm": tuned["blocks_per_sm"], "deep_blocks": tuned["deep_blocks"],
                      "picked_by": "apspie_autotune_batch on the same job list, untimed"},
            "timing": "CUDA events on the launching stream (plain: all single-source calls "
                      "back to back; batched: one apspie_batch_run, transposes included); "
                      "per_graph: each graph's two jobs in a launch of their own"}


def serving_leg(ctx, rates=(100, 1000, 10000, 100000), n_queries=600, seed=SEED, n_verify=120,
                serve_reps=3):
    """Serving: 8 device-resident graphs (R-MAT 12..23 symmetrised + the
    1024x1024 grid, uint32 weights in [1, 255]), a Poisson stream of 60% BFS
    / 30% SSSP / 10% MIS queries, graph chosen in proportion to its vertex
    count (the first 24 queries are one of every (graph, kind) pair), sources
    seed-chosen among vertices with edges.  Each rate is replayed open-loop
    through the server (continuous batching) and through the plain
    one-query-at-a-time path, serve_reps times each above 100 q/s (the
    median run by throughput is reported, every run's throughput listed);
    latency = arrival -> result row in (pinned) host memory.  During the server's replay the answers of a seeded sample of
    n_verify queries (every pair in the stream among them) are kept on the
    device and compared with the single-query path afterwards; a mismatch
    raises."""
    import torch
    import apspie_b200 as ap
    from apspie_b200 import workloads as wl
    from apspie_b200.serving import QUERY_DTYPE
    graphs = wl.serving_graphs(ctx, seed=seed)
    names = wl.serving_names()
    torch.cuda.synchronize()
    out = {"graphs": names, "mix": "60% BFS / 30% SSSP / 10% MIS", "queries_per_rate": n_queries,
           "latency": "arrival -> result row in host memory (device -> pinned host copy included)",
           "budget_gb": 120, "rates": []}
    kinds = ("bfs", "sssp", "mis")
    with ap.Server(budget_bytes=120 << 30, max_batch=256) as srv:
        gids = [srv.add_graph(g) for g in graphs]
        # untimed warm-up of both paths: every (graph, kind) alone and in
        # groups, so workspaces, result buffers and MIS priorities exist
        nonzero = [np.flatnonzero((g.ptr[1:] - g.ptr[:-1]).cpu().numpy() > 0) for g in graphs]
        wq = []
        for gi, g in enumerate(graphs):
            for kind in (0, 1, 2):
                for rep in (1, 3, 40):
                    for _ in range(rep):
                        wq.append((kind, gids[gi], int(nonzero[gi][len(wq) % len(nonzero[gi])])))
        warm = np.zeros(len(wq), dtype=QUERY_DTYPE)
        warm["type"] = [k for k, _, _ in wq]
        warm["graph"] = [gg for _, gg, _ in wq]
        warm["source"] = [sv for _, _, sv in wq]
        warm["seed"] = 1
        warm["t_us"] = 0.0
        srv.replay(warm)
        srv.replay(warm[::7], plain=True)
        for rate in rates:
            q, gi = wl.poisson_stream(graphs, gids, n_queries, float(rate), seed * 1000 + int(rate),
                                      cover=True)
            rng = np.random.default_rng(seed * 7 + int(rate))
            pick = {}
            for i in range(len(q)):   # the first query of every (graph, kind) pair
                pick.setdefault((int(gi[i]), int(q["type"][i])), i)
            sample = set(pick.values())
            for i in rng.permutation(len(q)):
                if len(sample) >= n_verify:
                    break
                sample.add(int(i))
            keep = {i: torch.empty(graphs[int(gi[i])].m, dtype=torch.int32, device="cuda")
                    for i in sorted(sample)}
            row = {"rate_qps": rate}
            lats = {}
            # the stream is replayed `reps` times on each path (alternating);
            # the reported run of each path is its median by throughput, and
            # every run's throughput is listed (runs differ by how arrivals
            # fall into batches)
            reps = 1 if rate <= 100 else serve_reps
            runs = {"batched": [], "plain": []}
            for rep in range(reps):
                for name, plain in (("batched", False), ("plain", True)):
                    srv.reset_stats()
                    lat, wall = srv.replay(q, plain=plain,
                                           keep=None if (plain or rep) else keep)
                    rec = {"qps": n_queries / (wall * 1e-3),
                           "p50_ms": float(np.percentile(lat, 50)),
                           "p99_ms": float(np.percentile(lat, 99)), "wall_ms": wall}
                    if not plain:
                        st = srv.stats()
                        rec["batches"] = int(st["batches"])
                        rec["admission_waits"] = int(st["admission_waits"])
                        rec["memory_cap_gb"] = round(st["memory_cap_bytes"] / 2**30, 1)
                        rec["max_launch_ms"] = round(st["max_launch_ms"], 2)
                    runs[name].append((rec, lat))
            for name in ("batched", "plain"):
                order = sorted(range(reps), key=lambda i: runs[name][i][0]["qps"])
                rec, lat = runs[name][order[reps // 2]]
                row[name] = dict(rec, runs_qps=[round(r["qps"], 1) for r, _ in runs[name]])
                lats[name] = lat
            row["throughput_ratio"] = row["batched"]["qps"] / row["plain"]["qps"]
            for i, t in keep.items():
                ref = wl.plain_answer(ctx, graphs[int(gi[i])], int(q["type"][i]),
                                      int(q["source"][i]), int(q["seed"][i]))
                if not torch.equal(t, ref):
                    raise RuntimeError(f"served answer of query {i} ({kinds[q['type'][i]]} on "
                                       f"{names[gi[i]]}) differs from the single-query path")
            row["verified"] = len(keep)
            row["pairs_in_stream"] = len(pick)
            table = {}
            for (g_i, k), _ in sorted(pick.items()):
                sel = (gi == g_i) & (q["type"] == k)
                table[f"{names[g_i]}/{kinds[k]}"] = [
                    int(sel.sum()), round(float(np.median(lats["batched"][sel])), 2),
                    round(float(np.median(lats["plain"][sel])), 2)]
            row["by_graph_kind"] = table
            row["by_graph_kind_columns"] = ["queries", "batched_p50_ms", "plain_p50_ms"]
            out["rates"].append(row)
            del keep
    return out


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import apspie_b200 as ap

    h = build_graph(args.scale)
    g = h.to_device(local)
    deg = h.degrees()
    nsrc = max(args.steps, 1)
    from apspie_b200.replicas import replica_sources
    sources = replica_sources(h, nsrc + args.warmup, rank)
    ctx = ap.Context(local)
    stream = torch.cuda.current_stream(local)
    depth = torch.empty(h.m, dtype=torch.int32, device=g.ptr.device)
    # one-time graph build step outside the timed region (like the CSR
    # itself): the in-adjacency the pull levels probe, each row ordered by
    # the neighbours' out-degree (apspie_bfs_prepare)
    prep_ms = None
    if not args.no_prepare:
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        ap.bfs_prepare(ctx, g)
        p1.record(stream)
        torch.cuda.synchronize()
        prep_ms = p0.elapsed_time(p1)

    # per-graph autotuning of the push/pull switch points on sources that are
    # not timed (cached under the graph's fingerprint), then an untimed pass:
    # edges traversed per source (and warm-up)
    tune = {"alpha": None, "beta": None}
    if args.switch:
        sa, sb = (int(x) for x in args.switch.split(","))
        ap.bfs_set_params(ctx, sa, sb)
        tune = {"alpha": sa, "beta": sb}
    elif not args.no_tune:
        tune_src = ap.seeded_sources(h, 64, seed=1000 + rank)
        tune = ap.autotune_bfs(ctx, g, tune_src)
    e_r = []
    for s in sources[:nsrc]:
        ap.bfs(ctx, g, s, depth)
        e_r.append(ap.bfs_stats(ctx)["edges_traversed"])
    reached = ap.bfs_stats(ctx)["vertices_reached"]
    trace = ap.bfs_trace(ctx)
    for s in sources[nsrc:]:
        ap.bfs(ctx, g, s, depth)
    torch.cuda.synchronize()

    # ---- timed: K traversals, inputs resident ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(nsrc)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.launches
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i, s in enumerate(sources[:nsrc]):
            ev[i][0].record(stream)
            ap.bfs(ctx, g, s, depth)
            ev[i][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
        launches = ctx.launches - launches0
        # keep sampling a little longer for a usable clock record on short runs
        total_ms = t0.elapsed_time(t1)
        if total_ms < 1500 and not args.profile_run:
            extra = int(1500 / max(total_ms / nsrc, 1e-3))
            for i in range(min(extra, 20000)):
                ap.bfs(ctx, g, sources[i % nsrc], depth)
            torch.cuda.synchronize()
    per = [a.elapsed_time(b) for a, b in ev]
    ms = total_ms
    from apspie_b200.replicas import aggregate
    ms, edges_all = aggregate(ms, float(sum(e_r)), device=g.ptr.device)
    value = edges_all / (ms * 1e-3) / 1e9

    # ---- roofline of the traversal kernel (bfs_persistent, one launch per traversal) ----
    pk, pk_kind = peaks()
    b_alg = 4.0 * np.mean(e_r) + 8.0 * reached + 4.0 * h.m
    avg_launch_s = float(np.mean(per)) * 1e-3
    achieved = b_alg / avg_launch_s / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "peak_kind": pk_kind,
            "kernel": "bfs_persistent (initialisation fused in)",
            "algorithmic_bytes_per_launch": b_alg,
            "traffic": profile_traffic("bfs_persistent"),
            "vs_nominal_8tbs": achieved / 8000.0}

    # ---- end to end through the C ABI with host buffers ----
    ptr_h = torch.from_numpy(h.ptr).pin_memory()
    ind_h = torch.from_numpy(h.ind).pin_memory()
    depth_h = torch.empty(h.m, dtype=torch.int32).pin_memory()
    e2e_steps = 0 if args.profile_run else min(nsrc, 10)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the uploaded CSR as given (no prepared in-adjacency: building it is a
    # per-graph step that an end-to-end call would have to repeat)
    g_e2e = ap.DeviceGraph(h.m, h.nnz, g.ptr, g.ind, symmetric=h.symmetric)
    a.record(stream)
    for s in sources[:e2e_steps]:
        g.ptr.copy_(ptr_h, non_blocking=True)
        g.ind.copy_(ind_h, non_blocking=True)
        ap.bfs(ctx, g_e2e, s, depth)
        depth_h.copy_(depth, non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(a.elapsed_time(b), 1e-6)
    e2e = {"value": sum(e_r[:e2e_steps]) / (e2e_ms * 1e-3) / 1e9, "unit": "GTEPS",
           "h2d_bytes_per_step": int(h.ptr.nbytes + h.ind.nbytes),
           "d2h_bytes_per_step": int(depth_h.numel() * 4),
           "note": "graph CSR copied host->device and depths device->host every step"}

    extras = {}
    # The other legs are single-GPU measurements of their own configurations.
    # They run at N=1 only: under torchrun the other ranks would wait at the
    # closing barrier for minutes, past the process group's timeout, while
    # holding their GPUs idle.
    if not args.profile_run and rank == 0 and world == 1:
        extras["sssp"] = sssp_leg(ctx, h)
        extras["mis_tc_spgemm"] = mis_tc_spgemm_leg(ctx)
        extras["batched"] = batched_leg(ctx, h)
        extras["serving"] = serving_leg(ctx)

    # ---- reference CPU BFS on a bounded sample (rank 0, N=1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.profile_run:
        import oracle
        if oracle.have_reference():
            edges, wall, n = cpu_reference_bfs(h, sources[:8], 20.0)
            cpu = {"value": edges / wall / 1e9, "unit": "GTEPS", "cores": 1,
                   "kind": "reference",
                   "sample": f"{n} BFS traversals of the same graph and sources, "
                             f"SimpleReferenceBfs (src/testBfs.cpp:7-72) -O3, 1 thread, "
                             f"host nproc={os.cpu_count()}"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": nsrc,
        "warmup": args.warmup, "ms_per_step": ms / nsrc, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": shared_config(args.scale, h.m, h.nnz, world),
        "workload_stats": {"edges_traversed_per_step": float(np.mean(e_r)),
                           "vertices_reached": int(reached),
                           "pull_adjacency": ("CSR as given" if prep_ms is None else
                                              "in-adjacency ordered by neighbour out-degree, "
                                              "built once by apspie_bfs_prepare in %.1f ms "
                                              "outside the timed region" % prep_ms),
                           "switch_points": {"alpha": tune.get("alpha"), "beta": tune.get("beta"),
                                             "blocks_per_sm": tune.get("blocks_per_sm"),
                                             "picked_by": "--switch" if args.switch else
                                             "defaults" if args.no_tune else
                                             "autotuner on 64 untimed sources (21 switch-point "
                                             "candidates ranked on 32, the best 4 and the "
                                             "reference point (32, 128) re-timed on the other "
                                             "32, two sweeps each; then 3 / 2 / 1 blocks per SM "
                                             "on all 64)"}},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "per_step_ms": {"min": min(per), "median": statistics.median(per), "max": max(per)},
        "level_trace": [[t["dir"], t["frontier"], t["frontier_edges"], round(t["us"], 1),
                         round(t["work_first_us"], 1), round(t["work_last_us"], 1)]
                        for t in trace],
        "level_trace_columns": ["dir", "frontier", "frontier_edges", "us", "first_block_done_us",
                                "last_block_done_us"],
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


def run_serving(args):
    """--workload serving: the full arrival-rate sweep of the serving leg."""
    import torch
    rank, _, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    import apspie_b200 as ap
    ctx = ap.Context(local)
    res = serving_leg(ctx, rates=(100, 1000, 10000, 100000), n_queries=max(args.steps, 200))
    best = max(res["rates"], key=lambda r: r["batched"]["qps"])
    line = {"metric": "serving throughput (queries/s), mixed BFS/SSSP/MIS on 8 resident graphs",
            "value": best["batched"]["qps"], "unit": "queries/s", "n_gpus": 1,
            "steps": res["queries_per_rate"], "warmup": 0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/uint32",
            "data": "synthetic", "config": {"workload": "serving: " + ", ".join(res["graphs"]),
                                            "mix": res["mix"], "budget_gb": res["budget_gb"]},
            "serving": res}
    print(json.dumps(line), flush=True)


def run_profile_case(args):
    """--profile-case NAME: run one workload of the MIS / TC / SpGEMM / batched
    / SpMSpV / SpMV / push-pull SSSP (R-MAT 22, two sources) / pull-adjacency
    sort (R-MAT 22) configurations
    three times and exit, for ncu captures of its kernels (no timing, no
    JSON)."""
    import torch
    import apspie_b200 as ap
    ctx = ap.Context(0)
    case = args.profile_case
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    if case in ("mis_er", "mis_grid"):
        h = ap.gen_er(1 << 20, 8, seed=SEED) if case == "mis_er" else ap.gen_grid(1024, 1024)
        g = h.to_device()
        prio = torch.from_numpy(ap.mt19937(5489, h.m).view(np.int32)).cuda()
        run = lambda: ap.mis(ctx, g, prio)
    elif case == "tc":
        h = ap.gen_rmat(18, EDGE_FACTOR, seed=SEED)
        _, lp, li = ap.tc_prepare(ctx, h.to_device())
        run = lambda: ap.triangle_count(ctx, h.m, lp, li)
    elif case == "spgemm":
        a = ap.gen_powerlaw(1 << 18, seed=SEED)
        A = (a.m, a.ncols, t(a.ptr), t(a.ind), t(a.w_f32))
        run = lambda: ap.spgemm(ctx, A, A)
    elif case == "sort":
        # the BFS pull-adjacency build of R-MAT 22: a 6-pass radix sort of
        # 128.3 M (u64 key, i32 value) pairs (graph built on the host, so the
        # first sort launches are this one's)
        h = ap.gen_rmat(22, EDGE_FACTOR, seed=SEED)
        g = h.to_device()
        run = lambda: ap.bfs_prepare(ctx, g)
    elif case == "batch":
        h = ap.gen_rmat(20, EDGE_FACTOR, seed=SEED)
        ap.weights_u32(h, seed=SEED)
        g = h.to_device()
        srcs = ap.seeded_sources(h, 96, seed=7)
        jobs = [{"type": "bfs", "graph": g, "sources": srcs[:64]},
                {"type": "sssp", "graph": g, "sources": srcs[64:]}]
        run = lambda: ap.batch_run(ctx, jobs)
    elif case == "sssp_pull":
        h = ap.gen_rmat(22, EDGE_FACTOR, seed=SEED)
        ap.weights_u32(h, seed=SEED)
        g = ap.sssp_prepare(ctx, h.to_device())
        ap.sssp_set_pull(ctx, 2)
        srcs = ap.seeded_sources(h, 2, seed=3)
        run = lambda: [ap.sssp(ctx, g, s, weights="u32") for s in srcs]
    elif case in ("spmspv", "spmv"):
        h = ap.gen_rmat(20, EDGE_FACTOR, seed=SEED)
        g = h.to_device()
        val = torch.ones(h.nnz, dtype=torch.float32, device="cuda")
        if case == "spmv":
            x = torch.rand(h.m, device="cuda")
            run = lambda: ap.spmv(ctx, h.m, g.ptr, g.ind, val, x)
        else:
            xi = t(np.arange(0, h.m, 64, dtype=np.int32))
            run = lambda: ap.spmspv(ctx, 0, g, xi, None, val)
    else:
        raise SystemExit(f"unknown profile case {case}")
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    print(f"profile case {case}: ok")


def main():
    args = parse()
    if args.profile_case:
        run_profile_case(args)
        return
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serving":
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
