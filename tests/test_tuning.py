"""Per-graph tuning: the autotuners' picks (BFS switch points and blocks per
SM, SSSP blocks per SM and pull switch, batched blocks per SM and deep-graph
share, SpGEMM table load / warp-row limit / long-row accumulator) are cached
by graph fingerprint, a cache hit applies the same choice to the context
again, and every choice a tuner may make gives the same results: BFS depths,
uint32 distances and SpGEMM structure exactly, SpGEMM values within 1e-5
relative of the FP64 oracle."""
import itertools

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

VAL_RTOL = 1e-5


def test_bfs_tuner_caches_and_every_grid_gives_the_same_depths(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(16, 16, seed=12)
    g = h.to_device()
    srcs = ap.seeded_sources(h, 8, seed=1)
    try:
        first = ap.autotune_bfs(ctx, g, srcs)
        assert first["blocks_per_sm"] in (0, 1, 2) and first["ms_per_bfs"] > 0
        picked = ap.get_tuning(ctx)
        ap.reset_tuning(ctx)
        again = ap.autotune_bfs(ctx, g, srcs)       # cache hit: the same choice, applied again
        assert again == first and ap.get_tuning(ctx) == picked
        ref, _ = oracle.bfs(h.m, h.ptr, h.ind, srcs[0])
        for bps in (0, 1, 2, 3):
            ap.set_tuning(ctx, bfs_blocks_per_sm=bps)
            np.testing.assert_array_equal(ap.bfs(ctx, g, srcs[0]).cpu().numpy(), ref)
    finally:
        ap.reset_tuning(ctx)


def test_sssp_tuner_caches_and_every_choice_gives_the_same_distances(ctx):
    import apspie_b200 as ap
    h = ap.gen_rmat(14, 16, seed=3)
    ap.weights_u32(h, seed=3)
    g = h.to_device()
    ap.sssp_prepare(ctx, g)                         # in-adjacency: the pull switch is a choice too
    srcs = ap.seeded_sources(h, 6, seed=2)
    try:
        first = ap.autotune_sssp(ctx, g, srcs)
        assert not first["cached"] and first["blocks_per_sm"] in (0, 1)
        assert first["pull_alpha"] in (0, 2, 8)
        ap.reset_tuning(ctx)
        again = ap.autotune_sssp(ctx, g, srcs)
        assert again["cached"]
        assert (again["blocks_per_sm"], again["pull_alpha"]) == (first["blocks_per_sm"],
                                                                  first["pull_alpha"])
        ref = oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, srcs[1])
        for bps, alpha in itertools.product((0, 1), (0, 2, 8)):
            ap.set_tuning(ctx, sssp_blocks_per_sm=bps, sssp_pull_alpha=alpha)
            d = ap.sssp(ctx, g, srcs[1], weights="u32").cpu().numpy().view(np.uint32)
            np.testing.assert_array_equal(d, ref, err_msg=f"blocks {bps} alpha {alpha}")
    finally:
        ap.reset_tuning(ctx)


def _dev_csr(h):
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return (h.m, getattr(h, "ncols", h.m), t(h.ptr), t(h.ind), t(h.w_f32))


def test_spgemm_tuner_caches_and_every_table_choice_gives_the_same_product(ctx):
    """Power-law rows reach every bin; each (table load, warp limit, bitmap)
    candidate moves rows between bins and resizes their tables."""
    import apspie_b200 as ap
    A = ap.gen_powerlaw(1 << 12, 1 << 11, max_deg=1024, seed=2)
    B = ap.gen_powerlaw(1 << 11, 1 << 14, max_deg=1024, seed=3)
    dA, dB = _dev_csr(A), _dev_csr(B)
    rp, ri, rv = oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, A.w_f32, B.ptr, B.ind, B.w_f32)
    _, _, mag = oracle.spgemm(A.m, B.ncols, A.ptr, A.ind, np.abs(A.w_f32), B.ptr, B.ind,
                              np.abs(B.w_f32))
    try:
        for load, warp, bitmap in itertools.product((2, 4), (256, 64, 0), (1 << 18, 0)):
            ap.set_tuning(ctx, spgemm_table_load=load, spgemm_warp_max_prod=warp,
                          spgemm_bitmap_max_cols=bitmap)
            cp, ci, cv = ap.spgemm(ctx, dA, dB)
            tag = f"load {load} warp {warp} bitmap {bitmap}"
            np.testing.assert_array_equal(cp.cpu().numpy(), rp.astype(np.int32), err_msg=tag)
            np.testing.assert_array_equal(ci.cpu().numpy(), ri, err_msg=tag)
            err = np.abs(cv.cpu().numpy().astype(np.float64) - rv)
            assert np.all(err <= VAL_RTOL * np.abs(rv) + 1e-12 * mag + 1e-30), (tag, err.max())
        ap.reset_tuning(ctx)
        first = ap.autotune_spgemm(ctx, dA, dB)
        assert not first["cached"] and first["table_load"] in (2, 4)
        assert first["warp_max_prod"] in (256, 64) and first["ms"] > 0
        ap.reset_tuning(ctx)
        again = ap.autotune_spgemm(ctx, dA, dB)
        assert again["cached"] and {k: again[k] for k in ("table_load", "warp_max_prod",
                                                          "bitmap_max_cols")} == \
            {k: first[k] for k in ("table_load", "warp_max_prod", "bitmap_max_cols")}
        cp, ci, _ = ap.spgemm(ctx, dA, dB)          # the tuner left no plan behind it
        np.testing.assert_array_equal(ci.cpu().numpy(), ri)
    finally:
        ap.reset_tuning(ctx)


def test_spgemm_tuning_is_validated(ctx):
    import apspie_b200 as ap
    for bad in ({"spgemm_table_load": 3}, {"spgemm_warp_max_prod": 512},
                {"bfs_blocks_per_sm": -1}, {"spgemm_bitmap_max_cols": -1}):
        with pytest.raises(ap.ApspieError):
            ap.set_tuning(ctx, **bad)
    ap.reset_tuning(ctx)


def test_batch_tuner_caches_and_keeps_every_row(ctx):
    """A mix with a deep graph (a grid: its sources run beside the
    multi-source launch) so that the deep share is a candidate too."""
    import torch
    import apspie_b200 as ap
    r = ap.gen_rmat(13, 16, seed=4)
    ap.weights_u32(r, seed=4)
    grid = ap.gen_grid(96, 96)
    ap.weights_u32(grid, seed=5)
    dr, dg = r.to_device(), grid.to_device()
    jobs = [{"type": "bfs", "graph": dr, "sources": ap.seeded_sources(r, 40, seed=1)},
            {"type": "sssp", "graph": dr, "sources": ap.seeded_sources(r, 12, seed=2)},
            {"type": "bfs", "graph": dg, "sources": list(range(0, grid.m, grid.m // 6))},
            {"type": "sssp", "graph": dg, "sources": [0, grid.m - 1]}]
    try:
        first = ap.autotune_batch(ctx, jobs)
        assert not first["cached"] and first["blocks_per_sm"] in (0, 1) and first["ms"] > 0
        ap.reset_tuning(ctx)
        again = ap.autotune_batch(ctx, jobs)
        assert again["cached"] and (again["blocks_per_sm"], again["deep_blocks"]) == \
            (first["blocks_per_sm"], first["deep_blocks"])
        import ctypes as C
        from apspie_b200._native import lib
        nres = C.c_int()
        assert lib.apspie_ctx_resident_blocks(ctx.handle, C.byref(nres)) == 0
        resident = nres.value
        for bps, deep in ((0, 0), (1, 0), (0, resident // 4), (1, (3 * resident) // 4)):
            ap.set_tuning(ctx, batch_blocks_per_sm=bps, batch_deep_blocks=deep)
            outs = ap.batch_run(ctx, jobs)
            for j, out in zip(jobs, outs):
                for i, s in enumerate(j["sources"]):
                    ref = (ap.bfs(ctx, j["graph"], s) if j["type"] == "bfs"
                           else ap.sssp(ctx, j["graph"], s, weights="u32"))
                    assert torch.equal(out[i], ref), f"{j['type']} src {s} blocks {bps} deep {deep}"
    finally:
        ap.reset_tuning(ctx)
