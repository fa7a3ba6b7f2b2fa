"""Failure paths: every device-side wait is bounded and ends in
APSPIE_ERR_TIMEOUT, an allocation failure is a status (never an exit), a
failed server request fails alone.  The failures are made without faulting
or hanging the GPU: a one-shot test hook (apspie_debug_inject) makes one
block leave a BFS launch before its first grid barrier (the others' bounded
barrier wait runs out), makes the first tile of a radix sort withhold its
look-back status (its successors' bounded waits run out), or fails the next
workspace allocation on the host; the server's hook fails one query group on
the host.  After each failure the context (or server) is used again and
must give correct results."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

APSPIE_ERR_OOM = 2
APSPIE_ERR_CUDA = 3
APSPIE_ERR_TIMEOUT = 4
INJECT_BFS_BARRIER, INJECT_SORT_LOOKBACK, INJECT_ALLOC_FAIL = 1, 2, 3


def test_bfs_barrier_timeout_is_reported_and_the_context_recovers():
    import apspie_b200 as ap
    from apspie_b200._native import lib
    h = ap.gen_rmat(12, 16, seed=2)
    g = h.to_device()
    src = ap.seeded_sources(h, 1, seed=3)[0]
    ref, _ = oracle.bfs(h.m, h.ptr, h.ind, src)
    with ap.Context(0) as ctx:
        np.testing.assert_array_equal(ap.bfs(ctx, g, src).cpu().numpy(), ref)
        assert lib.apspie_debug_inject(ctx.handle, INJECT_BFS_BARRIER) == 0
        ap.bfs(ctx, g, src)                     # launches; the wait runs out on the device
        with pytest.raises(ap.ApspieError) as e:
            ap.bfs_stats(ctx)
        assert e.value.status == APSPIE_ERR_TIMEOUT
        # the context is usable: both barrier counter sets come back clean
        for _ in range(3):
            np.testing.assert_array_equal(ap.bfs(ctx, g, src).cpu().numpy(), ref)
            assert ap.bfs_stats(ctx)["vertices_reached"] == int((ref >= 0).sum())


def test_sort_lookback_timeout_is_reported_by_spmspv():
    import torch
    import apspie_b200 as ap
    from apspie_b200._native import lib
    h = ap.gen_rmat(14, 16, seed=4, symmetric=False)
    g = h.to_device()
    val = torch.ones(h.nnz, dtype=torch.float32, device="cuda")
    xind = np.arange(0, h.m, 3, dtype=np.int32)
    xi = torch.from_numpy(xind).cuda()
    with ap.Context(0) as ctx:
        ap.spmspv_set_params(ctx, 0.0)         # always the radix-sort path
        yi, yv, _ = ap.spmspv(ctx, 0, g, xi, None, val)
        ryi, ryv = oracle.spmspv(0, h.m, h.ptr, h.ind, None, xind, None)
        np.testing.assert_array_equal(yi.cpu().numpy(), ryi)
        assert lib.apspie_debug_inject(ctx.handle, INJECT_SORT_LOOKBACK) == 0
        with pytest.raises(ap.ApspieError) as e:
            ap.spmspv(ctx, 0, g, xi, None, val)
        assert e.value.status == APSPIE_ERR_TIMEOUT
        # cleared: the next call sorts again, correctly
        yi, yv, _ = ap.spmspv(ctx, 0, g, xi, None, val)
        np.testing.assert_array_equal(yi.cpu().numpy(), ryi)
        np.testing.assert_allclose(yv.cpu().numpy(), ryv, rtol=1e-6)


def test_allocation_failure_is_a_status():
    import apspie_b200 as ap
    from apspie_b200._native import lib
    h = ap.gen_rmat(12, 16, seed=5)
    ap.weights_u32(h, seed=5)
    g = h.to_device()
    src = ap.seeded_sources(h, 1, seed=1)[0]
    with ap.Context(0) as ctx:
        assert lib.apspie_debug_inject(ctx.handle, INJECT_ALLOC_FAIL) == 0
        with pytest.raises(ap.ApspieError) as e:    # a fresh context must grow its workspace
            ap.sssp(ctx, g, src, weights="u32")
        assert e.value.status == APSPIE_ERR_OOM
        d = ap.sssp(ctx, g, src, weights="u32").cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(d, oracle.sssp_u32(h.m, h.ptr, h.ind, h.w_u32, src))


def test_server_failed_request_fails_alone():
    import apspie_b200 as ap
    hs = [ap.gen_rmat(12, 16, seed=6), ap.gen_rmat(13, 16, seed=7)]
    for i, h in enumerate(hs):
        ap.weights_u32(h, seed=i)
    ds = [h.to_device() for h in hs]
    rng = np.random.default_rng(9)
    with ap.Context(0) as ctx, ap.Server(budget_bytes=4 << 30, max_batch=64) as srv:
        gids = [srv.add_graph(d) for d in ds]
        srv.debug_fail_next(2)                   # the first MIS group launched fails
        qs = [(int(rng.integers(2)), int(rng.choice([0, 1])), 0) for _ in range(60)]
        qs = [(gi, k, int(rng.integers(hs[gi].m))) for gi, k, _ in qs]
        rids = [srv.submit(k, gids[gi], s) for gi, k, s in qs]
        bad = srv.submit(2, gids[0], 0, seed=777)   # a group of its own: (graph 0, seed 777)
        with pytest.raises(ap.ApspieError) as e:
            srv.wait(bad)
        assert e.value.status == APSPIE_ERR_CUDA
        for (gi, k, s), rid in zip(qs, rids):
            out, _ = srv.wait(rid)
            ref = ap.bfs(ctx, ds[gi], s) if k == 0 else ap.sssp(ctx, ds[gi], s, weights="u32")
            np.testing.assert_array_equal(out, ref.cpu().numpy())
        # the server keeps serving, MIS included
        again = srv.submit(2, gids[0], 0, seed=777)
        out, _ = srv.wait(again)
        prio = oracle.mt_fill(777, hs[0].m)
        np.testing.assert_array_equal(out, oracle.mis(hs[0].m, hs[0].ptr, hs[0].ind, prio))
