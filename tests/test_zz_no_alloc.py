"""apspie_bfs_noalloc -- the BFS entry point that allocates no memory.

Callers such as code running under CUDA graph stream capture, hosts with a
fixed device-memory budget, or plugins in a process whose allocator they do
not own cannot call cudaMalloc.  This entry point keeps its scratch in one
fixed device array (at most 2^20 vertices, 2^24 edges).  The test calls it
through the C ABI and checks it against apspie_bfs, the entry point that
draws scratch from a context workspace: BFS depths are integers, so the
tolerance is zero.  Two calls in a row on the same array show that the
contents left by one call do not leak into the next.  The status word,
copied out by apspie_bfs_noalloc_status after a traversal, reports 0 for a
finished traversal and APSPIE_ERR_TIMEOUT when a bounded grid-barrier wait
gave up (made to happen by a test hook that makes one block leave before
the barrier; the others' wait runs out, nothing faults or hangs).

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

APSPIE_ERR_TIMEOUT = 4
APSPIE_ERR_TOO_LARGE = 8
INJECT_BFS_BARRIER = 1


def _p(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _noalloc(lib, stream, g, src, out, tptr, tind, max_levels=0, status=None):
    """The traversal, then (status given) its status word copied to `status`
    on the same stream."""
    rc = lib.apspie_bfs_noalloc(C.c_void_p(stream.cuda_stream), int(src), int(g.nnz), int(g.m),
                                _p(g.ptr), _p(g.ind), _p(tptr), _p(tind), _p(out),
                                int(max_levels))
    if rc == 0 and status is not None:
        rc = lib.apspie_bfs_noalloc_status(C.c_void_p(stream.cuda_stream), _p(status))
    return rc


@pytest.mark.parametrize("symmetric", [True, False])
def test_noalloc_bfs_matches_bfs_twice(symmetric):
    import torch

    import apspie_b200 as ap
    from apspie_b200._native import lib

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = ap.gen_rmat(16, 16, seed=21, symmetric=symmetric)   # 65,536 vertices, within the limits
    g = h.to_device()
    tptr, tind = (g.ptr, g.ind) if symmetric else (g.tptr, g.tind)
    stream = torch.cuda.current_stream()
    with ap.Context(0) as ctx:
        sources = ap.seeded_sources(h, 2, seed=4)
        status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        for s in sources:                       # two calls in a row share the scratch array
            ref = ap.bfs(ctx, g, s).cpu().numpy()
            out = torch.full((h.m,), 7, dtype=torch.int32, device="cuda")
            assert _noalloc(lib, stream, g, s, out, tptr, tind, status=status) == 0
            torch.cuda.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), ref)
            assert int(status.item()) == 0      # finished: no wait gave up
        # the fixed iteration count and the push-only form (no in-adjacency)
        s = sources[0]
        ref = ap.bfs(ctx, g, s, max_levels=3).cpu().numpy()
        out = torch.empty(h.m, dtype=torch.int32, device="cuda")
        assert _noalloc(lib, stream, g, s, out, None, None, max_levels=3) == 0
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch

    from apspie_b200._native import lib

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    stream = torch.cuda.current_stream()
    ptr = torch.zeros(2, dtype=torch.int32, device="cuda")
    out = torch.empty(1, dtype=torch.int32, device="cuda")
    # more vertices than the array holds: refused before anything is launched
    rc = lib.apspie_bfs_noalloc(C.c_void_p(stream.cuda_stream), 0, 0, (1 << 20) + 1, _p(ptr),
                                None, None, None, _p(out), 0)
    assert rc == APSPIE_ERR_TOO_LARGE
    rc = lib.apspie_bfs_noalloc(C.c_void_p(stream.cuda_stream), 0, (1 << 24) + 1, 1, _p(ptr),
                                _p(ptr), None, None, _p(out), 0)
    assert rc == APSPIE_ERR_TOO_LARGE
    assert lib.apspie_status_string(rc) == b"input exceeds the fixed scratch size"
    # the status copy needs somewhere to write: refused, nothing launched
    assert lib.apspie_bfs_noalloc_status(C.c_void_p(stream.cuda_stream), None) == 1


def test_noalloc_bfs_inside_a_cuda_graph():
    """A caller captures apspie_bfs_noalloc (its init kernel and the
    cooperative persistent kernel) into a CUDA graph and replays it: the
    replay writes the same depths as a direct call."""
    import torch

    import apspie_b200 as ap
    import oracle
    from apspie_b200._native import lib

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = ap.gen_rmat(14, 16, seed=3)
    g = h.to_device()
    src = ap.seeded_sources(h, 1, seed=1)[0]
    depth = torch.empty(h.m, dtype=torch.int32, device="cuda")
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        assert _noalloc(lib, side, g, src, depth, g.ptr, g.ind) == 0   # first call: outside capture
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        assert _noalloc(lib, side, g, src, depth, g.ptr, g.ind) == 0
    depth.fill_(7)
    torch.cuda.synchronize()
    for _ in range(2):
        graph.replay()
        torch.cuda.synchronize()
        ref, _ = oracle.bfs(h.m, h.ptr, h.ind, src)
        np.testing.assert_array_equal(depth.cpu().numpy(), ref)
        depth.fill_(7)


def test_noalloc_status_reports_a_barrier_timeout():
    """The status word tells a caller that cannot synchronise whether the
    depths are complete: a timeout after a one-shot test hook made one block
    leave before the first grid barrier, then 0 again on the next call, whose
    depths are right."""
    import torch

    import apspie_b200 as ap
    import oracle
    from apspie_b200._native import lib

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = ap.gen_rmat(12, 16, seed=8)
    g = h.to_device()
    src = ap.seeded_sources(h, 1, seed=2)[0]
    ref, _ = oracle.bfs(h.m, h.ptr, h.ind, src)
    stream = torch.cuda.current_stream()
    out = torch.empty(h.m, dtype=torch.int32, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert _noalloc(lib, stream, g, src, out, g.ptr, g.ind, status=status) == 0   # set-up
    torch.cuda.synchronize()
    assert lib.apspie_debug_inject(None, INJECT_BFS_BARRIER) == 0
    assert _noalloc(lib, stream, g, src, out, g.ptr, g.ind, status=status) == 0
    torch.cuda.synchronize()
    assert int(status.item()) == APSPIE_ERR_TIMEOUT
    assert _noalloc(lib, stream, g, src, out, g.ptr, g.ind, status=status) == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    np.testing.assert_array_equal(out.cpu().numpy(), ref)
