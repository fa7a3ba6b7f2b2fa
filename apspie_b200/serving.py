"""Python handle on the native query server (apspie_server_* in
include/apspie.h): continuous batching of BFS / SSSP / MIS queries over
device-resident graphs, with per-query latency."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import ApspieError, ServerStats, check, lib
from .ops import _p

BFS, SSSP, MIS = 0, 1, 2

# apspie_query (include/apspie.h)
QUERY_DTYPE = np.dtype([("type", np.int32), ("graph", np.int32), ("source", np.int32),
                        ("seed", np.uint32), ("t_us", np.float64)])


class Server:
    def __init__(self, device: int = 0, budget_bytes: int = 120 << 30, max_batch: int = 256):
        self._h = C.c_void_p()
        check(lib.apspie_server_create(device, budget_bytes, max_batch, C.byref(self._h)),
              what="apspie_server_create")
        self._graphs = []      # keep the device tensors alive
        self._live = {}        # req id -> (result array, graph m)

    def add_graph(self, g) -> int:
        gid = C.c_int()
        sym = bool(getattr(g, "symmetric", False))
        tptr = None if sym else getattr(g, "tptr", None)
        tind = None if sym else getattr(g, "tind", None)
        p = _p
        check(lib.apspie_server_add_graph(self._h, int(g.m), int(g.nnz), p(g.ptr), p(g.ind),
                                          p(tptr), p(tind), p(g.w_u32), int(sym), C.byref(gid)),
              what="apspie_server_add_graph")
        sin = getattr(g, "extra", {}).get("sssp_in", {}).get("u32")
        if sin is not None:
            # in-adjacency with weights from sssp_prepare: push/pull SSSP queries
            check(lib.apspie_server_set_sssp_in(self._h, gid.value, p(sin[0]), p(sin[1]),
                                                p(sin[2])), what="apspie_server_set_sssp_in")
        self._graphs.append(g)
        return gid.value

    def submit(self, kind: int, graph: int, source: int = 0, seed: int = 0) -> int:
        if not 0 <= graph < len(self._graphs):
            raise ApspieError(2, f"apspie_server_submit: unknown graph {graph}")
        m = self._graphs[graph].m
        out = np.empty(m, dtype=np.int32)
        rid = C.c_uint64()
        check(lib.apspie_server_submit(self._h, int(kind), int(graph), int(source), int(seed),
                                       C.c_void_p(out.ctypes.data), C.byref(rid)),
              what="apspie_server_submit")
        self._live[rid.value] = out
        return rid.value

    def submit_device(self, kind: int, graph: int, source: int = 0, seed: int = 0,
                      out=None) -> int:
        """Submit with the result written to the device tensor `out` (int32,
        m entries), or dropped when out is None."""
        if not 0 <= graph < len(self._graphs):
            raise ApspieError(2, f"apspie_server_submit_device: unknown graph {graph}")
        m = self._graphs[graph].m
        if out is not None and (out.numel() < m or out.dtype.itemsize != 4):
            raise ValueError(f"out: needs a device row of {m} 32-bit entries")
        rid = C.c_uint64()
        check(lib.apspie_server_submit_device(self._h, int(kind), int(graph), int(source),
                                              int(seed), _p(out), C.byref(rid)),
              what="apspie_server_submit_device")
        self._live[rid.value] = out
        return rid.value

    def replay(self, queries, plain: bool = False, to_host: bool = True, keep=None):
        """Open-loop replay of a timed query stream: `queries` is a structured
        array with fields type, graph, source, seed, t_us (see QUERY_DTYPE).
        Returns (latencies_ms array, wall_ms); a latency runs from the query's
        arrival until its result is in host memory (to_host) or on the device.
        plain=True runs the stream one query at a time through the
        single-query kernels instead.  keep (batched replay only): a dict
        {query index: int32 device tensor of the graph's m entries} that
        receives those queries' answers (apspie_server_replay_keep)."""
        q = np.ascontiguousarray(queries, dtype=QUERY_DTYPE)
        lat = np.zeros(len(q), dtype=np.float64)
        wall = C.c_double()
        if keep:
            if plain:
                raise ValueError("keep is for the batched replay")
            rows = (C.c_void_p * len(q))()
            for i, t in keep.items():
                m = self._graphs[int(q["graph"][i])].m
                if t.numel() < m or t.dtype.itemsize != 4:
                    raise ValueError(f"keep[{i}]: needs a device row of {m} 32-bit entries")
                rows[i] = _p(t).value  # a contiguous CUDA tensor, or ValueError
            check(lib.apspie_server_replay_keep(self._h, len(q), C.c_void_p(q.ctypes.data),
                                                int(bool(to_host)), rows,
                                                C.c_void_p(lat.ctypes.data), C.byref(wall)),
                  what="apspie_server_replay_keep")
            return lat, wall.value
        fn = lib.apspie_server_replay_plain if plain else lib.apspie_server_replay
        check(fn(self._h, len(q), C.c_void_p(q.ctypes.data), int(bool(to_host)),
                 C.c_void_p(lat.ctypes.data), C.byref(wall)), what="apspie_server_replay")
        return lat, wall.value

    def wait(self, rid: int):
        lat = C.c_double()
        try:
            check(lib.apspie_server_wait(self._h, C.c_uint64(rid), C.byref(lat)),
                  what="apspie_server_wait")
        except ApspieError:
            self._live.pop(rid, None)
            raise
        return self._live.pop(rid), lat.value

    def debug_fail_next(self, kind: int) -> None:
        """Test hook: the next group of this kind fails without running."""
        check(lib.apspie_server_debug_fail_next(self._h, int(kind)),
              what="apspie_server_debug_fail_next")

    def poll(self, rid: int):
        done, lat = C.c_int(), C.c_double()
        check(lib.apspie_server_poll(self._h, C.c_uint64(rid), C.byref(done), C.byref(lat)),
              what="apspie_server_poll")
        if done.value:
            return self._live.pop(rid), lat.value
        return None

    def stats(self) -> dict:
        s = ServerStats()
        check(lib.apspie_server_get_stats(self._h, C.byref(s)), what="apspie_server_get_stats")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def reset_stats(self) -> None:
        check(lib.apspie_server_reset_stats(self._h), what="apspie_server_reset_stats")

    def close(self) -> None:
        if self._h:
            lib.apspie_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
