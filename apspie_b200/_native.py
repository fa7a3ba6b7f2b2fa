"""ctypes binding of libapspie_b200.so (the C ABI declared in include/apspie.h).

The library is built in-tree by ``python -m apspie_b200.build``.  There is no
fallback: importing this module raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libapspie_b200.so"

if not LIB_PATH.exists():
    raise ImportError(
        f"apspie_b200 native library not built: {LIB_PATH} is missing "
        "(run `python apspie_b200/build.py`)")

lib = C.CDLL(str(LIB_PATH))

c_int, c_i64, c_u64, c_u32, c_f32 = C.c_int, C.c_int64, C.c_uint64, C.c_uint32, C.c_float
vp = C.c_void_p
P_int = C.POINTER(C.c_int)
P_i64 = C.POINTER(C.c_int64)
P_u64 = C.POINTER(C.c_uint64)
P_size = C.POINTER(C.c_size_t)
P_vp = C.POINTER(C.c_void_p)


class BfsStats(C.Structure):
    _fields_ = [("levels", C.c_int32), ("pull_levels", C.c_int32),
                ("vertices_reached", C.c_int64), ("edges_traversed", C.c_int64)]


class SsspStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("phases", C.c_int32), ("vertices_reached", C.c_int64),
                ("edges_traversed", C.c_int64), ("relaxations", C.c_int64)]


class Csr(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int64), ("d_ptr", C.c_void_p),
                ("d_ind", C.c_void_p), ("d_val", C.c_void_p)]


class Job(C.Structure):
    _fields_ = [("type", C.c_int), ("m", C.c_int), ("nnz", C.c_int64), ("d_ptr", C.c_void_p),
                ("d_ind", C.c_void_p), ("d_tptr", C.c_void_p), ("d_tind", C.c_void_p),
                ("d_w", C.c_void_p), ("symmetric", C.c_int), ("nsrc", C.c_int),
                ("h_src", C.POINTER(C.c_int)), ("d_out", C.c_void_p), ("alpha", C.c_int),
                ("beta", C.c_int), ("d_stptr", C.c_void_p), ("d_stind", C.c_void_p),
                ("d_stw", C.c_void_p)]


class BatchStats(C.Structure):
    _fields_ = [("super_steps", C.c_int32), ("pad", C.c_int32), ("frontier_edges", C.c_int64)]


class Tuning(C.Structure):
    _fields_ = [("bfs_alpha", C.c_int32), ("bfs_beta", C.c_int32),
                ("bfs_blocks_per_sm", C.c_int32), ("sssp_blocks_per_sm", C.c_int32),
                ("sssp_pull_alpha", C.c_int32), ("batch_blocks_per_sm", C.c_int32),
                ("batch_deep_blocks", C.c_int32), ("spgemm_table_load", C.c_int32),
                ("spgemm_warp_max_prod", C.c_int32), ("spgemm_bitmap_max_cols", C.c_int64),
                ("spmspv_sort_factor", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("batches", C.c_uint64), ("jobs", C.c_uint64),
                ("pending", C.c_uint64), ("in_flight_bytes", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("max_ms", C.c_double), ("admission_waits", C.c_uint64),
                ("memory_cap_bytes", C.c_uint64), ("max_launch_ms", C.c_double)]


# name -> (restype, argtypes); every symbol declared in include/apspie.h
PROTOS: dict[str, tuple] = {
    "apspie_ctx_create": (c_int, [c_int, vp, P_vp]),
    "apspie_ctx_destroy": (c_int, [vp]),
    "apspie_ctx_set_stream": (c_int, [vp, vp]),
    "apspie_ctx_set_max_grid": (c_int, [vp, c_int]),
    "apspie_ctx_resident_blocks": (c_int, [vp, P_int]),
    "apspie_ctx_sync": (c_int, [vp]),
    "apspie_ctx_launch_count": (c_int, [vp, P_u64]),
    "apspie_ctx_workspace_bytes": (c_int, [vp, P_size]),
    "apspie_last_error": (C.c_char_p, [vp]),
    "apspie_status_string": (C.c_char_p, [c_int]),
    "apspie_bfs": (c_int, [vp, c_int, c_i64, c_int, vp, vp, vp, vp, vp, c_int]),
    "apspie_bfs_noalloc": (c_int, [vp, c_int, c_i64, c_int, vp, vp, vp, vp, vp, c_int]),
    "apspie_bfs_noalloc_status": (c_int, [vp, vp]),
    "apspie_debug_inject": (c_int, [vp, c_int]),
    "apspie_server_debug_fail_next": (c_int, [vp, c_int]),
    "apspie_bfs_get_stats": (c_int, [vp, C.POINTER(BfsStats)]),
    "apspie_csr_transpose": (c_int, [vp, c_int, c_int, c_i64, vp, vp, vp, vp, vp, vp]),
    "apspie_bfs_prepare": (c_int, [vp, c_int, c_i64, vp, vp, vp, vp]),
    "apspie_bfs_get_trace": (c_int, [vp, c_int, P_int, vp, vp, vp, vp, vp, vp, vp, vp]),
    "apspie_bfs_set_params": (c_int, [vp, c_int, c_int, c_int]),
    "apspie_sssp_u32": (c_int, [vp, c_int, c_i64, c_int, vp, vp, vp, vp, c_int]),
    "apspie_sssp_f32": (c_int, [vp, c_int, c_i64, c_int, vp, vp, vp, vp, c_int]),
    "apspie_sssp_set_params": (c_int, [vp, c_u32, c_f32]),
    "apspie_sssp_get_trace": (c_int, [vp, c_int, P_int, vp, vp, vp, vp]),
    "apspie_sssp_get_stats": (c_int, [vp, C.POINTER(SsspStats)]),
    "apspie_sssp_u32_pull": (c_int, [vp, c_int, c_i64, c_int, vp, vp, vp, vp, vp, vp, vp, c_int]),
    "apspie_sssp_f32_pull": (c_int, [vp, c_int, c_i64, c_int, vp, vp, vp, vp, vp, vp, vp, c_int]),
    "apspie_sssp_set_pull": (c_int, [vp, c_int]),
    "apspie_mis": (c_int, [vp, c_i64, c_int, vp, vp, vp, vp, c_f32]),
    "apspie_mis_get_rounds": (c_int, [vp, P_int]),
    "apspie_neighbor_flags": (c_int, [vp, c_i64, c_int, vp, vp, vp, vp]),
    "apspie_spmspv": (c_int, [vp, c_int, c_int, c_i64, vp, vp, vp, c_int, vp, vp, vp, vp, P_int,
                              P_i64]),
    "apspie_spmv": (c_int, [vp, c_int, c_int, c_i64, vp, vp, vp, vp, vp]),
    "apspie_mxv_dense": (c_int, [vp, c_int, c_int, c_i64, vp, vp, vp, vp, vp, P_i64]),
    "apspie_spmspv_set_params": (c_int, [vp, C.c_double]),
    "apspie_spgemm": (c_int, [vp, C.POINTER(Csr), C.POINTER(Csr), C.POINTER(Csr)]),
    "apspie_spgemm_symbolic": (c_int, [vp, C.POINTER(Csr), C.POINTER(Csr), vp, P_i64]),
    "apspie_spgemm_numeric": (c_int, [vp, C.POINTER(Csr), C.POINTER(Csr), vp, vp, vp]),
    "apspie_spgemm_set_params": (c_int, [vp, c_i64]),
    "apspie_csr_free": (c_int, [vp, C.POINTER(Csr)]),
    "apspie_csr_copy_out": (c_int, [vp, C.POINTER(Csr), vp, vp, vp]),
    "apspie_tc_prepare": (c_int, [vp, c_i64, c_int, vp, vp, vp, vp, vp, P_i64]),
    "apspie_tc": (c_int, [vp, c_int, c_i64, vp, vp, P_i64]),
    "apspie_batch_run": (c_int, [vp, c_int, C.POINTER(Job), c_int]),
    "apspie_batch_set_params": (c_int, [vp, c_int]),
    "apspie_batch_set_deep_mode": (c_int, [vp, c_int]),
    "apspie_batch_set_sssp_pull": (c_int, [vp, c_int]),
    "apspie_batch_get_stats": (c_int, [vp, C.POINTER(BatchStats)]),
    "apspie_autotune_bfs": (c_int, [vp, c_int, P_int, c_i64, c_int, vp, vp, vp, vp, vp, P_int,
                                    P_int, C.POINTER(C.c_float)]),
    "apspie_autotune_spmspv": (c_int, [vp, c_int, c_i64, vp, vp, vp, vp, vp, vp, vp,
                                       C.POINTER(C.c_double)]),
    "apspie_autotune_sssp": (c_int, [vp, c_int, P_int, c_i64, c_int, vp, vp, vp, vp, vp, vp, vp,
                                     C.POINTER(C.c_float), P_int]),
    "apspie_autotune_spgemm": (c_int, [vp, C.POINTER(Csr), C.POINTER(Csr),
                                       C.POINTER(C.c_float), P_int]),
    "apspie_autotune_batch": (c_int, [vp, c_int, C.POINTER(Job), C.POINTER(C.c_float), P_int]),
    "apspie_ctx_get_tuning": (c_int, [vp, C.POINTER(Tuning)]),
    "apspie_ctx_set_tuning": (c_int, [vp, C.POINTER(Tuning)]),
    "apspie_server_create": (c_int, [c_int, C.c_size_t, c_int, P_vp]),
    "apspie_server_add_graph": (c_int, [vp, c_int, c_i64, vp, vp, vp, vp, vp, c_int, P_int]),
    "apspie_server_set_sssp_in": (c_int, [vp, c_int, vp, vp, vp]),
    "apspie_server_submit": (c_int, [vp, c_int, c_int, c_int, c_u32, vp, P_u64]),
    "apspie_server_submit_device": (c_int, [vp, c_int, c_int, c_int, c_u32, vp, P_u64]),
    "apspie_server_replay": (c_int, [vp, c_int, vp, c_int, vp, C.POINTER(C.c_double)]),
    "apspie_server_replay_plain": (c_int, [vp, c_int, vp, c_int, vp, C.POINTER(C.c_double)]),
    "apspie_server_replay_keep": (c_int, [vp, c_int, vp, c_int, vp, vp, C.POINTER(C.c_double)]),
    "apspie_server_poll": (c_int, [vp, c_u64, P_int, C.POINTER(C.c_double)]),
    "apspie_server_wait": (c_int, [vp, c_u64, C.POINTER(C.c_double)]),
    "apspie_server_get_stats": (c_int, [vp, C.POINTER(ServerStats)]),
    "apspie_server_reset_stats": (c_int, [vp]),
    "apspie_server_destroy": (c_int, [vp]),
    "apspie_gen_rmat_host": (c_int, [c_int, c_int, c_u64, c_int, c_int, P_int, P_i64, P_vp, P_vp]),
    "apspie_gen_er_host": (c_int, [c_int, c_int, c_u64, P_i64, P_vp, P_vp]),
    "apspie_gen_rmat_device": (c_int, [vp, c_int, c_int, c_u64, c_int, c_int, C.POINTER(Csr)]),
    "apspie_gen_er_device": (c_int, [vp, c_int, c_int, c_u64, C.POINTER(Csr)]),
    "apspie_gen_weights_u32_device": (c_int, [vp, c_int, vp, vp, c_u64, c_u32, c_u32, vp]),
    "apspie_gen_weights_f32_device": (c_int, [vp, c_int, vp, vp, c_u64, vp]),
    "apspie_gen_grid_host": (c_int, [c_int, c_int, P_i64, P_vp, P_vp]),
    "apspie_gen_weights_u32_host": (c_int, [c_int, vp, vp, c_u64, c_u32, c_u32, vp]),
    "apspie_gen_weights_f32_host": (c_int, [c_int, vp, vp, c_u64, vp]),
    "apspie_gen_powerlaw_host": (c_int, [c_int, c_int, C.c_double, C.c_double, c_int, c_u64,
                                         C.POINTER(C.c_double), P_i64, P_vp, P_vp, P_vp]),
    "apspie_mt19937_fill_host": (c_int, [c_u32, c_i64, vp]),
    "apspie_read_mtx_host": (c_int, [C.c_char_p, c_int, P_int, P_i64, P_vp, P_vp, P_vp, P_int]),
    "apspie_host_free": (None, [vp]),
}

for _name, (_res, _args) in PROTOS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class ApspieError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def check(status: int, ctx=None, what: str = "") -> None:
    if status != 0:
        detail = ""
        if ctx is not None:
            detail = (lib.apspie_last_error(ctx) or b"").decode()
        if not detail:
            detail = (lib.apspie_status_string(status) or b"").decode()
        raise ApspieError(status, f"{what}: {detail}" if what else detail)
