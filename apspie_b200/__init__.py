"""apspie_b200 -- B200-native (sm_100a) SpMSpV / hash-SpGEMM hot path of apspie.

Python mirror of the reference's host entry points on top of the C ABI in
include/apspie.h (libapspie_b200.so).  Device arrays are torch tensors (torch
is the device allocator and stream provider only); every compute call goes
through the native library, which raises on import if it is not built.
"""
from ._native import ApspieError, lib  # noqa: F401  (raises if the .so is missing)
from .graph import (DeviceGraph, HostGraph, from_edges, gen_er, gen_grid, gen_powerlaw, gen_rmat,  # noqa: F401
                    largest_cc_vertex, mt19937, read_mtx, seeded_sources, weights_f32, weights_u32)
from .serving import Server  # noqa: F401
from .ops import (Context, bfs, bfs_prepare, bfs_set_params, csr_transpose, bfs_stats, bfs_trace, mis, mis_rounds,  # noqa: F401
                  neighbor_flags, sssp, sssp_stats, sssp_set_params, sssp_trace, sssp_prepare, sssp_set_pull, spmspv, spmv, mxv_dense, spmspv_set_params,
                  PLUS_TIMES, MIN_PLUS, MAX_TIMES, OR_AND, spgemm, spgemm_symbolic, spgemm_numeric, spgemm_set_params, tc_prepare,
                  triangle_count, batch_run, batch_stats, batch_set_params, batch_set_sssp_pull, autotune_bfs, autotune_spmspv,
                  autotune_sssp, autotune_spgemm, autotune_batch, get_tuning, set_tuning, reset_tuning,
                  gen_rmat_device, gen_er_device, weights_device)

__all__ = ["Server",
    "ApspieError", "Context", "DeviceGraph", "HostGraph", "bfs", "bfs_prepare", "bfs_set_params", "csr_transpose", "bfs_stats", "bfs_trace", "from_edges",
    "sssp", "sssp_set_params", "sssp_stats", "sssp_trace", "sssp_prepare", "sssp_set_pull", "mis", "mis_rounds", "neighbor_flags", "spmspv", "spmv", "mxv_dense", "spmspv_set_params", "spgemm", "spgemm_symbolic", "spgemm_numeric", "spgemm_set_params", "tc_prepare", "triangle_count", "batch_run", "batch_stats", "batch_set_params", "batch_set_sssp_pull", "autotune_bfs", "autotune_spmspv", "autotune_sssp", "autotune_spgemm", "autotune_batch", "get_tuning", "set_tuning", "reset_tuning", "gen_er", "gen_er_device", "gen_grid", "gen_powerlaw", "gen_rmat", "gen_rmat_device", "largest_cc_vertex", "mt19937", "read_mtx", "seeded_sources",
    "weights_device", "weights_f32", "weights_u32",
]
