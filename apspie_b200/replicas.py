"""Multi-GPU replicas: BFS / SSSP / MIS queries are independent, so N GPUs run
N independent replicas (one process per GPU, every graph resident on each)
with no collective on the data path.  torch.distributed (NCCL on GPUs, gloo
on CPU) is only the plumbing for the barrier around a timed region and for
combining the ranks' figures: the job's time is the slowest rank's, its work
the sum over ranks."""
from __future__ import annotations


def replica_sources(g, n: int, rank: int, base_seed: int = 0) -> list[int]:
    """n seed-chosen sources of graph g for replica `rank` (distinct seeds per
    rank, so the replicas share no queries; the same on every run)."""
    from .graph import seeded_sources
    return seeded_sources(g, n, seed=base_seed + rank)


def aggregate(ms_local: float, work_local: float, device="cpu") -> tuple[float, float]:
    """(max over ranks of ms_local, sum over ranks of work_local); the local
    values when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(ms_local), float(work_local)
    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    w = torch.tensor([float(work_local)], dtype=torch.float64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
