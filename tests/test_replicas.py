"""Multi-GPU replicas on the CPU: two gloo ranks (127.0.0.1) combine their
figures as bench.py --gpus N does (slowest rank's time, summed work), and the
ranks' seed-chosen sources are distinct and reproducible.  No GPU needed."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import apspie_b200 as ap
        from apspie_b200.replicas import aggregate, replica_sources
        ms, work = aggregate(1.5 + rank, 100.0 * (rank + 1))
        h = ap.gen_rmat(10, 8, seed=2)
        q.put((rank, ms, work, replica_sources(h, 5, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_combine_time_and_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, work, _ in res:
        assert ms == 2.5 and work == 300.0       # max over ranks, sum over ranks
    s0, s1 = res[0][3], res[1][3]
    assert s0 != s1                               # replicas share no queries
    import apspie_b200 as ap
    from apspie_b200.replicas import replica_sources
    h = ap.gen_rmat(10, 8, seed=2)
    assert replica_sources(h, 5, 0) == s0 and replica_sources(h, 5, 1) == s1


def test_aggregate_without_a_process_group():
    from apspie_b200.replicas import aggregate
    assert aggregate(3.0, 7.0) == (3.0, 7.0)
