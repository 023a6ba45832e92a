"""The multi-GPU path of bench.py runs independent replicas: every rank simulates
its own seeded networks and the job's time is the slowest rank's.  Here that host
logic runs as two gloo processes on the CPU (no GPU)."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    import numpy as np
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    from edlut_b200.configs import sweep_networks
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        slow = bench.max_over_ranks(0.25 * (rank + 1), world)
        specs = sweep_networks(seed=bench.rank_seed(1, rank), n_networks=3, t_end=0.005)
        sizes = [s["n"] for s in specs]
        # every rank takes the same collective steps: all ranks see all sizes
        gathered = [None] * world
        dist.all_gather_object(gathered, sizes)
        out.put((rank, slow, gathered))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_distinct_workloads():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [0.5, 0.5]           # max over ranks
    g0, g1 = res[0][2], res[1][2]
    assert g0 == g1                                      # same view on every rank
    assert g0[0] != g0[1]                                # rank seeds give different networks


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.max_over_ranks(1.5, 1) == 1.5
    assert bench.rank_seed(7, 0) == 7 and bench.rank_seed(7, 3) == 10
