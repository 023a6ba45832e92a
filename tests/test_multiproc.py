"""Multi-rank host logic, run as two gloo processes on the CPU (no GPU):

* bench.py's replicas: every rank simulates its own seeded networks and the job's
  time is the slowest rank's;
* sharding of independent networks (edlut_b200.shard): contiguous cost-balanced
  slices, one per rank, gathered on rank 0 in network order."""
import os
import socket

import numpy as np
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


# ---------------------------------------------------------------- sharding ----
def _shard_specs():
    """Independent LIF networks of uneven sizes with explicit connectivity."""
    from edlut_b200.configs import adjoint_networks
    specs = []
    for i, n in enumerate([40, 90, 60, 150, 30, 75, 120]):
        specs += adjoint_networks(seed=100 + i, n_networks=1, n=n, indeg=10, n_inputs=20, in_indeg=4,
                                  rate_hz=60.0, t_end=0.012, w_in_max=2.0)
    return specs


def _oracle_work(specs):
    """CPU stand-in for a rank's GPU sweep: the C oracle on each network, 100 steps."""
    from edlut_b200.network import Layer, NetworkDescription
    from oracle import oracle as O
    out = []
    for s in specs:
        n = s["n"]
        net = NetworkDescription()
        net.add_layer(Layer(n, "LIFTimeDrivenModel", dict(s["params"]), integrator="RK2", dt=1e-4))
        net.add_layer(Layer(s["n_in"], "InputSpikeNeuronModel", output=0))
        stype = ((s["src"] >= s["n_exc"]) & (s["src"] < n)).astype(np.int32)
        net.add_synapses(s["src"].astype(np.int64), s["tgt"].astype(np.int64), 1e-3, stype, s["w"], s["w"], -1)
        r = O.run(net, s["times"], s["cells"].astype(np.int64) + n, 100)
        keep = r["spike_cell"] < n
        out.append((r["spike_step"][keep].tolist(), r["spike_cell"][keep].tolist()))
    return out


def _shard_worker(rank, world, port, out):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from edlut_b200.shard import network_cost, partition, run_sharded
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        specs = _shard_specs()
        mine = partition([network_cost(s) for s in specs], world)[rank]
        res = run_sharded(specs, _oracle_work, rank, world)
        out.put((rank, mine, res))
    finally:
        dist.destroy_process_group()


def test_partition_covers_every_network_once_in_balanced_contiguous_slices():
    from edlut_b200.shard import partition
    rng = np.random.default_rng(4)
    for n, world in [(4096, 8), (64, 2), (7, 3), (3, 8), (1, 1), (0, 4)]:
        costs = rng.uniform(1.0, 10.0, n)
        sl = partition(costs, world)
        assert len(sl) == world and sl[0][0] == 0 and sl[-1][1] == n
        for (a, b), (c, d) in zip(sl, sl[1:]):
            assert b == c and a <= b
        covered = np.concatenate([np.arange(a, b) for a, b in sl]) if n else np.zeros(0)
        assert np.array_equal(covered, np.arange(n))
        if n:
            share = costs.sum() / world
            for a, b in sl:
                assert abs(costs[a:b].sum() - share) <= costs.max() + 1e-9


def test_sharded_networks_gather_to_the_single_rank_result():
    """Two gloo ranks each run their slice of independent networks (the C oracle
    standing in for the GPU); rank 0 gathers the per-network spike trains in network
    order, equal to one rank running every network."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, g0), (r1, s1, g1) = res
    assert g1 is None and g0 is not None
    specs = _shard_specs()
    assert s0[0] == 0 and s0[1] == s1[0] and s1[1] == len(specs) and s0[1] > 0 and s1[1] > s1[0]
    assert g0 == _oracle_work(specs)
