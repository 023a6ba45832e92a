"""Independent networks sharded across ranks (one process per GPU).

The batched parameter sweep and the adjoint batch are independent networks with
no synapse between them, so they partition by network with no data-path
collective: each rank takes a contiguous, cost-balanced slice of the network
table, runs it on its own GPU, and the per-network results are gathered on rank
0 in network order.  The reference runs one OpenMP queue per GPU the same way,
each queue owning its own neurons (src/openmp/openmp_GPU.cu:44-78); its only
exchange, spikes between queues, does not exist between independent networks.

Everything here is host logic over ``torch.distributed`` (NCCL on GPUs, gloo on
CPU); the per-rank work is any function of a slice of network specs, e.g.
:func:`run_sweep_slice` on a GPU.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def network_cost(spec: dict) -> float:
    """Work of one network per step, up to a constant: its neuron updates plus its
    synapses (explicit, or expected from the connection probability)."""
    n = float(spec["n"])
    if "src" in spec:
        m = float(len(spec["src"]))
    else:
        m = float(spec.get("p", 0.1)) * (n + float(spec.get("n_in", 0))) * n
    return n + m


def partition(costs: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous slices [lo, hi) of range(len(costs)), one per rank in rank order.

    The cut after rank r's slice is the network whose cost prefix is closest to
    (r + 1) / world of the total, so every network is in exactly one slice and each
    slice's cost is within one network's cost of an equal share.  Slices may be
    empty when there are fewer networks than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, np.float64)
    n = len(c)
    if n == 0:
        return [(0, 0)] * world
    pre = np.concatenate([[0.0], np.cumsum(c)])
    total = pre[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        j = int(np.searchsorted(pre, target))
        if j > 0 and abs(pre[j - 1] - target) <= abs(pre[min(j, n)] - target):
            j -= 1
        j = min(max(j, bounds[-1]), n)
        bounds.append(j)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def gather_in_order(local: list, rank: int, world: int, dst: int = 0) -> Optional[list]:
    """Concatenate every rank's per-network list on rank ``dst`` (rank order, so
    network order for the slices of :func:`partition`); None on the other ranks.
    Every rank takes the same collective step."""
    if world == 1:
        return list(local)
    import torch.distributed as dist
    parts = [None] * world if rank == dst else None
    dist.gather_object(local, parts, dst=dst)
    if rank != dst:
        return None
    out = []
    for p in parts:
        out.extend(p)
    return out


def run_sharded(specs: Sequence[dict], work: Callable[[Sequence[dict]], list], rank: int, world: int,
                dst: int = 0) -> Optional[list]:
    """Run ``work`` on this rank's slice of ``specs`` (it returns one result per
    network of the slice) and gather all results on ``dst`` in network order."""
    lo, hi = partition([network_cost(s) for s in specs], world)[rank]
    local = work(specs[lo:hi]) if hi > lo else []
    if len(local) != hi - lo:
        raise RuntimeError("work returned %d results for %d networks" % (len(local), hi - lo))
    return gather_in_order(local, rank, world, dst)


def run_sweep_slice(specs: Sequence[dict], n_steps: int, integrator: str = "RK2", device: int = 0,
                    autotune_steps: int = 0) -> list:
    """GPU work of one rank: its networks in one persistent sweep for ``n_steps``
    steps; returns each network's spikes as (steps, cells) arrays."""
    from .sweep import Sweep
    sw = Sweep.from_specs(list(specs), n_steps_max=n_steps, integrator=integrator, device=device)
    try:
        if autotune_steps:
            sw.autotune(autotune_steps)
        sw.reset()
        sw.run(n_steps)
        return [sw.spikes(i) for i in range(len(specs))]
    finally:
        sw.close()
