"""Independent systems across GPUs: one process per GPU, no collective in the
data path.

A sweep or a request trace is a set of independent systems, so it shards by
system: ``partition`` assigns systems to ranks by longest-processing-time
bin packing on ``beads x steps`` (deterministic, the same on every rank;
the populations of one box, coupled, go to one rank together), each
rank steps its own systems in one ``Batch`` on its own GPU, and only the
final host-side results travel (``torch.distributed.gather_object``), once,
after the run.  Timing across ranks is the max over ranks of each rank's
device time.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(costs, world_size):
    """LPT bin packing: list of system indices per rank.  Ties go to the
    lower rank; the result depends only on ``costs`` and ``world_size``."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def units(n, couplings=()):
    """Systems bundled into units that stay on one rank: the members of each
    coupled group (populations of one box, ``Batch.couple``) together, every
    other system alone."""
    grouped = set()
    out = []
    for members, *_ in couplings:
        members = [int(m) for m in members]
        if grouped & set(members):
            raise ValueError("a system belongs to two coupled groups")
        grouped |= set(members)
        out.append(sorted(members))
    out += [[i] for i in range(n) if i not in grouped]
    return out


def partition_units(costs, couplings, world_size):
    """``partition`` over units: a coupled group goes to one rank whole."""
    us = units(len(costs), couplings)
    parts = partition([sum(costs[i] for i in u) for u in us], world_size)
    return [sorted(i for k in p for i in us[k]) for p in parts]


def imbalance(costs, parts):
    loads = [sum(costs[i] for i in p) for p in parts]
    return max(loads) / (sum(loads) / len(loads)) if sum(loads) else 1.0


def run_sharded(specs, steps, runner, rank=None, world_size=None, group=None, couplings=()):
    """Run `steps` steps of every system, each rank running its share with
    `runner(list_of_specs, steps) -> list_of_results`; rank 0 returns the
    results of all systems in their original order, other ranks None.
    ``couplings``: groups ``(members, fixed, cross_wca)`` of systems that are
    populations of one box; each stays on one rank, and the runner is called
    as ``runner(specs, steps, local_couplings)`` with the members renumbered
    to positions in its own list."""
    import torch.distributed as dist
    if world_size is None:
        world_size = dist.get_world_size(group) if dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank(group) if dist.is_initialized() else 0
    costs = [s.n * steps for s in specs]
    parts = partition_units(costs, couplings, world_size)
    mine = parts[rank]
    if couplings:
        pos = {g: k for k, g in enumerate(mine)}
        local_c = [([pos[m] for m in members], fixed, cross) for members, fixed, cross in couplings
                   if all(m in pos for m in members)]
        local = runner([specs[i] for i in mine], steps, local_c) if mine else []
    else:
        local = runner([specs[i] for i in mine], steps) if mine else []
    payload = list(zip(mine, local))
    if world_size == 1:
        gathered = [payload]
    else:
        gathered = [None] * world_size if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(specs)
    for part in gathered:
        for i, res in part:
            out[i] = res
    return out


def gpu_runner(precision="mixed", device=None):
    """A runner that steps its systems in one Batch on this rank's GPU and
    returns final positions, tangents and [P, S, director] per system."""
    def run(specs, steps, couplings=()):
        from .batch import Batch
        b = Batch(specs, precision=precision, device=device)
        for members, fixed, cross in couplings:
            b.couple(members, fixed, cross)
        b.begin(steps)
        b.run(steps)
        b.engine.synchronize()
        res = []
        for st in b.states:
            op = b.engine.order_params(st.slot) if b.dim == 2 else np.full(3, np.nan)
            res.append({"pos": st.pos.cpu().numpy(), "tangent": st.tangent.double().cpu().numpy(),
                        "order": op, "status": b.engine.status(st.slot)})
        b.close()
        return res
    return run
