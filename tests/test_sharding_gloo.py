"""Sharding independent systems over ranks, tested with two gloo ranks on the
CPU.  The CPU oracle plays the per-rank device runner, so the test needs no
GPU; the sharded result must equal the single-rank result bit for bit (each
system is independent and its run deterministic)."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from gliding_collective_rotation_b200 import sharding


def test_partition_is_balanced_and_complete():
    rng = np.random.default_rng(3)
    costs = list(rng.lognormal(8, 1.5, size=257))
    for w in (1, 2, 3, 8):
        parts = sharding.partition(costs, w)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        # LPT is within 5% of the mean load unless one system alone exceeds it
        bound = max(1.05, max(costs) / (sum(costs) / w))
        assert sharding.imbalance(costs, parts) <= bound + 1e-9
        assert parts == sharding.partition(costs, w)  # deterministic


def _specs():
    from gliding_collective_rotation_b200 import workloads as W
    specs = W.config3(n_systems=256, param_seed=99)
    return sorted(specs, key=lambda s: s.n)[:5]


def _oracle_runner(specs, steps):
    from oracle import oracle as O
    out = []
    for sp in specs:
        p = sp.params
        ng = max(1, int(p.L / (2.0 * max(2 * sp.rest_lengths.max(), p.wca_params[3]))))
        sysm = O.OracleSystem(sp.pos, sp.tangent, sp.chain_id, sp.rest_lengths, p.L, p.spring_params,
                              p.wca_params, p.active_params, p.D, p.Dr, p.radius, p.n_nearby, ng, nbor_depth=64)
        sysm.build_lists(grid_window=1)
        sysm.run(steps, dt=sp.dt * 1e-3, noise_mode=O.NOISE_PHILOX, seed=int(p.seed))
        out.append(sysm.pos.copy())
    return out


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = sharding.run_sharded(_specs(), 5, _oracle_runner)
        if rank == 0:
            q.put([r.tolist() for r in res])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_rank():
    single = sharding.run_sharded(_specs(), 5, _oracle_runner, rank=0, world_size=1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert len(got) == len(single)
    for a, b in zip(got, single):
        assert np.array_equal(np.array(a), b)
