"""Sharding independent systems over ranks, tested with two gloo ranks on the
CPU.  The CPU oracle plays the per-rank device runner, so the test needs no
GPU; the sharded result must equal the single-rank result bit for bit (each
system is independent and its run deterministic)."""
import math
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


# -- populations of one box stay together --------------------------------

def _pop_specs():
    """Two boxes of two populations (from the reference fixture) and one
    independent system."""
    from gliding_collective_rotation_b200.engine import SystemParams
    from gliding_collective_rotation_b200.workloads import SystemSpec
    from tests.multipop_helpers import load, pop_arrays
    d, s = load("pops2_2d")
    specs = []
    for box in range(2):
        for k in range(2):
            a = pop_arrays(d, s, k)
            prm = SystemParams(L=s["L"], spring_params=a["spring"], wca_params=a["wca"], active_params=a["active"],
                               D=0.01, Dr=0.0, radius=a["radius"], n_nearby=a["n_nearby"],
                               calc_springs=a["longest"] > 1, seed=10 * box + k)
            specs.append(SystemSpec(f"box{box}_p{k}", 2, a["pos"], a["tangent"], a["chain_id"], a["rest_lengths"],
                                    prm, 1e-3, math.inf))
    specs.append(_specs()[0])
    couplings = [([0, 1], [False, False], d["cross_wca"]), ([2, 3], [False, False], d["cross_wca"])]
    return specs, couplings


def _oracle_group_runner(specs, steps, couplings=()):
    """Singles through OracleSystem, coupled groups through OracleGroup."""
    from oracle import oracle as O
    out = [None] * len(specs)
    grouped = set()
    for members, fixed, cross in couplings:
        systems = []
        for m in members:
            sp = specs[m]
            p = sp.params
            o = O.OracleSystem(sp.pos, sp.tangent, sp.chain_id, sp.rest_lengths, p.L, p.spring_params,
                               p.wca_params, p.active_params, p.D, p.Dr, p.radius, p.n_nearby, 4,
                               calc_springs=p.calc_springs)
            o.seed = int(p.seed)
            systems.append(o)
        O.OracleGroup(systems, fixed, cross).run(steps, dt=1e-4, noise_mode=O.NOISE_PHILOX)
        for m, o in zip(members, systems):
            out[m] = o.pos.copy()
            grouped.add(m)
    rest = [i for i in range(len(specs)) if i not in grouped]
    for i, r in zip(rest, _oracle_runner([specs[i] for i in rest], steps)):
        out[i] = r
    return out


def test_coupled_groups_stay_on_one_rank():
    specs, couplings = _pop_specs()
    costs = [sp.n for sp in specs]
    for w in (1, 2, 3, 5):
        parts = sharding.partition_units(costs, couplings, w)
        assert sorted(i for p in parts for i in p) == list(range(len(specs)))
        for members, _, _ in couplings:
            assert sum(1 for p in parts if set(members) <= set(p)) == 1


def _group_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        specs, couplings = _pop_specs()
        res = sharding.run_sharded(specs, 3, _oracle_group_runner, couplings=couplings)
        if rank == 0:
            q.put([r.tolist() for r in res])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_with_coupled_populations():
    specs, couplings = _pop_specs()
    single = sharding.run_sharded(specs, 3, _oracle_group_runner, rank=0, world_size=1, couplings=couplings)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_group_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert len(got) == len(single)
    for a, b in zip(got, single):
        assert np.array_equal(np.array(a), b)
