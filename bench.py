#!/usr/bin/env python3
"""Benchmark of the gliding-collective-rotation SRK2 step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gcr|reference]
                    [--workload sweep|large|config1|config5|pops|motors] [--precision mixed|fp64]

Default workload: the batched sweep -- 256 independent 2D systems (chains of
5-40 beads, 50-4000 chains per system, area fraction 0.1-0.4, chirality and
bending drawn per system, FP32 forces / FP64 positions, Philox seeds 0..255),
advanced together by one captured graph of persistent kernels.  One step is
one SRK2 step of every system.  Metric: bead-steps/s (beads x SRK2 steps per
second, one bead-step = two force evaluations).

Printed as one JSON line by rank 0.  Under torchrun every rank runs its own
256 systems (weak scaling, no collective in the data path); the timed region
is bracketed by barriers and its length is the max over ranks.

``--impl reference`` times the reference's algorithm on the host cores: the
CPU restatement of the reference's Numba step (oracle/), all host threads,
chain-aligned chunks, Verlet lists rebuilt every 40 steps, on a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        d["source"] = "measured"
        return d
    return dict(PEAKS_FALLBACK)


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------

def make_workload(name, rank=0, scale=1.0, systems=256):
    from gliding_collective_rotation_b200 import workloads as W
    if name == "sweep":
        specs = W.config3(n_systems=256, param_seed=12345 + rank)[:systems]
        desc = (f"batched sweep: {len(specs)} independent 2D systems, 50-4000 chains of 5-40 beads, area fraction "
                "0.1-0.4, chirality -0.5..0.5, bending 1..50, WCA r_c=1, T=0.01, dt=1e-3, SRK2")
    elif name == "large":
        specs = [W.config2(seed=rank, scale=scale)]
        desc = "large single system: 2D L=1000, 20,000 chains x 25 beads, LJ r_c=2.5 sigma eps 0.5, chiral 0.2, SRK2"
    elif name == "config1":
        specs = [W.config1(seed=rank)]
        desc = "small single system: 2D L=60, 200 chains x 10 beads, WCA, SRK2"
    elif name == "config5":
        specs = [W.config5(seed=rank, scale=scale)]
        desc = "3D precision stress: L=200, 40,000 chains x 25 beads, LJ eps 1, Dr 0.1, SRK2"
    elif name == "pops":
        specs, groups = W.populations(n_boxes=max(1, systems // 2), seed=rank)
        specs = _Specs(specs)
        specs.groups = groups
        desc = (f"two populations per box: {len(groups)} 2D boxes L=150, 1000 chains x 10 beads (WCA, v0=1) and "
                "3000 passive beads of diameter 0.7, one dt per box, cross WCA = mean parameters, SRK2")
    elif name == "motors":
        specs, groups, motors = W.motors(n_boxes=max(1, systems // 2), seed=rank, n_chains=1000, L=150.0)
        specs = _Specs(specs)
        specs.groups, specs.motors = groups, motors
        desc = (f"chains pushed by motors: {len(groups)} 2D boxes L=150, 1000 chains x 10 beads (v0 handed to the "
                "motors), 11,250 motors (density 0.5, D 0.1, k_on 0.9, k_off 0.2, reach a/2), SRK2")
    else:
        raise SystemExit(f"unknown workload {name}")
    return specs, desc


class _Specs(list):
    """Workload specs; ``groups``: populations coupled in one box; ``motors``:
    motor populations (motor index, chain index, params, hold)."""
    groups = ()
    motors = ()


def workload_config(args, specs, desc, world):
    """The ``config`` of the JSON line: what the workload is, the same in the
    GPU arm and the reference arm (measured quantities go elsewhere)."""
    n_beads = sum(s.n for s in specs)
    dim = specs[0].dim
    F = 8 if args.precision == "fp64" else 4
    # bytes per bead a step touches: pos, pos1, build positions (FP64), the
    # tangent, force, pair force and noise (FT), list count, topology, images
    touched = 3 * dim * 8 + 4 * dim * F + 4 + 1 + 4 * dim
    return {"workload": desc, "systems_per_gpu": len(specs), "beads_per_gpu": n_beads,
            "coupled_groups": len(getattr(specs, "groups", ())),
            "parallelism": f"{world} GPU(s), independent systems per GPU (no collective in the data path)",
            "l2": f"inputs larger than L2: a step touches ~{touched * n_beads / 1e6:.0f} MB per GPU > 126 MB",
            "dt_rule": "adaptive (SRK.py:323-353): dtmax = configured dt, max_dist_per_step of "
                       "config.grid_list_setup"}


def stratified(specs, m):
    """Indices of `m` systems at the bead-count quantiles (k + 1/2) / m of
    the workload: the CPU arms time a sample spread over the size range."""
    order = sorted(range(len(specs)), key=lambda i: (specs[i].n, i))
    if m >= len(order):
        return order
    return sorted({order[min(len(order) - 1, int((k + 0.5) * len(order) / m))] for k in range(m)})


# --------------------------------------------------------------------------
# algorithmic bytes (HBM roofline)
# --------------------------------------------------------------------------

def step_bytes(dim, precision):
    """Minimum HBM bytes per bead of one SRK2 step with one cell rebuild, by
    phase, as the hot path's measurement contract defines them (P = 8 B per
    FP64 position component, F = 4 B (mixed) or 8 B (FP64) per force
    component):
      predictor  read pos, write pos1, write F0, 4 B of metadata = 2dP + dF + 4
      corrector  read pos and pos1, read F0, write pos and the tangent, 4 B
                 of metadata                                     = 3dP + 2dF + 4
      cell build read pos, 8 B of cell key and sorted index, the sorted copy
                                                                 = 2dP + 8
    in all 7dP + 3dF + 16: 152 B in 2D mixed, 176 B 2D FP64, 220 B 3D mixed."""
    P = 8
    F = 8 if precision == "fp64" else 4
    out = {"predictor": 2 * dim * P + dim * F + 4, "corrector": 3 * dim * P + 2 * dim * F + 4,
           "cell_build": 2 * dim * P + 8}
    out["step"] = sum(out.values())
    return out


# the phase of the step each timed kernel group belongs to
KERNEL_PHASE = {"lists_pos": "cell_build", "pair_pos": "predictor", "stage0": "predictor", "lists_pos1": "cell_build",
                "pair_pos1": "corrector", "stage1": "corrector", "update": "corrector"}


def algorithmic_bytes(dim, precision, n_beads, n_cells, get_orient, rot_diff, list_mean, builds_per_stage):
    """This design's own byte model of one launch of each kernel group (the
    ``model_frac`` of the line): every input the kernel reads counted once
    and every output once.  A list build (bin + sort + build) reads the
    positions, writes and reads one cell slot per bead, writes the list and
    the build positions; it runs for a fraction `builds_per_stage` of the
    beads per stage (measured), and that fraction of its bytes is charged to
    each list launch."""
    P = 8                                   # FP64 position component
    F = 8 if precision == "fp64" else 4     # force / tangent / noise component
    tan = dim * F if get_orient else 0
    build = n_beads * (dim * P + 4 + 4 + 4 * list_mean + 4 + dim * P) + n_cells * 8
    lists = builds_per_stage * build
    pair = n_beads * (dim * P + 4 + 4 * list_mean + dim * F)
    stage0 = n_beads * (dim * P + 1 + dim * F + dim * F + dim * P + tan + dim * F + dim * P + 8)
    stage1 = n_beads * (dim * P + 1 + dim * F + dim * F + dim * F + tan)
    update = n_beads * (dim * P + dim * F + dim * F + dim * P + dim * P + 8 + (2 * dim * F if rot_diff else 0))
    return {"lists_pos": lists, "pair_pos": pair, "stage0": stage0, "lists_pos1": lists, "pair_pos1": pair,
            "stage1": stage1, "update": update}


KERNELS = ["lists_pos", "pair_pos", "stage0", "lists_pos1", "pair_pos1", "stage1", "update"]


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------

class ClockSampler:
    """SM clock, its maximum and the active clock-event reasons of one GPU,
    read through NVML (the library nvidia-smi queries) on a host thread every
    `period` seconds between ``start`` and ``stop``: the timed region of a
    20-step run lasts ~15 ms, far below nvidia-smi's sampling interval, so
    the sampler runs in-process.  The main thread waits on the GPU (CUDA
    events) while it samples."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device_index=0, period=0.002):
        self.device_index = device_index
        self.period = period
        self.samples = []
        self.error = None
        self._stop = None
        self._thread = None
        self._nvml = None
        self._h = None

    def _handle(self, nv):
        import torch
        props = torch.cuda.get_device_properties(self.device_index)
        uuid = getattr(props, "uuid", None)
        if uuid is not None:
            try:
                return nv.nvmlDeviceGetHandleByUUID(("GPU-" + str(uuid)).encode())
            except Exception:
                pass
        bus = getattr(props, "pci_bus_id", None)
        if bus is not None:
            pci = f"{getattr(props, 'pci_domain_id', 0):08x}:{bus:02x}:{getattr(props, 'pci_device_id', 0):02x}.0"
            try:
                return nv.nvmlDeviceGetHandleByPciBusId_v2(pci.encode())
            except Exception:
                pass
        return nv.nvmlDeviceGetHandleByIndex(self.device_index)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            self._nvml = nv
            self._h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self._h, nv.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: the line says so
            self.error = f"NVML unavailable: {e}"
            return
        self._stop = threading.Event()

        def loop():
            nv, h = self._nvml, self._h
            while not self._stop.is_set():
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                except Exception as e:
                    self.error = str(e)
                    return
                self._stop.wait(self.period)

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()

    def stop(self):
        if self._thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.error or "not started"]}
        self._stop.set()
        self._thread.join(timeout=5)
        try:
            self._nvml.nvmlShutdown()
        except Exception:
            pass
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"]}
        nv = self._nvml
        active = 0
        for _, r in self.samples:
            active |= r
        reasons = sorted(name for name, const in self.REASONS if active & getattr(nv, const, 0))
        sm = [s for s, _ in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, every 2 ms in the timed region"}


# --------------------------------------------------------------------------
# CPU arm: the reference's algorithm (oracle) on a bounded sample
# --------------------------------------------------------------------------

def cpu_sample_rate(specs, states_host, steps, threads, budget_s=20.0):
    """bead-steps/s of the oracle (the reference's Numba step restated in C,
    OpenMP threads over chain-aligned chunks) on the systems `specs` (a
    sample of the workload) from the states `states_host`, in rounds of
    `steps` steps per system after an untimed list build until `budget_s`
    seconds of stepping, under the reference's adaptive dt rule as the GPU
    arm (dtmax = the system's dt, max_dist_per_step of grid_list_setup; each
    system's dt carried)."""
    from oracle import oracle as O
    systems = []
    for spec, (pos, tan) in zip(specs, states_host):
        p = spec.params
        ng = max(1, int(p.L / (2.0 * max(2 * spec.rest_lengths.max(), p.wca_params[3]))))
        sysm = O.OracleSystem(pos, tan, spec.chain_id, spec.rest_lengths, p.L, p.spring_params, p.wca_params,
                              p.active_params, p.D, p.Dr, p.radius, p.n_nearby, ng, nbor_depth=32)
        sysm.build_lists(grid_window=1)
        sysm.seed_mt(int(p.seed), threads)
        systems.append([spec, sysm, spec.dt])
    # rounds of `steps` steps over the sample until the time budget is used
    total_bs, total_t, used = 0, 0.0, []
    rounds = 0
    while total_t < budget_s and rounds < 1000:
        for entry in systems:
            spec, sysm, dt = entry
            t0 = time.perf_counter()
            res = sysm.run(steps, dt=dt, dtmax=spec.dt, max_dist_per_step=spec.relax_mdps, n_threads=threads)
            total_t += time.perf_counter() - t0
            total_bs += spec.n * res["steps"]
            entry[2] = res["dt"]
            if res["flag"] < 0:
                sysm.build_lists(grid_window=1)
        rounds += 1
    used = [f"{spec.name}({spec.n} beads)" for spec, _, _ in systems]
    used.append(f"{rounds} rounds of {steps} steps")
    return total_bs / total_t, used, total_t


def relax_on_cpu(spec, max_steps=600):
    """Untimed adaptive-dt warm-up with the oracle (the reference's own
    adaptive step), used by the reference arm."""
    from oracle import oracle as O
    p = spec.params
    ng = max(1, int(p.L / (2.0 * max(2 * spec.rest_lengths.max(), p.wca_params[3]))))
    sysm = O.OracleSystem(spec.pos, spec.tangent, spec.chain_id, spec.rest_lengths, p.L, p.spring_params,
                          p.wca_params, p.active_params, p.D, p.Dr, p.radius, p.n_nearby, ng, nbor_depth=32)
    sysm.build_lists(grid_window=1)
    sysm.seed_mt(7, os.cpu_count() or 1)
    done = 0
    dt = spec.dt * 1e-4
    while done < max_steps:
        res = sysm.run(100, dt=dt, dtmax=spec.dt, max_dist_per_step=spec.relax_mdps, n_threads=os.cpu_count() or 1)
        done += res["steps"]
        dt = res["dt"]
        if res["flag"] < 0:
            sysm.build_lists(grid_window=1)
        if dt >= spec.dt * (1 - 1e-12):
            break
    return sysm.pos.copy(), sysm.tangent_list.copy()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    specs, desc = make_workload(args.workload, systems=args.systems)
    if getattr(specs, "groups", ()):
        # the CPU restatement couples populations over all pairs, not over the
        # reference's lists: its time would not be the reference's
        print(json.dumps({"impl": "reference", "unavailable": "coupled populations: no list-based CPU "
                          "restatement of the multi-population step to time"}), flush=True)
        return
    threads = os.cpu_count() or 1
    # a bounded sample spread over the size range, relaxed untimed with the
    # reference's adaptive dt
    sample = [specs[i] for i in stratified(specs, args.cpu_systems)]
    states = [relax_on_cpu(s) for s in sample]
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_sample_rate(sample[:1], states[:1], 2, threads)
    rates = []
    for _ in range(args.steps):
        r, used, secs = cpu_sample_rate(sample, states, args.cpu_steps, threads,
                                        budget_s=args.cpu_budget / max(args.steps, 1))
        rates.append(r)
    value = float(np.median(rates))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    line = {
        "impl": "reference", "metric": "bead-steps/s", "value": value, "unit": "bead-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, specs, desc, world),
        "cpu_baseline": {"value": value, "unit": "bead-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{len(sample)} systems at the bead-count quantiles of the workload, relaxed on "
                                   f"the CPU, {args.cpu_steps}-step rounds per timed step: {', '.join(used)}"},
        "e2e": {"value": value, "unit": "bead-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------

def run_gpu(args):
    import torch
    import torch.distributed as dist
    from gliding_collective_rotation_b200.batch import Batch, PlainRunner
    from gliding_collective_rotation_b200.engine import default_skin
    from gliding_collective_rotation_b200._lib import (FLAG_CELL_OVERFLOW, FLAG_LIST_CORRUPT, FLAG_LIST_OVERFLOW,
                                                       FLAG_NONFINITE)
    FLAG_FATAL = FLAG_CELL_OVERFLOW | FLAG_NONFINITE | FLAG_LIST_CORRUPT | FLAG_LIST_OVERFLOW
    regrows = 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    specs, desc = make_workload(args.workload, rank=rank, scale=args.scale, systems=args.systems)
    for sp in specs:
        sp.params.cell_factor = args.cell_factor
        sp.params.skin = args.skin if args.skin >= 0 else None
    batch = Batch(specs, precision=args.precision, device=dev, steps_per_graph=args.steps_per_graph,
                  ctas_per_sm=args.ctas_per_sm, block_beads=args.block_beads, list_depth=args.list_depth or None,
                  pair_mode=args.pair_mode)
    groups = list(getattr(specs, "groups", ()))
    for members, fixed, cross in groups:
        batch.couple(members, fixed, cross)
    for m in getattr(specs, "motors", ()):
        batch.set_motors(*m)
    eng = batch.engine
    n_beads = batch.n_beads
    # untimed warm-up; every step after it, timed or not, follows the
    # reference's default adaptive dt rule (dtmax = the configured dt)
    relax_steps = batch.relax(max_steps=args.relax_steps, adaptive_after=True)
    tuned = None
    if args.autotune:
        # launch shapes measured on copies of the relaxed systems (untimed);
        # the batch is rebuilt from the same relaxed state with the best one
        import dataclasses
        from gliding_collective_rotation_b200 import autotune
        relaxed = [dataclasses.replace(sp, pos=st.pos.cpu().numpy(), tangent=st.tangent.double().cpu().numpy())
                   for sp, st in zip(specs, batch.states)]
        tuned = autotune.tune(relaxed, precision=args.precision, device=dev, couplings=groups,
                              refresh=args.autotune > 1)
        batch.close()
        tspecs, kw = autotune.apply(relaxed, tuned)
        for sp, tsp in zip(specs, tspecs):
            sp.pos, sp.tangent, sp.params = tsp.pos, tsp.tangent, tsp.params
        batch = Batch(specs, precision=args.precision, device=dev, list_depth=args.list_depth or None, **kw)
        for members, fixed, cross in groups:
            batch.couple(members, fixed, cross)
        for m in getattr(specs, "motors", ()):
            batch.set_motors(*m)
        batch.set_adaptive(True)
        args.steps_per_graph, args.ctas_per_sm, args.block_beads = (kw["steps_per_graph"], kw["ctas_per_sm"],
                                                                    kw["block_beads"])
        args.pair_mode = kw["pair_mode"]
    # warm-up under the adaptive dt (regrows the cells if a system overflowed them)
    batch.run_checked(args.warmup)
    eng = batch.engine
    eng.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    def any_rank(flag):
        if world > 1:
            t = torch.tensor([int(flag)], device=dev, dtype=torch.int64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            flag = bool(t.item())
        return bool(flag)

    # ---- device-timed batched steps -------------------------------------
    # a system whose cells or lists overflow inside the timed steps stops
    # there: the depths are doubled and the steps timed again, so that the
    # number reported is of args.steps steps of every system
    for attempt in range(4):
        builds0 = [s["list_builds"] for s in batch.statuses()]
        batch.begin(args.steps)
        clocks = ClockSampler(local)
        barrier()
        torch.cuda.synchronize()
        clocks.start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed")
        ev0.record(eng.stream)
        batch.run(args.steps)
        ev1.record(eng.stream)
        torch.cuda.nvtx.range_pop()
        ev1.synchronize()
        clk = clocks.stop()
        torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1)
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        st = batch.statuses()
        if not any_rank(batch.overflowed(st)) or attempt == 3:
            break
        batch.regrow()
        eng = batch.engine
        regrows += 1
    steps_done = min(s["steps_done"] for s in st)
    flags = sorted({s["flags"] for s in st})
    if steps_done < args.steps or any(f & FLAG_FATAL for f in flags):
        raise SystemExit(f"timed run incomplete: {steps_done} of {args.steps} steps, flags {flags}")
    value = world * n_beads * args.steps / (ms / 1e3)
    # the dt the adaptive rule took: bead-weighted mean over the timed steps
    dt_mean = sum(s["dt_used"] * x.n for s, x in zip(st, batch.states)) / (args.steps * n_beads)
    # neighbour lists: mean length, and bead-builds per stage in the timed region
    list_entries = sum(eng.neighbour_list(x.slot, partners=False)[3] for x in batch.states)
    list_mean = list_entries / n_beads
    bead_builds = sum((s["list_builds"] - b0) * x.n for s, b0, x in zip(st, builds0, batch.states))
    builds_per_stage = bead_builds / (2.0 * args.steps * n_beads)

    # ---- the same steps over several contexts ---------------------------
    # workloads of several independent systems or boxes: the line's value is the
    # device time of all the contexts' steps (the one-context figure above is
    # kept beside it, and is what the per-kernel profile below explains)
    split = args.contexts >= 2 and len(context_parts([sp.n for sp in specs], args.contexts, groups)) >= 2
    tc = None
    one_context = {"value": value, "ms_per_step": ms / args.steps}
    if split:
        tc = SplitContexts(args, specs, batch, dev, k=args.contexts, groups=groups,
                           motors=getattr(specs, "motors", ()))
        clocks = ClockSampler(local)
        clocks.start()
        ms2, st2 = tc.timed(args.steps, barrier, any_rank)
        clk2 = clocks.stop()
        if world > 1:
            t = torch.tensor([ms2], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms2 = float(t.item())
        done2 = min(s["steps_done"] for s in st2)
        flags2 = sorted({s["flags"] for s in st2})
        if done2 < args.steps or any(f & FLAG_FATAL for f in flags2):
            raise SystemExit(f"split-context timed run incomplete: {done2} of {args.steps} steps, flags {flags2}")
        regrows += tc.regrows
        ms, clk = ms2, clk2
        value = world * n_beads * args.steps / (ms / 1e3)

    # ---- per-kernel profile (roofline) ----------------------------------
    # the same steps launched kernel group by kernel group with CUDA events
    # between the groups on the context stream (steady state: the lists
    # carry over from the timed run)
    batch.begin(args.profile_steps)
    kms = eng.profile_steps(args.profile_steps) / args.profile_steps
    cfg = eng.cfg
    from gliding_collective_rotation_b200.engine import footprint
    n_cells = sum(footprint(cfg, s.params, s.n, len(s.rest_lengths))[0] for s in specs)
    get_orient = bool(specs[0].params.spring_params[4])
    rot_diff = (not get_orient) and specs[0].params.Dr > 0
    model = algorithmic_bytes(batch.dim, args.precision, n_beads, n_cells, get_orient, rot_diff, list_mean,
                              builds_per_stage)
    sb = step_bytes(batch.dim, args.precision)
    dom = int(np.argmax(kms))
    kname = KERNELS[dom]
    pk = peaks()
    # the dominant kernel against the contract's bytes of its phase of the
    # step (beads x bytes per bead of that phase, per launch)
    alg_bytes = sb[KERNEL_PHASE[kname]] * n_beads
    achieved = alg_bytes / (kms[dom] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as fh:
            tr = json.load(fh).get(args.workload, {}).get(args.precision, {})
        if kname in tr:
            v = tr[kname]
            traffic = (v["bytes_per_bead"] if isinstance(v, dict) else float(v)) * n_beads
    step_achieved = sb["step"] * value / world / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                "algorithmic_bytes": alg_bytes,
                "algorithmic_bytes_source": f"{sb[KERNEL_PHASE[kname]]} B per bead: the {KERNEL_PHASE[kname]} "
                                            f"phase of the hot-path contract's {sb['step']} B per bead-step",
                "peak_source": f"{pk['source']} (MEASURED_PEAKS.json hbm_gbs)" if pk["source"] == "measured"
                else pk["source"],
                "kernel_ms": {k: float(v) for k, v in zip(KERNELS, kms)},
                "step_bytes_per_bead": sb["step"], "step_achieved": step_achieved,
                "step_frac": step_achieved / pk["hbm_gbs"],
                "model_bytes_per_bead": {k: float(v) / n_beads for k, v in model.items()},
                "model_frac": (model[kname] / (kms[dom] / 1e3) / 1e9) / pk["hbm_gbs"],
                "model_step_frac": (sum(model.values()) / (kms.sum() / 1e3) / 1e9) / pk["hbm_gbs"]}

    # ---- plain path: one system per launch sequence ---------------------
    plain = None
    if args.plain and len(specs) > 1 and not groups:
        pr = PlainRunner(specs, precision=args.precision, device=dev, steps_per_graph=args.steps_per_graph)
        pr.copy_state_from(batch)
        pr.begin(args.plain_steps)
        pr.run(min(args.plain_steps, 10))
        pr.synchronize()
        pr.begin(args.plain_steps)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(pr.stream)
        pr.run(args.plain_steps)
        e1.record(pr.stream)
        e1.synchronize()
        pms = e0.elapsed_time(e1)
        plain = {"value": pr.n_beads * args.plain_steps / (pms / 1e3), "unit": "bead-steps/s",
                 "steps": args.plain_steps, "ms_per_step": pms / args.plain_steps}
        pr.close()

    # ---- end to end through the public API with host buffers ------------
    # (timed again after a regrow, as above)
    spc = args.e2e_steps_per_call
    n_calls = max(1, args.steps // spc)
    for attempt in range(0 if split else 4):
        big = batch.big
        h_pos = torch.empty(big["pos"].shape, dtype=big["pos"].dtype, pin_memory=True)
        h_tan = torch.empty(big["tangent"].shape, dtype=big["tangent"].dtype, pin_memory=True)
        h_pos.copy_(big["pos"])
        h_tan.copy_(big["tangent"])
        torch.cuda.synchronize()
        e2e_bytes_in = h_pos.numel() * h_pos.element_size() + h_tan.numel() * h_tan.element_size()
        short = False
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n_calls):
            big["pos"].copy_(h_pos, non_blocking=True)
            big["tangent"].copy_(h_tan, non_blocking=True)
            batch.begin(spc)
            batch.run(spc)
            batch.engine.synchronize()
            h_pos.copy_(big["pos"], non_blocking=True)
            h_tan.copy_(big["tangent"], non_blocking=True)
            torch.cuda.synchronize()
            short = short or min(s["steps_done"] for s in batch.statuses()) < spc
        e2e_s = time.perf_counter() - t0
        if not any_rank(short) or attempt == 3:
            break
        batch.regrow()
        regrows += 1
    if split:
        e2e_s, e2e_bytes_in, short = tc.e2e(spc, n_calls, barrier)
        short = any_rank(short)
        tc.close()
    if short:
        raise SystemExit("end-to-end run incomplete after regrows")
    eng = batch.engine
    if world > 1:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * n_beads * spc * n_calls / e2e_s, "unit": "bead-steps/s",
           "h2d_bytes_per_step": e2e_bytes_in / spc, "d2h_bytes_per_step": e2e_bytes_in / spc,
           "steps_per_call": spc, "calls": n_calls,
           "api": "Batch.begin/run (gcr_call_begin_batch, gcr_run) with pinned host buffers"
           + (f"; {len(tc.parts)} Batch contexts, a share of the systems each, on their own streams: one "
              "context's copies run while the others step" if split else ""),
           "contexts": len(tc.parts) if split else 1}

    # ---- the same workload in FP64, and the mixed path's error against it
    fp64 = None
    if args.fp64_block and args.precision == "mixed" and not groups:
        fp64 = fp64_block(args, specs, batch, dev)

    # ---- CPU baseline (rank 0, N = 1) ------------------------------------
    cpu = None
    # (coupled populations: the CPU sampler steps single populations, so
    # no CPU line for them)
    if world == 1 and args.cpu_baseline and not groups:
        host_states = [(s.pos.cpu().numpy(), s.tangent.double().cpu().numpy()) for s in batch.states]
        threads = os.cpu_count() or 1
        idx = stratified(specs, args.cpu_systems)
        r, used, secs = cpu_sample_rate([specs[i] for i in idx], [host_states[i] for i in idx], args.cpu_steps,
                                        threads, budget_s=args.cpu_budget)
        idx1 = stratified(specs, 2)
        r1, used1, secs1 = cpu_sample_rate([specs[i] for i in idx1], [host_states[i] for i in idx1], args.cpu_steps,
                                           1, budget_s=max(2.0, args.cpu_budget / 3))
        cpu = {"value": r, "unit": "bead-steps/s", "cores": threads, "kind": "port",
               "sample": f"{len(idx)} systems at the bead-count quantiles of the workload from the GPU's relaxed "
                         f"states, {args.cpu_steps}-step rounds: {', '.join(used)} ({secs:.1f} s); adaptive dt as "
                         "the GPU arm",
               "single_thread_value": r1,
               "single_thread_sample": f"{args.cpu_steps}-step rounds of {', '.join(used1)} ({secs1:.1f} s)"}

    spg = args.steps_per_graph
    line = {
        "metric": "bead-steps/s", "value": value, "unit": "bead-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": workload_config(args, specs, desc, world),
        "run": {"precision": ("FP32 forces and SRK arithmetic, FP64 positions" if args.precision == "mixed"
                              else "FP64"),
                "relax_steps": relax_steps, "steps_done": steps_done, "flags": flags, "dt_mean": dt_mean,
                "regrows_in_timing": regrows, "cell_factor": args.cell_factor,
                "skin": specs[0].params.skin if specs[0].params.skin is not None
                else default_skin(specs[0].params.wca_params[3]),
                "steps_per_graph": spg, "cell_depth": batch.cell_depth,
                "list_depth": batch.list_depth, "list_mean": list_mean,
                "list_builds_per_stage": builds_per_stage, "block_beads": args.block_beads,
                "ctas_per_sm": args.ctas_per_sm, "pair_mode": args.pair_mode,
                "contexts": len(tc.parts) if split else 1,
                "split_ctas_per_sm": (args.ctas_per_sm or args.split_ctas_per_sm) if split else None,
                "autotune": None if tuned is None else {k: v for k, v in tuned.items() if k != "trials"}},
        "one_context": dict(one_context, note="the same steps in one context, device-timed; the per-kernel "
                            "profile of `roofline` is of this context") if split else None,
        "e2e": e2e, "roofline": roofline, "clocks": clk,
        # the run-start check, then 15 kernels per step (two list builds of
        # four, two pair, two stage, dt rule, update, bookkeeping; 13 when
        # the stages sum the pair forces; two motor-decision kernels more
        # with motor populations) in graphs of steps_per_graph steps
        # (per context: each context launches the whole sequence)
        "gpu_launches": (len(tc.parts) if split else 1) * (1 + ((13 if args.pair_mode == 1 and not groups else 15)
                                                  + (2 if getattr(specs, "motors", ()) else 0))
                                             * spg * math.ceil(args.steps / spg)),
    }
    if fp64 is not None:
        line["fp64"] = fp64
    if plain is not None:
        line["plain"] = plain
        line["batched_over_plain"] = value / world / plain["value"]
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    if world > 1:
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# precision: the mixed path against the FP64 path of the same kernels
# --------------------------------------------------------------------------

def split_by_beads(sizes, k):
    """Cut a list of system sizes into min(k, len) contiguous, non-empty runs
    of about equal beads: the boundaries [0, c1, ..., len].  Run q ends at
    the first system whose running bead count reaches q/k of the total."""
    n = len(sizes)
    k = max(1, min(int(k), n))
    cum = np.cumsum(sizes)
    cuts = [0]
    for q in range(1, k):
        c = int(np.searchsorted(cum, cum[-1] * q / k)) + 1
        cuts.append(min(max(c, cuts[-1] + 1), n - (k - q)))
    cuts.append(n)
    return cuts


def context_parts(sizes, k, groups=()):
    """The systems of each context, as index lists: contiguous runs of about
    equal beads (``split_by_beads``), or, with coupled populations, whole
    boxes (a coupled group stays together) balanced by beads."""
    if not groups:
        cuts = split_by_beads(sizes, k)
        return [list(range(a, b)) for a, b in zip(cuts[:-1], cuts[1:])]
    from gliding_collective_rotation_b200 import sharding
    return [p for p in sharding.partition_units(list(sizes), groups, k) if p]


class SplitContexts:
    """The workload's systems split, by beads, over `k` Batch contexts, each
    on its own stream, started from the batch's current positions and
    tangents and warmed up untimed (their lists are built at the first
    call).  Queued in turn, one context's kernels fill the others' tails and
    idle SMs (the list kernels of a few flagged systems, the ends of the
    persistent grids), and one context's host copies run while the others
    step."""

    def __init__(self, args, specs, batch, dev, k=2, groups=(), motors=()):
        import torch
        from gliding_collective_rotation_b200.batch import Batch
        self.args = args
        index_parts = context_parts([sp.n for sp in specs], max(2, k), groups)
        self.parts = []
        for idx in index_parts:
            part, states = [specs[i] for i in idx], [batch.states[i] for i in idx]
            # persistent grids of at most split_ctas_per_sm CTAs per SM: the
            # contexts' grids then share the SMs instead of each filling them
            cps = args.ctas_per_sm if args.ctas_per_sm else args.split_ctas_per_sm
            hb = Batch(part, precision=args.precision, device=dev, steps_per_graph=args.steps_per_graph,
                       ctas_per_sm=cps, block_beads=args.block_beads, list_depth=batch.list_depth,
                       cell_depth=batch.cell_depth, pair_mode=args.pair_mode)
            # the populations of a box, and its motors, stay in one context
            at = {g: j for j, g in enumerate(idx)}
            for members, fixed, cross in groups:
                if members[0] in at:
                    hb.couple([at[m] for m in members], fixed, cross)
            for m, c, prm, hold in motors:
                if m in at:
                    hb.set_motors(at[m], at[c], prm, hold)
            for dst, src in zip(hb.states, states):
                dst.pos.copy_(src.pos)
                dst.tangent.copy_(src.tangent)
            torch.cuda.synchronize()
            hb.set_adaptive(True)
            hb.run_checked(max(args.warmup, 1))
            self.parts.append(hb)
        self.regrows = 0

    def statuses(self):
        return [st for hb in self.parts for st in hb.statuses()]

    def timed(self, steps, barrier, any_rank):
        """Device milliseconds of `steps` steps of every context (CUDA events
        around all the streams) and their statuses; after an overflow inside
        the steps the overflowed context is regrown and the steps timed
        again (at most three times)."""
        import torch
        for attempt in range(4):
            for hb in self.parts:
                hb.begin(steps)
            torch.cuda.synchronize()
            streams = [hb.engine.stream for hb in self.parts]
            s0 = streams[0]
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            barrier()
            torch.cuda.nvtx.range_push("timed_contexts")
            ev0.record(s0)
            for st in streams[1:]:
                st.wait_event(ev0)
            for hb in self.parts:
                hb.run(steps)
            for st in streams[1:]:
                evb = torch.cuda.Event()
                evb.record(st)
                s0.wait_event(evb)
            ev1.record(s0)
            torch.cuda.nvtx.range_pop()
            ev1.synchronize()
            torch.cuda.synchronize()
            barrier()
            ms = ev0.elapsed_time(ev1)
            over = [hb.overflowed() for hb in self.parts]
            if not any_rank(any(over)) or attempt == 3:
                return ms, self.statuses()
            for hb, o in zip(self.parts, over):
                if o:
                    hb.regrow()
            self.regrows += 1

    def e2e(self, spc, n_calls, barrier):
        """Seconds of `n_calls` calls of `spc` steps with every call's state
        copied in from pinned host buffers and back; bytes copied in per
        call; whether a call fell short."""
        import torch
        hosts = []
        for hb in self.parts:
            hp = torch.empty(hb.big["pos"].shape, dtype=hb.big["pos"].dtype, pin_memory=True)
            ht = torch.empty(hb.big["tangent"].shape, dtype=hb.big["tangent"].dtype, pin_memory=True)
            hp.copy_(hb.big["pos"])
            ht.copy_(hb.big["tangent"])
            hosts.append((hp, ht))
        nbytes = sum(hp.numel() * hp.element_size() + ht.numel() * ht.element_size() for hp, ht in hosts)
        torch.cuda.synchronize()
        short = False
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for call in range(n_calls):
            for hb, (hp, ht) in zip(self.parts, hosts):
                with torch.cuda.stream(hb.engine.stream):
                    hb.big["pos"].copy_(hp, non_blocking=True)
                    hb.big["tangent"].copy_(ht, non_blocking=True)
                    # the wait that arming does anyway; then the previous
                    # call's statuses are final
                    hb.engine.stream.synchronize()
                    if call > 0:
                        short = short or min(st["steps_done"] for st in hb.statuses()) < spc
                    hb.begin(spc)
                    hb.run(spc)
                    hp.copy_(hb.big["pos"], non_blocking=True)
                    ht.copy_(hb.big["tangent"], non_blocking=True)
        for hb in self.parts:
            hb.engine.stream.synchronize()
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        short = short or min(st["steps_done"] for st in self.statuses()) < spc
        return secs, nbytes, short

    def close(self):
        for hb in self.parts:
            hb.close()


def specs_at(specs, positions, tangents, steps):
    """Copies of `specs` that start from the given device state and step
    counters (the Philox key), with parameter objects of their own."""
    import copy
    import dataclasses
    out = []
    for sp, p, t, k in zip(specs, positions, tangents, steps):
        prm = copy.copy(sp.params)
        prm.step = int(k)
        out.append(dataclasses.replace(sp, pos=p.cpu().numpy().copy(), tangent=t.double().cpu().numpy().copy(),
                                       params=prm))
    return out


def compare_precisions(specs, dt0, marks, depths):
    """The mixed path and the FP64 path of the same kernels from one state
    (`specs`, as ``specs_at`` makes them), same Philox seeds and the same
    adaptive dt rule, with an FP64 control whose positions start one ulp
    away (its divergence is the growth of any perturbation in these chaotic
    systems): per checkpoint in `marks`, the largest position difference
    over L of any system against FP64, that of the control, and after the
    first step the relative L2 error of the forces (F0 + F1)."""
    import torch
    from gliding_collective_rotation_b200.batch import Batch

    runs = {prec: Batch(specs, precision=prec, **depths) for prec in ("fp64", "mixed")}
    for b in runs.values():
        b.set_adaptive(True)
    ctl = Batch(specs, precision="fp64", **depths)
    ctl.set_adaptive(True)
    rng = np.random.default_rng(1)
    for st, sp in zip(ctl.states, specs):
        ulp = np.spacing(sp.params.L)
        st.pos.add_(torch.from_numpy(rng.choice([-ulp, ulp], size=tuple(st.pos.shape))).to(st.pos.device))
        st.pos.remainder_(sp.params.L)
    runs["fp64_ulp"] = ctl
    L = np.array([sp.params.L for sp in specs])
    rows = []
    done = 0
    for b in runs.values():
        b._carry_dt = list(dt0)  # the first call starts from the common state's dt
    for m in sorted(set(marks) | {1}):
        for b in runs.values():
            b.run_checked(m - done)  # regrows cells or lists if the run needs them
            b.engine.synchronize()
        done = m
        err, err_ctl = 0.0, 0.0
        num = den = 0.0
        for i, (s64, s32, sc) in enumerate(zip(runs["fp64"].states, runs["mixed"].states, runs["fp64_ulp"].states)):
            d = (s32.pos - s64.pos).cpu().numpy()
            d -= L[i] * np.round(d / L[i])
            err = max(err, float(np.abs(d).max()) / L[i])
            d = (sc.pos - s64.pos).cpu().numpy()
            d -= L[i] * np.round(d / L[i])
            err_ctl = max(err_ctl, float(np.abs(d).max()) / L[i])
            if m == 1:
                f64 = s64.forces.cpu().numpy()
                f32 = s32.forces.double().cpu().numpy()
                num += float(((f32 - f64) ** 2).sum())
                den += float((f64 ** 2).sum())
        row = {"steps": m, "max_pos_err_over_L": err, "fp64_ulp_control_over_L": err_ctl}
        if m == 1:
            row["force_rel_l2_err"] = (num / den) ** 0.5 if den > 0 else 0.0
        row["flags"] = sorted({s["flags"] for b in runs.values() for s in b.statuses()})
        rows.append(row)
    for b in runs.values():
        b.close()
    return rows


def fp64_block(args, specs, batch, dev):
    """The workload's FP64 throughput and the mixed path's error against
    FP64, both from the mixed run's state after its timed steps: an FP64
    batch of the same systems is warmed up and timed over `--steps` steps as
    the line's own value is, then ``compare_precisions`` runs to
    `--fp64-steps` steps."""
    import torch
    from gliding_collective_rotation_b200.batch import Batch

    sts = batch.statuses()
    start = ([s.pos for s in batch.states], [s.tangent for s in batch.states], [s["step"] for s in sts])
    state = specs_at(specs, *start)
    dt0 = [s["dt"] for s in sts]
    depths = dict(cell_depth=min(128, 2 * batch.cell_depth), list_depth=min(1024, 2 * batch.list_depth))
    b = Batch(specs_at(specs, *start), precision="fp64", device=dev, steps_per_graph=args.steps_per_graph,
              ctas_per_sm=args.ctas_per_sm, block_beads=args.block_beads, pair_mode=args.pair_mode, **depths)
    b.set_adaptive(True)
    b._carry_dt = list(dt0)
    b.run_checked(args.warmup)
    b.begin(args.steps)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(b.engine.stream)
    b.run(args.steps)
    e1.record(b.engine.stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    flags = sorted({s["flags"] for s in b.statuses()})
    b.close()
    marks = [m for m in (10, 100, 1000, 5000) if m <= args.fp64_steps]
    rows = compare_precisions(state, dt0, marks, depths)
    by = {r["steps"]: r for r in rows}
    return {"value": b.n_beads * args.steps / (ms / 1e3), "unit": "bead-steps/s", "ms_per_step": ms / args.steps,
            "steps": args.steps, "flags": flags,
            "force_rel_l2_err_1step": by[1]["force_rel_l2_err"],
            "max_pos_err_over_L": {str(m): by[m]["max_pos_err_over_L"] for m in marks},
            "fp64_ulp_control_over_L": {str(m): by[m]["fp64_ulp_control_over_L"] for m in marks},
            "error_run_flags": sorted({f for r in rows for f in r["flags"]}),
            "from": "the mixed run's state after its timed steps; same Philox seeds, same adaptive dt rule; the "
                    "control is FP64 with every position moved by one ulp"}


def run_precision_report(args):
    """Both precisions from one relaxed FP64 state, same Philox seeds and
    the same dt rule: the relative force error after one step and the
    position divergence over `--precision-report` steps."""
    import torch
    from gliding_collective_rotation_b200.batch import Batch

    torch.cuda.set_device(0)
    specs, desc = make_workload(args.workload, scale=args.scale, systems=args.systems)
    dim = specs[0].dim
    base = Batch(specs, precision="fp64")
    relax_steps = base.relax(max_steps=args.relax_steps, adaptive_after=True)
    sts = base.statuses()
    dt0 = [s["dt"] for s in sts]
    state = specs_at(specs, [s.pos for s in base.states], [s.tangent for s in base.states], [s["step"] for s in sts])
    # cells and lists as deep as the relaxed run needed, with a margin
    depths = dict(cell_depth=min(128, 2 * base.cell_depth), list_depth=min(1024, 2 * base.list_depth))
    base.close()
    marks = [m for m in (10, 100, 1000, 5000, args.precision_report) if m <= args.precision_report]
    rows = compare_precisions(state, dt0, marks, depths)
    line = {"metric": "mixed vs FP64 error", "workload": desc, "dim": dim, "relax_steps": relax_steps,
            "dt_rule": "adaptive (SRK.py:323-353), dtmax = configured dt", "checkpoints": rows}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# serving: a Poisson trace through the continuous-batching server
# --------------------------------------------------------------------------


def run_serve(args):
    import torch
    from gliding_collective_rotation_b200 import serve as S
    from gliding_collective_rotation_b200 import workloads as W

    torch.cuda.set_device(0)
    tr = W.serve_trace(args.requests, rate=args.rate, seed=7, max_beads=args.max_beads, min_steps=args.min_steps,
                       max_steps=args.max_steps)
    reqs = [S.request_from_trace(e, obs_every=args.obs_every) for e in tr]
    srv = S.Server(2, args.precision, hbm_budget=int(args.hbm_budget_gb * (1 << 30)), chunk=args.chunk)
    clocks = ClockSampler(0, period=0.05)
    clocks.start()
    res = srv.serve(reqs, timeout=args.serve_timeout)
    clk = clocks.stop()
    st = dict(srv.stats)
    rejected = list(srv.rejected)
    srv.close()
    s = S.summarize(res)
    dev = max(st["device_s"], 1e-12)
    # where the makespan went: the rounds' graphs on the device, the host
    # work of the rounds around them, and waiting with nothing resident
    gap = {"makespan_s": s["makespan_s"], "device_busy_s": st["device_s"],
           "round_host_s": st["round_wall_s"] - st["device_s"], "idle_s": st["idle_s"],
           "other_host_s": s["makespan_s"] - st["round_wall_s"] - st["idle_s"],
           "rounds": st["rounds"], "regrows": st["regrows"],
           "device_bead_steps_per_s": st["bead_steps_done"] / dev,
           "mean_resident_beads": st["resident_bead_s"] / dev,
           "armed_step_fraction": st["bead_steps_done"] / max(st["bead_steps_armed_max"], 1)}
    line = {
        "metric": "bead-steps/s", "value": s["bead_steps_per_s"], "unit": "bead-steps/s", "n_gpus": 1,
        "steps": None, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": f"served trace: {args.requests} requests, Poisson {args.rate}/s, beads log-uniform "
                               f"[1e3, {args.max_beads:.0e}], steps uniform [{args.min_steps}, {args.max_steps}], "
                               f"adaptive dt (dtmax 1e-3), P/S/angle every {args.obs_every} steps",
                   "chunk": args.chunk, "hbm_budget_gb": args.hbm_budget_gb},
        "serve": {**s, "rejected": len(rejected)}, "gap": gap, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="gcr", choices=["gcr", "reference"])
    ap.add_argument("--workload", default="sweep",
                    choices=["sweep", "large", "config1", "config5", "serve", "pops", "motors"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--systems", type=int, default=256, help="systems of the sweep workload")
    ap.add_argument("--cell-factor", type=float, default=1.0, help="GPU cell side / pair cutoff")
    ap.add_argument("--steps-per-graph", type=int, default=10)
    ap.add_argument("--ctas-per-sm", type=int, default=0,
                    help="CTAs per SM of the tile kernels (0: from occupancy, <0: one CTA per tile)")
    ap.add_argument("--block-beads", type=int, default=128)
    ap.add_argument("--pair-mode", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="pair forces: 0 list kernel, 1 list walk inside the stage kernels (no pair launch), "
                         "2 cell-staged kernel; -1: the measured best of the workload (1 for the 2D LJ "
                         "system, 0 otherwise)")
    ap.add_argument("--skin", type=float, default=-1.0,
                    help="Verlet skin of the neighbour lists (<0: 0.2 r_cut + 0.1, within [0.2, 1])")
    ap.add_argument("--list-depth", type=int, default=0, help="neighbour slots per bead (0: default)")
    ap.add_argument("--relax-steps", type=int, default=2000)
    ap.add_argument("--autotune", type=int, default=0,
                    help="1: launch shapes from the autotuner (cached per workload and device); 2: re-tune")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--plain", type=int, default=1)
    ap.add_argument("--plain-steps", type=int, default=50)
    ap.add_argument("--e2e-steps-per-call", type=int, default=100)
    ap.add_argument("--split-ctas-per-sm", type=int, default=6,
                    help="persistent CTAs per SM of each context when the systems are split over several "
                         "(0: as many as fit); --ctas-per-sm, when given, sets both")
    ap.add_argument("--contexts", type=int, default=4, choices=range(1, 9),
                    help="k > 1: the timed and end-to-end steps of a workload of several independent systems run "
                         "over k contexts on their own streams (a share of the systems each, by beads); 1: one")
    ap.add_argument("--cpu-baseline", type=int, default=1)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--cpu-systems", type=int, default=8, help="systems of the CPU sample (size quantiles)")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--fp64-block", type=int, default=1,
                    help="1: add the FP64 throughput and the mixed path's error against FP64 to the line")
    ap.add_argument("--fp64-steps", type=int, default=1000, help="steps of the mixed-vs-FP64 comparison")
    ap.add_argument("--precision-report", type=int, default=0,
                    help="report mixed vs FP64 error over this many steps instead of timing")
    # serving (--workload serve): the defaults are the serving configuration
    ap.add_argument("--requests", type=int, default=200, help="serve: requests in the trace")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: Poisson arrival rate per second")
    ap.add_argument("--max-beads", type=float, default=1e6, help="serve: largest request (log-uniform from 1e3)")
    ap.add_argument("--min-steps", type=int, default=1000)
    ap.add_argument("--max-steps", type=int, default=20000)
    ap.add_argument("--obs-every", type=int, default=100)
    ap.add_argument("--chunk", type=int, default=200)
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-timeout", type=float, default=900.0)
    args = ap.parse_args()
    if args.pair_mode < 0:
        # measured on a B200: the stage kernels' own list walk is 11% faster on
        # the 2D LJ system; the separate pair kernel elsewhere
        args.pair_mode = 1 if args.workload == "large" else 0
    if args.workload == "serve" and args.impl == "gcr":
        run_serve(args)
        return
    if args.precision_report > 0 and args.impl == "gcr":
        run_precision_report(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
