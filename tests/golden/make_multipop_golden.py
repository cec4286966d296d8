#!/usr/bin/env python3
"""Generate the golden fixtures of several populations in one box by running
the reference itself.

Run from the repository root in a container where the reference source is
mounted (read-only) at /root/reference and Numba is installed:

    python tests/golden/make_multipop_golden.py [--ref /root/reference] [--out tests/golden]

The reference is prepared as ``make_golden.py`` prepares it (a scratch copy,
matplotlib stubbed, the numpy aliases restored).  For every case the script

1. builds the populations the reference's way: ``defaults.set_defaults`` and
   overrides, ``config.configure``, one ``Equal_Size_Chain_Collection`` per
   population (the later ones resized with ``set_size`` and
   ``adjust_WCA_params``, given their own ``v0``, some of them ``fixed``),
   ``control.configure_start`` (placement, cells, every population pair's
   nbor_list);
2. relaxes the placement with the reference's own multi-population
   ``updates.SRK2_force_calc`` (adaptive dt) and records that state, every
   population's packed parameters, and the cross-population WCA parameters
   the reference derives (``updates.interpop_forces``);
3. records the single-kernel cross force (``forces.central_pair_force`` over
   a population's nbor_list of another population) on the relaxed state;
4. runs one ``updates.SRK2_force_calc`` step of the list of populations from
   that recorded state (positions, tangents, fresh lists, status restored
   each time) ``TRIALS`` times, recording every population's arrays and the
   ``status`` fields of each trial.

T = 0 in every case: with several populations the reference runs one thread
per population pair, and Numba draws each thread's noise from that thread's
own unseeded generator.  Even without noise the reference's multi-population
step is not reproducible: its threads meet at a spin barrier on a plain
counter array (``SRK.thread_wait``, SRK.py:487-495, no atomics or fences), and
repeated steps from one state give different positions for a few beads.
Hence several trials: a restatement is pinned by matching one of them.

The fixtures are ``<case>.npz``; their entries are merged into ``index.json``.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_golden import _install_shims, _status_fields  # noqa: E402

# LJ attraction (r_c = 2.5 sigma, eps 0.5) so that pairs of the relaxed state
# sit inside the cutoffs and the cross forces act from the first step
TRIALS = 6

COMMON = dict(a=0.5, k=100., kappa=20., repel_d_max=1., WCA_epsilon=0.5, LJ_cutoff_factor=2.5 / 2 ** (1 / 6),
              T=0., t_init_grow=0., a_init_factor=1.0)

CASES = {
    # chains of 8 beads with chiral propulsion and single smaller beads with
    # their own propulsion, 2D
    "pops2_2d": dict(
        sim=dict(Lx=24., n_chains=24, chain_length=8, v0=1., v_tan_angle=0.1, dim=2, seed=5, dtmax=1e-3,
                 **COMMON),
        others=[dict(name="beads", n=60, length=1, size=0.7, v0=0.5)],
        relax_steps=200),
    # three populations, the last fixed (obstacles): chains, beads, posts
    "pops3_fixed_2d": dict(
        sim=dict(Lx=24., n_chains=20, chain_length=8, v0=1., v_tan_angle=0., dim=2, seed=7, dtmax=1e-3,
                 **COMMON),
        others=[dict(name="beads", n=40, length=1, size=0.7, v0=0.5),
                dict(name="posts", n=12, length=1, size=1.6, v0=0., fixed=True)],
        relax_steps=200),
    # 3D: chains and short chains of a larger bead
    "pops2_3d": dict(
        sim=dict(Lx=12., n_chains=24, chain_length=6, v0=1., v_tan_angle=0., dim=3, seed=9, dtmax=5e-4,
                 **COMMON),
        others=[dict(name="dimers", n=20, length=2, size=1.3, v0=0.5)],
        relax_steps=200),
}


def _pop_record(pop):
    return dict(pos=pop.pos.copy(), tangent=pop.tangent_list.copy(), chain_id=pop.chain_id.astype(np.int64),
                rest_lengths=pop.rest_lengths.copy(), spring_params=pop.spring_params(),
                wca_params=pop.WCA_params.copy(), active_params=pop.active_params())


def run_case(name, spec, mods):
    populations, config, updates, forces, defaults, control = mods
    sim, _ = defaults.set_defaults()
    sim.update(dict(plot_every=-1, ticker_every=-1, save_state_every=-1., t_max=0., n_threads=1,
                    b_cached=True, filelabel="golden"))
    sim.update(spec["sim"])
    config.configure(sim)
    pops = [populations.Equal_Size_Chain_Collection(sim, name="chains")]
    for o in spec["others"]:
        p = populations.Equal_Size_Chain_Collection(sim, num_chains=o["n"], chain_length=o["length"],
                                                    name=o["name"])
        p.set_size(o["size"])
        p.adjust_WCA_params()
        p.v0 = o["v0"]
        if o.get("fixed"):
            p.fixed = True
        pops.append(p)
    status = config.status_class(sim)
    control.configure_start(sim, pops, status)
    t0 = time.time()
    status.next_output_step = status.stepnum + spec["relax_steps"]
    updates.SRK2_force_calc(pops, status, sim)
    relax_s = time.time() - t0

    out = {}
    n = len(pops)
    for k, pop in enumerate(pops):
        for key, val in _pop_record(pop).items():
            out[f"p{k}_{key}0" if key in ("pos", "tangent") else f"p{k}_{key}"] = val
    # the reference's own cross-population parameters: the WCA row of
    # interpop_forces(pop_k, pop_q) (updates.py:274-312)
    cross = np.zeros((n, n, 4))
    for k, pk in enumerate(pops):
        for q, pq in enumerate(pops):
            if k == q:
                continue
            names, params = updates.interpop_forces(pk, pq)
            for nm, row in zip(names, params):
                if nm == "WCA":
                    cross[k, q] = row[:4]
    out["cross_wca"] = cross
    scal = dict(L=config.Lx, dim=config.dim, n_pops=n, names=[p.name for p in pops],
                fixed=[bool(p.fixed) for p in pops], D=[float(p.D) for p in pops], Dr=[float(p.Dr) for p in pops],
                radius=[float(p.repel_d_max) for p in pops],
                n_nearby=[int(p.n_nearby_beads_dont_repel) for p in pops],
                longest=[int(p.longest_chain_length) for p in pops],
                rigid_rod=[float(p.rigid_rod_projection_factor) for p in pops],
                n_grid=int(sim["n_grid"]), grid_window=int(sim["grid_window"]), grid_factor=config.grid_factor,
                n_steps_update=int(config.n_steps_update_grid_list), rk_cheat=config.RK_cheat_factor,
                max_dist_per_step=config.max_dist_per_step, dtmax=status.dtmax, relax_steps=spec["relax_steps"],
                relax_seconds=relax_s, n_threads=int(config.n_threads), sim_overrides=spec["sim"],
                others=spec["others"])

    # single-kernel golden: the force on population k from population q over
    # k's nbor_list of q, built fresh at the relaxed state
    for pop in pops:
        pop.update_grid_list(overwrite=True)
    for pk in pops:
        for pq in pops:
            pk.update_nbor_list_with_pop2(pq, grid_window=sim["grid_window"])
    for k, pk in enumerate(pops):
        for q, pq in enumerate(pops):
            if k == q or pk.fixed:
                continue
            f = np.zeros_like(pk.pos)
            tl = pk.tangent_list.copy()
            forces.central_pair_force(np.array([0, 0, 0, 1, 0]), pk.pos, pk.nbor_list[q], f, tl, pk.where_active,
                                      config.Lx, pq.pos, cross[k, q], pq.tangent_list, config.Lx / 2)
            out[f"k_cross_{k}_{q}"] = f

    # one step from the recorded state, TRIALS times
    st0 = _status_fields(status)
    out["status_before"] = st0
    st_after = []
    for t in range(TRIALS):
        for k, pop in enumerate(pops):
            pop.pos[:] = out[f"p{k}_pos0"]
            pop.tangent_list[:] = out[f"p{k}_tangent0"]
        for pop in pops:
            pop.update_grid_list(overwrite=True)
        for pk in pops:
            for pq in pops:
                pk.update_nbor_list_with_pop2(pq, grid_window=sim["grid_window"])
        status.dt, status.dt_used, status.stepnum, status.t = st0[0], st0[1], int(st0[2]), st0[3]
        status.update_grid_list_counter = int(st0[4])
        status.next_output_step = status.stepnum + 1
        updates.SRK2_force_calc(pops, status, sim)
        st_after.append(_status_fields(status))
        for k, pop in enumerate(pops):
            out[f"trial{t}_p{k}_pos"] = pop.pos.copy()
            out[f"trial{t}_p{k}_tangent"] = pop.tangent_list.copy()
            out[f"trial{t}_p{k}_forces"] = pop.forces.copy()
    out["status_after"] = np.array(st_after)
    out["trials"] = np.array(TRIALS)
    out["scalars"] = np.array(json.dumps(scal, default=lambda o: o.item()))
    return out, scal


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--one", action="store_true", help="run the listed cases in this process (internal)")
    args = ap.parse_args()
    if not args.one:
        # Numba freezes module globals such as config.dim at first compile:
        # one fresh process per case
        index = {}
        for name in args.cases:
            subprocess.run([sys.executable, os.path.abspath(__file__), "--one", "--ref", args.ref,
                            "--out", args.out, "--cases", name], check=True)
            with open(os.path.join(args.out, f"{name}.json")) as fh:
                index[name] = json.load(fh)
            os.remove(os.path.join(args.out, f"{name}.json"))
        path = os.path.join(args.out, "index.json")
        if os.path.exists(path):
            with open(path) as fh:
                index = {**json.load(fh), **index}
        with open(path, "w") as fh:
            json.dump(index, fh, indent=1, sort_keys=True)
        return

    scratch = tempfile.mkdtemp(prefix="gcr_ref_")
    ref = os.path.join(scratch, "ref")
    shutil.copytree(args.ref, ref)
    for root, dirs, files in os.walk(ref):
        for d in dirs:
            os.chmod(os.path.join(root, d), 0o755)
        for fn in files:
            os.chmod(os.path.join(root, fn), 0o644)
    os.makedirs(os.path.join(ref, "Results"), exist_ok=True)
    cwd = os.getcwd()
    os.chdir(ref)
    sys.path.insert(0, ref)
    _install_shims()
    import populations  # noqa: F401  (must come first: circular imports)
    import config
    import updates
    import forces
    import defaults
    import control
    mods = (populations, config, updates, forces, defaults, control)
    index = {}
    for name in args.cases:
        os.chdir(ref)
        t0 = time.time()
        out, scal = run_case(name, CASES[name], mods)
        os.chdir(cwd)
        path = os.path.join(args.out, f"{name}.npz")
        np.savez_compressed(path, **out)
        index[name] = {"file": f"{name}.npz", "bytes": os.path.getsize(path),
                       "beads": int(sum(out[f"p{k}_pos0"].shape[0] for k in range(scal["n_pops"]))),
                       "seconds": round(time.time() - t0, 1), "L": scal["L"], "dim": scal["dim"],
                       "n_grid": scal["n_grid"], "n_pops": scal["n_pops"]}
        print(name, index[name], flush=True)
    for name, entry in index.items():
        with open(os.path.join(args.out, f"{name}.json"), "w") as fh:
            json.dump(entry, fh)
    shutil.rmtree(scratch, ignore_errors=True)


if __name__ == "__main__":
    main()
