#!/usr/bin/env python3
"""Generate the golden fixtures in this folder by running the reference itself.

Run from the repository root in a container where the reference source is
mounted (read-only) at /root/reference and Numba is installed:

    python tests/golden/make_golden.py [--ref /root/reference] [--out tests/golden]

The reference is copied to a scratch directory (its ``config.configure``
deletes ``__pycache__/*`` in the working directory and ``cline`` writes
``Results/``), matplotlib is stubbed (it is only needed for plotting), the
``np.float``/``np.int`` aliases removed in numpy 2 are restored, and
``populations`` is imported first (the import order of ``BDsim.py``).

For every case the script
1. builds the population the reference's way (``defaults.set_defaults`` +
   overrides, ``config.configure``, ``Equal_Size_Chain_Collection``,
   ``control.configure_start``), runs the reference's own init-grow protocol
   (``control.sim_loop`` until t >= 0, then ``early_time_procedures`` once more
   so that ``end_init_grow`` restores the physical parameters);
2. records that relaxed state and the packed parameters;
3. seeds Numba's RNG (``np.random.seed`` inside an ``@njit`` function) and calls
   ``updates.SRK2_force_calc`` repeatedly with ``n_threads = 1``, recording the
   ``status`` fields before and after each call and the arrays after it;
4. records single-kernel outputs (springs, pair forces, propulsion, cell and
   neighbour lists) on the relaxed state.

The fixtures are ``<case>.npz``; ``index.json`` lists them with their sizes.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import time
import types

import numpy as np


def _install_shims():
    np.float = float  # noqa: NPY001 -- removed alias the reference still uses
    np.int = int

    class _Stub(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)
            return lambda *a, **k: None

    for m in ["matplotlib", "matplotlib.pyplot", "matplotlib.colors", "matplotlib.cm",
              "matplotlib.collections", "matplotlib.patches", "mpl_toolkits",
              "mpl_toolkits.mplot3d", "mpl_toolkits.mplot3d.art3d", "mpl_toolkits.axes_grid1",
              "mpl_toolkits.axes_grid1.inset_locator"]:
        sys.modules[m] = _Stub(m)


CASES = {
    # benchmark config 1 exactly: 2D, Lx=60, 200 x 10 beads, a=0.5, k=100,
    # kappa=20, WCA (cutoff 1), v0=1 tangent-locked, T=0.01, dt=1e-3 fixed.
    "config1": dict(
        sim=dict(Lx=60., n_chains=200, chain_length=10, a=0.5, k=100., kappa=20.,
                 repel_d_max=1., WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0.,
                 T=0.01, dim=2, seed=0),
        dt=1e-3, fixed_dt=True, calls=[1, 9, 90, 900], noise_seed=0, save_every=None),
    # config-2 physics (LJ attraction r_c = 2.5 sigma, eps 0.5, chiral 0.2) on a
    # small box.  With a fixed dt of 1e-3 the reference's own trajectory blows
    # up on this state (max force ~1e10 within 50 steps), so the reference's
    # adaptive dt with dtmax = 1e-3 is used.
    "chiral_lj": dict(
        sim=dict(Lx=55., n_chains=60, chain_length=25, a=0.5, k=100., kappa=20.,
                 repel_d_max=1., WCA_epsilon=0.5, LJ_cutoff_factor=2.5 / 2 ** (1 / 6), v0=1.,
                 v_tan_angle=0.2, T=0.01, dim=2, seed=3, dtmax=1e-3),
        dt=None, fixed_dt=False, calls=[1, 49, 250], noise_seed=11, save_every=None),
    # 2D rotationally diffusing propulsion (not tangent-locked), Dr = 0.1.
    "rotdiff2d": dict(
        sim=dict(Lx=30., n_chains=40, chain_length=8, a=0.5, k=100., kappa=10.,
                 repel_d_max=1., WCA_epsilon=1., LJ_cutoff_factor=2.5 / 2 ** (1 / 6), v0=1.,
                 v_tan_angle=0., T=0.05, Dr=0.1, b_use_tangent_as_propulsion_direction=False,
                 dim=2, seed=5),
        dt=5e-4, fixed_dt=True, calls=[1, 99, 100], noise_seed=21, save_every=None),
    # config-5 physics in 3D on a small box: LJ eps 1, kappa 10, Dr 0.1,
    # T 0.05, dt 5e-4.
    "rotdiff3d": dict(
        sim=dict(Lx=16., n_chains=60, chain_length=10, a=0.5, k=100., kappa=10.,
                 repel_d_max=1., WCA_epsilon=1., LJ_cutoff_factor=2.5 / 2 ** (1 / 6), v0=1.,
                 v_tan_angle=0., T=0.05, Dr=0.1, b_use_tangent_as_propulsion_direction=False,
                 dim=3, seed=7, t_init_grow=0., a_init_factor=1.0),
        dt=5e-4, fixed_dt=True, calls=[1, 49, 150], noise_seed=31, save_every=None,
        init_grow=False, relax_steps=300),
    # adaptive dt (max_dist_per_step from grid_list_setup) with a save-time
    # limit on each call, so dt_used is clipped and calls end early.
    "adaptive": dict(
        sim=dict(Lx=30., n_chains=50, chain_length=10, a=0.5, k=100., kappa=20.,
                 repel_d_max=1., WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0.1,
                 T=0.01, dim=2, seed=9, dtmax=4e-3),
        dt=None, fixed_dt=False, calls=[50, 50, 50, 50, 50], noise_seed=41, save_every=0.05),
    # rigid rods (kappa < 0: projection factor 1, populations.py:325-329)
    # with translational noise, 2D, through the reference's own init-grow
    "rigid2d": dict(
        sim=dict(Lx=30., n_chains=40, chain_length=8, a=0.5, k=100., kappa=-1., repel_d_max=1.,
                 WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0., T=0.05, dim=2, seed=17,
                 dtmax=1e-3),
        dt=None, fixed_dt=False, calls=[1, 19, 80], noise_seed=61, save_every=None),
    # rigid rods in 3D, chains laid straight and relaxed by the reference's
    # own adaptive steps (with the projection on)
    "rigid3d": dict(
        sim=dict(Lx=16., n_chains=40, chain_length=6, a=0.5, k=100., kappa=-1., repel_d_max=1.,
                 WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0., T=0.05, dim=3, seed=19,
                 dtmax=5e-4, t_init_grow=0., a_init_factor=1.0),
        dt=None, fixed_dt=False, calls=[1, 19, 80], noise_seed=71, save_every=None,
        init_grow=False, relax_steps=200),
    # 3D growth: config-5 physics (LJ eps 1, kappa 10, Dr 0.1, T 0.05) on a
    # small box, grown by the reference's own init-grow (3D rigid-rod phase)
    "grow3d": dict(
        sim=dict(Lx=16., n_chains=60, chain_length=10, a=0.5, k=100., kappa=10., repel_d_max=1.,
                 WCA_epsilon=1., LJ_cutoff_factor=2.5 / 2 ** (1 / 6), v0=1., v_tan_angle=0., T=0.05, Dr=0.1,
                 b_use_tangent_as_propulsion_direction=False, dim=3, seed=37, dtmax=5e-4, dt0=5e-4),
        dt=None, fixed_dt=False, calls=[1, 19, 80], noise_seed=111, save_every=None),
    # SRK4 (SRK.py:186-215, 296-321): 2D with chirality, grown by the
    # reference's init-grow under SRK4
    "srk4_2d": dict(
        sim=dict(Lx=30., n_chains=40, chain_length=8, a=0.5, k=100., kappa=20., repel_d_max=1.,
                 WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0.1, T=0.05, dim=2, seed=23,
                 dtmax=1e-3, SRK_order=4),
        dt=None, fixed_dt=False, calls=[1, 19, 80], noise_seed=81, save_every=None),
    # SRK4 in 3D with LJ attraction and rotational diffusion
    "srk4_3d": dict(
        sim=dict(Lx=16., n_chains=40, chain_length=6, a=0.5, k=100., kappa=10., repel_d_max=1.,
                 WCA_epsilon=1., LJ_cutoff_factor=2.5 / 2 ** (1 / 6), v0=1., v_tan_angle=0., T=0.05, Dr=0.1,
                 b_use_tangent_as_propulsion_direction=False, dim=3, seed=29, dtmax=5e-4, SRK_order=4,
                 t_init_grow=0., a_init_factor=1.0),
        dt=None, fixed_dt=False, calls=[1, 19, 80], noise_seed=91, save_every=None,
        init_grow=False, relax_steps=200),
    # SRK4 with rigid rods (the projection at every stage)
    "srk4_rigid": dict(
        sim=dict(Lx=30., n_chains=40, chain_length=8, a=0.5, k=100., kappa=-1., repel_d_max=1.,
                 WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0., T=0.05, dim=2, seed=31,
                 dtmax=1e-3, SRK_order=4),
        dt=None, fixed_dt=False, calls=[1, 19, 80], noise_seed=101, save_every=None),
    # the paper's chiral run settings (Chiral_parameters_script.sh:3-17) on a
    # small box: chain length 30, kappa 100, v_tan_angle 0.1, WCA_epsilon 1e-8,
    # WCA_shift 0.1, bead_density 0.3, adaptive dt.
    "paper_chiral": dict(
        sim=dict(Lx=30., chain_length=30, kappa=100., v_tan_angle=0.1, bead_density=0.3,
                 WCA_epsilon=1e-8, WCA_shift=0.1, dim=2, seed=13),
        dt=None, fixed_dt=False, calls=[20, 20], noise_seed=51, save_every=None),
}


def _status_fields(status):
    return np.array([status.dt, status.dt_used, status.stepnum, status.t,
                     status.update_grid_list_counter, status.max_forces_strength,
                     status.next_output_step, status.next_save_time, status.dtmax], dtype=np.float64)


STATUS_FIELDS = ["dt", "dt_used", "stepnum", "t", "update_grid_list_counter", "max_forces_strength",
                 "next_output_step", "next_save_time", "dtmax"]


def _nbor_pairs(nbor_list):
    rows = []
    for b1 in range(nbor_list.shape[0]):
        n = nbor_list[b1, 0]
        for k in range(n):
            rows.append((b1, nbor_list[b1, 1 + k]))
    return np.array(rows, dtype=np.int32).reshape(-1, 2)


def _grid_pairs(grid_list):
    rows = []
    ng, _, nz, _ = grid_list.shape
    for gx in range(ng):
        for gy in range(ng):
            for gz in range(nz):
                c = grid_list[gx, gy, gz]
                for k in range(c[0]):
                    rows.append(((gx * ng + gy) * nz + gz, c[1 + k]))
    return np.array(rows, dtype=np.int32).reshape(-1, 2)


def run_case(name, spec, mods):
    populations, config, updates, forces, defaults, control = mods
    from numba import njit

    @njit
    def _seed(s):
        np.random.seed(s)

    sim, _ = defaults.set_defaults()
    sim.update(dict(plot_every=-1, ticker_every=-1, save_state_every=-1., t_max=0., n_threads=1,
                    b_cached=True, filelabel="golden"))
    sim.update(spec["sim"])
    if spec["dt"] is not None:
        sim["dtmax"] = spec["dt"]
        sim["dt0"] = spec["dt"]
    config.configure(sim)
    config.n_threads = 1
    pops = [populations.Equal_Size_Chain_Collection(sim)]
    status = config.status_class(sim)
    control.configure_start(sim, pops, status)
    pop = pops[0]
    # the reference's placement and derived settings, before any step
    init = dict(init_pos=pop.pos.copy(), init_tangent=pop.tangent_list.copy(),
                init_wca_params=pop.WCA_params.copy(), init_spring_params=pop.spring_params(),
                init_active_params=pop.active_params())
    init_scal = dict(n_chains=int(sim["n_chains"]), n_beads=int(sim["n_beads"]), n_grid_setup=int(sim["n_grid"]),
                     grid_spacing=float(sim["grid_spacing"]),
                     n_steps_update_grid_list=int(sim["n_steps_update_grid_list"]),
                     max_dist_per_step_setup=float(sim["max_dist_per_step"]), grid_window_setup=int(sim["grid_window"]),
                     D_init=float(pop.D), Dr_init=float(pop.Dr), b_init_growing=bool(sim["b_init_growing"]),
                     sim_overrides=spec["sim"], dt_override=spec["dt"])
    t0 = time.time()
    if spec.get("init_grow", True):
        control.sim_loop(pops, sim, status)        # init-grow until t > 0
        control.early_time_procedures(pops, status, sim)  # ends init-grow
    else:
        # Chains laid straight (a_init_factor = 1) and relaxed by the
        # reference's own adaptive-dt steps, without init-grow.  (The
        # reference's 3D projection divides by zero only for a one-bead
        # chain; these cases have none.)
        status.next_output_step = status.stepnum + spec["relax_steps"]
        updates.SRK2_force_calc(pops, status, sim)
    grow_s = time.time() - t0

    # relaxed state and the parameters the hot path sees
    out = dict(init)
    out["pos0"] = pop.pos.copy()
    out["tangent0"] = pop.tangent_list.copy()
    out["chain_id"] = pop.chain_id.astype(np.int64)
    out["rest_lengths"] = pop.rest_lengths.copy()
    out["spring_params"] = pop.spring_params()
    out["wca_params"] = pop.WCA_params.copy()
    out["active_params"] = pop.active_params()
    scal = dict(L=config.Lx, dim=config.dim, D=pop.D, Dr=pop.Dr, radius=pop.repel_d_max,
                n_nearby=pop.n_nearby_beads_dont_repel, n_grid=sim["n_grid"],
                grid_factor=config.grid_factor, n_steps_update=config.n_steps_update_grid_list,
                rk_cheat=config.RK_cheat_factor, grid_window=sim["grid_window"],
                longest_chain_length=pop.longest_chain_length,
                rigid_rod=float(pop.rigid_rod_projection_factor), srk_order=int(config.SRK_order),
                b_get_orientations=bool(pop.b_get_orientations), noise_seed=spec["noise_seed"],
                fixed_dt=spec["fixed_dt"], save_every=spec["save_every"],
                init_grow_steps=int(status.stepnum), init_grow_seconds=grow_s, **init_scal)

    # single-kernel goldens on the relaxed state
    dim = config.dim
    f = np.zeros_like(pop.pos)
    tl = pop.tangent_list.copy()
    forces.calc_chain_spring_forces(pop.pos, tl, pop.chain_id, f, config.Lx, pop.spring_params(),
                                    pop.rest_lengths)
    out["k_spring_forces"] = f.copy()
    out["k_spring_tangent"] = tl.copy()
    # fresh lists at the relaxed state, built the way configure_start builds them
    pop.update_grid_list(overwrite=True)
    pop.update_nbor_list_with_pop2(pop, grid_window=sim["grid_window"])
    out["k_where_is_bead"] = pop.where_is_bead.copy()
    out["k_grid_pairs"] = _grid_pairs(pop.grid_list)
    out["k_nbor_pairs"] = _nbor_pairs(pop.nbor_list[0])
    n_grid = pop.grid_list.shape[1]
    gw_loop = max(1, int(np.ceil(config.grid_factor * pop.WCA_params[3] / (config.Lx / n_grid))))
    fp = np.zeros_like(pop.pos)
    forces.central_pair_force(np.array([0, 0, 0, 1, 1]), pop.pos, pop.nbor_list[0], fp, tl,
                              pop.where_active, config.Lx, pop.pos, pop.WCA_params, tl,
                              gw_loop * config.Lx / n_grid)
    out["k_pair_forces"] = fp.copy()
    fprop = np.zeros_like(pop.pos)
    forces.self_propel(fprop, tl, pop.active_params())
    out["k_propel_forces"] = fprop.copy()
    scal["pbc_width"] = gw_loop * config.Lx / n_grid

    # the hot path: repeated SRK2_force_calc calls with a seeded Numba RNG
    if spec["fixed_dt"]:
        status.dt = spec["dt"]
        status.dtmax = spec["dt"]
        config.max_dist_per_step = math.inf
    if spec["save_every"]:
        sim["save_state_every"] = spec["save_every"]
        status.next_save_time = status.t + spec["save_every"]
    scal["max_dist_per_step"] = config.max_dist_per_step
    scal["grid_depth1"] = int(pop.grid_list.shape[-1])
    scal["nbor_depth1"] = int(pop.nbor_list.shape[-1])
    scal["dtmax"] = status.dtmax
    out["lists_before_pos"] = pop.pos.copy()
    _seed(spec["noise_seed"])
    st_before, st_after = [], []
    for ci, n in enumerate(spec["calls"]):
        status.next_output_step = status.stepnum + n
        st_before.append(_status_fields(status))
        updates.SRK2_force_calc(pops, status, sim)
        st_after.append(_status_fields(status))
        out[f"call{ci}_pos"] = pop.pos.copy()
        out[f"call{ci}_tangent"] = pop.tangent_list.copy()
        out[f"call{ci}_forces"] = pop.forces.copy()
        if config.SRK_order == 4:
            out[f"call{ci}_forces_aux"] = pop.forces_aux.copy()
        if spec["save_every"] and status.t >= status.next_save_time:
            status.next_save_time += spec["save_every"]
    out["status_before"] = np.array(st_before)
    out["status_after"] = np.array(st_after)
    out["calls"] = np.array(spec["calls"], dtype=np.int64)
    scal["final_nbor_depth1"] = int(pop.nbor_list.shape[-1])
    out["final_nbor_pairs"] = _nbor_pairs(pop.nbor_list[0])
    out["final_grid_pairs"] = _grid_pairs(pop.grid_list)
    out["final_where_is_bead"] = pop.where_is_bead.copy()
    out["scalars"] = np.array(json.dumps(scal, default=lambda o: o.item()))
    return out, scal


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--one", action="store_true",
                    help="run the listed cases in this process (internal)")
    args = ap.parse_args()
    if not args.one:
        # Numba freezes module globals such as config.dim at first compile, so
        # every case runs in a fresh process with its own scratch copy.
        index = {}
        for name in ["rng"] + list(args.cases):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--one", "--ref", args.ref,
                            "--out", args.out, "--cases", name], check=True)
            with open(os.path.join(args.out, f"{name}.json")) as fh:
                index[name] = json.load(fh)
            os.remove(os.path.join(args.out, f"{name}.json"))
        # a run over some cases keeps the index entries of the others
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

    # pin the RNG stream: Numba's standard_normal after np.random.seed
    from numba import njit

    @njit
    def _draw(s, n):
        np.random.seed(s)
        o = np.empty(n)
        for i in range(n):
            o[i] = np.random.standard_normal()
        return o

    index = {}
    os.chdir(cwd)
    os.makedirs(args.out, exist_ok=True)
    if args.cases == ["rng"]:
        rng = {"seed0": _draw(0, 1000), "seed12345": _draw(12345, 1000)}
        np.savez_compressed(os.path.join(args.out, "rng.npz"), **rng)
        index["rng"] = {"file": "rng.npz"}
    for name in [c for c in args.cases if c != "rng"]:
        os.chdir(ref)
        t0 = time.time()
        out, scal = run_case(name, CASES[name], mods)
        os.chdir(cwd)
        path = os.path.join(args.out, f"{name}.npz")
        np.savez_compressed(path, **out)
        index[name] = {"file": f"{name}.npz", "bytes": os.path.getsize(path),
                       "beads": int(out["pos0"].shape[0]), "seconds": round(time.time() - t0, 1),
                       **{k: scal[k] for k in ("L", "dim", "n_grid", "init_grow_steps")}}
        print(name, index[name], flush=True)
    for name, entry in index.items():
        with open(os.path.join(args.out, f"{name}.json"), "w") as fh:
            json.dump(entry, fh)
    shutil.rmtree(scratch, ignore_errors=True)


if __name__ == "__main__":
    main()
