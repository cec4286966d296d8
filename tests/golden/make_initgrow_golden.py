#!/usr/bin/env python3
"""Golden vectors of the reference's rigid-rod projection and init-grow
protocol, made by running the reference itself.

Run from the repository root where the reference source is mounted at
/root/reference (read-only; it is copied to a scratch directory) and Numba
is installed:

    python tests/golden/make_initgrow_golden.py [--ref /root/reference] [--out tests/golden]

Two fixtures:

``rigid_project.npz`` -- direct calls of updates.project_updates_for_rigid_rod
(updates.py:347-499) in 2D and 3D on seeded chains: bent, stretched and
wrapped across the periodic boundary, of mixed lengths (1, 2, 5 and 12
beads, two rest lengths; no one-bead chain in 3D, where the reference
divides by its zero moment of inertia), with forces and noise, for projection factors
0.3 and 1.  Inputs and the returned positions are stored per call.

``initgrow.npz`` -- the reference's init-grow loop (control.sim_loop while
growing: control.early_time_procedures, control.py:153-219, then
updates.SRK2_force_calc with growing_stepskip = 10 steps per call) on a 2D
system (Lx = 40, 100 chains x 10 beads, config-1 physics, the reference's
growth defaults t_init_grow = 1 and a_init_factor = 1e-8).  Two windows of
8 consecutive calls: ``repel`` (the first calls with progress >= 0.1:
repulsion radius ramped up, no projection) and ``rigid`` (the first calls
with progress >= 0.3: projection factor 0.025, kappa 10).  Earlier calls are
ill-conditioned (bonds of 5e-9 at coordinates ~40) and are not recorded.  Per call: the status before and after,
every parameter the step reads, and the positions, tangents and forces
after; per window, the state before its first call.  D = 0 while growing,
so these calls draw no translational noise.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_golden import _install_shims, _status_fields  # noqa: E402

WINDOW = 8


def _scratch_reference(src):
    scratch = tempfile.mkdtemp(prefix="gcr_grow_")
    ref = os.path.join(scratch, "ref")
    shutil.copytree(src, ref, ignore=shutil.ignore_patterns("*.zip", "*.ipynb"))
    for root, dirs, files in os.walk(ref):
        for d in dirs:
            os.chmod(os.path.join(root, d), 0o755)
        for fn in files:
            os.chmod(os.path.join(root, fn), 0o644)
    os.makedirs(os.path.join(ref, "Results"), exist_ok=True)
    os.chdir(ref)
    sys.path.insert(0, ref)
    _install_shims()
    return scratch


def _chains(rng, dim, L, lengths, rests):
    """Chains along random directions with bend and stretch, wrapped."""
    pos, chain_id = [], []
    for ci, (n, a) in enumerate(zip(lengths, rests)):
        x = rng.uniform(0, L, dim)
        u = rng.normal(size=dim)
        u /= np.linalg.norm(u)
        for b in range(n):
            pos.append(x.copy())
            chain_id.append(ci)
            step = u * a * rng.uniform(0.8, 1.3) + rng.normal(scale=0.15 * a, size=dim)
            x = x + step
    return np.mod(np.array(pos), L), np.array(chain_id, dtype=np.int64)


def part_project(dim, out_dir):
    import populations  # noqa: F401  (must come first: circular imports)
    import config
    import updates
    import defaults

    sim, _ = defaults.set_defaults()
    sim.update(dict(dim=dim, Lx=8., n_threads=1, b_cached=True, filelabel="golden_proj", plot_every=-1,
                    ticker_every=-1, save_state_every=-1.))
    config.configure(sim)
    config.n_threads = 1
    rng = np.random.default_rng(100 + dim)
    # a one-bead chain only in 2D: the 3D projection divides by its zero
    # moment of inertia (updates.py:493) and raises
    lengths = [12, 5, 1 if dim == 2 else 3, 2, 12, 5, 12, 12]
    rests = [0.5, 0.5, 0.5, 0.5, 0.35, 0.35, 0.5, 0.5]
    L = 8.
    out = {}
    k = 0
    for pf in (0.3, 1.0):
        for stage, (dt, D, radius) in enumerate([(1e-3, 0.01, 1.0), (5e-4, 0.05, 0.8)]):
            pos, chain_id = _chains(rng, dim, L, lengths, rests)
            n = len(pos)
            # the last two chains sit across the boundary
            for ci in (6, 7):
                sel = chain_id == ci
                pos[sel] = np.mod(pos[sel] - pos[sel][0] + (L - 0.3) + 0.05 * ci, L)
            forces = rng.normal(scale=5.0, size=(n, dim))
            noise = rng.normal(size=(n, 2 * dim))
            nch = len(lengths)
            book = np.full((nch, 1 + max(lengths)), -1, dtype=np.int64)
            book[:, 0] = 0
            for bi in range(n):
                c = chain_id[bi]
                book[c, 1 + book[c, 0]] = bi
                book[c, 0] += 1
            rest_lengths = np.array(rests, dtype=np.float64)
            rtn = np.zeros_like(pos)
            updates.project_updates_for_rigid_rod(np.array([0, 0], dtype=np.int64), rtn, pos, forces, noise,
                                                  book, chain_id, rest_lengths, pf, L, dt, D, radius)
            for nm, v in (("pos", pos), ("forces", forces), ("noise", noise), ("chain_id", chain_id),
                          ("rest", rest_lengths), ("out", rtn.copy())):
                out[f"c{k}_{nm}"] = v
            out[f"c{k}_scal"] = np.array([pf, L, dt, D, radius])
            k += 1
    out["n_calls"] = np.array(k)
    path = os.path.join(out_dir, f"_proj{dim}.npz")
    np.savez(path, **out)


def part_initgrow(out_dir):
    import populations
    import config
    import updates
    import defaults
    import control

    sim, _ = defaults.set_defaults()
    sim.update(dict(plot_every=-1, ticker_every=-1, save_state_every=-1., t_max=0., n_threads=1, b_cached=True,
                    filelabel="golden_grow", Lx=40., n_chains=100, chain_length=10, a=0.5, k=100., kappa=20.,
                    repel_d_max=1., WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., v_tan_angle=0., T=0.01, dim=2,
                    seed=2, dtmax=1e-3, dt0=1e-3))
    config.configure(sim)
    config.n_threads = 1
    pops = [populations.Equal_Size_Chain_Collection(sim)]
    status = config.status_class(sim)
    control.configure_start(sim, pops, status)
    pop = pops[0]

    def params():
        return dict(radius=pop.repel_d_max, rigid=pop.rigid_rod_projection_factor, spring=pop.spring_params(),
                    wca=pop.WCA_params.copy(), active=pop.active_params(), D=pop.D, Dr=pop.Dr,
                    n_nearby=pop.n_nearby_beads_dont_repel, rest=pop.rest_lengths.copy(),
                    rk=config.RK_cheat_factor, active_on=float(bool(status.b_calc_active_forces)),
                    mdps=config.max_dist_per_step, dtmax=status.dtmax)

    out = {"chain_id": pop.chain_id.astype(np.int64)}
    scal = dict(L=config.Lx, dim=config.dim, grid_factor=config.grid_factor, n_grid=int(sim["n_grid"]),
                n_steps_update=config.n_steps_update_grid_list, longest_chain_length=int(pop.longest_chain_length),
                t_init_grow=sim["t_init_grow"], t_start=status.t, growing_stepskip=sim["growing_stepskip"])
    # the first calls (progress < ~0.05) are ill-conditioned: bonds of 5e-9
    # at coordinates ~40 carry ~1e-6 relative resolution and one step moves a
    # bead farther than its bond, so the reference's own result hangs on its
    # fastmath rounding; the windows start where bonds are ~1e-2 long
    windows = {"repel": lambda prog: 0.1 <= prog < 0.25, "rigid": lambda prog: prog >= 0.3}
    recorded = {}
    n_calls = 0
    while sim["b_init_growing"]:
        control.early_time_procedures(pops, status, sim)
        if not sim["b_init_growing"]:
            break
        progress = (status.t - scal["t_start"]) / sim["t_init_grow"]
        status.next_output_step = status.stepnum + sim["growing_stepskip"]
        target = None
        for w, cond in windows.items():
            if cond(progress) and len(recorded.get(w, {"calls": []})["calls"]) < WINDOW:
                target = w
                break
        if target is None:
            updates.SRK2_force_calc(pops, status, sim)
        else:
            rec = recorded.setdefault(target, {"calls": []})
            if not rec["calls"]:
                rec["pos0"], rec["tangent0"] = pop.pos.copy(), pop.tangent_list.copy()
            call = {"before": _status_fields(status), "params": params(), "progress": progress}
            updates.SRK2_force_calc(pops, status, sim)
            call.update(after=_status_fields(status), pos=pop.pos.copy(), tangent=pop.tangent_list.copy(),
                        forces=pop.forces.copy())
            rec["calls"].append(call)
        n_calls += 1
        if all(len(recorded.get(w, {"calls": []})["calls"]) >= WINDOW for w in windows):
            break
    for w, rec in recorded.items():
        out[f"{w}_pos0"], out[f"{w}_tangent0"] = rec["pos0"], rec["tangent0"]
        calls = rec["calls"]
        out[f"{w}_status_before"] = np.array([c["before"] for c in calls])
        out[f"{w}_status_after"] = np.array([c["after"] for c in calls])
        for k in ("pos", "tangent", "forces"):
            out[f"{w}_{k}"] = np.array([c[k] for c in calls])
        for k in ("radius", "rigid", "D", "Dr", "n_nearby", "rk", "active_on", "mdps", "dtmax"):
            out[f"{w}_p_{k}"] = np.array([c["params"][k] for c in calls], dtype=np.float64)
        for k in ("spring", "wca", "active", "rest"):
            out[f"{w}_p_{k}"] = np.array([c["params"][k] for c in calls])
        out[f"{w}_progress"] = np.array([c["progress"] for c in calls])
    out["scalars"] = np.array(json.dumps(scal, default=lambda o: o.item()))
    path = os.path.join(out_dir, "initgrow.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {w: len(r["calls"]) for w, r in recorded.items()}, "calls run", n_calls,
          "rigid factors", sorted({float(c["params"]["rigid"]) for r in recorded.values() for c in r["calls"]}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--part", default=None, help="internal: one part per process")
    a = ap.parse_args()
    out_dir = os.path.abspath(a.out)
    if a.part is None:
        # Numba freezes config.dim at first compile: one process per part
        for part in ("project2", "project3", "initgrow"):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--ref", a.ref, "--out", out_dir,
                            "--part", part], check=True)
        merged = {}
        for dim in (2, 3):
            p = os.path.join(out_dir, f"_proj{dim}.npz")
            with np.load(p) as d:
                for k in d.files:
                    merged[f"d{dim}_{k}"] = d[k]
            os.remove(p)
        np.savez_compressed(os.path.join(out_dir, "rigid_project.npz"), **merged)
        return
    scratch = _scratch_reference(a.ref)
    try:
        if a.part.startswith("project"):
            part_project(int(a.part[-1]), out_dir)
        else:
            part_initgrow(out_dir)
    finally:
        shutil.rmtree(scratch, ignore_errors=True)


if __name__ == "__main__":
    main()
