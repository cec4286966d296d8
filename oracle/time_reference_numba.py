#!/usr/bin/env python3
"""Time the reference's own Numba step against the oracle's C restatement.

    python oracle/time_reference_numba.py [--ref /root/reference] [--systems 8] [--steps 40]

Test infrastructure, run where the reference source and Numba are present
(not on the GPU hosts): it backs the CPU baseline that ``bench.py`` reports,
which times the C restatement (``kind: port``) because the reference cannot
travel to the GPU hosts.

For `--systems` systems at the bead-count quantiles of the benchmark sweep
(the bench's own sample), each relaxed untimed by the oracle under the
reference's adaptive dt, the script times on the same state:
  * the reference's ``updates.SRK2_force_calc`` (Numba, chain-chunked Python
    threads), run on a scratch copy of the reference with the shims its
    fixtures use (numpy's removed aliases, a stubbed matplotlib), with
    ``config.n_threads`` = all host threads and = 1, after one untimed call
    that compiles it;
  * the oracle (``oracle.OracleSystem.run``, OpenMP over the same chunks)
    with all host threads and one.
Both follow the reference's adaptive dt rule (dtmax 1e-3, max_dist_per_step
of its grid_list_setup) and rebuild Verlet lists every 40 steps.  It prints
one JSON line per system and a summary line (bead-steps/s summed over the
sample as bench.py sums it: total bead-steps / total time).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

CHILD = r"""
import json, os, shutil, sys, tempfile, time, types
import numpy as np
ref_src, cases_path, steps, threads = sys.argv[1], sys.argv[2], int(sys.argv[3]), int(sys.argv[4])
scratch = tempfile.mkdtemp(prefix="gcr_numba_")
ref = os.path.join(scratch, "ref")
shutil.copytree(ref_src, ref, ignore=shutil.ignore_patterns("Chiral_paper_plots", "Images", "Results"))
for r, ds, fs in os.walk(ref):
    for d in ds:
        os.chmod(os.path.join(r, d), 0o755)
    for f in fs:
        os.chmod(os.path.join(r, f), 0o644)
os.makedirs(os.path.join(ref, "Results"), exist_ok=True)
np.float = float
np.int = int

class _Stub(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return lambda *a, **k: None

for m in ["matplotlib", "matplotlib.pyplot", "matplotlib.colors", "matplotlib.cm", "matplotlib.collections",
          "matplotlib.patches", "mpl_toolkits", "mpl_toolkits.mplot3d", "mpl_toolkits.mplot3d.art3d",
          "mpl_toolkits.axes_grid1", "mpl_toolkits.axes_grid1.inset_locator"]:
    sys.modules[m] = _Stub(m)
os.chdir(ref)
sys.path.insert(0, ref)
import populations  # noqa: F401  (first: the reference's circular imports)
import config, updates, defaults, control
cases = np.load(cases_path, allow_pickle=True)["cases"]
out = []
for case in cases:
    sim, _ = defaults.set_defaults()
    sim.update(case["sim"])
    sim.update(dict(plot_every=-1, ticker_every=-1, save_state_every=-1., t_init_grow=0., a_init_factor=1.,
                    dt0=1e-3, dtmax=1e-3, n_threads=threads))
    config.configure(sim)
    pops = [populations.Equal_Size_Chain_Collection(sim, name="beads")]
    pop = pops[0]
    pop.random_initialization()
    pop.pos[:] = case["pos"]
    pop.tangent_list[:] = case["tangent"]
    status = config.status_class(sim)
    control.configure_start(sim, pops, status)  # grids and lists of the relaxed state
    status.dt = float(case["dt"])
    row = {"name": case["name"], "beads": int(pop.total_pop)}
    for n_thr in (threads, 1):
        config.n_threads = n_thr
        sim["n_threads"] = n_thr
        status.next_output_step = status.stepnum + 2  # compiles / warms the threads
        updates.SRK2_force_calc(pops, status, sim)
        status.next_output_step = status.stepnum + steps
        s0 = status.stepnum
        t0 = time.perf_counter()
        updates.SRK2_force_calc(pops, status, sim)
        dt = time.perf_counter() - t0
        row[f"numba_{n_thr}"] = {"steps": status.stepnum - s0, "seconds": dt}
    out.append(row)
print("RESULT " + json.dumps(out))
shutil.rmtree(scratch, ignore_errors=True)
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--systems", type=int, default=8)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()

    import bench
    from gliding_collective_rotation_b200 import workloads as W
    from oracle import oracle as O

    specs = W.config3(n_systems=256, param_seed=12345)
    idx = bench.stratified(specs, a.systems)
    cases, states = [], []
    for i in idx:
        sp = specs[i]
        pos, tan = bench.relax_on_cpu(sp)
        p = sp.params
        states.append((sp, pos, tan))
        cases.append({"name": sp.name, "pos": pos, "tangent": tan, "dt": 1e-3,
                      "sim": dict(Lx=float(p.L), n_chains=len(sp.rest_lengths), chain_length=int(sp.n // len(sp.rest_lengths)),
                                  a=0.5, k=100., kappa=float(p.spring_params[1]), repel_d_max=1., WCA_epsilon=1.,
                                  LJ_cutoff_factor=1., v0=1., v_tan_angle=float(p.active_params[2]), T=0.01,
                                  dim=2, seed=int(p.seed))})
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "cases.npz")
        np.savez(path, cases=np.array(cases, dtype=object))
        res = subprocess.run([sys.executable, "-c", CHILD, a.ref, path, str(a.steps), str(a.threads)],
                             capture_output=True, text=True, timeout=3600)
    line = [ln for ln in res.stdout.splitlines() if ln.startswith("RESULT ")]
    if res.returncode != 0 or not line:
        sys.exit(res.stdout[-3000:] + res.stderr[-3000:])
    rows = json.loads(line[0][len("RESULT "):])
    # the oracle on the same relaxed states
    for row, (sp, pos, tan) in zip(rows, states):
        p = sp.params
        for n_thr in (a.threads, 1):
            ng = max(1, int(p.L / (2.0 * max(2 * sp.rest_lengths.max(), p.wca_params[3]))))
            o = O.OracleSystem(pos, tan, sp.chain_id, sp.rest_lengths, p.L, p.spring_params, p.wca_params,
                               p.active_params, p.D, p.Dr, p.radius, p.n_nearby, ng, nbor_depth=32)
            o.build_lists(grid_window=1)
            o.seed_mt(int(p.seed), n_thr)
            o.run(2, dt=1e-3, dtmax=sp.dt, max_dist_per_step=sp.relax_mdps, n_threads=n_thr)
            t0 = time.perf_counter()
            r = o.run(a.steps, dt=1e-3, dtmax=sp.dt, max_dist_per_step=sp.relax_mdps, n_threads=n_thr)
            row[f"port_{n_thr}"] = {"steps": r["steps"], "seconds": time.perf_counter() - t0}
        print(json.dumps(row), flush=True)
    summ = {"threads": a.threads, "systems": len(rows), "beads": sum(r["beads"] for r in rows), "steps": a.steps}
    for key in (f"numba_{a.threads}", "numba_1", f"port_{a.threads}", "port_1"):
        bs = sum(r["beads"] * r[key]["steps"] for r in rows)
        summ[key + "_bead_steps_per_s"] = bs / sum(r[key]["seconds"] for r in rows)
    summ["port_over_numba"] = summ[f"port_{a.threads}_bead_steps_per_s"] / summ[f"numba_{a.threads}_bead_steps_per_s"]
    summ["port_over_numba_1thread"] = summ["port_1_bead_steps_per_s"] / summ["numba_1_bead_steps_per_s"]
    print(json.dumps({"summary": summ}), flush=True)


if __name__ == "__main__":
    main()
