"""Systems of the benchmarked sweep on the GPU against the oracle.

The bench's default workload is 256 heterogeneous 2D systems (chains of
5-40 beads, bending 1..50, chirality -0.5..0.5, area fraction 0.1-0.4).  Six
of them -- the smallest, one of at least 50k beads, and the ones with the
smallest and largest bending constant and chirality -- are relaxed together
on the device in FP64 and then advanced in one batch with the Philox stream;
the oracle (the reference's step restated in C, same Philox stream, the
reference's 40-step Verlet lists and its own summation order) advances each
from the same state under the reference's adaptive dt rule.  Positions
agree within 1e-12 of the box after one step and 1e-9 after 200; the dt
each step took agrees within 1e-9 relative.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden_io import min_image  # noqa: E402

N_UPDATE = 40  # the reference's list cadence (config.grid_list_setup with dt safety 1/40)


def pick_systems(specs):
    """Indices of the smallest system, a system of >= 50k beads (the one
    closest to 50k), and the extremes of bending constant and chirality."""
    n = np.array([s.n for s in specs])
    kappa = np.array([s.params.spring_params[1] for s in specs])
    chir = np.array([s.params.active_params[2] for s in specs])
    big = np.flatnonzero(n >= 50000)
    picks = [int(np.argmin(n)), int(big[np.argmin(n[big])]), int(np.argmin(kappa)), int(np.argmax(kappa)),
             int(np.argmin(chir)), int(np.argmax(chir))]
    out = []
    for i in picks:
        if i not in out:
            out.append(i)
    return out


def _countdown(until, n):
    """Steps to the oracle's next list rebuild after `n` more steps."""
    if n < until:
        return until - n
    return N_UPDATE - (n - until) % N_UPDATE


def test_sweep_systems_match_the_oracle():
    specs = W.config3(n_systems=256, param_seed=12345)
    idx = pick_systems(specs)
    sel = [specs[i] for i in idx]
    assert any(s.n >= 50000 for s in sel)
    b = Batch(sel, precision="fp64")
    b.relax(max_steps=2000, adaptive_after=True)
    sts = b.statuses()
    assert not any(s["flags"] for s in sts)
    oracles, dts, step0 = [], [s["dt"] for s in sts], [s["step"] for s in sts]
    for st, sp in zip(b.states, sel):
        p = sp.params
        a = float(sp.rest_lengths.max())
        rc = float(p.wca_params[3])
        ng = max(1, int(p.L / (2.0 * max(2 * a, rc))))
        o = O.OracleSystem(st.pos.cpu().numpy(), st.tangent.cpu().numpy(), sp.chain_id, sp.rest_lengths, p.L,
                           p.spring_params, p.wca_params, p.active_params, p.D, p.Dr, p.radius, p.n_nearby, ng,
                           nbor_depth=64)
        o.build_lists(grid_window=max(1, math.ceil(max(2 * a, rc) / (p.L / ng))))
        oracles.append(o)
    until = [N_UPDATE] * len(sel)
    done = 0
    report, bad = [], []
    for n_steps, tol in ((1, 1e-12), (9, 1e-11), (40, 1e-10), (150, 1e-9)):
        b.begin(n_steps)
        b.run(n_steps)
        sts = b.statuses()
        for j, (st, sp, o) in enumerate(zip(b.states, sel, oracles)):
            p = sp.params
            assert sts[j]["steps_done"] == n_steps and sts[j]["flags"] == 0, (sp.name, sts[j])
            res = o.run(n_steps, dt=dts[j], dtmax=sp.dt, max_dist_per_step=sp.relax_mdps,
                        noise_mode=O.NOISE_PHILOX, seed=p.seed, step0=step0[j] + done, steps_until_update=until[j])
            assert res["steps"] == n_steps
            # the dt rule on the same forces: equal to rounding after the first
            # step; later the trajectories' own (tiny) differences feed it
            dt_tol = 1e-12 if done == 0 else 1e-6
            dt_err = abs(res["dt"] - sts[j]["dt"]) / res["dt"]
            dts[j] = res["dt"]
            until[j] = _countdown(until[j], n_steps)
            err = np.max(np.abs(min_image(st.pos.cpu().numpy() - o.pos, p.L))) / p.L
            report.append((sp.name, sp.n, done + n_steps, err, dt_err))
            if err >= tol or dt_err > dt_tol:
                bad.append(report[-1])
        done += n_steps
    b.close()
    assert not bad, (bad, report)
