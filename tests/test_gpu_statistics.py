"""Statistics of long runs: the GPU step against the CPU oracle (the
reference's algorithm, pinned to the reference's own trajectories).

Eight independent Philox seeds on each side (different seeds, so the two
samples are independent), all from the reference's relaxed state of the
2,000-bead system, 1,000 steps of dt = 1e-3 in FP64.  Compared per run and
then as means over the eight runs, within two standard errors of their
difference:

* mean-squared displacement of the beads (the GPU runs from the device's
  image counters; the oracle runs unwrapped every 40 steps, the
  oracle's list period, far below half a box per chunk);
* polar and nematic order parameters of the chain directions
  (analysis.polar_orderparameter, analysis.nematic_orderparameter);
* the contact number: beads within r < 1.1 of a bead of another chain (the
  first peak of the bead-bead g(r)).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.engine import SystemParams  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden_io import load, min_image  # noqa: E402

N_RUNS, STEPS, CHUNK = 8, 1000, 40


def _params(seed):
    d, s = load("config1")
    return d, s, SystemParams(L=s["L"], spring_params=d["spring_params"], wca_params=d["wca_params"],
                              active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                              n_nearby=s["n_nearby"], dtmax=1e-3, seed=seed)


def _observables(pos_unwrapped, pos0, pos, tangent, chain, L):
    msd = float(np.mean(np.sum((pos_unwrapped - pos0) ** 2, axis=1)))
    P, S, _ = O.order_params(tangent, np.concatenate(([0], np.flatnonzero(np.diff(chain)) + 1, [len(chain)])))
    # contacts with beads of other chains
    n = len(pos)
    cnt = 0
    for i in range(0, n, 500):
        d = min_image(pos[i:i + 500, None, :] - pos[None, :, :], L)
        r2 = np.sum(d * d, axis=2)
        other = chain[i:i + 500, None] != chain[None, :]
        cnt += int(np.sum((r2 < 1.1 ** 2) & other))
    return np.array([msd, P, S, cnt / n])


def _gpu_runs():
    specs = []
    for k in range(N_RUNS):
        d, s, prm = _params(1000 + k)
        specs.append(W.SystemSpec(f"c1_{k}", 2, d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], prm,
                                  1e-3, 0.0125))
    b = Batch(specs, precision="fp64")
    L = specs[0].params.L
    pos0 = [st.pos.cpu().numpy().copy() for st in b.states]
    # the device counts the periodic images: the whole run in one call, and the
    # unwrapped positions (hence the MSD) read once at the end
    b.begin(STEPS)
    b.run(STEPS)
    b.engine.synchronize()
    sts = b.statuses()
    assert all(s["flags"] == 0 and s["steps_done"] == STEPS for s in sts)
    unw = [u.cpu().numpy() for u in b.unwrapped()]
    out = [_observables(unw[i], pos0[i], st.pos.cpu().numpy(), st.tangent.cpu().numpy(), specs[i].chain_id, L)
           for i, st in enumerate(b.states)]
    b.close()
    return np.array(out)


def _oracle_runs():
    d, s, _ = _params(0)
    L = s["L"]
    out = []
    for k in range(N_RUNS):
        # the reference's grid and list depths for this system (recorded with the fixture)
        sysm = O.OracleSystem(d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], L, d["spring_params"],
                              d["wca_params"], d["active_params"], s["D"], s["Dr"], s["radius"], s["n_nearby"],
                              s["n_grid"], s["grid_factor"], grid_depth=s["grid_depth1"] - 1,
                              nbor_depth=2 * max(s["nbor_depth1"], s["final_nbor_depth1"]))
        sysm.build_lists(grid_window=s["grid_window"])
        pos0 = sysm.pos.copy()
        unw, prev = pos0.copy(), pos0.copy()
        for c in range(STEPS // CHUNK):
            res = sysm.run(CHUNK, dt=1e-3, noise_mode=O.NOISE_PHILOX, seed=5000 + k, step0=c * CHUNK,
                           steps_until_update=CHUNK, n_steps_update=CHUNK, n_threads=os.cpu_count() or 1)
            assert res["flag"] >= 0 and res["steps"] == CHUNK
            unw += min_image(sysm.pos - prev, L)
            prev = sysm.pos.copy()
        out.append(_observables(unw, pos0, prev, sysm.tangent_list, np.asarray(d["chain_id"]), L))
    return np.array(out)


def test_long_run_statistics_match_the_oracle():
    g, o = _gpu_runs(), _oracle_runs()
    names = ["msd", "polar P", "nematic S", "contacts per bead"]
    for j, name in enumerate(names):
        diff = g[:, j].mean() - o[:, j].mean()
        se = np.sqrt(g[:, j].var(ddof=1) / N_RUNS + o[:, j].var(ddof=1) / N_RUNS)
        assert abs(diff) <= 2 * se, (name, g[:, j].mean(), o[:, j].mean(), se)
