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


# ---------------------------------------------------------------------------
# the config-2 and config-5 physics, and the mixed path
# ---------------------------------------------------------------------------
#
# 24 independent Philox seeds on each side from the reference's relaxed
# state of each fixture, run to the same physical time T in 20 chunks of
# T/20 (the call's time limit, max_dt_usable, as the reference's save times
# cut its calls, SRK.py:128-130), the GPU in the given precision, the oracle
# in FP64:
#   chiral_lj  2D, LJ 2.5 sigma, eps 0.5, chirality 0.2, adaptive dt  (config-2 physics)
#   rotdiff3d  3D, LJ eps 1, kappa 10, rotational diffusion Dr 0.1    (config-5 physics)
#   config1    2D WCA, the mixed path
# Observables at T: the beads' mean-squared displacement (GPU: the device's
# image counters), the bead-bead g(r) of beads of different chains binned
# over [0, 3) in 15 bins, and per case: P and S and the chains' mean
# rotation rate (2D: the chain angle of calc_avg_phi_chain unwrapped from
# chunk to chunk, over T -- the chirality's signature), or the tangent
# autocorrelation <t(T).t(0)> (3D: the rotational diffusion).  Scalars agree
# within two standard errors of the difference of the means; the g(r) curve
# by a chi-square over its bins (sum of squared z-scores below the 99.9%
# point of chi2 with as many degrees of freedom as bins).

N_SEEDS = 24
GR_EDGES = np.linspace(0.0, 3.0, 16)
STAT_CASES = {  # fixture: (physical time, chunks)
    "chiral_lj": (1.0, 20),
    "rotdiff3d": (0.5, 20),
    "config1": (1.0, 20),
}


def _chain_starts(chain):
    return np.concatenate(([0], np.flatnonzero(np.diff(chain)) + 1, [len(chain)]))


def _gr_counts(pos, chain, L):
    """Pairs of beads of different chains per bead, binned by distance."""
    n = len(pos)
    counts = np.zeros(len(GR_EDGES) - 1)
    for i in range(0, n, 400):
        d = min_image(pos[i:i + 400, None, :] - pos[None, :, :], L)
        r = np.sqrt(np.sum(d * d, axis=2))
        other = chain[i:i + 400, None] != chain[None, :]
        counts += np.histogram(r[other], bins=GR_EDGES)[0]
    return counts / n


def _chain_angles(tangent, cs):
    from oracle.observables import avg_phi
    return avg_phi(tangent, cs, 1)


class _Tracker:
    """Chain angles unwrapped from chunk to chunk (2D), start tangents (3D)."""

    def __init__(self, tangent, cs, dim):
        self.dim, self.cs = dim, cs
        self.t0 = tangent.copy()
        self.phi = _chain_angles(tangent, cs) if dim == 2 else None
        self.turned = np.zeros(len(cs) - 1)

    def update(self, tangent):
        if self.dim == 2:
            phi = _chain_angles(tangent, self.cs)
            self.turned += np.angle(np.exp(1j * (phi - self.phi)))
            self.phi = phi

    def final(self, tangent, T):
        if self.dim == 2:
            return [float(np.mean(self.turned)) / T]
        return [float(np.mean(np.sum(tangent * self.t0, axis=1)))]


def _stats_row(unw, pos0, pos, tangent, chain, L, dim, tracker, T):
    msd = float(np.mean(np.sum((unw - pos0) ** 2, axis=1)))
    row = [msd]
    if dim == 2:
        P, S, _ = O.order_params(tangent, _chain_starts(chain))
        row += [P, S]
    row += tracker.final(tangent, T)
    return np.array(row), _gr_counts(pos, chain, L)


def _case(name):
    d, s = load(name)
    T, chunks = STAT_CASES[name]
    mdps = float(s["max_dist_per_step"]) if not s["fixed_dt"] else np.inf
    return d, s, T, chunks, mdps


def _stats_gpu(name, precision):
    d, s, T, chunks, mdps = _case(name)
    dim, L = int(s["dim"]), float(s["L"])
    specs = []
    for k in range(N_SEEDS):
        prm = SystemParams(L=L, spring_params=d["spring_params"], wca_params=d["wca_params"],
                           active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                           n_nearby=s["n_nearby"], dtmax=s["dtmax"], max_dist_per_step=mdps,
                           rk_cheat=s["rk_cheat"], seed=2000 + k)
        specs.append(W.SystemSpec(f"{name}_{k}", dim, d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"],
                                  prm, s["dtmax"], mdps))
    # lists deep enough for the LJ clusters (calls are armed directly here,
    # without the regrow that Batch.run_checked does after an overflow)
    b = Batch(specs, precision=precision, list_depth=256, cell_depth=64)
    chain = np.asarray(d["chain_id"])
    cs = _chain_starts(chain)
    pos0 = [st.pos.cpu().numpy().copy() for st in b.states]
    trackers = [_Tracker(st.tangent.double().cpu().numpy(), cs, dim) for st in b.states]
    dts = [float(s["dtmax"])] * N_SEEDS
    for c in range(chunks):
        b.engine.call_begin_many([st.slot for st in b.states], 100000, dts, max_dt_usable=T / chunks)
        b.run(100000, sync_every=4)
        b.engine.synchronize()
        sts = b.statuses()
        assert all(x["flags"] == 0 and not x["active"] for x in sts), sts
        dts = [x["dt"] for x in sts]
        for tr, st in zip(trackers, b.states):
            tr.update(st.tangent.double().cpu().numpy())
    unw = [u.cpu().numpy() for u in b.unwrapped()]
    rows = [_stats_row(unw[i], pos0[i], st.pos.cpu().numpy(), st.tangent.double().cpu().numpy(), chain, L, dim,
                       trackers[i], T) for i, st in enumerate(b.states)]
    b.close()
    return np.array([r[0] for r in rows]), np.array([r[1] for r in rows])


def _stats_oracle(name):
    d, s, T, chunks, mdps = _case(name)
    dim, L = int(s["dim"]), float(s["L"])
    chain = np.asarray(d["chain_id"])
    cs = _chain_starts(chain)
    rows = []
    for k in range(N_SEEDS):
        sysm = O.OracleSystem(d["pos0"], d["tangent0"], chain, d["rest_lengths"], L, d["spring_params"],
                              d["wca_params"], d["active_params"], s["D"], s["Dr"], s["radius"], s["n_nearby"],
                              s["n_grid"], s["grid_factor"], grid_depth=2 * s["grid_depth1"],
                              nbor_depth=2 * max(s["nbor_depth1"], s["final_nbor_depth1"]))
        sysm.build_lists(grid_window=s["grid_window"])
        pos0 = sysm.pos.copy()
        unw, prev = pos0.copy(), pos0.copy()
        tracker = _Tracker(sysm.tangent_list.copy(), cs, dim)
        dt, step, until = float(s["dtmax"]), 0, int(s["n_steps_update"])
        for c in range(chunks):
            res = sysm.run(100000, dt=dt, dtmax=s["dtmax"], max_dist_per_step=mdps, rk_cheat=s["rk_cheat"],
                           max_dt_usable=T / chunks, noise_mode=O.NOISE_PHILOX, seed=7000 + k, step0=step,
                           steps_until_update=until, n_steps_update=int(s["n_steps_update"]),
                           n_threads=os.cpu_count() or 1)
            assert res["flag"] >= 0, res
            n = res["steps"]
            step += n
            # the oracle's next list rebuild, counted across calls
            until = until - n if n < until else int(s["n_steps_update"]) - (n - until) % int(s["n_steps_update"])
            dt = res["dt"]
            unw += min_image(sysm.pos - prev, L)
            prev = sysm.pos.copy()
            tracker.update(sysm.tangent_list)
        rows.append(_stats_row(unw, pos0, prev, sysm.tangent_list.copy(), chain, L, dim, tracker, T))
    return np.array([r[0] for r in rows]), np.array([r[1] for r in rows])


@pytest.mark.parametrize("name,precision", [("chiral_lj", "fp64"), ("chiral_lj", "mixed"), ("rotdiff3d", "fp64"),
                                            ("rotdiff3d", "mixed"), ("config1", "mixed")])
def test_statistics_of_lj_3d_and_mixed_runs_match_the_oracle(name, precision):
    from scipy.stats import chi2
    (gs, gg), (os_, og) = _stats_gpu(name, precision), _stats_oracle(name)
    dim = int(load(name)[1]["dim"])
    names = ["msd"] + (["polar P", "nematic S", "chain rotation rate"] if dim == 2 else ["tangent autocorrelation"])
    report = {}
    for j, nm in enumerate(names):
        diff = gs[:, j].mean() - os_[:, j].mean()
        se = np.sqrt(gs[:, j].var(ddof=1) / N_SEEDS + os_[:, j].var(ddof=1) / N_SEEDS)
        report[nm] = (gs[:, j].mean(), os_[:, j].mean(), se)
        assert abs(diff) <= 2 * se, (name, precision, nm, report[nm])
    # g(r): bins with counts on either side
    gm, om = gg.mean(axis=0), og.mean(axis=0)
    se = np.sqrt(gg.var(axis=0, ddof=1) / N_SEEDS + og.var(axis=0, ddof=1) / N_SEEDS)
    live = se > 0
    z2 = float(np.sum(((gm - om)[live] / se[live]) ** 2))
    assert live.sum() >= 5 and z2 <= chi2.ppf(0.999, int(live.sum())), (name, precision, z2, gm, om, se)
