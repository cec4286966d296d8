"""Statistics of a grown state and the init-grow loop on the oracle.

Growth from bonds of 5e-9 is chaotic (the reference's own result hangs on
its last-bit rounding), so grown states are compared through statistics:
the bond-length distribution, close contacts between chains, the number of
growth steps and the time growth ends at."""
import math

import numpy as np

from gliding_collective_rotation_b200.engine import SystemParams
from gliding_collective_rotation_b200.growth import GrowSettings, GrowthConstants, grow_params
from tests.golden_io import load, min_image


def grown_stats(pos, chain, L, close=0.8):
    pos = np.asarray(pos, dtype=np.float64)
    chain = np.asarray(chain)
    same = np.diff(chain) == 0
    bl = np.linalg.norm(min_image(np.diff(pos, axis=0), L), axis=1)[same]
    n_close = 0
    for i0 in range(0, len(pos), 256):
        d = min_image(pos[i0:i0 + 256, None, :] - pos[None, :, :], L)
        r = np.linalg.norm(d, axis=2)
        other = chain[i0:i0 + 256, None] != chain[None, :]
        n_close += int(np.sum((r < close) & other))
    return dict(bond_mean=float(bl.mean()), bond_std=float(bl.std()), bond_min=float(bl.min()),
                bond_max=float(bl.max()), n_close=n_close // 2)


def growth_case(name="config1"):
    """A golden run the reference grew itself: its random placement
    (``init_pos``), its physical parameters and its grown state (``pos0``).
    Both runs used repel_d_max 1, WCA_epsilon 1, WCA_shift 0, rest length 0.5
    and dt0 = dtmax."""
    d, s = load(name)
    ov = s["sim_overrides"]
    base = SystemParams(L=s["L"], spring_params=np.array(d["spring_params"]), wca_params=np.array(d["wca_params"]),
                        active_params=np.array(d["active_params"]), D=s["D"], Dr=s["Dr"], radius=s["radius"],
                        n_nearby=s["n_nearby"], dtmax=s["dtmax"], max_dist_per_step=s["max_dist_per_step_setup"])
    consts = GrowthConstants(repel_d_max=1.0, WCA_epsilon=1.0, WCA_shift=0.0,
                             LJ_cutoff_factor=float(ov.get("LJ_cutoff_factor", 1.0)), reference_rest_length=0.5,
                             longest_chain_length=s["longest_chain_length"])
    settings = GrowSettings(dt0=s["dtmax"])
    return d, s, base, consts, settings


def config1_growth_case():
    return growth_case("config1")


def check_like_reference(stats, ref, steps, ref_steps, t):
    assert abs(stats["bond_mean"] - ref["bond_mean"]) <= 0.02, (stats, ref)
    assert stats["bond_std"] <= 2.0 * ref["bond_std"], (stats, ref)
    assert stats["bond_min"] > 0.02 and stats["bond_max"] < 0.8, stats
    assert stats["n_close"] == 0 == ref["n_close"], stats
    assert abs(steps - ref_steps) <= 0.2 * ref_steps, (steps, ref_steps)
    assert 0.0 < t <= 0.02, t


def oracle_grow(d, s, base, consts, settings):
    """control.sim_loop while growing, on the oracle: parameters from the
    schedule, then one call of ``growing_stepskip`` steps."""
    from oracle import oracle as O
    L = s["L"]
    n_chains = len(d["rest_lengths"])
    sysm = O.OracleSystem(d["init_pos"], d["init_tangent"], d["chain_id"], np.full(n_chains, 0.5), L,
                          base.spring_params, base.wca_params, base.active_params, 0.0, base.Dr, base.radius, -1,
                          s["n_grid_setup"], s["grid_factor"], nbor_depth=64)
    sysm.seed_mt(0)
    t = t_start = -settings.t_init_grow
    dt, steps, counter, built = settings.dt0, 0, 1, False
    n_upd = s["n_steps_update_grid_list"]
    while t <= 0:
        p, rest, active = grow_params(base, consts, t, t_start, settings)
        sysm.spring_params, sysm.WCA_params, sysm.active = p.spring_params, p.wca_params, p.active_params
        sysm.D, sysm.Dr, sysm.radius, sysm.rigid_rod = p.D, p.Dr, p.radius, p.rigid_rod
        sysm.n_nearby = p.n_nearby
        sysm.rest_lengths[:] = rest
        if not built:
            sysm.build_lists(grid_window=max(1, math.ceil(s["grid_factor"] * p.wca_params[3] / (L / s["n_grid_setup"]))))
            built = True
        res = sysm.run(settings.growing_stepskip, dt=dt, dtmax=p.dtmax, max_dist_per_step=p.max_dist_per_step,
                       rk_cheat=p.rk_cheat, steps_until_update=n_upd - counter, n_steps_update=n_upd,
                       calc_active=active)
        dt, t, steps = res["dt"], t + res["dt_used"], steps + res["steps"]
        counter = max(1, (res["steps"] + counter) % n_upd)
    return sysm, steps, t
