"""The oracle's rigid-rod projection and init-grow steps against the reference.

``tests/golden/rigid_project.npz`` holds direct calls of the reference's
updates.project_updates_for_rigid_rod (updates.py:347-499) in 2D and 3D;
``tests/golden/initgrow.npz`` holds windows of the reference's own init-grow
loop (control.early_time_procedures + updates.SRK2_force_calc): the repel
phase (radius ramped from 4e-8, no projection) and the rigid phase
(projection factor 0.025), both from progress 0.1 on.  Both were made by
``tests/golden/make_initgrow_golden.py``.

The reference is compiled by Numba with fastmath, which may contract
products and sums into FMAs: single projections agree to a few ulp.
"""
import json
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden_io import GOLDEN, min_image, status_dict


def _proj():
    return np.load(f"{GOLDEN}/rigid_project.npz")


@pytest.mark.parametrize("dim", [2, 3])
def test_projection_matches_reference(dim):
    d = _proj()
    for k in range(int(d[f"d{dim}_n_calls"])):
        g = lambda nm: d[f"d{dim}_c{k}_{nm}"]  # noqa: E731
        pf, L, dt, D, r = g("scal")
        out = O.project_rigid(g("pos"), g("forces"), g("noise"), g("chain_id"), g("rest"), pf, L, dt, D, r)
        assert np.max(np.abs(min_image(out - g("out"), L))) <= 4e-15 * L, (dim, k)


def test_projection_factor_one_makes_a_rigid_rod():
    """Factor 1, no forces or noise: every chain lands on a straight rod of
    its rest length, centred where the chain was (the reference's target)."""
    d = _proj()
    pos, chain, rest = d["d2_c2_pos"], d["d2_c2_chain_id"], d["d2_c2_rest"]
    L = float(d["d2_c2_scal"][1])
    out = O.project_rigid(pos, np.zeros_like(pos), np.zeros((len(pos), 4)), chain, rest, 1.0, L, 1e-3, 0.0, 1.0)
    for c in np.unique(chain):
        x = out[chain == c]
        if len(x) < 2:
            continue
        bonds = min_image(np.diff(x, axis=0), L)
        assert np.allclose(np.linalg.norm(bonds, axis=1), rest[c], rtol=0, atol=1e-12)
        u = bonds / np.linalg.norm(bonds, axis=1)[:, None]
        assert np.allclose(u, u[0], atol=1e-12)


def _initgrow():
    d = np.load(f"{GOLDEN}/initgrow.npz")
    return d, json.loads(str(d["scalars"]))


def grid_window(s, cutoff):
    """SRK.py:99-101: cells the neighbour search spans."""
    return max(1, int(math.ceil(s["grid_factor"] * cutoff / (s["L"] / s["n_grid"]))))


def call_params(d, w, ci):
    return {k: d[f"{w}_p_{k}"][ci] for k in ("radius", "rigid", "D", "Dr", "n_nearby", "rk", "active_on", "mdps",
                                               "dtmax", "spring", "wca", "active", "rest")}


@pytest.mark.parametrize("window", ["repel", "rigid"])
def test_initgrow_calls_match_reference(window):
    d, s = _initgrow()
    p0 = call_params(d, window, 0)
    sysm = O.OracleSystem(d[f"{window}_pos0"], d[f"{window}_tangent0"], d["chain_id"], p0["rest"], s["L"],
                          p0["spring"], p0["wca"], p0["active"], p0["D"], p0["Dr"], p0["radius"],
                          int(p0["n_nearby"]), s["n_grid"], s["grid_factor"], nbor_depth=64,
                          rigid_rod=p0["rigid"])
    sysm.build_lists(grid_window=grid_window(s, p0["wca"][3]))
    # Dr > 0 draws rotational deviates (unused: the tangents follow the bonds)
    sysm.seed_mt(0)
    for ci in range(len(d[f"{window}_progress"])):
        p = call_params(d, window, ci)
        sysm.spring_params, sysm.WCA_params, sysm.active = p["spring"], p["wca"], p["active"]
        sysm.D, sysm.Dr, sysm.radius, sysm.rigid_rod = float(p["D"]), float(p["Dr"]), float(p["radius"]), \
            float(p["rigid"])
        sysm.n_nearby = int(p["n_nearby"])
        sysm.rest_lengths[:] = p["rest"]
        before = status_dict(d[f"{window}_status_before"][ci])
        after = status_dict(d[f"{window}_status_after"][ci])
        res = sysm.run(int(before["next_output_step"] - before["stepnum"]), dt=before["dt"], dtmax=before["dtmax"],
                       max_dist_per_step=float(p["mdps"]), rk_cheat=float(p["rk"]),
                       steps_until_update=int(s["n_steps_update"] - before["update_grid_list_counter"]),
                       n_steps_update=s["n_steps_update"], calc_active=bool(p["active_on"]))
        assert res["steps"] == after["stepnum"] - before["stepnum"]
        assert abs(res["dt"] - after["dt"]) <= 1e-9 * abs(after["dt"]), (window, ci)
        assert abs(res["dt_used"] - after["dt_used"]) <= 1e-9 * abs(after["dt_used"]), (window, ci)
        assert abs(res["max_forces_strength"] - after["max_forces_strength"]) <= \
            1e-7 * abs(after["max_forces_strength"]), (window, ci)
        err = np.max(np.abs(min_image(sysm.pos - d[f"{window}_pos"][ci], s["L"])))
        # bitwise in the repel window; ulp-level (fastmath) differences in the
        # projection grow to ~1e-9 over the 80 steps of the rigid window
        assert err <= (1e-12 if window == "repel" else 2e-9), (window, ci, err)
        assert np.max(np.abs(sysm.tangent_list - d[f"{window}_tangent"][ci])) <= 1e-6, (window, ci)
