"""The init-grow schedule (control.early_time_procedures, control.py:153-219)
against the parameters the reference itself set before each recorded call
of its growth loop (``tests/golden/initgrow.npz``)."""
import json

import numpy as np
import pytest

from gliding_collective_rotation_b200.engine import SystemParams
from gliding_collective_rotation_b200.growth import GrowSettings, GrowthConstants, grow_params
from gliding_collective_rotation_b200.engine import wca_params as make_WCA_params
from tests.golden_io import GOLDEN, status_dict


def _base():
    # the grown system's own (physical) parameters: config-1 physics
    return SystemParams(L=40.0, spring_params=np.array([100.0, 20.0, 0.0, 0.0, 1.0, 0.1]),
                        wca_params=make_WCA_params(1.0, 1.0, 0.0, 1.0), active_params=np.array([1.0, 0.0, 0.0]),
                        D=0.01, Dr=0.0075, radius=1.0, n_nearby=4, dtmax=1e-3, max_dist_per_step=0.0125)


@pytest.mark.parametrize("window", ["repel", "rigid"])
def test_schedule_matches_reference(window):
    d = np.load(f"{GOLDEN}/initgrow.npz")
    s = json.loads(str(d["scalars"]))
    c = GrowthConstants(repel_d_max=1.0, WCA_epsilon=1.0, WCA_shift=0.0, LJ_cutoff_factor=1.0,
                        reference_rest_length=0.5, longest_chain_length=s["longest_chain_length"])
    settings = GrowSettings(t_init_grow=s["t_init_grow"], growing_stepskip=s["growing_stepskip"])
    for ci in range(len(d[f"{window}_progress"])):
        t = status_dict(d[f"{window}_status_before"][ci])["t"]
        p, rest, active = grow_params(_base(), c, t, s["t_start"], settings)
        assert p.radius == d[f"{window}_p_radius"][ci]
        assert p.rigid_rod == d[f"{window}_p_rigid"][ci]
        np.testing.assert_array_equal(p.spring_params, d[f"{window}_p_spring"][ci])
        wca = np.array(d[f"{window}_p_wca"][ci])
        wca[3] = (wca[1] / wca[0]) ** (1 / 6)  # updates.interpop_forces while growing
        np.testing.assert_array_equal(p.wca_params, wca)
        assert np.all(rest == d[f"{window}_p_rest"][ci])
        assert p.n_nearby == d[f"{window}_p_n_nearby"][ci]
        assert p.D == d[f"{window}_p_D"][ci] and p.Dr == d[f"{window}_p_Dr"][ci]
        assert p.rk_cheat == d[f"{window}_p_rk"][ci]
        assert active == bool(d[f"{window}_p_active_on"][ci]) and not p.self_propel


def test_schedule_phases():
    c = GrowthConstants(repel_d_max=1.0, WCA_epsilon=1.0, WCA_shift=0.1, LJ_cutoff_factor=1.0,
                        reference_rest_length=0.5, longest_chain_length=10, rigid_rod_projection_factor=0.5)
    st = GrowSettings()
    p, rest, _ = grow_params(_base(), c, -0.9, -1.0, st)      # progress 0.1: repel ramp
    assert p.rigid_rod == 0 and abs(p.radius - 0.4) < 1e-12 and p.spring_params[1] == 0
    p, rest, _ = grow_params(_base(), c, -0.5, -1.0, st)      # progress 0.5: rigid phase
    assert p.rigid_rod == 0.5 and p.radius == 1.0 and p.spring_params[1] == 10
    assert p.wca_params[2] == 0.0                            # WCA_shift is 0 while growing
    p, rest, _ = grow_params(_base(), c, 0.0, -1.0, st)       # progress 1
    assert p.rigid_rod == 0.0 and p.spring_params[0] == 100.0 and p.spring_params[1] == 20.0
    assert abs(rest - 0.5) < 1e-15
    single = GrowthConstants(1.0, 1.0, 0.0, 1.0, 0.5, longest_chain_length=1, rigid_rod_projection_factor=0.3)
    p, _, _ = grow_params(_base(), single, -0.9, -1.0, st)
    assert p.radius == 1.0 and p.rigid_rod == 0.3
