"""Host logic of several populations in one box: the cross parameters the
drop-in derives (interpop_forces, updates.py:274-312) and its refusals."""
from types import SimpleNamespace

import numpy as np
import pytest

from gliding_collective_rotation_b200 import updates
from gliding_collective_rotation_b200.engine import wca_params as make_WCA_params


def _pop(name, wca, growing=False, special=None, extra=()):
    return SimpleNamespace(name=name, b_init_growing=growing, special_interactions=special or {},
                           interactions=lambda other: [["WCA", 0.5 * (wca + other._wca)], *extra], _wca=wca)


def test_default_cross_parameters_are_the_mean():
    a = _pop("chains", make_WCA_params(1.0, 1.0, 0.0, 1.0))
    b = _pop("beads", make_WCA_params(0.7, 0.5, 0.0, 2.0))
    np.testing.assert_array_equal(updates._cross_wca(a, b), 0.5 * (a._wca + b._wca))
    np.testing.assert_array_equal(updates._cross_wca(b, a), updates._cross_wca(a, b))


def test_special_interaction_wins():
    """pop1.special_interactions[pop2.name] replaces interactions(pop2)."""
    special = np.array([3.0, 4.0, 0.0, 1.5])
    a = _pop("chains", make_WCA_params(1.0, 1.0, 0.0, 1.0), special={"beads": [["WCA", special]]})
    b = _pop("beads", make_WCA_params(0.7, 0.5, 0.0, 2.0))
    np.testing.assert_array_equal(updates._cross_wca(a, b), special)
    # not symmetric: b still takes the mean
    np.testing.assert_array_equal(updates._cross_wca(b, a), 0.5 * (a._wca + b._wca))


def test_growing_population_cuts_at_the_minimum():
    """repulsive_only while either population grows (updates.py:278, 304-310):
    r_cut = (p1 / p0)^(1/6)."""
    a = _pop("chains", make_WCA_params(1.0, 1.0, 0.0, 2.5 / 2 ** (1 / 6)), growing=True)
    b = _pop("beads", make_WCA_params(0.7, 0.5, 0.0, 2.5 / 2 ** (1 / 6)))
    w = updates._cross_wca(b, a)
    assert w[3] == pytest.approx((w[1] / w[0]) ** (1 / 6), rel=1e-15)
    assert w[3] < 0.5 * (a._wca[3] + b._wca[3])


def test_no_interaction_gives_zeros():
    a = SimpleNamespace(name="a", special_interactions={}, interactions=lambda other: [], b_init_growing=False)
    np.testing.assert_array_equal(updates._cross_wca(a, a), np.zeros(4))


def test_other_forces_between_populations_are_refused():
    a = _pop("chains", make_WCA_params(1.0, 1.0, 0.0, 1.0), extra=[["quadrupole_quadrupole", np.zeros(2)]])
    b = _pop("shells", make_WCA_params(1.0, 1.0, 0.0, 1.0))
    with pytest.raises(NotImplementedError, match="quadrupole_quadrupole"):
        updates._cross_wca(a, b)


def test_motor_push_is_no_pair_force():
    a = SimpleNamespace(name="chains", special_interactions={}, b_init_growing=False,
                        interactions=lambda other: [["motor_push", np.array([0.0625, 0, 1.0, 0.9, 0.2])]])
    b = SimpleNamespace(name="motors", special_interactions={}, b_init_growing=False, interactions=lambda o: [])
    np.testing.assert_array_equal(updates._cross_wca(a, b), np.zeros(4))


def test_motor_population_as_a_system(monkeypatch):
    """A Motor_Population maps to single diffusing beads with a zero-strength
    WCA whose cutoff is the chain-motor list radius: grid_window * Lx /
    n_grid with grid_window from the squared motor_max_dist (SRK.py:84-101)."""
    cfg = SimpleNamespace(Lx=60.0, n_grid=30, grid_factor=2.0, max_dist_per_step=0.0125, RK_cheat_factor=1.0,
                          dim=2)
    monkeypatch.setattr(updates, "_config", cfg)
    mot = SimpleNamespace(name="motors", total_pop=5, pos=np.zeros((5, 2)), D=0.1, Dr=0.3, fixed=False,
                          motor_max_dist_sq=0.0625, special_interactions={}, b_init_growing=False,
                          self_interactions=lambda: [["diffuse", np.array([1.0])]], where_active=np.zeros(5))
    status = SimpleNamespace(dtmax=1e-3, stepnum=7, b_calc_active_forces=True)
    prm = updates._pop_params(mot, status, {}, 3)
    assert updates._is_motors(mot)
    assert prm.wca_params.tolist() == [0.0, 0.0, 0.0, 2.0]
    assert prm.D == 0.1 and prm.Dr == 0.0 and not prm.calc_springs and not prm.self_propel and prm.calc_wca
    pos, tan, chain, rest = updates._pop_arrays(mot, 2)
    assert chain.tolist() == [0, 1, 2, 3, 4] and tan.shape == (5, 2) and rest.shape == (5,)
    # a wide motor reach widens the window: ceil(2 * 9 / 2) cells of 2
    assert updates._motor_list_radius(cfg, [9.0]) == 18.0
    # the list radius agrees with the workload's own derivation
    from gliding_collective_rotation_b200.workloads import motor_list_radius
    assert motor_list_radius(60.0, 1.0, 0.0625) == updates._motor_list_radius(cfg, [0.0625])
