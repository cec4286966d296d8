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
    a = _pop("chains", make_WCA_params(1.0, 1.0, 0.0, 1.0), extra=[["motor_push", np.zeros(5)]])
    b = _pop("motors", make_WCA_params(1.0, 1.0, 0.0, 1.0))
    with pytest.raises(NotImplementedError, match="motor_push"):
        updates._cross_wca(a, b)
