"""The rotation-rate estimator of the product against the reference's
notebook functions' outputs (tests/golden/observables.npz)."""
import os

import numpy as np
import pytest

from gliding_collective_rotation_b200 import observables as OBS

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_rotation_rate_matches_the_reference():
    g = np.load(os.path.join(GOLDEN, "observables.npz"))
    t, angle, omega = OBS.rotation_rate(g["series"])
    assert np.allclose(t, g["rot_time"], rtol=0, atol=0) and np.allclose(angle, g["rot_angle"], rtol=0, atol=0)
    assert np.allclose(omega, g["rot_omega"], rtol=1e-13, atol=1e-13)
    ct, co = OBS.remove_outliers(omega, t)
    assert np.array_equal(ct, g["rot_clean_time"]) and np.allclose(co, g["rot_clean_omega"], rtol=1e-13, atol=1e-13)


def test_rotation_rate_needs_an_ordered_state():
    s = np.zeros((20, 4))
    s[:, 0] = np.arange(20)
    s[:, 2] = 0.3
    assert OBS.rotation_rate(s) is None


@pytest.mark.parametrize("key", ["k30", "k100", "k300"])
def test_rotation_rate_of_the_papers_own_runs(key):
    """The paper's chiral runs (kappa 30, 100, 300; Data.zip of the paper's
    figures), through the notebook's estimator and through this one: the
    same rates, outliers and mean (the chirality reverses between kappa 100
    and 300)."""
    g = np.load(os.path.join(GOLDEN, "paper_rotation.npz"))
    t, angle, omega = OBS.rotation_rate(g[f"{key}_series"])
    assert np.allclose(t, g[f"{key}_time"], rtol=1e-14, atol=0)
    assert np.array_equal(angle, g[f"{key}_angle"])
    assert np.allclose(omega, g[f"{key}_omega"], rtol=1e-12, atol=1e-15)
    ct, co = OBS.remove_outliers(omega, t)
    assert np.array_equal(ct, np.asarray(g[f"{key}_clean_time"]))
    assert abs(co.mean() - float(g[f"{key}_mean_omega"])) <= 1e-12 * abs(float(g[f"{key}_mean_omega"]))
