"""The rotation-rate estimator of the product against the reference's
notebook functions' outputs (tests/golden/observables.npz)."""
import os

import numpy as np

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
