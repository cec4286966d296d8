"""The oracle's motor push against the reference's own ``calc_motor_push``.

``tests/golden/make_motor_golden.py`` ran ``forces.calc_motor_push``
(forces.py:248-283) twice on seeded synthetic states (2D, 2D with
``b_one_motor_per_bead``, 3D; some motors attached at the start) with Numba's
generator seeded; ``oracle.motor_push_mt`` restates the loop with the same
MT19937 stream and must reproduce every decision (both ``where_active``
arrays exactly) and the forces within a few ulp of the largest force (the
reference is compiled with fastmath, which may fuse its
``+= force * tangent``).  A second check pins the keyed draws that the group
step and the GPU use.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "motor_push.npz")
CASES = ["m2d", "m2d_one", "m3d"]


@pytest.mark.parametrize("case", CASES)
def test_oracle_motor_push_reproduces_the_reference(case):
    z = np.load(GOLD)
    g = {k[len(case) + 1:]: z[k] for k in z.files if k.startswith(case + "_")}
    forces_b = np.zeros_like(g["pos_b"])
    where_b, where_m = g["where_b"].copy(), g["where_m"].copy()
    mt = O.MT()
    O.lib().gcro_mt_seed(O.C.byref(mt), int(g["rng_seed"]))
    for call in range(2):
        O.lib().gcro_motor_push_mt(O._p(g["pos_b"]), len(g["pos_b"]), O._p(g["nbor"]), g["nbor"].shape[1],
                                   O._p(forces_b), O._p(where_b), O._p(g["tangent"]), float(g["L"]),
                                   O._p(g["pos_m"]), O._p(where_m), O._p(g["params"]), O.C.byref(mt),
                                   g["pos_b"].shape[1])
        np.testing.assert_array_equal(where_b, g[f"where_b{call}"])
        np.testing.assert_array_equal(where_m, g[f"where_m{call}"])
        scale = max(1.0, float(np.abs(g[f"forces{call}"]).max()))
        np.testing.assert_allclose(forces_b, g[f"forces{call}"], rtol=0, atol=1e-15 * scale)
    # the fixture exercises every branch: attachments, detachments, pushes
    assert (g["where_m1"] >= 0).sum() > 0 and (g["where_m0"] != g["where_m"]).sum() > 0
    assert np.abs(g["forces1"]).sum() > 0


def test_motor_push_mt_wrapper_matches_the_direct_call():
    z = np.load(GOLD)
    g = {k[4:]: z[k] for k in z.files if k.startswith("m2d_") and not k.startswith("m2d_one")}
    forces_b = np.zeros_like(g["pos_b"])
    where_b, where_m = g["where_b"].copy(), g["where_m"].copy()
    O.motor_push_mt(g["pos_b"], g["nbor"], forces_b, where_b, g["tangent"], float(g["L"]), g["pos_m"], where_m,
                    g["params"], int(g["rng_seed"]))
    np.testing.assert_array_equal(where_m, g["where_m0"])


def test_keyed_motor_draws_are_uniform_and_distinct():
    u = np.array([O.motor_uniforms(9, m, b, 123, s) for m in range(40) for b in range(25) for s in (0, 1)])
    assert u.shape == (2000, 2)
    assert np.all((u >= 0) & (u < 1))
    # mean and spread of U[0, 1): 2000 draws a column
    assert abs(u.mean() - 0.5) < 0.02 and abs(u.std() - np.sqrt(1 / 12)) < 0.02
    assert len(np.unique(u[:, 0])) == len(u)
    a, b = O.motor_uniforms(9, 1, 2, 123, 0), O.motor_uniforms(9, 1, 2, 123, 1)
    assert not np.array_equal(a, b)
    np.testing.assert_array_equal(O.motor_uniforms(9, 1, 2, 123, 0), a)
