"""The CPU restatement of the reference's observables against the
reference's own outputs (tests/golden/observables.npz)."""
import json
import os

import numpy as np

from oracle import observables as OB

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _state():
    d = np.load(os.path.join(GOLDEN, "config1.npz"))
    s = json.loads(str(d["scalars"]))
    chain = np.asarray(d["chain_id"])
    cs = np.concatenate(([0], np.flatnonzero(np.diff(chain)) + 1, [len(chain)]))
    return d["pos0"], d["tangent0"], cs, float(s["L"])


def test_chain_frames_match_the_reference():
    g = np.load(os.path.join(GOLDEN, "observables.npz"))
    pos, tan, cs, L = _state()
    assert np.allclose(OB.chain_com(pos, cs, L), g["com"], rtol=0, atol=1e-12)
    assert np.allclose(OB.avg_phi(tan, cs, 1), g["phi1"], rtol=0, atol=1e-13)
    assert np.allclose(OB.avg_phi(tan, cs, 2), g["phi2"], rtol=0, atol=1e-13)


def test_pair_correlations_match_the_reference():
    g = np.load(os.path.join(GOLDEN, "observables.npz"))
    pos, tan, cs, L = _state()
    com = OB.chain_com(pos, cs, L)
    phi1, phi2 = OB.avg_phi(tan, cs, 1), OB.avg_phi(tan, cs, 2)
    for kind, key in ((0, "g_of_r"), (1, "cvv"), (2, "cnn")):
        got = OB.correlation(com, L, kind, 0.25, phi1, phi2)
        want = g[key]
        assert got.shape == want.shape, key
        assert np.array_equal(got[:, 0], want[:, 0]), key
        assert np.allclose(got[:, 1], want[:, 1], rtol=1e-12, atol=1e-12), key


def test_rotation_rate_matches_the_reference():
    g = np.load(os.path.join(GOLDEN, "observables.npz"))
    t, angle, omega = OB.rotation_rate(g["series"])
    assert np.allclose(t, g["rot_time"]) and np.allclose(angle, g["rot_angle"])
    assert np.allclose(omega, g["rot_omega"], rtol=1e-12, atol=1e-12)
    ct, co = OB.remove_outliers(omega, t)
    assert np.allclose(ct, g["rot_clean_time"]) and np.allclose(co, g["rot_clean_omega"], rtol=1e-12)
