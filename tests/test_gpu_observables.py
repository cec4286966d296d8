"""GPU observables against the reference's outputs and the CPU restatement:
chain frames, g(r), Cvv and Cnn over chain centres, on the reference's
relaxed config-1 state (tests/golden/observables.npz) and on a state after
200 GPU steps."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import observables as OBS  # noqa: E402
from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.engine import SystemParams  # noqa: E402
from oracle import observables as OB  # noqa: E402
from tests.golden_io import load  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _batch(precision):
    d, s = load("config1")
    prm = SystemParams(L=s["L"], spring_params=d["spring_params"], wca_params=d["wca_params"],
                       active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                       n_nearby=s["n_nearby"], dtmax=1e-3, seed=9)
    spec = W.SystemSpec("c1", 2, d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], prm, 1e-3, 0.0125)
    return Batch([spec], precision=precision), spec


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_observables_match_the_reference_outputs(precision):
    g = np.load(os.path.join(GOLDEN, "observables.npz"))
    b, spec = _batch(precision)
    eng, slot = b.engine, b.states[0].slot
    com, phi = OBS.chain_frames(eng, slot)
    tol = 1e-12 if precision == "fp64" else 1e-6  # FP32 tangents on the mixed path
    assert np.allclose(com, g["com"], rtol=0, atol=1e-11)
    assert np.allclose(phi[:, 0], g["phi1"], rtol=0, atol=tol)
    assert np.allclose(phi[:, 1], g["phi2"], rtol=0, atol=tol)
    gr = OBS.pair_correlation(eng, slot, "g_of_r", 0.25)
    assert gr.shape == g["g_of_r"].shape and np.allclose(gr, g["g_of_r"], rtol=1e-12, atol=1e-12)
    for kind, key in (("Cvv", "cvv"), ("Cnn", "cnn")):
        c = OBS.pair_correlation(eng, slot, kind, 0.25)
        assert np.allclose(c, g[key], rtol=0, atol=1e-8 if precision == "fp64" else 1e-5), key
    b.close()


def test_observables_after_steps_match_the_oracle():
    b, spec = _batch("fp64")
    b.begin(200)
    b.run(200)
    b.engine.synchronize()
    eng, st = b.engine, b.states[0]
    pos, tan = st.pos.cpu().numpy(), st.tangent.cpu().numpy()
    chain = np.asarray(spec.chain_id)
    cs = np.concatenate(([0], np.flatnonzero(np.diff(chain)) + 1, [len(chain)]))
    L = spec.params.L
    com, phi = OBS.chain_frames(eng, st.slot)
    want_com = OB.chain_com(pos, cs, L)
    assert np.allclose(com, want_com, rtol=0, atol=1e-11)
    p1, p2 = OB.avg_phi(tan, cs, 1), OB.avg_phi(tan, cs, 2)
    for kind, k in (("g_of_r", 0), ("Cvv", 1), ("Cnn", 2)):
        got = OBS.pair_correlation(eng, st.slot, kind, 0.5)
        want = OB.correlation(want_com, L, k, 0.5, p1, p2)
        assert got.shape == want.shape and np.allclose(got, want, rtol=1e-9, atol=1e-8), kind
    b.close()


def test_series_recorded_in_the_graph_equals_order_params():
    """The in-graph series (gcr_call.series) holds, bit for bit, what
    gcr_order_params returns at the same steps, and recording it does not
    change the trajectory."""
    import copy
    first, base = _batch("fp64")
    first.close()

    def fresh():
        b = Batch([copy.deepcopy(base)], "fp64")
        b.run_checked(5)
        return b

    b = fresh()
    step0 = b.statuses()[0]["step"]
    b.begin(100, series_every=25)
    b.run(100)
    rows = b.series()[0]
    assert rows.shape == (4, 5)
    assert list(rows[:, 0] - step0) == [25, 50, 75, 100]
    assert np.array_equal(rows[-1, 2:], b.engine.order_params(b.states[0].slot))
    pos_series = b.states[0].pos.cpu().numpy()
    b.close()
    c = fresh()
    c.begin(25)
    c.run(25)
    assert np.array_equal(rows[0, 2:], c.engine.order_params(c.states[0].slot))
    c.begin(75)
    c.run(75)
    assert np.array_equal(c.states[0].pos.cpu().numpy(), pos_series)
    c.close()
