"""Batched and mixed-precision paths on the GPU.

* Systems advanced together in one context give bit-for-bit the results
  they give alone (per-system arithmetic does not depend on the batch).
* FP32 forces / FP64 positions stay within the stated error of the FP64 run
  of the same kernels over 1,000 steps.
* A cell-table overflow stops the system cleanly and the regrown context
  finishes the steps.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.engine import SystemParams  # noqa: E402
from tests.golden_io import load, min_image  # noqa: E402


def _small_sweep(k=6):
    specs = W.config3(n_systems=256, param_seed=777)
    specs = sorted(specs, key=lambda s: s.n)[:k]
    return specs


def _relaxed(specs, precision):
    b = Batch(specs, precision=precision)
    b.relax(max_steps=600)
    return b


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_equals_alone_bitwise(precision):
    specs = _small_sweep()
    # relax once, then give every run the same start
    b0 = _relaxed(specs, precision)
    pos0 = [st.pos.clone() for st in b0.states]
    tan0 = [st.tangent.clone() for st in b0.states]
    step0 = [s["step"] for s in b0.statuses()]
    b0.close()
    steps = 50

    def fresh(sel):
        sp = [specs[i] for i in sel]
        for i in sel:
            specs[i].params.step = step0[i]
        b = Batch(sp, precision=precision)
        for j, i in enumerate(sel):
            b.states[j].pos.copy_(pos0[i])
            b.states[j].tangent.copy_(tan0[i])
        torch.cuda.synchronize()
        b.begin(steps)
        b.run(steps)
        b.engine.synchronize()
        return b

    mix = fresh(list(range(len(specs))))
    # a parameter update of every resident system (as relax() makes) must not
    # disturb the batch: run on and compare with a fresh batch started from
    # the same state
    for st in mix.states:
        mix.engine.update_params(st)
    snap_pos = [st.pos.clone() for st in mix.states]
    snap_tan = [st.tangent.clone() for st in mix.states]
    snap_step = [s["step"] for s in mix.statuses()]
    mix.begin(steps)
    mix.run(steps)
    mix.engine.synchronize()
    for i in range(len(specs)):
        specs[i].params.step = snap_step[i]
    again = Batch(specs, precision=precision)
    for j in range(len(specs)):
        again.states[j].pos.copy_(snap_pos[j])
        again.states[j].tangent.copy_(snap_tan[j])
    torch.cuda.synchronize()
    again.begin(steps)
    again.run(steps)
    again.engine.synchronize()
    for j in range(len(specs)):
        assert torch.equal(again.states[j].pos, mix.states[j].pos), j
    assert not any(s["flags"] for s in mix.statuses())
    again.close()
    mix.close()
    mix = fresh(list(range(len(specs))))
    for i in range(len(specs)):
        alone = fresh([i])
        assert torch.equal(alone.states[0].pos, mix.states[i].pos), i
        assert torch.equal(alone.states[0].tangent, mix.states[i].tangent), i
        assert torch.equal(alone.states[0].forces, mix.states[i].forces), i
        alone.close()
    assert all(s["steps_done"] == steps for s in mix.statuses())
    mix.close()


def test_mixed_precision_error_vs_fp64():
    """FP32 forces and SRK arithmetic with FP64 positions vs the FP64 run of
    the same kernels, same Philox noise, config 1 (2,000 beads, WCA) from the
    reference's relaxed state, 1,000 steps."""
    d, s = load("config1")
    prm = lambda: SystemParams(L=s["L"], spring_params=d["spring_params"], wca_params=d["wca_params"],
                               active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                               n_nearby=s["n_nearby"], dtmax=1e-3, seed=3)
    out = {}
    for prec in ("fp64", "mixed"):
        spec = W.SystemSpec("config1", 2, d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], prm(),
                            1e-3, 0.0125)
        b = Batch([spec], precision=prec)
        b.begin(1000)
        b.run(1000)
        b.engine.synchronize()
        out[prec] = (b.states[0].pos.cpu().numpy(), b.statuses()[0])
        b.close()
    (p64, s64), (p32, s32) = out["fp64"], out["mixed"]
    assert s64["steps_done"] == s32["steps_done"] == 1000
    err = np.max(np.abs(min_image(p32 - p64, s["L"])))
    disp = np.sqrt(np.mean(min_image(p64 - d["pos0"], s["L"]) ** 2))
    # stated bound: max position error below 1e-5 of the box and 1e-3 of
    # the rms displacement over the 1,000 steps
    assert err / s["L"] < 1e-5, err
    assert err / disp < 1e-3, (err, disp)


def test_cell_overflow_regrows():
    specs = _small_sweep(3)
    b = Batch(specs, precision="mixed", cell_depth=8)
    b.relax(max_steps=400)
    sts = b.run_checked(30)
    assert all(st["steps_done"] == 30 for st in sts)
    assert not b.overflowed(sts)
    b.close()
