"""Independent systems split over several contexts, each on its own stream
and queued in turn (the bench's timed and end-to-end arms for the sweep),
step exactly as they do together in one context: every system's trajectory
depends only on itself."""
import copy

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402


def _relaxed(n):
    """n small sweep systems after a relaxation under the adaptive dt, with
    their step counters (the noise stream goes on from there)."""
    specs = sorted(W.config3(n_systems=48, param_seed=9), key=lambda s: s.n)[:n]
    b = Batch(specs, "mixed")
    b.relax(max_steps=1500, adaptive_after=True)
    out = []
    for sp, st, status in zip(specs, b.states, b.statuses()):
        sp = copy.deepcopy(sp)
        sp.pos = st.pos.cpu().numpy().copy()
        sp.tangent = st.tangent.double().cpu().numpy().copy()
        sp.params.step = status["step"]
        out.append(sp)
    b.close()
    return out


def test_systems_split_over_contexts_step_as_in_one():
    specs = _relaxed(9)
    whole = Batch(copy.deepcopy(specs), "mixed")
    whole.set_adaptive(True)
    parts = [Batch(copy.deepcopy(specs[a:b]), "mixed") for a, b in ((0, 3), (3, 7), (7, 9))]
    for b in parts:
        b.set_adaptive(True)
    steps, calls = 40, 3
    for _ in range(calls):
        whole.begin(steps)
        whole.run(steps)
        # the parts queued in turn on their own streams
        for b in parts:
            with torch.cuda.stream(b.engine.stream):
                b.begin(steps)
                b.run(steps)
    torch.cuda.synchronize()
    got = [st for b in parts for st in b.statuses()]
    ref = whole.statuses()
    assert all(s["flags"] == 0 and s["steps_done"] == steps for s in got + ref)
    pos_parts = [st.pos.cpu().numpy() for b in parts for st in b.states]
    for k, st in enumerate(whole.states):
        np.testing.assert_array_equal(st.pos.cpu().numpy(), pos_parts[k], err_msg=f"system {k}")
    assert [s["dt"] for s in got] == [s["dt"] for s in ref]
    whole.close()
    for b in parts:
        b.close()


def test_programmatic_launch_changes_no_bit(monkeypatch):
    """The step kernels launched with and without programmatic dependent
    launch (GCR_PDL, read when a context is created) end on the same bits."""
    specs = _relaxed(4)
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("GCR_PDL", flag)
        b = Batch(copy.deepcopy(specs), "mixed")
        b.set_adaptive(True)
        b.begin(60)
        b.run(60)
        assert all(s["flags"] == 0 and s["steps_done"] == 60 for s in b.statuses())
        out.append([st.pos.cpu().numpy() for st in b.states])
        b.close()
    for a, c in zip(*out):
        np.testing.assert_array_equal(a, c)
