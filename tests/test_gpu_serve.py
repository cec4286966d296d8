"""The serving loop on the GPU: a request served in a mix of others, split
into chunks at other requests' pace (its adaptive dt carried from chunk to
chunk), ends bit-for-bit where it ends when run alone in one call; its
order-parameter series ends at the alone value."""
import copy

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import serve as S  # noqa: E402
from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402


def _relaxed(n):
    """n small sweep systems, relaxed once under the adaptive dt, which
    they keep (the rule a request's steps follow)."""
    specs = sorted(W.config3(n_systems=64, param_seed=5), key=lambda s: s.n)[:n]
    b = Batch(specs, "mixed")
    b.relax(max_steps=2000, adaptive_after=True)
    out = []
    for sp, st, status in zip(specs, b.states, b.statuses()):
        sp = copy.deepcopy(sp)
        sp.pos = st.pos.cpu().numpy().copy()
        sp.tangent = st.tangent.double().cpu().numpy().copy()
        sp.params.step = status["step"]
        out.append(sp)
    b.engine.close()
    return out


def _alone(spec, steps):
    b = Batch([copy.deepcopy(spec)], "mixed")
    b.begin(steps)
    b.run(steps)
    st = b.statuses()[0]
    assert st["flags"] == 0 and st["steps_done"] == steps
    pos = b.states[0].pos.cpu().numpy()
    op = b.engine.order_params(b.states[0].slot)
    b.engine.close()
    return pos, op


def test_served_in_a_mix_equals_alone():
    specs = _relaxed(4)
    steps = [150, 90, 200, 61]
    reqs = [S.Request(i, copy.deepcopy(sp), steps[i], 0.0, 30 if i == 0 else 0, relax=False)
            for i, sp in enumerate(specs)]
    srv = S.Server(2, "mixed", hbm_budget=1 << 30, chunk=37)
    res = {r.id: r for r in srv.serve(reqs, timeout=300)}
    srv.close()
    for i, sp in enumerate(specs):
        r = res[i]
        assert r.flags == 0 and r.steps == steps[i]
        pos, op = _alone(sp, steps[i])
        assert np.array_equal(r.pos, pos), i
        if i == 0:
            assert list(r.series[:, 0]) == [30, 60, 90, 120, 150]
            assert np.allclose(r.series[-1, 1:], op, rtol=0, atol=1e-12)


def test_corrupt_requests_leave_the_mix_untouched():
    """Requests with zero beads, negative steps, chain ids out of order or a
    NaN position arrive while three valid ones are resident: each is
    rejected with its reason, and the valid ones end bit for bit where they
    end alone."""
    specs = _relaxed(3)
    steps = [400, 300, 350]
    good = [S.Request(i, copy.deepcopy(sp), steps[i], 0.0, 0, relax=False) for i, sp in enumerate(specs)]
    bad = []
    for k, fault in enumerate(["zero_beads", "negative_steps", "chain_order", "nan_pos"]):
        sp = copy.deepcopy(specs[k % 3])
        n_steps = 50
        if fault == "zero_beads":
            sp.pos, sp.tangent, sp.chain_id = sp.pos[:0], sp.tangent[:0], sp.chain_id[:0]
        elif fault == "negative_steps":
            n_steps = -1
        elif fault == "chain_order":
            sp.chain_id = sp.chain_id[::-1].copy()
        else:
            sp.pos = sp.pos.copy()
            sp.pos[0, 0] = np.nan
        # they arrive once the valid requests are on the device
        bad.append(S.Request(10 + k, sp, n_steps, 0.02 * (k + 1), 0, relax=False))
    srv = S.Server(2, "mixed", hbm_budget=1 << 30, chunk=25)
    res = {r.id: r for r in srv.serve(good + bad, timeout=300)}
    rejected = dict(srv.rejected)
    srv.close()
    assert sorted(res) == [0, 1, 2]
    assert sorted(rejected) == [10, 11, 12, 13]
    for i, sp in enumerate(specs):
        r = res[i]
        assert r.flags == 0 and r.steps == steps[i]
        pos, _ = _alone(sp, steps[i])
        assert np.array_equal(r.pos, pos), i


def test_fresh_requests_relax_then_run():
    tr = W.serve_trace(3, rate=1000.0, max_beads=4000, min_steps=50, max_steps=120, seed=3)
    reqs = [S.request_from_trace(e, relax=True, obs_every=25) for e in tr]
    srv = S.Server(2, "mixed", hbm_budget=1 << 30, chunk=100)
    res = srv.serve(reqs, timeout=300)
    srv.close()
    assert len(res) == 3
    for r in res:
        assert r.flags == 0 and r.relax_steps > 0
        assert r.steps == reqs[r.id].steps
        assert np.all(np.isfinite(r.pos))
        assert r.series.shape[0] == r.steps // 25
    s = S.summarize(res)
    assert s["failed"] == 0 and s["p99_s"] >= s["p50_s"] > 0
