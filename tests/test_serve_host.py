"""Host logic of the serving loop (admission, chunking, observation steps,
relaxation hand-over, overflow regrow), run on the CPU against a fake
engine that advances step counters instead of beads."""
import math

import numpy as np
import torch
import pytest

from gliding_collective_rotation_b200 import serve as S
from gliding_collective_rotation_b200 import workloads as W
from gliding_collective_rotation_b200._lib import FLAG_CELL_OVERFLOW


class FakeEngine:
    """Slots hold step counters; a relaxing system reaches the full dt after
    `relax_needed` steps; the first run with `overflow_at` systems resident
    stops one system half way with a cell overflow."""

    def __init__(self, bead_capacity, system_capacity, relax_needed=250, overflow_once=None):
        self.bead_capacity, self.system_capacity = bead_capacity, system_capacity
        self.relax_needed = relax_needed
        self.overflow_once = overflow_once
        self.sys = {}
        self.closed = False
        self.runs = []

    def try_admit(self, st):
        used = sum(v["st"].n for v in self.sys.values())
        if used + st.n > self.bead_capacity or len(self.sys) >= self.system_capacity:
            return None
        slot = min(set(range(self.system_capacity)) - set(self.sys))
        self.sys[slot] = dict(st=st, step=st.params.step, armed=0, done=0, relaxed=0, flags=0, dt=0.0)
        st.slot = slot
        return slot

    def admit(self, st):
        slot = self.try_admit(st)
        assert slot is not None
        return slot

    def evict(self, slot):
        self.sys.pop(slot)

    def update_params(self, st):
        assert st.slot in self.sys

    def call_begin_many(self, slots, max_steps, dts, series=None, series_every=0, series_phase=0):
        for i, (s, k, dt) in enumerate(zip(slots, max_steps, dts)):
            v = self.sys[s]
            every = int(series_every[i] if np.ndim(series_every) else series_every)
            phase = int(series_phase[i] if np.ndim(series_phase) else series_phase)
            # the device series: a row after each step j of the call with
            # (j + phase) % every == 0, in row i of `series`
            v.update(armed=int(k), done=0, flags=0, dt_call=dt, rows=0,
                     series=(series, i, every, phase) if series is not None and every > 0 else None)

    def run(self, n):
        self.runs.append(n)
        for s, v in self.sys.items():
            d = min(v["armed"], n)
            if self.overflow_once is not None and len(self.sys) >= self.overflow_once and d > 1:
                d //= 2
                v["flags"] = FLAG_CELL_OVERFLOW
                self.overflow_once = None
            if v.get("series") is not None:
                buf, row, every, phase = v["series"]
                for j in range(1, d + 1):
                    if (j + phase) % every == 0 and v["rows"] < buf.shape[1]:
                        step = v["step"] + j
                        buf[row, v["rows"]] = torch.tensor([step, 0.0, step * 1e-3, 0.5, 0.25], dtype=torch.float64)
                        v["rows"] += 1
            v["done"] = d
            v["step"] += d
            relaxing = math.isfinite(v["st"].params.max_dist_per_step)
            dtmax = v["st"].params.dtmax
            if relaxing:
                v["relaxed"] += d
                v["dt"] = dtmax if v["relaxed"] >= self.relax_needed else 0.1 * dtmax
            else:
                v["dt"] = dtmax
            v["armed"] = 0

    def status(self, slot):
        v = self.sys[slot]
        return {"dt": v["dt"], "dt_used": v["dt"], "max_forces_strength": 0.0, "steps_done": v["done"],
                "step": v["step"], "flags": v["flags"], "active": False, "series_rows": v.get("rows", 0)}

    def statuses(self, slots):
        return [self.status(s) for s in slots]

    def order_params(self, slot):
        return np.array([self.sys[slot]["step"] * 1e-3, 0.5, 0.25])

    def synchronize(self):
        pass

    def close(self):
        self.closed = True


class FakeServer(S.Server):
    def __init__(self, *a, relax_needed=250, overflow_once=None, **kw):
        self._fake_kw = dict(relax_needed=relax_needed, overflow_once=overflow_once)
        self.engines = []
        super().__init__(*a, device="cpu", **kw)

    def _make_engine(self):
        eng = FakeEngine(self.bead_capacity, self.max_systems, **self._fake_kw)
        self._fake_kw["overflow_once"] = None  # only the first engine overflows
        self.engines.append(eng)
        return eng


def _requests(n, steps, relax=False, obs_every=0, sizes=None, adaptive=True):
    out = []
    for i in range(n):
        nch = (sizes[i] if sizes else 20)
        spec = W.make_system(f"r{i}", 2, nch, 10, 40.0, seed=i)
        out.append(S.Request(i, spec, steps[i] if np.ndim(steps) else steps, 0.0, obs_every, relax, adaptive))
    return out


def test_every_request_runs_exactly_its_steps_with_observations():
    srv = FakeServer(hbm_budget=1 << 26, chunk=64)
    reqs = _requests(5, [100, 250, 64, 333, 1], obs_every=50)
    res = srv.serve(reqs, timeout=30)
    assert sorted(r.id for r in res) == list(range(5))
    for r in res:
        want = reqs[r.id].steps
        assert r.steps == want and r.flags == 0 and r.relax_steps == 0
        # an observation at every multiple of 50 of the request's steps, none
        # past the end, although calls of 64 steps cross them
        assert list(r.series[:, 0]) == list(range(50, want + 1, 50))
    assert max(srv.engines[0].runs) == 64


def test_relaxation_comes_first_and_is_counted_apart():
    srv = FakeServer(hbm_budget=1 << 26, chunk=100, relax_needed=250)
    reqs = _requests(2, 120, relax=True, adaptive=False)
    res = srv.serve(reqs, timeout=30)
    for r in res:
        assert r.relax_steps == 300  # three chunks of 100 until the dt is full
        assert r.steps == 120
    for rq in reqs:
        assert math.isinf(rq.spec.params.max_dist_per_step)  # handed over to the fixed dt


def test_adaptive_requests_keep_the_adaptive_rule_and_carry_dt():
    srv = FakeServer(hbm_budget=1 << 26, chunk=50)
    reqs = _requests(2, 120)
    res = srv.serve(reqs, timeout=30)
    assert all(r.steps == 120 and r.relax_steps == 0 for r in res)
    for rq in reqs:
        assert rq.spec.params.max_dist_per_step == rq.spec.relax_mdps


def test_admission_waits_for_room_and_backfills():
    # room for 400 beads: the 300-bead request must wait for the first to leave,
    # the 100-bead one may pass it
    srv = FakeServer(hbm_budget=1 << 20, chunk=50)
    srv.bead_capacity = 400
    srv.engine = srv._make_engine()
    reqs = _requests(3, [200, 50, 50], sizes=[30, 30, 10])
    res = srv.serve(reqs, timeout=30)
    by_id = {r.id: r for r in res}
    assert by_id[2].admitted <= by_id[1].admitted  # backfilled ahead of request 1
    assert by_id[1].admitted >= by_id[0].admitted
    assert all(r.steps == q.steps for r, q in zip(sorted(res, key=lambda r: r.id), reqs))


def test_overflow_regrows_and_keeps_step_counters():
    srv = FakeServer(hbm_budget=1 << 26, chunk=40, overflow_once=2)
    depth0 = srv.cell_depth
    reqs = _requests(3, 120)
    res = srv.serve(reqs, timeout=30)
    assert srv.cell_depth == 2 * depth0
    assert len(srv.engines) == 2 and srv.engines[0].closed
    for r in res:
        assert r.steps == 120 and r.flags == 0
    # the step counter (the noise key) carried over: params.step was set from the status
    assert all(q.spec.params.step > 0 for q in reqs if q.id in (r.id for r in res))


def test_summary():
    res = [S.Result(i, 1000, 100, 0.0, 0.0, 1.0 + i, 0, np.zeros((1, 2)), np.zeros((1, 2)), np.zeros((0, 4)), 0)
           for i in range(4)]
    s = S.summarize(res)
    assert s["requests"] == 4 and s["bead_steps"] == 4e5
    assert s["p50_s"] == pytest.approx(2.5) and s["bead_steps_per_s"] == pytest.approx(1e5)


def test_request_from_trace_shapes():
    tr = W.serve_trace(3, max_beads=5000)
    reqs = [S.request_from_trace(e, obs_every=100) for e in tr]
    for e, r in zip(tr, reqs):
        assert r.spec.n == e["n_chains"] * e["chain_length"] and r.steps == e["steps"]
        assert r.arrival == e["arrival"] and r.spec.params.seed == e["seed"]


def _corrupt_requests(first_id, arrival):
    """Requests the server must refuse, one fault each."""
    bad = []
    for k, fault in enumerate(["zero_beads", "negative_steps", "zero_steps", "chain_order", "chain_gap", "nan_pos",
                               "dim3", "huge"]):
        spec = W.make_system(f"bad{k}", 2, 20, 10, 40.0, seed=100 + k)
        steps = 50
        if fault == "zero_beads":
            spec.pos, spec.tangent, spec.chain_id = spec.pos[:0], spec.tangent[:0], spec.chain_id[:0]
        elif fault == "negative_steps":
            steps = -5
        elif fault == "zero_steps":
            steps = 0
        elif fault == "chain_order":
            spec.chain_id = spec.chain_id[::-1].copy()
        elif fault == "chain_gap":
            spec.chain_id = np.where(spec.chain_id >= 5, spec.chain_id + 1, spec.chain_id)
        elif fault == "nan_pos":
            spec.pos = spec.pos.copy()
            spec.pos[3, 1] = np.nan
        elif fault == "dim3":
            spec = W.make_system(f"bad{k}", 3, 20, 10, 40.0, seed=100 + k)
        elif fault == "huge":
            spec = W.make_system(f"bad{k}", 2, 2000, 10, 400.0, seed=100 + k)
        bad.append((fault, S.Request(first_id + k, spec, steps, arrival, 0, False, True)))
    return bad


def test_corrupt_requests_are_rejected_and_the_rest_run():
    srv = FakeServer(hbm_budget=1 << 20, chunk=40)
    srv.bead_capacity = 5000
    srv.engine = srv._make_engine()
    good = _requests(3, [120, 80, 100])
    bad = _corrupt_requests(10, arrival=0.0)
    res = srv.serve(good + [r for _, r in bad], timeout=30)
    assert sorted(r.id for r in res) == [0, 1, 2]
    assert all(r.steps == q.steps and r.flags == 0 for r, q in zip(sorted(res, key=lambda r: r.id), good))
    rejected = dict(srv.rejected)
    assert sorted(rejected) == [r.id for _, r in bad]
    reasons = {fault: rejected[r.id] for fault, r in bad}
    assert "n >= 1" in reasons["zero_beads"]
    assert "positive integer" in reasons["negative_steps"] and "positive integer" in reasons["zero_steps"]
    assert "chain ids" in reasons["chain_order"] and "chain ids" in reasons["chain_gap"]
    assert "non-finite" in reasons["nan_pos"]
    assert "dimension" in reasons["dim3"]
    assert "exceed" in reasons["huge"]


def test_check_request_accepts_the_trace():
    tr = W.serve_trace(5, max_beads=5000)
    for e in tr:
        assert S.check_request(S.request_from_trace(e), 2, 10_000) is None
