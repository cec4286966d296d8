"""Neighbour lists across calls, and a system that stops among others.

* A run start rebuilds only the lists that no longer cover their systems'
  positions: a run split into calls of a few steps gives bit for bit the
  trajectory, and the same number of list builds, as one call.
* Positions the host writes between calls are covered: chains moved by the
  host far beyond the skin give bit for bit what a fresh context started
  from the moved state gives.
* A non-finite position put into one system's host state before upload stops
  that system alone (GCR_FLAG_NONFINITE); every other system of the batch
  steps bit for bit as in a clean run.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200._lib import FLAG_NONFINITE  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402


def _specs(k=5, seed=321):
    specs = W.config3(n_systems=256, param_seed=seed)
    # the smallest systems, and one of about 20k beads
    order = sorted(specs, key=lambda s: s.n)
    return order[:k - 1] + [min(order, key=lambda s: abs(s.n - 20000))]


def _relaxed_state(specs, precision):
    b = Batch(specs, precision=precision)
    b.relax(max_steps=600, adaptive_after=True)
    sts = b.statuses()
    snap = dict(pos=[st.pos.clone() for st in b.states], tan=[st.tangent.clone() for st in b.states],
                step=[s["step"] for s in sts], dt=[s["dt"] for s in sts])
    b.close()
    return snap


def _batch_from(specs, snap, precision, pos=None):
    for i, sp in enumerate(specs):
        sp.params.step = snap["step"][i]
    b = Batch(specs, precision=precision)
    b.set_adaptive(True)
    for j, st in enumerate(b.states):
        st.pos.copy_(snap["pos"][j] if pos is None else pos[j])
        st.tangent.copy_(snap["tan"][j])
    torch.cuda.synchronize()
    return b


def _call(b, steps, dts=None):
    b.engine.call_begin_many([st.slot for st in b.states], steps, dts if dts is not None else 0.0)
    b.run(steps)
    b.engine.synchronize()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_chunked_calls_keep_lists(precision):
    specs = _specs()
    snap = _relaxed_state(specs, precision)
    one = _batch_from(specs, snap, precision)
    builds0 = [s["list_builds"] for s in one.statuses()]
    _call(one, 60, snap["dt"])
    many = _batch_from(specs, snap, precision)
    _call(many, 10, snap["dt"])
    for _ in range(5):
        _call(many, 10)
    s1, s6 = one.statuses(), many.statuses()
    for j in range(len(specs)):
        assert torch.equal(one.states[j].pos, many.states[j].pos), j
        assert torch.equal(one.states[j].tangent, many.states[j].tangent), j
        assert s1[j]["step"] == s6[j]["step"]
        assert s1[j]["flags"] == s6[j]["flags"] == 0
        # the admission build plus the skin-triggered ones, the same in both:
        # no call start rebuilt a list that still covered its system
        assert s1[j]["list_builds"] == s6[j]["list_builds"], (j, s1[j]["list_builds"], s6[j]["list_builds"])
        assert s1[j]["list_builds"] - builds0[j] < 2 * 60
    one.close()
    many.close()


def test_host_moved_positions_rebuild():
    precision = "mixed"
    specs = _specs()
    snap = _relaxed_state(specs, precision)
    b = _batch_from(specs, snap, precision)
    _call(b, 20, snap["dt"])
    sts = b.statuses()
    # the host moves every chain by its own random shift of 1.5 to 3 (far
    # beyond the skin) between calls; the tangents stay
    rs = np.random.default_rng(5)
    moved = []
    for st, sp in zip(b.states, specs):
        chain = sp.chain_id
        nc = int(chain.max()) + 1
        ang = rs.uniform(0, 2 * np.pi, nc)
        mag = rs.uniform(1.5, 3.0, nc)
        shift = np.stack([mag * np.cos(ang), mag * np.sin(ang)], axis=1)[chain]
        p = np.mod(st.pos.cpu().numpy() + shift, sp.params.L)
        moved.append(torch.from_numpy(p).to(st.pos.device))
    for st, p in zip(b.states, moved):
        st.pos.copy_(p)
    builds_before = [s["list_builds"] for s in sts]
    snap2 = dict(pos=moved, tan=[st.tangent.clone() for st in b.states], step=[s["step"] for s in sts],
                 dt=[s["dt"] for s in sts])
    torch.cuda.synchronize()
    _call(b, 30, snap2["dt"])
    fresh = _batch_from(specs, snap2, precision)
    _call(fresh, 30, snap2["dt"])
    after = b.statuses()
    for j in range(len(specs)):
        assert after[j]["list_builds"] > builds_before[j], j  # the run start flagged the moved system
        assert torch.equal(b.states[j].pos, fresh.states[j].pos), j
        assert torch.equal(b.states[j].forces, fresh.states[j].forces), j
    b.close()
    fresh.close()


@pytest.mark.parametrize("ids", [[1, 1, 2, 2, 3, 3], [0, 0, 2, 2, 3, 3], [0, 0, 1, 1, 2, 2]])
def test_admit_refuses_chain_ids_not_covering_every_chain(ids):
    """Chain ids must run 0, 1, ..., n_chains - 1 (here 4 chains) in
    contiguous ranges: a system whose first chain id is not 0, that skips a
    chain, or that ends before the last chain is refused at admission."""
    import dataclasses

    from gliding_collective_rotation_b200._lib import GcrError
    from gliding_collective_rotation_b200.engine import Engine, SystemState
    n = len(ids)
    params = dataclasses.replace(_specs(1)[0].params, L=20.0)
    pos = np.stack([np.arange(n) * 2.0 + 1.0, np.full(n, 5.0)], axis=1)
    with Engine(2, "fp64", bead_capacity=64, system_capacity=1, cell_capacity=4096) as eng:
        st = SystemState.from_host(pos, np.tile([1.0, 0.0], (n, 1)), np.array(ids), np.full(4, 0.5), params)
        with pytest.raises(GcrError) as e:
            eng.admit(st)
        assert e.value.code == -1 and "chain ids" in str(e.value)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_nonfinite_stops_one_system(precision):
    specs = _specs()
    snap = _relaxed_state(specs, precision)
    clean = _batch_from(specs, snap, precision)
    _call(clean, 40, snap["dt"])
    bad = 2
    pos = [p.clone() for p in snap["pos"]]
    host = pos[bad].cpu().numpy()
    host[7, 0] = np.nan  # a NaN in one system's host positions, uploaded with the rest
    pos[bad] = torch.from_numpy(host).to(pos[bad].device)
    hit = _batch_from(specs, snap, precision, pos=pos)
    _call(hit, 40, snap["dt"])
    sc, sh = clean.statuses(), hit.statuses()
    for j in range(len(specs)):
        if j == bad:
            # stopped in its first step: the flag keeps every kernel off it
            # until it is armed again
            assert sh[j]["flags"] & FLAG_NONFINITE, sh[j]
            assert sh[j]["steps_done"] == 0, sh[j]
        else:
            assert sh[j]["flags"] == 0, (j, sh[j])
            assert sh[j]["steps_done"] == sc[j]["steps_done"] == 40
            assert torch.equal(hit.states[j].pos, clean.states[j].pos), j
            assert torch.equal(hit.states[j].tangent, clean.states[j].tangent), j
    # re-armed with a finite state, the stopped system steps again
    hit.states[bad].pos.copy_(snap["pos"][bad])
    torch.cuda.synchronize()
    _call(hit, 5, snap["dt"])
    assert hit.statuses()[bad]["flags"] == 0 and hit.statuses()[bad]["steps_done"] == 5
    clean.close()
    hit.close()
