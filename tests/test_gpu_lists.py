"""The Verlet neighbour lists on the GPU.

* The list of every bead is exactly the set of non-excluded beads within
  r_cut + skin of the positions it was built from (brute force on the CPU,
  same FP64 arithmetic), for the 2D and 3D kernels.
* Lists are in ascending partner id, so the skin changes only when lists
  are rebuilt, not the forces: trajectories with skin 0 (a rebuild every
  stage), 0.3 and 0.8 are bit-for-bit equal over 200 steps, in FP64 and in
  mixed precision.
* A list overflow stops the system cleanly and the regrown context
  (deeper lists) finishes the steps.
"""
import copy

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.engine import SystemParams, default_skin  # noqa: E402
from tests.golden_io import load, min_image  # noqa: E402


def _config1_spec(skin):
    d, s = load("config1")
    prm = SystemParams(L=s["L"], spring_params=d["spring_params"], wca_params=d["wca_params"],
                       active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                       n_nearby=s["n_nearby"], dtmax=1e-3, seed=5, skin=skin)
    return W.SystemSpec("config1", 2, d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], prm, 1e-3,
                        0.0125)


def _brute_force(xb, chain, L, rl, nn):
    """Per bead: the set of partners within rl (FP64, min image), without
    the same-chain neighbours |i - j| <= nn (the whole chain when nn < 0),
    and the set of pairs with r^2 within 2e-6 of rl^2 (the list radius
    carries a 1e-6 margin in r^2: either answer is right for those)."""
    n = len(xb)
    want, edge = [], []
    for i in range(n):
        d = min_image(xb - xb[i], L)
        ds = np.zeros(n)
        for k in range(xb.shape[1]):
            ds = ds + d[:, k] * d[:, k]
        same = chain == chain[i]
        excl = same & ((np.abs(np.arange(n) - i) <= nn) if nn >= 0 else True)
        excl[i] = True
        want.append(set(np.nonzero((ds <= rl * rl) & ~excl)[0].tolist()))
        edge.append(set(np.nonzero((np.abs(ds - rl * rl) <= 2e-6 * rl * rl) & ~excl)[0].tolist()))
    return want, edge


def _check_lists(b, spec):
    eng = b.engine
    st = b.states[0]
    counts, part, xb, total = eng.neighbour_list(st.slot)
    counts, part, xb = counts.cpu().numpy(), part.cpu().numpy(), xb.cpu().numpy()
    assert total == counts.sum() and counts.max() <= eng.cfg.list_depth
    p = spec.params
    rl = p.wca_params[3] + (p.skin if p.skin is not None else default_skin(p.wca_params[3]))
    want, edge = _brute_force(xb, np.asarray(spec.chain_id), p.L, rl, p.n_nearby)
    for i in range(len(xb)):
        got = part[i, :counts[i]].tolist()
        assert got == sorted(got) and len(got) == len(set(got)), i  # ascending, no partner twice
        assert set(got) ^ want[i] <= edge[i], (i, sorted(set(got) ^ want[i]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_list_is_every_pair_within_the_list_radius_2d(precision):
    spec = _config1_spec(0.3)
    b = Batch([spec], precision=precision)
    b.begin(57)
    b.run(57)
    b.engine.synchronize()
    assert b.statuses()[0]["flags"] == 0
    assert b.statuses()[0]["list_builds"] >= 1
    _check_lists(b, spec)
    b.close()


def test_list_is_every_pair_within_the_list_radius_3d():
    spec = W.config5(seed=1, scale=0.002)  # 80 chains x 25 beads in 3D
    b = Batch([spec], precision="mixed")
    b.relax(max_steps=400)
    b.begin(20)
    b.run(20)
    b.engine.synchronize()
    assert b.statuses()[0]["flags"] == 0
    _check_lists(b, spec)
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_skin_does_not_change_the_trajectory(precision):
    out = {}
    for skin in (0.0, 0.3, 0.8):
        b = Batch([_config1_spec(skin)], precision=precision)
        # two calls: the second starts from the lists the first left, which
        # must not matter either
        b.begin(120)
        b.run(120)
        b.begin(80)
        b.run(80)
        b.engine.synchronize()
        st = b.statuses()[0]
        assert st["flags"] == 0 and st["steps_done"] == 80
        out[skin] = (b.states[0].pos.cpu().numpy(), st["list_builds"])
        b.close()
    # skin 0 rebuilds at every stage that moved a bead; a wide skin rarely
    assert out[0.0][1] >= 300 and out[0.8][1] < out[0.3][1] < out[0.0][1] / 4
    for skin in (0.3, 0.8):
        assert np.array_equal(out[skin][0], out[0.0][0]), skin


def test_list_overflow_regrows():
    specs = sorted(W.config3(n_systems=256, param_seed=777), key=lambda s: s.n)[:3]
    specs = [copy.deepcopy(s) for s in specs]
    b = Batch(specs, precision="mixed", list_depth=4)
    b.relax(max_steps=400)
    sts = b.run_checked(30)
    assert all(st["steps_done"] == 30 for st in sts)
    assert not b.overflowed(sts)
    assert b.list_depth > 4
    b.close()
