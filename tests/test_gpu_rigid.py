"""Rigid-rod projection and the init-grow protocol on the GPU.

* The drop-in replays the reference's own init-grow calls
  (``tests/golden/initgrow.npz``: the repel phase and the rigid phase with
  projection factor 0.025), parameters changing between calls as
  control.early_time_procedures changes them.
* A growing population steps in FP64 whatever precision is asked for.
* ``growth.init_grow`` grows the reference's config-1 placement and a 3D
  placement into states with the statistics of the reference's own grown
  states.
* Rigid rods (factor 1) with noise stay rods; a batch holding a rigid
  system steps every system as it steps alone, bit for bit, before and after
  the projection is switched off (the graph is re-captured without it).
* ``gcr_update_desc`` keeps or re-derives the cell grid when the cutoff or
  skin changes; the pair sum does not depend on the grid, so the results
  equal those of a context admitted with the new parameters.
"""
import copy
import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import config, updates  # noqa: E402
from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200._lib import GcrError  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.engine import SystemParams  # noqa: E402
from gliding_collective_rotation_b200.growth import init_grow  # noqa: E402
from gliding_collective_rotation_b200.workloads import SystemSpec  # noqa: E402
from tests.golden_io import GOLDEN, load, min_image, status_dict  # noqa: E402
from tests.gpu_helpers import pop_from_arrays, set_pop_params, status_from_row  # noqa: E402
from tests.grow_helpers import check_like_reference, growth_case, grown_stats  # noqa: E402


def _initgrow():
    d = np.load(f"{GOLDEN}/initgrow.npz")
    return d, json.loads(str(d["scalars"]))


def _params(d, w, ci):
    return {k: d[f"{w}_p_{k}"][ci] for k in ("radius", "rigid", "D", "Dr", "n_nearby", "rk", "active_on", "mdps",
                                               "dtmax", "spring", "wca", "active", "rest")}


def _replay_growth(window, precision):
    d, s = _initgrow()
    config.dim, config.Lx, config.SRK_order = int(s["dim"]), float(s["L"]), 2
    config.n_steps_update_grid_list = int(s["n_steps_update"])
    config.grid_factor = float(s["grid_factor"])
    config.walls = np.array([False, False, False])
    p0 = _params(d, window, 0)
    pop = pop_from_arrays(d[f"{window}_pos0"], d[f"{window}_tangent0"], d["chain_id"], p0["rest"], p0["spring"],
                          p0["wca"], p0["active"], p0["D"], p0["Dr"], p0["radius"], int(p0["n_nearby"]))
    sim = {"gpu_precision": precision, "gpu_noise": "mt", "seed": 0}
    st = status_from_row(d[f"{window}_status_before"][0])
    out = []
    for ci in range(len(d[f"{window}_progress"])):
        p = _params(d, window, ci)
        set_pop_params(pop, p["spring"], p["wca"], p["active"], p["D"], p["Dr"], p["radius"], p["n_nearby"],
                       p["rest"], p["rigid"], growing=True)
        config.max_dist_per_step, config.RK_cheat_factor = float(p["mdps"]), float(p["rk"])
        st.b_calc_active_forces = bool(p["active_on"])
        st.next_output_step = st.stepnum + 10
        updates.SRK2_force_calc([pop], st, sim)
        out.append((dict(st.__dict__), pop.pos.copy(), pop.tangent_list.copy()))
    return d, s, out


@pytest.mark.parametrize("window", ["repel", "rigid"])
def test_drop_in_replays_reference_growth(window):
    d, s, out = _replay_growth(window, "fp64")
    for ci, (st, pos, tan) in enumerate(out):
        after = status_dict(d[f"{window}_status_after"][ci])
        assert st["stepnum"] == int(after["stepnum"])
        assert abs(st["dt"] - after["dt"]) <= 1e-7 * abs(after["dt"]), (window, ci)
        assert abs(st["dt_used"] - after["dt_used"]) <= 1e-7 * abs(after["dt_used"]), (window, ci)
        assert abs(st["max_forces_strength"] - after["max_forces_strength"]) <= \
            1e-6 * abs(after["max_forces_strength"]), (window, ci)
        err = np.max(np.abs(min_image(pos - d[f"{window}_pos"][ci], s["L"])))
        # the oracle meets 1e-12 (repel) and 2e-9 (rigid) on these calls
        assert err <= (1e-9 if window == "repel" else 5e-9), (window, ci, err)
        assert np.max(np.abs(tan - d[f"{window}_tangent"][ci])) <= 1e-6


def test_growing_population_steps_in_fp64():
    _, _, a = _replay_growth("repel", "fp64")
    _, _, b = _replay_growth("repel", "mixed")
    for (sa, pa, ta), (sb, pb, tb) in zip(a, b):
        assert np.array_equal(pa, pb) and np.array_equal(ta, tb)
        assert sa["dt"] == sb["dt"]


@pytest.mark.parametrize("name", ["config1", "grow3d"])
def test_init_grow_on_device_matches_reference_statistics(name):
    d, s, base, consts, settings = growth_case(name)
    n_chains = len(d["rest_lengths"])
    spec = SystemSpec(name, int(s["dim"]), np.array(d["init_pos"]), np.array(d["init_tangent"]),
                      np.array(d["chain_id"]), np.full(n_chains, 0.5), copy.deepcopy(base), base.dtmax,
                      base.max_dist_per_step)
    res = init_grow([spec], settings, constants=[consts])
    ref = grown_stats(d["pos0"], d["chain_id"], s["L"])
    got = grown_stats(res.specs[0].pos, d["chain_id"], s["L"])
    check_like_reference(got, ref, int(res.steps[0]), s["init_grow_steps"], float(res.t[0]))
    assert res.specs[0].params.step == res.steps[0]
    # the grown spec steps on at mixed precision with its physical parameters
    b = Batch(res.specs, precision="mixed")
    b.begin(200, dt=float(res.dt[0]))
    b.run(200)
    sts = b.statuses()
    assert sts[0]["steps_done"] == 200 and sts[0]["flags"] == 0
    b.close()


def _rigid_spec(name="rigid2d"):
    """The reference's grown rigid-rod state and parameters (factor 1),
    stepped with the Philox stream under the reference's adaptive dt."""
    d, s = load(name)
    p = SystemParams(L=s["L"], spring_params=np.array(d["spring_params"]), wca_params=np.array(d["wca_params"]),
                     active_params=np.array(d["active_params"]), D=s["D"], Dr=s["Dr"], radius=s["radius"],
                     n_nearby=s["n_nearby"], dtmax=s["dtmax"], max_dist_per_step=s["max_dist_per_step"], seed=5,
                     rigid_rod=s["rigid_rod"])
    return SystemSpec(name, int(s["dim"]), np.array(d["pos0"]), np.array(d["tangent0"]), np.array(d["chain_id"]),
                      np.array(d["rest_lengths"]), p, s["dtmax"], s["max_dist_per_step"])


@pytest.mark.parametrize("name", ["rigid2d", "rigid3d"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rigid_rods_stay_rods(name, precision):
    spec = _rigid_spec(name)
    b = Batch([spec], precision=precision)
    b.begin(300, dt=spec.params.dtmax)
    b.run(300)
    st = b.statuses()[0]
    assert st["steps_done"] == 300 and st["flags"] == 0
    pos = b.states[0].pos.cpu().numpy()
    L = spec.params.L
    chain = spec.chain_id
    bonds = min_image(np.diff(pos, axis=0), L)[np.diff(chain) == 0]
    bl = np.linalg.norm(bonds, axis=1)
    # 3D: the projection puts every bead back on a rod of the rest length;
    # 2D: its per-component torque stretches bonds at first order in the
    # rotation (the reference's own runs show ~5e-4 at dt 1e-3)
    tol = 2e-3 if spec.dim == 2 else 1e-11
    assert np.max(np.abs(bl - spec.rest_lengths[0])) <= tol, np.max(np.abs(bl - spec.rest_lengths[0]))
    # the beads moved (noise and propulsion act on the rods)
    assert np.max(np.abs(min_image(pos - spec.pos, L))) > 1e-3
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_with_rigid_system_equals_alone(precision):
    rigid = _rigid_spec("rigid2d")
    plain = W.make_system("plain", 2, 40, 8, 30.0, seed=3)
    plain.params.max_dist_per_step = plain.relax_mdps

    def run(specs, steps, switch_off=False):
        b = Batch(copy.deepcopy(specs), precision=precision)
        b.begin(steps, dt=1e-4)
        b.run(steps)
        if switch_off:
            for st in b.states:
                st.params.rigid_rod = 0.0
                b.engine.update_params(st)
            b.begin(steps)
            b.run(steps)
        b.engine.synchronize()
        out = [(st.pos.cpu().numpy(), st.tangent.cpu().numpy()) for st in b.states]
        b.close()
        return out

    for switch in (False, True):
        both = run([rigid, plain], 40, switch)
        alone = [run([rigid], 40, switch)[0], run([plain], 40, switch)[0]]
        for (pa, ta), (pb, tb) in zip(both, alone):
            assert np.array_equal(pa, pb) and np.array_equal(ta, tb)


def test_update_desc_regrids_within_reserved_cells():
    base = W.make_system("plain", 2, 60, 10, 40.0, seed=11)
    base.params.max_dist_per_step = base.relax_mdps
    b = Batch([copy.deepcopy(base)], precision="fp64")
    b.relax(max_steps=400, adaptive_after=True)
    pos, tan = b.states[0].pos.clone(), b.states[0].tangent.clone()
    step = b.statuses()[0]["step"]
    b.close()

    def fresh(skin, start_skin=None):
        spec = copy.deepcopy(base)
        spec.params.step = step
        spec.params.skin = start_skin if start_skin is not None else skin
        b = Batch([spec], precision="fp64")
        b.states[0].pos.copy_(pos)
        b.states[0].tangent.copy_(tan)
        if start_skin is not None:
            b.states[0].params.skin = skin
            b.engine.update_params(b.states[0])
        b.begin(60, dt=1e-3)
        b.run(60)
        st = b.statuses()[0]
        assert st["steps_done"] == 60 and st["flags"] == 0, st
        out = b.states[0].pos.cpu().numpy()
        b.close()
        return out

    # a smaller cutoff keeps the (coarser) grid; a grid beyond the cells
    # reserved at admission -- pair forces switched on for a system admitted
    # without them -- is refused (the caller re-admits; the drop-in does so by
    # itself)
    spec = copy.deepcopy(base)
    b = Batch([spec], precision="fp64")
    st = b.states[0]
    st.params.wca_params = np.array(st.params.wca_params)
    st.params.wca_params[3] = 0.3
    b.engine.update_params(st)
    b.close()
    spec = copy.deepcopy(base)
    spec.params.calc_wca = False
    b = Batch([spec], precision="fp64")
    st = b.states[0]
    st.params.calc_wca = True
    with pytest.raises(GcrError) as err:
        b.engine.update_params(st)
    assert err.value.code == -6
    b.close()
    # a smaller skin keeps the grid; a larger one takes fewer, larger cells
    for start, new in ((0.3, 0.1), (0.3, 0.9)):
        a, b = fresh(new, start_skin=start), fresh(new)
        assert np.array_equal(a, b)
        assert np.max(np.abs(a - pos.cpu().numpy())) > 1e-6  # the steps ran
