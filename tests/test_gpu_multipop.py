"""Several populations in one box on the GPU (``gcr_couple``), against the
reference's own multi-population step (the trials of
``tests/golden/make_multipop_golden.py``; the reference does not reproduce
its own step exactly, so the GPU must land on one of its trials) and against
the oracle's multi-population step with the Philox noise."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import config, updates  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.engine import SystemParams  # noqa: E402
from gliding_collective_rotation_b200.workloads import SystemSpec  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.gpu_helpers import pop_from_arrays, status_from_row  # noqa: E402
from tests.multipop_helpers import CASES, load, oracle_group, pop_arrays  # noqa: E402


def _min_image(d, L):
    return d - L * np.round(d / L)


def _batch(d, s, precision="fp64", D=None, seeds=None, srk_order=2, list_depth=None, rigid=None):
    st0 = d["status_before"]
    specs = []
    for k in range(s["n_pops"]):
        a = pop_arrays(d, s, k)
        Dk = a["D"] if D is None or a["fixed"] else D
        params = SystemParams(L=s["L"], spring_params=a["spring"], wca_params=a["wca"], active_params=a["active"],
                              D=Dk, Dr=a["Dr"], radius=a["radius"], n_nearby=a["n_nearby"],
                              calc_springs=a["longest"] > 1, dtmax=st0[8], max_dist_per_step=s["max_dist_per_step"],
                              rk_cheat=s["rk_cheat"], seed=int(seeds[k]) if seeds is not None else 0,
                              rigid_rod=(rigid[k] if rigid is not None else 0.0))
        specs.append(SystemSpec(f"pop{k}", s["dim"], a["pos"], a["tangent"], a["chain_id"], a["rest_lengths"],
                                params, st0[8], s["max_dist_per_step"]))
    b = Batch(specs, precision=precision, srk_order=srk_order, list_depth=list_depth)
    b.couple(range(s["n_pops"]), s["fixed"], d["cross_wca"])
    return b


@pytest.mark.parametrize("name", CASES)
def test_one_step_lands_on_a_reference_trial(name):
    d, s = load(name)
    n, L = s["n_pops"], s["L"]
    st0 = d["status_before"]
    b = _batch(d, s)
    b.begin(1, dt=st0[0])
    b.run(1)
    sts = b.statuses()
    assert all(x["flags"] == 0 and x["steps_done"] == 1 for x in sts)
    gpu = [st.pos.cpu().numpy() for st in b.states]
    errs = [max(np.max(np.abs(_min_image(gpu[k] - d[f"trial{t}_p{k}_pos"], L))) for k in range(n))
            for t in range(int(d["trials"]))]
    best = int(np.argmin(errs))
    assert errs[best] < 1e-12, errs
    sa = d["status_after"][best]
    lead = s["fixed"].index(False)
    assert abs(sts[lead]["dt"] - sa[0]) <= 1e-12 * sa[0]
    assert abs(sts[lead]["max_forces_strength"] - sa[5]) <= 1e-10 * sa[5]
    for k in range(n):
        if s["fixed"][k]:
            np.testing.assert_array_equal(gpu[k], d[f"p{k}_pos0"])
        else:
            ref = d[f"trial{best}_p{k}_forces"]
            f = b.states[k].forces.cpu().numpy()
            assert np.max(np.abs(f - ref)) <= 1e-9 * max(1.0, np.max(np.abs(ref)))
    b.close()


def test_populations_write_one_state_file_each(tmp_path):
    from gliding_collective_rotation_b200 import state_io
    d, s = load("pops3_fixed_2d")
    b = _batch(d, s, D=0.01, seeds=[1, 2, 3])
    b.begin(3, dt=d["status_before"][0])
    b.run(3)
    files = state_io.save_populations(b, range(s["n_pops"]), s["names"], str(tmp_path / "run"), 7, 3, 0.003)
    for k, fn in enumerate(files):
        assert fn.endswith(f"run_{s['names'][k]}_00000007.dat")
        back = state_io.read_state(fn)
        np.testing.assert_allclose(back["pos"], b.states[k].pos.cpu().numpy(), rtol=1e-8, atol=0)
        assert back["stepnum"] == 3
    b.close()


@pytest.mark.parametrize("name", CASES)
def test_matches_the_oracle_with_noise(name):
    """T > 0 (D = 0.01 for the moving populations), the Philox stream with
    one seed per population: one step, then nine more."""
    d, s = load(name)
    n, L = s["n_pops"], s["L"]
    seeds = [101 + k for k in range(n)]
    st0 = d["status_before"]
    b = _batch(d, s, D=0.01, seeds=seeds)
    g = oracle_group(d, s, D=0.01, seeds=seeds)
    dt, step0 = st0[0], 0
    for n_steps, tol in ((1, 1e-12), (9, 1e-9)):
        b.begin(n_steps, dt=dt)
        b.run(n_steps)
        sts = b.statuses()
        assert all(x["flags"] == 0 and x["steps_done"] == n_steps for x in sts)
        res = g.run(n_steps, dt=dt, dtmax=st0[8], max_dist_per_step=s["max_dist_per_step"], rk_cheat=s["rk_cheat"],
                    noise_mode=O.NOISE_PHILOX, step0=step0)
        step0 += n_steps
        dt = res["dt"]
        lead = s["fixed"].index(False)
        assert abs(sts[lead]["dt"] - res["dt"]) <= 1e-9 * res["dt"]
        for k in range(n):
            err = np.max(np.abs(_min_image(b.states[k].pos.cpu().numpy() - g.systems[k].pos, L)))
            assert err < tol, (k, n_steps, err)
    b.close()


@pytest.mark.parametrize("name", CASES)
def test_mixed_precision_follows_fp64(name):
    d, s = load(name)
    L = s["L"]
    st0 = d["status_before"]
    out = {}
    for prec in ("fp64", "mixed"):
        b = _batch(d, s, precision=prec, D=0.01, seeds=[7, 8, 9])
        b.begin(1, dt=st0[0])
        b.run(1)
        assert all(x["flags"] == 0 for x in b.statuses())
        out[prec] = [st.pos.cpu().numpy() for st in b.states]
        b.close()
    for a, m in zip(out["fp64"], out["mixed"]):
        assert np.max(np.abs(_min_image(a - m, L))) < 1e-5


def test_decoupled_systems_step_alone():
    """After gcr_decouple every member steps exactly as it does uncoupled."""
    d, s = load("pops2_2d")
    st0 = d["status_before"]
    b = _batch(d, s, D=0.01, seeds=[3, 4])
    b.engine.decouple(b.states[0].slot)
    b.groups.clear()
    b.begin(5, dt=st0[0])
    b.run(5)
    single = Batch([b.specs[0]], precision="fp64")
    single.begin(5, dt=st0[0])
    single.run(5)
    np.testing.assert_array_equal(b.states[0].pos.cpu().numpy(), single.states[0].pos.cpu().numpy())
    for x in (b, single):
        x.close()


@pytest.mark.parametrize("name", CASES)
def test_srk4_coupled_matches_the_oracle(name):
    """The SRK4 branch (SRK.py:186-215, 296-321) with several populations:
    the cross forces enter every stage force."""
    d, s = load(name)
    n, L = s["n_pops"], s["L"]
    seeds = [31 + k for k in range(n)]
    st0 = d["status_before"]
    b = _batch(d, s, D=0.01, seeds=seeds, srk_order=4)
    g = oracle_group(d, s, D=0.01, seeds=seeds, srk_order=4)
    dt, step0 = st0[0], 0
    for n_steps, tol in ((1, 1e-12), (9, 1e-9)):
        b.begin(n_steps, dt=dt)
        b.run(n_steps)
        sts = b.statuses()
        assert all(x["flags"] == 0 and x["steps_done"] == n_steps for x in sts)
        res = g.run(n_steps, dt=dt, dtmax=st0[8], max_dist_per_step=s["max_dist_per_step"], rk_cheat=s["rk_cheat"],
                    noise_mode=O.NOISE_PHILOX, step0=step0, srk_order=4)
        step0 += n_steps
        dt = res["dt"]
        lead = s["fixed"].index(False)
        assert abs(sts[lead]["dt"] - res["dt"]) <= 1e-9 * res["dt"]
        for k in range(n):
            err = np.max(np.abs(_min_image(b.states[k].pos.cpu().numpy() - g.systems[k].pos, L)))
            assert err < tol, (k, n_steps, err)
            if not s["fixed"][k]:
                fa = b.states[k].forces_aux.cpu().numpy()
                assert np.max(np.abs(fa - g.systems[k].forces_aux)) <= 1e-8 * max(1.0, np.max(np.abs(fa)))
    b.close()


@pytest.mark.parametrize("name", ["pops2_2d", "pops3_fixed_2d"])
def test_drop_in_steps_a_list_of_populations(name):
    """updates.SRK2_force_calc(pops, status, sim) with the reference's
    population objects' interface: lands on a reference trial."""
    d, s = load(name)
    n, L = s["n_pops"], s["L"]
    config.dim, config.Lx = s["dim"], s["L"]
    config.SRK_order = 2
    config.n_steps_update_grid_list = s["n_steps_update"]
    config.max_dist_per_step = s["max_dist_per_step"]
    config.RK_cheat_factor = s["rk_cheat"]
    config.walls = np.array([False, False, False])
    pops = []
    for k in range(n):
        a = pop_arrays(d, s, k)
        p = pop_from_arrays(a["pos"], a["tangent"], a["chain_id"], a["rest_lengths"], a["spring"], a["wca"],
                            a["active"], a["D"], a["Dr"], a["radius"], a["n_nearby"])
        p.name, p.fixed = s["names"][k], bool(a["fixed"])
        p.interactions = (lambda kk: (lambda other: [["WCA", d["cross_wca"][kk, other._k]]]))(k)
        p._k = k
        pops.append(p)
    st = status_from_row(d["status_before"])
    st.next_output_step = st.stepnum + 1
    sim = {"gpu_precision": "fp64", "seed": 0}
    updates.SRK2_force_calc(pops, st, sim)
    errs = [max(np.max(np.abs(_min_image(pops[k].pos - d[f"trial{t}_p{k}_pos"], L))) for k in range(n))
            for t in range(int(d["trials"]))]
    assert min(errs) < 1e-12, errs
    best = int(np.argmin(errs))
    assert st.stepnum == int(d["status_before"][2]) + 1
    assert abs(st.dt - d["status_after"][best][0]) <= 1e-12 * st.dt
    assert abs(st.max_forces_strength - d["status_after"][best][5]) <= 1e-10 * st.max_forces_strength
    pops[0]._gcr_group.engine.close()


@pytest.mark.parametrize("name", ["pops2_2d", "pops3_fixed_2d"])
def test_a_member_overflow_stops_the_box(name):
    """Lists too short for one population: its overflow stops every
    population of the box before the real update, the batch regrows and
    re-runs the step for all of them, and the result is the run with deep
    enough lists from the start, bit for bit."""
    d, s = load(name)
    st0 = d["status_before"]
    b = _batch(d, s, D=0.01, seeds=[5, 6, 7], list_depth=4)
    b.begin(1, dt=st0[0])
    b.run(1)
    # the short lists overflow at the first build: no member took the step
    assert all(x["steps_done"] == 0 and x["flags"] & 16 for x in b.statuses())
    b.close()
    out = []
    for depth in (4, 128):
        b = _batch(d, s, D=0.01, seeds=[5, 6, 7], list_depth=depth)
        sts = b.run_checked(20)
        assert all(x["steps_done"] == 20 and x["flags"] == 0 for x in sts)
        out.append([st.pos.cpu().numpy() for st in b.states])
        b.close()
    for a, c in zip(*out):
        np.testing.assert_array_equal(a, c)


@pytest.mark.parametrize("name", ["pops2_2d", "pops2_3d"])
@pytest.mark.parametrize("srk_order", [2, 4])
def test_rigid_rods_among_populations_match_the_oracle(srk_order, name):
    """The chains blended towards rigid rods beside free beads: the
    projection uses each stage's force, cross forces included.  Factor 0.05:
    the relaxed chains are bent, and a larger factor snaps them onto their
    neighbours (forces of 1e4 to 1e6, dt down to 1e-8)."""
    d, s = load(name)
    n, L = s["n_pops"], s["L"]
    rigid = [0.05, 0.0]
    st0 = d["status_before"]
    b = _batch(d, s, D=0.01, seeds=[41, 42], srk_order=srk_order, rigid=rigid)
    g = oracle_group(d, s, D=0.01, seeds=[41, 42], srk_order=srk_order, rigid=rigid)
    dt, step0 = st0[0], 0
    for n_steps, tol in ((1, 1e-12), (9, 1e-9)):
        b.begin(n_steps, dt=dt)
        b.run(n_steps)
        assert all(x["flags"] == 0 and x["steps_done"] == n_steps for x in b.statuses())
        res = g.run(n_steps, dt=dt, dtmax=st0[8], max_dist_per_step=s["max_dist_per_step"], rk_cheat=s["rk_cheat"],
                    noise_mode=O.NOISE_PHILOX, step0=step0, srk_order=srk_order)
        step0 += n_steps
        dt = res["dt"]
        for k in range(n):
            err = np.max(np.abs(_min_image(b.states[k].pos.cpu().numpy() - g.systems[k].pos, L)))
            assert err < tol, (k, n_steps, err)
    b.close()
