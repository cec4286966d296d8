"""The CUDA path against the reference's own trajectories and the oracle.

Trajectories: the drop-in ``SRK2_force_calc`` (FP64, the reference's MT19937
noise stream injected) replays every golden call sequence and must land on
the reference's positions within the tolerances the oracle itself meets
(``tests/golden_io.TRAJ_TOL``).  Lists: the device builders reproduce the
reference's where_is_bead, grid_list and nbor_list arrays exactly.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import updates  # noqa: E402
from gliding_collective_rotation_b200.engine import Engine, SystemParams, SystemState, philox_noise  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden_io import CASES, TRAJ_TOL, load, min_image, pairs_from_nbor  # noqa: E402
from tests.gpu_helpers import pop_from_golden, set_config, status_from_row  # noqa: E402


def _replay(name, precision="fp64"):
    d, s = load(name)
    set_config(s)
    pop = pop_from_golden(d, s)
    sim = {"gpu_precision": precision, "gpu_noise": "mt", "seed": int(s["noise_seed"]),
           "save_state_every": float(s["save_every"] or -1.0)}
    results = []
    st = status_from_row(d["status_before"][0])
    for ci, n in enumerate(d["calls"]):
        # one status object across calls, as control.sim_loop keeps it
        row = status_from_row(d["status_before"][ci])
        st.next_output_step = st.stepnum + int(n)
        st.next_save_time = row.next_save_time
        updates.SRK2_force_calc([pop], st, sim)
        snap = status_from_row(d["status_before"][ci])
        snap.__dict__.update(st.__dict__)
        results.append((ci, snap, pop.pos.copy(), pop.tangent_list.copy(), pop.forces.copy()))
        if s.get("srk_order", 2) == 4:
            # the last stage's force (pop.forces_aux), SRK4 only
            ref_a = d[f"call{ci}_forces_aux"]
            tol = TRAJ_TOL[name][ci]
            if tol is not None:
                assert np.max(np.abs(pop.forces_aux - ref_a)) <= max(1e3 * tol, 1e-6) * np.max(np.abs(ref_a))
    return d, s, results


@pytest.mark.parametrize("name", CASES)
def test_drop_in_replays_reference_calls(name):
    d, s, results = _replay(name)
    for ci, st, pos, tan, frc in results:
        tol = TRAJ_TOL[name][ci]
        if tol is None:
            break
        after = d["status_after"][ci]
        assert st.stepnum == int(after[2]), (name, ci)
        rt = 1e-9 if tol <= 1e-9 else 1e-5
        assert abs(st.dt_used - after[1]) <= rt * abs(after[1]), (name, ci, st.dt_used, after[1])
        assert abs(st.dt - after[0]) <= 1e-5 * abs(after[0])
        assert abs(st.max_forces_strength - after[5]) <= 1e-5 * abs(after[5])
        assert st.update_grid_list_counter == int(after[4])
        err = np.max(np.abs(min_image(pos - d[f"call{ci}_pos"], s["L"])))
        assert err <= tol, (name, ci, err)
        assert np.max(np.abs(tan - d[f"call{ci}_tangent"])) <= 100 * tol
        ref_f = d[f"call{ci}_forces"]
        assert np.max(np.abs(frc - ref_f)) <= max(1e3 * tol, 1e-6) * np.max(np.abs(ref_f))


@pytest.mark.parametrize("name", ["config1", "chiral_lj", "rotdiff3d"])
def test_reference_lists_are_exact(name):
    d, s = load(name)
    n = d["pos0"].shape[0]
    prm = SystemParams(L=s["L"], spring_params=d["spring_params"], wca_params=d["wca_params"],
                       active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                       n_nearby=s["n_nearby"])
    with Engine(int(s["dim"]), "fp64", bead_capacity=n, system_capacity=1, cell_capacity=64 * n) as eng:
        st = SystemState.from_host(d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], prm)
        slot = eng.admit(st)
        wib, grid, nb = eng.reference_lists(slot, s["n_grid"], s["grid_window"], grid_depth1=s["grid_depth1"],
                                            nbor_depth1=9, mode=1)
        assert np.array_equal(wib.cpu().numpy(), d["k_where_is_bead"])
        assert np.array_equal(pairs_from_nbor(nb.cpu().numpy()), d["k_nbor_pairs"])
        g = grid.cpu().numpy()
        rows = []
        ng, _, nz, _ = g.shape
        for gx in range(ng):
            for gy in range(ng):
                for gz in range(nz):
                    for k in range(g[gx, gy, gz, 0]):
                        rows.append(((gx * ng + gy) * nz + gz, g[gx, gy, gz, 1 + k]))
        assert np.array_equal(np.array(rows, dtype=np.int32).reshape(-1, 2), d["k_grid_pairs"])


def test_philox_stream_matches_oracle():
    for dim in (2, 3):
        g = philox_noise(dim, 1234, 77, 5000).cpu().numpy()
        o = O.philox_noise(1234, 77, dim, 5000)
        assert np.max(np.abs(g - o)) < 1e-13
        assert abs(g.mean()) < 0.02 and abs(g.std() - 1) < 0.02


def test_philox_trajectory_matches_oracle():
    d, s = load("config1")
    set_config(s)
    pop = pop_from_golden(d, s)
    n_steps = 200
    st = status_from_row(d["status_before"][0])
    st.next_output_step = st.stepnum + n_steps
    sim = {"gpu_precision": "fp64", "gpu_noise": "philox", "seed": 5, "save_state_every": -1.0}
    step0 = st.stepnum
    updates.SRK2_force_calc([pop], st, sim)
    ref = O.OracleSystem(d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], s["L"], d["spring_params"],
                         d["wca_params"], d["active_params"], s["D"], s["Dr"], s["radius"], s["n_nearby"],
                         s["n_grid"], nbor_depth=64)
    ref.build_lists(grid_window=s["grid_window"])
    ref.run(n_steps, dt=1e-3, noise_mode=O.NOISE_PHILOX, seed=5, step0=step0)
    assert np.max(np.abs(min_image(pop.pos - ref.pos, s["L"]))) < 1e-9


def test_order_parameters_match_oracle():
    d, s = load("config1")
    prm = SystemParams(L=s["L"], spring_params=d["spring_params"], wca_params=d["wca_params"],
                       active_params=d["active_params"], D=s["D"], Dr=s["Dr"], radius=s["radius"],
                       n_nearby=s["n_nearby"])
    n = d["pos0"].shape[0]
    with Engine(2, "fp64", bead_capacity=n, system_capacity=1, cell_capacity=64 * n) as eng:
        tan = d["call3_tangent"]
        st = SystemState.from_host(d["call3_pos"], tan, d["chain_id"], d["rest_lengths"], prm)
        slot = eng.admit(st)
        got = eng.order_params(slot)
    cs = np.concatenate(([0], np.flatnonzero(np.diff(d["chain_id"])) + 1, [n]))
    want = O.order_params(tan, cs)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)
