"""Several populations in one box: the oracle against the reference's own
multi-population runs (``tests/golden/make_multipop_golden.py``).

The reference's multi-population step is not reproducible from run to run
(its threads meet at a spin barrier on a plain counter array,
SRK.py:487-495): the fixtures hold several one-step trials from one recorded
state, and the oracle must reproduce one of them.  The kernel-level cross
force is deterministic and is compared directly.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.multipop_helpers import CASES, load, oracle_group


def _min_image(d, L):
    return d - L * np.round(d / L)


@pytest.mark.parametrize("name", CASES)
def test_cross_force_matches_the_reference_kernel(name):
    """forces.central_pair_force over a population's nbor_list of another
    population, with the reference's interpop_forces parameters."""
    d, s = load(name)
    n = s["n_pops"]
    seen = 0
    for k in range(n):
        for q in range(n):
            key = f"k_cross_{k}_{q}"
            if key not in d:
                continue
            ref = d[key]
            f = O.cross_forces(d[f"p{k}_pos0"], d[f"p{q}_pos0"], d["cross_wca"][k, q], s["L"])
            assert np.max(np.abs(f - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref))), (key,)
            seen += 1
    assert seen >= 2
    # the relaxed states put partners inside the cross cutoffs
    assert any(np.max(np.abs(d[k])) > 0.1 for k in d if k.startswith("k_cross_"))


@pytest.mark.parametrize("name", CASES)
def test_cross_parameters_are_the_mean_of_the_populations(name):
    """interpop_forces of two WCA populations: 0.5 (WCA_params + other's)
    (populations.py:226-232), recorded from the reference."""
    d, s = load(name)
    n = s["n_pops"]
    for k in range(n):
        for q in range(n):
            if k != q:
                np.testing.assert_allclose(d["cross_wca"][k, q],
                                           O.mean_wca(d[f"p{k}_wca_params"], d[f"p{q}_wca_params"]), rtol=1e-15)


@pytest.mark.parametrize("name", CASES)
def test_one_step_reproduces_a_reference_trial(name):
    d, s = load(name)
    n, L = s["n_pops"], s["L"]
    st0 = d["status_before"]
    g = oracle_group(d, s)
    res = g.run(1, dt=st0[0], dtmax=st0[8], max_dist_per_step=s["max_dist_per_step"], rk_cheat=s["rk_cheat"],
                noise_mode=O.NOISE_PHILOX)
    assert res["steps"] == 1
    errs = []
    for t in range(int(d["trials"])):
        e = max(np.max(np.abs(_min_image(g.systems[k].pos - d[f"trial{t}_p{k}_pos"], L))) for k in range(n))
        errs.append(e)
    best = int(np.argmin(errs))
    assert errs[best] < 1e-12, errs
    sa = d["status_after"][best]
    assert abs(res["dt"] - sa[0]) <= 1e-12 * sa[0]
    assert abs(res["dt_used"] - sa[1]) <= 1e-12 * sa[1]
    # status.max_forces_strength: the first population's own value
    assert abs(res["max_forces_strength"] - sa[5]) <= 1e-10 * sa[5]
    for k in range(n):
        if not s["fixed"][k]:
            ref = d[f"trial{best}_p{k}_forces"]
            assert np.max(np.abs(g.systems[k].forces - ref)) <= 1e-9 * max(1.0, np.max(np.abs(ref)))
            if s["longest"][k] > 1:
                np.testing.assert_allclose(g.systems[k].tangent_list, d[f"trial{best}_p{k}_tangent"], atol=1e-12)


@pytest.mark.parametrize("name", ["pops3_fixed_2d"])
def test_fixed_population_never_moves(name):
    d, s = load(name)
    k = s["fixed"].index(True)
    for t in range(int(d["trials"])):
        np.testing.assert_array_equal(d[f"trial{t}_p{k}_pos"], d[f"p{k}_pos0"])
    g = oracle_group(d, s, D=0.01, seeds=[3, 4, 5])
    g.run(5, dt=1e-4, noise_mode=O.NOISE_PHILOX)
    np.testing.assert_array_equal(g.systems[k].pos, d[f"p{k}_pos0"])
    assert np.max(np.abs(_min_image(g.systems[0].pos - d["p0_pos0"], s["L"]))) > 0


def test_one_population_group_is_the_single_population_step():
    """A group of one population takes the single-population step: the same
    pairs, summed in ascending id instead of the list's order (FP64 rounding
    apart, the same trajectory as OracleSystem.run with fresh lists)."""
    d, s = load("pops2_2d")
    from tests.multipop_helpers import pop_arrays
    a = pop_arrays(d, s, 0)

    def make():
        return O.OracleSystem(a["pos"], a["tangent"], a["chain_id"], a["rest_lengths"], s["L"], a["spring"],
                              a["wca"], a["active"], 0.01, 0.0, a["radius"], a["n_nearby"], s["n_grid"],
                              nbor_depth=256)
    single = make()
    single.build_lists(grid_window=1)
    single.run(5, dt=1e-4, noise_mode=O.NOISE_PHILOX, seed=7, steps_until_update=1000)
    one = make()
    one.seed = 7
    O.OracleGroup([one], [False], np.zeros((1, 1, 4))).run(5, dt=1e-4, noise_mode=O.NOISE_PHILOX)
    assert np.max(np.abs(_min_image(one.pos - single.pos, s["L"]))) < 1e-12


def test_one_population_group_is_the_single_population_srk4_step():
    d, s = load("pops2_2d")
    from tests.multipop_helpers import pop_arrays
    a = pop_arrays(d, s, 0)

    def make():
        return O.OracleSystem(a["pos"], a["tangent"], a["chain_id"], a["rest_lengths"], s["L"], a["spring"],
                              a["wca"], a["active"], 0.01, 0.0, a["radius"], a["n_nearby"], s["n_grid"],
                              nbor_depth=256, srk_order=4)
    single = make()
    single.build_lists(grid_window=1)
    r1 = single.run(5, dt=1e-4, dtmax=1e-3, max_dist_per_step=0.01, noise_mode=O.NOISE_PHILOX, seed=7,
                    steps_until_update=1000)
    one = make()
    one.seed = 7
    r2 = O.OracleGroup([one], [False], np.zeros((1, 1, 4))).run(5, dt=1e-4, dtmax=1e-3, max_dist_per_step=0.01,
                                                               noise_mode=O.NOISE_PHILOX, srk_order=4)
    assert np.max(np.abs(_min_image(one.pos - single.pos, s["L"]))) < 1e-12
    assert np.max(np.abs(one.forces_aux - single.forces_aux)) < 1e-9
    assert abs(r1["dt"] - r2["dt"]) <= 1e-12 * r1["dt"]
