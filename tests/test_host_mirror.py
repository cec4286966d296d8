"""The packed parameters and derived settings this package computes equal
the ones the reference computed for the same options, as the golden
fixtures recorded them by running the reference: the WCA parameter array
(populations.make_WCA_params, populations.py:48-58) and the grid and dt-rule
settings of config.grid_list_setup (config.py:147-225) that the workloads
and the bench use (``workloads._relax_mdps``)."""
import numpy as np
import pytest

from gliding_collective_rotation_b200 import defaults
from gliding_collective_rotation_b200.engine import wca_params
from gliding_collective_rotation_b200.workloads import _relax_mdps
from tests.golden_io import CASES, load


def _sim(s):
    sim, _ = defaults.set_defaults()
    sim.update(s["sim_overrides"])
    return sim


@pytest.mark.parametrize("name", CASES)
def test_wca_params_match_reference(name):
    d, s = load(name)
    sim = _sim(s)
    got = wca_params(sim["repel_d_max"], sim["WCA_epsilon"], sim["WCA_shift"], sim["LJ_cutoff_factor"])
    assert np.array_equal(got, d["init_wca_params"])


@pytest.mark.parametrize("name", [c for c in CASES if not load(c)[1]["b_init_growing"]])
def test_grid_setup_matches_reference(name):
    """n_grid = max(n_grid_min, int(L / (grid_factor d))) and max_dist_per_step
    = (grid_factor - 1) d / (2 n_update), with d the largest interaction
    distance max(2 a, r_cut) and n_update = int(1 / (safety * rk_cheat))."""
    d, s = load(name)
    sim = _sim(s)
    a = float(sim["a"])
    rc = float(d["init_wca_params"][3])
    dist = max(2 * a, rc)
    n_update = max(1, int(1.0 / (sim["timestep_safety_factor"] * sim["RK_cheat_factor"])))
    assert n_update == s["n_steps_update_grid_list"]
    assert max(sim["n_grid_min"], int(s["L"] / (sim["grid_factor"] * dist))) == s["n_grid_setup"]
    assert _relax_mdps(a, rc, grid_factor=sim["grid_factor"], n_update=n_update) == s["max_dist_per_step_setup"]


def test_gpu_switches_in_defaults():
    sim, help = defaults.set_defaults()
    for k in ("gpu", "gpu_precision", "gpu_noise", "gpu_cell_factor", "gpu_steps_per_graph"):
        assert k in sim and k in help
