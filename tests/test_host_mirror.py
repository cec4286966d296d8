"""The host-side mirror of the reference interface (config, populations,
defaults) reproduces the reference's own initial placement and derived
settings, recorded in the golden fixtures by running the reference."""
import numpy as np
import pytest

from gliding_collective_rotation_b200 import config, defaults, populations
from tests.golden_io import CASES, load


def _build(s):
    sim, _ = defaults.set_defaults()
    sim.update(dict(plot_every=-1, ticker_every=-1, save_state_every=-1., t_max=0., n_threads=1))
    sim.update(s["sim_overrides"])
    if s["dt_override"] is not None:
        sim["dtmax"] = s["dt_override"]
        sim["dt0"] = s["dt_override"]
    config.configure(sim)
    pop = populations.Equal_Size_Chain_Collection(sim)
    pop.random_initialization()
    config.grid_list_setup(sim, [pop])
    return sim, pop


@pytest.mark.parametrize("name", CASES)
def test_initial_placement_matches_reference(name):
    d, s = load(name)
    sim, pop = _build(s)
    assert sim["n_chains"] == s["n_chains"] and sim["n_beads"] == s["n_beads"]
    assert np.array_equal(pop.pos, d["init_pos"])
    assert np.array_equal(pop.tangent_list, d["init_tangent"])
    assert np.array_equal(pop.WCA_params, d["init_wca_params"])
    # configure_start sets the init-grow parameters (v0 = 0, D = 0, ...) when
    # the reference grows chains; the physical values are those recorded
    # after init-grow ended
    want = d["init_active_params"] if not s["b_init_growing"] else d["active_params"]
    assert np.array_equal(pop.active_params(), want)


@pytest.mark.parametrize("name", CASES)
def test_grid_setup_matches_reference(name):
    d, s = load(name)
    sim, pop = _build(s)
    assert sim["n_grid"] == s["n_grid_setup"]
    assert sim["grid_spacing"] == s["grid_spacing"]
    assert sim["n_steps_update_grid_list"] == s["n_steps_update_grid_list"]
    assert sim["max_dist_per_step"] == s["max_dist_per_step_setup"]
    assert sim["grid_window"] == s["grid_window_setup"]
    if s["b_init_growing"]:
        assert pop.D == s["D"] and pop.Dr == s["Dr"]
    else:
        assert pop.D == s["D_init"] and pop.Dr == s["Dr_init"]
    assert config.n_steps_update_grid_list == s["n_steps_update_grid_list"]


def test_status_class_fields():
    sim, _ = defaults.set_defaults()
    st = config.status_class(sim)
    assert st.t == -sim["t_init_grow"] and st.dt == sim["dt0"] and st.dtmax == sim["dtmax"]
    assert st.update_grid_list_counter == 0 and st.next_output_step == 0 and st.stepnum == 0


def test_gpu_switches_in_defaults():
    sim, help = defaults.set_defaults()
    for k in ("gpu", "gpu_precision", "gpu_noise", "gpu_cell_factor", "gpu_steps_per_graph"):
        assert k in sim and k in help
