"""Helpers for the GPU tests: reference-shaped populations and status objects
built from the golden fixtures, and the module settings the step reads."""
from types import SimpleNamespace

import numpy as np

from gliding_collective_rotation_b200 import config


def pop_from_arrays(pos, tangent, chain_id, rest_lengths, spring, wca, active, D, Dr, radius, n_nearby,
                    b_get_orientations=True):
    chain_id = np.asarray(chain_id, dtype=np.int64)
    longest = int(np.max(np.bincount(chain_id)))
    sp = np.array(spring, dtype=np.float64)
    wc = np.array(wca, dtype=np.float64)
    ac = np.array(active, dtype=np.float64)
    return SimpleNamespace(
        name="beads", fixed=False, total_pop=len(pos), pos=np.array(pos, dtype=np.float64),
        pos1=np.zeros_like(pos, dtype=np.float64), tangent_list=np.array(tangent, dtype=np.float64),
        forces=np.zeros_like(pos, dtype=np.float64), chain_id=chain_id,
        rest_lengths=np.array(rest_lengths, dtype=np.float64), longest_chain_length=longest,
        rigid_rod_projection_factor=0.0, D=float(D), Dr=float(Dr), repel_d_max=float(radius),
        n_nearby_beads_dont_repel=int(n_nearby), b_init_growing=False, special_interactions={},
        b_get_orientations=b_get_orientations,
        self_interactions=lambda: ([["springs", sp]] if longest > 1 else []) + [["WCA", wc],
                                                                              ["self-propulsion", ac]])


def pop_from_golden(d, s):
    pop = pop_from_arrays(d["pos0"], d["tangent0"], d["chain_id"], d["rest_lengths"], d["spring_params"],
                          d["wca_params"], d["active_params"], s["D"], s["Dr"], s["radius"], s["n_nearby"])
    pop.rigid_rod_projection_factor = float(s.get("rigid_rod", 0.0))
    if s.get("srk_order", 2) == 4:
        pop.forces_aux = np.zeros_like(pop.pos)
    return pop


def set_pop_params(pop, spring, wca, active, D, Dr, radius, n_nearby, rest_lengths, rigid, growing):
    """Give a population new parameters between calls, as the reference's
    init-grow loop does (control.early_time_procedures)."""
    sp, wc, ac = (np.array(a, dtype=np.float64) for a in (spring, wca, active))
    longest = pop.longest_chain_length
    pop.self_interactions = lambda: ([["springs", sp]] if longest > 1 else []) + [["WCA", wc],
                                                                                   ["self-propulsion", ac]]
    pop.D, pop.Dr, pop.repel_d_max, pop.n_nearby_beads_dont_repel = float(D), float(Dr), float(radius), int(n_nearby)
    pop.rest_lengths[:] = rest_lengths
    pop.rigid_rod_projection_factor = float(rigid)
    pop.b_init_growing = bool(growing)


def set_config(s):
    config.dim = int(s["dim"])
    config.Lx = float(s["L"])
    config.SRK_order = int(s.get("srk_order", 2))
    config.n_steps_update_grid_list = int(s["n_steps_update"])
    config.max_dist_per_step = float(s["max_dist_per_step"])
    config.RK_cheat_factor = float(s["rk_cheat"])
    config.grid_factor = float(s["grid_factor"])
    config.walls = np.array([False, False, False])


def status_from_row(row):
    keys = ["dt", "dt_used", "stepnum", "t", "update_grid_list_counter", "max_forces_strength",
            "next_output_step", "next_save_time", "dtmax"]
    d = dict(zip(keys, row.tolist()))
    return SimpleNamespace(dt=d["dt"], dtmax=d["dtmax"], dt_used=d["dt_used"], stepnum=int(d["stepnum"]),
                           t=d["t"], next_output_step=int(d["next_output_step"]),
                           next_save_time=d["next_save_time"],
                           update_grid_list_counter=int(d["update_grid_list_counter"]),
                           max_forces_strength=d["max_forces_strength"], b_calc_active_forces=True)
