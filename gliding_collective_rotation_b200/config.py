"""Module-level settings, time keeping and derived step parameters.

Mirrors the parts of the reference's ``config`` module that the step path
reads (config.py:13-26 globals, ``status_class`` config.py:37-72,
``configure`` config.py:75-144, ``grid_list_setup`` config.py:147-225), with
the same names and meaning, so that host code written against the reference
runs unchanged on top of this package.  The Numba cache handling of
``configure`` (config.py:121-142) has no counterpart here.
"""
from __future__ import annotations

import numpy as np

b_cached = True
sliding_partner_maxdist = 0.
n_threads = 1
dim = 2
Lx = 1.
n_grid = 1
b_FENE = False
pop_name_list = []
b_announcements = True
n_steps_update_grid_list = 1
RK_cheat_factor = 1
max_dist_per_step = 1
grid_factor = 2.
SRK_order = 2
walls = np.array([False, False, False])


class status_class:
    """General time-keeping object (config.py:37-72)."""

    def __init__(self, sim, start_t=None, start_stepnum=0, start_filenumber=0):
        if start_t is None:
            self.t_start = -sim['t_init_grow']
        else:
            self.t_start = start_t
        self.stepnum = start_stepnum
        self.filenumber = start_filenumber
        self.SRK2_step = 1
        self.b_calc_active_forces = True
        self.reset_timekeeping(sim)

    def reset_timekeeping(self, sim):
        self.t = self.t_start
        self.dt = sim['dt0']
        self.update_nborlists_count = 0
        self.update_mtr_nborlists_count = 0
        self.max_forces_strength = 0
        self.t_prev = 0
        self.clocktime_prev = 0
        self.dt_used = 0
        self.next_save_time = self.t_start
        self.next_output_step = 0
        self.update_grid_list_counter = 0
        self.dtmax = sim['dtmax']
        self.prev_ticker_step = 0

    def dt_SRK2(self):
        return self.dt if self.SRK2_step == 1 else self.dt_used


def configure(sim):
    """Derived values of ``sim`` and module settings (config.py:75-119)."""
    global dim, SRK_order, Lx, walls
    sim['epsilon'] = 1e-8
    sim['chain_density'] = sim['bead_density'] / (
        sim['repel_d_max'] * (sim['a'] * (sim['chain_length'] - 1) + sim['repel_d_max']))
    if sim['n_chains'] < 0:
        sim['n_chains'] = max(1, round(sim['Lx'] * sim['Lx'] * sim['chain_density']))
    sim['n_beads'] = sim['chain_length'] * sim['n_chains']
    if sim.get('motor_density', 0) > 0:
        sim['n_motors'] = int(round(sim['Lx'] * sim['Lx'] * sim['motor_density']))
    if sim.get('n_motors', 0) > 0:
        raise NotImplementedError("motor populations are not part of the GPU step path")
    sim['motor_imparts_force'] = 0
    if sim['Dr'] < 0 and sim['D'] > 0:
        sim['Dr'] = 3 * sim['D'] / (4 * sim['repel_d_max'] * 2)
    sim['outfileprefix'] = sim['resultspath'] + sim['filelabel']
    dim = sim['dim']
    SRK_order = sim['SRK_order']
    Lx = sim['Lx']
    walls = np.array([(st in sim['walls'] or sim['walls'] in ['all', 'True']) for st in ['x', 'y', 'z']])
    np.random.seed(sim['seed'])


def grid_list_setup(sim, pops):
    """Grid spacing, rebuild cadence and the dt safety step (config.py:147-225)."""
    global n_grid, grid_factor, n_steps_update_grid_list, max_dist_per_step
    from . import populations
    dists = []
    for pop in pops:
        d = [0.0]
        if isinstance(pop, populations.Chain_Collection) and pop.longest_chain_length > 1:
            d.append(2 * max(pop.rest_lengths))
        if isinstance(pop, populations.Chain_Collection):
            d.append(max(pop.WCA_params[-1], pop.sliding_partner_maxdist))
        dists.append(max(d))
    sim['biggest_interaction_distance'] = max(dists)
    sim['n_grid'] = max(sim['n_grid_min'], int(sim['Lx'] / (sim['grid_factor'] * sim['biggest_interaction_distance'])))
    if sim['n_grid_max'] > 0:
        sim['n_grid'] = min(sim['n_grid'], sim['n_grid_max'])
    sim['grid_spacing'] = sim['Lx'] / sim['n_grid']
    relevant = [d for d in dists if d < sim['Lx'] / 2]
    sim['n_steps_update_grid_list'] = max(1, int(1. / (sim['timestep_safety_factor'] * sim['RK_cheat_factor'])))
    sim['max_dist_per_step'] = 0.5 * (sim['grid_factor'] - 1) * min(relevant) / sim['n_steps_update_grid_list']
    sim['grid_window'] = int(np.ceil(sim['biggest_interaction_distance'] / sim['grid_spacing']))
    n_grid = sim['n_grid']
    grid_factor = sim['grid_factor']
    n_steps_update_grid_list = sim['n_steps_update_grid_list']
    max_dist_per_step = sim['max_dist_per_step']
    for pop in pops:
        pop.make_empty_grid_list(num_pops=len(pops))
