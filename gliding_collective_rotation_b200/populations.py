"""Bead-spring-chain populations as the step path sees them.

A host-side mirror of the reference's population classes
(populations.py:61-614) restricted to what the step path reads: the same
class names, attribute names, parameter packing (``make_WCA_params``,
``spring_params``, ``active_params``, ``self_interactions``) and the same
order of numpy random draws in construction and ``random_initialization``,
so that a seed gives the reference's initial state.  Motors, shells,
growth/division and special interactions are not mirrored; the init-grow
protocol (``set_init_grow`` / ``early_time_procedures`` / ``end_init_grow``)
is restated as a schedule in ``growth.py``.
"""
from __future__ import annotations

import math

import numpy as np

from . import config


def unit_vector(angle_list):
    """populations.py:12-20"""
    if angle_list.shape[0] == 1:
        return np.array([math.cos(angle_list[0]), math.sin(angle_list[0])])
    sin_theta = math.sin(angle_list[1])
    return np.array([sin_theta * math.cos(angle_list[0]), sin_theta * math.sin(angle_list[0]),
                     math.cos(angle_list[1])])


def make_WCA_params(repel_d_max, WCA_epsilon, WCA_shift, LJ_cutoff_factor):
    """populations.py:48-58: [12 eps r^6, 12 eps r^12, shift, cutoff]."""
    LJ_cutoff_dist = LJ_cutoff_factor * repel_d_max - WCA_shift
    two_WCA_sigma_6 = repel_d_max ** 6
    WCA_factor = 12 * two_WCA_sigma_6 * WCA_epsilon
    return np.array([WCA_factor, WCA_factor * two_WCA_sigma_6, WCA_shift, LJ_cutoff_dist])


class Population:
    """populations.py:61-141 (base arrays and flags)."""

    def __init__(self, total_pop, sim, name="pop"):
        self.total_pop = total_pop
        self.pos = np.empty((total_pop, config.dim), dtype=float)
        self.pos1 = np.empty_like(self.pos)
        self.noise_vec = np.empty((total_pop, 2 * config.dim), dtype=float)
        self.name = name
        self.special_interactions = {}
        self.v0 = 0.
        self.where_active = np.full(total_pop, 0)
        self.n_nearby_beads_dont_repel = 0
        self.b_init_growing = False
        self.pos_init_noise = sim['pos_init_noise']
        self.D = sim['D']
        self.Dr = sim['Dr']
        self.initialized = False
        self.fixed = False
        self.fix_after_grow = False

    def how_many(self):
        return self.total_pop

    def make_empty_grid_list(self, num_pops=1):
        self.n_grid = config.n_grid
        n_grid_z = 1 if config.dim == 2 else self.n_grid
        depth = max(1, int(8 * self.total_pop / self.n_grid ** config.dim))
        self.grid_list = np.zeros((self.n_grid, self.n_grid, n_grid_z, 1 + depth), dtype=np.int64)
        self.where_is_bead = np.zeros((self.total_pop, 3), dtype=np.int64)

    def interactions(self, pop):
        return []

    def self_interactions(self):
        return []


class Forces_Population(Population):
    def __init__(self, total_pop, sim, name="beads"):
        super().__init__(total_pop, sim, name=name)
        self.reset_force_arrays()

    def reset_force_arrays(self):
        """populations.py:149-154: SRK4 keeps the force of its last stage."""
        self.forces = np.zeros((self.total_pop, config.dim))
        if config.SRK_order == 4:
            self.forces_aux = np.empty_like(self.forces)
        else:
            self.forces_aux = np.empty((self.total_pop, 0))

    def make_empty_grid_list(self, num_pops=1):
        super().make_empty_grid_list(num_pops=num_pops)
        self.nbor_list = np.zeros((num_pops, self.total_pop, 1 + 8), dtype=np.int64)


class WCA_Population(Forces_Population):
    def __init__(self, total_pop, sim, name="beads"):
        super().__init__(total_pop, sim, name=name)
        self.reset_WCA_consts(sim)
        self.set_size(self.repel_d_max, sim=sim)
        self.sim = sim

    def set_size(self, diam, sim=None):
        sim = self.sim if sim is None else sim
        self.repel_d_max = diam
        self.diam = diam
        if self.D < 0:
            self.D = sim['T'] / self.repel_d_max
        if self.Dr < 0:
            self.Dr = 3 * self.D / (4 * self.repel_d_max ** 2)

    def reset_WCA_consts(self, sim):
        self.repel_d_max = sim['repel_d_max']
        self.WCA_epsilon = sim['WCA_epsilon']
        self.WCA_shift = sim['WCA_shift']
        self.LJ_cutoff_factor = sim['LJ_cutoff_factor']
        self.adjust_WCA_params()
        super().reset_force_arrays()

    def adjust_WCA_params(self):
        self.WCA_params = make_WCA_params(self.repel_d_max, self.WCA_epsilon, self.WCA_shift,
                                          self.LJ_cutoff_factor)

    def size_scale(self):
        return self.repel_d_max

    def self_interactions(self):
        forces_list = super().self_interactions()
        forces_list.append(["WCA", self.WCA_params])
        if np.any(config.walls):
            forces_list.append(["walls", np.append(self.WCA_params, config.walls)])
        return forces_list


class Oriented_WCA_Population(WCA_Population):
    def __init__(self, total_pop, sim, name="beads"):
        super().__init__(total_pop, sim, name=name)
        self.reset_v0(sim)
        self.tangent_list = np.empty((self.total_pop, config.dim))
        self.orientations = np.empty((self.total_pop, config.dim - 1))
        self.orientations[:, 0] = (sim['phi_init'] * np.ones((self.how_many()))
                                   + sim['phi_init_noise'] * np.random.normal(size=(self.how_many())))
        if config.dim == 3:
            self.orientations[:, 1] = np.full((self.total_pop), 0.5 * np.pi)
        for bi in range(self.total_pop):
            self.tangent_list[bi] = unit_vector(self.orientations[bi])
        self.phi_init = sim['phi_init']
        self.phi_init_noise = sim['phi_init_noise']
        self.Efield = np.zeros(config.dim)

    def reset_v0(self, sim):
        self.v0 = sim['v0']
        self.where_active = np.full((self.total_pop), 0)

    def self_interactions(self):
        forces_list = super().self_interactions()
        if self.Efield.dot(self.Efield) > 0:
            forces_list.append(["Efield", self.Efield])
        return forces_list


class Chain_Collection(Oriented_WCA_Population):
    def __init__(self, num_subpops, total_pop, sim, name="beads", chain_id=None):
        super().__init__(total_pop, sim, name=name)
        self.num_subpops = num_subpops
        if chain_id is None:
            self.chain_id = np.asarray(np.floor(np.arange(self.total_pop)) / (self.total_pop / self.num_subpops),
                                       dtype=np.int64)
        self.inherited_label = self.chain_id.copy()
        self.reset_constants(sim)
        self.make_phonebook()

    def reset_constants(self, sim):
        self.k = sim['k']
        self.reference_rest_length = sim['a']
        self.rest_lengths = np.full(self.num_subpops, sim['a'])
        self.a_init_factor = sim['a_init_factor']
        self.spontaneous_bond_angle = sim['spontaneous_bond_angle']
        if sim['kappa'] >= 0:
            self.rigid_rod_projection_factor = sim['rigid_rod_projection_factor']
            self.kappa = sim['kappa']
        else:
            self.rigid_rod_projection_factor = 1
            self.kappa = 0
        self.n_nearby_beads_dont_repel = sim['n_nearby_beads_dont_repel']
        self.v_tan_angle = sim['v_tan_angle']
        self.b_use_tangent_as_propulsion_direction = sim['b_use_tangent_as_propulsion_direction']
        self.sliding_partner_maxdist = sim['sliding_partner_maxdist']
        self.b_init_growing = False
        self.b_grow = sim['b_grow']
        self.b_FENE = sim['b_FENE']
        self.FENE_tolerance = sim['FENE_tolerance']
        self.reset_v0(sim)
        self.reset_WCA_consts(sim)

    def spring_params(self):
        """populations.py:345-353"""
        return np.array([self.k, self.kappa, self.spontaneous_bond_angle, float(int(self.b_FENE)),
                         float(self.b_get_orientations), self.FENE_tolerance])

    def active_params(self):
        """populations.py:355-358"""
        return np.array([self.v0, self.sliding_partner_maxdist, self.v_tan_angle])

    def make_phonebook(self):
        self.longest_chain_length = int(np.max(np.bincount(self.chain_id)))
        self.phonebook = np.full((self.num_chains(), 1 + self.longest_chain_length), -1)
        self.phonebook[:, 0] = 0
        for bi in range(self.total_pop):
            c = self.chain_id[bi]
            self.phonebook[c, 1 + self.phonebook[c, 0]] = bi
            self.phonebook[c, 0] += 1
        self.set_order_on_chain()

    def num_chains(self):
        return self.num_subpops

    def set_order_on_chain(self):
        self.order_on_chain = np.empty_like(self.chain_id)
        for chain_contents in self.phonebook:
            for i in range(chain_contents[0]):
                self.order_on_chain[chain_contents[1 + i]] = i
        return self.order_on_chain

    def random_initialization(self, already_know_head_pos=False):
        """populations.py:530-557: head bead uniform in the box, chain angle
        uniform, beads laid back along the angle at a_init_factor * rest length."""
        bi = 0
        head_index, ci = 0, 0
        while bi < self.total_pop:
            if self.order_on_chain[bi] == 0:
                head_index = bi
                if not already_know_head_pos:
                    self.pos[head_index] = np.mod(config.Lx / 2 * (1. + self.pos_init_noise * (
                        2 * np.random.rand(config.dim) - 1)), config.Lx)
                    self.orientations[head_index, 0] = np.mod(
                        np.pi * (np.random.rand() > 0.5) + self.phi_init
                        + 2 * np.pi * self.phi_init_noise * np.random.rand() + np.pi, 2 * np.pi) - np.pi
                    if config.dim == 3:
                        self.orientations[head_index, 1] = math.acos(2 * np.random.rand() - 1)
                self.tangent_list[head_index] = unit_vector(self.orientations[head_index])
                ci = self.chain_id[bi]
                bi += 1
            j = 1
            if bi < self.total_pop:
                while self.chain_id[bi] == ci:
                    self.tangent_list[bi] = self.tangent_list[head_index]
                    self.pos[bi] = (self.pos[head_index]
                                    - self.a_init_factor * self.rest_lengths[ci] * self.tangent_list[head_index] * j)
                    bi += 1
                    j += 1
                    if bi > self.total_pop - 1:
                        break
        self.pos = np.mod(self.pos, config.Lx)
        self.initialized = True

    def tangents_to_orientations(self):
        self.orientations[:, 0] = np.arctan2(self.tangent_list[:, 1], self.tangent_list[:, 0])
        if config.dim == 3:
            self.orientations[:, 1] = np.arccos(self.tangent_list[:, 2])

    def chain_members(self, chain_num):
        return self.phonebook[chain_num, 1:1 + self.phonebook[chain_num, 0]]

    def self_interactions(self):
        """populations.py:570-591 (springs first: they update the tangents)."""
        forces_list = super().self_interactions()
        forces_list.append(["self-propulsion", self.active_params()])
        if self.longest_chain_length > 1:
            forces_list.insert(0, ["springs", self.spring_params()])
        if self.sliding_partner_maxdist > 0 and self.v0 > 0:
            for force_name in ["WCA", "self-propulsion"]:
                names = [item[0] for item in forces_list]
                if force_name in names:
                    forces_list.pop(names.index(force_name))
            forces_list.append(["active_sliding_and_WCA", np.append(self.WCA_params, self.active_params())])
        return forces_list


class Equal_Size_Chain_Collection(Chain_Collection):
    """populations.py:593-614"""

    def __init__(self, sim, num_chains=-1, chain_length=-1, name="beads"):
        self.num_subpops = sim['n_chains'] if num_chains < 0 else num_chains
        self.subpop_size = sim['chain_length'] if chain_length < 0 else chain_length
        self.total_pop = self.num_subpops * self.subpop_size
        self.chain_id = np.asarray(np.floor(np.arange(self.total_pop) / self.subpop_size), dtype=np.int64)
        super().__init__(self.num_subpops, self.total_pop, sim, name=name, chain_id=self.chain_id)
        self.b_get_orientations = (self.subpop_size > 1 and self.b_use_tangent_as_propulsion_direction)

    def chain_length(self):
        return self.subpop_size
