"""Synthetic workloads with the shapes of the five benchmark configurations.

Initial states follow the reference's placement rule
(``Chain_Collection.random_initialization``, populations.py:530-557): chain
heads uniform in the box, chain angles uniform, beads laid straight behind
the head at the rest length.  Overlapping placements are relaxed before any
timed step by the step itself under the reference's adaptive dt
(``relax``).  All randomness is seeded.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .engine import SystemParams, wca_params

LJ_CUTOFF = 2.5 / 2 ** (1 / 6)  # 2.5 sigma in units of r_WCA = 2^(1/6) sigma


@dataclass
class SystemSpec:
    name: str
    dim: int
    pos: np.ndarray
    tangent: np.ndarray
    chain_id: np.ndarray
    rest_lengths: np.ndarray
    params: SystemParams
    dt: float
    relax_mdps: float

    @property
    def n(self):
        return self.pos.shape[0]


def lay_chains(rs, n_chains, chain_length, L, a, dim):
    """Head uniform in [0, L)^dim, direction uniform (on the circle / sphere),
    beads at head - j a t (populations.py:530-557 with a_init_factor = 1)."""
    heads = rs.uniform(0.0, L, size=(n_chains, dim))
    if dim == 2:
        ang = rs.uniform(0.0, 2 * np.pi, size=n_chains)
        t = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    else:
        phi = rs.uniform(0.0, 2 * np.pi, size=n_chains)
        ct = rs.uniform(-1.0, 1.0, size=n_chains)
        st = np.sqrt(1 - ct * ct)
        t = np.stack([st * np.cos(phi), st * np.sin(phi), ct], axis=1)
    j = np.arange(chain_length, dtype=np.float64)
    pos = heads[:, None, :] - a * j[None, :, None] * t[:, None, :]
    pos = np.mod(pos.reshape(-1, dim), L)
    tan = np.repeat(t, chain_length, axis=0)
    chain = np.repeat(np.arange(n_chains), chain_length)
    return pos, tan, chain


def _relax_mdps(a, rc, grid_factor=2.0, n_update=40):
    # config.grid_list_setup: 0.5 (grid_factor - 1) min_dist / n_steps_update
    return 0.5 * (grid_factor - 1) * max(2 * a, rc) / n_update


def make_system(name, dim, n_chains, chain_length, L, seed, *, a=0.5, k=100.0, kappa=20.0, eps=1.0,
                cutoff=1.0, v0=1.0, v_tan_angle=0.0, T=0.01, Dr=None, tangent_locked=True, dt=1e-3,
                noise_seed=None, cell_factor=1.0):
    rs = np.random.RandomState(seed)
    pos, tan, chain = lay_chains(rs, n_chains, chain_length, L, a, dim)
    radius = 1.0
    D = T / radius
    if Dr is None:
        Dr = 3 * D / (4 * radius ** 2)
    get_orient = tangent_locked and chain_length > 1
    wca = wca_params(radius, eps, 0.0, cutoff)
    params = SystemParams(
        L=L, spring_params=np.array([k, kappa, 0.0, 0.0, float(get_orient), 0.1]), wca_params=wca,
        active_params=np.array([v0, 0.0, v_tan_angle]), D=D, Dr=Dr, radius=radius, n_nearby=4,
        calc_springs=chain_length > 1, calc_wca=True, self_propel=True, dtmax=dt, max_dist_per_step=math.inf,
        rk_cheat=1.0, seed=seed if noise_seed is None else noise_seed, step=0, cell_factor=cell_factor)
    return SystemSpec(name, dim, pos, tan, chain, np.full(n_chains, a), params, dt, _relax_mdps(a, wca[3]))


def config1(seed=0):
    """2D, Lx=60, 200 x 10 beads, WCA, v0 = 1 tangent-locked, T = 0.01, dt = 1e-3."""
    return make_system("config1", 2, 200, 10, 60.0, seed)


def config2(seed=0, scale=1.0):
    """2D, Lx=1000, 20,000 x 25 beads, LJ (2.5 sigma, eps 0.5), chiral 0.2."""
    n_chains = int(round(20000 * scale))
    L = 1000.0 * math.sqrt(scale)
    return make_system("config2", 2, n_chains, 25, L, seed, eps=0.5, cutoff=LJ_CUTOFF, v_tan_angle=0.2)


def config3(n_systems=256, param_seed=12345, first=0):
    """Batched sweep: per system n_chains log-uniform [50, 4000], chain length
    uniform integer [5, 40], area fraction uniform [0.1, 0.4], chirality
    uniform [-0.5, 0.5], bending uniform [1, 50]; otherwise config 1; the
    Philox seed of system i is i."""
    rng = np.random.default_rng(param_seed)
    nch = np.exp(rng.uniform(np.log(50), np.log(4000), size=n_systems)).astype(int)
    clen = rng.integers(5, 41, size=n_systems)
    phi = rng.uniform(0.1, 0.4, size=n_systems)
    ang = rng.uniform(-0.5, 0.5, size=n_systems)
    kap = rng.uniform(1.0, 50.0, size=n_systems)
    out = []
    for i in range(first, n_systems):
        a = 0.5
        # excluded area of a chain r (a (L-1) + r) with r = 1 (config.py:81-82)
        L = math.sqrt(nch[i] * (a * (clen[i] - 1) + 1.0) / phi[i])
        out.append(make_system(f"sweep{i}", 2, int(nch[i]), int(clen[i]), L, seed=1000 + i, kappa=float(kap[i]),
                               v_tan_angle=float(ang[i]), noise_seed=i))
    return out


def config5(seed=0, scale=1.0):
    """3D, L=200, 40,000 x 25 beads, LJ eps 1 (2.5 sigma), kappa 10,
    rotationally diffusing propulsion (Dr 0.1), T 0.05, dt 5e-4."""
    n_chains = int(round(40000 * scale))
    L = 200.0 * scale ** (1 / 3)
    return make_system("config5", 3, n_chains, 25, L, seed, kappa=10.0, eps=1.0, cutoff=LJ_CUTOFF, T=0.05,
                       Dr=0.1, tangent_locked=False, dt=5e-4)


def populations(n_boxes=128, seed=0):
    """Boxes of two populations each (the multi-population step,
    updates.py:146-247): 2D, L = 150, 1000 chains x 10 beads as config 1
    (WCA, v0 = 1 tangent-locked) and 3000 single passive beads of diameter
    0.7; cross parameters the mean of the two WCA sets (populations.py:226-232).
    Returns the specs (chains of box i at 2i, beads at 2i + 1) and the
    groups ``(members, fixed, cross_wca)``."""
    specs, groups = [], []
    for i in range(n_boxes):
        rs = np.random.RandomState(seed * 100003 + i)
        chains = make_system(f"box{i}_chains", 2, 1000, 10, 150.0, seed=5000 + i, noise_seed=2 * i)
        L = 150.0
        nb = 3000
        pos = rs.uniform(0.0, L, size=(nb, 2))
        ang = rs.uniform(0.0, 2 * math.pi, size=nb)
        tan = np.stack([np.cos(ang), np.sin(ang)], axis=1)
        r = 0.7
        wca = wca_params(r, 1.0, 0.0, 1.0)
        D = 0.01 / r
        params = SystemParams(
            L=L, spring_params=np.array([100.0, 20.0, 0.0, 0.0, 0.0, 0.1]), wca_params=wca,
            active_params=np.array([0.0, 0.0, 0.0]), D=D, Dr=3 * D / (4 * r * r), radius=r, n_nearby=4,
            calc_springs=False, calc_wca=True, self_propel=False, dtmax=1e-3, max_dist_per_step=math.inf,
            rk_cheat=1.0, seed=2 * i + 1, step=0)
        beads = SystemSpec(f"box{i}_beads", 2, pos, tan, np.arange(nb), np.full(nb, 0.5), params, 1e-3,
                           chains.relax_mdps)
        cross = np.zeros((2, 2, 4))
        cross[0, 1] = cross[1, 0] = 0.5 * (chains.params.wca_params + wca)
        specs += [chains, beads]
        groups.append(([2 * i, 2 * i + 1], [False, False], cross))
    return specs, groups


def motor_params(a=0.5, force=1.0, k_on=0.9, k_off=0.2, one_per_bead=False):
    """The motor_push parameters of Chain_Collection.interactions
    (populations.py:276-287) with the reference's defaults: motor_max_dist =
    a / 2 (squared), imparts_force = v0 (config.py:95-98), k_on 0.9, k_off 0.2
    (defaults.py:185-201)."""
    return np.array([(a / 2) ** 2, float(one_per_bead), force, k_on, k_off])


def motor_list_radius(L, biggest_interaction, max_dist_sq, grid_factor=2.0, n_grid_min=1):
    """The list radius of the reference's chain-motor lists: grid_window *
    Lx / n_grid with n_grid of config.grid_list_setup (config.py:147-193) and
    the chain-motor thread's grid_window = max(1, ceil(grid_factor *
    nbor_length_scale / grid_spacing)), whose length scale is the squared
    motor_max_dist (SRK.py:84-87, 99-101); the list holds the motors within
    that radius (updates.py:603-604)."""
    n_grid = max(n_grid_min, int(L / (grid_factor * biggest_interaction)))
    h = L / n_grid
    window = max(1, int(math.ceil(grid_factor * max_dist_sq / h)))
    return window * h


def motors(n_boxes=16, seed=0, n_chains=200, chain_length=10, L=60.0, motor_density=0.5, D_motors=0.1,
           k_on=0.9, k_off=0.2, hold=True):
    """Boxes of chains pushed by motors (Motor_Population,
    populations.py:617-661; BDsim.py:24-25): config-1 chains whose
    propulsion v0 = 1 is handed to the motors (config.py:95-98: chains keep v0
    = 0), and round(L^2 motor_density) motors of diffusion D_motors
    (defaults.py:179-201).  Returns specs (chains of box i at 2i, motors at
    2i + 1), the groups ``(members, fixed, cross_wca)`` and the motor settings
    ``(motor index, chain index, params, hold)``; the motors' cross r_cut is
    the reference's chain-motor list radius."""
    specs, groups, mots = [], [], []
    a = 0.5
    prm = motor_params(a, 1.0, k_on, k_off)
    for i in range(n_boxes):
        rs = np.random.RandomState(seed * 100019 + i)
        chains = make_system(f"box{i}_chains", 2, n_chains, chain_length, L, seed=7000 + i, v0=0.0,
                             noise_seed=2 * i)
        nm = int(round(L * L * motor_density))
        pos = rs.uniform(0.0, L, size=(nm, 2))
        tan = np.tile([1.0, 0.0], (nm, 1))
        # biggest interaction distance: 2 a (springs), r_cut (WCA), motor_max_dist
        r_list = motor_list_radius(L, max(2 * a, float(chains.params.wca_params[3]), a / 2), prm[0])
        params = SystemParams(
            L=L, spring_params=np.array([0.0, 0.0, 0.0, 0.0, 0.0, 0.1]), wca_params=np.array([0.0, 0.0, 0.0, r_list]),
            active_params=np.array([0.0, 0.0, 0.0]), D=D_motors, Dr=0.0, radius=1.0, n_nearby=0,
            calc_springs=False, calc_wca=True, self_propel=False, dtmax=chains.params.dtmax,
            max_dist_per_step=math.inf, rk_cheat=1.0, seed=2 * i + 1, step=0)
        mot = SystemSpec(f"box{i}_motors", 2, pos, tan, np.arange(nm), np.full(nm, a), params, chains.dt,
                         chains.relax_mdps)
        cross = np.zeros((2, 2, 4))
        cross[1, 0] = [0.0, 0.0, 0.0, r_list]
        specs += [chains, mot]
        groups.append(([2 * i, 2 * i + 1], [False, False], cross))
        mots.append((2 * i + 1, 2 * i, prm, hold))
    return specs, groups, mots


def serve_trace(n_requests, rate=20.0, seed=7, min_beads=1000, max_beads=1_000_000, min_steps=1000,
                max_steps=20000):
    """Poisson arrivals at `rate`/s of config-3-style systems with bead count
    log-uniform in [min_beads, max_beads] and a step count uniform in
    [min_steps, max_steps]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
    beads = np.exp(rng.uniform(np.log(min_beads), np.log(max_beads), size=n_requests))
    steps = rng.integers(min_steps, max_steps + 1, size=n_requests)
    clen = rng.integers(5, 41, size=n_requests)
    phi = rng.uniform(0.1, 0.4, size=n_requests)
    ang = rng.uniform(-0.5, 0.5, size=n_requests)
    kap = rng.uniform(1.0, 50.0, size=n_requests)
    reqs = []
    for i in range(n_requests):
        nch = max(1, int(round(beads[i] / clen[i])))
        L = math.sqrt(nch * (0.5 * (clen[i] - 1) + 1.0) / phi[i])
        reqs.append(dict(id=i, arrival=float(t[i]), n_chains=nch, chain_length=int(clen[i]), L=L,
                         steps=int(steps[i]), kappa=float(kap[i]), v_tan_angle=float(ang[i]), seed=i))
    return reqs
