"""``SRK2_force_calc(pops, status, sim)`` on the B200: the drop-in step.

Same signature, inputs, outputs and bookkeeping as the reference's
``updates.SRK2_force_calc`` (updates.py:132-267):

* runs up to ``status.next_output_step - status.stepnum`` SRK2 steps, stops
  early when the elapsed time reaches ``status.next_save_time - status.t``
  (if saving) -- SRK.py:128-130, 345-346;
* writes back ``status.dt`` (last dt), ``status.dt_used`` (time elapsed in the
  call), ``status.stepnum``, ``status.t``, ``status.max_forces_strength`` and
  ``status.update_grid_list_counter`` -- updates.py:249-256;
* leaves the population's ``pos``, ``pos1``, ``tangent_list`` and ``forces``
  as the reference leaves them (F0 + F1 of the last step, tangents at pos1);
* raises no exception for numerical trouble: a GPU cell or neighbour-list
  overflow makes the next call use deeper cells or lists (the reference
  regrows its lists the same way, updates.py:257-267) and non-finite values
  are reported in ``status.gpu_flags``.

The bead state stays on the device between calls; each call uploads the
host arrays (the caller may have changed them) and downloads the result.
The rigid-rod projection (updates.project_updates_for_rigid_rod,
updates.py:347-499) runs on the device whenever the population's
``rigid_rod_projection_factor`` is on and a chain has more than 2 beads, so
the reference's init-grow protocol (control.early_time_procedures,
control.py:153-219), which changes the radius, WCA parameters, spring
constants, rest lengths and projection factor between calls, runs through
this step unchanged; while a population grows the step computes in FP64
whatever ``gpu_precision`` says (radii down to 1e-8 put the WCA prefactors
below the FP32 range).  ``config.SRK_order`` 4 runs the reference's SRK4
branch (SRK.py:144-215, 296-321) and fills ``pop.forces_aux`` with the last
stage's force.  A list of several populations (up to 4, fixed ones
included) steps as the reference steps it (updates.py:146-247): one dt from
the largest max-force value over the moving populations, and each moving
population feels the others' WCA force (``interpop_forces``,
updates.py:274-312), through ``gcr_couple``.  A Motor_Population in the
list pushes the chains it interacts with (``motor_push``,
forces.py:248-283, through ``gcr_set_motors``; SRK2) and ``where_active``
of every population is written back.  Features outside the GPU path (walls,
FENE, active sliding, E-field) raise ``NotImplementedError``.

``install(updates_module, config_module)`` rebinds a reference checkout's
``updates.SRK2_force_calc`` to this function and makes it read that
checkout's ``config`` module.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import config as _default_config
from ._lib import FLAG_CELL_OVERFLOW, FLAG_LIST_OVERFLOW, GcrError
from .batch import MAX_DEPTH, MAX_LIST_DEPTH, cell_scale, default_depth, default_list_depth
from .engine import Engine, SystemParams, SystemState, default_config, footprint

_config = _default_config
_pair_rule_check = None


def install(updates_module, config_module, force_rules_module=None, forces_module=None):
    """Use this step inside a reference checkout: ``updates.SRK2_force_calc``
    becomes the GPU step and reads the checkout's ``config`` globals."""
    global _config, _pair_rule_check
    _config = config_module
    if force_rules_module is not None and forces_module is not None:
        _pair_rule_check = (force_rules_module, forces_module)
    updates_module.SRK2_force_calc = SRK2_force_calc
    return SRK2_force_calc


def _force_list(pop):
    """interpop_forces(pop, pop) (updates.py:274-312) as a dict of name -> params."""
    if pop.name in getattr(pop, "special_interactions", {}):
        forces_list = pop.special_interactions[pop.name]
    else:
        forces_list = pop.self_interactions()
    out = {}
    for name, params in forces_list:
        out[name] = np.array(params, dtype=np.float64)
    if getattr(pop, "b_init_growing", False):
        for name in ("WCA", "active_sliding_and_WCA"):
            if name in out and out[name][0] != 0:
                out[name][3] = (out[name][1] / out[name][0]) ** (1 / 6)
    return out


_SUPPORTED = {"springs", "WCA", "self-propulsion"}


def _is_motors(pop):
    """A Motor_Population (populations.py:617-661): single beads that only
    diffuse and push the chains near them."""
    return type(pop).__name__ == "Motor_Population" or hasattr(pop, "motor_max_dist_sq")


def _pop_arrays(pop, dim):
    """Positions, tangents, chain ids and rest lengths of a population; a
    motor population has no chains or tangents: one chain per motor."""
    if _is_motors(pop):
        n = pop.total_pop
        return pop.pos, np.tile(np.eye(dim)[0], (n, 1)), np.arange(n), np.ones(n)
    return pop.pos, pop.tangent_list, pop.chain_id, pop.rest_lengths


def _motor_list_radius(cfg, params):
    """The radius of the reference's chain-motor lists: grid_window * Lx /
    n_grid (updates.py:603-604), grid_window of the chain-motor thread from
    its length scale, the squared motor_max_dist (SRK.py:84-87, 99-101)."""
    L = float(cfg.Lx)
    n_grid = int(getattr(cfg, "n_grid", 0) or 0)
    grid_factor = float(getattr(cfg, "grid_factor", 2.0))
    if n_grid <= 0:
        raise NotImplementedError("motors need config.n_grid (config.grid_list_setup)")
    h = L / n_grid
    return max(1, int(np.ceil(grid_factor * float(params[0]) / h))) * h


def _motor_params(pop, status, sim, seed):
    """A motor population as a system: single beads with D = D_motors and
    no force of their own (their diffusion, SRK.py:389-395), binned with a
    zero-strength WCA of cutoff the chain-motor list radius.  A motor
    population with D = 0 (pop.fixed) steps with D = 0: it keeps its place."""
    cfg = _config
    names = [f[0] for f in pop.self_interactions()]
    if set(names) - {"diffuse"}:
        raise NotImplementedError(f"forces not on the GPU step: {sorted(set(names) - {'diffuse'})}")
    r_list = _motor_list_radius(cfg, [float(pop.motor_max_dist_sq)])
    return SystemParams(
        L=float(cfg.Lx), spring_params=np.zeros(6), wca_params=np.array([0.0, 0.0, 0.0, r_list]),
        active_params=np.zeros(3), D=float(pop.D), Dr=0.0, radius=1.0, n_nearby=0, calc_springs=False,
        calc_wca=True, self_propel=False, dtmax=float(status.dtmax), max_dist_per_step=float(cfg.max_dist_per_step),
        rk_cheat=float(cfg.RK_cheat_factor), seed=seed, step=int(status.stepnum),
        cell_factor=float(sim.get('gpu_cell_factor', 1.0)), skin=sim.get('gpu_skin', None))


def _pop_params(pop, status, sim, seed):
    """The packed parameters of one population (its self_interactions, as
    SRK.py:58-97 reads them) as a ``SystemParams``."""
    if _is_motors(pop):
        return _motor_params(pop, status, sim, seed)
    cfg = _config
    forces = _force_list(pop)
    extra = set(forces) - _SUPPORTED
    if extra:
        raise NotImplementedError(f"forces not on the GPU step: {sorted(extra)}")
    longest = int(pop.longest_chain_length)
    calc_springs = "springs" in forces and longest > 1
    spring = forces.get("springs", np.zeros(6))
    if calc_springs and spring[3] != 0:
        raise NotImplementedError("FENE springs are not part of the GPU step")
    calc_wca = "WCA" in forces
    wca = forces.get("WCA", np.zeros(4))
    self_propel = "self-propulsion" in forces and bool(status.b_calc_active_forces)
    active = forces.get("self-propulsion", np.zeros(3))
    return SystemParams(
        L=float(cfg.Lx), spring_params=spring, wca_params=wca, active_params=active, D=float(pop.D),
        Dr=float(pop.Dr), radius=float(pop.repel_d_max), n_nearby=int(pop.n_nearby_beads_dont_repel),
        calc_springs=calc_springs, calc_wca=calc_wca, self_propel=self_propel, dtmax=float(status.dtmax),
        max_dist_per_step=float(cfg.max_dist_per_step), rk_cheat=float(cfg.RK_cheat_factor), seed=seed,
        step=int(status.stepnum), cell_factor=float(sim.get('gpu_cell_factor', 1.0)),
        skin=sim.get('gpu_skin', None), rigid_rod=float(getattr(pop, "rigid_rod_projection_factor", 0.0)))


def _cross_wca(pop1, pop2):
    """The WCA parameters of the force on ``pop1`` from ``pop2``:
    interpop_forces(pop1, pop2) (updates.py:274-312) -- a special interaction
    if ``pop1`` has one for ``pop2``, else ``pop1.interactions(pop2)`` -- with
    the cutoff at the potential's minimum while either population grows.
    Zeros: no pair force."""
    if pop2.name in getattr(pop1, "special_interactions", {}):
        forces_list = pop1.special_interactions[pop2.name]
    else:
        forces_list = pop1.interactions(pop2)
    out = np.zeros(4)
    for name, params in forces_list or []:
        if name == "motor_push":
            continue  # the motors' push: gcr_set_motors, not a pair force
        if name != "WCA":
            raise NotImplementedError(f"force between populations not on the GPU step: {name}")
        out = np.array(params, dtype=np.float64)[:4].copy()
    if (getattr(pop1, "b_init_growing", False) or getattr(pop2, "b_init_growing", False)) and out[0] != 0:
        out[3] = (out[1] / out[0]) ** (1 / 6)
    return out


class _GpuPop:
    """Device copy of one population and the context that steps it."""

    def __init__(self, pop, sim, dim, precision, params, cell_depth, list_depth, key, srk_order=2):
        self.key = key
        self.dim, self.precision, self.srk_order = dim, precision, srk_order
        self.n, self.n_chains = pop.total_pop, len(pop.rest_lengths)
        self.spg = int(sim.get('gpu_steps_per_graph', 10))
        self.state = SystemState.from_host(pop.pos, pop.tangent_list, pop.chain_id, pop.rest_lengths, params,
                                           precision=precision, device=torch.device("cuda"), srk_order=srk_order)
        self.engine = None
        self.make_engine(params, cell_depth, list_depth)
        n = self.n
        ft = torch.float64 if precision == "fp64" else torch.float32
        self.h_pos = torch.empty((n, dim), dtype=torch.float64, pin_memory=True)
        self.h_tan = torch.empty((n, dim), dtype=ft, pin_memory=True)
        self.h_frc = torch.empty((n, dim), dtype=ft, pin_memory=True)
        self.h_pos1 = torch.empty((n, dim), dtype=torch.float64, pin_memory=True)
        self.h_faux = torch.empty((n, dim), dtype=ft, pin_memory=True) if srk_order == 4 else None
        self.rng = None

    def make_engine(self, params, cell_depth, list_depth):
        """(Re)create the context and bind the device state to it; the state
        tensors, and so the bead state, carry over."""
        if self.engine is not None:
            self.engine.close()
        cfg = default_config(self.dim, self.precision, cell_depth=cell_depth, list_depth=list_depth,
                             srk_order=self.srk_order)
        cells = footprint(cfg, params, self.n, self.n_chains)[0]
        self.engine = Engine(self.dim, self.precision, bead_capacity=max(self.n, 1), system_capacity=1,
                             cell_capacity=max(cells, 1), cell_depth=cell_depth, list_depth=list_depth,
                             steps_per_graph=self.spg, device=self.state.pos.device, srk_order=self.srk_order)
        self.engine.admit(self.state)


def _key(pop, dim, precision, params, depth, ldepth, srk_order=2):
    # the pair cutoff and skin may change from call to call (init-grow): the
    # context re-derives its cell grid within the cells it reserved
    return (pop.total_pop, len(pop.rest_lengths), dim, precision, float(params.L), float(params.cell_factor), depth,
            ldepth, bool(params.calc_wca), srk_order)


def _gpu_state(pop, sim, dim, precision, params, srk_order=2):
    depth = getattr(pop, "_gcr_cell_depth", default_depth(dim, cell_scale(params)))
    ldepth = getattr(pop, "_gcr_list_depth", default_list_depth(dim))
    g = getattr(pop, "_gcr", None)
    key = _key(pop, dim, precision, params, depth, ldepth, srk_order)
    if g is None or g.key != key:
        if g is not None:
            g.engine.close()
        g = _GpuPop(pop, sim, dim, precision, params, depth, ldepth, key, srk_order)
        pop._gcr = g
    return g


def SRK2_force_calc(pops, status, sim):
    """Stochastic Runge-Kutta 2nd-order update (Branka and Heyes, PRE 60:2381,
    1999) of one bead-spring-chain population on the GPU."""
    cfg = _config
    srk_order = int(getattr(cfg, "SRK_order", 2))
    if srk_order not in (2, 4):
        raise NotImplementedError("the GPU step implements SRK_order 2 and 4")
    if np.any(getattr(cfg, "walls", np.zeros(3, dtype=bool))):
        raise NotImplementedError("walls are not part of the GPU step")
    movers = [p for p in pops if not p.fixed]
    if not movers:
        raise NotImplementedError("the GPU step needs a population that moves")
    if _pair_rule_check is not None:
        fr, fm = _pair_rule_check
        if fr.central_pair_force_rule is not fm.WCA:
            raise NotImplementedError("the GPU step implements the forces.WCA pair rule")
    if not torch.cuda.is_available():
        raise GcrError(-2, "no CUDA device: the gcr hot path runs on the GPU only")
    if len(pops) > 1:
        return _srk2_populations(pops, status, sim, srk_order)
    pop = pops[0]
    dim = int(cfg.dim)
    precision = sim.get('gpu_precision', 'fp64')
    if getattr(pop, "b_init_growing", False):
        precision = 'fp64'

    # time_vals, updates.py:138-146
    max_dt_usable = (status.next_save_time - status.t) if sim.get('save_state_every', -1) > 0 else -1.0
    max_steps = status.next_output_step - status.stepnum
    seed = int(sim.get('seed', 0))
    params = _pop_params(pop, status, sim, seed)
    g = _gpu_state(pop, sim, dim, precision, params, srk_order)
    st, eng = g.state, g.engine

    # upload the host state (the caller may have changed it between calls)
    g.h_pos.numpy()[:] = pop.pos
    g.h_tan.numpy()[:] = pop.tangent_list
    st.pos.copy_(g.h_pos, non_blocking=True)
    st.tangent.copy_(g.h_tan, non_blocking=True)
    st.rest_lengths.copy_(torch.from_numpy(np.asarray(pop.rest_lengths, dtype=np.float64)))
    st.params = params
    try:
        eng.update_params(st)
    except GcrError as e:
        if e.code != -6:
            raise
        # the new cell grid needs more cells than the context reserved
        g.make_engine(params, g.engine.cfg.cell_depth, g.engine.cfg.list_depth)
        eng = g.engine

    noise = None
    n_noise = 0
    mode = sim.get('gpu_noise', 'philox')
    if mode == 'mt':
        # the reference's MT19937 stream, drawn on the host in SRK.py:134-142 order
        if g.rng is None:
            g.rng = np.random.RandomState(seed)
        if max_steps < 0:
            raise NotImplementedError("injected noise needs a bounded step count per call")
        per = st.n * dim * (int(pop.D > 0) + int(pop.Dr > 0))
        rng_state = g.rng.get_state()
        flat = g.rng.standard_normal(per * max_steps)
        snaps = np.zeros((max_steps, st.n, 2 * dim))
        k = 0
        for s in range(max_steps):
            if pop.D > 0:
                snaps[s, :, :dim] = flat[k:k + st.n * dim].reshape(st.n, dim)
                k += st.n * dim
            if pop.Dr > 0:
                snaps[s, :, dim:] = flat[k:k + st.n * dim].reshape(st.n, dim)
                k += st.n * dim
        noise = torch.from_numpy(snaps).to(eng.device)
        n_noise = max_steps
    elif mode != 'philox':
        raise ValueError(f"unknown gpu_noise {mode!r}")

    # An overflow of the GPU cells or lists is the library's capacity, not the
    # model's: grow them in place and finish the call (steps already taken
    # stand; the step counter, and so the noise stream, carries on).
    done, elapsed, dt = 0, 0.0, float(status.dt)
    while True:
        left = max_steps - done if max_steps >= 0 else -1
        lim = max_dt_usable - elapsed if max_dt_usable >= 0 else -1.0
        eng.call_begin(st.slot, max_steps=left, dt=dt, max_dt_usable=lim,
                       noise=noise[done:] if noise is not None else None)
        if left >= 0 and max_dt_usable < 0:
            eng.run(left, sync_every=0)
        else:
            # time-limited: check between graphs whether the system is done
            eng.run(left if left >= 0 else (1 << 62), sync_every=1)
        res = eng.status(st.slot)
        done += int(res['steps_done'])
        elapsed += res['dt_used']
        dt = res['dt']
        grow_cells = bool(res['flags'] & FLAG_CELL_OVERFLOW) and eng.cfg.cell_depth < MAX_DEPTH
        grow_lists = bool(res['flags'] & FLAG_LIST_OVERFLOW) and eng.cfg.list_depth < MAX_LIST_DEPTH
        if not (grow_cells or grow_lists) or done == max_steps or (max_dt_usable >= 0 and elapsed >= max_dt_usable):
            break
        depth = min(MAX_DEPTH, 2 * eng.cfg.cell_depth) if grow_cells else eng.cfg.cell_depth
        ldepth = min(MAX_LIST_DEPTH, 2 * eng.cfg.list_depth) if grow_lists else eng.cfg.list_depth
        pop._gcr_cell_depth, pop._gcr_list_depth = depth, ldepth
        st.params.step = int(res['step'])
        g.make_engine(st.params, depth, ldepth)
        g.key = _key(pop, dim, precision, params, depth, ldepth, srk_order)
        eng = g.engine
    steps_done = done
    if mode == 'mt' and steps_done < n_noise:
        # give back the deviates of steps that did not run
        g.rng.set_state(rng_state)
        g.rng.standard_normal(per * steps_done)

    # download into the population's arrays
    g.h_pos.copy_(st.pos, non_blocking=True)
    g.h_pos1.copy_(st.pos1, non_blocking=True)
    g.h_tan.copy_(st.tangent, non_blocking=True)
    g.h_frc.copy_(st.forces, non_blocking=True)
    if g.h_faux is not None:
        g.h_faux.copy_(st.forces_aux, non_blocking=True)
    torch.cuda.synchronize(eng.device)
    pop.pos[:] = g.h_pos.numpy()
    pop.pos1[:] = g.h_pos1.numpy()
    pop.tangent_list[:] = g.h_tan.numpy()
    pop.forces[:] = g.h_frc.numpy()
    if g.h_faux is not None and getattr(pop, "forces_aux", np.empty((0, 0))).shape == pop.forces.shape:
        pop.forces_aux[:] = g.h_faux.numpy()

    # write-back, updates.py:249-256
    status.dt = dt
    status.dt_used = elapsed
    status.stepnum += steps_done
    status.t += status.dt_used
    status.max_forces_strength = res['max_forces_strength']
    status.update_grid_list_counter = max(
        1, (steps_done + status.update_grid_list_counter) % cfg.n_steps_update_grid_list)
    status.gpu_flags = res['flags']
    return None


class _GpuGroup:
    """Device copies of several populations in one context, coupled as one
    box (``Engine.couple``)."""

    def __init__(self, pops, sim, dim, precision, params, fixed, cell_depth, list_depth, key, srk_order):
        self.key = key
        self.dim, self.precision, self.srk_order = dim, precision, srk_order
        self.fixed = list(fixed)
        self.spg = int(sim.get('gpu_steps_per_graph', 10))
        dev = torch.device("cuda")
        self.states = [SystemState.from_host(*_pop_arrays(p, dim), prm, precision=precision, device=dev,
                                             srk_order=srk_order)
                       for p, prm in zip(pops, params)]
        ft = torch.float64 if precision == "fp64" else torch.float32
        self.host = []
        for p in pops:
            n = p.total_pop
            self.host.append(dict(pos=torch.empty((n, dim), dtype=torch.float64, pin_memory=True),
                                  pos1=torch.empty((n, dim), dtype=torch.float64, pin_memory=True),
                                  tan=torch.empty((n, dim), dtype=ft, pin_memory=True),
                                  frc=torch.empty((n, dim), dtype=ft, pin_memory=True)))
        self.engine = None
        self.cross = None
        self.motors = []
        self.make_engine(cell_depth, list_depth)

    def make_engine(self, cell_depth, list_depth):
        if self.engine is not None:
            self.engine.close()
        cfg = default_config(self.dim, self.precision, cell_depth=cell_depth, list_depth=list_depth,
                             srk_order=self.srk_order)
        cells = sum(footprint(cfg, st.params, st.n, st.n_chains)[0] for st in self.states)
        self.engine = Engine(self.dim, self.precision, bead_capacity=sum(st.n for st in self.states),
                             system_capacity=len(self.states), cell_capacity=max(cells, 1), cell_depth=cell_depth,
                             list_depth=list_depth, steps_per_graph=self.spg, device=self.states[0].pos.device,
                             srk_order=self.srk_order)
        for st in self.states:
            self.engine.admit(st)
        if self.cross is not None:
            self.engine.couple([st.slot for st in self.states], self.fixed, self.cross)
        for motor, chains, prm, hold in self.motors:
            self.engine.set_motors(self.states[motor].slot, self.states[chains].slot, prm, hold)

    def set_motors(self, motors):
        """Motor populations: (motor index, chain index, params, hold)."""
        same = len(motors) == len(self.motors) and all(
            a[:2] == b[:2] and np.array_equal(a[2], b[2]) and a[3] == b[3] for a, b in zip(motors, self.motors))
        if not same:
            for motor, _, _, _ in self.motors:
                self.engine.set_motors(self.states[motor].slot, -1, None)
            self.motors = list(motors)
            for motor, chains, prm, hold in self.motors:
                self.engine.set_motors(self.states[motor].slot, self.states[chains].slot, prm, hold)

    def set_cross(self, cross):
        if self.cross is None or not np.array_equal(cross, self.cross):
            self.cross = cross
            self.engine.couple([st.slot for st in self.states], self.fixed, cross)


def _srk2_populations(pops, status, sim, srk_order):
    """SRK2_force_calc over several populations (updates.py:146-247): each
    population is a system of one context; the systems step under one dt,
    rebuild their lists together and feel each other's WCA force
    (interpop_forces, SRK.py:229-245, 287-294).  Fixed populations
    (pop.fixed) never move.  Philox noise with the seed ``sim['seed'] + k``
    for population k."""
    cfg = _config
    dim = int(cfg.dim)
    if sim.get('gpu_noise', 'philox') != 'philox':
        raise NotImplementedError("several populations draw the Philox stream")
    precision = sim.get('gpu_precision', 'fp64')
    if any(getattr(p, "b_init_growing", False) for p in pops):
        precision = 'fp64'
    if len(pops) > 4:
        raise NotImplementedError("the GPU step couples at most 4 populations")
    seed = int(sim.get('seed', 0))
    params = [_pop_params(p, status, sim, seed + k) for k, p in enumerate(pops)]
    if not all(prm.calc_wca for prm in params):
        raise NotImplementedError("every population of the GPU step has the WCA force")
    # motors step even when they do not diffuse (D = 0 moves them by nothing)
    fixed = [bool(p.fixed) and not _is_motors(p) for p in pops]
    n = len(pops)
    cross = np.zeros((n, n, 4))
    for k, pk in enumerate(pops):
        for q, pq in enumerate(pops):
            if k != q and not fixed[k]:
                cross[k, q] = _cross_wca(pk, pq)
    # motor pushes (Chain_Collection.interactions, populations.py:276-287),
    # gated like every active force (SRK.py:84-87); the motors' cross entry
    # carries the chain-motor list radius
    motors = []
    for k, pk in enumerate(pops):
        for q, pq in enumerate(pops):
            if k == q or not _is_motors(pq) or _is_motors(pk):
                continue
            for name, prm in pk.interactions(pq) or []:
                if name != "motor_push":
                    continue
                prm = np.array(prm, dtype=np.float64)[:5].copy()
                if not status.b_calc_active_forces:
                    prm[3] = 0.0  # no motor attaches while active forces are off
                if any(m[0] == q for m in motors):
                    raise NotImplementedError("a motor population pushes one chain population on the GPU step")
                motors.append((q, k, prm, bool(getattr(pq, "b_motors_dont_diffuse_while_pushing", True))))
                cross[q, k] = [0.0, 0.0, 0.0, params[q].wca_params[3]]
    max_dt_usable = (status.next_save_time - status.t) if sim.get('save_state_every', -1) > 0 else -1.0
    max_steps = status.next_output_step - status.stepnum
    depth = getattr(pops[0], "_gcr_cell_depth",
                    default_depth(dim, max(cell_scale(prm) for prm in params)))
    ldepth = getattr(pops[0], "_gcr_list_depth", default_list_depth(dim))
    key = (tuple((p.total_pop, len(_pop_arrays(p, dim)[3])) for p in pops), tuple(fixed), dim, precision,
           float(cfg.Lx), depth, ldepth, srk_order)
    if motors and srk_order != 2:
        raise NotImplementedError("motors are stepped by the SRK2 branch on the GPU")
    g = getattr(pops[0], "_gcr_group", None)
    if g is None or g.key != key:
        if g is not None:
            g.engine.close()
        g = _GpuGroup(pops, sim, dim, precision, params, fixed, depth, ldepth, key, srk_order)
        pops[0]._gcr_group = g
    eng = g.engine
    for p, st, prm, h in zip(pops, g.states, params, g.host):
        h["pos"].numpy()[:] = p.pos
        st.pos.copy_(h["pos"], non_blocking=True)
        if not _is_motors(p):
            h["tan"].numpy()[:] = p.tangent_list
            st.tangent.copy_(h["tan"], non_blocking=True)
            st.rest_lengths.copy_(torch.from_numpy(np.asarray(p.rest_lengths, dtype=np.float64)))
        st.params = prm
    try:
        for st in g.states:
            eng.update_params(st)
    except GcrError as e:
        if e.code != -6:
            raise
        g.make_engine(eng.cfg.cell_depth, eng.cfg.list_depth)
        eng = g.engine
    g.set_cross(cross)
    g.set_motors(motors)

    done, elapsed, dt = 0, 0.0, float(status.dt)
    lead = fixed.index(False)  # the first moving population reports status (shared_arr[0])
    while True:
        left = max_steps - done if max_steps >= 0 else -1
        lim = max_dt_usable - elapsed if max_dt_usable >= 0 else -1.0
        eng.call_begin_many([st.slot for st in g.states], left, [dt] * n, lim)
        if left >= 0 and max_dt_usable < 0:
            eng.run(left, sync_every=0)
        else:
            eng.run(left if left >= 0 else (1 << 62), sync_every=1)
        sts = [eng.status(st.slot) for st in g.states]
        res = sts[lead]
        done += int(res['steps_done'])
        elapsed += res['dt_used']
        dt = res['dt']
        flags = 0
        for r in sts:
            flags |= r['flags']
        grow_cells = bool(flags & FLAG_CELL_OVERFLOW) and eng.cfg.cell_depth < MAX_DEPTH
        grow_lists = bool(flags & FLAG_LIST_OVERFLOW) and eng.cfg.list_depth < MAX_LIST_DEPTH
        if not (grow_cells or grow_lists) or done == max_steps or (max_dt_usable >= 0 and elapsed >= max_dt_usable):
            break
        depth = min(MAX_DEPTH, 2 * eng.cfg.cell_depth) if grow_cells else eng.cfg.cell_depth
        ldepth = min(MAX_LIST_DEPTH, 2 * eng.cfg.list_depth) if grow_lists else eng.cfg.list_depth
        pops[0]._gcr_cell_depth, pops[0]._gcr_list_depth = depth, ldepth
        for st, r in zip(g.states, sts):
            st.params.step = int(r['step'])
        g.make_engine(depth, ldepth)
        g.key = key[:5] + (depth, ldepth, srk_order)
        eng = g.engine
    for st, h in zip(g.states, g.host):
        h["pos"].copy_(st.pos, non_blocking=True)
        h["pos1"].copy_(st.pos1, non_blocking=True)
        h["tan"].copy_(st.tangent, non_blocking=True)
        h["frc"].copy_(st.forces, non_blocking=True)
    torch.cuda.synchronize(eng.device)
    for p, h, fx in zip(pops, g.host, fixed):
        if fx:
            continue
        p.pos[:] = h["pos"].numpy()
        p.pos1[:] = h["pos1"].numpy()
        if _is_motors(p):
            continue
        p.tangent_list[:] = h["tan"].numpy()
        p.forces[:] = h["frc"].numpy()
    if g.motors:
        for p, st in zip(pops, g.states):
            p.where_active[:] = eng.where_active(st.slot).cpu().numpy()
    status.dt = dt
    status.dt_used = elapsed
    status.stepnum += done
    status.t += status.dt_used
    status.max_forces_strength = res['max_forces_strength']
    status.update_grid_list_counter = max(
        1, (done + status.update_grid_list_counter) % cfg.n_steps_update_grid_list)
    status.gpu_flags = flags
    return None
