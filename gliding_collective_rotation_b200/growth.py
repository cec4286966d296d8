"""The reference's init-grow protocol for systems stepped on the device.

Chains start compressed (bonds of ``a_init_factor`` times the rest length,
populations.py:530-557) and grow to their rest length over a time
``t_init_grow`` before the run proper starts at t = 0.  The schedule is the
reference's:

* ``set_init_grow`` (populations.py:134-135, 234-236, 294-296, 376-389):
  n_nearby_beads_dont_repel = -1 (no pair force within a chain), kappa = 0,
  k = 1, WCA_shift = 0, D = 0, v0 = 0, and no active forces
  (control.py:173-174), RK_cheat_factor = 1;
* every ``growing_stepskip`` steps, ``control.early_time_procedures``
  (control.py:153-219) sets, from progress = max((t - t_start) / t_init_grow,
  epsilon):
  - progress < 0.25: repulsion radius repel_d_max * progress / 0.25, no
    rigid-rod projection;
  - progress < 1: full radius, kappa = 10, projection factor
    max(0.025, the population's own factor);
  - rest lengths a * a_init_factor ** (1 - progress ** 0.1);
  - WCA parameters packed at the current radius (``engine.wca_params``,
    the layout of the reference's make_WCA_params), with the
    pair cutoff at the potential minimum while growing
    (updates.interpop_forces, updates.py:304-310);
* once t > 0, ``end_init_grow`` (populations.py:137-140, 238-240, 297-299,
  391-403) restores every parameter.

``grow_params`` is that schedule as a pure function; ``init_grow`` runs it
for a list of ``SystemSpec`` in one FP64 ``Batch`` (radii down to 1e-8 put
the WCA prefactors below the FP32 range) and returns the grown specs, which
may then be stepped at any precision.  Every step, the rigid-rod projection
included, runs on the device; the host only sets parameters between calls,
as the reference's own loop does.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

import numpy as np
import torch

from .batch import Batch
from .engine import wca_params


@dataclass
class GrowSettings:
    """Growth settings (defaults.py:159-166, 252-253; config.py:78)."""
    t_init_grow: float = 1.0
    a_init_factor: float = 1e-8
    growing_stepskip: int = 10
    epsilon: float = 1e-8
    dt0: float | None = None      # dt of the first step (default: 1e-4 dtmax, defaults.py:59)


@dataclass
class GrowthConstants:
    """The population constants the schedule reads (its saved values)."""
    repel_d_max: float
    WCA_epsilon: float
    WCA_shift: float
    LJ_cutoff_factor: float
    reference_rest_length: float
    longest_chain_length: int
    rigid_rod_projection_factor: float = 0.0

    @classmethod
    def from_spec(cls, spec, WCA_epsilon=None, LJ_cutoff_factor=None):
        """Read the constants off a spec's packed parameters; give
        ``WCA_epsilon`` and ``LJ_cutoff_factor`` to avoid the round trip
        through ``wca_params``."""
        p = spec.params
        r = float(p.radius)
        shift = float(p.wca_params[2])
        eps = WCA_epsilon if WCA_epsilon is not None else float(p.wca_params[0]) / (12 * r ** 6)
        lj = LJ_cutoff_factor if LJ_cutoff_factor is not None else (float(p.wca_params[3]) + shift) / r
        rest = np.asarray(spec.rest_lengths, dtype=np.float64)
        longest = int(np.max(np.bincount(np.asarray(spec.chain_id))))
        return cls(repel_d_max=r, WCA_epsilon=float(eps), WCA_shift=shift, LJ_cutoff_factor=float(lj),
                   reference_rest_length=float(rest[0]), longest_chain_length=longest,
                   rigid_rod_projection_factor=float(p.rigid_rod))


def grow_progress(t, t_start, settings):
    """control.py:180-181"""
    return max((t - t_start) / settings.t_init_grow, settings.epsilon)


def grow_params(base, c, t, t_start, settings):
    """The parameters of one growth call at time ``t`` (control.py:176-216):
    ``(params, rest_length, active)``.  ``base`` is the system's own
    ``SystemParams``; the returned copy keeps its step counter, seed, dtmax,
    max_dist_per_step, Dr, skin and cell factor."""
    prog = grow_progress(t, t_start, settings)
    p = copy.deepcopy(base)
    # set_init_grow
    k, kappa = 1.0, 0.0
    radius = c.repel_d_max
    rigid = c.rigid_rod_projection_factor
    if c.longest_chain_length != 1:
        init_repel_frac, init_rigid_frac = 0.25, 1.0
        repel_portion_frac = min(init_repel_frac, prog) / init_repel_frac
        radius = c.repel_d_max
        rigid = max(0.025, c.rigid_rod_projection_factor)
        if prog < init_repel_frac:
            rigid = 0
            radius = c.repel_d_max * repel_portion_frac
        elif prog < init_rigid_frac:
            radius = c.repel_d_max
            kappa = 10
        else:
            rigid = 0.0
            kappa = float(base.spring_params[1])
            k = float(base.spring_params[0])
    wca = wca_params(radius, c.WCA_epsilon, 0.0, c.LJ_cutoff_factor)
    if wca[0] != 0:
        # repulsive only while growing: cutoff at the potential minimum
        wca[3] = (wca[1] / wca[0]) ** (1 / 6)
    rest = c.reference_rest_length * (settings.a_init_factor ** (1 - prog ** 0.1))
    spring = np.array(base.spring_params, dtype=np.float64)
    spring[0], spring[1] = k, kappa
    p.spring_params = spring
    p.wca_params = wca
    p.radius = float(radius)
    p.rigid_rod = float(rigid)
    p.n_nearby = -1
    p.D = 0.0
    p.active_params = np.array([0.0, base.active_params[1], base.active_params[2]])
    p.self_propel = False
    p.rk_cheat = 1.0
    return p, rest, False


@dataclass
class GrowResult:
    specs: list          # grown specs: positions, tangents, step counters after growth
    t: np.ndarray        # time of each system after its last growth call (> 0)
    dt: np.ndarray       # dt each system carries into its next call
    steps: np.ndarray    # growth steps per system
    calls: int           # growth calls (parameter updates) of the batch


def init_grow(specs, settings=None, constants=None, device=None, max_calls=1_000_000, **batch_kw):
    """Grow every system of ``specs`` (placed with ``a_init_factor``-short
    bonds) on the device; returns a ``GrowResult``.  ``constants`` defaults
    to ``GrowthConstants.from_spec`` of each spec."""
    settings = settings or GrowSettings()
    consts = constants or [GrowthConstants.from_spec(s) for s in specs]
    n_sys = len(specs)
    base = [copy.deepcopy(s.params) for s in specs]
    work = []
    for s in specs:
        w = copy.copy(s)
        w.params = copy.deepcopy(s.params)
        w.rest_lengths = np.array(s.rest_lengths, dtype=np.float64)
        work.append(w)
    batch = Batch(work, precision="fp64", device=device, **batch_kw)
    t_start = np.full(n_sys, -settings.t_init_grow)
    t = t_start.copy()
    growing = np.full(n_sys, settings.t_init_grow > 0)
    steps = np.zeros(n_sys, dtype=np.int64)
    dts = [settings.dt0 if settings.dt0 is not None else 1e-4 * b.dtmax for b in base]
    n_ch = [len(s.rest_lengths) for s in specs]
    calls = 0
    try:
        while growing.any() and calls < max_calls:
            # control.early_time_procedures: growth ends once t > 0
            rest_all = []
            for i, st in enumerate(batch.states):
                if growing[i] and t[i] > 0:
                    growing[i] = False
                if growing[i]:
                    p, rest, _ = grow_params(base[i], consts[i], t[i], t_start[i], settings)
                    p.step = st.params.step
                    rest_all.append(np.full(n_ch[i], rest))
                else:
                    p = copy.deepcopy(base[i])
                    p.step = st.params.step
                    rest_all.append(np.asarray(specs[i].rest_lengths, dtype=np.float64))
                st.params = p
                batch.specs[i].params = p
                batch.engine.update_params(st)
            if not growing.any():
                break
            batch.big["rest"].copy_(torch.from_numpy(np.concatenate(rest_all)))
            left = [settings.growing_stepskip if g else 0 for g in growing]
            slots = [st.slot for st in batch.states]
            batch.engine.call_begin_many(slots, left, dts if calls == 0 else batch._dts())
            batch.run(settings.growing_stepskip)
            elapsed = np.zeros(n_sys)
            regrows = 0
            while True:
                sts = batch.statuses()
                for i, s in enumerate(sts):
                    left[i] -= s["steps_done"]
                    steps[i] += s["steps_done"]
                    elapsed[i] += s["dt_used"]
                    batch.states[i].params.step = s["step"]
                if not batch.overflowed(sts) or regrows >= 6:
                    break
                batch.regrow()
                regrows += 1
                batch.engine.call_begin_many(slots, left, batch._dts())
                batch.run(max(left))
            for i, s in enumerate(sts):
                if s["flags"] & 2:
                    raise FloatingPointError(f"system {i}: non-finite state while growing")
            t += np.where(growing, elapsed, 0.0)
            calls += 1
        sts = batch.statuses()
        for i, st in enumerate(batch.states):
            p = copy.deepcopy(base[i])
            p.step = sts[i]["step"]
            st.params = p
        out = []
        for i, st in enumerate(batch.states):
            g = copy.copy(specs[i])
            g.pos = st.pos.cpu().numpy().copy()
            g.tangent = st.tangent.cpu().numpy().copy()
            g.params = copy.deepcopy(base[i])
            g.params.step = int(sts[i]["step"])
            out.append(g)
        return GrowResult(specs=out, t=t, dt=np.array([s["dt"] for s in sts]), steps=steps, calls=calls)
    finally:
        batch.close()


def compressed_chains(spec, a_init_factor=1e-8):
    """``spec`` with its chains shrunk about each head bead to
    ``a_init_factor`` times their bond vectors (the placement of
    Chain_Collection.random_initialization, populations.py:530-557)."""
    L = float(spec.params.L)
    pos = np.asarray(spec.pos, dtype=np.float64)
    chain = np.asarray(spec.chain_id)
    heads = np.concatenate(([0], np.flatnonzero(np.diff(chain)) + 1))
    head_of = heads[np.searchsorted(heads, np.arange(len(pos)), side="right") - 1]
    d = pos - pos[head_of]
    d -= L * np.round(d / L)
    out = copy.copy(spec)
    out.pos = np.mod(pos[head_of] + a_init_factor * d, L)
    return out
