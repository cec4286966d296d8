"""Many independent systems of different sizes advanced together.

All systems of a ``Batch`` share one ``Engine`` (one ``libgcr`` context), so
one captured CUDA graph of persistent kernels steps every system: the
kernels walk a per-system tile table in device memory, each system keeps its
own parameters, adaptive dt, step counter and Philox seed.  The bead state of
all systems lives in a few large device tensors (per-system views), so the
host <-> device copies of a call are single bulk transfers.

The plain path (``PlainRunner``) advances the same systems one system per
launch sequence, as the drop-in does; it is the baseline the batched path is
measured against.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ._lib import FLAG_CELL_OVERFLOW, FLAG_LIST_OVERFLOW, FLAG_NEXT_OVERFLOW
from .engine import Engine, SystemState, default_config, default_skin, footprint

OVERFLOW = FLAG_CELL_OVERFLOW | FLAG_NEXT_OVERFLOW | FLAG_LIST_OVERFLOW
MAX_DEPTH = 128
MAX_LIST_DEPTH = 1024


def default_depth(dim, cell_factor):
    """Slots per GPU cell: 16 (2D) / 32 (3D) for a cell of side r_cut, scaled
    with the cell volume and rounded up to a power of two."""
    base = 16 if dim == 2 else 32
    want = base * max(1.0, cell_factor) ** dim
    d = 8
    while d < want and d < MAX_DEPTH:
        d *= 2
    return d


def cell_scale(params):
    """GPU cell side over the pair cutoff: (r_cut + skin) * cell_factor / r_cut."""
    rc = float(params.wca_params[3])
    skin = params.skin if params.skin is not None else default_skin(rc)
    return max(1.0, params.cell_factor) * (rc + max(0.0, skin)) / rc


def default_list_depth(dim):
    return 32 if dim == 2 else 96


def _views(specs, precision, device, srk_order=2):
    ft = torch.float64 if precision == "fp64" else torch.float32
    dim = specs[0].dim
    n_tot = sum(s.n for s in specs)
    c_tot = sum(len(s.rest_lengths) for s in specs)
    big = {
        "pos": torch.empty((n_tot, dim), dtype=torch.float64, device=device),
        "pos1": torch.zeros((n_tot, dim), dtype=torch.float64, device=device),
        "tangent": torch.empty((n_tot, dim), dtype=ft, device=device),
        "forces": torch.zeros((n_tot, dim), dtype=ft, device=device),
        "chain_id": torch.empty(n_tot, dtype=torch.int32, device=device),
        "rest": torch.empty(c_tot, dtype=torch.float64, device=device),
    }
    if srk_order == 4:
        big["forces_aux"] = torch.zeros((n_tot, dim), dtype=ft, device=device)
    h_pos = np.concatenate([s.pos for s in specs])
    h_tan = np.concatenate([s.tangent for s in specs])
    h_chain = np.concatenate([s.chain_id for s in specs]).astype(np.int32)
    h_rest = np.concatenate([s.rest_lengths for s in specs])
    big["pos"].copy_(torch.from_numpy(h_pos))
    # pos1 starts at pos: a motor attached in its first predictor keeps its
    # previous pos1 (SRK.py:389-395)
    big["pos1"].copy_(big["pos"])
    big["tangent"].copy_(torch.from_numpy(h_tan))
    big["chain_id"].copy_(torch.from_numpy(h_chain))
    big["rest"].copy_(torch.from_numpy(h_rest))
    states, bo, co = [], 0, 0
    for s in specs:
        n, nc = s.n, len(s.rest_lengths)
        states.append(SystemState(pos=big["pos"][bo:bo + n], pos1=big["pos1"][bo:bo + n],
                                  tangent=big["tangent"][bo:bo + n], forces=big["forces"][bo:bo + n],
                                  chain_id=big["chain_id"][bo:bo + n], rest_lengths=big["rest"][co:co + nc],
                                  params=s.params,
                                  forces_aux=big["forces_aux"][bo:bo + n] if srk_order == 4 else None))
        bo += n
        co += nc
    return big, states


class Batch:
    """Systems of one dimension and precision resident in one context.

    Each system's parameters are its spec's own ``params`` object, shared:
    ``relax``/``set_adaptive`` write the dt rule into it and ``regrow`` the
    step counter, so the specs follow the batch (pass copies to keep the
    originals)."""

    def __init__(self, specs, precision="mixed", device=None, steps_per_graph=10, cell_depth=None,
                 block_beads=128, block_cells=256, stream=None, ctas_per_sm=0, list_depth=None, srk_order=2,
                 pair_mode=0):
        if not specs:
            raise ValueError("empty batch")
        dims = {s.dim for s in specs}
        if len(dims) != 1:
            raise ValueError("a batch holds systems of one dimension")
        self.dim = dims.pop()
        self.specs = specs
        self.precision = precision
        self.device = torch.device(device or "cuda")
        if cell_depth is None:
            cell_depth = default_depth(self.dim, max(cell_scale(s.params) for s in specs))
        self.cell_depth = cell_depth
        self.list_depth = list_depth or default_list_depth(self.dim)
        self._engine_kw = dict(block_beads=block_beads, block_cells=block_cells, steps_per_graph=steps_per_graph,
                               stream=stream, ctas_per_sm=ctas_per_sm, pair_mode=pair_mode)
        self.n_beads = sum(s.n for s in specs)
        self.srk_order = srk_order
        self.big, self.states = _views(specs, precision, self.device, srk_order)
        torch.cuda.synchronize(self.device)
        self.engine = None
        self._carry_dt = None  # dts to hand to the next call after a regrow
        self.series_buf = None
        self.groups = []  # coupled populations: (member indices, fixed flags, cross WCA parameters)
        self.motors = []  # motor populations: (motor index, chain index, params, hold)
        self._img_carry = [None] * len(specs)  # L * images crossed before the last regrow
        self._make_engine()

    def _make_engine(self):
        cfg = default_config(self.dim, self.precision, cell_depth=self.cell_depth, list_depth=self.list_depth,
                             srk_order=self.srk_order)
        cells = sum(footprint(cfg, s.params, s.n, len(s.rest_lengths))[0] for s in self.specs)
        self.engine = Engine(self.dim, self.precision, device=self.device, bead_capacity=self.n_beads,
                             system_capacity=len(self.specs), cell_capacity=max(cells, 1),
                             cell_depth=self.cell_depth, list_depth=self.list_depth, srk_order=self.srk_order,
                             **self._engine_kw)
        for st in self.states:
            self.engine.admit(st)
        for g in self.groups:
            self._couple(*g)
        for m in self.motors:
            self._set_motors(*m)

    def set_motors(self, motor, chains, params, hold=True):
        """System ``motor`` (single beads, coupled with ``chains`` by
        ``couple`` whose cross r_cut of motor from chains is the list radius)
        is a motor population pushing the beads of system ``chains``
        (forces.calc_motor_push, forces.py:248-283): params =
        [motor_max_dist_sq, b_one_motor_per_bead, imparts_force, k_on,
        k_off]; ``hold``: b_motors_dont_diffuse_while_pushing.  Survives a
        regrow."""
        m = (int(motor), int(chains), np.asarray(params, dtype=np.float64), bool(hold))
        self._set_motors(*m)
        self.motors.append(m)

    def _set_motors(self, motor, chains, params, hold):
        self.engine.set_motors(self.states[motor].slot, self.states[chains].slot, params, hold)

    def where_active(self, i):
        """pop.where_active of system i after the last step (int32 numpy)."""
        return self.engine.where_active(self.states[i].slot).cpu().numpy()

    def couple(self, members, fixed, cross_wca):
        """Step the systems ``members`` (indices into this batch, in the
        reference's population order) as the populations of one box, as
        ``updates.SRK2_force_calc`` steps a list of populations
        (updates.py:146-247): one dt per step, joint list builds, and the WCA
        force ``cross_wca[i][j]`` = [p0, p1, shift, r_cut] of population j on
        population i (``interpop_forces``, updates.py:274-312).  ``fixed[i]``:
        population i never moves (pop.fixed).  The coupling survives a regrow."""
        g = (list(members), [bool(f) for f in fixed], np.asarray(cross_wca, dtype=np.float64))
        self._couple(*g)
        self.groups.append(g)

    def _couple(self, members, fixed, cross_wca):
        self.engine.couple([self.states[i].slot for i in members], fixed, cross_wca)

    def overflowed(self, statuses=None):
        statuses = statuses if statuses is not None else self.statuses()
        return any(s["flags"] & OVERFLOW for s in statuses)

    def regrow(self):
        """Double the slots per GPU cell or per neighbour list after an
        overflow (the reference doubles its list depths the same way,
        updates.py:257-267) and re-admit every system; step counters carry
        over, so the noise stream goes on."""
        sts = self.statuses()
        flags = 0
        for st, s in zip(self.states, sts):
            st.params.step = s["step"]
            flags |= s["flags"]
        # a re-admitted system starts from dtmax: its dt is handed over by the next call
        self._carry_dt = [s["dt"] for s in sts]
        # the new context counts images from 0: keep those crossed so far
        for i, st in enumerate(self.states):
            img = self.engine.unwrapped(st.slot) - st.pos
            self._img_carry[i] = img if self._img_carry[i] is None else self._img_carry[i] + img
        cell = bool(flags & FLAG_CELL_OVERFLOW)
        lst = bool(flags & FLAG_LIST_OVERFLOW) or not cell
        if (cell and self.cell_depth >= MAX_DEPTH) or (lst and self.list_depth >= MAX_LIST_DEPTH):
            bad = [(x.name if hasattr(x, "name") else i, s["flags"]) for i, (x, s) in enumerate(zip(self.specs, sts))
                   if s["flags"]]
            raise RuntimeError(f"GPU cell or list depth limit reached (cell depth {self.cell_depth}, list depth "
                               f"{self.list_depth}; flags {bad[:8]})")
        self.engine.close()
        if cell:
            self.cell_depth *= 2
        if lst:
            self.list_depth *= 2
        self._make_engine()

    # -- calls -------------------------------------------------------------------
    def begin(self, max_steps, dt=None, max_dist_per_step=None, max_dt_usable=-1.0, series_every=0):
        """Arm every system for the next run (one SRK2_force_calc call each).
        Without `dt` each system keeps the dt its last step chose, as the
        reference's status.dt carries from call to call.  With
        `series_every`, the device records the order parameters of every
        system after every `series_every` steps of the call (``series``)."""
        for st in self.states:
            if max_dist_per_step is not None and st.params.max_dist_per_step != max_dist_per_step:
                st.params.max_dist_per_step = max_dist_per_step
                self.engine.update_params(st)
        self.series_buf = None
        if series_every > 0:
            rows = int(np.max(max_steps)) // series_every + 1
            self.series_buf = torch.zeros((len(self.states), rows, 5), dtype=torch.float64, device=self.device)
        self.engine.call_begin_many([st.slot for st in self.states], max_steps, self._dts(dt), max_dt_usable,
                                    series=self.series_buf, series_every=series_every)

    def series(self):
        """Rows (step, time in the call, P, S, director angle) recorded on
        the device in the last call, per system."""
        if self.series_buf is None:
            return [np.zeros((0, 5)) for _ in self.states]
        rows = [s["series_rows"] for s in self.statuses()]
        buf = self.series_buf.cpu().numpy()
        return [buf[i, :r].copy() for i, r in enumerate(rows)]

    def _dts(self, dt=None):
        """Per-system dt of the next call: `dt`, else the dts carried over a
        regrow, else 0 (each system keeps its own)."""
        if dt is not None:
            return [dt] * len(self.states)
        carry, self._carry_dt = self._carry_dt, None
        return carry if carry is not None else [0.0] * len(self.states)

    def set_adaptive(self, on=True):
        """The reference's adaptive dt (dtmax = the system's dt,
        max_dist_per_step of config.grid_list_setup, SRK.py:323-353) or a
        fixed dt (max_dist_per_step = inf) for every system."""
        for st, spec in zip(self.states, self.specs):
            want = spec.relax_mdps if on else math.inf
            if st.params.max_dist_per_step != want:
                st.params.max_dist_per_step = want
                self.engine.update_params(st)

    def run(self, max_steps, sync_every=0):
        self.engine.run(max_steps, sync_every)

    def relax(self, max_steps=2000, chunk=200, adaptive_after=False):
        """Untimed warm-up under the reference's adaptive dt (dtmax = the
        system's dt, max_dist_per_step from grid_list_setup) until every
        system takes full steps or `max_steps` have run; removes the overlaps
        of random placement.  Afterwards the systems keep the adaptive rule
        (`adaptive_after`) or take a fixed dt."""
        done = 0
        first = True
        while done < max_steps:
            self.set_adaptive(True)
            dts = [s.dt for s in self.specs] if first else self._dts()
            first = False
            self.engine.call_begin_many([st.slot for st in self.states], chunk, dts)
            self.engine.run(chunk)
            done += chunk
            sts = self.statuses()
            if self.overflowed(sts):
                self.regrow()
                continue
            if all(s["dt"] >= spec.dt * (1 - 1e-12) for s, spec in zip(sts, self.specs)):
                break
        self.set_adaptive(adaptive_after)
        return done

    def statuses(self):
        return self.engine.statuses([st.slot for st in self.states])

    def run_checked(self, steps, max_regrow=6):
        """Run `steps` steps of every system; after a cell or list overflow
        regrow and run the remaining steps of the systems that stopped.  The
        returned statuses count in ``steps_done`` the steps of all calls."""
        self.begin(steps)
        self.run(steps)
        done = [0] * len(self.states)
        regrows = 0
        while True:
            sts = self.statuses()
            done = [d + s["steps_done"] for d, s in zip(done, sts)]
            if not self.overflowed(sts) or regrows >= max_regrow:
                break
            left = [steps - d for d in done]
            self.regrow()
            regrows += 1
            slots = [st.slot for st in self.states]
            self.engine.call_begin_many(slots, left, self._dts())
            self.run(max(left))
        for s, d in zip(sts, done):
            s["steps_done"] = d
        return sts

    def order_params(self):
        return np.array([self.engine.order_params(st.slot) for st in self.states])

    def unwrapped(self):
        """Per system, its positions plus the periodic images its beads
        crossed since the batch was made (float64 [n, dim] on the device):
        mean-squared displacements without host round trips."""
        out = []
        for st, carry in zip(self.states, self._img_carry):
            u = self.engine.unwrapped(st.slot)
            out.append(u if carry is None else u + carry)
        return out

    def msd(self, reference):
        """Mean-squared displacement per system from ``reference`` (a list of
        unwrapped positions, e.g. an earlier ``unwrapped()``), in FP64."""
        return np.array([float(((u - r) ** 2).sum(dim=1).mean()) for u, r in zip(self.unwrapped(), reference)])

    def close(self):
        self.engine.close()


class PlainRunner:
    """The same systems, one context and one launch sequence per system."""

    def __init__(self, specs, precision="mixed", device=None, steps_per_graph=10, cell_depth=None):
        # one stream for every context: launches of different systems do not overlap
        self.stream = torch.cuda.Stream(device=device)
        self.batches = [Batch([s], precision, device, steps_per_graph, cell_depth, stream=self.stream)
                        for s in specs]
        self.n_beads = sum(s.n for s in specs)

    def copy_state_from(self, batch):
        for b, st in zip(self.batches, batch.states):
            b.states[0].pos.copy_(st.pos)
            b.states[0].tangent.copy_(st.tangent)
        torch.cuda.synchronize()

    def begin(self, max_steps):
        for b in self.batches:
            b.begin(max_steps)

    def run(self, max_steps):
        for b in self.batches:
            b.run(max_steps)

    def synchronize(self):
        for b in self.batches:
            b.engine.synchronize()

    def close(self):
        for b in self.batches:
            b.close()
