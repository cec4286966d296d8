"""Torch-facing wrapper of one ``libgcr`` context.

State of every system lives in torch CUDA tensors that the context binds by
device pointer (``gcr_admit``); the context owns only its scratch.  An
``Engine`` can hold one system (the drop-in ``SRK2_force_calc`` path) or many
systems of different sizes (batched sweeps, serving).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import Call, Config, GcrError, Status, SystemBuffers, SystemDesc, check

PRECISIONS = {"fp64": _lib.GCR_FP64, "mixed": _lib.GCR_MIXED}


def wca_params(radius, epsilon, shift, cutoff_factor):
    """The packed pair parameters the step reads, in the reference's layout
    (the array populations.make_WCA_params returns, populations.py:48-58):
    [12 eps r^6, 12 eps r^12, shift, cutoff], the cutoff being
    cutoff_factor * r - shift, for the rule coeff = ds^-4 (p0 - p1 ds^-3)
    of forces.WCA."""
    r6 = float(radius) ** 6
    p0 = 12.0 * r6 * float(epsilon)
    return np.array([p0, p0 * r6, float(shift), float(cutoff_factor) * float(radius) - float(shift)])


def default_skin(r_cut):
    """Verlet skin for a pair cutoff: 0.2 r_cut + 0.1, within [0.2, 1].  A
    wider skin means rarer list builds but longer lists; measured on B200 the
    best was 0.3 for r_cut = 1 (WCA sweep) and 0.5 for r_cut = 2.23 (LJ)."""
    return min(1.0, max(0.2, 0.2 * float(r_cut) + 0.1))


@dataclass
class SystemParams:
    """One system's parameters, packed the way the reference packs them.

    ``spring_params`` = Chain_Collection.spring_params() (populations.py:345-353),
    ``wca_params`` = make_WCA_params(...) (populations.py:48-58),
    ``active_params`` = Chain_Collection.active_params() (populations.py:355-358).
    """
    L: float
    spring_params: np.ndarray
    wca_params: np.ndarray
    active_params: np.ndarray
    D: float
    Dr: float
    radius: float
    n_nearby: int
    calc_springs: bool = True
    calc_wca: bool = True
    self_propel: bool = True
    dtmax: float = 1e-3
    max_dist_per_step: float = math.inf
    rk_cheat: float = 1.0
    seed: int = 0
    step: int = 0
    cell_factor: float = 1.0
    skin: float | None = None    # Verlet skin of the neighbour list; None: default_skin(r_cut)
    rigid_rod: float = 0.0       # rigid_rod_projection_factor (updates.py:347-499); 0: off

    def desc(self, n_beads, n_chains):
        d = SystemDesc()
        d.n_beads, d.n_chains, d.L = int(n_beads), int(n_chains), float(self.L)
        for i in range(6):
            d.spring_params[i] = float(self.spring_params[i])
        for i in range(4):
            d.wca_params[i] = float(self.wca_params[i])
        for i in range(3):
            d.active_params[i] = float(self.active_params[i])
        d.calc_springs, d.calc_wca = int(bool(self.calc_springs)), int(bool(self.calc_wca))
        d.self_propel, d.n_nearby = int(bool(self.self_propel)), int(self.n_nearby)
        d.D, d.Dr, d.radius = float(self.D), float(self.Dr), float(self.radius)
        d.dtmax, d.max_dist_per_step, d.rk_cheat = float(self.dtmax), float(self.max_dist_per_step), \
            float(self.rk_cheat)
        d.seed, d.step, d.cell_factor = int(self.seed) & (2 ** 64 - 1), int(self.step), float(self.cell_factor)
        d.skin = float(self.skin if self.skin is not None else default_skin(self.wca_params[3]))
        d.rigid_rod = float(self.rigid_rod)
        return d


@dataclass
class SystemState:
    """Device state of one system (bead order, chains contiguous)."""
    pos: torch.Tensor            # float64 [n, d]
    pos1: torch.Tensor           # float64 [n, d]
    tangent: torch.Tensor        # float64 | float32 [n, d]
    forces: torch.Tensor         # float64 | float32 [n, d]
    chain_id: torch.Tensor       # int32 [n]
    rest_lengths: torch.Tensor   # float64 [n_chains]
    params: SystemParams
    slot: int = -1
    extra: dict = field(default_factory=dict)
    forces_aux: torch.Tensor | None = None  # SRK4: force of the last stage (pop.forces_aux)

    @property
    def n(self):
        return self.pos.shape[0]

    @property
    def n_chains(self):
        return self.rest_lengths.shape[0]

    @staticmethod
    def from_host(pos, tangent, chain_id, rest_lengths, params, precision="fp64", device="cuda", srk_order=2):
        ft = torch.float64 if precision == "fp64" else torch.float32
        pos_t = torch.as_tensor(np.ascontiguousarray(pos), dtype=torch.float64, device=device)
        chain = np.asarray(chain_id)
        if np.any(np.diff(chain) < 0):
            raise ValueError("chains must be contiguous, increasing ranges of beads")
        return SystemState(
            pos=pos_t.clone(),
            # pos1 starts at pos: a motor that is attached in its first
            # predictor keeps its previous pos1 (SRK.py:389-395)
            pos1=pos_t.clone(),
            tangent=torch.as_tensor(np.ascontiguousarray(tangent), dtype=ft, device=device).clone(),
            forces=torch.zeros(pos_t.shape, dtype=ft, device=device),
            chain_id=torch.as_tensor(chain.astype(np.int32), device=device),
            rest_lengths=torch.as_tensor(np.asarray(rest_lengths, dtype=np.float64), device=device).clone(),
            params=params,
            forces_aux=torch.zeros(pos_t.shape, dtype=ft, device=device) if srk_order == 4 else None)

    def buffers(self):
        b = SystemBuffers()
        b.pos, b.pos1 = self.pos.data_ptr(), self.pos1.data_ptr()
        b.tangent, b.forces = self.tangent.data_ptr(), self.forces.data_ptr()
        b.chain_id, b.rest_lengths = self.chain_id.data_ptr(), self.rest_lengths.data_ptr()
        b.forces_aux = self.forces_aux.data_ptr() if self.forces_aux is not None else None
        return b


def default_config(dim, precision="fp64", bead_capacity=1 << 20, system_capacity=1,
                   cell_capacity=None, cell_depth=None, block_beads=256, block_cells=256,
                   steps_per_graph=10, ctas_per_sm=0, list_depth=0, srk_order=2, pair_mode=0):
    cfg = Config()
    cfg.dim = dim
    cfg.precision = PRECISIONS[precision]
    cfg.bead_capacity = int(bead_capacity)
    cfg.system_capacity = int(system_capacity)
    cfg.cell_capacity = int(cell_capacity if cell_capacity is not None else 4 * bead_capacity)
    cfg.cell_depth = int(cell_depth if cell_depth is not None else (16 if dim == 2 else 32))
    if cfg.cell_depth not in (8, 16, 32, 64, 128):
        raise ValueError("cell_depth must be 8, 16, 32, 64 or 128")
    cfg.block_beads, cfg.block_cells = int(block_beads), int(block_cells)
    cfg.steps_per_graph, cfg.ctas_per_sm = int(steps_per_graph), int(ctas_per_sm)
    cfg.list_depth = int(list_depth)
    if srk_order not in (2, 4):
        raise ValueError("srk_order must be 2 or 4")
    cfg.srk_order = int(srk_order)
    # pair forces: 0 list kernel, 1 list walk inside the stage kernels (same
    # bits), 2 cell-staged kernel (same pairs, another summation order)
    if pair_mode not in (0, 1, 2):
        raise ValueError("pair_mode must be 0, 1 or 2")
    cfg.pair_mode = int(pair_mode)
    return cfg


def footprint(cfg, params, n_beads, n_chains):
    cells, byts = C.c_int64(), C.c_int64()
    check(_lib.load().gcr_footprint(C.byref(cfg), C.byref(params.desc(n_beads, n_chains)), C.byref(cells),
                                    C.byref(byts)))
    return cells.value, byts.value


class Engine:
    """A ``gcr_ctx``: scratch for up to ``system_capacity`` resident systems."""

    def __init__(self, dim, precision="fp64", device=None, stream=None, **cfg_kwargs):
        if not torch.cuda.is_available():
            raise GcrError(-2, "no CUDA device: the gcr hot path runs on the GPU only")
        self.lib = _lib.load()
        self.dim = dim
        self.precision = precision
        self.device = torch.device(device or "cuda")
        self.cfg = default_config(dim, precision, **cfg_kwargs)
        self.stream = stream or torch.cuda.Stream(device=self.device)
        self._ctx = C.c_void_p()
        with torch.cuda.device(self.device):
            check(self.lib.gcr_create(C.byref(self.cfg), C.c_void_p(self.stream.cuda_stream),
                                      C.byref(self._ctx)))
        self.systems = {}

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.gcr_destroy(self._ctx)
            self._ctx = C.c_void_p()
            self.systems.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- systems -------------------------------------------------------------
    def admit(self, st: SystemState):
        torch.cuda.current_stream(self.device).synchronize()
        slot = C.c_int32()
        check(self.lib.gcr_admit(self._ctx, C.byref(st.params.desc(st.n, st.n_chains)), C.byref(st.buffers()),
                                 C.byref(slot)))
        st.slot = slot.value
        self.systems[st.slot] = st
        return st.slot

    def try_admit(self, st: SystemState):
        try:
            return self.admit(st)
        except GcrError as e:
            if e.code == -6:
                return None
            raise

    def evict(self, slot):
        check(self.lib.gcr_evict(self._ctx, int(slot)))
        st = self.systems.pop(int(slot), None)
        if st is not None:
            st.slot = -1

    def update_params(self, st: SystemState):
        check(self.lib.gcr_update_desc(self._ctx, st.slot, C.byref(st.params.desc(st.n, st.n_chains))))

    def couple(self, slots, fixed, cross_wca):
        """Step the resident systems ``slots`` as the populations of one box
        (``gcr_couple``): one dt, joint list builds, and the WCA force
        ``cross_wca[i][j] = [p0, p1, shift, r_cut]`` of population j on
        population i.  ``fixed[i]``: population i never moves."""
        n = len(slots)
        cw = np.ascontiguousarray(np.asarray(cross_wca, dtype=np.float64).reshape(n, n, 4))
        s_arr = (C.c_int32 * n)(*[int(s) for s in slots])
        f_arr = (C.c_int32 * n)(*[1 if f else 0 for f in fixed])
        check(self.lib.gcr_couple(self._ctx, n, s_arr, f_arr, cw.ctypes.data_as(C.POINTER(C.c_double))))

    def set_motors(self, motor_slot, chain_slot, params, hold=True):
        """``motor_slot`` (single beads, coupled with ``chain_slot`` by
        ``couple`` with the list radius as the cross r_cut of motor from
        chains) pushes the chains' beads (``gcr_set_motors``): params =
        [motor_max_dist_sq, b_one_motor_per_bead, imparts_force, k_on,
        k_off] (populations.py:276-287); ``hold``:
        b_motors_dont_diffuse_while_pushing.  ``chain_slot=-1`` undoes it."""
        prm = np.ascontiguousarray(np.asarray(params if params is not None else np.zeros(5), dtype=np.float64))
        if prm.shape != (5,):
            raise ValueError("motor params are [max_dist_sq, one_per_bead, force, k_on, k_off]")
        check(self.lib.gcr_set_motors(self._ctx, int(motor_slot), int(chain_slot),
                                      prm.ctypes.data_as(C.POINTER(C.c_double)), 1 if hold else 0))

    def where_active(self, slot):
        """pop.where_active of a resident system after the last step: int32
        [n] on the device (chains: motors attached minus one; motors: the
        bead pushed or -1)."""
        st = self.systems[int(slot)]
        out = torch.empty(st.n, dtype=torch.int32, device=st.pos.device)
        torch.cuda.current_stream(self.device).synchronize()
        check(self.lib.gcr_where_active(self._ctx, int(slot), C.c_void_p(out.data_ptr())))
        self.synchronize()
        return out

    def unwrapped(self, slot):
        """Positions plus the periodic images each bead crossed since
        admission (or ``reset_images``): float64 [n, dim] on the device."""
        st = self.systems[int(slot)]
        out = torch.empty_like(st.pos)
        torch.cuda.current_stream(self.device).synchronize()
        check(self.lib.gcr_unwrapped_positions(self._ctx, int(slot), C.c_void_p(out.data_ptr())))
        return out

    def reset_images(self, slot):
        check(self.lib.gcr_reset_images(self._ctx, int(slot)))

    def decouple(self, slot):
        check(self.lib.gcr_decouple(self._ctx, int(slot)))

    def call_begin(self, slot, max_steps, dt, max_dt_usable=-1.0, noise=None):
        """Arm one system for the next ``run``: the arguments of one
        ``SRK2_force_calc`` call (updates.py:138-146)."""
        c = Call()
        c.max_steps, c.max_dt_usable, c.dt = int(max_steps), float(max_dt_usable), float(dt)
        if noise is not None:
            assert noise.dtype == torch.float64 and noise.is_cuda and noise.is_contiguous()
            c.noise, c.noise_steps = noise.data_ptr(), noise.shape[0]
            self.systems[slot].extra["noise_ref"] = noise  # keep alive while in use
        else:
            c.noise, c.noise_steps = None, 0
        torch.cuda.current_stream(self.device).synchronize()
        check(self.lib.gcr_call_begin(self._ctx, int(slot), C.byref(c)))

    def call_begin_many(self, slots, max_steps, dts, max_dt_usable=-1.0, series=None, series_every=0,
                        series_phase=0):
        """Arm many systems with one copy of the state table each way.
        ``series``: a float64 device tensor [len(slots), rows, 5] that
        receives, on the device, (step, time in the call, P, S, angle) after
        each step k of the call with (k + phase) % series_every == 0."""
        n = len(slots)
        calls = (Call * n)()
        arr = (C.c_int32 * n)(*[int(s) for s in slots])
        if series is not None:
            assert series.dtype == torch.float64 and series.is_cuda and series.is_contiguous()
            assert series.shape[0] >= n and series.shape[2] == 5
            self._series_ref = series  # keep alive while in use
        for i in range(n):
            calls[i].max_steps = int(max_steps[i] if np.ndim(max_steps) else max_steps)
            calls[i].max_dt_usable = float(max_dt_usable[i] if np.ndim(max_dt_usable) else max_dt_usable)
            calls[i].dt = float(dts[i] if np.ndim(dts) else dts)
            calls[i].noise, calls[i].noise_steps = None, 0
            every = int(series_every[i] if np.ndim(series_every) else series_every)
            if series is not None and every > 0:
                calls[i].series = series[i].data_ptr()
                calls[i].series_every = every
                calls[i].series_phase = int(series_phase[i] if np.ndim(series_phase) else series_phase)
                calls[i].series_capacity = series.shape[1]
        torch.cuda.current_stream(self.device).synchronize()
        check(self.lib.gcr_call_begin_batch(self._ctx, n, arr, calls))

    # -- stepping ------------------------------------------------------------
    def run(self, max_steps, sync_every=0):
        """Queue up to ``max_steps`` steps of every armed system on the
        context stream.  Work queued afterwards on the caller's current torch
        stream (reading the state tensors, say) is ordered after them; the
        host does not wait."""
        check(self.lib.gcr_run(self._ctx, int(max_steps), int(sync_every)))
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def synchronize(self):
        check(self.lib.gcr_synchronize(self._ctx))

    PROFILE_GROUPS = ["lists_pos", "pair_pos", "stage0", "lists_pos1", "pair_pos1", "stage1", "update"]

    def profile_steps(self, n_steps):
        """Milliseconds per kernel group over ``n_steps`` individually
        launched steps, in the order of ``PROFILE_GROUPS``."""
        out = (C.c_float * 7)()
        check(self.lib.gcr_profile_steps(self._ctx, int(n_steps), out))
        return np.array(out[:], dtype=np.float64)

    def count_active(self):
        n = C.c_int32()
        check(self.lib.gcr_count_active(self._ctx, C.byref(n)))
        return n.value

    @staticmethod
    def _status_dict(s):
        return {"dt": s.dt, "dt_used": s.dt_used, "max_forces_strength": s.max_forces_strength,
                "steps_done": s.steps_done, "step": s.step, "flags": s.flags, "active": bool(s.active),
                "list_builds": s.list_builds, "series_rows": s.series_rows}

    def status(self, slot):
        s = Status()
        check(self.lib.gcr_get_status(self._ctx, int(slot), C.byref(s)))
        return self._status_dict(s)

    def statuses(self, slots):
        """The statuses of many systems with one copy of the state table."""
        n = len(slots)
        out = (Status * max(n, 1))()
        arr = (C.c_int32 * max(n, 1))(*[int(s) for s in slots])
        check(self.lib.gcr_get_statuses(self._ctx, n, arr, out))
        return [self._status_dict(out[i]) for i in range(n)]

    # -- observables and exports --------------------------------------------
    def order_params(self, slot):
        out = (C.c_double * 3)()
        check(self.lib.gcr_order_params(self._ctx, int(slot), out))
        return np.array(out[:])

    def reference_lists(self, slot, n_grid, grid_window, grid_depth1=None, nbor_depth1=9, mode=1):
        """The reference's where_is_bead / grid_list / nbor_list, built on the
        device; depths double on overflow as populations.py:104-112, 176-180 do."""
        st = self.systems[slot]
        n = st.n
        nz = 1 if self.dim == 2 else n_grid
        if grid_depth1 is None:
            grid_depth1 = 1 + max(1, int(8 * n / n_grid ** self.dim))
        dev = st.pos.device
        while True:
            wib = torch.zeros((n, 3), dtype=torch.int64, device=dev)
            grid = torch.zeros((n_grid, n_grid, nz, grid_depth1), dtype=torch.int64, device=dev)
            nb = torch.zeros((n, nbor_depth1), dtype=torch.int64, device=dev)
            torch.cuda.current_stream(dev).synchronize()
            rc = self.lib.gcr_reference_lists(self._ctx, int(slot), int(n_grid), int(grid_window),
                                              wib.data_ptr(), grid.data_ptr(), grid_depth1, nb.data_ptr(),
                                              nbor_depth1, int(mode))
            if rc == 0:
                return wib, grid, nb
            msg = self.lib.gcr_last_error().decode()
            if rc != -8:
                raise GcrError(rc, msg)
            if "grid" in msg:
                grid_depth1 = 2 * grid_depth1
            else:
                nbor_depth1 = 2 * nbor_depth1

    def neighbour_list(self, slot, partners=True):
        """Counts [n], partners [n, list_depth] (bead ids in summation order,
        -1 past the count), the FP64 positions of the build [n, d] and the
        total entries of a system's list as of its last build."""
        st = self.systems[slot]
        dev = st.pos.device
        counts = torch.zeros(st.n, dtype=torch.int32, device=dev)
        part = torch.full((st.n, self.cfg.list_depth), -1, dtype=torch.int32, device=dev) if partners else None
        xb = torch.zeros((st.n, self.dim), dtype=torch.float64, device=dev)
        total = C.c_int64()
        torch.cuda.current_stream(dev).synchronize()
        check(self.lib.gcr_neighbour_list(self._ctx, int(slot), C.c_void_p(counts.data_ptr()),
                                          C.c_void_p(part.data_ptr()) if part is not None else None,
                                          self.cfg.list_depth, C.c_void_p(xb.data_ptr()), C.byref(total)))
        return counts, part, xb, total.value

    def cell_assignment(self, slot):
        st = self.systems[slot]
        out = torch.empty(st.n, dtype=torch.int32, device=st.pos.device)
        ncs = C.c_int32()
        torch.cuda.current_stream(st.pos.device).synchronize()
        check(self.lib.gcr_cell_assignment(self._ctx, int(slot), out.data_ptr(), C.byref(ncs)))
        return out, ncs.value


def philox_noise(dim, seed, step, n, do_trans=True, do_rot=True, device="cuda"):
    out = torch.zeros((n, 2 * dim), dtype=torch.float64, device=device)
    torch.cuda.current_stream().synchronize()
    check(_lib.load().gcr_philox_noise(dim, int(seed) & (2 ** 64 - 1), int(step), int(n), int(do_trans),
                                       int(do_rot), out.data_ptr(), None))
    return out
