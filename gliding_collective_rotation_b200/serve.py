"""Continuous batching of simulation requests on one GPU.

A request is one independent system (a ``SystemSpec``) to be advanced a
given number of SRK2 steps, with the order parameters P, S and the director
angle (``output_methods.calc_avg_phi_chain`` + ``analysis.polar_orderparameter``
+ ``analysis.nematic_orderparameter``, output_methods.py:492-510,
analysis.py:294-328) sampled every ``obs_every`` steps.  The server keeps
every resident system in one ``Engine`` context, so one captured graph of
persistent kernels advances all of them at once.  Requests are admitted as
soon as the context's bead, cell and slot ranges have room (the library's
allocator is the memory budget); a finished request is evicted at once and
its ranges go to the next one.  Admission is first come first served, and a
later request that fits may go ahead of a head request that does not
(backfill) unless the head has waited longer than ``max_head_wait`` seconds.

Steps follow the reference's adaptive dt by default (dtmax = the request's
dt, ``max_dist_per_step`` of ``config.grid_list_setup``, config.py:189), which
also takes fresh chains laid straight at random through their overlaps; a
request may instead ask for a fixed dt, and then for an untimed relaxation
under the adaptive rule first (until the step takes the full dt), reported
apart from the requested steps.  Each system's dt carries from call to call,
as the reference's ``status.dt`` does.

Calls are chunked: every system is armed for at most ``chunk`` steps, the
graph runs, statuses come back in one copy, finished requests leave.  The
order parameters are sampled on the device inside the steps' graph (the
call's series, counted from the request's first step), so a chunk does not
stop at observation steps and a sample costs no host round trip.  With a fixed dt a system's trajectory
does not depend on how its steps are split into calls (the Philox noise is
keyed by bead and step, and the pair sums are taken in a fixed order), so a
request served in a busy mix ends bit-for-bit where it ends alone.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import FLAG_CELL_OVERFLOW, FLAG_LIST_OVERFLOW, GcrError
from .batch import MAX_DEPTH, MAX_LIST_DEPTH, OVERFLOW, default_depth, default_list_depth
from .engine import Engine, SystemState
from .workloads import SystemSpec, make_system

# resident bytes per bead of the state tensors (FP64 pos/pos1, FT tangent/forces, chain id)
_STATE_BYTES = {"mixed": 2 * 16 + 2 * 8 + 4, "fp64": 2 * 16 + 2 * 16 + 4}


@dataclass
class Request:
    id: int
    spec: SystemSpec
    steps: int
    arrival: float = 0.0
    obs_every: int = 0
    relax: bool = False
    adaptive: bool = True


@dataclass
class Result:
    id: int
    n_beads: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    relax_steps: int
    pos: np.ndarray
    tangent: np.ndarray
    series: np.ndarray          # rows (step, P, S, angle)
    flags: int

    @property
    def latency(self):
        return self.finished - self.arrival


@dataclass
class _Live:
    req: Request
    state: SystemState
    admitted: float
    relaxing: bool
    relax_steps: int = 0
    done: int = 0
    dt: float | None = None
    series: list = field(default_factory=list)


def check_request(req, dim, bead_capacity):
    """Why ``req`` cannot be served (a short reason), or None.  A request
    must ask for at least one step, hold at least one bead, have arrays of
    matching shapes with finite values, chain ids 0, 1, ..., n_chains - 1 in
    contiguous increasing ranges (the layout the step kernels index by), a
    positive box side and rest lengths, and fit an empty context."""
    sp = getattr(req, "spec", None)
    if sp is None:
        return "no system"
    steps = req.steps
    if not isinstance(steps, (int, np.integer)) or steps < 1:
        return f"steps must be a positive integer (got {steps!r})"
    if not isinstance(req.obs_every, (int, np.integer)) or req.obs_every < 0:
        return f"obs_every must be a non-negative integer (got {req.obs_every!r})"
    if sp.dim != dim:
        return f"dimension {sp.dim} in a {dim}D server"
    pos, tan = np.asarray(sp.pos), np.asarray(sp.tangent)
    chain, rest = np.asarray(sp.chain_id), np.asarray(sp.rest_lengths)
    n = pos.shape[0] if pos.ndim == 2 else -1
    if n < 1 or pos.shape[1] != dim:
        return f"positions must be [n >= 1, {dim}] (got {pos.shape})"
    if tan.shape != pos.shape or chain.shape != (n,):
        return "tangent [n, dim] and chain_id [n] must match the positions"
    if rest.ndim != 1 or rest.shape[0] < 1:
        return "rest_lengths must be [n_chains >= 1]"
    if not np.issubdtype(chain.dtype, np.integer):
        return "chain ids must be integers"
    steps_c = np.diff(chain)
    if chain[0] != 0 or np.any((steps_c != 0) & (steps_c != 1)) or chain[-1] != rest.shape[0] - 1:
        return "chain ids must run 0, 1, ..., n_chains - 1 in contiguous increasing ranges"
    L = float(sp.params.L)
    if not (math.isfinite(L) and L > 0):
        return f"box side must be positive and finite (got {L})"
    if not (np.all(np.isfinite(pos)) and np.all(np.isfinite(tan)) and np.all(np.isfinite(rest))):
        return "non-finite positions, tangents or rest lengths"
    if np.any(rest <= 0):
        return "rest lengths must be positive"
    if n > bead_capacity:
        return f"{n} beads exceed the context ({bead_capacity})"
    return None


def request_from_trace(entry, relax=False, obs_every=0, adaptive=True):
    """A ``Request`` from one entry of ``workloads.serve_trace``."""
    spec = make_system(f"req{entry['id']}", 2, entry["n_chains"], entry["chain_length"], entry["L"],
                       seed=10_000 + entry["id"], kappa=entry["kappa"], v_tan_angle=entry["v_tan_angle"],
                       noise_seed=entry["seed"])
    return Request(entry["id"], spec, entry["steps"], entry["arrival"], obs_every, relax, adaptive)


class Server:
    """One GPU, one context, many resident requests."""

    def __init__(self, dim=2, precision="mixed", hbm_budget=8 << 30, cells_per_bead=4.0, max_systems=256,
                 chunk=200, device=None, cell_depth=None, relax_max_steps=4000, max_head_wait=5.0,
                 steps_per_graph=10):
        self.dim, self.precision = dim, precision
        self.device = torch.device(device or "cuda")
        self.chunk = int(chunk)
        self._series = None  # device rows of the in-graph order-parameter series
        self.relax_max_steps = int(relax_max_steps)
        self.max_head_wait = float(max_head_wait)
        self.cell_depth = cell_depth or default_depth(dim, 1.3)  # cells of side r_cut + skin
        self.list_depth = default_list_depth(dim)
        self.max_systems = int(max_systems)
        self.cells_per_bead = float(cells_per_bead)
        self.steps_per_graph = int(steps_per_graph)
        self.hbm_budget = int(hbm_budget)
        self._size_context()
        self.engine = self._make_engine()
        self.live: dict[int, _Live] = {}
        self.queue: list[Request] = []
        self.results: list[Result] = []
        self.rejected: list[tuple[int, str]] = []  # (request id, reason)
        self.t0 = None
        # where the time of a served trace goes: device time of the rounds'
        # graphs (CUDA events on the context stream), wall time of the rounds
        # (arming, statuses, series, finished requests, regrows around them),
        # and time with nothing resident waiting for arrivals
        self.stats = {"rounds": 0, "device_s": 0.0, "round_wall_s": 0.0, "idle_s": 0.0, "regrows": 0,
                      "resident_bead_s": 0.0, "bead_steps_done": 0, "bead_steps_armed_max": 0}

    # -- memory ----------------------------------------------------------------
    def _per_bead_bytes(self):
        ft = 4 if self.precision == "mixed" else 8
        # fp, xi, topo, list, xref, rest length
        scratch = 2 * self.dim * ft + 1 + 4 * self.list_depth + 4 + 8 * self.dim + 8
        per_cell = 4 * (self.cell_depth + 2)               # slots, count, count at the build
        return _STATE_BYTES[self.precision] + scratch + self.cells_per_bead * per_cell

    def _size_context(self):
        self.bead_capacity = max(1024, int(self.hbm_budget / self._per_bead_bytes()))
        self.cell_capacity = int(self.cells_per_bead * self.bead_capacity)

    def _make_engine(self):
        return Engine(self.dim, self.precision, device=self.device, bead_capacity=self.bead_capacity,
                      system_capacity=self.max_systems, cell_capacity=self.cell_capacity,
                      cell_depth=self.cell_depth, list_depth=self.list_depth, steps_per_graph=self.steps_per_graph)

    def fits_ever(self, req: Request):
        return req.spec.n <= self.bead_capacity

    # -- clock -----------------------------------------------------------------
    def now(self):
        return time.perf_counter() - self.t0

    # -- admission -------------------------------------------------------------
    def _admit_one(self, req: Request):
        """Admit the queued request ``req``: True when it left the queue
        (admitted, or rejected), False when the context has no room yet."""
        why = check_request(req, self.dim, self.bead_capacity)
        if why is not None:
            self._reject(req, why)
            return True
        sp = req.spec
        p = sp.params
        if req.relax or req.adaptive:
            p.max_dist_per_step = sp.relax_mdps
        st = SystemState.from_host(sp.pos, sp.tangent, sp.chain_id, sp.rest_lengths, p, precision=self.precision,
                                   device=self.device)
        try:
            slot = self.engine.try_admit(st)
        except GcrError as e:
            if e.code != -1:  # GCR_ERR_BAD_ARG: the library refused the system itself
                raise
            del st
            self._reject(req, str(e))
            return True
        if slot is None:
            del st
            return False
        self.queue.remove(req)
        self.live[slot] = _Live(req, st, self.now(), relaxing=req.relax)
        return True

    def _reject(self, req, reason):
        """A request that cannot be served leaves the queue with its reason;
        the resident requests are not touched."""
        self.queue.remove(req)
        self.rejected.append((req.id, reason))

    def _admit(self):
        now = self.now()
        arrived = [r for r in self.queue if r.arrival <= now]
        if not arrived:
            return
        blocked = None  # the first arrived request that did not fit
        for r in arrived:
            if len(self.live) >= self.max_systems and check_request(r, self.dim, self.bead_capacity) is None:
                break
            if blocked is not None and now - blocked.arrival > self.max_head_wait:
                break  # no backfill past a head that has waited too long
            if not self._admit_one(r) and blocked is None:
                blocked = r

    # -- overflow --------------------------------------------------------------
    def _regrow(self, statuses):
        flags = 0
        for slot, lv in self.live.items():
            lv.state.params.step = statuses[slot]["step"]
            flags |= statuses[slot]["flags"]
        cell = bool(flags & FLAG_CELL_OVERFLOW)
        lst = bool(flags & FLAG_LIST_OVERFLOW) or not cell
        if (cell and self.cell_depth >= MAX_DEPTH) or (lst and self.list_depth >= MAX_LIST_DEPTH):
            raise RuntimeError("GPU cell or list depth limit reached")
        old = list(self.live.values())
        self.engine.close()
        if cell:
            self.cell_depth *= 2
        if lst:
            self.list_depth *= 2
        self._size_context()
        self.engine = self._make_engine()
        self.live = {}
        for lv in old:
            slot = self.engine.admit(lv.state)
            self.live[slot] = lv

    # -- one round of calls ----------------------------------------------------
    def _plan(self, lv: _Live):
        if lv.relaxing:
            return min(self.chunk, self.relax_max_steps - lv.relax_steps)
        return min(self.chunk, lv.req.steps - lv.done)

    def _round(self):
        slots = sorted(self.live)
        plan = [self._plan(self.live[s]) for s in slots]
        # each system's dt carries from call to call (the reference's status.dt)
        dts = [self.live[s].dt if self.live[s].dt is not None else self.live[s].req.spec.dt for s in slots]
        # the order parameters are sampled on the device, inside the steps'
        # graph, every obs_every steps counted from the request's start
        every = [0 if self.live[s].relaxing else max(0, self.live[s].req.obs_every) for s in slots]
        phase = [self.live[s].done % e if e > 0 else 0 for s, e in zip(slots, every)]
        series = None
        if any(every):
            rows = max(k // e + 1 for k, e in zip(plan, every) if e > 0)
            if self._series is None or self._series.shape[0] < len(slots) or self._series.shape[1] < rows:
                self._series = torch.zeros((max(self.max_systems, len(slots)), max(rows, self.chunk + 1), 5),
                                           dtype=torch.float64, device=self.device)
            series = self._series
        t_round = time.perf_counter()
        self.engine.call_begin_many(slots, plan, dts, series=series, series_every=every, series_phase=phase)
        ev = None
        if self.device.type == "cuda":
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record(self.engine.stream)
        self.engine.run(max(plan))
        if ev is not None:
            ev[1].record(self.engine.stream)
        statuses = dict(zip(slots, self.engine.statuses(slots)))
        st_ = self.stats
        st_["rounds"] += 1
        if ev is not None:
            dev_s = ev[0].elapsed_time(ev[1]) / 1e3
            st_["device_s"] += dev_s
            st_["resident_bead_s"] += dev_s * sum(self.live[s].state.n for s in slots)
        st_["bead_steps_done"] += sum(self.live[s].state.n * statuses[s]["steps_done"] for s in slots)
        st_["bead_steps_armed_max"] += sum(self.live[s].state.n for s in slots) * max(plan)
        rows_host = None
        if series is not None and any(statuses[s]["series_rows"] for s in slots):
            rows_host = series.cpu().numpy()
        for i, s in enumerate(slots):
            st, lv = statuses[s], self.live[s]
            if rows_host is None or not st["series_rows"]:
                continue
            # a row's global step -> steps of the request
            start = st["step"] - st["steps_done"]
            for r in rows_host[i, :st["series_rows"]]:
                lv.series.append((lv.done + int(r[0]) - start, r[2], r[3], r[4]))
        finished, overflow = [], False
        for s, k in zip(slots, plan):
            lv, st = self.live[s], statuses[s]
            # steps completed before a stop are valid; an overflowed system
            # resumes from there once the cells have grown
            n_done = st["steps_done"]
            lv.dt = st["dt"]
            if st["flags"] & OVERFLOW:
                overflow = True
                if lv.relaxing:
                    lv.relax_steps += n_done
                else:
                    lv.done += n_done
                continue
            if lv.relaxing:
                lv.relax_steps += n_done
                full = st["dt"] >= lv.req.spec.dt * (1 - 1e-12)
                if full or lv.relax_steps >= self.relax_max_steps:
                    lv.relaxing = False
                    if not lv.req.adaptive:
                        lv.state.params.max_dist_per_step = math.inf
                        self.engine.update_params(lv.state)
                continue
            lv.done += n_done
            if st["flags"] or n_done < k:
                finished.append(s)  # a failed system leaves with its flags
                continue
            if lv.done >= lv.req.steps:
                finished.append(s)
        for s in finished:
            self._finish(s, statuses[s]["flags"])
        if overflow:
            self._regrow({s: statuses[s] for s in self.live})
            st_["regrows"] += 1
        st_["round_wall_s"] += time.perf_counter() - t_round

    def _finish(self, slot, flags):
        lv = self.live.pop(slot)
        st = lv.state
        self.engine.synchronize()
        res = Result(lv.req.id, st.n, lv.done, lv.req.arrival, lv.admitted, self.now(), lv.relax_steps,
                     st.pos.cpu().numpy(), st.tangent.double().cpu().numpy(),
                     np.array(lv.series, dtype=np.float64).reshape(-1, 4), int(flags))
        self.engine.evict(slot)
        self.results.append(res)

    # -- driver ----------------------------------------------------------------
    def serve(self, requests, timeout=None):
        """Serve ``requests`` (arrival times in seconds from the start) until
        all are done; returns the results in completion order.  A request that
        cannot be served (``check_request``) is rejected when it arrives and
        listed in ``rejected`` as (id, reason); the others run as if it had
        never come."""
        self.queue = sorted(requests, key=lambda r: (r.arrival, r.id))
        self.t0 = time.perf_counter()
        while self.queue or self.live:
            if timeout is not None and self.now() > timeout:
                raise TimeoutError(f"serving did not finish in {timeout} s")
            self._admit()
            if not self.live:
                if self.queue:
                    wait = self.queue[0].arrival - self.now()
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                        self.stats["idle_s"] += min(wait, 0.05)
                    elif not self._admit_one_blocking():
                        raise RuntimeError("a request does not fit an empty context")
                continue
            self._round()
        return self.results

    def _admit_one_blocking(self):
        return self._admit_one(self.queue[0])

    def close(self):
        self.engine.close()


def summarize(results, makespan=None):
    """Latency percentiles and throughput of a served trace."""
    lat = np.array([r.latency for r in results])
    bead_steps = float(sum(r.n_beads * r.steps for r in results))
    relax = float(sum(r.n_beads * r.relax_steps for r in results))
    span = makespan if makespan is not None else max(r.finished for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "bead_steps": bead_steps, "relax_bead_steps": relax, "makespan_s": span,
            "bead_steps_per_s": bead_steps / span if span > 0 else float("nan"),
            "failed": sum(1 for r in results if r.flags)}
