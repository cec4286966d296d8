"""CPU oracle for the gliding-collective-rotation hot path (test infrastructure).

This module is the parity checker and the timed CPU baseline.  Only the test
suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
it; the product package never imports it.

It wraps ``gcr_oracle.c`` (a loop-for-loop C restatement of the reference's
Numba step) and mirrors the reference's host-side set-up:

* ``OracleSystem`` holds a population's arrays in the reference's numpy layouts
  (``populations.py:63-82, 150-154, 182-184``) and runs the multi-step SRK2 loop
  (``SRK.py:13-484``) the way ``updates.SRK2_force_calc`` (``updates.py:132-267``)
  drives it, including the ``status`` write-back and the list regrow on
  overflow.
* ``build_lists`` reproduces ``Population.update_grid_list(overwrite=True)``
  (``populations.py:104-112``) and ``update_nbor_list_with_pop2``
  (``populations.py:156-180``).

Parity anchors: the golden fixtures under ``tests/golden`` were produced by the
reference itself (Numba, single thread, seeded RNG); ``tests/test_oracle_golden.py``
checks this oracle against them.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libgcr_oracle.so")
# the same restatement compiled with FMA contraction (a * b + c fused, as
# nvcc does by default): a second valid FP64 evaluation of every step whose
# divergence from the first measures how sensitive a trajectory is to
# rounding (tests only; it needs a CPU with FMA and AVX2)
_FMA_LIB_PATH = os.path.join(_HERE, "libgcr_oracle_fma.so")

NOISE_MT, NOISE_INJECT, NOISE_PHILOX = 0, 1, 2


class MT(C.Structure):
    _fields_ = [("mt", C.c_uint32 * 624), ("idx", C.c_int), ("has_gauss", C.c_int),
                ("gauss", C.c_double)]


class Params(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("n_threads", C.c_int32), ("L", C.c_double),
        ("n_beads", C.c_int64), ("n_chains", C.c_int64),
        ("calc_springs", C.c_int32), ("calc_wca", C.c_int32), ("self_propel", C.c_int32),
        ("noise_mode", C.c_int32),
        ("spring", C.c_double * 6), ("wca", C.c_double * 4), ("active", C.c_double * 3),
        ("D", C.c_double), ("Dr", C.c_double), ("radius", C.c_double),
        ("rigid_rod", C.c_double),
        ("n_nearby", C.c_int64), ("longest_chain_length", C.c_int64),
        ("grid_factor", C.c_double),
        ("dt", C.c_double), ("dtmax", C.c_double), ("max_dist_per_step", C.c_double),
        ("rk_cheat", C.c_double), ("max_dt_usable", C.c_double),
        ("steps_until_update", C.c_int64), ("n_steps_update", C.c_int64),
        ("max_steps", C.c_int64),
        ("seed", C.c_uint64), ("step0", C.c_int64), ("srk_order", C.c_int64),
    ]


class State(C.Structure):
    _fields_ = [
        ("pos", C.c_void_p), ("pos1", C.c_void_p), ("noise", C.c_void_p),
        ("tangent", C.c_void_p), ("forces", C.c_void_p),
        ("where_active", C.c_void_p), ("where_is_bead", C.c_void_p),
        ("chain_id", C.c_void_p), ("rest_lengths", C.c_void_p),
        ("grid_list", C.c_void_p), ("n_grid", C.c_int64), ("n_grid_z", C.c_int64),
        ("grid_depth1", C.c_int64),
        ("nbor_list", C.c_void_p), ("nbor_depth1", C.c_int64),
        ("noise_inject", C.c_void_p), ("noise_inject_steps", C.c_int64),
        ("mt", C.c_void_p), ("forces_aux", C.c_void_p),
    ]


class Motors(C.Structure):
    """A motor population of a group (gcro_motors)."""
    _fields_ = [("motor_pop", C.c_int32), ("chain_pop", C.c_int32), ("dont_diffuse", C.c_int32),
                ("pad", C.c_int32), ("params", C.c_double * 5), ("list_r2", C.c_double),
                ("act", C.c_void_p * 8)]


class Result(C.Structure):
    _fields_ = [("dt", C.c_double), ("dt_used_total", C.c_double), ("steps", C.c_double),
                ("max_forces_strength", C.c_double), ("counter", C.c_double),
                ("flag", C.c_double)]


_libs = {}


def fma_available():
    """The host CPU runs the contracted build (x86-64-v3: FMA and AVX2)."""
    try:
        with open("/proc/cpuinfo") as fh:
            flags = next((ln.split(":", 1)[1].split() for ln in fh if ln.startswith("flags")), [])
    except OSError:
        return False
    return "fma" in flags and "avx2" in flags


def build():
    """Compile ``libgcr_oracle.so`` with the recipe in ``oracle/Makefile``."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(variant=""):
    """The oracle library: ``""`` the reference's arithmetic (no
    contraction), ``"fma"`` the contracted control build."""
    if variant not in _libs:
        path = {"": _LIB_PATH, "fma": _FMA_LIB_PATH}[variant]
        if variant == "fma" and not fma_available():
            raise RuntimeError("the contracted oracle needs a CPU with FMA and AVX2")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.gcro_srk2_run.restype = C.c_int
        L.gcro_srk2_run.argtypes = [C.POINTER(Params), C.POINTER(State), C.POINTER(Result)]
        L.gcro_mt_seed.argtypes = [C.POINTER(MT), C.c_uint32]
        L.gcro_mt_normals.argtypes = [C.c_uint32, C.c_int64, C.c_void_p]
        L.gcro_philox_pair.argtypes = [C.c_uint64, C.c_uint32, C.c_int64, C.c_uint32, C.c_void_p]
        L.gcro_philox_noise.argtypes = [C.c_uint64, C.c_int64, C.c_int, C.c_int64, C.c_int,
                                        C.c_int, C.c_void_p]
        L.gcro_spring_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_int64, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        L.gcro_pair_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                       C.c_double, C.c_void_p, C.c_double, C.c_int]
        L.gcro_self_propel.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int]
        L.gcro_update_grid_list.restype = C.c_int
        L.gcro_update_grid_list.argtypes = [C.POINTER(State), C.c_void_p, C.c_int64, C.c_double,
                                            C.c_int, C.c_int, C.c_int, C.c_int64]
        L.gcro_update_nbor_list.restype = C.c_int
        L.gcro_update_nbor_list.argtypes = [C.POINTER(State), C.c_void_p, C.c_int64, C.c_double,
                                            C.c_int64, C.c_int64, C.c_int]
        L.gcro_update_nbor_list_few.restype = C.c_int
        L.gcro_update_nbor_list_few.argtypes = L.gcro_update_nbor_list.argtypes
        L.gcro_chunk_chain.restype = C.c_int
        L.gcro_chunk_chain.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        L.gcro_order_params.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        L.gcro_pair_forces_all.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                           C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_void_p]
        L.gcro_motor_uniforms.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_int64, C.c_int, C.c_void_p]
        L.gcro_motor_push_mt.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(MT), C.c_int]
        L.gcro_group_run_motors.restype = C.c_int
        L.gcro_group_run_motors.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.POINTER(Params), C.POINTER(Result), C.POINTER(Motors)]
        L.gcro_group_run.restype = C.c_int
        L.gcro_group_run.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Params),
                                     C.POINTER(Result)]
        L.gcro_project_rigid.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                         C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_int]
        assert L.gcro_sizeof_params() == C.sizeof(Params)
        assert L.gcro_sizeof_state() == C.sizeof(State)
        assert L.gcro_sizeof_mt() == C.sizeof(MT)
        assert L.gcro_sizeof_motors() == C.sizeof(Motors)
        _libs[variant] = L
    return _libs[variant]


def _p(a):
    return a.ctypes.data if a is not None else None


# ---------------------------------------------------------------------------
# random streams
# ---------------------------------------------------------------------------

def mt_normals(seed, n):
    """``n`` normals of the stream Numba draws after ``np.random.seed(seed)``."""
    out = np.empty(n)
    lib().gcro_mt_normals(seed, n, _p(out))
    return out


def philox_pair(seed, bead, step, stream):
    out = np.empty(2)
    lib().gcro_philox_pair(seed, bead, step, stream, _p(out))
    return out


def philox_noise(seed, step, dim, n, do_trans=True, do_rot=True):
    out = np.zeros((n, 2 * dim))
    lib().gcro_philox_noise(seed, step, dim, n, int(do_trans), int(do_rot), _p(out))
    return out


def split_mt_stream(stream, n_beads, dim, n_steps, D_pos, Dr_pos):
    """Cut the reference's sequential normal stream into per-step ``noise_vec``
    snapshots ``[n_steps, N, 2*dim]`` in the order ``SRK.py:134-142`` consumes it
    (all translational deviates of a step bead-major, then all rotational ones)."""
    out = np.zeros((n_steps, n_beads, 2 * dim))
    k = 0
    for s in range(n_steps):
        if D_pos:
            out[s, :, :dim] = stream[k:k + n_beads * dim].reshape(n_beads, dim)
            k += n_beads * dim
        if Dr_pos:
            out[s, :, dim:] = stream[k:k + n_beads * dim].reshape(n_beads, dim)
            k += n_beads * dim
    return out


def normals_per_step(n_beads, dim, D_pos, Dr_pos):
    return n_beads * dim * (int(bool(D_pos)) + int(bool(Dr_pos)))


# ---------------------------------------------------------------------------
# kernels as unit functions
# ---------------------------------------------------------------------------

def spring_forces(pos, tangent, chain_id, forces, L, spring_params, rest_lengths):
    n, dim = pos.shape
    lib().gcro_spring_forces(_p(pos), _p(tangent), _p(chain_id), _p(forces), n, L,
                             _p(np.ascontiguousarray(spring_params, dtype=np.float64)),
                             _p(rest_lengths), dim)


def pair_forces(pos, nbor_list, forces, L, wca_params, pbc_width):
    n, dim = pos.shape
    lib().gcro_pair_forces(_p(pos), _p(nbor_list), nbor_list.shape[1], _p(forces), n, L,
                           _p(np.ascontiguousarray(wca_params, dtype=np.float64)), pbc_width, dim)


def self_propel(forces, tangent, active_params):
    n, dim = forces.shape
    lib().gcro_self_propel(_p(forces), _p(tangent), n,
                           _p(np.ascontiguousarray(active_params, dtype=np.float64)), dim)


def project_rigid(prev, forces, noise, chain_id, rest_lengths, factor, L, dt, D, radius):
    """updates.project_updates_for_rigid_rod (updates.py:347-499) on one
    chunk: the projected positions.  ``noise`` is the [N, 2*dim] noise_vec."""
    prev = np.ascontiguousarray(prev, dtype=np.float64)
    forces = np.ascontiguousarray(forces, dtype=np.float64)
    noise = np.ascontiguousarray(noise, dtype=np.float64)
    chain_id = np.ascontiguousarray(chain_id, dtype=np.int64)
    rest_lengths = np.ascontiguousarray(rest_lengths, dtype=np.float64)
    out = np.zeros_like(prev)
    lib().gcro_project_rigid(_p(out), _p(prev), _p(forces), _p(noise), len(prev), _p(chain_id), _p(rest_lengths),
                             float(factor), float(L), float(dt), float(D), float(radius), prev.shape[1])
    return out


def chunk_chain(n_threads, chain_id):
    split = np.zeros(max(n_threads - 1, 0), dtype=np.int64)
    k = lib().gcro_chunk_chain(n_threads, len(chain_id), _p(chain_id), _p(split))
    return split[:k]


def motor_uniforms(seed, motor, bead, step, stage):
    """The keyed (u_off, u_on) draws of one (motor, bead) decision."""
    out = np.zeros(2)
    lib().gcro_motor_uniforms(seed, motor, bead, step, stage, _p(out))
    return out


def motor_push_mt(pos_b, nbor_list, forces_b, where_active_b, tangent, L, pos_m, where_active_m, params, seed):
    """forces.calc_motor_push (forces.py:248-283) on the reference's arrays,
    with its draws from MT19937 seeded with `seed` (np.random.seed(seed) in
    a Numba-compiled function gives the same stream).  Arrays are updated in
    place: forces_b, where_active_b, where_active_m (int64)."""
    pos_b = np.ascontiguousarray(pos_b, dtype=np.float64)
    pos_m = np.ascontiguousarray(pos_m, dtype=np.float64)
    tangent = np.ascontiguousarray(tangent, dtype=np.float64)
    nbor = np.ascontiguousarray(nbor_list, dtype=np.int64)
    for a, t in ((forces_b, np.float64), (where_active_b, np.int64), (where_active_m, np.int64)):
        assert a.dtype == t and a.flags.c_contiguous
    mt = MT()
    lib().gcro_mt_seed(C.byref(mt), seed & 0xFFFFFFFF)
    prm = np.ascontiguousarray(params, dtype=np.float64)
    lib().gcro_motor_push_mt(_p(pos_b), len(pos_b), _p(nbor), nbor.shape[1], _p(forces_b), _p(where_active_b),
                             _p(tangent), float(L), _p(pos_m), _p(where_active_m), _p(prm), C.byref(mt),
                             pos_b.shape[1])


def order_params(tangent, chain_start):
    """``[P, S, director_angle]`` as ``analysis.polar_orderparameter`` and
    ``analysis.nematic_orderparameter`` compute them."""
    out = np.empty(3)
    cs = np.ascontiguousarray(chain_start, dtype=np.int64)
    lib().gcro_order_params(_p(np.ascontiguousarray(tangent)), _p(cs), len(cs) - 1,
                            tangent.shape[1], _p(out))
    return out


# ---------------------------------------------------------------------------
# a population in the reference's layouts
# ---------------------------------------------------------------------------

class OracleSystem:
    """One bead-spring-chain population with the reference's arrays.

    Parameters are the packed arrays the reference passes to ``SRK_jit``:
    ``spring_params`` (populations.py:345-353), ``wca_params``
    (populations.py:48-58), ``active_params`` (populations.py:355-358).
    """

    def __init__(self, pos, tangent, chain_id, rest_lengths, L, spring_params, wca_params,
                 active_params, D, Dr, radius, n_nearby, n_grid, grid_factor=2.0,
                 calc_springs=True, calc_wca=True, self_propel=True, grid_depth=None,
                 nbor_depth=8, rigid_rod=0.0, srk_order=2, variant=""):
        self.variant = variant  # oracle library: "" or "fma" (see lib())
        self.pos = np.ascontiguousarray(pos, dtype=np.float64).copy()
        self.N, self.dim = self.pos.shape
        self.pos1 = np.zeros_like(self.pos)
        self.noise_vec = np.zeros((self.N, 2 * self.dim))
        self.tangent_list = np.ascontiguousarray(tangent, dtype=np.float64).copy()
        self.forces = np.zeros_like(self.pos)
        self.where_active = np.zeros(self.N, dtype=np.int64)
        self.chain_id = np.ascontiguousarray(chain_id, dtype=np.int64)
        self.rest_lengths = np.ascontiguousarray(rest_lengths, dtype=np.float64).copy()
        self.L = float(L)
        self.spring_params = np.asarray(spring_params, dtype=np.float64)
        self.WCA_params = np.asarray(wca_params, dtype=np.float64)
        self.active = np.asarray(active_params, dtype=np.float64)
        self.D, self.Dr, self.radius = float(D), float(Dr), float(radius)
        self.n_nearby = int(n_nearby)
        self.n_grid = int(n_grid)
        self.grid_factor = float(grid_factor)
        self.calc_springs = bool(calc_springs) and np.max(np.bincount(self.chain_id)) > 1
        self.calc_wca, self.do_self_propel = bool(calc_wca), bool(self_propel)
        self.longest_chain_length = int(np.max(np.bincount(self.chain_id)))
        self.rigid_rod = float(rigid_rod)
        self.srk_order = int(srk_order)
        # SRK4 keeps the force of the last stage (populations.py:149-154)
        self.forces_aux = np.zeros_like(self.pos) if self.srk_order == 4 else None
        nz = 1 if self.dim == 2 else self.n_grid
        if grid_depth is None:
            grid_depth = max(1, int(8 * self.N / self.n_grid ** self.dim))
        self.grid_list = np.zeros((self.n_grid, self.n_grid, nz, 1 + grid_depth), dtype=np.int64)
        self.where_is_bead = np.zeros((self.N, 3), dtype=np.int64)
        self.nbor_list = np.zeros((self.N, 1 + nbor_depth), dtype=np.int64)
        self.mt = (MT * 64)()
        self._inject = None
        self.n_threads = 1

    # -- struct plumbing --------------------------------------------------
    def _state(self):
        st = State()
        st.pos, st.pos1, st.noise = _p(self.pos), _p(self.pos1), _p(self.noise_vec)
        st.tangent, st.forces = _p(self.tangent_list), _p(self.forces)
        st.where_active, st.where_is_bead = _p(self.where_active), _p(self.where_is_bead)
        st.chain_id, st.rest_lengths = _p(self.chain_id), _p(self.rest_lengths)
        st.grid_list = _p(self.grid_list)
        st.n_grid, st.n_grid_z, st.grid_depth1 = self.grid_list.shape[0], self.grid_list.shape[2], \
            self.grid_list.shape[3]
        st.nbor_list, st.nbor_depth1 = _p(self.nbor_list), self.nbor_list.shape[1]
        if self._inject is not None:
            st.noise_inject, st.noise_inject_steps = _p(self._inject), self._inject.shape[0]
        st.mt = C.addressof(self.mt)
        st.forces_aux = _p(self.forces_aux)
        return st

    def seed_mt(self, seed, n_threads=1):
        """Seed the per-thread MT19937 streams (thread t gets seed + t)."""
        for t in range(min(n_threads, 64)):
            lib(self.variant).gcro_mt_seed(C.byref(self.mt[t]), (seed + t) & 0xFFFFFFFF)

    def set_injected_noise(self, snapshots):
        self._inject = np.ascontiguousarray(snapshots, dtype=np.float64)

    # -- list construction -------------------------------------------------
    def build_lists(self, grid_window=None):
        """Initial lists as ``configure_start`` builds them (control.py:116-150)."""
        L = lib(self.variant)
        while True:
            st = self._state()
            if L.gcro_update_grid_list(C.byref(st), _p(self.pos), self.N, self.L, self.dim, 0, 1, 0):
                break
            g = self.grid_list
            self.grid_list = np.zeros(g.shape[:-1] + (2 * g.shape[-1],), dtype=np.int64)
        if grid_window is None:
            grid_window = max(1, int(math.ceil(self.radius * self.n_grid / self.L)))
        while True:
            st = self._state()
            L.gcro_update_nbor_list(C.byref(st), _p(self.pos), self.N, self.L, self.n_nearby,
                                    grid_window, self.dim)
            if np.all(self.nbor_list[:, 0] >= 0):
                break
            self.nbor_list = np.concatenate((self.nbor_list, np.zeros_like(self.nbor_list)), axis=1)

    # -- the step ---------------------------------------------------------
    def run(self, n_steps, dt, dtmax=None, max_dist_per_step=math.inf, rk_cheat=1.0,
            max_dt_usable=-1.0, steps_until_update=40, n_steps_update=40, noise_mode=NOISE_MT,
            seed=0, step0=0, n_threads=1, calc_active=True):
        """Run ``SRK_jit`` for up to ``n_steps`` steps.  Returns the row
        ``shared_arr[0]`` as a dict (dt, elapsed, steps, max force, flag)."""
        p = self._params(n_threads, noise_mode, calc_active)
        p.dt = dt
        p.dtmax = dt if dtmax is None else dtmax
        p.max_dist_per_step, p.rk_cheat, p.max_dt_usable = max_dist_per_step, rk_cheat, max_dt_usable
        p.steps_until_update, p.n_steps_update, p.max_steps = steps_until_update, n_steps_update, n_steps
        p.seed, p.step0 = seed, step0
        res = Result()
        st = self._state()
        rc = lib(self.variant).gcro_srk2_run(C.byref(p), C.byref(st), C.byref(res))
        if rc != 0:
            raise RuntimeError(f"oracle srk2 run failed ({rc})")
        return {"dt": res.dt, "dt_used": res.dt_used_total, "steps": int(res.steps),
                "max_forces_strength": res.max_forces_strength, "flag": res.flag}

    def _params(self, n_threads=1, noise_mode=NOISE_MT, calc_active=True):
        p = Params()
        p.dim, p.n_threads, p.L = self.dim, n_threads, self.L
        p.n_beads, p.n_chains = self.N, len(self.rest_lengths)
        p.calc_springs, p.calc_wca = int(self.calc_springs), int(self.calc_wca)
        p.self_propel = int(self.do_self_propel and calc_active)
        p.noise_mode = noise_mode
        for i in range(6):
            p.spring[i] = self.spring_params[i]
        for i in range(4):
            p.wca[i] = self.WCA_params[i]
        for i in range(3):
            p.active[i] = self.active[i]
        p.D, p.Dr, p.radius, p.rigid_rod = self.D, self.Dr, self.radius, self.rigid_rod
        p.n_nearby, p.longest_chain_length = self.n_nearby, self.longest_chain_length
        p.grid_factor = self.grid_factor
        p.srk_order = self.srk_order
        p.seed = getattr(self, "seed", 0)
        return p

    def chain_start(self):
        cs = np.flatnonzero(np.diff(self.chain_id)) + 1
        return np.concatenate(([0], cs, [self.N])).astype(np.int64)

    def order_params(self):
        return order_params(self.tangent_list, self.chain_start())


# ---------------------------------------------------------------------------
# several populations in one box
# ---------------------------------------------------------------------------

def mean_wca(wca_a, wca_b):
    """The default cross parameters: ``0.5 * (WCA_params + other.WCA_params)``
    (``WCA_Population.interactions``, populations.py:226-232)."""
    return 0.5 * (np.asarray(wca_a, dtype=np.float64) + np.asarray(wca_b, dtype=np.float64))


def cross_forces(pos_p, pos_q, wca_params, L):
    """The WCA force on every bead of population P from the beads of
    population Q (forces.central_pair_force over P's nbor_list of Q), over all
    pairs within the cutoff."""
    pos_p = np.ascontiguousarray(pos_p, dtype=np.float64)
    pos_q = np.ascontiguousarray(pos_q, dtype=np.float64)
    out = np.zeros_like(pos_p)
    chain = np.zeros(len(pos_p), dtype=np.int64)
    lib().gcro_pair_forces_all(_p(pos_p), len(pos_p), _p(chain), 0, _p(pos_q), len(pos_q), 0,
                               _p(np.ascontiguousarray(wca_params, dtype=np.float64)), float(L), pos_p.shape[1],
                               _p(out))
    return out


class OracleGroup:
    """Populations stepped together as ``updates.SRK2_force_calc`` steps a list
    of populations (updates.py:146-247): one dt from the largest max-force
    value over the moving populations, and the force of every other
    population added after a population's own forces (SRK.py:229-245,
    287-294).  SRK2, one thread per population; pair forces over all pairs.

    ``systems``: ``OracleSystem`` per population (each with a ``seed``
    attribute for the Philox stream), ``fixed[k]``: population k never moves,
    ``cross[k][q]``: the WCA parameters of the force on k from q."""

    def __init__(self, systems, fixed, cross, motors=None):
        self.systems = list(systems)
        n = len(self.systems)
        self.fixed = np.asarray([1 if f else 0 for f in fixed], dtype=np.int32)
        self.cross = np.ascontiguousarray(np.asarray(cross, dtype=np.float64).reshape(n, n, 4))
        # motors: dict(motor_pop, chain_pop, params [5], dont_diffuse, list_r2); where_active of
        # every population is kept in self.where_active (int32, -1 at each step start)
        self.motors = motors
        self.where_active = [np.zeros(s.N, dtype=np.int32) for s in self.systems]

    def run(self, n_steps, dt, dtmax=None, max_dist_per_step=math.inf, rk_cheat=1.0, max_dt_usable=-1.0,
            noise_mode=NOISE_PHILOX, step0=0, calc_active=True, srk_order=2):
        """SRK2, or the SRK4 branch with ``srk_order=4`` (every system made
        with ``srk_order=4``, so that it has its ``forces_aux``)."""
        L = lib()
        n = len(self.systems)
        ps = [s._params(1, noise_mode, calc_active) for s in self.systems]
        sts = [s._state() for s in self.systems]
        g = Params()
        s0 = self.systems[0]
        g.dim, g.L, g.dt = s0.dim, s0.L, dt
        g.dtmax = dt if dtmax is None else dtmax
        g.max_dist_per_step, g.rk_cheat, g.max_dt_usable = max_dist_per_step, rk_cheat, max_dt_usable
        g.max_steps, g.noise_mode, g.step0 = n_steps, noise_mode, step0
        g.srk_order = srk_order
        p_arr = (C.POINTER(Params) * n)(*[C.pointer(p) for p in ps])
        s_arr = (C.POINTER(State) * n)(*[C.pointer(st) for st in sts])
        res = Result()
        if self.motors is not None:
            mo = Motors()
            mo.motor_pop, mo.chain_pop = self.motors["motor_pop"], self.motors["chain_pop"]
            mo.dont_diffuse = 1 if self.motors.get("dont_diffuse", True) else 0
            for i, v in enumerate(self.motors["params"]):
                mo.params[i] = v
            mo.list_r2 = self.motors["list_r2"]
            for k, a in enumerate(self.where_active):
                mo.act[k] = a.ctypes.data
            rc = L.gcro_group_run_motors(n, p_arr, s_arr, _p(self.fixed), _p(self.cross), C.byref(g),
                                         C.byref(res), C.byref(mo))
        else:
            rc = L.gcro_group_run(n, p_arr, s_arr, _p(self.fixed), _p(self.cross), C.byref(g), C.byref(res))
        if rc != 0:
            raise RuntimeError(f"oracle group run failed ({rc})")
        return {"dt": res.dt, "dt_used": res.dt_used_total, "steps": int(res.steps),
                "max_forces_strength": res.max_forces_strength}
