"""ctypes binding of ``libgcr.so`` (the C ABI in ``include/gcr.h``).

The library is built in-tree by ``gliding_collective_rotation_b200.build``.
There is no fallback: if the shared library is missing or a call fails, a
``GcrError`` is raised.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; GCR_LIBRARY names another build of the same sources (a
# different revision to compare against, say)
LIB_PATH = os.environ.get("GCR_LIBRARY") or os.path.join(HERE, "libgcr.so")

GCR_OK = 0
ERRORS = {-1: "BAD_ARG", -2: "CUDA", -3: "OOM", -4: "NONFINITE", -5: "TIMEOUT", -6: "CAPACITY",
          -7: "STATE", -8: "OVERFLOW"}
GCR_FP64, GCR_MIXED = 0, 1
FLAG_CELL_OVERFLOW, FLAG_NONFINITE, FLAG_NEXT_OVERFLOW, FLAG_LIST_CORRUPT, FLAG_LIST_OVERFLOW = 1, 2, 4, 8, 16
FLAG_SERIES_FULL = 32


class GcrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"gcr error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("dim", C.c_int32), ("precision", C.c_int32), ("bead_capacity", C.c_int64),
                ("system_capacity", C.c_int32), ("cell_capacity", C.c_int64), ("cell_depth", C.c_int32),
                ("block_beads", C.c_int32), ("block_cells", C.c_int32), ("steps_per_graph", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("list_depth", C.c_int32), ("srk_order", C.c_int32),
                ("pair_mode", C.c_int32)]


class SystemDesc(C.Structure):
    _fields_ = [("n_beads", C.c_int64), ("n_chains", C.c_int64), ("L", C.c_double),
                ("spring_params", C.c_double * 6), ("wca_params", C.c_double * 4),
                ("active_params", C.c_double * 3), ("calc_springs", C.c_int32), ("calc_wca", C.c_int32),
                ("self_propel", C.c_int32), ("n_nearby", C.c_int32), ("D", C.c_double), ("Dr", C.c_double),
                ("radius", C.c_double), ("dtmax", C.c_double), ("max_dist_per_step", C.c_double),
                ("rk_cheat", C.c_double), ("seed", C.c_uint64), ("step", C.c_int64),
                ("cell_factor", C.c_double), ("skin", C.c_double), ("rigid_rod", C.c_double)]


class SystemBuffers(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("pos1", C.c_void_p), ("tangent", C.c_void_p), ("forces", C.c_void_p),
                ("chain_id", C.c_void_p), ("rest_lengths", C.c_void_p), ("forces_aux", C.c_void_p)]


class Call(C.Structure):
    _fields_ = [("max_steps", C.c_int64), ("max_dt_usable", C.c_double), ("dt", C.c_double),
                ("noise", C.c_void_p), ("noise_steps", C.c_int64), ("series", C.c_void_p),
                ("series_every", C.c_int64), ("series_phase", C.c_int64), ("series_capacity", C.c_int64)]


class Status(C.Structure):
    _fields_ = [("dt", C.c_double), ("dt_used", C.c_double), ("max_forces_strength", C.c_double),
                ("steps_done", C.c_int64), ("step", C.c_int64), ("flags", C.c_int32), ("active", C.c_int32),
                ("list_builds", C.c_int64), ("series_rows", C.c_int64)]


# exported symbols and their signatures (every declaration of include/gcr.h)
SIGNATURES = {
    "gcr_create": (C.c_int, [C.POINTER(Config), C.c_void_p, C.POINTER(C.c_void_p)]),
    "gcr_destroy": (C.c_int, [C.c_void_p]),
    "gcr_last_error": (C.c_char_p, []),
    "gcr_version": (C.c_int, []),
    "gcr_admit": (C.c_int, [C.c_void_p, C.POINTER(SystemDesc), C.POINTER(SystemBuffers),
                            C.POINTER(C.c_int32)]),
    "gcr_evict": (C.c_int, [C.c_void_p, C.c_int32]),
    "gcr_update_desc": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(SystemDesc)]),
    "gcr_call_begin": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Call)]),
    "gcr_call_begin_batch": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(Call)]),
    "gcr_footprint": (C.c_int, [C.POINTER(Config), C.POINTER(SystemDesc), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int64)]),
    "gcr_run": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32]),
    "gcr_get_status": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Status)]),
    "gcr_get_statuses": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(Status)]),
    "gcr_count_active": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "gcr_synchronize": (C.c_int, [C.c_void_p]),
    "gcr_profile_steps": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_float)]),
    "gcr_order_params": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "gcr_reference_lists": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                                      C.c_int64, C.c_void_p, C.c_int64, C.c_int32]),
    "gcr_cell_assignment": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int32)]),
    "gcr_chain_frames": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "gcr_pair_correlation": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.POINTER(C.c_double),
                                       C.c_int32, C.POINTER(C.c_int32)]),
    "gcr_neighbour_list": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                     C.POINTER(C.c_int64)]),
    "gcr_philox_noise": (C.c_int, [C.c_int32, C.c_uint64, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                   C.c_void_p, C.c_void_p]),
    "gcr_unwrapped_positions": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "gcr_reset_images": (C.c_int, [C.c_void_p, C.c_int32]),
    "gcr_couple": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                             C.POINTER(C.c_double)]),
    "gcr_decouple": (C.c_int, [C.c_void_p, C.c_int32]),
    "gcr_set_motors": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.c_int32]),
    "gcr_where_active": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "gcr_order_params_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64,
                                           C.POINTER(C.c_double), C.c_void_p]),
}

_lib = None


def load(path=None):
    """Load ``libgcr.so``; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise GcrError(-2, f"{path} is missing; build it with "
                           "`python -m gliding_collective_rotation_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    if rc != GCR_OK:
        msg = load().gcr_last_error()
        raise GcrError(rc, msg.decode() if msg else "")
    return rc
