"""The reference's analysis observables for resident systems.

* ``chain_frames``: per chain, the centre that ``analysis.chain_COM``
  computes (analysis.py:288-292 -- the head plus the *summed* separations
  head - x_i, wrapped, exactly as the reference writes it) and the mean chain
  angle of ``output_methods.calc_avg_phi_chain`` (output_methods.py:492-510)
  with 1- and 2-fold symmetry; on the GPU (``gcr_chain_frames``).
* ``pair_correlation``: ``analysis.g_of_r``, ``analysis.Cvv`` and
  ``analysis.Cnn`` (analysis.py:203-275) over the chain centres, one GPU
  thread per chain pair (``gcr_pair_correlation``); 2D.
* ``order_parameters``: P, S and the director angle
  (analysis.py:294-328, ``gcr_order_params``).
* ``rotation_rate`` and ``remove_outliers``: the collective rotation rate of
  the paper's analysis (``rotation_rate1`` and ``remove_outliers_zscore`` of
  Chiral_paper_plots/Main_figs/Plots.ipynb) from a series of
  (t, P, S, director angle) rows, e.g. ``serve.Result.series``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import check

KINDS = {"g_of_r": 0, "Cvv": 1, "Cnn": 2}


def chain_frames(engine, slot):
    """(centres [n_chains, d], phi [n_chains, 2]) as numpy arrays."""
    st = engine.systems[slot]
    dev = st.pos.device
    com = torch.zeros((st.n_chains, engine.dim), dtype=torch.float64, device=dev)
    phi = torch.zeros((st.n_chains, 2), dtype=torch.float64, device=dev)
    torch.cuda.current_stream(dev).synchronize()
    check(engine.lib.gcr_chain_frames(engine._ctx, int(slot), C.c_void_p(com.data_ptr()), C.c_void_p(phi.data_ptr())))
    return com.cpu().numpy(), phi.cpu().numpy()


def pair_correlation(engine, slot, kind="g_of_r", binsize=0.25):
    """Rows (r, value) with r < L/2, as ``analysis.correlation_func``."""
    st = engine.systems[slot]
    L = float(st.params.L)
    rows = int(np.ceil(L / 2 / binsize)) + 2
    out = (C.c_double * (2 * rows))()
    n = C.c_int32()
    torch.cuda.current_stream(st.pos.device).synchronize()
    check(engine.lib.gcr_pair_correlation(engine._ctx, int(slot), KINDS[kind], float(binsize), out, rows,
                                          C.byref(n)))
    return np.array(out[:2 * n.value]).reshape(-1, 2)


def order_parameters(engine, slot):
    """[P, S, director angle]."""
    return engine.order_params(slot)


def _angle_differences(a2, a1):
    return np.angle(np.exp(1j * a2) / np.exp(1j * a1))


def rotation_rate(series, lag=4, time_rescale=15.5, s_threshold=0.7):
    """(time, angle, omega) from rows (t, P, S, angle): from the first row
    with S above the threshold, the director rotation over `lag` rows divided
    by the elapsed rescaled time; None if S never exceeds the threshold."""
    series = np.asarray(series, dtype=np.float64)
    t, S, angle = series[:, 0], series[:, 2], series[:, 3]
    index = int(np.argmax(S > s_threshold))
    if not S[index] > s_threshold:
        return None
    k = np.arange(index, len(t) - lag)
    dtime = (t[k + lag] - t[k]) / time_rescale
    return t[k + lag] / time_rescale, angle[k + lag], _angle_differences(angle[k + lag], angle[k]) / dtime


def remove_outliers(omega, time, threshold=2.0):
    """Rates within `threshold` population standard deviations of the mean."""
    z = np.abs((omega - omega.mean()) / omega.std())
    keep = np.nonzero(z <= threshold)[0]
    return time[keep], omega[keep]
