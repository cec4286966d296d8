"""CPU restatement of the reference's observables -- test infrastructure.

Only the tests (and the bench's CPU arm) use this module, to check the GPU
observables in ``gliding_collective_rotation_b200/observables.py``.
It follows the reference definition by definition and is pinned to the
reference's own outputs in ``tests/golden/observables.npz`` (made by
``tests/golden/make_observables_golden.py``).

* ``chain_com``: analysis.chain_COM (analysis.py:288-292).  The reference
  adds, to the head bead, the sum (not the mean) of the min-image
  separations head - x_i over the chain, then wraps; reproduced as is.
* ``avg_phi``: output_methods.calc_avg_phi_chain (output_methods.py:492-510).
* ``correlation``: analysis.correlation_func (analysis.py:203-241) with the
  pair functions of g_of_r, Cvv and Cnn (analysis.py:243-275).  Distances
  past the last bin (possible when L/2 is not an integer) are not counted;
  the reference would index past its array there.
* ``rotation_rate`` and ``remove_outliers``: rotation_rate1 and
  remove_outliers_zscore of the paper's analysis notebook
  (Chiral_paper_plots/Main_figs/Plots.ipynb).
"""
from __future__ import annotations

import numpy as np


def _true_sep(pt1, pt2, L):
    # analysis.true_sep (analysis.py:185-187): floor-mod wrap of pt2 - pt1
    return np.mod(pt2 - pt1 + L / 2, L) - L / 2


def chain_com(pos, chain_start, L):
    out = np.empty((len(chain_start) - 1, pos.shape[1]))
    for c in range(len(chain_start) - 1):
        b0, b1 = chain_start[c], chain_start[c + 1]
        head = pos[b0]
        out[c] = np.mod(head + np.sum(_true_sep(pos[b0:b1], head, L), axis=0), L)
    return out


def avg_phi(tangent, chain_start, n_fold=1):
    out = np.empty(len(chain_start) - 1)
    for c in range(len(chain_start) - 1):
        t = tangent[chain_start[c]:chain_start[c + 1]]
        if n_fold == 1:
            out[c] = np.arctan2(np.sum(t[:, 1]), np.sum(t[:, 0]))
        else:
            phi = np.arctan2(t[:, 1], t[:, 0])
            out[c] = np.arctan2(np.sum(np.sin(n_fold * phi)), np.sum(np.cos(n_fold * phi))) / n_fold
    return out


def correlation(com, L, kind, binsize=0.25, phi1=None, phi2=None, chunk=512):
    """``kind`` 0: g(r) (norm 'all'), 1: Cvv, 2: Cnn (norm 'bin').  Returns
    rows (r, value) with r < L/2, as correlation_func does."""
    bin_ranges = np.arange(0, int(L / 2) * np.sqrt(2), binsize)
    nb = bin_ranges.shape[0]
    sums = np.zeros(nb)
    counts = np.zeros(nb, dtype=np.int64)
    nc = len(com)
    for i0 in range(0, nc, chunk):
        ci = np.arange(i0, min(nc, i0 + chunk))
        for i in ci:
            cj = np.arange(i)
            if len(cj) == 0:
                continue
            sep = _true_sep(com[i], com[cj], L)
            dist = np.sqrt(np.sum(sep ** 2, axis=1))
            b = (dist / binsize).astype(np.int64)
            ok = b < nb
            if kind == 0:
                f = np.ones(len(cj))
            elif kind == 1:
                f = np.cos(phi1[i]) * np.cos(phi1[cj]) + np.sin(phi1[i]) * np.sin(phi1[cj])
            else:
                f = np.abs(np.cos(phi2[i]) * np.cos(phi2[cj]) + np.sin(phi2[i]) * np.sin(phi2[cj]))
            np.add.at(sums, b[ok], 2 * f[ok])
            np.add.at(counts, b[ok], 2)
    if kind == 0:
        density = np.sum(counts) / (L * L)
        denom = density * 2 * np.pi * binsize * (bin_ranges + binsize / 2)
    else:
        denom = np.maximum(counts, 1)
    values = sums / denom
    keep = bin_ranges < L / 2
    return np.stack((bin_ranges[keep], values[keep]), axis=1)


def rotation_rate(series, lag=4, time_rescale=15.5, s_threshold=0.7):
    """(time, angle, omega) from rows (t, P, S, angle), or None if S never
    exceeds the threshold."""
    t, S, angle = series[:, 0], series[:, 2], series[:, 3]
    index = int(np.argmax(S > s_threshold))
    if not S[index] > s_threshold:
        return None
    k = np.arange(index, len(t) - lag)
    dtime = (t[k + lag] - t[k]) / time_rescale
    dangle = np.angle(np.exp(1j * angle[k + lag]) / np.exp(1j * angle[k]))
    return t[k + lag] / time_rescale, angle[k + lag], dangle / dtime


def remove_outliers(omega, time, threshold=2.0):
    z = np.abs((omega - omega.mean()) / omega.std())
    keep = np.nonzero(z <= threshold)[0]
    return time[keep], omega[keep]
