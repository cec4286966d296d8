#!/usr/bin/env python3
"""Golden vectors of the reference's observables, made by running the
reference's own functions.

Run from the repository root where the reference source is mounted at
/root/reference (read-only; nothing is written there):

    python tests/golden/make_observables_golden.py [--ref /root/reference] [--out tests/golden]

Inputs are the relaxed 2,000-bead state of ``config1.npz`` (200 chains of 10
beads, L = 60) and, for the rotation rate, a seeded synthetic series of
(t, P, S, director angle).  Recorded (``observables.npz``):

* ``analysis.chain_COM`` of every chain (analysis.py:288-292);
* ``output_methods.calc_avg_phi_chain`` with n-fold symmetry 1 and 2
  (output_methods.py:492-510);
* ``analysis.g_of_r``, ``analysis.Cvv``, ``analysis.Cnn`` with bin size 0.25
  (analysis.py:203-275);
* ``rotation_rate1`` and ``remove_outliers_zscore`` of the paper's analysis
  notebook (Chiral_paper_plots/Main_figs/Plots.ipynb), whose source cells are
  executed as they are.

The reference is imported with the shims of ``make_golden.py`` (matplotlib
stubbed, ``np.float``/``np.int`` restored), from a scratch copy.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import sys
import tempfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_golden import _install_shims  # noqa: E402


class _Beads:
    """The parts of a reference chain population the observables read."""

    def __init__(self, pos, tangent, chain_id):
        self.pos = pos
        self.tangent_list = tangent
        self.total_pop = len(pos)
        n_chains = int(chain_id.max()) + 1
        lengths = np.bincount(chain_id, minlength=n_chains)
        self.phonebook = np.zeros((n_chains, 1 + lengths.max()), dtype=np.int64)
        start = 0
        for c in range(n_chains):
            self.phonebook[c, 0] = lengths[c]
            self.phonebook[c, 1:1 + lengths[c]] = np.arange(start, start + lengths[c])
            start += lengths[c]

    def num_chains(self):
        return self.phonebook.shape[0]


def _notebook_functions(path, names):
    nb = json.load(open(path))
    ns = {"np": np}
    from scipy import stats
    ns["stats"] = stats
    for cell in nb["cells"]:
        src = "".join(cell.get("source", []))
        if cell.get("cell_type") == "code" and any(f"def {n}(" in src for n in names):
            exec(compile(src, path, "exec"), ns)
    return ns


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__))))
    a = ap.parse_args()
    _install_shims()
    # `import matplotlib.pyplot as plt` reads the attribute of the parent stub
    for name in [m for m in list(sys.modules) if "." in m]:
        parent, child = name.rsplit(".", 1)
        if parent in sys.modules and type(sys.modules[name]).__name__ == "_Stub":
            setattr(sys.modules[parent], child, sys.modules[name])
    work = tempfile.mkdtemp(prefix="gcr_obs_")
    shutil.copytree(a.ref, os.path.join(work, "ref"), ignore=shutil.ignore_patterns("*.zip", "*.ipynb"))
    sys.path.insert(0, os.path.join(work, "ref"))
    os.chdir(os.path.join(work, "ref"))
    import populations  # noqa: F401  (import order of BDsim.py)
    import analysis
    import output_methods

    d = np.load(os.path.join(a.out, "config1.npz"))
    s = json.loads(str(d["scalars"]))
    pos, tan = d["pos0"].astype(np.float64), d["tangent0"].astype(np.float64)
    chain = np.asarray(d["chain_id"], dtype=np.int64)
    L = float(s["L"])
    beads = _Beads(pos, tan, chain)
    record = {"sim": {"Lx": L}, "pops": {"beads": beads}}
    nc = beads.num_chains()
    com = np.array([analysis.chain_COM(beads, c, L) for c in range(nc)])
    phi1 = np.array([output_methods.calc_avg_phi_chain(beads, c) for c in range(nc)])
    phi2 = np.array([output_methods.calc_avg_phi_chain(beads, c, n_fold_symmetry=2) for c in range(nc)])
    g = analysis.g_of_r(record, binsize=0.25)
    cvv = analysis.Cvv(record, binsize=0.25)
    cnn = analysis.Cnn(record, binsize=0.25)

    # a director-angle series: isotropic start, then ordered and rotating
    rng = np.random.default_rng(4)
    t = np.arange(0, 400.0, 2.0)
    S = np.clip(np.minimum(1.0, t / 150.0) + 0.02 * rng.standard_normal(len(t)), 0, 1)
    P = 0.5 * S
    angle = np.angle(np.exp(1j * (0.01 * t + 0.05 * rng.standard_normal(len(t)))))
    series = np.stack([t, P, S, angle], axis=1)
    fn = os.path.join(work, "series.txt")
    np.savetxt(fn, series)
    ns = _notebook_functions(os.path.join(a.ref, "Chiral_paper_plots", "Main_figs", "Plots.ipynb"),
                             ["angle_differences", "rotation_rate1", "remove_outliers_zscore"])
    rt, rangle, omega = ns["rotation_rate1"](fn)
    ct, comega = ns["remove_outliers_zscore"](omega, rt)

    out = os.path.join(a.out, "observables.npz")
    np.savez_compressed(out, com=com, phi1=phi1, phi2=phi2, g_of_r=g, cvv=cvv, cnn=cnn, series=series,
                        rot_time=rt, rot_angle=rangle, rot_omega=omega, rot_clean_time=ct, rot_clean_omega=comega,
                        L=L, binsize=0.25)
    print("wrote", out, "chains", nc, "bins", len(g))


if __name__ == "__main__":
    main()
