#!/usr/bin/env python3
"""Golden vectors of the paper's rotation-rate analysis on the paper's own
runs.

Run from the repository root where the reference source is mounted at
/root/reference (read-only; nothing is written there):

    python tests/golden/make_paper_rotation_golden.py [--ref /root/reference] [--out tests/golden]

Three (t, P, S, director angle) series of the reference's chiral runs
(``Chiral_paper_plots/Main_figs/Data.zip``: kappa 30, 100 and 300, case 0;
the output of ``global_op-chiral.py`` for runs of ``Chiral_parameters_script.sh``)
go through the paper notebook's ``rotation_rate1`` and
``remove_outliers_zscore`` (``Plots.ipynb``, its source cells executed as they
are).  Recorded (``paper_rotation.npz``): each series, the estimator's
(time, angle, omega), the outlier-free (time, omega) and their mean.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import zipfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_observables_golden import _notebook_functions  # noqa: E402

CASES = {"k30": "Data/Ckappa_30Case0", "k100": "Data/Ckappa_100Case0", "k300": "Data/Ckappa_300Case0"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args()
    main_figs = os.path.join(a.ref, "Chiral_paper_plots", "Main_figs")
    ns = _notebook_functions(os.path.join(main_figs, "Plots.ipynb"),
                             ["angle_differences", "rotation_rate1", "remove_outliers_zscore"])
    z = zipfile.ZipFile(os.path.join(main_figs, "Data.zip"))
    work = tempfile.mkdtemp(prefix="gcr_paper_")
    out = {}
    for key, member in CASES.items():
        series = np.loadtxt(z.read(member).decode().splitlines())
        fn = os.path.join(work, key + ".txt")
        np.savetxt(fn, series)
        rt, rangle, omega = ns["rotation_rate1"](fn)
        ct, comega = ns["remove_outliers_zscore"](omega, rt)
        out.update({f"{key}_series": series, f"{key}_time": rt, f"{key}_angle": rangle, f"{key}_omega": omega,
                    f"{key}_clean_time": ct, f"{key}_clean_omega": comega,
                    f"{key}_mean_omega": np.mean(comega)})
        print(key, member, "rows", len(series), "mean omega", np.mean(comega))
    path = os.path.join(a.out, "paper_rotation.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
