"""Loading helpers for the golden fixtures made by ``tests/golden/make_golden.py``."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["config1", "chiral_lj", "rotdiff2d", "rotdiff3d", "adaptive", "paper_chiral", "rigid2d", "rigid3d",
         "srk4_2d", "srk4_3d", "srk4_rigid", "grow3d"]
STATUS_FIELDS = ["dt", "dt_used", "stepnum", "t", "update_grid_list_counter", "max_forces_strength",
                 "next_output_step", "next_save_time", "dtmax"]


def load(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return d, json.loads(str(d["scalars"]))


def status_dict(row):
    return dict(zip(STATUS_FIELDS, row.tolist()))


def pairs_from_nbor(nbor_list):
    rows = []
    for b1 in range(nbor_list.shape[0]):
        for k in range(nbor_list[b1, 0]):
            rows.append((b1, nbor_list[b1, 1 + k]))
    return np.array(rows, dtype=np.int32).reshape(-1, 2)


def min_image(d, L):
    return (d + L / 2) % L - L / 2


# Trajectory tolerances (max abs position difference, in box units) per call
# index.  Cases with LJ attraction or kappa=100 plus adaptive dt are chaotic:
# ulp-level differences in the bend force (acos(c)/sqrt(1-c^2) for nearly
# straight chains) grow by ~1e3 per 50 steps, so only the first calls are
# inside the predictability horizon there.
TRAJ_TOL = {
    "config1": [1e-9, 1e-9, 1e-9, 1e-9],
    "chiral_lj": [1e-9, 1e-6, None],
    "rotdiff2d": [1e-11, 1e-11, 1e-11],
    "rotdiff3d": [1e-11, 1e-11, 1e-11],
    "adaptive": [1e-9, 1e-9, 1e-9, 1e-9, 1e-9],
    "paper_chiral": [1e-9, 1e-6],
    "rigid2d": [1e-9, 1e-9, 1e-9],
    "rigid3d": [1e-9, 1e-9, 1e-9],
    "srk4_2d": [1e-9, 1e-9, 1e-9],
    "srk4_3d": [1e-9, 1e-9, 1e-9],
    "srk4_rigid": [1e-9, 1e-9, 1e-9],
    "grow3d": [1e-9, 1e-9, 1e-9],
}
