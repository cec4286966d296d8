#!/usr/bin/env python3
"""Golden vectors of the motor push: the reference's own
``forces.calc_motor_push`` (forces.py:248-283) run on seeded synthetic
states.

Run from the repository root where the reference source is mounted
(read-only) at /root/reference and Numba is installed:

    python tests/golden/make_motor_golden.py [--ref /root/reference] [--out tests/golden]

The reference is prepared as ``make_golden.py`` prepares it (a scratch copy,
matplotlib stubbed, the numpy aliases restored); each dimension runs in a
fresh process because Numba freezes ``config.dim`` at the first compile.
Per case the script draws chain beads (positions, unit tangents) and motors
in a box, with some motors already attached, builds every bead's
motor-neighbour list in the reference's format (``[count, ids...]``, the
motors within the list radius in ascending id), seeds Numba's generator
(``np.random.seed`` inside an ``@njit`` function, the stream
``np.random.random`` then draws from) and calls ``calc_motor_push`` twice,
as the two stages of an SRK2 step do, recording the forces and both
``where_active`` arrays after each call.  The fixture is
``motor_push.npz``.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_golden import _install_shims  # noqa: E402

CASES = {
    # dim, beads, motors, box side, list radius, params [max_dist_sq, one_per_bead, force, k_on, k_off], seeds
    "m2d": dict(dim=2, nb=240, nm=160, L=12.0, list_r=0.9, params=[0.16, 0.0, 1.5, 0.6, 0.3], seed=3, rng=11),
    "m2d_one": dict(dim=2, nb=200, nm=200, L=10.0, list_r=1.0, params=[0.25, 1.0, 0.8, 0.9, 0.5], seed=5, rng=13),
    "m3d": dict(dim=3, nb=300, nm=200, L=6.0, list_r=1.1, params=[0.3, 0.0, 2.0, 0.7, 0.2], seed=7, rng=17),
}


def make_inputs(c):
    rs = np.random.RandomState(c["seed"])
    dim, nb, nm, L = c["dim"], c["nb"], c["nm"], c["L"]
    pos_b = rs.uniform(0, L, (nb, dim))
    t = rs.normal(size=(nb, dim))
    t /= np.linalg.norm(t, axis=1)[:, None]
    pos_m = rs.uniform(0, L, (nm, dim))
    where_m = np.full(nm, -1, dtype=np.int64)
    attached = rs.rand(nm) < 0.3
    where_m[attached] = rs.randint(0, nb, attached.sum())
    where_b = np.full(nb, -1, dtype=np.int64)
    d = pos_m[None, :, :] - pos_b[:, None, :]
    d -= L * np.round(d / L)
    r2 = np.sum(d * d, axis=2)
    lists = [np.flatnonzero(r2[b] <= c["list_r"] ** 2) for b in range(nb)]
    depth = max(1, max(len(x) for x in lists))
    nbor = np.zeros((nb, 1 + depth), dtype=np.int64)
    for b, x in enumerate(lists):
        nbor[b, 0] = len(x)
        nbor[b, 1:1 + len(x)] = x
    return dict(pos_b=pos_b, tangent=t, pos_m=pos_m, where_m=where_m, where_b=where_b, nbor=nbor,
                params=np.array(c["params"], dtype=np.float64), L=np.float64(L))


def run_one(name, ref, out):
    c = CASES[name]
    scratch = tempfile.mkdtemp(prefix="gcr_ref_")
    dst = os.path.join(scratch, "ref")
    shutil.copytree(ref, dst)
    for root, dirs, files in os.walk(dst):
        for d in dirs:
            os.chmod(os.path.join(root, d), 0o755)
        for fn in files:
            os.chmod(os.path.join(root, fn), 0o644)
    cwd = os.getcwd()
    os.chdir(dst)
    sys.path.insert(0, dst)
    _install_shims()
    import populations  # noqa: F401  (must come first: circular imports)
    import config
    config.dim = c["dim"]
    import forces
    from numba import njit

    @njit
    def _seed(s):
        np.random.seed(s)

    os.chdir(cwd)
    inp = make_inputs(c)
    rec = {f"{name}_{k}": v for k, v in inp.items()}
    forces_b = np.zeros_like(inp["pos_b"])
    where_b, where_m = inp["where_b"].copy(), inp["where_m"].copy()
    _seed(c["rng"])
    rec[f"{name}_rng_seed"] = np.int64(c["rng"])
    for call in range(2):
        forces.calc_motor_push(inp["pos_b"], inp["nbor"], forces_b, where_b, inp["tangent"], inp["L"],
                               inp["pos_m"], where_m, inp["params"])
        rec[f"{name}_forces{call}"] = forces_b.copy()
        rec[f"{name}_where_b{call}"] = where_b.copy()
        rec[f"{name}_where_m{call}"] = where_m.copy()
    np.savez_compressed(os.path.join(out, f"motor_{name}.npz"), **rec)
    shutil.rmtree(scratch)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--one", default=None, help="run one case in this process (internal)")
    args = ap.parse_args()
    if args.one:
        run_one(args.one, args.ref, args.out)
        return
    merged = {}
    for name in CASES:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--one", name, "--ref", args.ref,
                        "--out", args.out], check=True)
        part = os.path.join(args.out, f"motor_{name}.npz")
        with np.load(part) as z:
            merged.update({k: z[k] for k in z.files})
        os.remove(part)
    np.savez_compressed(os.path.join(args.out, "motor_push.npz"), **merged)


if __name__ == "__main__":
    main()
