#!/usr/bin/env python3
"""State files written by the reference's own ``output_methods.save_state``
(output_methods.py:420-466), for the format tests of ``state_io``.

Run from the repository root where the reference source is mounted at
/root/reference (read-only; nothing is written there):

    python tests/golden/make_state_golden.py [--ref /root/reference] [--out tests/golden]

A 2D population (the relaxed state of ``config1.npz``) and a small 3D one
(seeded chains) are written by ``save_state`` as the reference writes them
during a run: the population object is a reference ``Equal_Size_Chain_Collection``
carrying only the arrays ``save_state`` reads.  Output: ``state2d_beads_00000007.dat``
and ``state3d_beads_00000012.dat``.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import sys
import tempfile
import types

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_golden import _install_shims  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__))))
    a = ap.parse_args()
    out = os.path.abspath(a.out)
    _install_shims()
    for name in [m for m in list(sys.modules) if "." in m]:
        parent, child = name.rsplit(".", 1)
        if parent in sys.modules and type(sys.modules[name]).__name__ == "_Stub":
            setattr(sys.modules[parent], child, sys.modules[name])
    work = tempfile.mkdtemp(prefix="gcr_state_")
    shutil.copytree(a.ref, os.path.join(work, "ref"), ignore=shutil.ignore_patterns("*.zip", "*.ipynb"))
    sys.path.insert(0, os.path.join(work, "ref"))
    os.chdir(os.path.join(work, "ref"))
    import populations
    import config
    import output_methods

    def pop_of(pos, tangent, chain):
        pop = object.__new__(populations.Equal_Size_Chain_Collection)
        pop.name = "beads"
        pop.pos = pos
        pop.tangent_list = tangent
        pop.chain_id = chain
        pop.inherited_label = chain.copy()
        pop.orientations = np.zeros((len(pos), pos.shape[1] - 1))
        pop.where_active = np.zeros(len(pos), dtype=np.int64)
        return pop

    d = np.load(os.path.join(out, "config1.npz"))
    sim = {"b_save_most_recent_only": False, "n_digits_stepnum_str": 8}
    config.dim = 2
    sim["outfileprefix"] = os.path.join(out, "state2d")
    status = types.SimpleNamespace(filenumber=7, stepnum=1234, t=1.2345678)
    output_methods.save_state(sim, [pop_of(d["pos0"].copy(), d["tangent0"].copy(),
                                           np.asarray(d["chain_id"], dtype=np.int64))], status)
    rng = np.random.default_rng(5)
    n_chains, clen, L = 12, 6, 20.0
    t = rng.standard_normal((n_chains, 3))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    heads = rng.uniform(0, L, size=(n_chains, 3))
    pos = np.mod((heads[:, None, :] - 0.5 * np.arange(clen)[None, :, None] * t[:, None, :]).reshape(-1, 3), L)
    tan = np.repeat(t, clen, axis=0)
    config.dim = 3
    sim["outfileprefix"] = os.path.join(out, "state3d")
    status = types.SimpleNamespace(filenumber=12, stepnum=99, t=0.5)
    output_methods.save_state(sim, [pop_of(pos, tan, np.repeat(np.arange(n_chains), clen))], status)
    json.dump({"state3d_L": L}, open(os.path.join(out, "state_index.json"), "w"))
    print("wrote", sorted(f for f in os.listdir(out) if f.startswith("state")))


if __name__ == "__main__":
    main()
