"""Several populations in one box: the golden fixtures made by
``tests/golden/make_multipop_golden.py`` (the reference's own multi-population
runs), and the oracle and GPU groups built from them."""
import json
import os

import numpy as np

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["pops2_2d", "pops3_fixed_2d", "pops2_3d"]


def load(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    d = {k: z[k] for k in z.files if k != "scalars"}
    s = json.loads(str(z["scalars"]))
    return d, s


def pop_arrays(d, s, k):
    """Population k of a case: its relaxed state and packed parameters."""
    return dict(pos=d[f"p{k}_pos0"], tangent=d[f"p{k}_tangent0"], chain_id=d[f"p{k}_chain_id"],
                rest_lengths=d[f"p{k}_rest_lengths"], spring=d[f"p{k}_spring_params"], wca=d[f"p{k}_wca_params"],
                active=d[f"p{k}_active_params"], D=s["D"][k], Dr=s["Dr"][k], radius=s["radius"][k],
                n_nearby=s["n_nearby"][k], longest=s["longest"][k], fixed=s["fixed"][k])


def oracle_group(d, s, D=None, seeds=None, srk_order=2, rigid=None):
    """An ``OracleGroup`` at the case's relaxed state (``D`` replaces every
    moving population's translational diffusion constant)."""
    systems = []
    for k in range(s["n_pops"]):
        a = pop_arrays(d, s, k)
        Dk = a["D"] if D is None or a["fixed"] else D
        o = O.OracleSystem(a["pos"], a["tangent"], a["chain_id"], a["rest_lengths"], s["L"], a["spring"], a["wca"],
                           a["active"], Dk, a["Dr"], a["radius"], a["n_nearby"], s["n_grid"],
                           calc_springs=a["longest"] > 1, srk_order=srk_order,
                           rigid_rod=(rigid[k] if rigid is not None else 0.0))
        o.seed = int(seeds[k]) if seeds is not None else 0
        systems.append(o)
    return O.OracleGroup(systems, s["fixed"], d["cross_wca"])
