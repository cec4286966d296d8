"""The cell-staged pair kernel (``pair_mode = 2``) on the GPU.

It sums the same pairs as the list kernel (``pair_mode = 0``) in another
order (cell by cell instead of ascending partner id), so in FP64 the two
agree to rounding: positions within 1e-12 of the box after one step and
1e-9 after twenty, on sweep systems, the 2D LJ physics of the 500k-bead
system, the 3D LJ physics with rotational diffusion, and a dense strip in an
otherwise empty box whose row tiles hold more beads than a CTA stages (the
kernel then reads the same cells from global memory).  Its summation order
does not depend on the tile, grid or graph shape: launch shapes change no
bit.  The mixed path stays within FP32 rounding of the list kernel's.
"""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from tests.golden_io import min_image  # noqa: E402


def _strip(n_chains=800, L=400.0, height=100.0, seed=3):
    """LJ chains (config-2 physics) with heads in a strip of `height` across
    a box of side L: the strip's cells are four times denser than the box's
    mean, which sets the row tiles' width."""
    base = W.config2(seed=seed, scale=n_chains / 20000)
    rs = np.random.RandomState(seed)
    heads = np.stack([rs.uniform(0, L, n_chains), rs.uniform(0, height, n_chains)], axis=1)
    ang = rs.uniform(0, 2 * np.pi, n_chains)
    t = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    m = base.chain_id.size // n_chains
    j = np.arange(m, dtype=np.float64)
    pos = np.mod((heads[:, None, :] - 0.5 * j[None, :, None] * t[:, None, :]).reshape(-1, 2), L)
    params = dataclasses.replace(base.params, L=L)
    return dataclasses.replace(base, name="strip", pos=pos, tangent=np.repeat(t, m, axis=0), params=params)


CASES = {
    "sweep": lambda: sorted(W.config3(n_systems=64, param_seed=7), key=lambda s: s.n)[:4],
    "lj2d": lambda: [W.config2(seed=1, scale=0.01)],
    "lj3d": lambda: [W.config5(seed=2, scale=0.005)],
    "strip": lambda: [_strip()],
}


def _relaxed(specs):
    b = Batch(specs, precision="fp64", cell_depth=64, list_depth=256)
    b.relax(max_steps=600, adaptive_after=True)
    out = [dataclasses.replace(sp, pos=st.pos.cpu().numpy(), tangent=st.tangent.cpu().numpy())
           for sp, st in zip(specs, b.states)]
    b.close()
    return out


def _run(specs, precision, steps, **kw):
    # lists and cells deep enough for the LJ clusters (no regrow inside the comparison)
    b = Batch([dataclasses.replace(s, params=dataclasses.replace(s.params)) for s in specs],
              precision=precision, cell_depth=64, list_depth=256, **kw)
    b.set_adaptive(True)
    b.begin(steps)
    b.run(steps)
    st = b.statuses()
    assert all(s["flags"] == 0 and s["steps_done"] == steps for s in st), st
    pos = [x.pos.cpu().numpy().copy() for x in b.states]
    frc = [x.forces.double().cpu().numpy().copy() for x in b.states]
    dts = [s["dt"] for s in st]
    b.close()
    return pos, frc, dts


@pytest.mark.parametrize("case", sorted(CASES))
def test_cell_kernel_matches_list_kernel_fp64(case):
    specs = _relaxed(CASES[case]())
    for steps, tol in ((1, 1e-12), (20, 1e-9)):
        p0, f0, d0 = _run(specs, "fp64", steps, pair_mode=0)
        p2, f2, d2 = _run(specs, "fp64", steps, pair_mode=2)
        for sp, a, b in zip(specs, p0, p2):
            err = np.max(np.abs(min_image(a - b, sp.params.L))) / sp.params.L
            assert err < tol, (case, sp.name, steps, err)
        if steps == 1:
            for a, b in zip(f0, f2):
                scale = max(1.0, float(np.max(np.abs(a))))
                assert np.max(np.abs(a - b)) / scale < 1e-12
            np.testing.assert_allclose(d2, d0, rtol=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cell_kernel_is_independent_of_the_launch_shape(precision):
    specs = _relaxed(CASES["sweep"]() + [_strip(n_chains=200, L=200.0, height=50.0)])
    ref = _run(specs, precision, 30, pair_mode=2, block_beads=128, ctas_per_sm=0, steps_per_graph=10)
    for kw in (dict(block_beads=64, ctas_per_sm=2, steps_per_graph=5),
               dict(block_beads=256, ctas_per_sm=1, steps_per_graph=20)):
        out = _run(specs, precision, 30, pair_mode=2, **kw)
        for a, b in zip(ref[0], out[0]):
            np.testing.assert_array_equal(a, b)
        assert out[2] == ref[2]


def test_cell_kernel_mixed_within_fp32_rounding_of_the_list_kernel():
    specs = _relaxed(CASES["lj2d"]() + CASES["sweep"]())
    p0, f0, _ = _run(specs, "mixed", 1, pair_mode=0)
    p2, f2, _ = _run(specs, "mixed", 1, pair_mode=2)
    for sp, a, b, fa, fb in zip(specs, p0, p2, f0, f2):
        assert np.max(np.abs(min_image(a - b, sp.params.L))) / sp.params.L < 1e-9
        rel = np.linalg.norm(fa - fb) / np.linalg.norm(fa)
        assert rel < 1e-5, (sp.name, rel)
