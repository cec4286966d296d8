"""``updates.install`` inside a real reference checkout, on the CPU.

The reference is copied to a scratch directory (its ``config.configure``
deletes ``__pycache__/*`` in the working directory), imported with the shims
its own test fixtures need (numpy's removed ``np.float``/``np.int`` aliases,
a stubbed matplotlib, ``populations`` first), and the drop-in is installed
into its modules.  Then:

* ``updates.SRK2_force_calc`` of the checkout is the GPU step, and the
  reference's driver ``control.sim_loop`` (control.py:84) reaches it: with
  no GPU in this process the step stops at the device boundary with
  ``GcrError`` ("no CUDA device") -- after it has read the reference's own
  population object (its ``self_interactions``, packed parameters and
  arrays) and the checkout's ``config`` globals; nothing falls back to the
  CPU;
* a pair rule other than ``forces.WCA`` in ``force_rules`` is refused with
  ``NotImplementedError`` before any device work.

Skipped where the reference or Numba is not present (the GPU boxes carry
neither); the GPU parity of the step itself is pinned by the fixtures the
reference wrote (``tests/test_gpu_parity.py``).
"""
import os
import subprocess
import sys
import textwrap

import pytest

REF = os.environ.get("GCR_REFERENCE_DIR", "/root/reference")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.skipif(not os.path.isdir(REF), reason="reference checkout not present")

SCRIPT = textwrap.dedent(r"""
    import os, shutil, sys, tempfile, types
    import numpy as np
    ref_src, root, mode = sys.argv[1], sys.argv[2], sys.argv[3]
    scratch = tempfile.mkdtemp(prefix="gcr_bind_")
    ref = os.path.join(scratch, "ref")
    shutil.copytree(ref_src, ref, ignore=shutil.ignore_patterns("Chiral_paper_plots", "Images", "Results"))
    for r, ds, fs in os.walk(ref):
        for d in ds:
            os.chmod(os.path.join(r, d), 0o755)
        for f in fs:
            os.chmod(os.path.join(r, f), 0o644)
    os.makedirs(os.path.join(ref, "Results"), exist_ok=True)
    np.float = float
    np.int = int

    class _Stub(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)
            return lambda *a, **k: None

    for m in ["matplotlib", "matplotlib.pyplot", "matplotlib.colors", "matplotlib.cm", "matplotlib.collections",
              "matplotlib.patches", "mpl_toolkits", "mpl_toolkits.mplot3d", "mpl_toolkits.mplot3d.art3d",
              "mpl_toolkits.axes_grid1", "mpl_toolkits.axes_grid1.inset_locator"]:
        sys.modules[m] = _Stub(m)
    os.chdir(ref)
    sys.path.insert(0, ref)
    import populations  # noqa: F401  (first: the reference's circular imports)
    import config, updates, forces, force_rules, defaults, control
    sys.path.insert(0, root)
    from gliding_collective_rotation_b200 import updates as gpu_updates
    from gliding_collective_rotation_b200._lib import GcrError

    assert gpu_updates.install(updates, config, force_rules, forces) is gpu_updates.SRK2_force_calc
    assert updates.SRK2_force_calc is gpu_updates.SRK2_force_calc
    assert control.updates is updates  # the driver looks the step up on this module

    sim, _ = defaults.set_defaults()
    sim.update(dict(Lx=20., n_chains=12, chain_length=6, a=0.5, k=100., kappa=20., repel_d_max=1.,
                    WCA_epsilon=1., LJ_cutoff_factor=1., v0=1., T=0.01, dim=2, seed=1, t_init_grow=0.,
                    a_init_factor=1., plot_every=-1, ticker_every=5, save_state_every=-1., t_max=0.01,
                    stepnum_max=5, n_threads=1, gpu=True))
    config.configure(sim)
    pops = [populations.Equal_Size_Chain_Collection(sim, name="beads")]
    status = config.status_class(sim)
    # what control.run_sim does before its loop: placement, grids, lists
    control.configure_start(sim, pops, status)
    if mode == "sim_loop":
        try:
            control.sim_loop(pops, sim, status)
        except GcrError as e:
            assert "no CUDA device" in str(e), e
            # the step read the reference's population and the checkout's config
            p = gpu_updates._pop_params(pops[0], status, sim, 0)
            assert p.L == config.Lx and p.max_dist_per_step == config.max_dist_per_step
            assert np.array_equal(p.wca_params, pops[0].WCA_params)
            assert np.array_equal(p.spring_params, pops[0].spring_params())
            print("REACHED_DEVICE_BOUNDARY")
        else:
            raise AssertionError("the installed step ran without a GPU")
    else:
        force_rules.central_pair_force_rule = forces.general_pair_force if hasattr(forces, "general_pair_force") \
            else (lambda *a: None)
        try:
            updates.SRK2_force_calc(pops, status, sim)
        except NotImplementedError as e:
            assert "forces.WCA" in str(e), e
            print("REFUSED_OTHER_RULE")
        else:
            raise AssertionError("another pair rule was accepted")
    shutil.rmtree(scratch, ignore_errors=True)
""")


def _run(mode):
    pytest.importorskip("numba")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")  # this process must not reach a GPU
    res = subprocess.run([sys.executable, "-c", SCRIPT, REF, ROOT, mode], capture_output=True, text=True,
                         timeout=600, env=env)
    assert res.returncode == 0, res.stdout[-3000:] + res.stderr[-3000:]
    return res.stdout


def test_install_rebinds_the_reference_step_and_sim_loop_reaches_it():
    assert "REACHED_DEVICE_BOUNDARY" in _run("sim_loop")


def test_install_refuses_another_pair_rule():
    assert "REFUSED_OTHER_RULE" in _run("rule")
