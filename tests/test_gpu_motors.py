"""Motors on the GPU (``gcr_set_motors``): chains pushed by a motor
population (Motor_Population, populations.py:617-661; forces.calc_motor_push,
forces.py:248-283; the motors' diffusion, SRK.py:389-395) against the
oracle's group step, which restates the reference's bead-by-bead loop and is
itself pinned to the reference's ``calc_motor_push``
(``tests/test_motor_oracle.py``).

Both sides draw the keyed Philox numbers, so in FP64 every decision must be
the same: where_active of the chains and of the motors equal element by
element, positions of chains and motors within 1e-12 of the box after one
step and 1e-10 after five, dt within 1e-12.  Run with and without
b_motors_dont_diffuse_while_pushing (an attached motor keeps its position
and, after the predictor, its previous pos1).
"""
import dataclasses

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import workloads as W  # noqa: E402
from gliding_collective_rotation_b200._lib import GcrError  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden_io import min_image  # noqa: E402


def _box(hold=True, seed=0, k_on=0.9, k_off=0.2):
    return W.motors(n_boxes=1, seed=seed, n_chains=60, chain_length=8, L=24.0, motor_density=0.6, k_on=k_on,
                    k_off=k_off, hold=hold)


def _batch(specs, groups, mots, precision="fp64"):
    b = Batch(specs, precision=precision, cell_depth=32, list_depth=128)
    for g in groups:
        b.couple(*g)
    for m in mots:
        b.set_motors(*m)
    return b


def _oracle(b, specs, groups, mots):
    """The oracle group at the batch's current state (pos1 of the motors
    included: an attached motor's pos1 carries over)."""
    systems = []
    for st, sp in zip(b.states, specs):
        p = sp.params
        o = O.OracleSystem(st.pos.cpu().numpy(), st.tangent.double().cpu().numpy(), sp.chain_id, sp.rest_lengths,
                           p.L, p.spring_params, p.wca_params, p.active_params, p.D, p.Dr, p.radius, p.n_nearby, 4,
                           calc_springs=p.calc_springs, calc_wca=p.calc_wca and p.wca_params[0] != 0.0,
                           self_propel=p.self_propel)
        o.pos1[:] = st.pos1.cpu().numpy()
        o.seed = int(p.seed)
        systems.append(o)
    members, fixed, cross = groups[0]
    motor, chains, prm, hold = mots[0]
    r_list = float(cross[motor][chains][3])
    return O.OracleGroup(systems, fixed, cross, motors=dict(motor_pop=motor, chain_pop=chains, params=prm,
                                                            dont_diffuse=hold, list_r2=r_list * r_list))


@pytest.mark.parametrize("hold", [True, False])
def test_motors_match_the_oracle(hold):
    specs, groups, mots = _box(hold=hold)
    b = _batch(specs, groups, mots)
    b.relax(max_steps=400, adaptive_after=True)
    sts = b.statuses()
    assert not any(s["flags"] for s in sts)
    g = _oracle(b, specs, groups, mots)
    dt, step0 = sts[0]["dt"], sts[0]["step"]
    chains = specs[0]
    L = chains.params.L
    attached = pushed = 0
    for n_steps, tol in ((1, 1e-12), (4, 1e-10)):
        b.begin(n_steps)
        b.run(n_steps)
        sts = b.statuses()
        assert all(s["flags"] == 0 and s["steps_done"] == n_steps for s in sts), sts
        res = g.run(n_steps, dt=dt, dtmax=chains.params.dtmax, max_dist_per_step=chains.relax_mdps,
                    noise_mode=O.NOISE_PHILOX, step0=step0)
        assert res["steps"] == n_steps
        assert abs(sts[0]["dt"] - res["dt"]) <= 1e-12 * res["dt"], (sts[0]["dt"], res["dt"])
        dt, step0 = res["dt"], step0 + n_steps
        for k in range(2):
            np.testing.assert_array_equal(b.where_active(k), g.where_active[k], err_msg=f"where_active of {k}")
            err = np.max(np.abs(min_image(b.states[k].pos.cpu().numpy() - g.systems[k].pos, L))) / L
            assert err < tol, (k, n_steps, err)
        attached += int((g.where_active[1] >= 0).sum())
        pushed += int((g.where_active[0] >= 0).sum())
    b.close()
    # the comparison exercised attachments and pushes
    assert attached > 0 and pushed > 0


def test_attached_motors_hold_their_position():
    specs, groups, mots = _box(hold=True, k_on=1.0, k_off=0.0)
    b = _batch(specs, groups, mots)
    b.relax(max_steps=200, adaptive_after=True)
    before = b.states[1].pos.cpu().numpy().copy()
    b.begin(1)
    b.run(1)
    wa = b.where_active(1)
    after = b.states[1].pos.cpu().numpy()
    held = wa >= 0
    assert held.sum() > 0 and (~held).sum() > 0
    np.testing.assert_array_equal(after[held], before[held])
    assert np.all(np.any(after[~held] != before[~held], axis=1))
    b.close()


def test_mixed_precision_motors_run_and_push():
    specs, groups, mots = _box(seed=3)
    b = _batch(specs, groups, mots, precision="mixed")
    b.relax(max_steps=400, adaptive_after=True)
    b.begin(200)
    b.run(200)
    sts = b.statuses()
    assert all(s["flags"] == 0 and s["steps_done"] == 200 for s in sts), sts
    wa = b.where_active(1)
    assert 0 < (wa >= 0).sum() < len(wa)
    b.close()


def test_set_motors_refuses_what_it_cannot_step():
    specs, groups, mots = _box()
    b = Batch(specs, precision="fp64", srk_order=4)
    with pytest.raises(GcrError):
        b.engine.set_motors(b.states[1].slot, b.states[0].slot, mots[0][2])
    b.close()
    b = Batch(specs, precision="fp64")
    # chains are no motor population (springs, several beads per chain)
    with pytest.raises(GcrError):
        b.engine.set_motors(b.states[0].slot, b.states[1].slot, mots[0][2])
    with pytest.raises(GcrError):
        b.engine.where_active(b.states[0].slot)
    b.close()


def _fake_pops(specs, mots):
    """The reference's population objects as the drop-in reads them: the
    chains (Chain_Collection with motor_push toward the motors,
    populations.py:276-287) and a Motor_Population."""
    from types import SimpleNamespace
    from tests.gpu_helpers import pop_from_arrays
    ch, mo = specs
    p = ch.params
    chains = pop_from_arrays(ch.pos.copy(), ch.tangent.copy(), ch.chain_id, ch.rest_lengths, p.spring_params,
                             p.wca_params, p.active_params, p.D, p.Dr, p.radius, p.n_nearby)
    chains.name = "chains"
    chains.where_active = np.zeros(ch.n, dtype=np.int64)
    prm = mots[0][2]
    motors = SimpleNamespace(
        name="motors", total_pop=mo.n, pos=mo.pos.copy(), pos1=np.zeros_like(mo.pos), D=mo.params.D, Dr=0.0,
        fixed=False, motor_max_dist_sq=float(prm[0]), b_motors_dont_diffuse_while_pushing=bool(mots[0][3]),
        special_interactions={}, b_init_growing=False, n_nearby_beads_dont_repel=0,
        where_active=np.zeros(mo.n, dtype=np.int64), interactions=lambda other: [],
        self_interactions=lambda: [["diffuse", np.array([1.0])]])
    chains.interactions = lambda other: [["motor_push", prm]] if other is motors else []
    return chains, motors


def test_drop_in_steps_chains_and_motors_as_the_batch_does(monkeypatch):
    """updates.SRK2_force_calc over [chains, motors] (seeds sim['seed'] + k)
    equals the Batch path with the same systems bit for bit, and writes
    where_active back into both populations."""
    from types import SimpleNamespace
    from gliding_collective_rotation_b200 import config, updates
    specs, groups, mots = _box()
    ch = specs[0]
    L = ch.params.L
    for k, v in dict(dim=2, Lx=L, SRK_order=2, max_dist_per_step=ch.relax_mdps, RK_cheat_factor=1.0,
                     n_steps_update_grid_list=40, grid_factor=2.0, n_grid=int(L / 2.0)).items():
        monkeypatch.setattr(config, k, v)
    monkeypatch.setattr(updates, "_config", config)
    chains, motors = _fake_pops(specs, mots)
    # the batch's depths: no regrow inside the call (a regrow repeats the
    # interrupted step, whose predictor may have moved a motor's pos1)
    chains._gcr_cell_depth, chains._gcr_list_depth = 32, 128
    status = SimpleNamespace(dt=ch.dt, dtmax=ch.dt, stepnum=0, t=0.0, next_output_step=20, next_save_time=1e9,
                             update_grid_list_counter=1, b_calc_active_forces=True, max_forces_strength=0.0)
    sim = dict(seed=0, gpu_precision="fp64", save_state_every=-1)
    updates.SRK2_force_calc([chains, motors], status, sim)
    assert status.stepnum == 20
    b = _batch(specs, groups, mots)
    b.set_adaptive(True)
    b.begin(20, dt=ch.dt)
    b.run(20)
    np.testing.assert_array_equal(chains.pos, b.states[0].pos.cpu().numpy())
    np.testing.assert_array_equal(motors.pos, b.states[1].pos.cpu().numpy())
    np.testing.assert_array_equal(chains.where_active, b.where_active(0))
    np.testing.assert_array_equal(motors.where_active, b.where_active(1))
    assert (motors.where_active >= 0).any()
    b.close()
