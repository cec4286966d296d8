"""The init-grow protocol on the oracle against the reference's own growth.

The reference grew config 1 (200 chains x 10 beads in a 60 x 60 box) and a
3D system (60 chains x 10 beads in a box of 16, LJ attraction, rotational
diffusion) from their random placements before recording
``tests/golden/config1.npz`` and ``grow3d.npz``: the placement is
``init_pos``, the grown state ``pos0``.  The schedule of
``gliding_collective_rotation_b200.growth`` stepped by the oracle must grow
the same placement into a state with the reference's statistics."""
import pytest

from tests.grow_helpers import check_like_reference, growth_case, grown_stats, oracle_grow


@pytest.mark.parametrize("name", ["config1", "grow3d"])
def test_oracle_growth_matches_reference_statistics(name):
    d, s, base, consts, settings = growth_case(name)
    sysm, steps, t = oracle_grow(d, s, base, consts, settings)
    ref = grown_stats(d["pos0"], d["chain_id"], s["L"])
    got = grown_stats(sysm.pos, d["chain_id"], s["L"])
    check_like_reference(got, ref, steps, s["init_grow_steps"], t)
