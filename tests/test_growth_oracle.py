"""The init-grow protocol on the oracle against the reference's own growth.

The reference grew config 1 (200 chains x 10 beads in a 60 x 60 box) from
its random placement before recording ``tests/golden/config1.npz``: the
placement is ``init_pos``, the grown state ``pos0``.  The schedule of
``gliding_collective_rotation_b200.growth`` stepped by the oracle must grow
the same placement into a state with the reference's statistics."""
from tests.grow_helpers import check_like_reference, config1_growth_case, grown_stats, oracle_grow


def test_oracle_growth_matches_reference_statistics():
    d, s, base, consts, settings = config1_growth_case()
    sysm, steps, t = oracle_grow(d, s, base, consts, settings)
    ref = grown_stats(d["pos0"], d["chain_id"], s["L"])
    got = grown_stats(sysm.pos, d["chain_id"], s["L"])
    check_like_reference(got, ref, steps, s["init_grow_steps"], t)
