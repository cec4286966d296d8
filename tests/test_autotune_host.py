"""The launch-shape search of the autotuner, on the host with a fake timer."""
import json
import math

from gliding_collective_rotation_b200 import autotune
from gliding_collective_rotation_b200.workloads import config3


def _fake(best):
    """ms per step: a bowl around `best`, one unit per step away in each parameter."""
    def measure(shape):
        d = 0.0
        for k, v in shape.items():
            vals = autotune.SPACE[k]
            d += abs(vals.index(v) - vals.index(best[k]))
        return 1.0 + d
    return measure


def test_search_finds_the_minimum_of_a_separable_cost():
    best = {"block_beads": 256, "ctas_per_sm": 4, "steps_per_graph": 20, "skin_scale": 0.67, "pair_mode": 1}
    shape, ms, trials = autotune.search(_fake(best))
    assert shape == best and ms == 1.0
    # coordinate descent: far fewer runs than the full grid
    full = math.prod(len(v) for v in autotune.SPACE.values())
    assert len(trials) < full / 4


def test_search_starts_from_the_defaults_and_keeps_them_when_best():
    shape, ms, trials = autotune.search(_fake(autotune.DEFAULT))
    assert shape == autotune.DEFAULT and ms == 1.0
    assert trials[0] == {**autotune.DEFAULT, "ms_per_step": 1.0}


def test_failed_shapes_are_never_chosen():
    def measure(shape):
        return math.inf if shape["block_beads"] == 256 else (2.0 if shape["block_beads"] == 128 else 1.5)
    shape, ms, _ = autotune.search(measure)
    assert shape["block_beads"] == 64 and ms == 1.5


def test_signature_separates_workloads():
    a = config3(n_systems=8, param_seed=1)
    b = config3(n_systems=16, param_seed=1)
    sa, sb = autotune.signature(a, "mixed"), autotune.signature(b, "mixed")
    assert sa != sb
    assert sa == autotune.signature(list(a), "mixed")
    assert autotune.signature(a, "mixed") != autotune.signature(a, "fp64")
    assert json.loads(sa)["systems"] == 8


def test_apply_scales_the_skin_and_keeps_the_physics():
    specs = config3(n_systems=3, param_seed=2)
    res = {"block_beads": 64, "ctas_per_sm": 2, "steps_per_graph": 5, "skin_scale": 1.5, "pair_mode": 1}
    out, kw = autotune.apply(specs, res)
    assert kw == {"block_beads": 64, "ctas_per_sm": 2, "steps_per_graph": 5, "pair_mode": 1}
    from gliding_collective_rotation_b200.engine import default_skin
    for s, o in zip(specs, out):
        assert o.params.skin == default_skin(s.params.wca_params[3]) * 1.5
        assert (o.pos is s.pos) and o.params.wca_params is s.params.wca_params
        assert s.params.skin is None  # the caller's specs are not changed
