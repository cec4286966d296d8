"""The autotuner on the GPU: it measures, caches, and its shapes leave the
trajectory unchanged bit for bit."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200 import autotune  # noqa: E402
from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.workloads import config3  # noqa: E402

SMALL_SPACE = {"block_beads": (64, 128), "ctas_per_sm": (0, 2), "steps_per_graph": (5, 10),
               "skin_scale": (1.0, 1.5)}


def _specs(n=6):
    return sorted(config3(n_systems=64, param_seed=7), key=lambda s: s.n)[:n]


def test_tune_measures_and_caches(tmp_path, monkeypatch):
    cache = str(tmp_path / "tune.json")
    res = autotune.tune(_specs(), precision="mixed", steps=10, warmup=3, space=SMALL_SPACE, cache=cache)
    for k, vals in SMALL_SPACE.items():
        assert res[k] in vals
    assert np.isfinite(res["ms_per_step"]) and res["ms_per_step"] > 0
    assert min(t["ms_per_step"] for t in res["trials"]) == res["ms_per_step"]

    def refuse(*a, **k):
        raise AssertionError("a cached workload is not measured again")
    monkeypatch.setattr(autotune, "measure_shape", refuse)
    again = autotune.tune(_specs(), precision="mixed", steps=10, warmup=3, space=SMALL_SPACE, cache=cache)
    assert again == res


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_shape_gives_the_same_trajectory(precision):
    """Tile size, persistent grid, graph length, skin and whether the stage
    kernels sum the pair forces themselves change no bit of a trajectory."""
    specs = _specs(4)
    out = []
    for res in ({"block_beads": 128, "ctas_per_sm": 0, "steps_per_graph": 10, "skin_scale": 1.0, "pair_mode": 0},
                {"block_beads": 64, "ctas_per_sm": 2, "steps_per_graph": 5, "skin_scale": 1.5, "pair_mode": 1},
                {"block_beads": 256, "ctas_per_sm": 4, "steps_per_graph": 20, "skin_scale": 0.67, "pair_mode": 0},
                {"block_beads": 128, "ctas_per_sm": 0, "steps_per_graph": 10, "skin_scale": 1.0, "pair_mode": 1}):
        sp, kw = autotune.apply(specs, res)
        b = Batch(sp, precision=precision, **kw)
        b.set_adaptive(True)
        b.begin(60)
        b.run(60)
        st = b.statuses()
        assert all(s["flags"] == 0 and s["steps_done"] == 60 for s in st)
        out.append((np.concatenate([x.pos.cpu().numpy() for x in b.states]), [s["dt"] for s in st]))
        b.close()
    for pos, dts in out[1:]:
        np.testing.assert_array_equal(pos, out[0][0])
        assert dts == out[0][1]
