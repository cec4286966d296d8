"""Periodic image counters on the GPU: the unwrapped positions the device
keeps (pos + L * images crossed in the real updates) against the host's
unwrapping of the same trajectory by minimum-image steps."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from gliding_collective_rotation_b200.batch import Batch  # noqa: E402
from gliding_collective_rotation_b200.workloads import config3  # noqa: E402
from tests.golden_io import min_image  # noqa: E402


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_unwrapping_matches_host_unwrapping(precision):
    specs = sorted(config3(n_systems=64, param_seed=11), key=lambda s: s.n)[:3]
    b = Batch(specs, precision=precision)
    b.set_adaptive(True)
    ref = [u.clone() for u in b.unwrapped()]
    host = [st.pos.cpu().numpy().copy() for st in b.states]
    prev = [h.copy() for h in host]
    crossed = 0
    for _ in range(60):
        b.begin(10)
        b.run(10)
        for i, st in enumerate(b.states):
            cur = st.pos.cpu().numpy()
            host[i] += min_image(cur - prev[i], specs[i].params.L)
            prev[i] = cur.copy()
    assert all(s["flags"] == 0 for s in b.statuses())
    for i, (u, h) in enumerate(zip(b.unwrapped(), host)):
        u = u.cpu().numpy()
        L = specs[i].params.L
        crossed += int(np.sum(np.abs(u - b.states[i].pos.cpu().numpy()) > 0.5 * L))
        assert np.max(np.abs(u - h)) < 1e-9 * L
    assert crossed > 0  # some beads left the box and came in from the other side
    msd = b.msd(ref)
    for i, h in enumerate(host):
        r = ref[i].cpu().numpy()
        assert msd[i] == pytest.approx(np.mean(np.sum((h - r) ** 2, axis=1)), rel=1e-9)
    b.close()


def test_images_survive_a_regrow():
    specs = sorted(config3(n_systems=64, param_seed=12), key=lambda s: s.n)[:2]
    b = Batch(specs, precision="fp64")
    b.set_adaptive(True)
    for _ in range(30):
        b.begin(20)
        b.run(20)
    before = [u.cpu().numpy() for u in b.unwrapped()]
    b.regrow()
    after = [u.cpu().numpy() for u in b.unwrapped()]
    for x, y in zip(before, after):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-10)
    b.close()
