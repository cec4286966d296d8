"""Host logic of the bench: how the split-context arm cuts a workload's
systems into contexts (no GPU)."""
import numpy as np
import pytest

import bench


@pytest.mark.parametrize("k", [1, 2, 3, 4, 8])
def test_split_by_beads_is_contiguous_nonempty_and_balanced(k):
    rs = np.random.default_rng(3)
    sizes = [int(x) for x in np.exp(rs.uniform(np.log(250), np.log(160000), size=256))]
    cuts = bench.split_by_beads(sizes, k)
    assert cuts[0] == 0 and cuts[-1] == len(sizes) and len(cuts) == k + 1
    assert all(a < b for a, b in zip(cuts[:-1], cuts[1:]))
    parts = [sum(sizes[a:b]) for a, b in zip(cuts[:-1], cuts[1:])]
    # each run is within one system of an even share
    assert max(parts) - sum(sizes) / k <= max(sizes)


def test_split_by_beads_with_few_systems():
    assert bench.split_by_beads([5, 7], 4) == [0, 1, 2]
    assert bench.split_by_beads([100, 1, 1, 1], 2) == [0, 1, 4]
    assert bench.split_by_beads([3], 3) == [0, 1]
