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


def test_context_parts_keep_coupled_boxes_whole():
    # 8 boxes of two populations each: chains then passive beads
    sizes = [10000 + 500 * b if p == 0 else 3000 for b in range(8) for p in range(2)]
    groups = [([2 * b, 2 * b + 1], [False, False], None) for b in range(8)]
    parts = bench.context_parts(sizes, 4, groups)
    assert len(parts) == 4
    assert sorted(i for p in parts for i in p) == list(range(16))
    for p in parts:
        assert all((i ^ 1) in p for i in p)  # a box's populations together
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes) + 3000
    # without couplings: the contiguous bead split
    assert bench.context_parts([5, 7, 9], 2) == [[0, 1], [2]]
