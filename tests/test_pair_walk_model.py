"""The index arithmetic of the warp-wide list walk (``warp_list_pair_force``
in ``csrc/gcr_step.cu``), restated lane by lane in Python: for any list
counts of a warp's 32 beads, every bead gets each of its list entries
exactly once and adds them in ascending slot order -- first the rows walked
one lane per bead, then its flattened tail, round by round -- so the sums are
those of a one-bead walk.  No GPU."""
import numpy as np
import pytest

CHUNK, ROW_BUSY, LIST_DEPTH = 2, 16, 256


def walk_order(counts, chunk=CHUNK, row_busy=ROW_BUSY, list_depth=LIST_DEPTH):
    """The (bead, slot) pairs in the order each bead adds them, as the kernel
    computes them: a list per lane."""
    cnt = [min(max(int(c), 0), list_depth) for c in counts]
    q_round = 32 * chunk
    added = [[] for _ in range(32)]
    # walked rows: only when the warp's pairs fill more than one round
    rows = 0
    if sum(cnt) > q_round:
        while rows < list_depth and sum(c > rows for c in cnt) >= row_busy:
            rows += 1
    for lane in range(32):
        for k in range(min(cnt[lane], rows)):
            added[lane].append(k)
    # the tails, flattened: an inclusive warp scan of the remaining counts
    rem = [c - rows if c > rows else 0 for c in cnt]
    incl = list(np.cumsum(rem))
    excl = [i - r for i, r in zip(incl, rem)]
    total = incl[31]
    for base in range(0, total, q_round):
        buf = {}
        for c in range(chunk):
            for lane in range(32):
                q = base + 32 * c + lane
                # binary search: the last lane whose prefix is <= q
                lo = 0
                for step in (16, 8, 4, 2, 1):
                    if excl[lo + step] <= q:
                        lo += step
                if q < total:
                    k = q - excl[lo]
                    assert 0 <= k < rem[lo], (q, lo, k)
                    buf[q - base] = (lo, rows + k)
        # each owner adds its pairs of this round in ascending q
        for lane in range(32):
            q0, q1 = max(excl[lane], base), min(incl[lane], base + q_round)
            for q in range(q0, q1):
                owner, slot = buf[q - base]
                assert owner == lane
                added[lane].append(slot)
    return added


def _check(counts):
    added = walk_order(counts)
    for lane, c in enumerate(counts):
        assert added[lane] == list(range(min(max(c, 0), LIST_DEPTH))), lane


@pytest.mark.parametrize("seed", range(40))
def test_random_counts_add_every_entry_once_in_order(seed):
    rs = np.random.default_rng(seed)
    mean = rs.choice([0.5, 2.0, 6.0, 13.0, 30.0])
    _check([int(x) for x in rs.poisson(mean, size=32)])


@pytest.mark.parametrize("counts", [
    [0] * 32,                                  # no pairs at all
    [1] * 32,                                  # exactly one round
    [2] * 32 + [],                             # 64 pairs: one round, no walked row
    [3] * 32,                                  # more than a round: walked rows
    [0] * 31 + [LIST_DEPTH],                   # one full list, the rest empty
    [LIST_DEPTH] * 32,                         # every list full
    [LIST_DEPTH + 5, -3] + [7] * 30,           # counts clamped to [0, list_depth]
    list(range(32)),                           # a staircase
    [16] * 16 + [0] * 16,                      # half the warp busy: rows walked
    [15] * 15 + [40] * 17,                     # just above the busy threshold
])
def test_edge_counts(counts):
    _check(counts)
