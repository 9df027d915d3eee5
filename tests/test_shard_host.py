"""Host logic of the sharded parse (alpacc_b200/shard.py), no GPU: the halo
terminals gathered across short and empty slices, the prefix of position
sums (depth, v, terminals and the last head restart after a head), and the
pairs the next non-empty slice closes."""

import numpy as np

from alpacc_b200 import shard

E = 99  # the empty terminal


def _edge(ids):
    """A slice's gathered edge record from its position terminals."""
    e = np.full(2 * shard.HALO, E, np.uint32)
    k = min(shard.HALO, len(ids))
    e[:k] = ids[:k]
    if k:
        e[2 * shard.HALO - k:] = ids[len(ids) - k:]
    return e, len(ids)


def test_halos_walk_past_short_and_empty_slices():
    slices = [list(range(100, 140)), [7], [], list(range(200, 203)), list(range(300, 330))]
    edges = [_edge(s) for s in slices]
    whole = [x for s in slices for x in s]
    starts = np.cumsum([0] + [len(s) for s in slices])
    for r in range(len(slices)):
        hl, hr = shard.halos(edges, r, E)
        a, b = starts[r], starts[r + 1]
        want_l = [whole[i] if i >= 0 else E for i in range(a - shard.HALO, a)]
        want_r = [whole[i] if i < len(whole) else E for i in range(b, b + shard.HALO)]
        assert hl.tolist() == want_l, r
        assert hr.tolist() == want_r, r


def test_prefix_restarts_after_a_head():
    # nodes, brackets, depth, v, terminals, heads, last head, closed pairs
    sums = [np.array([5, 4, 2, -1, 3, 1, 0, 1, 0, 0]), np.array([2, 2, -1, 1, 1, 0, -1, 0, 1, 0]),
            np.array([4, 0, 0, 0, 2, 0, -1, 0, 0, 0])]
    assert shard.prefix(sums, 0) == (0, 0, 0, 0, 0, 0, -1, 0)
    assert shard.prefix(sums, 1) == (5, 4, 2, -1, 3, 1, 0, 1)
    assert shard.prefix(sums, 2) == (7, 6, 1, 0, 4, 1, 0, 1)
    headed = [np.array([1, 0, 5, 5, 5, 0, -1, 0, 0, 0]), np.array([1, 0, 1, 2, 3, 1, 40, 0, 0, 0])]
    assert shard.prefix(headed, 2) == (2, 0, 1, 2, 3, 1, 40, 0)


def test_closed_next_skips_empty_slices():
    sums = [np.zeros(10, np.int64) for _ in range(4)]
    sums[1][8], sums[3][8] = 4, 2
    edges = [(None, 10), (None, 0), (None, 0), (None, 5)]
    assert shard.closed_next(sums, edges, 0) == 2
    edges[1] = (None, 3)
    assert shard.closed_next(sums, edges, 0) == 4
    assert shard.closed_next(sums, edges, 3) == 0
    edges[1] = (None, 0)
    assert shard.closed_next(sums, edges, 1) == 0  # an empty slice closes nothing
