"""The community ordering run before partitioning (cola_community_order: the
reference's Rabbit Order step, rabbit_order_write.py:48-55, written from the
published method): a permutation, deterministic, robust to isolated vertices,
self-loops and duplicates, and it puts connected vertices near each other --
on planted-partition graphs with shuffled ids, about three times as many edges
join vertices at most one community size apart as in the input order."""
import numpy as np
import pytest

import cola_b200 as cb
from cola_b200 import ColaError


def planted(seed, k=8, sz=400, m_in=20000, m_out=1500):
    rng = np.random.default_rng(seed)
    n = k * sz
    comm = np.repeat(np.arange(k), sz)
    a = rng.integers(0, n, m_in * 3)
    b = rng.integers(0, n, m_in * 3)
    keep = (comm[a] == comm[b]) & (a != b)
    a, b = a[keep][:m_in], b[keep][:m_in]
    c = rng.integers(0, n, m_out)
    d = rng.integers(0, n, m_out)
    perm = rng.permutation(n)
    r = perm[np.concatenate([a, c])]
    s = perm[np.concatenate([b, d])]
    return n, np.concatenate([r, s]).astype(np.int32), np.concatenate([s, r]).astype(np.int32), sz


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_planted_communities_placed_together(seed):
    n, row, col, sz = planted(seed)
    mp, nc = cb.community_order(n, row, col)
    assert np.array_equal(np.sort(mp), np.arange(n))
    near_new = np.mean(np.abs(mp[row].astype(np.int64) - mp[col]) <= sz)
    near_in = np.mean(np.abs(row.astype(np.int64) - col) <= sz)
    assert near_new >= 2.5 * near_in and near_new > 0.6
    assert 1 <= nc < n // 10
    again, nc2 = cb.community_order(n, row, col)
    assert np.array_equal(again, mp) and nc2 == nc  # deterministic


def test_edge_cases():
    mp, nc = cb.community_order(0, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert len(mp) == 0 and nc == 0
    # no edges: every vertex its own community, ids kept
    mp, nc = cb.community_order(5, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert np.array_equal(mp, np.arange(5)) and nc == 5
    # self-loops only, duplicates, one directed entry per edge
    mp, nc = cb.community_order(4, np.array([0, 1, 1, 2], np.int32), np.array([0, 1, 2, 1], np.int32))
    assert np.array_equal(np.sort(mp), np.arange(4))
    assert abs(int(mp[1]) - int(mp[2])) == 1  # the one edge's endpoints adjacent
    with pytest.raises(ColaError):
        cb.community_order(3, np.array([0, 3], np.int32), np.array([1, 1], np.int32))


def test_rmat_ordering_is_a_permutation():
    n, row, col, _ = cb.rmat(12, 16, seed=4)
    mp, nc = cb.community_order(n, row, col)
    assert np.array_equal(np.sort(mp), np.arange(n)) and nc >= 1
    r2, c2 = cb.relabel_edges(n, row, col, mp)
    assert np.array_equal(np.sort(r2), np.sort(mp[row]))
