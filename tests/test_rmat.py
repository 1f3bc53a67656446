"""The synthetic R-MAT inputs: the library's generator (cola_rmat_generate)
and the oracle's C restatement give the same graph, entry for entry and bit
for bit in the values, so a benchmark leg that must not load the product can
build the identical workload from the oracle."""
import numpy as np
import pytest

import cola_b200 as cb
from oracle import oracle


@pytest.mark.parametrize("scale,deg,seed,self_loops,values", [
    (1, 1, 0, False, 0),
    (6, 3.5, 9, False, 1),
    (10, 8, 1, False, 0),
    (12, 16, 1, True, 1),
    (14, 16, 1, True, 1),   # the CPU-runnable configuration: self-loops, 1/deg(row)
    (13, 32, 2, False, 2),  # D^-1/2 A D^-1/2
])
def test_oracle_rmat_matches_library(scale, deg, seed, self_loops, values):
    a = cb.rmat(scale, deg, seed, self_loops=self_loops, values=values)
    b = oracle.rmat(scale, deg, seed, self_loops=self_loops, values=values)
    assert a[0] == b[0] == 1 << scale
    for x, y in zip(a[1:], b[1:]):
        assert x.dtype == y.dtype and np.array_equal(x, y)
    n, row, col, val = b
    # sorted by (row, col), no duplicates, symmetric, self-loops only on request
    key = row.astype(np.int64) * n + col
    assert np.all(np.diff(key) > 0)
    assert np.array_equal(np.sort(col.astype(np.int64) * n + row), key)
    assert bool(np.any(row == col)) == (self_loops and len(row) > 0)
