"""Property tests (hypothesis) of the host preprocessing against the oracle on
random small COO inputs: duplicates, empty rows and columns, values, any
number of partitions (more partitions than rows included).  CPU only."""
import numpy as np
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import cola_b200 as cb
from oracle import oracle

NAMES = ["csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l", "csc_colPtr_r", "csc_rowIdx_r", "csc_colIdx_r"]


@st.composite
def coo(draw):
    n = draw(st.integers(1, 40))
    nnz = draw(st.integers(0, 160))
    row = np.array(draw(st.lists(st.integers(0, n - 1), min_size=nnz, max_size=nnz)), np.int32)
    col = np.array(draw(st.lists(st.integers(0, n - 1), min_size=nnz, max_size=nnz)), np.int32)
    val = np.array(draw(st.lists(st.floats(-4, 4, width=32), min_size=nnz, max_size=nnz)), np.float32)
    P = draw(st.integers(1, 12))
    return n, row, col, val, P


@settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(coo())
def test_partition_matches_oracle(case):
    n, row, col, val, P = case
    ps = cb.PartitionSet.from_coo(n, row, col, val, P)
    for r in range(P):
        got, want = ps.part(r), oracle.row_partition(n, row, col, P, r, val)
        for nm in NAMES:
            np.testing.assert_array_equal(got[nm], want[nm], err_msg=nm)
        for nm in ("csr_val_l", "csc_val_r"):
            np.testing.assert_array_equal(got[nm].view(np.uint32), want[nm].view(np.uint32), err_msg=nm)
        # structural facts of prep_torch_par.py:24-79
        assert got["csr_rowPtr_l"][0] == 0 and got["csc_colPtr_r"][0] == 0
        assert len(got["csr_rowPtr_l"]) == len(got["csr_rowIdx_l"]) + 1
        assert len(got["csc_colPtr_r"]) == len(got["csc_colIdx_r"]) + 1
        assert np.all(np.diff(got["csr_rowPtr_l"]) > 0) and np.all(np.diff(got["csc_colPtr_r"]) > 0)
        assert np.all(np.diff(got["csr_rowIdx_l"]) > 0) and np.all(np.diff(got["csc_colIdx_r"]) > 0)


@settings(max_examples=150, deadline=None)
@given(coo())
def test_nnz_split_matches_oracle(case):
    n, row, col, val, P = case
    ps = cb.PartitionSet.from_coo(n, row, col, val, P)
    for r in range(P):
        p = ps.part(r)
        for ids, ptr, ent in (("csr_rowIdx_l", "csr_rowPtr_l", "csr_colIdx_l"),
                              ("csc_colIdx_r", "csc_colPtr_r", "csc_rowIdx_r")):
            t, q = cb.nnz_split(p[ids], p[ptr], len(p[ent]))
            wt, wq = oracle.nnz_split(p[ids], p[ptr], len(p[ent]))
            np.testing.assert_array_equal(t, wt)
            np.testing.assert_array_equal(q, wq)
            if len(t):  # chunks tile every row's entries in order
                assert q[0] == 0 and q[-1] == len(p[ent]) and np.all(np.diff(q) > 0)


@settings(max_examples=100, deadline=None)
@given(coo(), st.randoms(use_true_random=False))
def test_relabel_is_a_permutation_of_the_product(case, rnd):
    n, row, col, val, P = case
    mapping = np.arange(n, dtype=np.int32)
    rnd.shuffle(mapping)
    r2, c2 = cb.relabel_edges(n, row, col, mapping)
    wr, wc = oracle.relabel_edges(row, col, mapping)
    np.testing.assert_array_equal(r2, wr)
    np.testing.assert_array_equal(c2, wc)
    # the relabelled graph's product is the permuted product (FP64 oracle)
    X = np.random.Generator(np.random.Philox(n)).standard_normal((n, 3), dtype=np.float32)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    Y = oracle.spmm_csr_f64(rp, ci, vv, X)
    rp2, ci2, vv2 = oracle.global_csr(n, r2, c2, val)
    Xp = np.empty_like(X)
    Xp[mapping] = X
    Y2 = oracle.spmm_csr_f64(rp2, ci2, vv2, Xp)
    np.testing.assert_allclose(Y2[mapping], Y, rtol=1e-5, atol=1e-4)
