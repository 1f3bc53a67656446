"""The oracle's restatements against the golden vectors the reference's own
preprocessing wrote (tests/golden/make_golden.py)."""
import numpy as np

from oracle import oracle

NAMES = ["csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l", "csc_colPtr_r", "csc_rowIdx_r", "csc_colIdx_r"]


def test_row_partition_matches_reference(golden):
    name, fx = golden
    n = int(fx["num_nodes"])
    for P in fx["nparts_list"]:
        for r in range(P):
            got = oracle.row_partition(n, fx["row"], fx["col"], int(P), r)
            for nm in NAMES:
                want = fx["P{}_r{}_{}".format(P, r, nm)]
                assert want.dtype == np.int32
                np.testing.assert_array_equal(got[nm], want, err_msg="{} P={} r={} {}".format(name, P, r, nm))


def test_global_csr_matches_reference(golden):
    _, fx = golden
    rp, ci, _ = oracle.global_csr(int(fx["num_nodes"]), fx["row"], fx["col"])
    np.testing.assert_array_equal(rp, fx["global_rowPtr"])
    np.testing.assert_array_equal(ci, fx["global_colIdx"])


def test_nnz_split_matches_reference(golden):
    _, fx = golden
    for P in fx["nparts_list"]:
        for r in range(P):
            pre = "P{}_r{}_".format(P, r)
            t, p = oracle.nnz_split(fx[pre + "csr_rowIdx_l"], fx[pre + "csr_rowPtr_l"], len(fx[pre + "csr_colIdx_l"]))
            np.testing.assert_array_equal(t, fx[pre + "lsplit_target"])
            np.testing.assert_array_equal(p, fx[pre + "lsplit_ptr"])
            t, p = oracle.nnz_split(fx[pre + "csc_colIdx_r"], fx[pre + "csc_colPtr_r"], len(fx[pre + "csc_rowIdx_r"]))
            np.testing.assert_array_equal(t, fx[pre + "rsplit_target"])
            np.testing.assert_array_equal(p, fx[pre + "rsplit_ptr"])


def test_workgroup_cols_match_reference(golden):
    _, fx = golden
    n = int(fx["num_nodes"])
    seen = 0
    for P in fx["nparts_list"]:
        key = "P{}_gs_list".format(P)
        if key not in fx:
            continue
        for gs in fx[key]:
            for s in range(P // gs):
                want = fx["P{}_gs{}_wg{}".format(P, gs, s)]
                got = oracle.workgroup_cols(n, fx["row"], fx["col"], int(P), int(gs), s)
                np.testing.assert_array_equal(got, want)
                seen += 1
    assert seen > 0


def test_values_follow_index_order():
    """Values ride with their indices and merged duplicates sum in input order."""
    row = np.array([0, 0, 1, 0], np.int32)
    col = np.array([3, 1, 2, 3], np.int32)
    val = np.array([1.0, 2.0, 3.0, 0.5], np.float32)
    got = oracle.row_partition(4, row, col, 2, 0, val)
    np.testing.assert_array_equal(got["csr_colIdx_l"], [1])
    np.testing.assert_array_equal(got["csr_val_l"], [2.0])
    np.testing.assert_array_equal(got["csc_colIdx_r"], [2, 3])
    np.testing.assert_array_equal(got["csc_rowIdx_r"], [1, 0])
    np.testing.assert_array_equal(got["csc_val_r"], [3.0, 1.5])


def test_openmp_partition_loop_matches_fp64():
    """The OpenMP FP32 loop over the partitions (a reported CPU baseline)
    computes the product: within 1e-5 of the FP64 oracle."""
    import cola_b200 as cb
    n, row, col, val = cb.rmat(11, 12, seed=8)
    ps = cb.PartitionSet.from_coo(n, row, col, val, 5)
    X = np.random.Generator(np.random.Philox(8)).standard_normal((n, 24), dtype=np.float32)
    Y = oracle.partitions_f32_omp([ps.part(r) for r in range(5)], ps.nodes_per_part, X)(3)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    ref = oracle.spmm_csr_f64(rp, ci, vv, X)
    assert oracle.rel_frobenius(Y[:n], ref) <= 1e-5


def test_ordered_fp32_restatement_against_fp64():
    """orc_spmm_rows_f32_ordered (the row-major schedule's summation order,
    compared bit for bit with the GPU in test_zz_rows_order_gpu.py) computes the
    FP64 oracle's product to FP32 accuracy for every hub setting, and the same
    bits on every call."""
    import cola_b200 as cb
    n, row, col, val = cb.rmat(11, 16, seed=4)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    X = np.random.Generator(np.random.Philox(2)).standard_normal((n, 128), dtype=np.float32)
    ref = oracle.spmm_csr_f64(rp, ci, vv, X)
    for thr, seg in ((256, 256), (16, 8), (1, 1), (10 ** 6, 256)):
        Y = oracle.spmm_rows_f32_ordered(rp, ci, vv, X, thr, seg)
        assert np.linalg.norm(Y - ref) / np.linalg.norm(ref) < 1e-6
        assert np.array_equal(Y, oracle.spmm_rows_f32_ordered(rp, ci, vv, X, thr, seg))
