"""The product's host preprocessing (cola_b200.prep, native) against the
reference's golden vectors and the oracle.  CPU only."""
import os

import numpy as np
import pytest

import cola_b200 as cb
from oracle import oracle
from conftest import GOLDEN_CASES, load_golden

NAMES = ["csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l", "csc_colPtr_r", "csc_rowIdx_r", "csc_colIdx_r"]


def test_row_partition_bit_exact(golden):
    name, fx = golden
    n = int(fx["num_nodes"])
    for P in fx["nparts_list"]:
        ps = cb.PartitionSet.from_coo(n, fx["row"], fx["col"], None, int(P))
        for r in range(P):
            got = ps.part(r)
            for nm in NAMES:
                want = fx["P{}_r{}_{}".format(P, r, nm)]
                assert got[nm].dtype == np.int32
                np.testing.assert_array_equal(got[nm], want, err_msg="{} P={} r={} {}".format(name, P, r, nm))


def test_global_csr_bit_exact(golden):
    _, fx = golden
    rp, ci, _ = cb.global_csr(int(fx["num_nodes"]), fx["row"], fx["col"])
    np.testing.assert_array_equal(rp, fx["global_rowPtr"])
    np.testing.assert_array_equal(ci, fx["global_colIdx"])


def test_nnz_split_bit_exact(golden):
    _, fx = golden
    for P in fx["nparts_list"]:
        for r in range(P):
            pre = "P{}_r{}_".format(P, r)
            t, p = cb.nnz_split(fx[pre + "csr_rowIdx_l"], fx[pre + "csr_rowPtr_l"], len(fx[pre + "csr_colIdx_l"]))
            np.testing.assert_array_equal(t, fx[pre + "lsplit_target"])
            np.testing.assert_array_equal(p, fx[pre + "lsplit_ptr"])
            t, p = cb.nnz_split(fx[pre + "csc_colIdx_r"], fx[pre + "csc_colPtr_r"], len(fx[pre + "csc_rowIdx_r"]))
            np.testing.assert_array_equal(t, fx[pre + "rsplit_target"])
            np.testing.assert_array_equal(p, fx[pre + "rsplit_ptr"])


def test_workgroup_cols_bit_exact(golden):
    _, fx = golden
    n = int(fx["num_nodes"])
    for P in fx["nparts_list"]:
        key = "P{}_gs_list".format(P)
        if key not in fx:
            continue
        for gs in fx[key]:
            for s in range(P // gs):
                got = cb.workgroup_cols(n, fx["row"], fx["col"], int(P), int(gs), s)
                np.testing.assert_array_equal(got, fx["P{}_gs{}_wg{}".format(P, gs, s)])


def test_stage_tables_match_oracle(golden):
    _, fx = golden
    n = int(fx["num_nodes"])
    checked = 0
    for P in fx["nparts_list"]:
        key = "P{}_gs_list".format(P)
        gss = [int(P)] + ([int(g) for g in fx[key]] if key in fx else [])
        for gs in gss:
            wg = [fx["P{}_gs{}_wg{}".format(P, gs, s)] for s in range(P // gs)] if gs < P else []
            for me in range(P):
                pre = "P{}_r{}_".format(P, me)
                zr = fx[pre + "rsplit_target"]
                nl = len(fx[pre + "lsplit_target"])
                got = cb.stage_tables(me, int(P), gs, n, zr, nl, wg)
                want = oracle.stage_tables(me, int(P), gs, n, zr, nl, wg)
                for k in ("local_offset", "remote_offset", "put_offset"):
                    np.testing.assert_array_equal(got[k], want[k])
                for a, b in zip(got["idx_ppl"], want["idx_ppl"]):
                    np.testing.assert_array_equal(a, b)
                for a, b in zip(got["put_colIdx"], want["put_colIdx"]):
                    np.testing.assert_array_equal(a, b)
                checked += 1
    assert checked > 0


def test_stage_tables_known_answer():
    """Hand-worked case: N=8, P=4 (npp=2), group_size=2 -> 2 stages.
    Rows 0-1 (PE0) reference cols {1, 4, 5, 6}; rows 2-3 (PE1) cols {0, 7}.
    Work group 0 = PEs 0,1 -> cols {0,1,4,5,6,7}; work group 1 = PEs 2,3."""
    row = np.array([0, 0, 1, 1, 2, 3, 4, 5, 6, 7], np.int32)
    col = np.array([1, 4, 5, 6, 0, 7, 4, 2, 1, 3], np.int32)
    n, P, gs = 8, 4, 2
    ps = cb.PartitionSet.from_coo(n, row, col, None, P)
    wg = [cb.workgroup_cols(n, row, col, P, gs, s) for s in range(2)]
    np.testing.assert_array_equal(wg[0], [0, 1, 4, 5, 6, 7])
    np.testing.assert_array_equal(wg[1], [1, 2, 3, 4])
    p0 = ps.part(0)
    # PE0 remote columns 4,5,6 (global ids), one chunk each
    zr, _ = cb.nnz_split(p0["csc_colIdx_r"], p0["csc_colPtr_r"], len(p0["csc_rowIdx_r"]))
    np.testing.assert_array_equal(zr, [4, 5, 6])
    t = cb.stage_tables(0, P, gs, n, zr, 1, wg)
    # stage 0: my group's cols [0, 4) -> no remote chunk; stage 1: PE2's range
    # [4, 6) is the partner (local_offset [0,2)), group range [4, 8) -> chunks [0, 3)
    np.testing.assert_array_equal(t["local_offset"], [0, 1, 0, 2])
    np.testing.assert_array_equal(t["remote_offset"], [0, 0, 0, 3])
    # positions of 4, 5 in wg0 restricted to PE2 ([4, 6) -> [4, 5]) and of 6 in PE3's part ([6, 8) -> [6, 7])
    np.testing.assert_array_equal(t["idx_ppl"][0], [0, 1, 0])
    # PE0 sends to target (0 - 2) mod 4 = PE2, whose work group 1 needs cols
    # {1,2,3,4} -> the ones PE0 owns ([0, 2)) = [1]
    np.testing.assert_array_equal(t["put_offset"][:2], [0, 1])
    np.testing.assert_array_equal(t["put_colIdx"][0], [1])


def test_values_match_oracle():
    n, row, col, val = cb.rmat(10, 8, seed=3)
    for P in (1, 3, 4):
        ps = cb.PartitionSet.from_coo(n, row, col, val, P)
        for r in range(P):
            got = ps.part(r)
            want = oracle.row_partition(n, row, col, P, r, val)
            for k in ("csr_val_l", "csc_val_r", "csr_colIdx_l", "csc_rowIdx_r"):
                np.testing.assert_array_equal(got[k], want[k])


def test_duplicate_values_sum_in_input_order():
    row = np.array([0, 0, 1, 0, 0], np.int32)
    col = np.array([3, 1, 2, 3, 3], np.int32)
    val = np.array([1.0, 2.0, 3.0, 0.5, 0.25], np.float32)
    ps = cb.PartitionSet.from_coo(4, row, col, val, 2)
    p = ps.part(0)
    np.testing.assert_array_equal(p["csc_colIdx_r"], [2, 3])
    np.testing.assert_array_equal(p["csc_val_r"], [3.0, np.float32(np.float32(1.0) + np.float32(0.5)) + np.float32(0.25)])


def test_bin_round_trip(tmp_path):
    name = GOLDEN_CASES[-1]
    fx = load_golden(name)
    n = int(fx["num_nodes"])
    P = int(fx["nparts_list"][0])
    ps = cb.PartitionSet.from_coo(n, fx["row"], fx["col"], None, P)
    d = str(tmp_path / name)
    ps.write_bin(d)
    # the files are the reference's own: compare against its golden arrays
    for r in range(P):
        for nm in NAMES:
            a = np.fromfile(os.path.join(d, "GPU{}".format(P), "{}_{}_{}.bin".format(nm, P, r)), dtype=np.int32)
            np.testing.assert_array_equal(a, fx["P{}_r{}_{}".format(P, r, nm)])
            np.testing.assert_array_equal(cb.bin2vec(os.path.join(d, "GPU{}".format(P),
                                                                   "{}_{}_{}.bin".format(nm, P, r))), a)
    back = cb.PartitionSet.read_bin(d, n, P)
    for r in range(P):
        a, b = ps.part(r), back.part(r)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])


def test_read_bin_without_values_defaults_to_ones(tmp_path):
    fx = load_golden("uniform1000")
    n = int(fx["num_nodes"])
    d = tmp_path / "g"
    (d / "GPU2").mkdir(parents=True)
    for r in range(2):
        for nm in NAMES:
            fx["P2_r{}_{}".format(r, nm)].tofile(str(d / "GPU2" / "{}_2_{}.bin".format(nm, r)))
    ps = cb.PartitionSet.read_bin(str(d), n, 2)
    p = ps.part(1)
    assert np.all(p["csr_val_l"] == 1.0) and np.all(p["csc_val_r"] == 1.0)
    np.testing.assert_array_equal(p["csc_colIdx_r"], fx["P2_r1_csc_colIdx_r"])


def test_read_bin_rejects_corrupt_indices(tmp_path):
    fx = load_golden("uniform1000")
    n = int(fx["num_nodes"])
    d = tmp_path / "g"
    (d / "GPU2").mkdir(parents=True)
    for r in range(2):
        for nm in NAMES:
            a = fx["P2_r{}_{}".format(r, nm)].copy()
            if r == 1 and nm == "csc_rowIdx_r":
                a[3] = 10 ** 6
            a.tofile(str(d / "GPU2" / "{}_2_{}.bin".format(nm, r)))
    with pytest.raises(cb.ColaError):
        cb.PartitionSet.read_bin(str(d), n, 2)


def test_bad_coo_rejected():
    with pytest.raises(cb.ColaError):
        cb.PartitionSet.from_coo(4, np.array([0, 5], np.int32), np.array([1, 1], np.int32), None, 2)
    with pytest.raises(cb.ColaError):
        cb.PartitionSet.from_coo(4, np.array([0], np.int32), np.array([-1], np.int32), None, 2)


def test_empty_graph_and_more_parts_than_rows():
    ps = cb.PartitionSet.from_coo(3, np.zeros(0, np.int32), np.zeros(0, np.int32), None, 5)
    for r in range(5):
        p = ps.part(r)
        assert len(p["csr_rowPtr_l"]) == 1 and len(p["csc_colPtr_r"]) == 1
        assert len(p["csr_colIdx_l"]) == 0 and len(p["csc_colIdx_r"]) == 0


def test_nnz_split_empty_rows_list():
    t, p = cb.nnz_split(np.zeros(0, np.int32), np.array([0], np.int32), 0)
    assert len(t) == 0 and len(p) == 0


def test_rmat_properties():
    n, row, col, val = cb.rmat(12, 16, seed=11)
    n2, row2, col2, val2 = cb.rmat(12, 16, seed=11)
    np.testing.assert_array_equal(row, row2)
    np.testing.assert_array_equal(col, col2)
    np.testing.assert_array_equal(val, val2)
    assert n == 4096
    assert np.all(row != col)
    key = row.astype(np.int64) * n + col
    assert np.all(np.diff(key) > 0)  # sorted, unique
    tkey = np.sort(col.astype(np.int64) * n + row)
    np.testing.assert_array_equal(key, tkey)  # symmetric
    deg = np.bincount(row, minlength=n).astype(np.float64)
    np.testing.assert_allclose(val, 1.0 / np.sqrt(deg[row] * deg[col]), rtol=1e-6)
    assert 0.6 * 16 * n < len(row) <= 16 * n
    assert deg.max() > 20 * deg.mean()  # power-law hub
    _, r3, c3, v3 = cb.rmat(10, 8, seed=2, self_loops=True, values=cb.prep.VALUES_ROW_NORMALISED)
    d3 = np.bincount(r3, minlength=1024)
    assert np.all(np.isin(np.arange(1024), r3[r3 == c3]))
    np.testing.assert_allclose(v3, 1.0 / d3[r3], rtol=1e-6)


def test_relabel_edges_matches_oracle():
    n, row, col, _ = cb.rmat(10, 8, seed=5)
    mapping = np.random.Generator(np.random.Philox(5)).permutation(n).astype(np.int32)
    r, c = cb.relabel_edges(n, row, col, mapping)
    wr, wc = oracle.relabel_edges(row, col, mapping)
    np.testing.assert_array_equal(r, wr)
    np.testing.assert_array_equal(c, wc)


def test_relabel_edges_rejects_bad_ids():
    row = np.array([0, 1], np.int32)
    col = np.array([1, 4], np.int32)
    with pytest.raises(cb.ColaError):
        cb.relabel_edges(4, row, col, np.arange(4, dtype=np.int32))  # col 4 outside
    with pytest.raises(cb.ColaError):
        cb.relabel_edges(4, row, col[:1].repeat(2), np.array([0, 9, 1, 2], np.int32))  # maps to 9
