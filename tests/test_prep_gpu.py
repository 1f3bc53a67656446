"""Preprocessing on the device (cola_partition_build_device,
cola_nnz_split_device, cola_relabel_edges_device) against the reference's
golden vectors, the oracle and the host build: every array bit for bit."""
import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200 import spmm as S
from oracle import oracle

from gpu_util import TOL_F32, dense_x, fp64_reference, rel

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
NAMES = ["csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l", "csc_colPtr_r", "csc_rowIdx_r", "csc_colIdx_r"]
VALS = ["csr_val_l", "csc_val_r"]


def dev(a, dtype=torch.int32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).to(DEV)


def build_device(n, row, col, val, P):
    return cb.PartitionSet.from_coo_device(n, dev(row), dev(col), None if val is None else dev(val, torch.float32),
                                           P)


def assert_same_sets(got, want, P, what):
    for r in range(P):
        g, w = got.part(r), want.part(r)
        for nm in NAMES:
            np.testing.assert_array_equal(g[nm], w[nm], err_msg="{} r={} {}".format(what, r, nm))
        for nm in VALS:  # bit for bit
            np.testing.assert_array_equal(g[nm].view(np.uint32), w[nm].view(np.uint32),
                                          err_msg="{} r={} {}".format(what, r, nm))


def test_device_partition_matches_golden(golden):
    name, fx = golden
    n = int(fx["num_nodes"])
    for P in fx["nparts_list"]:
        ps = build_device(n, fx["row"], fx["col"], None, int(P))
        for r in range(P):
            got = ps.part(r)
            for nm in NAMES:
                np.testing.assert_array_equal(got[nm], fx["P{}_r{}_{}".format(P, r, nm)],
                                              err_msg="{} P={} r={} {}".format(name, P, r, nm))
        # values (duplicates merged into sums of ones) as the host build has them
        assert_same_sets(ps, cb.PartitionSet.from_coo(n, fx["row"], fx["col"], None, int(P)), P, name)


def with_duplicates(n, row, col, val, seed):
    """Append shuffled duplicate entries with their own values."""
    g = np.random.Generator(np.random.Philox(seed))
    pick = g.integers(0, len(row), len(row) // 5)
    row = np.concatenate([row, row[pick]])
    col = np.concatenate([col, col[pick]])
    val = np.concatenate([val, g.standard_normal(len(pick)).astype(np.float32)])
    perm = g.permutation(len(row))
    return row[perm].astype(np.int32), col[perm].astype(np.int32), val[perm]


@pytest.mark.parametrize("scale,deg,P", [(10, 8, 1), (10, 8, 3), (11, 12, 4), (12, 16, 8), (9, 4, 16)])
def test_device_partition_with_values_matches_oracle(scale, deg, P):
    n, row, col, val = cb.rmat(scale, deg, seed=scale * 10 + P)
    keep = n - 37  # N not a multiple of P
    m = (row < keep) & (col < keep)
    row, col, val = with_duplicates(keep, row[m], col[m], val[m], seed=P)
    ps = build_device(keep, row, col, val, P)
    assert_same_sets(ps, cb.PartitionSet.from_coo(keep, row, col, val, P), P, "host")
    for r in range(P):
        got, want = ps.part(r), oracle.row_partition(keep, row, col, P, r, val)
        for nm in NAMES:
            np.testing.assert_array_equal(got[nm], want[nm])
        for nm in VALS:
            np.testing.assert_array_equal(got[nm].view(np.uint32), want[nm].view(np.uint32))


def test_device_partition_large_matches_host():
    # 8.4 M entries (six radix passes), hub rows and columns
    n, row, col, val = cb.rmat(18, 32, seed=7)
    ps = build_device(n, row, col, val, 8)
    assert_same_sets(ps, cb.PartitionSet.from_coo(n, row, col, val, 8), 8, "scale 18")


def test_device_partition_edge_cases():
    # no entries
    ps = build_device(10, np.zeros(0, np.int32), np.zeros(0, np.int32), None, 3)
    assert_same_sets(ps, cb.PartitionSet.from_coo(10, np.zeros(0, np.int32), np.zeros(0, np.int32), None, 3), 3,
                     "empty")
    # more partitions than rows, one node, all entries in one partition
    for n, row, col, P in [(3, [0, 2, 1, 2], [2, 0, 1, 2], 5), (1, [0, 0], [0, 0], 2), (64, [5] * 7, [9, 1, 9, 60, 5, 9, 1], 4)]:
        row = np.array(row, np.int32)
        col = np.array(col, np.int32)
        val = np.linspace(0.5, 3.0, len(row)).astype(np.float32)
        assert_same_sets(build_device(n, row, col, val, P), cb.PartitionSet.from_coo(n, row, col, val, P), P,
                         "n={} P={}".format(n, P))


def test_device_partition_rejects_bad_coo():
    row = np.array([0, 1, 2], np.int32)
    col = np.array([1, 5, 0], np.int32)
    with pytest.raises(cb.ColaError, match="entry 1"):
        build_device(4, row, col, None, 2)
    with pytest.raises(cb.ColaError):
        build_device(4, np.array([-1], np.int32), np.array([0], np.int32), None, 2)
    # the context stays usable
    ps = build_device(4, row, np.array([1, 3, 0], np.int32), None, 2)
    assert ps.part(0)["csr_rowPtr_l"].tolist() == [0, 1] and ps.part(0)["csc_colIdx_r"].tolist() == [3]


def test_nnz_split_device_matches_golden(golden):
    _, fx = golden
    for P in fx["nparts_list"]:
        for r in range(P):
            pre = "P{}_r{}_".format(P, r)
            for ids, ptr, ent, sp in (("csr_rowIdx_l", "csr_rowPtr_l", "csr_colIdx_l", "lsplit"),
                                      ("csc_colIdx_r", "csc_colPtr_r", "csc_rowIdx_r", "rsplit")):
                t, p = cb.nnz_split_device(dev(fx[pre + ids]), dev(fx[pre + ptr]), len(fx[pre + ent]))
                np.testing.assert_array_equal(t.cpu().numpy(), fx[pre + sp + "_target"])
                np.testing.assert_array_equal(p.cpu().numpy(), fx[pre + sp + "_ptr"])


def test_nnz_split_device_hub_rows():
    n, row, col, val = cb.rmat(16, 24, seed=11)
    ps = cb.PartitionSet.from_coo(n, row, col, val, 4)
    for r in range(4):
        p = ps.part(r)
        for ids, ptr, ent in (("csr_rowIdx_l", "csr_rowPtr_l", "csr_colIdx_l"),
                              ("csc_colIdx_r", "csc_colPtr_r", "csc_rowIdx_r")):
            wt, wp = oracle.nnz_split(p[ids], p[ptr], len(p[ent]))
            t, q = cb.nnz_split_device(dev(p[ids]), dev(p[ptr]), len(p[ent]))
            np.testing.assert_array_equal(t.cpu().numpy(), wt)
            np.testing.assert_array_equal(q.cpu().numpy(), wp)


def test_relabel_device_matches_oracle_and_rejects_bad_ids():
    n, row, col, _ = cb.rmat(12, 8, seed=3)
    mapping = np.random.Generator(np.random.Philox(3)).permutation(n).astype(np.int32)
    r, c = cb.relabel_edges(n, dev(row), dev(col), dev(mapping))
    wr, wc = oracle.relabel_edges(row, col, mapping)
    np.testing.assert_array_equal(r.cpu().numpy(), wr)
    np.testing.assert_array_equal(c.cpu().numpy(), wc)
    bad = mapping.copy()
    bad[int(row[0])] = n
    with pytest.raises(cb.ColaError):
        cb.relabel_edges(n, dev(row), dev(col), dev(bad))


def test_relabelled_graph_spmm_is_the_permuted_product():
    # A' = Q A Q^T for the relabelling Q: Y'[mapping[v]] = (A X)[v] when
    # X'[mapping[v]] = X[v]: reorder, partition and multiply all on the device
    n, row, col, val = cb.rmat(13, 16, seed=9)
    mapping = np.random.Generator(np.random.Philox(9)).permutation(n).astype(np.int32)
    r2, c2 = cb.relabel_edges(n, dev(row), dev(col), dev(mapping))
    ps = cb.PartitionSet.from_coo_device(n, r2, c2, dev(val, torch.float32), 8)
    X = dense_x(n, 64, seed=9)
    Xp = np.empty_like(X)
    Xp[mapping] = X
    Yp = S.Graph(ps).spmm(torch.from_numpy(Xp).to(DEV)).cpu().numpy()
    ref = fp64_reference(n, row, col, val, X)
    assert rel(Yp[mapping], ref) <= TOL_F32


# ---------------------------------------------------------------------------
# the whole graph built on the device (row view, hub segments, tasks)
# ---------------------------------------------------------------------------
def device_graph(n, row, col, val, P, **kw):
    return S.Graph.from_coo_device(n, dev(row), dev(col), None if val is None else dev(val, torch.float32), P, **kw)


@pytest.mark.parametrize("scale,deg,P,thr,seg,te", [(12, 16, 4, 0, 0, 0), (11, 8, 3, 8, 4, 64), (13, 24, 8, 32, 16, 300),
                                                    (10, 4, 1, 10 ** 6, 256, 1), (12, 16, 16, 1, 1, 0)])
def test_device_graph_equals_uploaded_graph(scale, deg, P, thr, seg, te):
    """Same statistics as the host upload of the same COO's partitions, and
    bit-identical SpMM results for every width (narrow widths interleave
    entries over lane groups relative to each task's start, so equal bits
    mean equal tasks and hub segments too)."""
    n, row, col, val = cb.rmat(scale, deg, seed=scale + P)
    keep = n - 5
    m = (row < keep) & (col < keep)
    row, col, val = with_duplicates(keep, row[m], col[m], val[m], seed=P)
    kw = dict(hub_threshold=thr, hub_segment=seg, task_entries=te)
    gd = device_graph(keep, row, col, val, P, **kw)
    gh = S.Graph(cb.PartitionSet.from_coo(keep, row, col, val, P), **kw)
    di, hi = gd.info, gh.info
    for k in ("num_nodes", "nparts", "nodes_per_part", "nnz", "nnz_local", "nnz_remote", "hub_rows", "hub_segments",
              "row_tasks"):
        assert getattr(di, k) == getattr(hi, k), k
    for K, xdt, ydt in [(8, torch.float32, torch.float32), (16, torch.float32, torch.float32),
                        (64, torch.float32, torch.float32), (128, torch.float32, torch.float32),
                        (256, torch.bfloat16, torch.bfloat16), (32, torch.bfloat16, torch.float32)]:
        X = torch.from_numpy(dense_x(keep, K, seed=K)).to(DEV).to(xdt)
        yd = gd.spmm(X, out_dtype=ydt)
        yh = gh.spmm(X, out_dtype=ydt, schedule=S.SCHEDULE_ROWS)
        torch.cuda.synchronize()
        assert torch.equal(yd, yh), (K, xdt, ydt)
    ref = fp64_reference(keep, row, col, val, dense_x(keep, 64, seed=64))
    y = gd.spmm(torch.from_numpy(dense_x(keep, 64, seed=64)).to(DEV))
    assert rel(y.cpu().numpy(), ref) <= TOL_F32


def test_device_graph_is_rows_only_and_edge_cases():
    n, row, col, val = cb.rmat(10, 8, seed=1)
    g = device_graph(n, row, col, val, 4)
    X = torch.ones((n, 16), device=DEV)
    for sched in (S.SCHEDULE_FUSED, S.SCHEDULE_BUFFER):
        with pytest.raises(cb.ColaError, match="row-major"):
            g.spmm(X, schedule=sched)
    with pytest.raises(cb.ColaError):
        g.zip_view(0)
    # no entries: Y is all zeros; rows of a one-node graph
    e = torch.zeros(0, dtype=torch.int32, device=DEV)
    g0 = S.Graph.from_coo_device(50, e, e, None, 3)
    assert g0.info.nnz == 0 and g0.info.row_tasks > 0
    y0 = g0.spmm(torch.ones((50, 32), device=DEV))
    g1 = device_graph(1, np.array([0, 0], np.int32), np.array([0, 0], np.int32), np.array([0.5, 2.0], np.float32), 2)
    y1 = g1.spmm(torch.full((1, 8), 3.0, device=DEV))
    torch.cuda.synchronize()
    assert torch.all(y0 == 0) and torch.all(y1 == 7.5)
    with pytest.raises(cb.ColaError, match="entry 1"):
        device_graph(4, np.array([0, 4], np.int32), np.array([1, 1], np.int32), None, 2)


try:
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    @st.composite
    def small_coo(draw):
        n = draw(st.integers(1, 60))
        nnz = draw(st.integers(0, 300))
        row = np.array(draw(st.lists(st.integers(0, n - 1), min_size=nnz, max_size=nnz)), np.int32)
        col = np.array(draw(st.lists(st.integers(0, n - 1), min_size=nnz, max_size=nnz)), np.int32)
        val = np.array(draw(st.lists(st.floats(-4, 4, width=32), min_size=nnz, max_size=nnz)), np.float32)
        P = draw(st.integers(1, 9))
        thr = draw(st.sampled_from([0, 1, 3, 8]))
        seg = draw(st.sampled_from([0, 1, 2, 5]))
        te = draw(st.sampled_from([0, 1, 4, 16]))
        return n, row, col, val, P, thr, seg, te

    @settings(max_examples=60, deadline=None, suppress_health_check=[HealthCheck.too_slow])
    @given(small_coo())
    def test_device_builds_match_host_on_random_coo(case):
        n, row, col, val, P, thr, seg, te = case
        assert_same_sets(build_device(n, row, col, val, P), cb.PartitionSet.from_coo(n, row, col, val, P), P,
                         "random")
        kw = dict(hub_threshold=thr, hub_segment=seg, task_entries=te)
        gd = device_graph(n, row, col, val, P, **kw)
        gh = S.Graph(cb.PartitionSet.from_coo(n, row, col, val, P), **kw)
        for k in ("nnz", "nnz_local", "hub_rows", "hub_segments", "row_tasks"):
            assert getattr(gd.info, k) == getattr(gh.info, k), k
        for K in (4, 64):
            X = torch.from_numpy(dense_x(n, K, seed=K)).to(DEV)
            a = gd.spmm(X)
            b = gh.spmm(X, schedule=S.SCHEDULE_ROWS)
            torch.cuda.synchronize()
            assert torch.equal(a, b)
except ImportError:  # hypothesis is optional for the GPU run
    pass
