"""GPU parity of the partitioned SpMM: every schedule and launcher against the
FP64 oracle, and the kernel-level drop-ins against the reference's own CUDA
kernels (oracle/_ref, compiled from the reference tree through the NVSHMEM
shim) on the same seeded inputs.  Tolerances: FP32 paths 1e-5 relative
Frobenius; BF16 storage 1e-2 against FP64 on the FP32 features."""
import ctypes

import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200 import spmm as S
from oracle import oracle

from gpu_util import TOL_BF16, TOL_F32, bf16_bits, dense_x, fp64_reference, graph_case, ptr, rel

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def case12():
    n, row, col, val, ps = graph_case(12, 16, seed=5, nparts=4)
    return n, row, col, val, ps


@pytest.mark.parametrize("K", [1, 3, 16, 32, 33, 64, 96, 100, 128, 256, 512])
def test_fused_fp32_matches_fp64(case12, K):
    n, row, col, val, ps = case12
    g = S.Graph(ps)
    X = dense_x(n, K, seed=K)
    ref = fp64_reference(n, row, col, val, X)
    Y = g.spmm(torch.from_numpy(X).to(DEV), schedule=S.SCHEDULE_FUSED)
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), ref) <= TOL_F32


@pytest.mark.parametrize("P", [1, 2, 3, 8, 16])
def test_partition_counts(P):
    n, row, col, val, ps = graph_case(11, 12, seed=P, nparts=P)
    g = S.Graph(ps)
    X = dense_x(n, 64, seed=1)
    ref = fp64_reference(n, row, col, val, X)
    Y = g.spmm(torch.from_numpy(X).to(DEV))
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), ref) <= TOL_F32


@pytest.mark.parametrize("if_split", [True, False])
@pytest.mark.parametrize("schedule,batch", [(S.SCHEDULE_FUSED, 0), (S.SCHEDULE_BUFFER, 0),
                                            (S.SCHEDULE_BUFFER, 64)])
def test_schedules_fp32(case12, if_split, schedule, batch):
    n, row, col, val, ps = case12
    g = S.Graph(ps, if_split=if_split)
    X = dense_x(n, 128, seed=2)
    ref = fp64_reference(n, row, col, val, X)
    Y = g.spmm(torch.from_numpy(X).to(DEV), schedule=schedule, gather_batch_rows=batch)
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), ref) <= TOL_F32


@pytest.mark.parametrize("P,gs", [(4, 1), (4, 2), (8, 2), (8, 4)])
@pytest.mark.parametrize("K", [32, 128])
def test_pipelined_schedule(P, gs, K):
    n, row, col, val, ps = graph_case(12, 16, seed=9, nparts=P)
    g = S.Graph(ps, group_size=gs)
    X = dense_x(n, K, seed=3)
    ref = fp64_reference(n, row, col, val, X)
    Y = g.spmm(torch.from_numpy(X).to(DEV), schedule=S.SCHEDULE_PIPELINE)
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), ref) <= TOL_F32


@pytest.mark.parametrize("K", [64, 256])
def test_bf16_storage(case12, K):
    n, row, col, val, ps = case12
    g = S.Graph(ps)
    X = dense_x(n, K, seed=4)
    Xb = bf16_bits(X)
    ref_f32x = fp64_reference(n, row, col, val, X)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    ref_bf16x = oracle.spmm_csr_f64(rp, ci, vv, Xb)
    xt = torch.from_numpy(Xb.view(np.int16)).view(torch.bfloat16).to(DEV)
    Y32 = g.spmm(xt, out_dtype=torch.float32)
    Y16 = g.spmm(xt, out_dtype=torch.bfloat16)
    torch.cuda.synchronize()
    y32 = Y32.cpu().numpy()
    y16 = Y16.float().cpu().numpy()
    # FP32 accumulation of exactly-widened BF16 features: FP32-level error
    assert rel(y32, ref_bf16x) <= TOL_F32
    # against FP64 on the FP32 features: BF16 storage error only
    assert rel(y32, ref_f32x) <= TOL_BF16
    assert rel(y16, ref_f32x) <= TOL_BF16
    # BF16 output is the FP32 result rounded once (the two runs may sum in a
    # different order, so compare to BF16 rounding, not bit for bit)
    assert rel(y16, y32) <= 2.0 ** -8


def test_accumulate_and_strides(case12):
    n, row, col, val, ps = case12
    g = S.Graph(ps)
    K = 64
    X = dense_x(n, K, seed=6)
    ref = fp64_reference(n, row, col, val, X)
    big = torch.zeros((n, 80), device=DEV)
    big[:, :K] = torch.from_numpy(X).to(DEV)
    xv = big[:, :K]  # ldx = 80
    Y = torch.zeros((n, 72), device=DEV)
    yv = Y[:, :K]  # ldy = 72
    g.spmm(xv, yv)
    g.spmm(xv, yv, accumulate=True)
    torch.cuda.synchronize()
    assert rel(yv.cpu().numpy(), 2 * ref) <= TOL_F32
    assert torch.all(Y[:, K:] == 0)


def test_pipeline_and_buffer_bf16(case12):
    n, row, col, val, _ = case12
    ps = cb.PartitionSet.from_coo(n, row, col, val, 4)
    g = S.Graph(ps, group_size=2)
    X = dense_x(n, 128, seed=8)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    Xb = bf16_bits(X)
    ref = oracle.spmm_csr_f64(rp, ci, vv, Xb)
    xt = torch.from_numpy(Xb.view(np.int16)).view(torch.bfloat16).to(DEV)
    for sch in (S.SCHEDULE_PIPELINE, S.SCHEDULE_BUFFER, S.SCHEDULE_FUSED):
        Y = g.spmm(xt, schedule=sch, gather_batch_rows=100)
        torch.cuda.synchronize()
        assert rel(Y.cpu().numpy(), ref) <= TOL_F32, sch


def test_golden_graphs_on_gpu():
    from conftest import GOLDEN_CASES, load_golden
    for name in GOLDEN_CASES:
        fx = load_golden(name)
        n = int(fx["num_nodes"])
        rng = np.random.Generator(np.random.Philox(17))
        val = rng.random(len(fx["row"]), dtype=np.float32)
        for P in fx["nparts_list"]:
            ps = cb.PartitionSet.from_coo(n, fx["row"], fx["col"], val, int(P))
            g = S.Graph(ps)
            X = dense_x(n, 32, seed=int(P))
            ref = fp64_reference(n, fx["row"], fx["col"], val, X)
            Y = g.spmm(torch.from_numpy(X).to(DEV))
            torch.cuda.synchronize()
            assert rel(Y.cpu().numpy(), ref) <= TOL_F32, (name, P)


def test_empty_graph():
    ps = cb.PartitionSet.from_coo(10, np.zeros(0, np.int32), np.zeros(0, np.int32), None, 4)
    g = S.Graph(ps)
    Y = g.spmm(torch.ones((10, 16), device=DEV))
    torch.cuda.synchronize()
    assert torch.all(Y == 0)


def test_bad_arguments_raise(case12):
    n, row, col, val, ps = case12
    g = S.Graph(ps)
    with pytest.raises(ValueError):
        g.spmm(torch.ones((n - 1, 16), device=DEV))
    with pytest.raises(cb.ColaError):
        g.spmm(torch.ones((n, 16), device=DEV), torch.empty((n, 16), dtype=torch.bfloat16, device=DEV),
               accumulate=True)
    with pytest.raises(cb.ColaError):
        g.spmm(torch.ones((n, 16), device=DEV), schedule=S.SCHEDULE_PIPELINE)
    with pytest.raises(cb.ColaError):
        S.Graph(ps, group_size=3)


# ---------------------------------------------------------------------------
# kernel-level drop-ins vs the reference's own kernels
# ---------------------------------------------------------------------------
def _padded_x(n, P, npp, K, seed):
    X = np.zeros((P * npp, K), np.float32)
    X[:n] = dense_x(n, K, seed)
    return X


def _run_dropin(fn, g, Xd, npp, K, P, buf=None):
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        args = [ptr(Y[p * npp:]), ptr(Xd[p * npp:])]
        if buf is not None:
            args.append(ptr(buf))
        args += [z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx,
                 z.csc_colIdx_zip, z.csc_val]
        args = [a if a is None or isinstance(a, ctypes.c_void_p) else ctypes.c_void_p(a) for a in args]
        fn(*args, 0, 0, z.local_chunks, z.remote_chunks, K, npp, p, None)
    torch.cuda.synchronize()
    return Y


def _run_reference(g, Xd, npp, K, P):
    R = oracle.ref()
    CF = (K + 31) // 32
    res = 1 if K & 31 else 0
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        assert R.ref_set_pe(p, npp * K, None) == 0
        rc = R.ref_ppl0_batch_spmm(CF, res, ptr(Y[p * npp:]), ptr(Xd[p * npp:]), z.csr_rowPtr, z.csr_colIdx,
                                   z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx, z.csc_colIdx_zip,
                                   z.csc_val, 0, 0, z.local_chunks, z.remote_chunks, K, npp, p, None)
        assert rc == 0
    torch.cuda.synchronize()
    return Y


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")


@needs_ref
@pytest.mark.parametrize("K", [16, 32, 64, 100, 128, 256])
def test_ppl0_dropin_matches_reference_kernels(K):
    P = 4
    n, row, col, val, ps = graph_case(12, 16, seed=21, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X = _padded_x(n, P, npp, K, seed=K)
    Xd = torch.from_numpy(X).to(DEV)
    ref64 = fp64_reference(n, row, col, val, X[:n])
    L = cb.lib()
    ours = _run_dropin(L.cola_ppl0_batch_spmm, g, Xd, npp, K, P)[:n].cpu().numpy()
    theirs = _run_reference(g, Xd, npp, K, P)[:n].cpu().numpy()
    assert rel(theirs, ref64) <= TOL_F32
    assert rel(ours, ref64) <= TOL_F32
    assert rel(ours, theirs) <= TOL_F32
    seq = _run_dropin(L.cola_ppl0_batch_spmm_seq, g, Xd, npp, K, P)[:n].cpu().numpy()
    assert rel(seq, theirs) <= TOL_F32
    nr = max(g.zip_view(p).remote_chunks for p in range(P))
    buf = torch.empty((max(nr, 1), K), device=DEV)
    bufd = _run_dropin(L.cola_ppl0_batch_buffer_spmm, g, Xd, npp, K, P, buf=buf)[:n].cpu().numpy()
    assert rel(bufd, theirs) <= TOL_F32


def _pipeline_tables(n, row, col, ps, P, gs):
    wg = [cb.workgroup_cols(n, row, col, P, gs, s) for s in range(P // gs)]
    tabs = []
    for me in range(P):
        p = ps.part(me)
        lt, lp = cb.nnz_split(p["csr_rowIdx_l"], p["csr_rowPtr_l"], len(p["csr_colIdx_l"]))
        rt, rp = cb.nnz_split(p["csc_colIdx_r"], p["csc_colPtr_r"], len(p["csc_rowIdx_r"]))
        tabs.append(oracle.stage_tables(me, P, gs, n, rt, len(lt), wg))
    return tabs


@needs_ref
@pytest.mark.parametrize("P,gs", [(4, 1), (4, 2), (8, 2)])
def test_pipelined_dropins_match_reference_kernels(P, gs):
    """The multi-stage schedule of include/dist_spmm_ppl_batch.cuh:785-836 run
    in lockstep over P virtual PEs, once with the reference's kernels and once
    with the drop-ins, on the oracle's stage tables."""
    K = 64
    n, row, col, val, ps = graph_case(12, 16, seed=31, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X = _padded_x(n, P, npp, K, seed=5)
    Xd = torch.from_numpy(X).to(DEV)
    ref64 = fp64_reference(n, row, col, val, X[:n])
    tabs = _pipeline_tables(n, row, col, ps, P, gs)
    nstages = P // gs
    R = oracle.ref()
    L = cb.lib()
    CF, res = (K + 31) // 32, 1 if K & 31 else 0
    results = {}
    for impl in ("ref", "ours"):
        Y = torch.zeros((P * npp, K), device=DEV)
        bufs = [torch.zeros((P * npp, K), device=DEV) for _ in range(2)]
        send = torch.zeros((P * npp, K), device=DEV)
        dev_idx = [[torch.from_numpy(t["idx_ppl"][i]).to(DEV) for i in range(nstages - 1)] for t in tabs]
        dev_put = [[torch.from_numpy(t["put_colIdx"][i]).to(DEV) for i in range(nstages - 1)] for t in tabs]
        # stage 0 for every PE (dist_spmm_ppl_batch.cuh:797-805)
        for me in range(P):
            z = g.zip_view(me)
            t = tabs[me]
            lo, ro = t["local_offset"], t["remote_offset"]
            args = (ptr(Y[me * npp:]), ptr(Xd[me * npp:]), z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val,
                    z.csc_colPtr, z.csc_rowIdx, z.csc_colIdx_zip, z.csc_val, int(lo[0]), int(ro[0]),
                    int(lo[1] - lo[0]), int(ro[1] - ro[0]), K, npp, me, None)
            if impl == "ref":
                assert R.ref_set_pe(me, npp * K, None) == 0
                assert R.ref_ppl0_batch_spmm(CF, res, *args) == 0
            else:
                cb._lib.check(L.cola_ppl0_batch_spmm(*args))
        for i in range(1, nstages):
            buf = bufs[(i - 1) % 2]
            # every PE's put for stage i (:788-793, :811-816)
            for me in range(P):
                t = tabs[me]
                target = ((me - i * gs) % P + P) % P
                nemb = int(t["put_offset"][2 * (i - 1) + 1] - t["put_offset"][2 * (i - 1)])
                if nemb == 0:
                    continue
                if impl == "ref":
                    assert R.ref_set_pe(me, npp * K, None) == 0
                    assert R.ref_batching_data_ppl(ptr(Xd[me * npp:]), ptr(send[me * npp:]), ptr(dev_put[me][i - 1]),
                                                   nemb, K, npp, gs, None) == 0
                else:
                    cb._lib.check(L.cola_batching_data_ppl(ptr(Xd[me * npp:]), ptr(send[me * npp:]),
                                                           ptr(dev_put[me][i - 1]), nemb, K, npp, gs, None))
                buf[target * npp: target * npp + nemb].copy_(send[me * npp: me * npp + nemb])
            # every PE's stage-i compute (:822-835)
            for me in range(P):
                z = g.zip_view(me)
                t = tabs[me]
                lo, ro = t["local_offset"], t["remote_offset"]
                if ro[2 * i + 1] - ro[2 * i] == 0:
                    continue
                args = (ptr(Y[me * npp:]), ptr(buf[me * npp:]), z.csc_colPtr, z.csc_rowIdx, z.csc_colIdx_zip,
                        z.csc_val, int(lo[2 * i]), int(lo[2 * i + 1]), int(ro[2 * i]), int(ro[2 * i + 1]), i,
                        ptr(dev_idx[me][i - 1]), K, npp, gs, me // gs * gs, me, None)
                if impl == "ref":
                    assert R.ref_set_pe(me, npp * K, None) == 0
                    assert R.ref_ppl_batch_spmm(CF, res, *args) == 0
                else:
                    cb._lib.check(L.cola_ppl_batch_spmm(*args))
        torch.cuda.synchronize()
        results[impl] = Y[:n].cpu().numpy()
    assert rel(results["ref"], ref64) <= TOL_F32  # pins the stage tables' meaning
    assert rel(results["ours"], ref64) <= TOL_F32
    assert rel(results["ours"], results["ref"]) <= TOL_F32


@needs_ref
def test_batching_data_ppl_matches_reference_bit_exact():
    K, npp, P = 96, 500, 4
    X = torch.from_numpy(dense_x(P * npp, K, seed=12)).to(DEV)
    rng = np.random.Generator(np.random.Philox(3))
    idx = torch.from_numpy(rng.integers(0, P * npp, 700).astype(np.int32)).to(DEV)
    a = torch.zeros((700, K), device=DEV)
    b = torch.zeros((700, K), device=DEV)
    R = oracle.ref()
    assert R.ref_set_pe(0, npp * K, None) == 0
    assert R.ref_batching_data_ppl(ptr(X), ptr(a), ptr(idx), 700, K, npp, 1, None) == 0
    cb._lib.check(cb.lib().cola_batching_data_ppl(ptr(X), ptr(b), ptr(idx), 700, K, npp, 1, None))
    torch.cuda.synchronize()
    assert torch.equal(a, b)


# ---------------------------------------------------------------------------
# row-major schedule (remote CSC transposed at upload; one writer per row)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("K", [1, 3, 16, 32, 33, 64, 96, 100, 128, 256, 512])
def test_rows_fp32_matches_fp64(case12, K):
    n, row, col, val, ps = case12
    g = S.Graph(ps)
    assert g.info.hub_rows > 0  # the R-MAT hubs exceed the default threshold
    X = dense_x(n, K, seed=100 + K)
    ref = fp64_reference(n, row, col, val, X)
    Y = g.spmm(torch.from_numpy(X).to(DEV), schedule=S.SCHEDULE_ROWS)
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), ref) <= TOL_F32


@pytest.mark.parametrize("thr,seg", [(0, 0), (8, 4), (1, 1), (40, 16), (10 ** 6, 256)])
def test_rows_hub_segments(case12, thr, seg):
    n, row, col, val, ps = case12
    g = S.Graph(ps, hub_threshold=thr, hub_segment=seg)
    X = dense_x(n, 64, seed=7)
    ref = fp64_reference(n, row, col, val, X)
    Y = g.spmm(torch.from_numpy(X).to(DEV), schedule=S.SCHEDULE_ROWS)
    Y2 = g.spmm(torch.from_numpy(X).to(DEV), schedule=S.SCHEDULE_ROWS)
    torch.cuda.synchronize()
    assert rel(Y.cpu().numpy(), ref) <= TOL_F32
    assert torch.equal(Y, Y2)  # no atomics: bitwise reproducible


@pytest.mark.parametrize("K", [32, 64, 256])
def test_rows_bf16_in_out(case12, K):
    n, row, col, val, ps = case12
    g = S.Graph(ps, hub_threshold=64, hub_segment=32)
    X = dense_x(n, K, seed=9)
    Xb = bf16_bits(X)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    ref_b = oracle.spmm_csr_f64(rp, ci, vv, Xb)
    ref_f = oracle.spmm_csr_f64(rp, ci, vv, X)
    xt = torch.from_numpy(Xb.view(np.int16)).view(torch.bfloat16).to(DEV)
    xf = torch.from_numpy(X).to(DEV)
    y32 = g.spmm(xt, out_dtype=torch.float32, schedule=S.SCHEDULE_ROWS)
    y16 = g.spmm(xt, out_dtype=torch.bfloat16, schedule=S.SCHEDULE_ROWS)
    yf16 = g.spmm(xf, out_dtype=torch.bfloat16, schedule=S.SCHEDULE_ROWS)
    torch.cuda.synchronize()
    assert rel(y32.cpu().numpy(), ref_b) <= TOL_F32
    assert rel(y16.float().cpu().numpy(), ref_f) <= TOL_BF16
    assert rel(yf16.float().cpu().numpy(), ref_f) <= TOL_BF16
    # the BF16 output is the FP32 accumulation rounded once (same order: exact)
    assert torch.equal(y16, y32.to(torch.bfloat16))


def test_rows_accumulate_strides_and_agreement(case12):
    n, row, col, val, ps = case12
    g = S.Graph(ps, hub_threshold=32, hub_segment=16)
    K = 64
    X = dense_x(n, K, seed=12)
    ref = fp64_reference(n, row, col, val, X)
    big = torch.zeros((n, 80), device=DEV)
    big[:, :K] = torch.from_numpy(X).to(DEV)
    Y = torch.zeros((n, 72), device=DEV)
    g.spmm(big[:, :K], Y[:, :K], schedule=S.SCHEDULE_ROWS)
    g.spmm(big[:, :K], Y[:, :K], accumulate=True, schedule=S.SCHEDULE_ROWS)
    yf = g.spmm(big[:, :K], schedule=S.SCHEDULE_FUSED)
    torch.cuda.synchronize()
    assert rel(Y[:, :K].cpu().numpy(), 2 * ref) <= TOL_F32
    assert torch.all(Y[:, K:] == 0)
    assert rel(yf.cpu().numpy(), Y[:, :K].cpu().numpy() / 2) <= TOL_F32


def test_rows_view_optional(case12):
    n, row, col, val, ps = case12
    g = S.Graph(ps, row_view=False)
    with pytest.raises(cb.ColaError):
        g.spmm(torch.ones((n, 16), device=DEV), schedule=S.SCHEDULE_ROWS)
    Y = g.spmm(torch.ones((n, 16), device=DEV))  # AUTO falls back to the fused schedule
    torch.cuda.synchronize()
    assert Y.shape == (n, 16)


@pytest.mark.parametrize("K,thr,seg", [(128, 16, 8), (1024, 32, 16), (256, 1, 1)])
def test_rows_hub_combine_tiles_and_repeats(case12, K, thr, seg):
    """Hub rows: segment partials from the streaming kernel, combined pairwise
    by the vector combine kernel -- right on every call, over several feature
    tiles (K = 1024 FP32 is two tiles), two launches per call."""
    n, row, col, val, ps = case12
    g = S.Graph(ps, hub_threshold=thr, hub_segment=seg)
    assert g.info.hub_rows > 0
    X = dense_x(n, K, seed=K + thr)
    ref = fp64_reference(n, row, col, val, X)
    xt = torch.from_numpy(X).to(DEV)
    outs = [g.spmm(xt, schedule=S.SCHEDULE_ROWS) for _ in range(3)]
    torch.cuda.synchronize()
    assert g.get_info().last_launches == 2
    for y in outs:
        assert rel(y.cpu().numpy(), ref) <= TOL_F32
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[1], outs[2])


def test_row_view_sizes_follow_the_graph():
    """Without options the row view's item size follows the graph's size: a
    graph of a few thousand entries (far under 128 x 4 entries per warp of a
    full wave) cuts rows longer than 128 entries into 128-entry segments, the
    same from the host upload and the device build; options override it; the
    product is right either way."""
    n = 1000
    lens = {0: 300, 1: 200, 2: 129, 3: 128}
    rows, cols = [], []
    for r in range(n):
        k = lens.get(r, 1)
        rows += [r] * k
        cols += [(r * 7 + j * 3) % n for j in range(k)]
    row = np.array(rows, np.int32)
    col = np.array(cols, np.int32)
    key = row.astype(np.int64) * n + col
    _, first = np.unique(key, return_index=True)
    row, col = row[np.sort(first)], col[np.sort(first)]
    assert np.bincount(row, minlength=n)[:4].tolist() == [300, 200, 129, 128]
    val = np.linspace(0.5, 1.5, len(row)).astype(np.float32)
    gh = S.Graph(cb.PartitionSet.from_coo(n, row, col, val, 1))
    gd = S.Graph.from_coo_device(n, torch.from_numpy(row).to(DEV), torch.from_numpy(col).to(DEV),
                                 torch.from_numpy(val).to(DEV), nparts=1)
    for g in (gh, gd):
        assert (g.info.hub_rows, g.info.hub_segments) == (3, 3 + 2 + 2)
    go = S.Graph(cb.PartitionSet.from_coo(n, row, col, val, 1), hub_threshold=256, hub_segment=100)
    assert (go.info.hub_rows, go.info.hub_segments) == (1, 3)
    X = dense_x(n, 32, seed=11)
    ref = fp64_reference(n, row, col, val, X)
    xt = torch.from_numpy(X).to(DEV)
    for g in (gh, gd, go):
        y = g.spmm(xt, schedule=S.SCHEDULE_ROWS)
        torch.cuda.synchronize()
        assert rel(y.cpu().numpy(), ref) <= TOL_F32


def test_rows_item_counters_across_tile_counts(case12):
    """Work items are drawn from counters kept in the graph (one per feature
    tile) and put back to zero by the last warp of each launch: calls with 1,
    2 and 4 feature tiles, interleaved on one graph, each give the right
    result and the same bits as a fresh graph's first call."""
    n, row, col, val, ps = case12
    g = S.Graph(ps, hub_threshold=32, hub_segment=16)
    assert g.info.hub_rows > 0
    xs = {K: torch.from_numpy(dense_x(n, K, seed=K)).to(DEV) for K in (128, 1024, 2048)}
    first = {}
    for K in (1024, 128, 2048, 128, 1024, 2048):
        y = g.spmm(xs[K], schedule=S.SCHEDULE_ROWS)
        torch.cuda.synchronize()
        if K not in first:
            first[K] = y
            ref = fp64_reference(n, row, col, val, xs[K].cpu().numpy())
            assert rel(y.cpu().numpy(), ref) <= TOL_F32
        else:
            assert torch.equal(y, first[K])
    fresh = S.Graph(ps, hub_threshold=32, hub_segment=16)
    assert torch.equal(fresh.spmm(xs[2048], schedule=S.SCHEDULE_ROWS), first[2048])


# ---------------------------------------------------------------------------
# staged gathers by bulk asynchronous copies (TMA) vs 16-byte vectors
# ---------------------------------------------------------------------------
def _device_error():
    code = ctypes.c_int32(-1)
    assert cb.lib().cola_device_error_check(ctypes.byref(code)) == 0
    return code.value


@pytest.mark.parametrize("K", [4, 96, 256, 512, 1000, 4096, 3])
def test_bulk_gather_copies_rows_exactly(K):
    """The staged gather send[b] = X[idx[b] % npp] through bulk copies (rows of
    1 KB .. 4 KB; narrower rows, 3 columns and 16 KB rows take the vector
    gather) gives exactly
    the rows the vector gather and a plain index copy give, on repeated
    calls, and no bounded wait runs out."""
    npp, P, nemb = 700, 4, 2500
    X = torch.from_numpy(dense_x(P * npp, K, seed=K)).to(DEV)
    rng = np.random.Generator(np.random.Philox(K))
    idx = torch.from_numpy(rng.integers(0, P * npp, nemb).astype(np.int32)).to(DEV)
    want = X[(idx.long() % npp)]
    outs = []
    try:
        for bulk in (1, 0, 1):
            assert cb.lib().cola_set_gather_bulk(bulk) == 0
            out = torch.full((nemb, K), float("nan"), device=DEV)
            cb._lib.check(cb.lib().cola_batching_data_ppl(ptr(X), ptr(out), ptr(idx), nemb, K, npp, 1, None))
            torch.cuda.synchronize()
            outs.append(out)
    finally:
        cb.lib().cola_set_gather_bulk(0)  # the default
    for o in outs:
        assert torch.equal(o, want)
    assert _device_error() == 0


@pytest.mark.parametrize("K,xdt", [(4, torch.float32), (256, torch.float32), (512, torch.bfloat16),
                                   (1000, torch.float32), (4096, torch.float32), (3, torch.float32)])
def test_bulk_gather_schedules(case12, K, xdt):
    """BUFFER staging and PIPELINE puts through bulk copies against the vector
    gather (their float atomics sum in varying order, so within 1e-6) and the
    FP64 oracle, and no bounded wait runs out."""
    n, row, col, val, ps = case12
    X = torch.from_numpy(dense_x(n, K, seed=K)).to(DEV).to(xdt)
    outs = {}
    try:
        for bulk in (1, 0):
            assert cb.lib().cola_set_gather_bulk(bulk) == 0
            g = S.Graph(ps)
            gp = S.Graph(ps, group_size=2)
            outs[bulk] = (g.spmm(X, schedule=S.SCHEDULE_BUFFER, gather_batch_rows=300),
                          gp.spmm(X, schedule=S.SCHEDULE_PIPELINE))
            torch.cuda.synchronize()
    finally:
        cb.lib().cola_set_gather_bulk(0)  # the default
    for j in range(2):
        assert rel(outs[1][j].cpu().numpy(), outs[0][j].cpu().numpy()) <= 1e-6
    assert _device_error() == 0
    ref = fp64_reference(n, row, col, val, X.float().cpu().numpy())
    assert rel(outs[1][0].cpu().numpy(), ref) <= TOL_F32
    assert rel(outs[1][1].cpu().numpy(), ref) <= TOL_F32


def test_bulk_gather_wait_limit_reports_and_drains():
    """A bulk-copy gather whose per-row wait is cut to one poll gives up on
    its first row, reports error 1 (it stopped early and drained every load it
    had issued: no copy is left in flight), and the device stays usable: with
    the default limit the same gather is exact again and reports nothing."""
    npp, P, nemb, K = 4096, 4, 20000, 1024  # 4 KB rows, far slower than one poll
    X = torch.from_numpy(dense_x(P * npp, K, seed=5)).to(DEV)
    rng = np.random.Generator(np.random.Philox(5))
    idx = torch.from_numpy(rng.integers(0, P * npp, nemb).astype(np.int32)).to(DEV)
    want = X[(idx.long() % npp)]
    out = torch.zeros((nemb, K), device=DEV)
    assert _device_error() == 0
    try:
        assert cb.lib().cola_set_gather_bulk(1) == 0
        assert cb.lib().cola_set_gather_wait_limit(1) == 0
        cb._lib.check(cb.lib().cola_batching_data_ppl(ptr(X), ptr(out), ptr(idx), nemb, K, npp, 1, None))
        torch.cuda.synchronize()
        assert _device_error() == 1
        assert cb.lib().cola_set_gather_wait_limit(0) == 0
        out.zero_()
        cb._lib.check(cb.lib().cola_batching_data_ppl(ptr(X), ptr(out), ptr(idx), nemb, K, npp, 1, None))
        torch.cuda.synchronize()
        assert _device_error() == 0
        assert torch.equal(out, want)
    finally:
        cb.lib().cola_set_gather_wait_limit(0)
        cb.lib().cola_set_gather_bulk(0)
    assert cb.lib().cola_set_gather_wait_limit(-1) == 1  # COLA_ERROR_INVALID_ARGUMENT


def _zip_rows(g, p, P):
    z = g.zip_view(p)
    h = ctypes.c_void_p()
    args = [z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx, z.csc_colIdx_zip,
            z.csc_val]
    args = [a if a is None or isinstance(a, ctypes.c_void_p) else ctypes.c_void_p(a) for a in args]
    cb._lib.check(cb.lib().cola_zip_rows_create(*args, 0, 0, z.local_chunks, z.remote_chunks, g.nodes_per_part, p,
                                                None, ctypes.byref(h)))
    return h


@pytest.mark.parametrize("K", [16, 100, 128, 256])
def test_zip_rows_view_matches_reference_kernels_and_rows(K):
    """The row view built from a PE's split blocks (what compat.h's
    ppl0_batch_SpMM keeps per d_csr_zip / d_csc_zip pair) adds the same
    product as the chunk launcher: within 1e-5 of FP64 and of the reference's
    kernels, equal to the graph's own row-major output for the partition's
    rows (the same entries in the same order; bit for bit where one lane group
    takes a row), the same bits on a repeated call, and exactly twice that
    after two calls into one output."""
    P = 4
    n, row, col, val, ps = graph_case(12, 16, seed=21, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X = _padded_x(n, P, npp, K, seed=K)
    Xd = torch.from_numpy(X).to(DEV)
    ref64 = fp64_reference(n, row, col, val, X[:n])
    rows = g.spmm(Xd[:n], schedule=S.SCHEDULE_ROWS)
    L = cb.lib()
    hs = [_zip_rows(g, p, P) for p in range(P)]
    try:
        outs = []
        for rep in range(2):
            Y = torch.zeros((P * npp, K), device=DEV)
            for p in range(P):
                cb._lib.check(L.cola_zip_rows_spmm(hs[p], ptr(Y[p * npp:]), ptr(Xd[p * npp:]), K, None))
            torch.cuda.synchronize()
            outs.append(Y)
        Y2 = outs[1].clone()
        for p in range(P):
            cb._lib.check(L.cola_zip_rows_spmm(hs[p], ptr(Y2[p * npp:]), ptr(Xd[p * npp:]), K, None))
        torch.cuda.synchronize()
        nnz = ctypes.c_int64()
        cb._lib.check(L.cola_zip_rows_get_info(hs[0], None, ctypes.byref(nnz), None, None))
        z0 = g.zip_view(0)
        assert nnz.value == z0.nnz_l + z0.nnz_r
    finally:
        for h in hs:
            L.cola_zip_rows_free(h)
    y = outs[0][:n]
    assert rel(y.cpu().numpy(), ref64) <= TOL_F32
    assert torch.equal(outs[0], outs[1])
    if K // 4 > 16:
        # one lane group per row (K > 64 FP32): each element is one FMA chain
        # in column order, whichever tasks the rows fall in
        assert torch.equal(y, rows)  # value equality (+0 and -0 compare equal)
    else:
        # narrower rows share a warp between lane groups, whose split of a row
        # follows the row's offset in its task: the same sum in another order
        assert rel(y.cpu().numpy(), rows.cpu().numpy()) <= 1e-6
    assert torch.equal(Y2, 2 * outs[0])
    if oracle.ref_available():
        theirs = _run_reference(g, Xd, npp, K, P)[:n].cpu().numpy()
        assert rel(y.cpu().numpy(), theirs) <= TOL_F32


@pytest.mark.parametrize("K", [32, 128])
def test_zip_rows_all_pes_one_view(K):
    """Every PE's chunks in one row view (cola_zip_rows_create_all, what
    compat.h's single-stage distSpMM_ppl_batch_all keeps): one call adds the
    whole product, equal to the graph's own row-major output (bit for bit
    where one lane group takes a row), within 1e-5 of FP64."""
    P = 4
    n, row, col, val, ps = graph_case(12, 16, seed=23, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X = _padded_x(n, P, npp, K, seed=K)
    Xd = torch.from_numpy(X).to(DEV)
    parts = (cb._lib.ZipPart * P)()
    for p in range(P):
        z = g.zip_view(p)
        q = parts[p]
        q.csr_rowPtr_l, q.csr_colIdx_l, q.csr_rowIdx_zip_l, q.csr_val_l = (z.csr_rowPtr, z.csr_colIdx,
                                                                           z.csr_rowIdx_zip, z.csr_val)
        q.csc_colPtr_r, q.csc_rowIdx_r, q.csc_colIdx_zip_r, q.csc_val_r = (z.csc_colPtr, z.csc_rowIdx,
                                                                           z.csc_colIdx_zip, z.csc_val)
        q.local_row_lb, q.remote_col_lb, q.local_row_num, q.remote_col_num = 0, 0, z.local_chunks, z.remote_chunks
    L = cb.lib()
    h = ctypes.c_void_p()
    cb._lib.check(L.cola_zip_rows_create_all(parts, P, npp, None, ctypes.byref(h)))
    try:
        Y = torch.zeros((P * npp, K), device=DEV)
        cb._lib.check(L.cola_zip_rows_spmm(h, ptr(Y), ptr(Xd), K, None))
        torch.cuda.synchronize()
        nnz = ctypes.c_int64()
        cb._lib.check(L.cola_zip_rows_get_info(h, None, ctypes.byref(nnz), None, None))
        assert nnz.value == g.info.nnz
    finally:
        L.cola_zip_rows_free(h)
    rows = g.spmm(Xd[:n], schedule=S.SCHEDULE_ROWS)
    y = Y[:n]
    assert rel(y.cpu().numpy(), fp64_reference(n, row, col, val, X[:n])) <= TOL_F32
    if K // 4 > 16:
        assert torch.equal(y, rows)
    else:
        assert rel(y.cpu().numpy(), rows.cpu().numpy()) <= 1e-6
    assert torch.all(Y[n:] == 0)


@pytest.mark.parametrize("xdt,ydt", [(torch.float32, torch.float32), (torch.bfloat16, torch.bfloat16)])
def test_spmm_host_pipelined_calls(case12, xdt, ydt):
    """cola_spmm_host: host X in, SpMM, host Y out, consecutive calls
    overlapped by the library (two staging sets); every call's Y equals the
    device call's bits, strided host rows included, and accumulate is
    refused."""
    n, row, col, val, ps = case12
    g = S.Graph(ps)
    K = 128
    xs = [torch.from_numpy(dense_x(n, K, seed=s)).to(xdt).pin_memory() for s in (1, 2, 3)]
    ys = [torch.empty((n, K), dtype=ydt).pin_memory() for _ in range(3)]
    for x, y in zip(xs, ys):
        g.spmm_host(x, y)
    g.sync_host()
    for x, y in zip(xs, ys):
        want = g.spmm(x.to(DEV), out_dtype=ydt).cpu()
        assert torch.equal(y, want)
    # strided host rows: a view of wider matrices
    xw = torch.zeros((n, K + 8), dtype=xdt).pin_memory()
    xw[:, :K] = xs[0]
    yw = torch.full((n, K + 4), 7.0, dtype=ydt).pin_memory()
    g.spmm_host(xw[:, :K], yw[:, :K])
    g.sync_host()
    assert torch.equal(yw[:, :K], ys[0]) and torch.all(yw[:, K:] == 7.0)
    o = cb._lib.SpmmOpts()
    o.accumulate = 1
    rc = cb.lib().cola_spmm_host(g._h, ptr(xs[0]), 0 if xdt == torch.float32 else 1, K, ptr(ys[0]),
                                 0 if ydt == torch.float32 else 1, K, K, ctypes.byref(o), None)
    assert rc == 4  # COLA_ERROR_UNSUPPORTED


def test_community_order_then_spmm_is_the_permuted_product():
    """Vertices relabelled by the community ordering, then partitioned and
    multiplied: row mapping[i] of the result is row i of the product on the
    original numbering (features permuted alike), within 1e-5 of FP64."""
    n, row, col, val = cb.rmat(12, 16, seed=6)
    mp, _ = cb.community_order(n, row, col)
    r2, c2 = cb.relabel_edges(n, row, col, mp)
    ps = cb.PartitionSet.from_coo(n, r2, c2, val, 4)
    g = S.Graph(ps)
    X = dense_x(n, 64, seed=6)
    Xp = np.empty_like(X)
    Xp[mp] = X
    Y = g.spmm(torch.from_numpy(Xp).to(DEV)).cpu().numpy()
    ref = fp64_reference(n, row, col, val, X)
    assert rel(Y[mp], ref) <= TOL_F32
