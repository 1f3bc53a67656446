"""GPU parity at the benchmark configurations' own sizes, collected before the
slower tests.

* Configuration 1 exactly (R-MAT scale 14, degree 16, self-loops, values
  1/deg(row), K = 32, P = 4): the row-major, fused and buffer schedules and
  the kernel-level drop-ins against the FP64 oracle over every row, against
  the reference's own CUDA kernels, and against torch.sparse.mm on the host.
* Configuration 2 (scale 20, degree 32, K = 128, FP32, P = 8): the row-major
  schedule and the drop-in launcher against the reference's kernels
  (ppl0_batch_SpMM<4, false>) and FP64 on sampled rows.
* Configuration 3 (scale 21, degree 48, K = 256, hub rows of tens of thousands
  of entries): FP32 within 1e-5 and BF16 storage within 1e-2 of FP64 on
  sampled rows including the 64 longest; those hub rows bit for bit equal to
  the oracle's restatement of the schedule's summation order; every feature
  tile width gives the same bits.

Inputs follow the configurations (prep_torch_par.py:24-79 partitions,
include/dist_spmm_ppl_batch.cuh:76-245 kernels); the FP64 products are the
oracle's (oracle/cola_oracle.c)."""
import warnings

import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200 import spmm as S
from oracle import oracle

from gpu_util import TOL_BF16, TOL_F32, bf16_bits, dense_x, ptr, rel

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")


def sampled_rows(n, row, samples, longest, seed=0):
    """Evenly spaced rows plus the `longest` rows with the most entries."""
    counts = np.bincount(row, minlength=n)
    pick = np.unique(np.concatenate([np.linspace(0, n - 1, samples).astype(np.int64),
                                     np.argsort(counts, kind="stable")[-longest:].astype(np.int64)]))
    return pick, counts


def sub_csr(rp, ci, vv, rows):
    """The CSR of the given rows only (their entries in the same order)."""
    lens = (rp[rows + 1] - rp[rows]).astype(np.int64)
    sp = np.zeros(len(rows) + 1, np.int64)
    np.cumsum(lens, out=sp[1:])
    idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
    return sp, ci[idx], vv[idx]


def run_dropin(fn, g, Xd, npp, K, P, buf=None):
    import ctypes
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        args = [ptr(Y[p * npp:]), ptr(Xd[p * npp:])] + ([ptr(buf)] if buf is not None else [])
        args += [z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx,
                 z.csc_colIdx_zip, z.csc_val]
        args = [a if a is None or isinstance(a, ctypes.c_void_p) else ctypes.c_void_p(a) for a in args]
        assert fn(*args, 0, 0, z.local_chunks, z.remote_chunks, K, npp, p, None) == 0
    torch.cuda.synchronize()
    return Y


def run_reference(g, Xd, npp, K, P):
    R = oracle.ref()
    CF, res = (K + 31) // 32, 1 if K & 31 else 0
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        assert R.ref_set_pe(p, npp * K, None) == 0
        assert R.ref_ppl0_batch_spmm(CF, res, ptr(Y[p * npp:]), ptr(Xd[p * npp:]), z.csr_rowPtr, z.csr_colIdx,
                                     z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx, z.csc_colIdx_zip,
                                     z.csc_val, 0, 0, z.local_chunks, z.remote_chunks, K, npp, p, None) == 0
    torch.cuda.synchronize()
    return Y


def padded(n, P, npp, K, seed):
    X = np.zeros((P * npp, K), np.float32)
    X[:n] = dense_x(n, K, seed)
    return X


# ---------------------------------------------------------------------------
def test_config1_exact_every_path():
    P, K = 4, 32
    n, row, col, val = cb.rmat(14, 16, seed=1, self_loops=True, values=cb.prep.VALUES_ROW_NORMALISED)
    ps = cb.PartitionSet.from_coo(n, row, col, val, P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X = padded(n, P, npp, K, seed=1)
    Xd = torch.from_numpy(X).to(DEV)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    ref = oracle.spmm_csr_f64(rp, ci, vv, X[:n])
    outs = {"rows": g.spmm(Xd[:n], schedule=S.SCHEDULE_ROWS),
            "fused": g.spmm(Xd[:n], schedule=S.SCHEDULE_FUSED),
            "buffer": g.spmm(Xd[:n], schedule=S.SCHEDULE_BUFFER)}
    L = cb.lib()
    nr = max(g.zip_view(p).remote_chunks for p in range(P))
    outs["ppl0"] = run_dropin(L.cola_ppl0_batch_spmm, g, Xd, npp, K, P)[:n]
    outs["ppl0_seq"] = run_dropin(L.cola_ppl0_batch_spmm_seq, g, Xd, npp, K, P)[:n]
    outs["ppl0_buffer"] = run_dropin(L.cola_ppl0_batch_buffer_spmm, g, Xd, npp, K, P,
                                     buf=torch.empty((nr, K), device=DEV))[:n]
    torch.cuda.synchronize()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # torch marks sparse CSR as beta
        A = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)), torch.from_numpy(ci.astype(np.int64)),
                                    torch.from_numpy(vv), size=(n, n))
        host = torch.sparse.mm(A, torch.from_numpy(X[:n])).numpy()
    assert rel(host, ref) <= TOL_F32
    for name, y in outs.items():
        y = y.cpu().numpy()
        assert rel(y, ref) <= TOL_F32, name
        assert rel(y, host) <= TOL_F32, name
    if oracle.ref_available():
        theirs = run_reference(g, Xd, npp, K, P)[:n].cpu().numpy()
        assert rel(theirs, ref) <= TOL_F32
        for name, y in outs.items():
            assert rel(y.cpu().numpy(), theirs) <= TOL_F32, name


@needs_ref
def test_config2_against_reference_kernels():
    P, K = 8, 128
    n, row, col, val = cb.rmat(20, 32, seed=2)
    ps = cb.PartitionSet.from_coo(n, row, col, val, P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X = padded(n, P, npp, K, seed=2)
    Xd = torch.from_numpy(X).to(DEV)
    theirs = run_reference(g, Xd, npp, K, P)[:n]
    ours = g.spmm(Xd[:n])
    dropin = run_dropin(cb.lib().cola_ppl0_batch_spmm, g, Xd, npp, K, P)[:n]
    torch.cuda.synchronize()
    pick, _ = sampled_rows(n, row, 4096, 64)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    sp, sc, sv = sub_csr(rp, ci, vv, pick)
    ref = oracle.spmm_csr_f64(sp, sc, sv, X)
    idx = torch.from_numpy(pick).to(DEV)
    t, o, d = (a[idx].cpu().numpy() for a in (theirs, ours, dropin))
    assert rel(t, ref) <= TOL_F32
    assert rel(o, t) <= TOL_F32 and rel(o, ref) <= TOL_F32
    assert rel(d, t) <= TOL_F32 and rel(d, ref) <= TOL_F32


@pytest.fixture(scope="module")
def config3():
    n, row, col, val = cb.rmat(21, 48, seed=3)
    g = S.Graph.from_coo_device(n, torch.from_numpy(row).to(DEV), torch.from_numpy(col).to(DEV),
                                torch.from_numpy(val).to(DEV), nparts=8)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    pick, counts = sampled_rows(n, row, 4096, 64)
    assert counts.max() > 10000  # hub rows of tens of thousands of entries
    return n, g, rp, ci, vv, pick, counts


def test_config3_fp32_and_bf16_against_fp64(config3):
    n, g, rp, ci, vv, pick, _ = config3
    K = 256
    X = dense_x(n, K, seed=3)
    sp, sc, sv = sub_csr(rp, ci, vv, pick)
    ref = oracle.spmm_csr_f64(sp, sc, sv, X)
    idx = torch.from_numpy(pick).to(DEV)
    X32 = torch.from_numpy(X).to(DEV)
    y32 = g.spmm(X32)[idx].cpu().numpy()
    assert rel(y32, ref) <= TOL_F32
    Xb = X32.to(torch.bfloat16)
    del X32
    ref_b = oracle.spmm_csr_f64(sp, sc, sv, bf16_bits(X))  # FP64 on the BF16-rounded features
    for ydt in (torch.float32, torch.bfloat16):
        y = g.spmm(Xb, out_dtype=ydt)[idx].float().cpu().numpy()
        assert rel(y, ref) <= TOL_BF16
        if ydt == torch.float32:
            assert rel(y, ref_b) <= TOL_F32


@pytest.mark.parametrize("xdt,tiles", [(torch.float32, (0, 64, 128, 256)),
                                       (torch.bfloat16, (0, 64, 128, 256))])
def test_config3_hub_rows_bitwise_and_tile_widths(config3, xdt, tiles):
    """The 64 longest rows (each cut into 512-entry segments, the default) equal the
    oracle's restatement of the summation order bit for bit, and the whole
    output is the same bits at every feature tile width."""
    n, g, rp, ci, vv, pick, counts = config3
    K = 256
    Xd = torch.from_numpy(dense_x(n, K, seed=30)).to(DEV).to(xdt)
    outs = [g.spmm(Xd, out_dtype=torch.float32, k_tile=t) for t in tiles]
    torch.cuda.synchronize()
    for y in outs[1:]:
        assert torch.equal(y, outs[0])
    hubs = np.argsort(counts, kind="stable")[-64:].astype(np.int64)
    sp, sc, sv = sub_csr(rp, ci, vv, hubs)
    want = oracle.spmm_rows_f32_ordered(sp, sc, sv, Xd.float().cpu().numpy(), hub_threshold=512,
                                        hub_segment=512)
    got = outs[0][torch.from_numpy(hubs).to(DEV)].cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
