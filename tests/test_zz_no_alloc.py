"""The staging variant that allocates nothing, cola_ppl0_batch_buffer_spmm_noalloc.

Some callers of this library cannot allocate device memory and have none to
lend: code that runs under a host framework owning every device allocation, or
a latency-bound loop that must not call cudaMalloc (it synchronises the device
and can fail under memory pressure).  For them the buffer-staged launcher has a
variant that stages the remote rows in a fixed array inside the library.  This
file checks it through the C ABI against the FP64 oracle and against the
ordinary launcher, which stages into a caller buffer:

* on two calls in a row with different features, so rows the first call left
  in the shared array would show up as a wrong second answer;
* with a partition's remote range split over two calls (the second starting
  at remote_col_lb > 0, where the staged rows are numbered from that offset);
* at exactly the array's capacity (the last staged row is the array's last);
* and that an over-size request is refused before anything is launched.

The two launchers scatter remote rows with float atomics whose order varies
from run to run, so they are compared within 1e-6, not bit for bit.

It sits in a file of its own, named to be collected last, so that a run that
stops at the first failure has run every other test first; it builds all its
inputs itself, so it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200 import _lib
from cola_b200 import spmm as S

from gpu_util import TOL_F32, dense_x, fp64_reference, graph_case, ptr, rel

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
SAME = 1e-6  # the two launchers: same gathers and kernel, atomics in another order


def _vp(a):
    return a if a is None or isinstance(a, ctypes.c_void_p) else ctypes.c_void_p(a)


def _call(fn, Y, X, z, local_num, r_lb, r_num, K, npp, p, buf=None):
    args = [ptr(Y[p * npp:]), ptr(X[p * npp:])]
    if buf is not None:
        args.append(ptr(buf))
    args += [z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx,
             z.csc_colIdx_zip, z.csc_val]
    _lib.check(fn(*[_vp(a) for a in args], 0, r_lb, local_num, r_num, K, npp, p, None))


def _launch(fn, g, Xd, npp, K, P, buf=None):
    """Run one launcher over every virtual partition into a zeroed output."""
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        _call(fn, Y, Xd, z, z.local_chunks, 0, z.remote_chunks, K, npp, p, buf)
    torch.cuda.synchronize()
    return Y


def _features(n, npp, P, K, seed):
    X = torch.zeros((P * npp, K), device=DEV)
    Xh = dense_x(n, K, seed=seed)
    X[:n] = torch.from_numpy(Xh).to(DEV)
    return X, Xh


@pytest.mark.parametrize("K", [64, 100])
def test_noalloc_matches_buffer_launcher_and_fp64_twice(K):
    P = 4
    n, row, col, val, ps = graph_case(12, 16, seed=41, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    nr = max(g.zip_view(p).remote_chunks for p in range(P))
    assert nr * K <= _lib.NOALLOC_STAGE_FLOATS
    L = cb.lib()
    buf = torch.empty((nr, K), device=DEV)
    for seed in (K, K + 1000):  # the second call's features differ from the first's
        X, Xh = _features(n, npp, P, K, seed)
        ref = fp64_reference(n, row, col, val, Xh)
        want = _launch(L.cola_ppl0_batch_buffer_spmm, g, X, npp, K, P, buf=buf)[:n].cpu().numpy()
        got = _launch(L.cola_ppl0_batch_buffer_spmm_noalloc, g, X, npp, K, P)[:n].cpu().numpy()
        assert rel(got, ref) <= TOL_F32
        assert rel(got, want) <= SAME


def test_noalloc_remote_range_split_over_two_calls():
    """Every partition's remote chunks in two calls: [0, h) together with the
    local chunks, then [h, nr) alone (remote_col_lb = h); the sum is the FP64
    product."""
    P, K = 4, 96
    n, row, col, val, ps = graph_case(12, 16, seed=43, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    X, Xh = _features(n, npp, P, K, seed=7)
    ref = fp64_reference(n, row, col, val, Xh)
    fn = cb.lib().cola_ppl0_batch_buffer_spmm_noalloc
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        h = z.remote_chunks // 3
        assert 0 < h < z.remote_chunks
        _call(fn, Y, X, z, z.local_chunks, 0, h, K, npp, p)
        _call(fn, Y, X, z, 0, h, z.remote_chunks - h, K, npp, p)
    torch.cuda.synchronize()
    assert rel(Y[:n].cpu().numpy(), ref) <= TOL_F32


def test_noalloc_at_exact_capacity():
    """remote_col_num * dim equal to the array's capacity (8,192 rows of 256
    floats): one remote entry per column, so every staged row, the last one
    included, lands in its own output row."""
    dim = 256
    nr = _lib.NOALLOC_STAGE_FLOATS // dim
    assert nr * dim == _lib.NOALLOC_STAGE_FLOATS
    npp, P = nr, 2
    rng = np.random.Generator(np.random.Philox(3))
    rows = rng.permutation(npp).astype(np.int32)             # partition 0's row of remote column j
    cols = (npp + np.arange(nr)).astype(np.int32)             # global columns owned by partition 1
    vals = rng.standard_normal(nr).astype(np.float32)
    Xh = dense_x(P * npp, dim, seed=9)
    want = np.zeros((npp, dim))
    want[rows] = vals[:, None].astype(np.float64) * Xh[cols].astype(np.float64)
    dev = {k: torch.from_numpy(v).to(DEV) for k, v in
           dict(colptr=np.arange(nr + 1, dtype=np.int32), rowidx=rows, colidx=cols, val=vals,
                lptr=np.zeros(1, np.int32), lcol=np.zeros(1, np.int32), lrow=np.zeros(1, np.int32),
                lval=np.zeros(1, np.float32)).items()}
    X = torch.from_numpy(Xh).to(DEV)
    L = cb.lib()
    outs = []
    for fn, buf in ((L.cola_ppl0_batch_buffer_spmm_noalloc, None),
                    (L.cola_ppl0_batch_buffer_spmm, torch.empty((nr, dim), device=DEV))):
        Y = torch.zeros((npp, dim), device=DEV)
        args = [ptr(Y), ptr(X)] + ([ptr(buf)] if buf is not None else [])
        args += [ptr(dev[k]) for k in ("lptr", "lcol", "lrow", "lval", "colptr", "rowidx", "colidx", "val")]
        _lib.check(fn(*args, 0, 0, 0, nr, dim, npp, 0, None))
        torch.cuda.synchronize()
        outs.append(Y.cpu().numpy())
    assert rel(outs[0], want) <= TOL_F32
    assert np.array_equal(outs[0], outs[1])  # one entry per output row: no atomic order to differ


def test_noalloc_rejects_oversize_request():
    L = cb.lib()
    dim = 256
    rows = _lib.NOALLOC_STAGE_FLOATS // dim + 1  # one row more than the array holds
    out = torch.zeros((1, dim), device=DEV)
    st = L.cola_ppl0_batch_buffer_spmm_noalloc(ptr(out), ptr(out), None, None, None, None, None, None, None, None,
                                               0, 0, 0, rows, dim, 1, 0, None)
    assert st == 1  # COLA_ERROR_INVALID_ARGUMENT, nothing launched
    assert b"fixed array holds" in L.cola_last_error()
    torch.cuda.synchronize()
    assert torch.all(out == 0)
