"""The staging variant that allocates nothing, cola_ppl0_batch_buffer_spmm_noalloc.

Some callers of this library cannot allocate device memory and have none to
lend: code that runs under a host framework owning every device allocation, or
a latency-bound loop that must not call cudaMalloc (it synchronises the device
and can fail under memory pressure).  For them the buffer-staged launcher has a
variant that stages the remote rows in a fixed array inside the library.  This
file checks it through the C ABI against the ordinary launcher, which stages
into a caller buffer, on two calls in a row (the second call reuses the array
the first call left behind), and that an over-size request is refused before
anything is launched.

It sits in a file of its own, named to be collected last, so that a run that
stops at the first failure has run every other test first; it builds all its
inputs itself, so it also passes alone in a fresh process.
"""
import ctypes

import pytest
import torch

import cola_b200 as cb
from cola_b200 import _lib
from cola_b200 import spmm as S

from gpu_util import TOL_F32, dense_x, graph_case, ptr, rel

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _launch(fn, g, Xd, npp, K, P, buf=None):
    """Run one launcher over every virtual partition into a zeroed output."""
    Y = torch.zeros((P * npp, K), device=DEV)
    for p in range(P):
        z = g.zip_view(p)
        args = [ptr(Y[p * npp:]), ptr(Xd[p * npp:])]
        if buf is not None:
            args.append(ptr(buf))
        args += [z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx,
                 z.csc_colIdx_zip, z.csc_val]
        args = [a if a is None or isinstance(a, ctypes.c_void_p) else ctypes.c_void_p(a) for a in args]
        _lib.check(fn(*args, 0, 0, z.local_chunks, z.remote_chunks, K, npp, p, None))
    torch.cuda.synchronize()
    return Y


@pytest.mark.parametrize("K", [64, 100])
def test_noalloc_matches_buffer_launcher_twice(K):
    P = 4
    n, row, col, val, ps = graph_case(12, 16, seed=41, nparts=P)
    g = S.Graph(ps)
    npp = g.nodes_per_part
    nr = max(g.zip_view(p).remote_chunks for p in range(P))
    assert nr * K <= _lib.NOALLOC_STAGE_FLOATS
    X = torch.zeros((P * npp, K), device=DEV)
    X[:n] = torch.from_numpy(dense_x(n, K, seed=K)).to(DEV)
    L = cb.lib()
    buf = torch.empty((nr, K), device=DEV)
    want = _launch(L.cola_ppl0_batch_buffer_spmm, g, X, npp, K, P, buf=buf)[:n].cpu().numpy()
    first = _launch(L.cola_ppl0_batch_buffer_spmm_noalloc, g, X, npp, K, P)[:n].cpu().numpy()
    second = _launch(L.cola_ppl0_batch_buffer_spmm_noalloc, g, X, npp, K, P)[:n].cpu().numpy()
    assert rel(first, want) <= TOL_F32
    assert rel(second, want) <= TOL_F32


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
