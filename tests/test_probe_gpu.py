"""The gather-ceiling probe (cola_probe_gather) the bench reports beside the
SpMM: it runs, a table that fits in L2 gathers faster than one far larger than
L2, and bad arguments are refused before anything is allocated."""
import ctypes

import pytest
import torch

import cola_b200 as cb

pytestmark = pytest.mark.gpu


def test_probe_l2_faster_than_dram():
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    l2, dram = ctypes.c_double(), ctypes.c_double()
    assert cb.lib().cola_probe_gather(32 << 20, 512, 1 << 22, 2, st, ctypes.byref(l2)) == 0
    assert cb.lib().cola_probe_gather(2 << 30, 512, 1 << 22, 2, st, ctypes.byref(dram)) == 0
    assert dram.value > 100 and l2.value > dram.value


def test_probe_rejects_bad_rows():
    v = ctypes.c_double()
    assert cb.lib().cola_probe_gather(1 << 20, 24, 100, 1, None, ctypes.byref(v)) == 1
    assert cb.lib().cola_probe_gather(1 << 20, 1024, 100, 1, None, ctypes.byref(v)) == 1


def test_graph_pattern_probe():
    """cola_probe_graph_gather reads the X rows a graph's entries name, in
    the row view's order: it runs for narrow and wide rows, its rate is
    entries x row bytes over its pass time, and it refuses a graph without
    a row view or unaligned rows."""
    import numpy as np
    from cola_b200 import spmm as S
    n, row, col, val = cb.rmat(12, 16, seed=2)
    g = S.Graph(cb.PartitionSet.from_coo(n, row, col, val, 4))
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for K, dt in ((128, torch.float32), (256, torch.bfloat16), (512, torch.float32)):
        X = torch.randn(n, K, device="cuda").to(dt)
        rb = K * X.element_size()
        v, t = ctypes.c_double(), ctypes.c_float()
        assert cb.lib().cola_probe_graph_gather(g._h, ctypes.c_void_p(X.data_ptr()), rb, rb, 2, st, ctypes.byref(v),
                                                ctypes.byref(t)) == 0
        assert v.value > 0 and t.value > 0
        assert abs(v.value - len(row) * rb / (t.value * 1e-3) / 1e9) <= 1e-6 * v.value
    X = torch.randn(n, 128, device="cuda")
    v = ctypes.c_double()
    assert cb.lib().cola_probe_graph_gather(g._h, ctypes.c_void_p(X.data_ptr() + 4), 512, 512, 1, st,
                                            ctypes.byref(v), None) == 1
    assert cb.lib().cola_probe_graph_gather(g._h, ctypes.c_void_p(X.data_ptr()), 512, 24, 1, st,
                                            ctypes.byref(v), None) == 1
    assert np.isfinite(v.value)
