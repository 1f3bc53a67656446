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
