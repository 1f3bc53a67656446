"""Helpers shared by the GPU parity tests: seeded inputs and the checkers."""
import ctypes

import numpy as np
import torch

import cola_b200 as cb
from oracle import oracle

# FP32 SpMM vs FP64: relative Frobenius error bound required of every FP32 path
TOL_F32 = 1e-5
# BF16-stored features (or BF16 output) vs FP64 on FP32 features
TOL_BF16 = 1e-2


def dense_x(n_rows, K, seed):
    """X ~ N(0, 1), FP32, from a Philox stream with the given seed."""
    g = np.random.Generator(np.random.Philox(seed))
    return g.standard_normal((n_rows, K), dtype=np.float32)


def bf16_bits(x):
    """Round FP32 to BF16 (nearest even) and return the raw uint16 bits."""
    t = torch.from_numpy(np.ascontiguousarray(x)).to(torch.bfloat16)
    return t.view(torch.int16).numpy().view(np.uint16)


def fp64_reference(n, row, col, val, X):
    """FP64 oracle Y = A X over the global CSR (prep_torch_par.py:93-101)."""
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    return oracle.spmm_csr_f64(rp, ci, vv, X)


def graph_case(scale, deg, seed, nparts, self_loops=False):
    n, row, col, val = cb.rmat(scale, deg, seed, self_loops=self_loops)
    ps = cb.PartitionSet.from_coo(n, row, col, val, nparts)
    return n, row, col, val, ps


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


def rel(y, ref):
    return oracle.rel_frobenius(y, ref)
