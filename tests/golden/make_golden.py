"""Write the golden fixtures for the partition preprocessing.

Runs the reference's OWN preprocessing on seeded COO inputs and stores what it
writes, so the parity tests can run where the reference tree is absent:

* ``prep_torch_par.row_partition`` (prep_torch_par.py:24-79) -> per partition the
  six int32 ``.bin`` arrays (local CSR rowPtr/colIdx/rowIdx, remote CSC
  colPtr/rowIdx/colIdx);
* ``prep_torch_par.serialize``'s global CSR (prep_torch_par.py:93-101), computed
  by the same ``A.tocsr()`` call;
* ``prep_torch_ppl.row_partition`` (prep_torch_ppl.py:24-49) -> the work-group
  column lists ``colIdx_{P}_{stages}_{s}.bin``;
* the reference's C++ ``nnz_split`` (include/dist_spmm_ppl_batch.cuh:29-56),
  compiled from the reference tree by oracle/Makefile, on every partition's
  local CSR and remote CSC.

Usage (in a container that has the reference tree and oracle/_ref built)::

    python tests/golden/make_golden.py [--ref-root DIR]   (default: $COLA_REF_ROOT, else
    a checkout named `reference` beside this repository's directory)

The inputs are generated here from fixed seeds (numpy PCG64) and stored in the
fixture next to the outputs.
"""
import argparse
import ctypes
import importlib.util
import os
import sys
import tempfile

import numpy as np
import scipy
from scipy.sparse import coo_matrix

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def rmat_coo(scale, deg, seed, a=0.57, b=0.19, c=0.19):
    """Small seeded R-MAT edge list, symmetrised, self-loops dropped, duplicates kept."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = 1 << scale
    m = n * deg // 2
    row = np.zeros(m, dtype=np.int64)
    col = np.zeros(m, dtype=np.int64)
    for _ in range(scale):
        u = rng.random(m)
        rbit = u >= a + b
        cbit = ((u >= a) & (u < a + b)) | (u >= a + b + c)
        row = (row << 1) | rbit
        col = (col << 1) | cbit
    keep = row != col
    row, col = row[keep], col[keep]
    r = np.concatenate([row, col]).astype(np.int32)
    c2 = np.concatenate([col, row]).astype(np.int32)
    return n, r, c2


def cases():
    out = []
    # 1. hand-made: duplicates, unsorted input, empty rows and columns,
    #    N not a multiple of P, a partition with no local entries.
    row = np.array([0, 3, 3, 1, 9, 9, 2, 5, 3, 8, 0, 7, 4, 4, 6], dtype=np.int32)
    col = np.array([5, 0, 0, 9, 1, 1, 8, 2, 7, 3, 6, 7, 4, 0, 6], dtype=np.int32)
    out.append(("hand10", 10, row, col, [3, 4], {3: [1], 4: [1, 2]}))
    # 2. more partitions than a clean split: N=9, P=4 -> npp=3, last partition empty.
    row = np.array([0, 1, 2, 8, 8, 3, 6, 5], dtype=np.int32)
    col = np.array([8, 2, 2, 0, 7, 3, 1, 4], dtype=np.int32)
    out.append(("short9", 9, row, col, [4], {4: [1, 2]}))
    # 3. a seeded random graph, uniform.
    rng = np.random.Generator(np.random.PCG64(7))
    n = 1000
    m = 6000
    row = rng.integers(0, n, m).astype(np.int32)
    col = rng.integers(0, n, m).astype(np.int32)
    out.append(("uniform1000", n, row, col, [2, 4, 8], {4: [1, 2], 8: [1, 2, 4]}))
    # 4. power-law R-MAT, scale 12, avg degree 16 (duplicates kept, hubs present).
    n, row, col = rmat_coo(12, 16, seed=1)
    out.append(("rmat12", n, row, col, [4, 8], {4: [1, 2], 8: [1, 2, 4]}))
    return out


def ref_nnz_split(lib, rowIdx, rowPtr, nnz):
    nrows = len(rowIdx)
    cap = nnz // 32 + nrows + 1
    target = np.zeros(cap, dtype=np.int32)
    ptr = np.zeros(cap + 1, dtype=np.int32)
    nch = ctypes.c_longlong()
    plen = ctypes.c_longlong()
    ri = np.ascontiguousarray(rowIdx, dtype=np.int32)
    rp = np.ascontiguousarray(rowPtr, dtype=np.int32)
    rc = lib.ref_nnz_split(ri.ctypes.data, nrows, rp.ctypes.data, nnz, target.ctypes.data,
                           ptr.ctypes.data, cap, ctypes.byref(nch), ctypes.byref(plen))
    assert rc == 0
    return target[: nch.value].copy(), ptr[: plen.value].copy()


def main():
    ap = argparse.ArgumentParser()
    repo = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ap.add_argument("--ref-root", default=os.environ.get("COLA_REF_ROOT") or
                    os.path.join(os.path.dirname(repo), "reference"))
    args = ap.parse_args()
    par = load_module(os.path.join(args.ref_root, "prep_torch_par.py"), "ref_prep_torch_par")
    ppl = load_module(os.path.join(args.ref_root, "prep_torch_ppl.py"), "ref_prep_torch_ppl")
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_ref", "libcola_ref.so"))
    lib.ref_nnz_split.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_longlong,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                  ctypes.c_void_p, ctypes.c_void_p]
    names = ["csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l", "csc_colPtr_r", "csc_rowIdx_r", "csc_colIdx_r"]
    for name, n, row, col, plist, gsmap in cases():
        fx = {"num_nodes": np.int64(n), "row": row, "col": col, "nparts_list": np.array(plist, dtype=np.int32),
              "scipy_version": np.array(scipy.__version__)}
        coo = coo_matrix((np.ones(len(row)), (row, col)), shape=(n, n))
        g = coo.tocsr()  # prep_torch_par.py:97
        fx["global_rowPtr"] = np.array(g.indptr, dtype=np.int32)
        fx["global_colIdx"] = np.array(g.indices, dtype=np.int32)
        with tempfile.TemporaryDirectory() as td:
            cwd = os.getcwd()
            os.chdir(td)
            try:
                for P in plist:
                    par.row_partition(coo, P, name, td)
                    d = os.path.join(td, name, "GPU{}".format(P))
                    for r in range(P):
                        arrs = {}
                        for nm in names:
                            a = np.fromfile(os.path.join(d, "{}_{}_{}.bin".format(nm, P, r)), dtype=np.int32)
                            fx["P{}_r{}_{}".format(P, r, nm)] = a
                            arrs[nm] = a
                        lt, lp = ref_nnz_split(lib, arrs["csr_rowIdx_l"], arrs["csr_rowPtr_l"],
                                               len(arrs["csr_colIdx_l"]))
                        rt, rp = ref_nnz_split(lib, arrs["csc_colIdx_r"], arrs["csc_colPtr_r"],
                                               len(arrs["csc_rowIdx_r"]))
                        fx["P{}_r{}_lsplit_target".format(P, r)] = lt
                        fx["P{}_r{}_lsplit_ptr".format(P, r)] = lp
                        fx["P{}_r{}_rsplit_target".format(P, r)] = rt
                        fx["P{}_r{}_rsplit_ptr".format(P, r)] = rp
                    for gs in gsmap.get(P, []):
                        if gs >= P:
                            continue
                        ppl.row_partition(coo, name, P, gs)
                        stages = P // gs
                        dp = os.path.join(td, "storage", "SP", name, "ppl{}".format(stages))
                        for s in range(stages):
                            fx["P{}_gs{}_wg{}".format(P, gs, s)] = np.fromfile(
                                os.path.join(dp, "colIdx_{}_{}_{}.bin".format(P, stages, s)), dtype=np.int32)
                        fx["P{}_gs_list".format(P)] = np.array([x for x in gsmap.get(P, []) if x < P],
                                                               dtype=np.int32)
            finally:
                os.chdir(cwd)
        path = os.path.join(HERE, "{}.npz".format(name))
        np.savez_compressed(path, **fx)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    sys.exit(main())
