"""ctypes binding of the CPU oracle (oracle/cola_oracle.c) and of the reference
library built from the reference tree (oracle/_ref/libcola_ref.so).

TEST INFRASTRUCTURE.  Imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, as the checker or the timed CPU
baseline.  The cola_b200 package never imports this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcola_ref.so")

_lib = None
_ref = None

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64


def _ptr(a):
    return None if a is None else a.ctypes.data


def lib():
    """The oracle library (built by `make -C oracle oracle`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle library missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_partition_count.restype = I64
        L.orc_partition_count.argtypes = [I32, I64, P, I32, I32]
        L.orc_row_partition.argtypes = [I32, I64, P, P, P, I32, I32] + [P] * 8 + [P]
        L.orc_global_csr.argtypes = [I32, I64, P, P, P, P, P, P, P]
        L.orc_workgroup_cols.argtypes = [I32, I64, P, P, I32, I32, I32, P, P]
        L.orc_nnz_split.argtypes = [P, I64, P, I64, P, P, I64, P, P]
        L.orc_stage_tables.argtypes = [I32, I32, I32, I32, P, I64, I64, P, P, P, P, P, P, P, I64, P, P, I64]
        L.orc_spmm_csr_f64.argtypes = [I64, P, P, P, P, I64, I32, P, I64]
        L.orc_spmm_csr_f64_bf16x.argtypes = [I64, P, P, P, P, I64, I32, P, I64]
        L.orc_spmm_rows_f32_ordered.argtypes = [I64, P, P, P, P, I64, I32, I64, I64, P, I64]
        L.orc_spmm_partition_f64.argtypes = [I32, I32, P, P, P, P, I64, P, P, P, P, I64, P, I64, I32, P, I64]
        L.orc_spmm_partitions_f32_omp.argtypes = [I32, I32] + [P] * 15 + [I64, I32, P, I64, I32]
        L.orc_max_threads.restype = I32
        L.orc_rmat_generate.argtypes = [I32, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_uint64, I32, I32, P, P, P, I64, P]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    """The reference's own code compiled from its tree (oracle/_ref)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference library missing: run `make -C oracle ref` where the reference tree exists")
        L = ctypes.CDLL(REF_SO)
        L.ref_set_pe.argtypes = [ctypes.c_int, ctypes.c_longlong, P]
        spmm_args = [ctypes.c_int, ctypes.c_int, P, P] + [P] * 8 + [ctypes.c_int] * 7 + [P]
        L.ref_ppl0_batch_spmm.argtypes = spmm_args
        L.ref_ppl0_batch_spmm_seq.argtypes = spmm_args
        L.ref_ppl0_batch_buffer_spmm.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P] + [P] * 8 + \
            [ctypes.c_int] * 7 + [P]
        L.ref_ppl_batch_spmm.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P, P, P] + [ctypes.c_int] * 5 + \
            [P] + [ctypes.c_int] * 5 + [P]
        L.ref_batching_data_ppl.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P]
        L.ref_nnz_split.argtypes = [P, ctypes.c_longlong, P, ctypes.c_longlong, P, P, ctypes.c_longlong, P, P]
        L.ref_sag_reference_host.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P, P, ctypes.c_int]
        L.ref_sag_reference_host.restype = None
        _ref = L
    return _ref


# --------------------------------------------------------------------------
# preprocessing restatements
# --------------------------------------------------------------------------
def row_partition(num_nodes, row, col, nparts, r, val=None):
    """prep_torch_par.py:24-79 for partition r (+ values in the same order)."""
    L = lib()
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    if val is not None:
        val = np.ascontiguousarray(val, dtype=np.float32)
    cap = int(L.orc_partition_count(num_nodes, len(row), _ptr(row), nparts, r))
    l_rowPtr = np.zeros(cap + 1, np.int32)
    l_colIdx = np.zeros(cap, np.int32)
    l_val = np.zeros(cap, np.float32)
    l_rowIdx = np.zeros(cap, np.int32)
    r_colPtr = np.zeros(cap + 1, np.int32)
    r_rowIdx = np.zeros(cap, np.int32)
    r_val = np.zeros(cap, np.float32)
    r_colIdx = np.zeros(cap, np.int32)
    counts = np.zeros(6, np.int64)
    rc = L.orc_row_partition(num_nodes, len(row), _ptr(row), _ptr(col), _ptr(val), nparts, r,
                             _ptr(l_rowPtr), _ptr(l_colIdx), _ptr(l_val), _ptr(l_rowIdx),
                             _ptr(r_colPtr), _ptr(r_rowIdx), _ptr(r_val), _ptr(r_colIdx), _ptr(counts))
    if rc != 0:
        raise RuntimeError("orc_row_partition failed")
    c = counts
    return {
        "csr_rowPtr_l": l_rowPtr[: c[0]], "csr_colIdx_l": l_colIdx[: c[1]], "csr_val_l": l_val[: c[1]],
        "csr_rowIdx_l": l_rowIdx[: c[2]], "csc_colPtr_r": r_colPtr[: c[3]], "csc_rowIdx_r": r_rowIdx[: c[4]],
        "csc_val_r": r_val[: c[4]], "csc_colIdx_r": r_colIdx[: c[5]],
    }


def relabel_edges(row, col, mapping):
    """rabbit_module/src/reorder.cpp:283-288: out_row[i] = mapping[src],
    out_col[i] = mapping[dst] for the old -> new id mapping."""
    mapping = np.asarray(mapping)
    return mapping[np.asarray(row)].astype(np.int32), mapping[np.asarray(col)].astype(np.int32)


def global_csr(num_nodes, row, col, val=None):
    """prep_torch_par.py:93-101 (A.tocsr())."""
    L = lib()
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    if val is not None:
        val = np.ascontiguousarray(val, dtype=np.float32)
    rp = np.zeros(num_nodes + 1, np.int32)
    ci = np.zeros(max(len(row), 1), np.int32)
    vo = np.zeros(max(len(row), 1), np.float32)
    m = ctypes.c_int64()
    if L.orc_global_csr(num_nodes, len(row), _ptr(row), _ptr(col), _ptr(val), _ptr(rp), _ptr(ci), _ptr(vo),
                        ctypes.byref(m)) != 0:
        raise RuntimeError("orc_global_csr failed")
    return rp, ci[: m.value], vo[: m.value]


def rmat(scale, avg_degree, seed, a=0.57, b=0.19, c=0.19, self_loops=False, values=2):
    """The seeded R-MAT graph the library's cola_rmat_generate defines,
    restated in C (orc_rmat_generate).  values: 0 ones, 1 1/deg(row),
    2 D^-1/2 A D^-1/2.  Returns (num_nodes, row, col, val)."""
    L = lib()
    cnt = ctypes.c_int64()
    args = (int(scale), float(avg_degree), float(a), float(b), float(c), ctypes.c_uint64(int(seed)),
            1 if self_loops else 0, int(values))
    if L.orc_rmat_generate(*args, None, None, None, 0, ctypes.byref(cnt)) != 0:
        raise RuntimeError("orc_rmat_generate failed")
    m = cnt.value
    row = np.zeros(max(m, 1), np.int32)
    col = np.zeros(max(m, 1), np.int32)
    val = np.zeros(max(m, 1), np.float32)
    if L.orc_rmat_generate(*args, _ptr(row), _ptr(col), _ptr(val), m, ctypes.byref(cnt)) != 0:
        raise RuntimeError("orc_rmat_generate failed")
    return 1 << int(scale), row[:m], col[:m], val[:m]


def workgroup_cols(num_nodes, row, col, nparts, gs, stage):
    """prep_torch_ppl.py:24-49 for one work group."""
    L = lib()
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    out = np.zeros(max(num_nodes, 1), np.int32)
    cnt = ctypes.c_int64()
    if L.orc_workgroup_cols(num_nodes, len(row), _ptr(row), _ptr(col), nparts, gs, stage, _ptr(out),
                            ctypes.byref(cnt)) != 0:
        raise RuntimeError("orc_workgroup_cols failed")
    return out[: cnt.value].copy()


def nnz_split(rowIdx, rowPtr, nnz):
    """include/dist_spmm_ppl_batch.cuh:29-56.  Returns (target, ptr)."""
    L = lib()
    rowIdx = np.ascontiguousarray(rowIdx, dtype=np.int32)
    rowPtr = np.ascontiguousarray(rowPtr, dtype=np.int32)
    cap = nnz // 32 + len(rowIdx) + 1
    target = np.zeros(cap, np.int32)
    ptr = np.zeros(cap + 1, np.int32)
    nch = ctypes.c_int64()
    plen = ctypes.c_int64()
    if L.orc_nnz_split(_ptr(rowIdx), len(rowIdx), _ptr(rowPtr), nnz, _ptr(target), _ptr(ptr), cap,
                       ctypes.byref(nch), ctypes.byref(plen)) != 0:
        raise RuntimeError("orc_nnz_split failed")
    return target[: nch.value].copy(), ptr[: plen.value].copy()


def stage_tables(me, nranks, gs, num_nodes, csc_colIdx_zip_r, nchunks_l, wg_lists):
    """src/distSpMM_ppl_batch.cu:101-193.  wg_lists: list of work-group column arrays."""
    L = lib()
    nstages = nranks // gs
    zr = np.ascontiguousarray(csc_colIdx_zip_r, dtype=np.int32)
    if wg_lists:
        wg = np.ascontiguousarray(np.concatenate([np.asarray(w, np.int32) for w in wg_lists]), dtype=np.int32)
        wg_off = np.zeros(len(wg_lists) + 1, np.int64)
        wg_off[1:] = np.cumsum([len(w) for w in wg_lists])
    else:
        wg = np.zeros(1, np.int32)
        wg_off = np.zeros(1, np.int64)
    lo = np.zeros(2 * nstages, np.int32)
    ro = np.zeros(2 * nstages, np.int32)
    po = np.zeros(2 * nstages, np.int32)
    idx_cap = len(zr) + 1
    idx = np.zeros(idx_cap, np.int32)
    idx_off = np.zeros(nstages + 1, np.int64)
    put_cap = max(num_nodes, 1)
    put = np.zeros(put_cap, np.int32)
    put_off = np.zeros(nstages + 1, np.int64)
    rc = L.orc_stage_tables(me, nranks, gs, num_nodes, _ptr(zr), len(zr), nchunks_l,
                            _ptr(wg) if wg_lists else None, _ptr(wg_off) if wg_lists else None,
                            _ptr(lo), _ptr(ro), _ptr(po), _ptr(idx), _ptr(idx_off), idx_cap,
                            _ptr(put), _ptr(put_off), put_cap)
    if rc != 0:
        raise RuntimeError("orc_stage_tables failed")
    idx_lists = [idx[idx_off[i - 1] if i > 1 else 0: idx_off[i]].copy() for i in range(1, nstages)]
    put_lists = [put[put_off[i]: put_off[i + 1]].copy() for i in range(nstages - 1)]
    return {"local_offset": lo, "remote_offset": ro, "put_offset": po, "idx_ppl": idx_lists,
            "put_colIdx": put_lists}


# --------------------------------------------------------------------------
# FP64 SpMM oracles
# --------------------------------------------------------------------------
def spmm_csr_f64(rowPtr, colIdx, val, X):
    """Y = A X in double over a CSR; X float32 (n x K) or bf16 bits (uint16)."""
    L = lib()
    nrows = len(rowPtr) - 1
    K = X.shape[1]
    Y = np.zeros((nrows, K), np.float64)
    rowPtr = np.ascontiguousarray(rowPtr, np.int32)
    colIdx = np.ascontiguousarray(colIdx, np.int32)
    val = None if val is None else np.ascontiguousarray(val, np.float32)
    X = np.ascontiguousarray(X)
    if X.dtype == np.float32:
        L.orc_spmm_csr_f64(nrows, _ptr(rowPtr), _ptr(colIdx), _ptr(val), _ptr(X), X.shape[1], K, _ptr(Y), K)
    elif X.dtype == np.uint16:
        L.orc_spmm_csr_f64_bf16x(nrows, _ptr(rowPtr), _ptr(colIdx), _ptr(val), _ptr(X), X.shape[1], K, _ptr(Y), K)
    else:
        raise TypeError(X.dtype)
    return Y


def spmm_rows_f32_ordered(rowPtr, colIdx, val, X, hub_threshold=512, hub_segment=512):
    """FP32 Y = A X summed in the row-major schedule's fixed order (fused
    multiply-adds in CSR order per row; rows over hub_threshold entries as
    hub_segment-entry segments added by a binary counter), to be compared bit
    for bit.  X float32 (n x K)."""
    L = lib()
    nrows = len(rowPtr) - 1
    X = np.ascontiguousarray(X, np.float32)
    K = X.shape[1]
    Y = np.zeros((nrows, K), np.float32)
    rowPtr = np.ascontiguousarray(rowPtr, np.int64)
    colIdx = np.ascontiguousarray(colIdx, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    if L.orc_spmm_rows_f32_ordered(nrows, _ptr(rowPtr), _ptr(colIdx), _ptr(val), _ptr(X), K, K,
                                   int(hub_threshold), int(hub_segment), _ptr(Y), K) != 0:
        raise RuntimeError("orc_spmm_rows_f32_ordered failed")
    return Y


def spmm_partition_f64(part, npp, lz, rz, X):
    """One partition from its split arrays (ppl0_batch_SpMM_kernel restated).
    lz = (ptr, colIdx, rowIdx_zip, val), rz = (ptr, rowIdx, colIdx_zip, val)."""
    L = lib()
    K = X.shape[1]
    Y = np.zeros((npp, K), np.float64)
    lz = [np.ascontiguousarray(a, np.float32 if i == 3 else np.int32) for i, a in enumerate(lz)]
    rz = [np.ascontiguousarray(a, np.float32 if i == 3 else np.int32) for i, a in enumerate(rz)]
    X = np.ascontiguousarray(X, np.float32)
    L.orc_spmm_partition_f64(part, npp, _ptr(lz[0]), _ptr(lz[1]), _ptr(lz[2]), _ptr(lz[3]), len(lz[2]),
                             _ptr(rz[0]), _ptr(rz[1]), _ptr(rz[2]), _ptr(rz[3]), len(rz[2]),
                             _ptr(X), X.shape[1], K, _ptr(Y), K)
    return Y


def partitions_f32_omp(parts, npp, X):
    """The OpenMP FP32 loop over the partitions (orc_spmm_partitions_f32_omp:
    each partition's split local CSR chunks and remote CSC chunks, as
    nnz_split makes them, one thread per partition).  parts: the partition
    dicts (csr_* / csc_* arrays with values).  Returns run(nthreads) -> Y
    ((P * npp) x K, FP32); the arrays are prepared once."""
    L = lib()
    P = len(parts)
    K = X.shape[1]
    cols = {k: [] for k in ("l_ptr", "l_col", "l_val", "l_row", "r_ptr", "r_row", "r_val", "r_col")}
    for p in parts:
        lt, lq = nnz_split(p["csr_rowIdx_l"], p["csr_rowPtr_l"], len(p["csr_colIdx_l"]))
        rt, rq = nnz_split(p["csc_colIdx_r"], p["csc_colPtr_r"], len(p["csc_rowIdx_r"]))
        z = np.zeros(1, np.int32)
        for k, a in (("l_ptr", lq if len(lq) else z), ("l_col", p["csr_colIdx_l"]), ("l_val", p["csr_val_l"]),
                     ("l_row", lt), ("r_ptr", rq if len(rq) else z), ("r_row", p["csc_rowIdx_r"]),
                     ("r_val", p["csc_val_r"]), ("r_col", rt)):
            cols[k].append(np.ascontiguousarray(a))
    arr = {}
    for k, v in cols.items():
        dt = np.float32 if k.endswith("val") else np.int32
        arr[k] = (np.ascontiguousarray(np.concatenate(v).astype(dt)),
                  np.concatenate([[0], np.cumsum([len(x) for x in v])]).astype(np.int64))
    Xp = np.zeros((P * npp, K), np.float32)
    Xp[:X.shape[0]] = X
    Y = np.empty((P * npp, K), np.float32)

    def run(nthreads):
        L.orc_spmm_partitions_f32_omp(
            P, npp, _ptr(arr["l_ptr"][0]), _ptr(arr["l_ptr"][1]), _ptr(arr["l_col"][0]), _ptr(arr["l_val"][0]),
            _ptr(arr["l_col"][1]), _ptr(arr["l_row"][0]), _ptr(arr["l_row"][1]), _ptr(arr["r_ptr"][0]),
            _ptr(arr["r_ptr"][1]), _ptr(arr["r_row"][0]), _ptr(arr["r_val"][0]), _ptr(arr["r_row"][1]),
            _ptr(arr["r_col"][0]), _ptr(arr["r_col"][1]), _ptr(Xp), K, K, _ptr(Y), K, int(nthreads))
        return Y
    return run


def rel_frobenius(y, ref):
    """||y - ref||_F / ||ref||_F in double."""
    y = np.asarray(y, np.float64)
    ref = np.asarray(ref, np.float64)
    den = np.linalg.norm(ref)
    num = np.linalg.norm(y - ref)
    return float(num / den) if den > 0 else float(num)
