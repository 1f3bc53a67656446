"""Host preprocessing of the partitioned SpMM, backed by the native library.

Mirrors the reference's preprocessing entry points with the same names and
argument meaning:

* :func:`row_partition` -- prep_torch_par.py:24-79 (writes the same .bin files)
* :func:`serialize`     -- prep_torch_par.py:93-110 (global CSR + partitions)
* :func:`ppl_row_partition` -- prep_torch_ppl.py:24-49 (work-group lists)
* :func:`nnz_split`     -- include/dist_spmm_ppl_batch.cuh:29-56
* :func:`stage_tables`  -- src/distSpMM_ppl_batch.cu:101-193
* :func:`bin2vec`       -- include/dist_spmm_ppl_batch.cuh:7-27
* :func:`relabel_edges` -- rabbit_module/src/reorder.cpp:283-288 (apply a
  vertex ordering computed elsewhere)
plus :class:`PartitionSet` (the partitions in memory) and :func:`rmat`.
:meth:`PartitionSet.from_coo_device`, :func:`nnz_split_device` and
:func:`relabel_edges` on CUDA tensors run the same steps on the GPU (torch
tensors in, identical results out).
"""
import ctypes
import os

import numpy as np

from ._lib import GraphInfo, PartitionView, check, lib  # noqa: F401

I32 = np.int32


def _p(a):
    return None if a is None else a.ctypes.data


def _i32(a):
    return np.ascontiguousarray(a, dtype=I32)


class PartitionSet:
    """P virtual row partitions of an N x N matrix: local CSR + compacted
    remote CSC each (prep_torch_par.py:24-79), with values."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)
        v = self.part_view(0)
        self.num_nodes = v.num_nodes
        self.nparts = v.nparts
        self.nodes_per_part = v.nodes_per_part

    @classmethod
    def from_coo(cls, num_nodes, row, col, val=None, nparts=1):
        row = _i32(row)
        col = _i32(col)
        if len(row) != len(col):
            raise ValueError("row and col differ in length")
        vv = None if val is None else np.ascontiguousarray(val, dtype=np.float32)
        h = ctypes.c_void_p()
        check(lib().cola_partition_build(int(num_nodes), len(row), _p(row), _p(col), _p(vv), int(nparts),
                                         ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_coo_device(cls, num_nodes, row, col, val=None, nparts=1):
        """from_coo with the COO as CUDA tensors (int32 row/col, float32 val):
        the partitions are built on the GPU, bit-identical to from_coo."""
        import torch
        _dev_i32(row, "row")
        _dev_i32(col, "col")
        if row.numel() != col.numel() or (val is not None and val.numel() != row.numel()):
            raise ValueError("row, col and val differ in length")
        if val is not None and (not val.is_cuda or val.dtype != torch.float32 or not val.is_contiguous()):
            raise ValueError("val must be a contiguous float32 CUDA tensor")
        h = ctypes.c_void_p()
        st = torch.cuda.current_stream(row.device).cuda_stream
        check(lib().cola_partition_build_device(int(num_nodes), row.numel(), row.data_ptr(), col.data_ptr(),
                                                None if val is None else val.data_ptr(), int(nparts), st,
                                                ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def read_bin(cls, graph_dir, num_nodes, nparts):
        """Load <graph_dir>/GPU<P>/*.bin (the reference's layout; values optional)."""
        h = ctypes.c_void_p()
        check(lib().cola_partition_read_bin(os.fsencode(graph_dir), int(num_nodes), int(nparts), ctypes.byref(h)))
        return cls(h.value)

    def write_bin(self, graph_dir):
        """Write <graph_dir>/GPU<P>/*.bin as prep_torch_par.py does, plus value files."""
        os.makedirs(graph_dir, exist_ok=True)
        check(lib().cola_partition_write_bin(self._h, os.fsencode(graph_dir)))

    def part_view(self, r):
        v = PartitionView()
        check(lib().cola_partition_get(self._h, int(r), ctypes.byref(v)))
        return v

    def part(self, r):
        """Copies of partition r's arrays, keyed by the reference's file names."""
        v = self.part_view(r)

        def arr(ptr, n, dt):
            if n == 0:
                return np.zeros(0, dt)
            ct = ctypes.c_int32 if dt == np.int32 else ctypes.c_float
            return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ct)), shape=(n,)).copy()

        return {
            "csr_rowPtr_l": arr(v.csr_rowPtr_l, v.n_rowPtr_l, np.int32),
            "csr_colIdx_l": arr(v.csr_colIdx_l, v.nnz_l, np.int32),
            "csr_val_l": arr(v.csr_val_l, v.nnz_l, np.float32),
            "csr_rowIdx_l": arr(v.csr_rowIdx_l, v.n_rows_l, np.int32),
            "csc_colPtr_r": arr(v.csc_colPtr_r, v.n_colPtr_r, np.int32),
            "csc_rowIdx_r": arr(v.csc_rowIdx_r, v.nnz_r, np.int32),
            "csc_val_r": arr(v.csc_val_r, v.nnz_r, np.float32),
            "csc_colIdx_r": arr(v.csc_colIdx_r, v.n_cols_r, np.int32),
            "row_lb": v.row_lb, "row_ub": v.row_ub,
        }

    def close(self):
        if self._h is not None and self._h.value:
            lib().cola_partition_set_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h


def row_partition(COO, nGPU, graph_name, bin_path, val=None):
    """prep_torch_par.py:24-79: partition a scipy COO matrix (or any object with
    .row/.col/.shape) into nGPU row blocks and write
    <bin_path>/<graph_name>/GPU<nGPU>/*_<nGPU>_<r>.bin.  Values: COO.data when
    `val` is None and the matrix carries data, written as csr_val_l/csc_val_r."""
    if val is None and getattr(COO, "data", None) is not None:
        val = COO.data
    ps = PartitionSet.from_coo(COO.shape[0], COO.row, COO.col, val, nGPU)
    ps.write_bin(os.path.join(bin_path, graph_name))
    return ps


def global_csr(num_nodes, row, col, val=None):
    """prep_torch_par.py:93-101: global CSR (rowPtr, colIdx, val) of the COO."""
    row = _i32(row)
    col = _i32(col)
    vin = None if val is None else np.ascontiguousarray(val, np.float32)
    rp = np.zeros(num_nodes + 1, I32)
    ci = np.zeros(max(len(row), 1), I32)
    vo = np.zeros(max(len(row), 1), np.float32)
    m = ctypes.c_int64()
    check(lib().cola_global_csr(int(num_nodes), len(row), _p(row), _p(col), _p(vin), _p(rp), _p(ci), _p(vo),
                                ctypes.byref(m)))
    return rp, ci[: m.value].copy(), vo[: m.value].copy()


def serialize(COO, graph_name, bin_path, nGPU_list):
    """prep_torch_par.py:93-110: global_rowPtr.bin / global_colIdx.bin plus the
    partitions for every P in nGPU_list."""
    d = os.path.join(bin_path, graph_name)
    os.makedirs(d, exist_ok=True)
    rp, ci, _ = global_csr(COO.shape[0], COO.row, COO.col)
    write_bin(os.path.join(d, "global_rowPtr.bin"), rp)
    write_bin(os.path.join(d, "global_colIdx.bin"), ci)
    return {P: row_partition(COO, P, graph_name, bin_path) for P in nGPU_list}


def workgroup_cols(num_nodes, row, col, nparts, group_size, stage):
    """prep_torch_ppl.py:24-49 for one work group."""
    row = _i32(row)
    col = _i32(col)
    out = np.zeros(max(int(num_nodes), 1), I32)
    n = ctypes.c_int64()
    check(lib().cola_workgroup_cols(int(num_nodes), len(row), _p(row), _p(col), int(nparts), int(group_size),
                                    int(stage), _p(out), ctypes.byref(n)))
    return out[: n.value].copy()


def ppl_row_partition(COO, graph_name, nGPU, gs, bin_path="./storage/SP"):
    """prep_torch_ppl.py:24-49: writes <bin_path>/<graph>/ppl<stages>/colIdx_<nGPU>_<stages>_<s>.bin."""
    stages = nGPU // gs
    d = os.path.join(bin_path, graph_name, "ppl{}".format(stages))
    os.makedirs(d, exist_ok=True)
    lists = []
    for s in range(stages):
        w = workgroup_cols(COO.shape[0], COO.row, COO.col, nGPU, gs, s)
        write_bin(os.path.join(d, "colIdx_{}_{}_{}.bin".format(nGPU, stages, s)), w)
        lists.append(w)
    return lists


def nnz_split(rowIdx, rowPtr, nnz):
    """include/dist_spmm_ppl_batch.cuh:29-56 -> (target, ptr)."""
    rowIdx = _i32(rowIdx)
    rowPtr = _i32(rowPtr)
    n = ctypes.c_int64()
    check(lib().cola_nnz_split(_p(rowIdx), len(rowIdx), _p(rowPtr), int(nnz), None, None, 0, ctypes.byref(n)))
    target = np.zeros(max(n.value, 1), I32)
    ptr = np.zeros(n.value + 1, I32)
    check(lib().cola_nnz_split(_p(rowIdx), len(rowIdx), _p(rowPtr), int(nnz), _p(target), _p(ptr), n.value,
                               ctypes.byref(n)))
    return target[: n.value].copy(), (ptr.copy() if len(rowIdx) else np.zeros(0, I32))


def _dev_i32(t, name):
    import torch
    if not t.is_cuda or t.dtype != torch.int32 or not t.is_contiguous():
        raise ValueError("{} must be a contiguous int32 CUDA tensor".format(name))


def nnz_split_device(rowIdx, rowPtr, nnz):
    """nnz_split on CUDA tensors (computed on the GPU) -> (target, ptr) tensors."""
    import torch
    _dev_i32(rowIdx, "rowIdx")
    _dev_i32(rowPtr, "rowPtr")
    st = torch.cuda.current_stream(rowIdx.device).cuda_stream
    n = ctypes.c_int64()
    nrows = rowIdx.numel()
    check(lib().cola_nnz_split_device(rowIdx.data_ptr(), nrows, rowPtr.data_ptr(), int(nnz), None, None, 0,
                                      ctypes.byref(n), st))
    target = torch.empty(max(n.value, 1), dtype=torch.int32, device=rowIdx.device)
    ptr = torch.empty(n.value + 1, dtype=torch.int32, device=rowIdx.device)
    if nrows:
        check(lib().cola_nnz_split_device(rowIdx.data_ptr(), nrows, rowPtr.data_ptr(), int(nnz), target.data_ptr(),
                                          ptr.data_ptr(), n.value, ctypes.byref(n), st))
        return target[: n.value], ptr
    return target[:0], ptr[:0]


def relabel_edges(num_nodes, row, col, mapping):
    """rabbit_module/src/reorder.cpp:283-288: (mapping[row], mapping[col]) for an
    old -> new vertex mapping computed elsewhere.  numpy arrays are relabelled
    on the host, CUDA tensors on the GPU."""
    if hasattr(row, "is_cuda") and row.is_cuda:
        import torch
        _dev_i32(row, "row")
        _dev_i32(col, "col")
        _dev_i32(mapping, "mapping")
        out_r = torch.empty_like(row)
        out_c = torch.empty_like(col)
        st = torch.cuda.current_stream(row.device).cuda_stream
        check(lib().cola_relabel_edges_device(int(num_nodes), row.numel(), row.data_ptr(), col.data_ptr(),
                                              mapping.data_ptr(), out_r.data_ptr(), out_c.data_ptr(), st))
        return out_r, out_c
    row = _i32(row)
    col = _i32(col)
    mapping = _i32(mapping)
    if len(row) != len(col):
        raise ValueError("row and col differ in length")
    out_r = np.empty_like(row)
    out_c = np.empty_like(col)
    check(lib().cola_relabel_edges(int(num_nodes), len(row), _p(row), _p(col), _p(mapping), _p(out_r), _p(out_c)))
    return out_r, out_c


def community_order(num_nodes, row, col):
    """The reordering step run before partitioning (rabbit_order_write.py:48-55;
    cola_community_order): communities by incremental aggregation, numbered
    community by community.  Returns (mapping old -> new, communities); with
    relabel_edges it gives the reordered edge list rabbit.reorder returns."""
    row = _i32(row)
    col = _i32(col)
    if len(row) != len(col):
        raise ValueError("row and col differ in length")
    mapping = np.empty(int(num_nodes), np.int32)
    nc = ctypes.c_int64()
    check(lib().cola_community_order(int(num_nodes), len(row), _p(row), _p(col), _p(mapping), ctypes.byref(nc)))
    return mapping, nc.value


def stage_tables(me, nranks, group_size, num_nodes, csc_colIdx_zip_r, nchunks_l, wg_lists):
    """src/distSpMM_ppl_batch.cu:101-193 for PE `me`."""
    nstages = nranks // group_size
    zr = _i32(csc_colIdx_zip_r)
    if wg_lists:
        wg = _i32(np.concatenate([np.asarray(w, I32) for w in wg_lists]))
        wg_off = np.zeros(len(wg_lists) + 1, np.int64)
        wg_off[1:] = np.cumsum([len(w) for w in wg_lists])
    else:
        wg, wg_off = None, None
    lo = np.zeros(2 * nstages, I32)
    ro = np.zeros(2 * nstages, I32)
    po = np.zeros(2 * nstages, I32)
    idx_cap = len(zr) + 1
    idx = np.zeros(idx_cap, I32)
    idx_off = np.zeros(nstages, np.int64)
    put_cap = max(int(num_nodes), 1)
    put = np.zeros(put_cap, I32)
    put_off = np.zeros(nstages, np.int64)
    check(lib().cola_stage_tables(int(me), int(nranks), int(group_size), int(num_nodes), _p(zr), len(zr),
                                  int(nchunks_l), _p(wg), _p(wg_off), _p(lo), _p(ro), _p(po), _p(idx),
                                  _p(idx_off), idx_cap, _p(put), _p(put_off), put_cap))
    idx_lists = [idx[(idx_off[i - 1] if i > 1 else 0): idx_off[i]].copy() for i in range(1, nstages)]
    put_lists = [put[put_off[i]: put_off[i + 1]].copy() for i in range(nstages - 1)]
    return {"local_offset": lo, "remote_offset": ro, "put_offset": po, "idx_ppl": idx_lists,
            "put_colIdx": put_lists}


def bin2vec(path, dtype=np.int32):
    """include/dist_spmm_ppl_batch.cuh:7-27 (64-bit sizes)."""
    L = lib()
    rd = L.cola_bin_read_i32 if np.dtype(dtype) == np.int32 else L.cola_bin_read_f32
    n = ctypes.c_int64()
    check(rd(os.fsencode(path), None, 0, ctypes.byref(n)))
    out = np.zeros(max(n.value, 1), dtype)
    check(rd(os.fsencode(path), _p(out), n.value, ctypes.byref(n)))
    return out[: n.value]


def write_bin(path, arr):
    arr = np.ascontiguousarray(arr)
    L = lib()
    if arr.dtype == np.int32:
        check(L.cola_bin_write_i32(os.fsencode(path), _p(arr), arr.size))
    elif arr.dtype == np.float32:
        check(L.cola_bin_write_f32(os.fsencode(path), _p(arr), arr.size))
    else:
        raise TypeError("write_bin: int32 or float32 only, got {}".format(arr.dtype))


VALUES_NONE = 0
VALUES_ROW_NORMALISED = 1   # 1/deg(row)
VALUES_SYM_NORMALISED = 2   # D^-1/2 A D^-1/2


def rmat(scale, avg_degree, seed, a=0.57, b=0.19, c=0.19, self_loops=False, values=VALUES_SYM_NORMALISED):
    """Seeded R-MAT graph: ceil(deg*N/2) draws, self-loops dropped, symmetrised,
    deduplicated, optional self-loops; COO sorted by (row, col).
    Returns (num_nodes, row, col, val)."""
    n = 1 << int(scale)
    cap = 2 * int(np.ceil(avg_degree * n / 2.0)) + (n if self_loops else 0)
    row = np.zeros(cap, I32)
    col = np.zeros(cap, I32)
    val = np.zeros(cap, np.float32)
    m = ctypes.c_int64()
    check(lib().cola_rmat_generate(int(scale), float(avg_degree), float(a), float(b), float(c), int(seed),
                                   1 if self_loops else 0, int(values), _p(row), _p(col), _p(val), cap,
                                   ctypes.byref(m)))
    k = m.value
    return n, row[:k].copy(), col[:k].copy(), val[:k].copy()
