"""Device side of the partitioned SpMM: the graph handle and the kernel-level
launchers, with the reference's names (include/dist_spmm_ppl_batch.cuh).

Dense operands are torch CUDA tensors (row-major); torch only supplies device
memory and streams.  Every call goes through the native library; nothing here
computes on the host.
"""
import ctypes

import torch

from . import _lib
from ._lib import (BFLOAT16, FLOAT32, SCHEDULE_AUTO, SCHEDULE_BUFFER, SCHEDULE_FUSED,  # noqa: F401
                   SCHEDULE_PIPELINE, SCHEDULE_ROWS, GraphInfo, SpmmOpts, UploadOpts, ZipView, check, lib)

_DT = {torch.float32: FLOAT32, torch.bfloat16: BFLOAT16}


def _stream(stream):
    if stream is None:
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _dense(t, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("{} must be a CUDA tensor".format(name))
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError("{} must be 2-D row-major (stride(1) == 1)".format(name))
    if t.dtype not in _DT:
        raise TypeError("{} must be float32 or bfloat16, got {}".format(name, t.dtype))
    return t


class Graph:
    """All P virtual partitions of one matrix resident on the current device
    (the d_csr_zip / d_csc_zip holders of include/sparse_data.h for every PE,
    plus the pipelined schedule's stage tables)."""

    def __init__(self, pset, if_split=True, group_size=None, row_view=True, hub_threshold=0, hub_segment=0,
                 task_entries=0, stream=None):
        o = UploadOpts()
        o.if_split = 1 if if_split else 0
        o.group_size = int(group_size or 0)
        o.no_row_view = 0 if row_view else 1
        o.hub_threshold = int(hub_threshold)
        o.hub_segment = int(hub_segment)
        o.task_entries = int(task_entries)
        h = ctypes.c_void_p()
        check(lib().cola_graph_upload(pset.handle, ctypes.byref(o), ctypes.byref(h), _stream(stream)))
        self._h = h
        self.info = self.get_info()
        self.num_nodes = self.info.num_nodes
        self.nparts = self.info.nparts
        self.nodes_per_part = self.info.nodes_per_part

    @classmethod
    def from_coo_device(cls, num_nodes, row, col, val=None, nparts=1, hub_threshold=0, hub_segment=0,
                        task_entries=0, stream=None):
        """The graph built on the GPU straight from a COO in CUDA tensors
        (int32 row/col, optional float32 val): the row view only (the
        row-major schedule), identical to Graph(PartitionSet.from_coo(...))'s."""
        for t, name in ((row, "row"), (col, "col")):
            if not t.is_cuda or t.dtype != torch.int32 or not t.is_contiguous():
                raise ValueError("{} must be a contiguous int32 CUDA tensor".format(name))
        if row.numel() != col.numel() or (val is not None and val.numel() != row.numel()):
            raise ValueError("row, col and val differ in length")
        if val is not None and (not val.is_cuda or val.dtype != torch.float32 or not val.is_contiguous()):
            raise ValueError("val must be a contiguous float32 CUDA tensor")
        o = UploadOpts()
        o.if_split = 1
        o.hub_threshold = int(hub_threshold)
        o.hub_segment = int(hub_segment)
        o.task_entries = int(task_entries)
        h = ctypes.c_void_p()
        check(lib().cola_graph_build_device(int(num_nodes), row.numel(), _ptr(row), _ptr(col), _ptr(val),
                                            int(nparts), ctypes.byref(o), _stream(stream), ctypes.byref(h)))
        g = cls.__new__(cls)
        g._h = h
        g.info = g.get_info()
        g.num_nodes = g.info.num_nodes
        g.nparts = g.info.nparts
        g.nodes_per_part = g.info.nodes_per_part
        return g

    def get_info(self):
        i = GraphInfo()
        check(lib().cola_graph_get_info(self._h, ctypes.byref(i)))
        return i

    def zip_view(self, part):
        z = ZipView()
        check(lib().cola_graph_zip_view(self._h, int(part), ctypes.byref(z)))
        return z

    def spmm(self, X, Y=None, out_dtype=None, accumulate=False, schedule=SCHEDULE_AUTO, gather_batch_rows=0,
             unroll=0, min_blocks=0, k_tile=0, stream=None):
        """Y = A X (Y += A X with accumulate).  X: (>= N) x K CUDA tensor,
        float32 or bfloat16; Y: N x K float32 or bfloat16 (allocated when None).
        unroll, min_blocks and k_tile tune the row-major schedule (0 = the
        library's choice; every choice gives the same bits).  Calls on one
        graph share its work-item counters and hub workspace: issue them on
        one stream (or order the streams), not concurrently."""
        _dense(X, "X")
        K = X.shape[1]
        if X.shape[0] < self.num_nodes:
            raise ValueError("X has {} rows, the graph {}".format(X.shape[0], self.num_nodes))
        if Y is None:
            Y = torch.empty((self.num_nodes, K), dtype=out_dtype or torch.float32, device=X.device)
        _dense(Y, "Y")
        if Y.shape[0] < self.num_nodes or Y.shape[1] != K:
            raise ValueError("Y must be {} x {}".format(self.num_nodes, K))
        o = SpmmOpts()
        o.accumulate = 1 if accumulate else 0
        o.schedule = int(schedule)
        o.gather_batch_rows = int(gather_batch_rows)
        o.unroll = int(unroll)
        o.min_blocks = int(min_blocks)
        o.k_tile = int(k_tile)
        check(lib().cola_spmm(self._h, _ptr(X), _DT[X.dtype], X.stride(0), _ptr(Y), _DT[Y.dtype], Y.stride(0), K,
                              ctypes.byref(o), _stream(stream)))
        return Y

    def spmm_host(self, X, Y, schedule=SCHEDULE_AUTO, stream=None):
        """cola_spmm_host: Y = A X with X and Y host tensors (pinned for
        overlap); returns at once, the result is in Y after sync_host()."""
        for t, name in ((X, "X"), (Y, "Y")):
            if not isinstance(t, torch.Tensor) or t.is_cuda or t.dim() != 2 or t.stride(1) != 1:
                raise ValueError("{} must be a 2-D row-major host tensor".format(name))
            if t.dtype not in _DT:
                raise TypeError("{} must be float32 or bfloat16".format(name))
        K = X.shape[1]
        if X.shape[0] < self.num_nodes or Y.shape[0] < self.num_nodes or Y.shape[1] != K:
            raise ValueError("X must have >= N rows and Y must be N x K")
        o = SpmmOpts()
        o.schedule = int(schedule)
        check(lib().cola_spmm_host(self._h, _ptr(X), _DT[X.dtype], X.stride(0), _ptr(Y), _DT[Y.dtype], Y.stride(0),
                                   K, ctypes.byref(o), _stream(stream)))
        return Y

    def sync_host(self):
        """Wait for every spmm_host call made on this graph."""
        check(lib().cola_spmm_host_sync(self._h))

    def join_host(self, stream=None):
        """Make `stream` wait for every spmm_host call made so far."""
        check(lib().cola_spmm_host_join(self._h, _stream(stream)))

    def autotune(self, X, Y=None, out_dtype=None, schedule=SCHEDULE_AUTO, reps=5, cache_path=None, stream=None):
        """cola_spmm_autotune on these operands: returns (options dict for
        spmm(), best ms, whether it came from the cache file)."""
        _dense(X, "X")
        K = X.shape[1]
        if Y is None:
            Y = torch.empty((self.num_nodes, K), dtype=out_dtype or torch.float32, device=X.device)
        _dense(Y, "Y")
        o = SpmmOpts()
        ms = ctypes.c_float()
        hit = ctypes.c_int32()
        check(lib().cola_spmm_autotune(self._h, _ptr(X), _DT[X.dtype], X.stride(0), _ptr(Y), _DT[Y.dtype],
                                       Y.stride(0), K, int(schedule), int(reps),
                                       None if cache_path is None else str(cache_path).encode(), _stream(stream),
                                       ctypes.byref(o), ctypes.byref(ms), ctypes.byref(hit)))
        opts = dict(schedule=o.schedule, k_tile=o.k_tile, unroll=o.unroll, min_blocks=o.min_blocks,
                    gather_batch_rows=o.gather_batch_rows)
        return opts, ms.value, bool(hit.value)

    def close(self):
        if self._h is not None and self._h.value:
            lib().cola_graph_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h


# ---------------------------------------------------------------------------
# kernel-level launchers (reference names, same argument meaning)
# ---------------------------------------------------------------------------
def ppl0_batch_SpMM(output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r,
                    csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb, remote_col_lb, local_row_num,
                    remote_col_num, dim, nodesPerPE, peid, stream=None):
    """include/dist_spmm_ppl_batch.cuh:202-245.  Pointer arguments: torch
    tensors or raw device addresses (int)."""
    a = [_any(x) for x in (output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r,
                           csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r)]
    check(lib().cola_ppl0_batch_spmm(*a, int(local_row_lb), int(remote_col_lb), int(local_row_num),
                                     int(remote_col_num), int(dim), int(nodesPerPE), int(peid), _stream(stream)))


def ppl0_batch_SpMM_seq(output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r,
                        csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb, remote_col_lb, local_row_num,
                        remote_col_num, dim, nodesPerPE, peid, stream=None):
    """include/dist_spmm_ppl_batch.cuh:543-587."""
    a = [_any(x) for x in (output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r,
                           csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r)]
    check(lib().cola_ppl0_batch_spmm_seq(*a, int(local_row_lb), int(remote_col_lb), int(local_row_num),
                                         int(remote_col_num), int(dim), int(nodesPerPE), int(peid),
                                         _stream(stream)))


def ppl0_batch_buffer_SpMM(output, input, comm_buffer, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l,
                           csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb, remote_col_lb,
                           local_row_num, remote_col_num, dim, nodesPerPE, peid, stream=None):
    """include/dist_spmm_ppl_batch.cuh:373-417."""
    a = [_any(x) for x in (output, input, comm_buffer, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l,
                           csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r)]
    check(lib().cola_ppl0_batch_buffer_spmm(*a, int(local_row_lb), int(remote_col_lb), int(local_row_num),
                                            int(remote_col_num), int(dim), int(nodesPerPE), int(peid),
                                            _stream(stream)))


def ppl_batch_SpMM(output, input, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_col_lb,
                   local_col_ub, remote_col_lb, remote_col_ub, stage, idx_ppl, dim, nodesPerPE, group_size,
                   group_offset, peid, stream=None):
    """include/dist_spmm_ppl_batch.cuh:709-760."""
    a = [_any(x) for x in (output, input, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r)]
    check(lib().cola_ppl_batch_spmm(*a, int(local_col_lb), int(local_col_ub), int(remote_col_lb),
                                    int(remote_col_ub), int(stage), _any(idx_ppl), int(dim), int(nodesPerPE),
                                    int(group_size), int(group_offset), int(peid), _stream(stream)))


def batching_data_ppl(input, send, put_colIdx, nemb, dim, nodesPerPE, group_size, stream=None):
    """include/dist_spmm_ppl_batch.cuh:59-73 (launched as at :792)."""
    check(lib().cola_batching_data_ppl(_any(input), _any(send), _any(put_colIdx), int(nemb), int(dim),
                                       int(nodesPerPE), int(group_size), _stream(stream)))


def _any(x):
    if x is None:
        return None
    if isinstance(x, torch.Tensor):
        if x.numel() and not x.is_cuda:
            raise TypeError("device pointer argument must be a CUDA tensor")
        return ctypes.c_void_p(x.data_ptr()) if x.numel() else None
    return ctypes.c_void_p(int(x))
