"""Batched form: many graphs, each with its own X, Y and feature width, in one
persistent launch (plus one for hub rows), capturable in a CUDA graph, with the
project's launch-parameter autotuner.  Backed by the cola_batch_* C ABI."""
import ctypes
import os

import torch

from ._lib import BatchInfo, SpmmOpts, UploadOpts, check, lib
from .spmm import _DT, _dense, _stream


class Batch:
    """Partition sets uploaded together (each split and given its row view)."""

    def __init__(self, psets, if_split=True, hub_threshold=0, hub_segment=0, task_entries=0, stream=None):
        o = UploadOpts()
        o.if_split = 1 if if_split else 0
        o.hub_threshold = int(hub_threshold)
        o.hub_segment = int(hub_segment)
        o.task_entries = int(task_entries)
        arr = (ctypes.c_void_p * max(len(psets), 1))(*[p.handle.value for p in psets])
        h = ctypes.c_void_p()
        check(lib().cola_batch_create(arr, len(psets), ctypes.byref(o), ctypes.byref(h), _stream(stream)))
        self._h = h
        self.ngraphs = len(psets)
        self.num_nodes = [p.num_nodes for p in psets]
        self._bound = None

    @classmethod
    def from_graphs(cls, graphs):
        """A batch over existing Graph objects (uploaded with their row view, or
        built on the device); the batch keeps them alive and borrows them."""
        arr = (ctypes.c_void_p * max(len(graphs), 1))(*[g._h.value for g in graphs])
        h = ctypes.c_void_p()
        check(lib().cola_batch_create_from_graphs(arr, len(graphs), ctypes.byref(h)))
        b = cls.__new__(cls)
        b._h = h
        b.ngraphs = len(graphs)
        b.num_nodes = [g.num_nodes for g in graphs]
        b._bound = None
        b._graphs = list(graphs)
        return b

    def bind(self, Xs, Ys, stream=None):
        """Bind per-graph dense operands (CUDA tensors; all X one dtype, all Y one dtype)."""
        if len(Xs) != self.ngraphs or len(Ys) != self.ngraphs:
            raise ValueError("need one X and one Y per graph")
        for i, (x, y) in enumerate(zip(Xs, Ys)):
            _dense(x, "X[%d]" % i)
            _dense(y, "Y[%d]" % i)
            if x.shape[0] < self.num_nodes[i] or y.shape[0] < self.num_nodes[i] or x.shape[1] != y.shape[1]:
                raise ValueError("graph %d: X %s / Y %s do not fit %d nodes" % (i, tuple(x.shape), tuple(y.shape),
                                                                                  self.num_nodes[i]))
        if len({x.dtype for x in Xs}) > 1 or len({y.dtype for y in Ys}) > 1:
            raise TypeError("all X must share one dtype and all Y another")
        n = self.ngraphs
        P = ctypes.c_void_p
        xs = (P * n)(*[x.data_ptr() for x in Xs])
        ys = (P * n)(*[y.data_ptr() for y in Ys])
        ldx = (ctypes.c_int64 * n)(*[x.stride(0) for x in Xs])
        ldy = (ctypes.c_int64 * n)(*[y.stride(0) for y in Ys])
        ks = (ctypes.c_int32 * n)(*[x.shape[1] for x in Xs])
        check(lib().cola_batch_bind(self._h, xs, ldx, ys, ldy, ks, _DT[Xs[0].dtype], _DT[Ys[0].dtype],
                                    _stream(stream)))
        self._bound = (list(Xs), list(Ys))  # keep the tensors alive while bound

    def run(self, accumulate=False, stream=None):
        o = SpmmOpts()
        o.accumulate = 1 if accumulate else 0
        check(lib().cola_batch_run(self._h, ctypes.byref(o), _stream(stream)))

    def capture(self, accumulate=False, stream=None):
        """Record run() into a CUDA graph kept by the batch."""
        o = SpmmOpts()
        o.accumulate = 1 if accumulate else 0
        st = stream or torch.cuda.Stream()
        check(lib().cola_batch_capture(self._h, ctypes.byref(o), _stream(st)))

    def replay(self, stream=None):
        check(lib().cola_batch_replay(self._h, _stream(stream)))

    def set_params(self, unroll=4, grid_pct=100, blocks_per_sm=4):
        check(lib().cola_batch_set_params(self._h, int(unroll), int(grid_pct), int(blocks_per_sm)))

    def autotune(self, reps=3, stream=None, cache=None):
        """Time the launch-parameter candidates on the bound operands; keep the
        fastest.  With `cache` (a file path) a batch tuned before on this device
        model takes its stored parameters without timing; self.tuned_from_cache
        tells which happened."""
        ms = ctypes.c_float()
        if cache is None:
            check(lib().cola_batch_autotune(self._h, int(reps), _stream(stream), ctypes.byref(ms)))
            self.tuned_from_cache = False
        else:
            hit = ctypes.c_int32()
            check(lib().cola_batch_autotune_cached(self._h, int(reps), os.fsencode(cache), _stream(stream),
                                                   ctypes.byref(ms), ctypes.byref(hit)))
            self.tuned_from_cache = bool(hit.value)
        return ms.value

    @property
    def info(self):
        i = BatchInfo()
        check(lib().cola_batch_get_info(self._h, ctypes.byref(i)))
        return i

    def close(self):
        if self._h is not None and self._h.value:
            lib().cola_batch_free(self._h)
        self._h = None
        self._bound = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
