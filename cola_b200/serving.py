"""Serving loop (cola_server_* C ABI): graphs registered once stay resident;
requests with host X are admitted by a device-memory budget, grouped by
feature width and dtype into one batched launch across graphs, and run on
several streams, so new requests start as soon as a slot and memory free up."""
import ctypes

import torch

from ._lib import ServerOpts, ServerStats, UploadOpts, check, lib
from .spmm import _DT


class Request:
    def __init__(self, server, rid, X, Y):
        self.server = server
        self.id = rid
        self.X = X  # kept alive until the request finishes
        self.Y = Y
        self.done = False

    def wait(self, timeout_ms=-1):
        """Block until the result is in self.Y (returned); raises ColaError on
        timeout (the request stays queryable), cancellation or failure."""
        if not self.done:
            st = lib().cola_server_wait(self.server._h, ctypes.c_uint64(self.id), int(timeout_ms))
            if st != 7:  # anything but a timeout ends the request
                self.done = True
                self.server._live.pop(self.id, None)
            check(st)
        return self.Y

    def cancel(self):
        check(lib().cola_server_cancel(self.server._h, ctypes.c_uint64(self.id)))


class Server:
    def __init__(self, memory_budget=0, slots=0, max_group=0, group_mib=0, small_mib=0, copy_chunk_mib=0,
                 copy_engines_only=False):
        """small_mib: requests with at most this many MiB of copies are small
        (a slot is kept for them and they may pass a large request that waits;
        0 = 16, -1 = plain FIFO).  copy_chunk_mib: copies move in pieces of at
        most this size (0 = 32).  copy_engines_only: small groups copy with the
        copy engines too, instead of with a kernel on pinned host memory."""
        o = ServerOpts()
        o.memory_budget = int(memory_budget)
        o.slots = int(slots)
        o.max_group = int(max_group)
        o.group_mib = int(group_mib)
        o.small_mib = int(small_mib)
        o.copy_chunk_mib = int(copy_chunk_mib)
        o.copy_engines_only = 1 if copy_engines_only else 0
        h = ctypes.c_void_p()
        check(lib().cola_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.num_nodes = []
        self._live = {}  # request id -> (X, Y): host buffers the GPU may still read or write

    def register(self, pset, if_split=True, hub_threshold=0, hub_segment=0, task_entries=0):
        o = UploadOpts()
        o.if_split = 1 if if_split else 0
        o.hub_threshold = int(hub_threshold)
        o.hub_segment = int(hub_segment)
        o.task_entries = int(task_entries)
        gid = ctypes.c_int32()
        check(lib().cola_server_register(self._h, pset.handle, ctypes.byref(o), ctypes.byref(gid)))
        self.num_nodes.append(pset.num_nodes)
        return gid.value

    def register_graph(self, graph):
        """Register an existing Graph (for example Graph.from_coo_device); the
        server takes it over: the Graph object is empty afterwards."""
        h, graph._h = graph._h, None
        gid = ctypes.c_int32()
        check(lib().cola_server_register_graph(self._h, h, ctypes.byref(gid)))
        self.num_nodes.append(graph.num_nodes)
        return gid.value

    def submit(self, graph_id, X, out_dtype=torch.float32, Y=None):
        """X: host tensor N x K (float32 or bfloat16; pinned memory lets copies
        overlap).  Returns a Request whose wait() gives Y (host, out_dtype)."""
        if X.is_cuda or X.dim() != 2 or not X.is_contiguous() or X.dtype not in _DT:
            raise ValueError("X must be a contiguous 2-D host tensor of float32 or bfloat16")
        if not 0 <= int(graph_id) < len(self.num_nodes):
            raise ValueError("unknown graph {}".format(graph_id))
        n = self.num_nodes[graph_id]
        if X.shape[0] != n:
            raise ValueError("X has {} rows, graph {} has {}".format(X.shape[0], graph_id, n))
        K = X.shape[1]
        if Y is None:
            Y = torch.empty((n, K), dtype=out_dtype, pin_memory=True)
        if Y.is_cuda or Y.shape != (n, K) or not Y.is_contiguous() or Y.dtype not in _DT:
            raise ValueError("Y must be a contiguous host tensor of shape {}".format((n, K)))
        rid = ctypes.c_uint64()
        check(lib().cola_server_submit(self._h, int(graph_id), ctypes.c_void_p(X.data_ptr()), _DT[X.dtype], K,
                                       ctypes.c_void_p(Y.data_ptr()), _DT[Y.dtype], ctypes.byref(rid)))
        self._live[rid.value] = (X, Y)
        return Request(self, rid.value, X, Y)

    def reset_stats(self):
        """Start a new measurement window (latencies, counts, peaks)."""
        check(lib().cola_server_reset_stats(self._h))

    def stats(self):
        s = ServerStats()
        check(lib().cola_server_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self._h is not None and self._h.value:
            lib().cola_server_destroy(self._h)  # waits for the requests on the GPU
        self._h = None
        self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
