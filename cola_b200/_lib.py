"""ctypes binding of libcola_b200.so (the C ABI declared in include/cola_spmm.h).

The library is built in-tree (cola_b200/lib/).  Loading fails loudly when it
is missing: there is no fallback implementation.
"""
import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libcola_b200.so")

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
F64 = ctypes.c_double

SUCCESS = 0
STATUS = {0: "success", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "unsupported",
          5: "I/O error", 6: "over memory budget", 7: "timed out", 8: "not ready", 9: "cancelled"}

FLOAT32 = 0
BFLOAT16 = 1

SCHEDULE_AUTO = 0
SCHEDULE_FUSED = 1
SCHEDULE_BUFFER = 2
SCHEDULE_PIPELINE = 3
SCHEDULE_ROWS = 4

# capacity (floats) of the library's fixed staging array (include/cola_spmm.h)
NOALLOC_STAGE_FLOATS = 2 * 1024 * 1024


class ColaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("{} ({}): {}".format(STATUS.get(status, "status %d" % status), status, msg))
        self.status = status


class PartitionView(ctypes.Structure):
    _fields_ = [("part", I32), ("nparts", I32), ("num_nodes", I32), ("nodes_per_part", I32), ("row_lb", I32),
                ("row_ub", I32),
                ("csr_rowPtr_l", P), ("csr_colIdx_l", P), ("csr_val_l", P), ("csr_rowIdx_l", P),
                ("csc_colPtr_r", P), ("csc_rowIdx_r", P), ("csc_val_r", P), ("csc_colIdx_r", P),
                ("n_rowPtr_l", I64), ("nnz_l", I64), ("n_rows_l", I64), ("n_colPtr_r", I64), ("nnz_r", I64),
                ("n_cols_r", I64)]


class UploadOpts(ctypes.Structure):
    _fields_ = [("if_split", I32), ("group_size", I32), ("no_row_view", I32), ("hub_threshold", I32),
                ("hub_segment", I32), ("task_entries", I32), ("reserved", I32 * 2)]


class GraphInfo(ctypes.Structure):
    _fields_ = [("num_nodes", I32), ("nparts", I32), ("nodes_per_part", I32), ("group_size", I32),
                ("nnz", I64), ("nnz_local", I64), ("nnz_remote", I64), ("local_chunks", I64),
                ("remote_chunks", I64), ("remote_cols", I64), ("device_bytes", I64), ("hub_rows", I64),
                ("hub_segments", I64), ("row_tasks", I64), ("last_launches", I64)]


class ZipView(ctypes.Structure):
    _fields_ = [("csr_rowPtr", P), ("csr_colIdx", P), ("csr_rowIdx_zip", P), ("csr_val", P),
                ("csc_colPtr", P), ("csc_rowIdx", P), ("csc_colIdx_zip", P), ("csc_val", P),
                ("local_chunks", I32), ("remote_chunks", I32), ("nnz_l", I64), ("nnz_r", I64)]


class SpmmOpts(ctypes.Structure):
    _fields_ = [("accumulate", I32), ("schedule", I32), ("gather_batch_rows", I32), ("unroll", I32),
                ("min_blocks", I32), ("k_tile", I32), ("reserved", I32 * 2)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("ngraphs", I32), ("batched_graphs", I32), ("work_items", I64), ("hub_items", I64),
                ("nnz", I64), ("device_bytes", I64), ("unroll", I32), ("grid_pct", I32), ("blocks_per_sm", I32),
                ("last_launches", I64)]


class ZipPart(ctypes.Structure):
    _fields_ = [("csr_rowPtr_l", P), ("csr_colIdx_l", P), ("csr_rowIdx_zip_l", P), ("csr_val_l", P),
                ("csc_colPtr_r", P), ("csc_rowIdx_r", P), ("csc_colIdx_zip_r", P), ("csc_val_r", P),
                ("local_row_lb", I32), ("remote_col_lb", I32), ("local_row_num", I32), ("remote_col_num", I32)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("memory_budget", I64), ("slots", I32), ("max_group", I32), ("group_mib", I32),
                ("small_mib", I32), ("copy_chunk_mib", I32), ("copy_engines_only", I32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", I64), ("completed", I64), ("rejected", I64), ("cancelled", I64), ("failed", I64),
                ("pending", I64), ("inflight", I32), ("max_inflight", I32), ("groups_launched", I32),
                ("max_group", I32), ("bytes_in_use", I64), ("peak_bytes", I64), ("budget", I64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("req_per_s", ctypes.c_double), ("queue_ms_mean", ctypes.c_double),
                ("copy_in_ms_mean", ctypes.c_double), ("kernel_ms_mean", ctypes.c_double),
                ("copy_out_ms_mean", ctypes.c_double)]


# name -> (restype, argtypes)
SIGNATURES = {
    "cola_status_string": (ctypes.c_char_p, [I32]),
    "cola_last_error": (ctypes.c_char_p, []),
    "cola_version": (ctypes.c_char_p, []),
    "cola_partition_build": (I32, [I32, I64, P, P, P, I32, P]),
    "cola_partition_set_free": (None, [P]),
    "cola_partition_get": (I32, [P, I32, P]),
    "cola_nnz_split": (I32, [P, I64, P, I64, P, P, I64, P]),
    "cola_partition_build_device": (I32, [I32, I64, P, P, P, I32, P, P]),
    "cola_set_gather_bulk": (I32, [I32]),
    "cola_set_gather_wait_limit": (I32, [I64]),
    "cola_probe_gather": (I32, [I64, I32, I64, I32, P, P]),
    "cola_probe_graph_gather": (I32, [P, P, I64, I32, I32, P, P, P]),
    "cola_device_error_check": (I32, [P]),
    "cola_graph_build_device": (I32, [I32, I64, P, P, P, I32, P, P, P]),
    "cola_nnz_split_device": (I32, [P, I64, P, I64, P, P, I64, P, P]),
    "cola_relabel_edges": (I32, [I32, I64, P, P, P, P, P]),
    "cola_community_order": (I32, [I32, I64, P, P, P, P]),
    "cola_relabel_edges_device": (I32, [I32, I64, P, P, P, P, P, P]),
    "cola_global_csr": (I32, [I32, I64, P, P, P, P, P, P, P]),
    "cola_workgroup_cols": (I32, [I32, I64, P, P, I32, I32, I32, P, P]),
    "cola_stage_tables": (I32, [I32, I32, I32, I32, P, I64, I64, P, P, P, P, P, P, P, I64, P, P, I64]),
    "cola_bin_read_i32": (I32, [ctypes.c_char_p, P, I64, P]),
    "cola_bin_write_i32": (I32, [ctypes.c_char_p, P, I64]),
    "cola_bin_read_f32": (I32, [ctypes.c_char_p, P, I64, P]),
    "cola_bin_write_f32": (I32, [ctypes.c_char_p, P, I64]),
    "cola_partition_write_bin": (I32, [P, ctypes.c_char_p]),
    "cola_partition_read_bin": (I32, [ctypes.c_char_p, I32, I32, P]),
    "cola_rmat_generate": (I32, [I32, F64, F64, F64, F64, ctypes.c_uint64, I32, I32, P, P, P, I64, P]),
    "cola_ppl0_batch_spmm": (I32, [P, P] + [P] * 8 + [I32] * 7 + [P]),
    "cola_ppl0_batch_spmm_seq": (I32, [P, P] + [P] * 8 + [I32] * 7 + [P]),
    "cola_ppl0_batch_buffer_spmm": (I32, [P, P, P] + [P] * 8 + [I32] * 7 + [P]),
    "cola_ppl0_batch_buffer_spmm_noalloc": (I32, [P, P] + [P] * 8 + [I32] * 7 + [P]),
    "cola_ppl_batch_spmm": (I32, [P, P, P, P, P, P] + [I32] * 5 + [P] + [I32] * 5 + [P]),
    "cola_zip_rows_create": (I32, [P] * 8 + [I32] * 6 + [P, P]),
    "cola_zip_rows_create_all": (I32, [P, I32, I32, P, P]),
    "cola_zip_rows_spmm": (I32, [P, P, P, I32, P]),
    "cola_zip_rows_free": (I32, [P]),
    "cola_zip_rows_get_info": (I32, [P, P, P, P, P]),
    "cola_batching_data_ppl": (I32, [P, P, P, I32, I32, I32, I32, P]),
    "cola_graph_upload": (I32, [P, P, P, P]),
    "cola_graph_free": (I32, [P]),
    "cola_graph_get_info": (I32, [P, P]),
    "cola_graph_zip_view": (I32, [P, I32, P]),
    "cola_spmm": (I32, [P, P, I32, I64, P, I32, I64, I32, P, P]),
    "cola_spmm_host": (I32, [P, P, I32, I64, P, I32, I64, I32, P, P]),
    "cola_spmm_host_sync": (I32, [P]),
    "cola_spmm_host_join": (I32, [P, P]),
    "cola_spmm_autotune": (I32, [P, P, I32, I64, P, I32, I64, I32, I32, I32, ctypes.c_char_p, P, P, P, P]),
    "cola_batch_create": (I32, [P, I32, P, P, P]),
    "cola_batch_create_from_graphs": (I32, [P, I32, P]),
    "cola_batch_free": (I32, [P]),
    "cola_batch_bind": (I32, [P, P, P, P, P, P, I32, I32, P]),
    "cola_batch_run": (I32, [P, P, P]),
    "cola_batch_capture": (I32, [P, P, P]),
    "cola_batch_replay": (I32, [P, P]),
    "cola_batch_set_params": (I32, [P, I32, I32, I32]),
    "cola_batch_autotune": (I32, [P, I32, P, P]),
    "cola_batch_autotune_cached": (I32, [P, I32, ctypes.c_char_p, P, P, P]),
    "cola_batch_get_info": (I32, [P, P]),
    "cola_server_create": (I32, [P, P]),
    "cola_server_destroy": (I32, [P]),
    "cola_server_register": (I32, [P, P, P, P]),
    "cola_server_register_graph": (I32, [P, P, P]),
    "cola_server_submit": (I32, [P, I32, P, I32, I32, P, I32, P]),
    "cola_server_wait": (I32, [P, ctypes.c_uint64, I32]),
    "cola_server_cancel": (I32, [P, ctypes.c_uint64]),
    "cola_server_get_stats": (I32, [P, P]),
    "cola_server_reset_stats": (I32, [P]),
}

_lib = None


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("cola_b200 native library missing at {}: run `python -m cola_b200._build` "
                               "(or __graft_entry__.build())".format(LIB_PATH))
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status):
    """Raise ColaError for a non-success status with the library's message."""
    if status != SUCCESS:
        msg = lib().cola_last_error()
        raise ColaError(status, msg.decode() if msg else "")
    return status
