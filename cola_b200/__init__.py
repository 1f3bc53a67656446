"""cola_b200: CoLa's partitioned SpMM (zzzlxhhh/CoLa) on one B200 (sm_100a).

P virtual row partitions, each a local CSR block plus a compacted remote CSC
block; the reference's NVSHMEM exchanges become on-device staged gathers.
Preprocessing is bit-identical to the reference's; the SpMM runs in hand-written
sm_100a CUDA kernels behind the C ABI in include/cola_spmm.h.
"""
from . import _lib
from ._lib import ColaError, lib  # noqa: F401
from .prep import (PartitionSet, bin2vec, community_order, global_csr, nnz_split, nnz_split_device,  # noqa: F401
                   ppl_row_partition, relabel_edges, rmat, row_partition, serialize, stage_tables, workgroup_cols, write_bin)

__all__ = ["PartitionSet", "row_partition", "serialize", "ppl_row_partition", "nnz_split", "nnz_split_device",
           "relabel_edges", "community_order", "stage_tables",
           "workgroup_cols", "global_csr", "bin2vec", "write_bin", "rmat", "ColaError", "lib", "version"]


def version():
    return _lib.lib().cola_version().decode()


def __getattr__(name):
    # the device API needs torch; import it on first use
    if name in ("Graph", "spmm"):
        import importlib
        mod = importlib.import_module(__name__ + ".spmm")
        return mod.Graph if name == "Graph" else mod
    raise AttributeError(name)
