"""Argument errors at the C ABI come back as status codes with a message,
before any device work (so these run on a machine without a GPU): the
reference's launchers called exit(); these return COLA_ERROR_INVALID_ARGUMENT
(1) or COLA_ERROR_UNSUPPORTED (4) and leave the reason in cola_last_error()."""
import ctypes

import cola_b200 as cb

P = ctypes.c_void_p
NULL = P(0)


def last_error():
    return cb.lib().cola_last_error().decode()


def ppl0(L, out, inp, local_rows, remote_cols, dim, npp, peid=0, ptr=NULL):
    return L.cola_ppl0_batch_spmm(out, inp, ptr, ptr, ptr, ptr, ptr, ptr, ptr, ptr, 0, 0, local_rows, remote_cols,
                                  dim, npp, peid, NULL)


def test_kernel_level_launcher_arguments():
    L = cb.lib()
    dummy = P(16)  # never dereferenced: every call below is rejected first
    assert ppl0(L, dummy, dummy, 1, 0, 0, 8) == 1 and "dim" in last_error()
    assert ppl0(L, dummy, dummy, 1, 0, 128, 0) == 1 and "nodesPerPE" in last_error()
    assert ppl0(L, dummy, dummy, -1, 0, 128, 8) == 1 and "negative" in last_error()
    assert ppl0(L, dummy, dummy, 0, 0, 128, 8, peid=-1) == 1
    assert ppl0(L, NULL, dummy, 4, 0, 128, 8) == 1 and "null dense pointer" in last_error()
    assert ppl0(L, dummy, dummy, 4, 0, 128, 8) == 1 and "null local CSR" in last_error()
    assert ppl0(L, dummy, dummy, 0, 4, 128, 8) == 1 and "null remote CSC" in last_error()
    # nothing to do is not an error (the reference's launcher returns as well)
    assert ppl0(L, NULL, NULL, 0, 0, 128, 8) == 0


def test_graph_and_gather_arguments():
    L = cb.lib()
    assert L.cola_spmm(NULL, NULL, 0, 128, NULL, 0, 128, 128, NULL, NULL) == 1
    assert "graph is NULL" in last_error()
    assert L.cola_batching_data_ppl(NULL, NULL, NULL, 4, 128, 8, 1, NULL) == 1
    assert "null pointer" in last_error()


def test_server_and_batch_arguments():
    L = cb.lib()
    rid = ctypes.c_uint64()
    assert L.cola_server_submit(NULL, 0, NULL, 0, 64, NULL, 0, ctypes.byref(rid)) == 1
    assert "null argument" in last_error()
    assert L.cola_server_wait(NULL, ctypes.c_uint64(1), 0) == 1
    assert L.cola_batch_bind(NULL, NULL, NULL, NULL, NULL, 0, 0, 0, NULL) == 1
    assert "null argument" in last_error()
