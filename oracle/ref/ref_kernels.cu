/*
 * ref_kernels.cu -- C entry points around the reference's OWN code, compiled
 * from the reference tree (include/dist_spmm_ppl_batch.cuh, include/utils.cuh,
 * include/sparse_data.h) through the single-GPU NVSHMEM/MPI shim in ./shim.
 *
 * TEST INFRASTRUCTURE.  Built by oracle/Makefile into oracle/_ref/ when the
 * reference tree is present; loaded only by tests/ (GPU checker for the
 * product's kernels, host checker for nnz_split) and by bench.py's reference
 * leg (SAG_reference_host, the reference's CPU SpMM).  Nothing of the
 * reference's source is copied here: the headers are included in place.
 */
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "mpi.h"
#include "dist_spmm_ppl_batch.cuh"

extern "C" {

/* Select the emulated PE for the launches that follow on `stream`. */
int ref_set_pe(int me, long long pe_stride_elems, cudaStream_t stream)
{
    cola_shim_host_me = me;
    cola_shim_host_pe_stride = pe_stride_elems;
    cudaError_t e = cudaMemcpyToSymbolAsync(cola_shim_me, &me, sizeof(int), 0, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbolAsync(cola_shim_pe_stride, &pe_stride_elems, sizeof(long long), 0,
                                    cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream); /* the host copies above read stack memory */
    return (int)e;
}

#define REF_CF_DISPATCH(FN, ...)                      \
    switch (CF) {                                     \
    case 1: if (res) FN<1, true>(__VA_ARGS__); else FN<1, false>(__VA_ARGS__); break;   \
    case 2: if (res) FN<2, true>(__VA_ARGS__); else FN<2, false>(__VA_ARGS__); break;   \
    case 3: if (res) FN<3, true>(__VA_ARGS__); else FN<3, false>(__VA_ARGS__); break;   \
    case 4: if (res) FN<4, true>(__VA_ARGS__); else FN<4, false>(__VA_ARGS__); break;   \
    case 8: if (res) FN<8, true>(__VA_ARGS__); else FN<8, false>(__VA_ARGS__); break;   \
    case 16: if (res) FN<16, true>(__VA_ARGS__); else FN<16, false>(__VA_ARGS__); break; \
    default: return -1;                               \
    }

/* ppl0_batch_SpMM<CF, is_residue> (include/dist_spmm_ppl_batch.cuh:202-245). */
int ref_ppl0_batch_spmm(int CF, int res, float *output, const float *input,
                        const int *csr_rowPtr_l, const int *csr_colIdx_l, const int *csr_rowIdx_zip_l,
                        const float *csr_val_l, const int *csc_colPtr_r, const int *csc_rowIdx_r,
                        const int *csc_colIdx_zip_r, const float *csc_val_r, int local_row_lb,
                        int remote_col_lb, int local_row_num, int remote_col_num, int dim,
                        int nodesPerPE, int peid, cudaStream_t stream)
{
    REF_CF_DISPATCH(ppl0_batch_SpMM, output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l,
                    csr_val_l, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb,
                    remote_col_lb, local_row_num, remote_col_num, dim, nodesPerPE, peid, stream)
    return 0;
}

/* ppl0_batch_buffer_SpMM<CF, is_residue> (include/dist_spmm_ppl_batch.cuh:373-417). */
int ref_ppl0_batch_buffer_spmm(int CF, int res, float *output, const float *input, const float *comm_buffer,
                               const int *csr_rowPtr_l, const int *csr_colIdx_l,
                               const int *csr_rowIdx_zip_l, const float *csr_val_l,
                               const int *csc_colPtr_r, const int *csc_rowIdx_r,
                               const int *csc_colIdx_zip_r, const float *csc_val_r, int local_row_lb,
                               int remote_col_lb, int local_row_num, int remote_col_num, int dim,
                               int nodesPerPE, int peid, cudaStream_t stream)
{
    REF_CF_DISPATCH(ppl0_batch_buffer_SpMM, output, input, comm_buffer, csr_rowPtr_l, csr_colIdx_l,
                    csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r,
                    local_row_lb, remote_col_lb, local_row_num, remote_col_num, dim, nodesPerPE, peid,
                    stream)
    return 0;
}

/* ppl0_batch_SpMM_seq<CF, is_residue> (include/dist_spmm_ppl_batch.cuh:543-587). */
int ref_ppl0_batch_spmm_seq(int CF, int res, float *output, const float *input,
                            const int *csr_rowPtr_l, const int *csr_colIdx_l, const int *csr_rowIdx_zip_l,
                            const float *csr_val_l, const int *csc_colPtr_r, const int *csc_rowIdx_r,
                            const int *csc_colIdx_zip_r, const float *csc_val_r, int local_row_lb,
                            int remote_col_lb, int local_row_num, int remote_col_num, int dim,
                            int nodesPerPE, int peid, cudaStream_t stream)
{
    REF_CF_DISPATCH(ppl0_batch_SpMM_seq, output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l,
                    csr_val_l, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb,
                    remote_col_lb, local_row_num, remote_col_num, dim, nodesPerPE, peid, stream)
    return 0;
}

/* ppl_batch_SpMM<CF, is_residue> (include/dist_spmm_ppl_batch.cuh:709-760). */
int ref_ppl_batch_spmm(int CF, int res, float *output, const float *input, const int *csc_colPtr_r,
                       const int *csc_rowIdx_r, const int *csc_colIdx_zip_r, const float *csc_val_r,
                       int local_col_lb, int local_col_ub, int remote_col_lb, int remote_col_ub, int stage,
                       const int *idx_ppl, int dim, int nodesPerPE, int group_size, int group_offset,
                       int peid, cudaStream_t stream)
{
    REF_CF_DISPATCH(ppl_batch_SpMM, output, input, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r,
                    local_col_lb, local_col_ub, remote_col_lb, remote_col_ub, stage, idx_ppl, dim,
                    nodesPerPE, group_size, group_offset, peid, stream)
    return 0;
}

/* batching_data_ppl (include/dist_spmm_ppl_batch.cuh:59-73), launched as the
 * reference launches it (:792): grid nemb, block 32. */
int ref_batching_data_ppl(const float *input, float *send, int *put_colIdx, int nemb, int dim, int nodesPerPE,
                          int group_size, cudaStream_t stream)
{
    if (nemb > 0)
        batching_data_ppl<<<nemb, 32, 0, stream>>>(input, send, put_colIdx, dim, nodesPerPE, group_size);
    return (int)cudaGetLastError();
}

/* nnz_split (include/dist_spmm_ppl_batch.cuh:29-56).  Outputs are copied into
 * caller buffers of capacity cap (target) and cap+1 (ptr). */
int ref_nnz_split(const int *rowIdx, long long nrows, const int *rowPtr, long long nnz, int *target, int *ptr,
                  long long cap, long long *nchunks, long long *ptr_len)
{
    std::vector<int> ri(rowIdx, rowIdx + nrows);
    std::vector<int> rp(rowPtr, rowPtr + (nrows > 0 ? nrows + 1 : 0));
    std::vector<int> ci((size_t)nnz, 0);
    std::vector<int> tg, pt;
    nnz_split(ri, rp, ci, tg, pt, 0, true);
    if ((long long)tg.size() > cap)
        return -1;
    std::copy(tg.begin(), tg.end(), target);
    std::copy(pt.begin(), pt.end(), ptr);
    *nchunks = (long long)tg.size();
    *ptr_len = (long long)pt.size();
    return 0;
}

/* SAG_reference_host<int, float> (include/utils.cuh:45-69): the reference's
 * CPU SpMM over global CSR rows [lb, ub), ignoring values. */
void ref_sag_reference_host(int lb, int ub, int N, const int *csr_indptr, const int *csr_indices, const float *B,
                            float *C_ref, int peid)
{
    SAG_reference_host<int, float>(lb, ub, N, csr_indptr, csr_indices, B, C_ref, peid);
}

} /* extern "C" */
