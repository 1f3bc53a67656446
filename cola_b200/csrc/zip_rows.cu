// The row view of one virtual PE's split blocks (the reference's d_csr_zip /
// d_csc_zip arrays, include/sparse_data.h:28-77) for callers of the
// kernel-level launcher: the chunks a ppl0_batch_SpMM call covers
// (include/dist_spmm_ppl_batch.cuh:202-245) are expanded on the device into
// (partition row, global column, value) entries, and the device graph build
// turns them into the row-major view -- every row's entries in column order,
// rows longer than 256 entries cut into segments, row-block tasks.  Built once
// per zip pair and chunk range; each SpMM through it is the row-major
// schedule accumulating into the caller's output, the same sum the chunk
// kernel computes with atomics.
#include <algorithm>
#include <cstdint>
#include <new>

#include <cuda_runtime.h>

#include "common.h"
#include "graph.h"

struct cola_zip_rows {
    cola_graph *g = nullptr;
    int32_t npp = 0, peid = 0;
    int64_t nnz = 0;
};

namespace cola {
namespace zr {

// Entries [e0, e0 + count) of a chunked block: chunk c (c0 <= c < c0 + nch)
// covers [ptr[c], ptr[c+1]) and names target[c]; the entry's own index array
// holds the other coordinate.  Local CSR chunks: row = target, column =
// col_off + index.  Remote CSC chunks (remote = 1): column = target, row =
// index.
__global__ void expand_chunks_kernel(const int32_t *__restrict__ ptr, const int32_t *__restrict__ target,
                                     const int32_t *__restrict__ index, const float *__restrict__ val, int64_t c0,
                                     int64_t nch, int64_t e0, int64_t count, int64_t col_off, int remote,
                                     int32_t *__restrict__ out_row, int32_t *__restrict__ out_col,
                                     float *__restrict__ out_val, unsigned int *__restrict__ max_row,
                                     unsigned int *__restrict__ max_col, unsigned int *__restrict__ ok)
{
    unsigned int mr = 0, mc = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = e0 + i;
        // the chunk holding entry e: the last c with ptr[c] <= e
        int64_t lo = c0, hi = c0 + nch;
        while (hi - lo > 1) {
            const int64_t m = (lo + hi) >> 1;
            if (__ldg(ptr + m) <= e)
                lo = m;
            else
                hi = m;
        }
        const int64_t t = __ldg(target + lo), x = __ldg(index + e);
        const int64_t r = remote ? x : t;
        const int64_t c = remote ? t : col_off + x;
        if (r < 0 || c < 0 || r > INT32_MAX || c > INT32_MAX) {
            atomicMin(ok, 0u);  // reported by the host
            out_row[i] = out_col[i] = 0;
            out_val[i] = 0.f;
            continue;
        }
        out_row[i] = (int32_t)r;
        out_col[i] = (int32_t)c;
        out_val[i] = val ? __ldg(val + e) : 1.0f;
        mr = max(mr, (unsigned int)r);
        mc = max(mc, (unsigned int)c);
    }
    atomicMax(max_row, mr);
    atomicMax(max_col, mc);
}

static int blocks_for(int64_t n)
{
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8));
}

static cola_status read_i32(const int32_t *d, int64_t i, int32_t &v, cudaStream_t st)
{
    COLA_CUDA(cudaMemcpyAsync(&v, d + i, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    return COLA_SUCCESS;
}

}  // namespace zr
}  // namespace cola

using namespace cola;

extern "C" {

cola_status cola_zip_rows_create(const int32_t *csr_rowPtr_l, const int32_t *csr_colIdx_l,
                                 const int32_t *csr_rowIdx_zip_l, const float *csr_val_l, const int32_t *csc_colPtr_r,
                                 const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r, const float *csc_val_r,
                                 int32_t local_row_lb, int32_t remote_col_lb, int32_t local_row_num,
                                 int32_t remote_col_num, int32_t nodesPerPE, int32_t peid, cola_stream_t stream,
                                 cola_zip_rows **out)
{
    const char *who = "cola_zip_rows_create";
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "%s: out is NULL", who);
    *out = nullptr;
    clear_error();
    COLA_REQUIRE(local_row_lb >= 0 && remote_col_lb >= 0 && local_row_num >= 0 && remote_col_num >= 0 &&
                     nodesPerPE >= 1 && peid >= 0,
                 COLA_ERROR_INVALID_ARGUMENT, "%s: negative chunk range, nodesPerPE %d or peid %d", who, nodesPerPE,
                 peid);
    COLA_REQUIRE(local_row_num == 0 || (csr_rowPtr_l && csr_colIdx_l && csr_rowIdx_zip_l), COLA_ERROR_INVALID_ARGUMENT,
                 "%s: null local CSR arrays", who);
    COLA_REQUIRE(remote_col_num == 0 || (csc_colPtr_r && csc_rowIdx_r && csc_colIdx_zip_r),
                 COLA_ERROR_INVALID_ARGUMENT, "%s: null remote CSC arrays", who);
    cudaStream_t st = (cudaStream_t)stream;
    // entry ranges of the chunks the call covers (chunk pointers are monotonic)
    int32_t lb_e = 0, le_e = 0, rb_e = 0, re_e = 0;
    if (local_row_num > 0) {
        COLA_TRY(zr::read_i32(csr_rowPtr_l, local_row_lb, lb_e, st));
        COLA_TRY(zr::read_i32(csr_rowPtr_l, (int64_t)local_row_lb + local_row_num, le_e, st));
    }
    if (remote_col_num > 0) {
        COLA_TRY(zr::read_i32(csc_colPtr_r, remote_col_lb, rb_e, st));
        COLA_TRY(zr::read_i32(csc_colPtr_r, (int64_t)remote_col_lb + remote_col_num, re_e, st));
    }
    COLA_CUDA(cudaStreamSynchronize(st));
    COLA_REQUIRE(le_e >= lb_e && re_e >= rb_e, COLA_ERROR_INVALID_ARGUMENT, "%s: chunk pointers decrease", who);
    const int64_t nl = (int64_t)le_e - lb_e, nr = (int64_t)re_e - rb_e, nnz = nl + nr;

    void *arena = nullptr;
    const size_t a = 256, n = (size_t)std::max<int64_t>(nnz, 1);
    const size_t bytes = 3 * ((4 * n + a - 1) / a * a) + a;
    COLA_CUDA(cudaMallocAsync(&arena, bytes, st));
    char *base = static_cast<char *>(arena);
    const size_t slice = (4 * n + a - 1) / a * a;
    int32_t *row = reinterpret_cast<int32_t *>(base);
    int32_t *col = reinterpret_cast<int32_t *>(base + slice);
    float *val = reinterpret_cast<float *>(base + 2 * slice);
    unsigned int *mx = reinterpret_cast<unsigned int *>(base + 3 * slice);  // max row, max col, all in range
    cola_status rc = COLA_SUCCESS;
    unsigned int h_mx[3] = {0, 0, 1};
    {
        const unsigned int init[3] = {0u, 0u, 1u};
        cudaError_t e = cudaMemcpyAsync(mx, init, sizeof init, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && nl > 0) {
            zr::expand_chunks_kernel<<<zr::blocks_for(nl), 256, 0, st>>>(
                csr_rowPtr_l, csr_rowIdx_zip_l, csr_colIdx_l, csr_val_l, local_row_lb, local_row_num, lb_e, nl,
                (int64_t)peid * nodesPerPE, 0, row, col, val, mx, mx + 1, mx + 2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && nr > 0) {
            zr::expand_chunks_kernel<<<zr::blocks_for(nr), 256, 0, st>>>(
                csc_colPtr_r, csc_colIdx_zip_r, csc_rowIdx_r, csc_val_r, remote_col_lb, remote_col_num, rb_e, nr, 0,
                1, row + nl, col + nl, val + nl, mx, mx + 1, mx + 2);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h_mx, mx, sizeof h_mx, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            rc = fail(COLA_ERROR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    }
    if (rc == COLA_SUCCESS && h_mx[2] == 0)
        rc = fail(COLA_ERROR_INVALID_ARGUMENT, "%s: an entry's row or column is negative or too large", who);
    cola_graph *g = nullptr;
    if (rc == COLA_SUCCESS) {
        // rows: up to the last one that has an entry (rows past it are never
        // touched, as the chunk kernel touches none); columns: global ids
        const int64_t nrows = nnz > 0 ? (int64_t)h_mx[0] + 1 : 0;
        const int64_t ncols = std::max<int64_t>(nrows, nnz > 0 ? (int64_t)h_mx[1] + 1 : 0);
        rc = graph_build_device_rect((int32_t)nrows, (int32_t)ncols, nnz, row, col, val, nullptr, st, g, who);
    }
    cudaFreeAsync(arena, st);
    if (rc != COLA_SUCCESS)
        return rc;
    cola_zip_rows *h = new (std::nothrow) cola_zip_rows();
    if (!h) {
        graph_release(g);
        return fail(COLA_ERROR_OUT_OF_MEMORY, "%s: host allocation failed", who);
    }
    h->g = g;
    h->npp = nodesPerPE;
    h->peid = peid;
    h->nnz = nnz;
    *out = h;
    return COLA_SUCCESS;
}

cola_status cola_zip_rows_spmm(cola_zip_rows *h, float *output, const float *input, int32_t dim,
                               cola_stream_t stream)
{
    COLA_REQUIRE(h && h->g, COLA_ERROR_INVALID_ARGUMENT, "cola_zip_rows_spmm: handle is NULL");
    COLA_REQUIRE(dim >= 1, COLA_ERROR_INVALID_ARGUMENT, "cola_zip_rows_spmm: dim %d", dim);
    if (h->g->N == 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(output && input, COLA_ERROR_INVALID_ARGUMENT, "cola_zip_rows_spmm: null dense pointer");
    // global column c is row c of the symmetric X, whose PE `peid` slice is `input`
    const float *x0 = input - (int64_t)h->peid * h->npp * dim;
    cola_spmm_opts o = {};
    o.accumulate = 1;
    o.schedule = COLA_SCHEDULE_ROWS;
    return cola_spmm(h->g, x0, COLA_FLOAT32, dim, output, COLA_FLOAT32, dim, dim, &o, stream);
}

cola_status cola_zip_rows_free(cola_zip_rows *h)
{
    if (h) {
        cola_status s = cola_graph_free(h->g);
        delete h;
        return s;
    }
    return COLA_SUCCESS;
}

cola_status cola_zip_rows_get_info(const cola_zip_rows *h, int64_t *rows, int64_t *nnz, int64_t *hub_rows,
                                   int64_t *device_bytes)
{
    COLA_REQUIRE(h && h->g, COLA_ERROR_INVALID_ARGUMENT, "cola_zip_rows_get_info: handle is NULL");
    if (rows)
        *rows = h->g->N;
    if (nnz)
        *nnz = h->nnz;
    if (hub_rows)
        *hub_rows = h->g->nhub;
    if (device_bytes)
        *device_bytes = (int64_t)(h->g->dbytes + h->g->ws_hub_bytes);
    return COLA_SUCCESS;
}

}  // extern "C"
