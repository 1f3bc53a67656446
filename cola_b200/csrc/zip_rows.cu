// The row view of one virtual PE's split blocks (the reference's d_csr_zip /
// d_csc_zip arrays, include/sparse_data.h:28-77) for callers of the
// kernel-level launcher: the chunks a ppl0_batch_SpMM call covers
// (include/dist_spmm_ppl_batch.cuh:202-245) are expanded on the device into
// (partition row, global column, value) entries, and the device graph build
// turns them into the row-major view -- every row's entries in column order,
// long rows cut into segments, row-block tasks (sized by the view).  Built once
// per zip pair and chunk range; each SpMM through it is the row-major
// schedule accumulating into the caller's output, the same sum the chunk
// kernel computes with atomics.
#include <algorithm>
#include <cstdint>
#include <new>
#include <vector>

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
// holds the other coordinate.  Local CSR chunks: row = row_off + target,
// column = col_off + index.  Remote CSC chunks (remote = 1): column = target,
// row = row_off + index.
__global__ void expand_chunks_kernel(const int32_t *__restrict__ ptr, const int32_t *__restrict__ target,
                                     const int32_t *__restrict__ index, const float *__restrict__ val, int64_t c0,
                                     int64_t nch, int64_t e0, int64_t count, int64_t col_off, int64_t row_off,
                                     int remote,
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
        const int64_t r = row_off + (remote ? x : t);
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

namespace cola {
namespace zr {

// The row view of the chunks of several PEs' calls: PE part[i] (whose rows
// start at output row row0[i]) contributes its local chunks [llb, +lnum) and
// remote chunks [rlb, +rnum).  x_peid: the PE whose X slice the SpMM calls
// will pass as `input`.
static cola_status build(const cola_zip_part *parts, int32_t nparts, const int64_t *row0, int32_t nodesPerPE,
                         const int32_t *peids, int32_t x_peid, cudaStream_t st, cola_zip_rows **out, const char *who)
{
    std::vector<int32_t> ends((size_t)nparts * 4, 0);
    for (int32_t i = 0; i < nparts; i++) {
        const cola_zip_part &z = parts[i];
        COLA_REQUIRE(z.local_row_lb >= 0 && z.remote_col_lb >= 0 && z.local_row_num >= 0 && z.remote_col_num >= 0,
                     COLA_ERROR_INVALID_ARGUMENT, "%s: PE %d: negative chunk range", who, i);
        COLA_REQUIRE(z.local_row_num == 0 || (z.csr_rowPtr_l && z.csr_colIdx_l && z.csr_rowIdx_zip_l),
                     COLA_ERROR_INVALID_ARGUMENT, "%s: PE %d: null local CSR arrays", who, i);
        COLA_REQUIRE(z.remote_col_num == 0 || (z.csc_colPtr_r && z.csc_rowIdx_r && z.csc_colIdx_zip_r),
                     COLA_ERROR_INVALID_ARGUMENT, "%s: PE %d: null remote CSC arrays", who, i);
        // entry ranges of the chunks the call covers (chunk pointers are monotonic)
        if (z.local_row_num > 0) {
            COLA_TRY(read_i32(z.csr_rowPtr_l, z.local_row_lb, ends[(size_t)i * 4], st));
            COLA_TRY(read_i32(z.csr_rowPtr_l, (int64_t)z.local_row_lb + z.local_row_num, ends[(size_t)i * 4 + 1], st));
        }
        if (z.remote_col_num > 0) {
            COLA_TRY(read_i32(z.csc_colPtr_r, z.remote_col_lb, ends[(size_t)i * 4 + 2], st));
            COLA_TRY(read_i32(z.csc_colPtr_r, (int64_t)z.remote_col_lb + z.remote_col_num, ends[(size_t)i * 4 + 3],
                              st));
        }
    }
    COLA_CUDA(cudaStreamSynchronize(st));
    int64_t nnz = 0;
    for (int32_t i = 0; i < nparts; i++) {
        const int32_t *e = ends.data() + (size_t)i * 4;
        COLA_REQUIRE(e[1] >= e[0] && e[3] >= e[2], COLA_ERROR_INVALID_ARGUMENT, "%s: PE %d: chunk pointers decrease",
                     who, i);
        nnz += (int64_t)(e[1] - e[0]) + (e[3] - e[2]);
    }
    COLA_REQUIRE(nnz < (int64_t)INT32_MAX, COLA_ERROR_UNSUPPORTED, "%s: %lld entries (at most 2^31 - 1)", who,
                 (long long)nnz);

    void *arena = nullptr;
    const size_t a = 256, n = (size_t)std::max<int64_t>(nnz, 1);
    const size_t slice = (4 * n + a - 1) / a * a;
    COLA_CUDA(cudaMallocAsync(&arena, 3 * slice + a, st));
    char *base = static_cast<char *>(arena);
    int32_t *row = reinterpret_cast<int32_t *>(base);
    int32_t *col = reinterpret_cast<int32_t *>(base + slice);
    float *val = reinterpret_cast<float *>(base + 2 * slice);
    unsigned int *mx = reinterpret_cast<unsigned int *>(base + 3 * slice);  // max row, max col, all in range
    cola_status rc = COLA_SUCCESS;
    unsigned int h_mx[3] = {0, 0, 1};
    {
        const unsigned int init[3] = {0u, 0u, 1u};
        cudaError_t e = cudaMemcpyAsync(mx, init, sizeof init, cudaMemcpyHostToDevice, st);
        int64_t at = 0;
        for (int32_t i = 0; i < nparts && e == cudaSuccess; i++) {
            const cola_zip_part &z = parts[i];
            const int32_t *en = ends.data() + (size_t)i * 4;
            const int64_t nl = (int64_t)en[1] - en[0], nr = (int64_t)en[3] - en[2];
            if (nl > 0) {
                expand_chunks_kernel<<<blocks_for(nl), 256, 0, st>>>(
                    z.csr_rowPtr_l, z.csr_rowIdx_zip_l, z.csr_colIdx_l, z.csr_val_l, z.local_row_lb, z.local_row_num,
                    en[0], nl, (int64_t)peids[i] * nodesPerPE, row0[i], 0, row + at, col + at, val + at, mx, mx + 1,
                    mx + 2);
                e = cudaGetLastError();
                at += nl;
            }
            if (e == cudaSuccess && nr > 0) {
                expand_chunks_kernel<<<blocks_for(nr), 256, 0, st>>>(
                    z.csc_colPtr_r, z.csc_colIdx_zip_r, z.csc_rowIdx_r, z.csc_val_r, z.remote_col_lb,
                    z.remote_col_num, en[2], nr, 0, row0[i], 1, row + at, col + at, val + at, mx, mx + 1, mx + 2);
                e = cudaGetLastError();
                at += nr;
            }
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
    h->peid = x_peid;
    h->nnz = nnz;
    *out = h;
    return COLA_SUCCESS;
}

}  // namespace zr
}  // namespace cola

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
    COLA_REQUIRE(nodesPerPE >= 1 && peid >= 0, COLA_ERROR_INVALID_ARGUMENT, "%s: nodesPerPE %d, peid %d", who,
                 nodesPerPE, peid);
    const cola_zip_part z = {csr_rowPtr_l,  csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l,     csc_colPtr_r,
                             csc_rowIdx_r,  csc_colIdx_zip_r, csc_val_r,    local_row_lb,  remote_col_lb,
                             local_row_num, remote_col_num};
    const int64_t row0 = 0;
    return zr::build(&z, 1, &row0, nodesPerPE, &peid, peid, (cudaStream_t)stream, out, who);
}

cola_status cola_zip_rows_create_all(const cola_zip_part *parts, int32_t nparts, int32_t nodesPerPE,
                                     cola_stream_t stream, cola_zip_rows **out)
{
    const char *who = "cola_zip_rows_create_all";
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "%s: out is NULL", who);
    *out = nullptr;
    clear_error();
    COLA_REQUIRE(parts && nparts >= 1 && nodesPerPE >= 1, COLA_ERROR_INVALID_ARGUMENT,
                 "%s: %d PEs, nodesPerPE %d", who, nparts, nodesPerPE);
    std::vector<int64_t> row0((size_t)nparts);
    std::vector<int32_t> peids((size_t)nparts);
    for (int32_t i = 0; i < nparts; i++) {
        row0[(size_t)i] = (int64_t)i * nodesPerPE;
        peids[(size_t)i] = i;
    }
    return zr::build(parts, nparts, row0.data(), nodesPerPE, peids.data(), 0, (cudaStream_t)stream, out, who);
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
