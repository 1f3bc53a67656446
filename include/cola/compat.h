/*
 * cola/compat.h -- the reference's C++ surface (include/sparse_data.h and
 * include/dist_spmm_ppl_batch.cuh of zzzlxhhh/CoLa) on top of the cola_b200 C
 * ABI, so a caller written against those headers builds unchanged for one B200
 * with P virtual PEs.  Header-only host C++; link libcola_b200.so and cudart.
 *
 * Differences a caller sees:
 *  - errors throw cola_compat::error instead of calling exit();
 *  - the device holders cannot be copied (the reference's can, and then double
 *    free their memory);
 *  - CF / is_residue template arguments are accepted and ignored: the library
 *    dispatches on dim itself, for every dim >= 1 (the reference's wrapper
 *    launches nothing for dim 65-96 or dim > 128);
 *  - "symmetric" buffers (X slices, pipeline buffers) of the P virtual PEs must
 *    be laid out back to back, nodesPerPE*dim floats apart, in one allocation
 *    (see cola_spmm.h); NVSHMEM puts/gets become reads of that memory.
 *  - the multi-stage schedule (group_size < nranks) runs all PEs together:
 *    distSpMM_ppl_batch_all().  The per-PE wrapper supports group_size == nranks,
 *    which is what P virtual partitions on one GPU map to.
 *  - ppl0_batch_SpMM (and the wrapper, which calls it) on the arrays of a
 *    d_csr_zip / d_csc_zip pair builds, on its first call for that pair and
 *    chunk range, the pair's row view on the device (cola_zip_rows_create: it
 *    synchronises the stream once) and keeps it until either holder is
 *    destroyed; every call then runs the row-major schedule on it (one writer
 *    per row, no atomics, the same bits every call) instead of the chunk
 *    kernel.  The result is the same product; arrays not owned by a holder
 *    run the chunk kernel.  distSpMM_ppl_batch_all with a single stage does
 *    the same with one row view of every PE's chunks: one launch (plus one for
 *    hub rows) for all PEs.  cola_compat::set_row_view_cache(false) turns the
 *    cache off.
 */
#ifndef COLA_COMPAT_H
#define COLA_COMPAT_H

#include <cuda_runtime_api.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../cola_spmm.h"

namespace cola_compat {

struct error : std::runtime_error {
    cola_status status;
    error(cola_status s, const std::string &what) : std::runtime_error(what), status(s) {}
};

inline void check(cola_status s, const char *where)
{
    if (s != COLA_SUCCESS)
        throw error(s, std::string(where) + ": " + cola_status_string(s) + ": " + cola_last_error());
}

inline void check_cuda(cudaError_t e, const char *where)
{
    if (e != cudaSuccess)
        throw error(COLA_ERROR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

template <typename T>
inline T *upload(const std::vector<T> &v, const char *where)
{
    T *p = nullptr;
    check_cuda(cudaMalloc((void **)&p, v.size() * sizeof(T)), where);
    if (!v.empty())
        check_cuda(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), where);
    return p;
}

// Row views of d_csr_zip / d_csc_zip pairs, built on first use by
// ppl0_batch_SpMM and dropped when either holder is destroyed.  Holders enter
// the registry with their device arrays, so arrays a holder does not own are
// never looked up in it.
struct zip_registry {
    using arrays = std::tuple<const void *, const void *, const void *, const void *>;
    using view_key = std::tuple<const void *, const void *, int, int, int, int, int, int>;
    std::mutex mu;
    std::map<const void *, arrays> csr, csc;  // holder -> its four device arrays
    std::map<view_key, cola_zip_rows *> views;
    // all PEs at once: nparts, nodesPerPE, then per PE its two holders and four offsets
    std::map<std::vector<intptr_t>, cola_zip_rows *> all_views;
    bool enabled = true;
};

inline zip_registry &registry()
{
    static zip_registry r;
    return r;
}

inline void set_row_view_cache(bool on)
{
    std::lock_guard<std::mutex> lk(registry().mu);
    registry().enabled = on;
}

inline void register_holder(bool is_csr, const void *holder, zip_registry::arrays a)
{
    std::lock_guard<std::mutex> lk(registry().mu);
    (is_csr ? registry().csr : registry().csc)[holder] = a;
}

// Forget a holder and free the row views built on its arrays.
inline void forget_holder(bool is_csr, const void *holder)
{
    zip_registry &R = registry();
    std::lock_guard<std::mutex> lk(R.mu);
    (is_csr ? R.csr : R.csc).erase(holder);
    for (auto it = R.views.begin(); it != R.views.end();) {
        if ((is_csr ? std::get<0>(it->first) : std::get<1>(it->first)) == holder) {
            cola_zip_rows_free(it->second);
            it = R.views.erase(it);
        } else {
            ++it;
        }
    }
    for (auto it = R.all_views.begin(); it != R.all_views.end();) {
        bool uses = false;
        for (size_t i = 2; i < it->first.size(); i += 6)
            uses = uses || it->first[i + (is_csr ? 0 : 1)] == (intptr_t)holder;
        if (uses) {
            cola_zip_rows_free(it->second);
            it = R.all_views.erase(it);
        } else {
            ++it;
        }
    }
}

// The row view of every PE's single-stage call at once (PE p's holders and
// chunk ranges), built on first use, when every block belongs to a holder.
inline cola_zip_rows *cached_all_view(int nranks, int nodesPerPE, void *const *csr_holders,
                                      void *const *csc_holders, int *const *local_offset, int *const *remote_offset,
                                      cudaStream_t stream)
{
    zip_registry &R = registry();
    std::lock_guard<std::mutex> lk(R.mu);
    if (!R.enabled)
        return nullptr;
    std::vector<intptr_t> key{(intptr_t)nranks, (intptr_t)nodesPerPE};
    for (int p = 0; p < nranks; p++) {
        if (!R.csr.count(csr_holders[p]) || !R.csc.count(csc_holders[p]))
            return nullptr;
        key.insert(key.end(), {(intptr_t)csr_holders[p], (intptr_t)csc_holders[p], (intptr_t)local_offset[p][0],
                               (intptr_t)remote_offset[p][0], (intptr_t)(local_offset[p][1] - local_offset[p][0]),
                               (intptr_t)(remote_offset[p][1] - remote_offset[p][0])});
    }
    auto it = R.all_views.find(key);
    if (it != R.all_views.end())
        return it->second;
    std::vector<cola_zip_part> parts((size_t)nranks);
    for (int p = 0; p < nranks; p++) {
        const auto &l = R.csr[csr_holders[p]];
        const auto &r = R.csc[csc_holders[p]];
        cola_zip_part &z = parts[(size_t)p];
        z.csr_rowPtr_l = static_cast<const int32_t *>(std::get<0>(l));
        z.csr_colIdx_l = static_cast<const int32_t *>(std::get<1>(l));
        z.csr_rowIdx_zip_l = static_cast<const int32_t *>(std::get<2>(l));
        z.csr_val_l = static_cast<const float *>(std::get<3>(l));
        z.csc_colPtr_r = static_cast<const int32_t *>(std::get<0>(r));
        z.csc_rowIdx_r = static_cast<const int32_t *>(std::get<1>(r));
        z.csc_colIdx_zip_r = static_cast<const int32_t *>(std::get<2>(r));
        z.csc_val_r = static_cast<const float *>(std::get<3>(r));
        z.local_row_lb = local_offset[p][0];
        z.remote_col_lb = remote_offset[p][0];
        z.local_row_num = local_offset[p][1] - local_offset[p][0];
        z.remote_col_num = remote_offset[p][1] - remote_offset[p][0];
    }
    cola_zip_rows *h = nullptr;
    check(cola_zip_rows_create_all(parts.data(), nranks, nodesPerPE, (cola_stream_t)stream, &h),
          "distSpMM_ppl_batch_all (row view)");
    R.all_views[key] = h;
    return h;
}

// The row view for these arrays and chunk range when both blocks belong to
// holders (built now if this is the first call), else nullptr.
inline cola_zip_rows *cached_row_view(const int *csr_rowPtr_l, const int *csr_colIdx_l, const int *csr_rowIdx_zip_l,
                                      const float *csr_val_l, const int *csc_colPtr_r, const int *csc_rowIdx_r,
                                      const int *csc_colIdx_zip_r, const float *csc_val_r, int local_row_lb,
                                      int remote_col_lb, int local_row_num, int remote_col_num, int nodesPerPE,
                                      int peid, cudaStream_t stream)
{
    zip_registry &R = registry();
    std::lock_guard<std::mutex> lk(R.mu);
    if (!R.enabled)
        return nullptr;
    const zip_registry::arrays want_l{csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l};
    const zip_registry::arrays want_r{csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r};
    const void *hl = nullptr, *hr = nullptr;
    for (const auto &kv : R.csr)
        if (kv.second == want_l)
            hl = kv.first;
    for (const auto &kv : R.csc)
        if (kv.second == want_r)
            hr = kv.first;
    if (!hl || !hr)
        return nullptr;
    const zip_registry::view_key k{hl, hr, local_row_lb, remote_col_lb, local_row_num, remote_col_num, nodesPerPE,
                                   peid};
    auto it = R.views.find(k);
    if (it != R.views.end())
        return it->second;
    cola_zip_rows *h = nullptr;
    check(cola_zip_rows_create(csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r, csc_rowIdx_r,
                               csc_colIdx_zip_r, csc_val_r, local_row_lb, remote_col_lb, local_row_num,
                               remote_col_num, nodesPerPE, peid, (cola_stream_t)stream, &h),
          "ppl0_batch_SpMM (row view)");
    R.views[k] = h;
    return h;
}

}  // namespace cola_compat

/* include/sparse_data.h:6-27 */
struct d_csr {
    int *d_csr_rowPtr = nullptr;
    int *d_csr_colIdx = nullptr;
    float *d_csr_val = nullptr;
    d_csr(std::vector<int> rowPtr, std::vector<int> colIdx, std::vector<float> val)
    {
        d_csr_rowPtr = cola_compat::upload(rowPtr, "d_csr");
        d_csr_colIdx = cola_compat::upload(colIdx, "d_csr");
        d_csr_val = cola_compat::upload(val, "d_csr");
    }
    d_csr(const d_csr &) = delete;
    d_csr &operator=(const d_csr &) = delete;
    ~d_csr()
    {
        cudaFree(d_csr_rowPtr);
        cudaFree(d_csr_colIdx);
        cudaFree(d_csr_val);
    }
};

/* include/sparse_data.h:28-52 */
struct d_csc_zip {
    int *d_csc_colPtr = nullptr;
    int *d_csc_rowIdx = nullptr;
    int *d_csc_colIdx_zip = nullptr;
    float *d_csc_val = nullptr;
    d_csc_zip(std::vector<int> colPtr, std::vector<int> rowIdx, std::vector<int> colIdx_zip, std::vector<float> val)
    {
        d_csc_colPtr = cola_compat::upload(colPtr, "d_csc_zip");
        d_csc_rowIdx = cola_compat::upload(rowIdx, "d_csc_zip");
        d_csc_colIdx_zip = cola_compat::upload(colIdx_zip, "d_csc_zip");
        d_csc_val = cola_compat::upload(val, "d_csc_zip");
        cola_compat::register_holder(false, this, {d_csc_colPtr, d_csc_rowIdx, d_csc_colIdx_zip, d_csc_val});
    }
    d_csc_zip(const d_csc_zip &) = delete;
    d_csc_zip &operator=(const d_csc_zip &) = delete;
    ~d_csc_zip()
    {
        cola_compat::forget_holder(false, this);
        cudaFree(d_csc_colPtr);
        cudaFree(d_csc_rowIdx);
        cudaFree(d_csc_colIdx_zip);
        cudaFree(d_csc_val);
    }
};

/* include/sparse_data.h:54-77 */
struct d_csr_zip {
    int *d_csr_rowPtr = nullptr;
    int *d_csr_colIdx = nullptr;
    int *d_csr_rowIdx_zip = nullptr;
    float *d_csr_val = nullptr;
    d_csr_zip(std::vector<int> rowPtr, std::vector<int> colIdx, std::vector<int> rowIdx_zip, std::vector<float> val)
    {
        d_csr_rowPtr = cola_compat::upload(rowPtr, "d_csr_zip");
        d_csr_colIdx = cola_compat::upload(colIdx, "d_csr_zip");
        d_csr_rowIdx_zip = cola_compat::upload(rowIdx_zip, "d_csr_zip");
        d_csr_val = cola_compat::upload(val, "d_csr_zip");
        cola_compat::register_holder(true, this, {d_csr_rowPtr, d_csr_colIdx, d_csr_rowIdx_zip, d_csr_val});
    }
    d_csr_zip(const d_csr_zip &) = delete;
    d_csr_zip &operator=(const d_csr_zip &) = delete;
    ~d_csr_zip()
    {
        cola_compat::forget_holder(true, this);
        cudaFree(d_csr_rowPtr);
        cudaFree(d_csr_colIdx);
        cudaFree(d_csr_rowIdx_zip);
        cudaFree(d_csr_val);
    }
};

/* include/dist_spmm_ppl_batch.cuh:7-27 (64-bit sizes; throws instead of exit) */
template <typename T>
std::vector<T> bin2vec(const std::string filename)
{
    static_assert(sizeof(T) == 4, "bin2vec: 4-byte element types only");
    int64_t n = 0;
    cola_compat::check(cola_bin_read_i32(filename.c_str(), nullptr, 0, &n), "bin2vec");
    std::vector<T> v((size_t)n);
    cola_compat::check(cola_bin_read_i32(filename.c_str(), reinterpret_cast<int32_t *>(v.data()), n, &n),
                       "bin2vec");
    return v;
}

/* include/dist_spmm_ppl_batch.cuh:29-56 */
inline void nnz_split(std::vector<int> &rowIdx, std::vector<int> &rowPtr, std::vector<int> &colIdx,
                      std::vector<int> &target, std::vector<int> &ptr, const int peid, bool local)
{
    int64_t n = 0;
    cola_compat::check(cola_nnz_split(rowIdx.data(), (int64_t)rowIdx.size(), rowPtr.data(), (int64_t)colIdx.size(),
                                      nullptr, nullptr, 0, &n),
                       "nnz_split");
    size_t t0 = target.size(), p0 = ptr.size();
    target.resize(t0 + (size_t)n);
    ptr.resize(p0 + (rowIdx.empty() ? 0 : (size_t)n + 1));
    if (!rowIdx.empty())
        cola_compat::check(cola_nnz_split(rowIdx.data(), (int64_t)rowIdx.size(), rowPtr.data(),
                                          (int64_t)colIdx.size(), target.data() + t0, ptr.data() + p0, n, &n),
                           "nnz_split");
    if (!rowIdx.empty())
        printf("PE-%d, %s_split_ratio:%.3f \n", peid, local ? "l" : "r", (float)n / rowIdx.size());
}

/* include/dist_spmm_ppl_batch.cuh:59-73 as a host call (launch shape is the library's) */
inline void batching_data_ppl(const float *input_nvsh, float *ppl_send_nvsh, int *put_colIdx, const int nemb,
                              const int dim, const int nodesPerPE, const int group_size, cudaStream_t stream)
{
    cola_compat::check(cola_batching_data_ppl(input_nvsh, ppl_send_nvsh, put_colIdx, nemb, dim, nodesPerPE,
                                              group_size, (cola_stream_t)stream),
                       "batching_data_ppl");
}

/* include/dist_spmm_ppl_batch.cuh:202-245 */
template <int CF, bool is_residue>
void ppl0_batch_SpMM(float *output, const float *input, const int *csr_rowPtr_l, const int *csr_colIdx_l,
                     const int *csr_rowIdx_zip_l, const float *csr_val_l, const int *csc_colPtr_r,
                     const int *csc_rowIdx_r, const int *csc_colIdx_zip_r, const float *csc_val_r,
                     const int local_row_lb, const int remote_col_lb, const int local_row_num,
                     const int remote_col_num, const int dim, const int nodesPerPE, const int peid,
                     cudaStream_t stream)
{
    if (cola_zip_rows *h = cola_compat::cached_row_view(csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l,
                                                        csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r,
                                                        local_row_lb, remote_col_lb, local_row_num, remote_col_num,
                                                        nodesPerPE, peid, stream)) {
        cola_compat::check(cola_zip_rows_spmm(h, output, input, dim, (cola_stream_t)stream), "ppl0_batch_SpMM");
        return;
    }
    cola_compat::check(cola_ppl0_batch_spmm(output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l,
                                            csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb,
                                            remote_col_lb, local_row_num, remote_col_num, dim, nodesPerPE, peid,
                                            (cola_stream_t)stream),
                       "ppl0_batch_SpMM");
}

/* include/dist_spmm_ppl_batch.cuh:543-587 */
template <int CF, bool is_residue>
void ppl0_batch_SpMM_seq(float *output, const float *input, const int *csr_rowPtr_l, const int *csr_colIdx_l,
                         const int *csr_rowIdx_zip_l, const float *csr_val_l, const int *csc_colPtr_r,
                         const int *csc_rowIdx_r, const int *csc_colIdx_zip_r, const float *csc_val_r,
                         const int local_row_lb, const int remote_col_lb, const int local_row_num,
                         const int remote_col_num, const int dim, const int nodesPerPE, const int peid,
                         cudaStream_t stream)
{
    cola_compat::check(cola_ppl0_batch_spmm_seq(output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l,
                                                csr_val_l, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r,
                                                local_row_lb, remote_col_lb, local_row_num, remote_col_num, dim,
                                                nodesPerPE, peid, (cola_stream_t)stream),
                       "ppl0_batch_SpMM_seq");
}

/* include/dist_spmm_ppl_batch.cuh:373-417 */
template <int CF, bool is_residue>
void ppl0_batch_buffer_SpMM(float *output, const float *input, const float *comm_buffer, const int *csr_rowPtr_l,
                            const int *csr_colIdx_l, const int *csr_rowIdx_zip_l, const float *csr_val_l,
                            const int *csc_colPtr_r, const int *csc_rowIdx_r, const int *csc_colIdx_zip_r,
                            const float *csc_val_r, const int local_row_lb, const int remote_col_lb,
                            const int local_row_num, const int remote_col_num, const int dim, const int nodesPerPE,
                            const int peid, cudaStream_t stream)
{
    cola_compat::check(cola_ppl0_batch_buffer_spmm(output, input, const_cast<float *>(comm_buffer), csr_rowPtr_l,
                                                   csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l, csc_colPtr_r,
                                                   csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb,
                                                   remote_col_lb, local_row_num, remote_col_num, dim, nodesPerPE,
                                                   peid, (cola_stream_t)stream),
                       "ppl0_batch_buffer_SpMM");
}

/* include/dist_spmm_ppl_batch.cuh:709-760 */
template <int CF, bool is_residue>
void ppl_batch_SpMM(float *output, const float *input, const int *csc_colPtr_r, const int *csc_rowIdx_r,
                    const int *csc_colIdx_zip_r, const float *csc_val_r, const int local_col_lb,
                    const int local_col_ub, const int remote_col_lb, const int remote_col_ub, const int stage,
                    const int *idx_ppl, const int dim, const int nodesPerPE, const int group_size,
                    const int group_offset, const int peid, cudaStream_t stream)
{
    cola_compat::check(cola_ppl_batch_spmm(output, input, csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r,
                                           local_col_lb, local_col_ub, remote_col_lb, remote_col_ub, stage, idx_ppl,
                                           dim, nodesPerPE, group_size, group_offset, peid, (cola_stream_t)stream),
                       "ppl_batch_SpMM");
}

/* include/dist_spmm_ppl_batch.cuh:851-918, one virtual PE, single stage.
 * The reference routes group_size == nranks > 8 through the buffer kernel with
 * CF = 1 (:872-883); here that case runs the same fused kernel (the result is
 * the same; comm_buffer is not needed). */
inline void distSpMM_ppl_batch_wrapper(const int group_size, float *output, const float *input_nvsh,
                                       float **ppl_buffer_nvsh, float *ppl_send_nvsh, float *comm_buffer_nvsh,
                                       int *local_offset_ppl, int *remote_offset_ppl, int *put_offset_ppl,
                                       int **put_colIdx_ppl, int **idx_ppl, d_csr_zip *csr_zip_l,
                                       d_csc_zip *csc_zip_r, const int block_lb, const int block_ub, const int dim,
                                       const int nodesPerPE, const int nranks, const int mype_node,
                                       cudaStream_t stream)
{
    (void)ppl_buffer_nvsh;
    (void)ppl_send_nvsh;
    (void)comm_buffer_nvsh;
    (void)put_offset_ppl;
    (void)put_colIdx_ppl;
    (void)idx_ppl;
    (void)block_lb;
    (void)block_ub;
    if (group_size != nranks)
        throw cola_compat::error(COLA_ERROR_UNSUPPORTED,
                                 "distSpMM_ppl_batch_wrapper: on one GPU the multi-stage schedule runs all virtual PEs "
                                 "together; call distSpMM_ppl_batch_all()");
    ppl0_batch_SpMM<1, false>(output, input_nvsh, csr_zip_l->d_csr_rowPtr, csr_zip_l->d_csr_colIdx,
                              csr_zip_l->d_csr_rowIdx_zip, csr_zip_l->d_csr_val, csc_zip_r->d_csc_colPtr,
                              csc_zip_r->d_csc_rowIdx, csc_zip_r->d_csc_colIdx_zip, csc_zip_r->d_csc_val,
                              local_offset_ppl[0], remote_offset_ppl[0], local_offset_ppl[1] - local_offset_ppl[0],
                              remote_offset_ppl[1] - remote_offset_ppl[0], dim, nodesPerPE, mype_node, stream);
}

/* The multi-stage schedule of include/dist_spmm_ppl_batch.cuh:785-836 for all
 * nranks virtual PEs at once, in lockstep: stage 0 of every PE, then per stage
 * i >= 1 every PE's put (a staged gather straight into the target PE's
 * pipeline buffer) followed by every PE's stage-i compute.  Arrays are indexed
 * by PE: offsets[pe] are the per-PE host tables of src/distSpMM_ppl_batch.cu,
 * put_colIdx_ppl[pe][i] / idx_ppl[pe][i] device lists.  input_nvsh and
 * output point at PE 0's slices; ppl_buffer_nvsh[0..1] at PE 0's copies of the
 * two pipeline buffers (each holds nranks*nodesPerPE*dim floats). */
inline void distSpMM_ppl_batch_all(const int group_size, float *output, const float *input_nvsh,
                                   float **ppl_buffer_nvsh, int **local_offset_ppl, int **remote_offset_ppl,
                                   int **put_offset_ppl, int ***put_colIdx_ppl, int ***idx_ppl,
                                   d_csr_zip **csr_zip_l, d_csc_zip **csc_zip_r, const int dim, const int nodesPerPE,
                                   const int nranks, cudaStream_t stream)
{
    const int nstages = nranks / group_size;
    const long long pe = (long long)nodesPerPE * dim;
    if (nstages == 1) {
        // one stage: every PE's chunks in one row view, one launch for all of them
        std::vector<void *> hl((size_t)nranks), hr((size_t)nranks);
        for (int me = 0; me < nranks; me++) {
            hl[(size_t)me] = csr_zip_l[me];
            hr[(size_t)me] = csc_zip_r[me];
        }
        if (cola_zip_rows *h = cola_compat::cached_all_view(nranks, nodesPerPE, hl.data(), hr.data(),
                                                             local_offset_ppl, remote_offset_ppl, stream)) {
            cola_compat::check(cola_zip_rows_spmm(h, output, input_nvsh, dim, (cola_stream_t)stream),
                               "distSpMM_ppl_batch_all");
            return;
        }
    }
    for (int me = 0; me < nranks; me++)
        ppl0_batch_SpMM<1, false>(output + me * pe, input_nvsh + me * pe, csr_zip_l[me]->d_csr_rowPtr,
                                  csr_zip_l[me]->d_csr_colIdx, csr_zip_l[me]->d_csr_rowIdx_zip,
                                  csr_zip_l[me]->d_csr_val, csc_zip_r[me]->d_csc_colPtr, csc_zip_r[me]->d_csc_rowIdx,
                                  csc_zip_r[me]->d_csc_colIdx_zip, csc_zip_r[me]->d_csc_val,
                                  local_offset_ppl[me][0], remote_offset_ppl[me][0],
                                  local_offset_ppl[me][1] - local_offset_ppl[me][0],
                                  remote_offset_ppl[me][1] - remote_offset_ppl[me][0], dim, nodesPerPE, me, stream);
    for (int i = 1; i < nstages; i++) {
        float *buf = ppl_buffer_nvsh[(i - 1) % 2];
        for (int me = 0; me < nranks; me++) {
            const int target = ((me - i * group_size) % nranks + nranks) % nranks;
            const int nemb = put_offset_ppl[me][2 * (i - 1) + 1] - put_offset_ppl[me][2 * (i - 1)];
            batching_data_ppl(input_nvsh + me * pe, buf + target * pe, put_colIdx_ppl[me][i - 1], nemb, dim,
                              nodesPerPE, group_size, stream);
        }
        for (int me = 0; me < nranks; me++)
            ppl_batch_SpMM<1, false>(output + me * pe, buf + me * pe, csc_zip_r[me]->d_csc_colPtr,
                                     csc_zip_r[me]->d_csc_rowIdx, csc_zip_r[me]->d_csc_colIdx_zip,
                                     csc_zip_r[me]->d_csc_val, local_offset_ppl[me][2 * i],
                                     local_offset_ppl[me][2 * i + 1], remote_offset_ppl[me][2 * i],
                                     remote_offset_ppl[me][2 * i + 1], i, idx_ppl[me][i - 1], dim, nodesPerPE,
                                     group_size, me / group_size * group_size, me, stream);
    }
}

/* include/utils.cuh:45-69: the unweighted host reference of rows [lb, ub):
 * C_ref[i, :] = sum over the row's stored columns k of B[k, :] (values are not
 * read; the reference's are all 1). */
template <typename Index, typename DType>
void SAG_reference_host(int lb, int ub, int N, const Index *csr_indptr, const int *csr_indices, const DType *B,
                        DType *C_ref, int peid)
{
    (void)peid;
    const int64_t M = ub > lb ? ub - lb : 0;
    for (int64_t x = 0; x < M * (int64_t)N; x++)
        C_ref[x] = DType(0);
    for (int64_t i = 0; i < M; i++) {
        DType *c = C_ref + i * N;
        for (Index p = csr_indptr[lb + i]; p < csr_indptr[lb + i + 1]; p++) {
            const DType *b = B + (int64_t)csr_indices[p] * N;
            for (int64_t j = 0; j < N; j++)
                c[j] += b[j];
        }
    }
}

/* include/utils.cuh:71-101: element-wise check with relative tolerance 1e-2.
 * Prints the first 33 mismatches as the reference does; returns whether all
 * elements passed (the reference exits the process after 33 mismatches). */
template <typename DType>
bool check_result(int M, int N, const DType *C, const DType *C_ref, int PEid)
{
    int64_t bad = 0;
    for (int64_t i = 0; i < M; i++)
        for (int64_t j = 0; j < N; j++) {
            const double c = (double)C[i * N + j], r = (double)C_ref[i * N + j];
            if (!(std::fabs(c - r) <= 1e-2 * std::fabs(r))) {
                if (bad <= 32)
                    printf("peid-%d Wrong result: i = %lld, j = %lld, result = %lf, reference = %lf.\n", PEid,
                           (long long)i, (long long)j, c, r);
                bad++;
            }
        }
    if (bad == 0)
        printf("PEid-%d passed\n", PEid);
    return bad == 0;
}

/* include/dist_spmm_ppl_batch.cuh:920-987 for one virtual PE: one SpMM into
 * `output` (accumulated, as the reference's kernels do), then optionally a
 * validation of rows [block_lb, block_ub) against SAG_reference_host over the
 * global CSR with host features h_in (the caller zeroes output first, as the
 * reference's main does), then optionally 200 timed SpMMs after warm-up,
 * timed with CUDA events on `stream` (the reference: MPI_Wtime between
 * barriers).  Returns the average milliseconds per SpMM when profiling, else
 * 0; throws cola_compat::error when validation fails. */
template <bool validate, bool profiling, bool profile_detail = false>
double run_distSpMM_ppl_batch(const int group_size, float *output, const float *input_nvsh, float **ppl_buffer_nvsh,
                              float *ppl_send_nvsh, float *comm_buffer_nvsh, int *local_offset_ppl,
                              int *remote_offset_ppl, int *put_offset_ppl, int **put_colIdx_ppl, int **idx_ppl,
                              d_csr_zip *csr_zip_l, d_csc_zip *csc_zip_r, const int block_lb, const int block_ub,
                              const int dim, const int nodesPerPE, const int nranks, const int mype_node,
                              const int *global_rowPtr, const int *global_colIdx, const float *h_in,
                              cudaStream_t stream)
{
    if (mype_node == 0 && (validate || profiling))
        printf("Running ppl_batch SpMM with group_size:%d\n", group_size);
    auto once = [&]() {
        distSpMM_ppl_batch_wrapper(group_size, output, input_nvsh, ppl_buffer_nvsh, ppl_send_nvsh, comm_buffer_nvsh,
                                   local_offset_ppl, remote_offset_ppl, put_offset_ppl, put_colIdx_ppl, idx_ppl,
                                   csr_zip_l, csc_zip_r, block_lb, block_ub, dim, nodesPerPE, nranks, mype_node,
                                   stream);
    };
    once();
    cola_compat::check_cuda(cudaStreamSynchronize(stream), "run_distSpMM_ppl_batch");
    if (validate) {
        const int M = block_ub - block_lb;
        std::vector<float> out((size_t)M * dim), ref((size_t)M * dim);
        SAG_reference_host<int, float>(block_lb, block_ub, dim, global_rowPtr, global_colIdx, h_in, ref.data(),
                                       mype_node);
        cola_compat::check_cuda(cudaMemcpy(out.data(), output, out.size() * sizeof(float), cudaMemcpyDeviceToHost),
                                "run_distSpMM_ppl_batch");
        if (!check_result(M, dim, out.data(), ref.data(), mype_node))
            throw cola_compat::error(COLA_ERROR_INVALID_ARGUMENT, "run_distSpMM_ppl_batch: validation failed");
    }
    double ms = 0.0;
    if (profiling) {
        const int num_profiling = 200;
        for (int i = 0; i < 50; i++)
            once();
        cudaEvent_t e0, e1;
        cola_compat::check_cuda(cudaEventCreate(&e0), "run_distSpMM_ppl_batch");
        cola_compat::check_cuda(cudaEventCreate(&e1), "run_distSpMM_ppl_batch");
        cola_compat::check_cuda(cudaEventRecord(e0, stream), "run_distSpMM_ppl_batch");
        for (int i = 0; i < num_profiling; i++)
            once();
        cola_compat::check_cuda(cudaEventRecord(e1, stream), "run_distSpMM_ppl_batch");
        cola_compat::check_cuda(cudaEventSynchronize(e1), "run_distSpMM_ppl_batch");
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        ms = (double)t / num_profiling;
        if (mype_node == 0) {
            printf("nodesPerPE:%d\n", nodesPerPE);
            printf("PE-%d time (ms) %.3f\n", mype_node, ms);
        }
    }
    return ms;
}

#endif /* COLA_COMPAT_H */
