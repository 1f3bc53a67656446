// Internal: the device-resident graph and the launch helpers shared by the
// translation units of the library (not part of the C ABI).
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "prep.h"
#include "spmm_kernels.cuh"

namespace cola {

#define COLA_CUDA(expr)                                                                                   \
    do {                                                                                                  \
        cudaError_t _e = (expr);                                                                          \
        if (_e != cudaSuccess)                                                                            \
            return ::cola::fail(_e == cudaErrorMemoryAllocation ? COLA_ERROR_OUT_OF_MEMORY : COLA_ERROR_CUDA, \
                                "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__);    \
    } while (0)

// Kernel launches issued by this thread (cola_spmm reports the count of its last call).
extern thread_local int64_t t_launches;

int sm_count();
// Resident blocks per SM for a kernel (cached by function address).
int blocks_per_sm(const void *fn, int threads);
// Persistent grid: enough warps for `items`, at most one full wave.
int64_t grid_for(const void *fn, int64_t items);
inline bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }
// Vector path of the row-major schedule for these operands.
bool vec_ok_rows(cola_dtype xdt, const void *X, int64_t ldx, cola_dtype ydt, const void *Y, int64_t ldy, int K);
// Grow a device allocation to at least `need` bytes (contents not kept).
cola_status ensure(void *&p, size_t &have, size_t need);

}  // namespace cola

using cola::dev::GatherSeg;
using cola::dev::PartDesc;

namespace cola {
struct HostPipe;  // cola_spmm_host's staging sets and copy streams
void host_pipe_release(HostPipe *p);
}  // namespace cola

struct cola_graph {
    int device = 0;
    int32_t N = 0, P = 0, npp = 0, gs = 0, nstages = 1, if_split = 1;
    int64_t nnz_l = 0, nnz_r = 0, lchunks = 0, rchunks = 0, rcols = 0;
    void *dmem = nullptr;
    size_t dbytes = 0;
    std::vector<cola_zip_view> zips;
    // fused schedule: all parts, all chunks
    PartDesc *d_fused = nullptr;
    int64_t fused_total = 0;
    std::vector<PartDesc> h_fused;
    // pipelined schedule (group_size < P)
    std::vector<cola::StageTables> tables;
    PartDesc *d_stage0 = nullptr;  // local + intra-group remote of every PE
    int64_t stage0_total = 0;
    std::vector<PartDesc *> d_stage;  // stage s >= 1 (index s-1), mode 2
    std::vector<int64_t> stage_total;
    std::vector<std::vector<PartDesc>> h_stage;
    std::vector<GatherSeg *> d_put;  // puts feeding stage s (index s-1)
    std::vector<int64_t> put_total;
    std::vector<std::vector<GatherSeg>> h_put;
    // lazily sized workspaces
    void *ppl_buf = nullptr;  // 2 x P x npp x K elements
    size_t ppl_bytes = 0;
    void *stage_buf = nullptr;  // BUFFER schedule staging
    size_t stage_bytes = 0;
    float *ws = nullptr;  // FP32 accumulator for BF16 output
    size_t ws_bytes = 0;
    int64_t last_launches = 0;       // kernels launched by the last cola_spmm call
    GatherSeg *d_bufsegs = nullptr;  // BUFFER schedule gather segments
    std::vector<GatherSeg> h_bufsegs;
    // the split local CSR / remote CSC blocks (FUSED, BUFFER, PIPELINE, zip
    // views); false for a graph built on the device, which has the row view only
    bool has_split = true;
    // row-major view (ROWS schedule): merged local + transposed remote entries
    bool has_rows = false;
    const int64_t *rv_ptr = nullptr;  // N+1
    const int32_t *rv_col = nullptr;
    const float *rv_val = nullptr;
    const int32_t *seg_row = nullptr;
    const int64_t *seg_beg = nullptr;
    const int32_t *hub_row = nullptr;
    const int64_t *hub_seg = nullptr;
    const int32_t *task_rb = nullptr, *task_re = nullptr;
    int64_t nseg = 0, nhub = 0, ntask = 0;
    int32_t hub_threshold = 256, hub_segment = 256, task_entries = 128;
    float *ws_hub = nullptr;  // nseg x K partials
    // dev::kMaxItemQueues + 1 work-item counters of the row-major schedule,
    // in dmem, zero between launches
    unsigned int *item_queue = nullptr;
    size_t ws_hub_bytes = 0;
    cola::HostPipe *host_pipe = nullptr;  // created by the first cola_spmm_host call
};

namespace cola {
void graph_release(cola_graph *g);

// Row view parameters: the caller's cola_upload_opts fields where non-zero,
// else chosen by the graph's size: with W warps in a full wave (32 per SM),
// T = 512 when each still draws 16 or more 512-entry items (nnz >= 512 x 16 x
// W), T = 128 when fewer than 4 128-entry items each (nnz < 128 x 4 x W), else
// 256; rows longer than T entries are cut into T-entry segments, the other
// rows packed into row blocks of about T / 2 entries.  Measured with the
// dynamic item schedule: T = 512 is 2-5 % faster than 256 on a scale-21 R-MAT
// graph (94 M entries, BF16 features), the same at scale 20 (31 M); T = 128 is
// faster than 256 on graphs of 0.46 and 1.4 M entries and slower at 4.4 and
// 13 M (the per-partition views of the scale-20 graph).
struct RowViewParams {
    int32_t hub_threshold, hub_segment, task_entries;
};
RowViewParams row_view_params(int64_t nnz, const cola_upload_opts *opts);
// The row-view graph of an nrows x ncols COO in device memory (entries sorted
// by (row, col), duplicates merged, hub segments and row-block tasks), for
// the row-major schedule; ncols >= nrows.
cola_status graph_build_device_rect(int32_t nrows, int32_t ncols, int64_t nnz, const int32_t *row, const int32_t *col,
                                    const float *val, const cola_upload_opts *opts, cudaStream_t st, cola_graph *&out,
                                    const char *who);
cola_status graph_upload(const cola_partition_set *ps, const cola_upload_opts *opts, cola_graph *&out,
                         cudaStream_t st);
}  // namespace cola
