// Batched form of the partitioned SpMM: many graphs of uneven size, each with
// its own dense operands and feature width, in one persistent launch (plus one
// for hub rows), capturable in a CUDA graph; and the launch-parameter autotuner.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "graph.h"
#include "batch.h"
#include "spmm_batch.cuh"
#include "tune_cache.h"

using cola::dev::BatchGraph;
static_assert(cola::kBatchQueueBytes >= (cola::dev::kMaxItemQueues + 1) * sizeof(unsigned int),
              "the batch counters must hold the kernel's counters");

struct cola_batch {
    int device = 0;
    std::vector<cola_graph *> graphs;
    bool own_graphs = true;
    // bound operands
    bool bound = false;
    cola_dtype xdt = COLA_FLOAT32, ydt = COLA_FLOAT32;
    std::vector<BatchGraph> h_desc;  // graphs that run in the batched launch
    BatchGraph *d_desc = nullptr;
    size_t d_desc_bytes = 0;
    int64_t total_items = 0, total_hub = 0;
    struct Solo {  // graphs that run through cola_spmm (scalar path or K > 32 vectors)
        int g;
        const void *X;
        int64_t ldx;
        void *Y;
        int64_t ldy;
        int32_t K;
    };
    std::vector<Solo> solo;
    // launch parameters (autotuned)
    int32_t unroll = 4;
    int32_t grid_pct = 100;  // persistent grid as a percentage of one full wave
    int32_t blocks_per_sm = 4;
    // captured CUDA graph
    cudaGraph_t cgraph = nullptr;
    cudaGraphExec_t cexec = nullptr;
    int64_t last_launches = 0;
};

namespace cola {

static void batch_release(cola_batch *b)
{
    if (!b)
        return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(b->device);
    if (b->cexec)
        cudaGraphExecDestroy(b->cexec);
    if (b->cgraph)
        cudaGraphDestroy(b->cgraph);
    cudaFree(b->d_desc);
    if (b->own_graphs)
        for (cola_graph *g : b->graphs)
            graph_release(g);
    cudaSetDevice(cur);
    delete b;
}

template <typename TR, typename TY, int UNROLL, int MINB>
static cola_status launch_batch_t(const BatchLaunch &L, cudaStream_t st)
{
    const bool dyn = L.queue && L.total_items < INT32_MAX;
    auto fn = dyn ? dev::batch_rowblock_kernel<TR, TY, UNROLL, MINB, true>
                  : dev::batch_rowblock_kernel<TR, TY, UNROLL, MINB, false>;
    int64_t gx = grid_for((const void *)fn, L.total_items);
    gx = std::max<int64_t>(1, gx * L.grid_pct / 100);
    t_launches++;
    fn<<<(unsigned)gx, dev::kThreads, 0, st>>>(L.desc, L.ngraphs, L.total_items, L.accumulate,
                                               dyn ? L.queue : nullptr);
    COLA_CUDA(cudaGetLastError());
    return COLA_SUCCESS;
}

template <typename TR, typename TY>
static cola_status launch_batch_u(const BatchLaunch &L, cudaStream_t st)
{
    if (L.blocks_per_sm == 3)
        return L.unroll == 2 ? launch_batch_t<TR, TY, 2, 3>(L, st) : launch_batch_t<TR, TY, 4, 3>(L, st);
    return L.unroll == 2 ? launch_batch_t<TR, TY, 2, 4>(L, st) : launch_batch_t<TR, TY, 4, 4>(L, st);
}

cola_status launch_batch(const BatchLaunch &L, cudaStream_t st)
{
    using BF = __nv_bfloat16;
    if (L.total_items > 0) {
        cola_status s;
        if (L.xdt == COLA_FLOAT32)
            s = L.ydt == COLA_FLOAT32 ? launch_batch_u<dev::VecTraits<float>, float>(L, st)
                                      : launch_batch_u<dev::VecTraits<float>, BF>(L, st);
        else
            s = L.ydt == COLA_FLOAT32 ? launch_batch_u<dev::VecTraits<BF>, float>(L, st)
                                      : launch_batch_u<dev::VecTraits<BF>, BF>(L, st);
        COLA_TRY(s);
    }
    if (L.total_hub > 0) {
        const int64_t blocks = std::min<int64_t>((L.total_hub + dev::kWarpsPerBlock - 1) / dev::kWarpsPerBlock,
                                                 (int64_t)sm_count() * 16);
        t_launches++;
        if (L.ydt == COLA_FLOAT32)
            dev::batch_hub_combine_kernel<float, 4><<<(unsigned)blocks, dev::kThreads, 0, st>>>(
                L.desc, L.ngraphs, L.total_hub, L.accumulate);
        else
            dev::batch_hub_combine_kernel<BF, 4><<<(unsigned)blocks, dev::kThreads, 0, st>>>(
                L.desc, L.ngraphs, L.total_hub, L.accumulate);
        COLA_CUDA(cudaGetLastError());
    }
    return COLA_SUCCESS;
}

void fill_batch_graph(BatchGraph &d, const cola_graph *g, const void *X, int64_t ldx, void *Y, int64_t ldy, int32_t K,
                      cola_dtype xdt, float *ws)
{
    std::memset(&d, 0, sizeof d);
    d.ba.rowptr = g->rv_ptr;
    d.ba.col = g->rv_col;
    d.ba.val = g->rv_val;
    d.ba.task_rb = g->task_rb;
    d.ba.task_re = g->task_re;
    d.ba.ntask = g->ntask;
    d.ba.seg_row = g->seg_row;
    d.ba.seg_beg = g->seg_beg;
    d.ba.nseg = g->nseg;
    d.ba.seg_len = g->hub_segment;
    d.ba.queue = nullptr;  // the batch kernel assigns items statically
    d.ba.ws = ws;
    d.ba.ld_ws = K;
    d.X = X;
    d.ldx = ldx;
    d.Y = Y;
    d.ldy = ldy;
    d.K = K;
    d.lg = dev::batch_lane_width(K, xdt == COLA_FLOAT32 ? 4 : 8);
    d.hub_row = g->hub_row;
    d.hub_seg = g->hub_seg;
    d.nhub = g->nhub;
}

static cola_status batch_run(cola_batch *b, const cola_spmm_opts *opts, cudaStream_t st)
{
    COLA_REQUIRE(b->bound, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_run: bind the dense operands first");
    const int accumulate = opts ? opts->accumulate : 0;
    COLA_REQUIRE(!(accumulate && b->ydt != COLA_FLOAT32), COLA_ERROR_UNSUPPORTED,
                 "cola_batch_run: accumulate needs FP32 outputs");
    const int64_t before = t_launches;
    BatchLaunch L;
    L.desc = b->d_desc;
    L.ngraphs = (int)b->h_desc.size();
    L.total_items = b->total_items;
    L.total_hub = b->total_hub;
    L.xdt = b->xdt;
    L.ydt = b->ydt;
    L.unroll = b->unroll;
    L.grid_pct = b->grid_pct;
    L.blocks_per_sm = b->blocks_per_sm;
    L.accumulate = accumulate;
    L.queue = reinterpret_cast<unsigned int *>(reinterpret_cast<char *>(b->d_desc) +
                                               batch_queue_offset(b->h_desc.size() * sizeof(BatchGraph)));
    COLA_TRY(launch_batch(L, st));
    for (const cola_batch::Solo &s : b->solo) {
        cola_spmm_opts o;
        std::memset(&o, 0, sizeof o);
        o.accumulate = accumulate;
        o.schedule = COLA_SCHEDULE_ROWS;
        COLA_TRY(cola_spmm(b->graphs[(size_t)s.g], s.X, b->xdt, s.ldx, s.Y, b->ydt, s.ldy, s.K, &o,
                           (cola_stream_t)st));
    }
    b->last_launches = t_launches - before;
    return COLA_SUCCESS;
}

}  // namespace cola

using namespace cola;

namespace cola {
// Key of a bound batch in the tuning cache: device model and SM count, then a
// 64-bit FNV-1a digest of the operand dtypes and, per graph, its rows,
// entries, width, tasks and hub segments (what the launch's cost depends on).
static std::string tune_key(const cola_batch *b)
{
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, b->device) != cudaSuccess)
        std::strcpy(prop.name, "unknown");
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int i = 0; i < 8; i++) {
            h ^= (v >> (8 * i)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    mix((uint64_t)b->xdt);
    mix((uint64_t)b->ydt);
    mix(b->graphs.size());
    for (const cola_graph *g : b->graphs) {
        mix((uint64_t)g->N);
        mix((uint64_t)(g->nnz_l + g->nnz_r));
        mix((uint64_t)g->ntask);
        mix((uint64_t)g->nseg);
    }
    for (const BatchGraph &d : b->h_desc)
        mix((uint64_t)d.K);
    for (const cola_batch::Solo &so : b->solo) {
        mix((uint64_t)so.g);
        mix((uint64_t)so.K);
    }
    std::string name(prop.name);
    for (char &c : name)
        if (c == ' ' || c == '\t')
            c = '_';
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s|%d|%016llx", name.c_str(), prop.multiProcessorCount, (unsigned long long)h);
    return buf;
}

}  // namespace cola

extern "C" {

cola_status cola_batch_create(const cola_partition_set *const *parts, int32_t ngraphs, const cola_upload_opts *opts,
                              cola_batch **out, cola_stream_t stream)
{
    COLA_REQUIRE(out && (ngraphs == 0 || parts) && ngraphs >= 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_batch_create: bad argument");
    *out = nullptr;
    COLA_REQUIRE(!(opts && opts->no_row_view), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_batch_create: the batched form runs on the row view");
    std::unique_ptr<cola_batch, void (*)(cola_batch *)> b(new (std::nothrow) cola_batch(), batch_release);
    COLA_REQUIRE(b, COLA_ERROR_OUT_OF_MEMORY, "cola_batch_create: host allocation failed");
    COLA_CUDA(cudaGetDevice(&b->device));
    try {
        for (int32_t i = 0; i < ngraphs; i++) {
            cola_graph *g = nullptr;
            COLA_TRY(graph_upload(parts[i], opts, g, (cudaStream_t)stream));
            b->graphs.push_back(g);
        }
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_batch_create: host allocation failed");
    }
    *out = b.release();
    return COLA_SUCCESS;
}

cola_status cola_batch_create_from_graphs(cola_graph *const *graphs, int32_t ngraphs, cola_batch **out)
{
    COLA_REQUIRE(out && (ngraphs == 0 || graphs) && ngraphs >= 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_batch_create_from_graphs: bad argument");
    *out = nullptr;
    std::unique_ptr<cola_batch, void (*)(cola_batch *)> b(new (std::nothrow) cola_batch(), batch_release);
    COLA_REQUIRE(b, COLA_ERROR_OUT_OF_MEMORY, "cola_batch_create_from_graphs: host allocation failed");
    b->own_graphs = false;
    COLA_CUDA(cudaGetDevice(&b->device));
    for (int32_t i = 0; i < ngraphs; i++) {
        COLA_REQUIRE(graphs[i] && graphs[i]->has_rows, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_batch_create_from_graphs: graph %d is NULL or has no row view", i);
        COLA_REQUIRE(graphs[i]->device == b->device, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_batch_create_from_graphs: graph %d lives on device %d, current device is %d", i,
                     graphs[i]->device, b->device);
    }
    try {
        b->graphs.assign(graphs, graphs + ngraphs);
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_batch_create_from_graphs: host allocation failed");
    }
    *out = b.release();
    return COLA_SUCCESS;
}

cola_status cola_batch_free(cola_batch *b)
{
    batch_release(b);
    return COLA_SUCCESS;
}

cola_status cola_batch_bind(cola_batch *b, const void *const *X, const int64_t *ldx, void *const *Y,
                            const int64_t *ldy, const int32_t *K, cola_dtype xdt, cola_dtype ydt,
                            cola_stream_t stream)
{
    COLA_REQUIRE(b && X && ldx && Y && ldy && K, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_bind: null argument");
    COLA_REQUIRE((xdt == COLA_FLOAT32 || xdt == COLA_BFLOAT16) && (ydt == COLA_FLOAT32 || ydt == COLA_BFLOAT16),
                 COLA_ERROR_INVALID_ARGUMENT, "cola_batch_bind: unknown dtype");
    cudaStream_t st = (cudaStream_t)stream;
    b->bound = false;
    b->xdt = xdt;
    b->ydt = ydt;
    b->h_desc.clear();
    b->solo.clear();
    b->total_items = 0;
    b->total_hub = 0;
    for (size_t i = 0; i < b->graphs.size(); i++) {
        cola_graph *g = b->graphs[i];
        COLA_REQUIRE(K[i] >= 1 && ldx[i] >= K[i] && ldy[i] >= K[i] && (g->N == 0 || (X[i] && Y[i])),
                     COLA_ERROR_INVALID_ARGUMENT, "cola_batch_bind: graph %zu: K=%d ldx=%lld ldy=%lld", i, K[i],
                     (long long)ldx[i], (long long)ldy[i]);
        if (g->N == 0)
            continue;
        COLA_REQUIRE(g->nseg + g->ntask < INT32_MAX, COLA_ERROR_UNSUPPORTED,
                     "cola_batch_bind: graph %zu has %lld work items (2^31 at most)", i, (long long)(g->nseg + g->ntask));
        if (g->nseg > 0)
            COLA_TRY(ensure(reinterpret_cast<void *&>(g->ws_hub), g->ws_hub_bytes,
                            (size_t)g->nseg * K[i] * sizeof(float)));
        const bool vec = vec_ok_rows(xdt, X[i], ldx[i], ydt, Y[i], ldy[i], K[i]) && aligned16(g->ws_hub);
        if (!vec) {
            b->solo.push_back({(int)i, X[i], ldx[i], Y[i], ldy[i], K[i]});
            continue;
        }
        BatchGraph d;
        fill_batch_graph(d, g, X[i], ldx[i], Y[i], ldy[i], K[i], xdt, g->ws_hub);
        d.item0 = b->total_items;
        d.hub0 = b->total_hub;
        b->total_items += g->nseg + g->ntask;
        b->total_hub += g->nhub * ((K[i] + 127) / 128);
        b->h_desc.push_back(d);
    }
    const size_t qoff = batch_queue_offset(b->h_desc.size() * sizeof(BatchGraph));
    const size_t need = qoff + kBatchQueueBytes;
    void *p = b->d_desc;
    COLA_TRY(ensure(p, b->d_desc_bytes, need));
    b->d_desc = static_cast<BatchGraph *>(p);
    // the work-item counters start at zero (each launch leaves them so)
    COLA_CUDA(cudaMemsetAsync(static_cast<char *>(p) + qoff, 0, kBatchQueueBytes, st));
    if (!b->h_desc.empty())
        COLA_CUDA(cudaMemcpyAsync(b->d_desc, b->h_desc.data(), b->h_desc.size() * sizeof(BatchGraph),
                                  cudaMemcpyHostToDevice, st));
    COLA_CUDA(cudaStreamSynchronize(st));
    if (b->cexec) {  // a captured graph refers to the old operands
        cudaGraphExecDestroy(b->cexec);
        cudaGraphDestroy(b->cgraph);
        b->cexec = nullptr;
        b->cgraph = nullptr;
    }
    b->bound = true;
    return COLA_SUCCESS;
}

cola_status cola_batch_run(cola_batch *b, const cola_spmm_opts *opts, cola_stream_t stream)
{
    COLA_REQUIRE(b, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_run: batch is NULL");
    return batch_run(b, opts, (cudaStream_t)stream);
}

cola_status cola_batch_capture(cola_batch *b, const cola_spmm_opts *opts, cola_stream_t stream)
{
    COLA_REQUIRE(b && b->bound, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_capture: bind the dense operands first");
    cudaStream_t st = (cudaStream_t)stream;
    if (b->cexec) {
        cudaGraphExecDestroy(b->cexec);
        cudaGraphDestroy(b->cgraph);
        b->cexec = nullptr;
        b->cgraph = nullptr;
    }
    COLA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const cola_status s = batch_run(b, opts, st);
    cudaGraph_t cg = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &cg);
    if (s != COLA_SUCCESS) {
        if (cg)
            cudaGraphDestroy(cg);
        return s;
    }
    COLA_CUDA(e);
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ex, cg, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(cg);
        COLA_CUDA(ie);
    }
    b->cgraph = cg;
    b->cexec = ex;
    return COLA_SUCCESS;
}

cola_status cola_batch_replay(cola_batch *b, cola_stream_t stream)
{
    COLA_REQUIRE(b && b->cexec, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_replay: nothing captured");
    COLA_CUDA(cudaGraphLaunch(b->cexec, (cudaStream_t)stream));
    return COLA_SUCCESS;
}

cola_status cola_batch_get_info(const cola_batch *b, cola_batch_info *o)
{
    COLA_REQUIRE(b && o, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_get_info: null argument");
    std::memset(o, 0, sizeof *o);
    o->ngraphs = (int32_t)b->graphs.size();
    o->batched_graphs = (int32_t)b->h_desc.size();
    o->work_items = b->total_items;
    o->hub_items = b->total_hub;
    for (const cola_graph *g : b->graphs) {
        o->nnz += g->nnz_l + g->nnz_r;
        o->device_bytes += (int64_t)(g->dbytes + g->ws_hub_bytes);
    }
    o->device_bytes += (int64_t)b->d_desc_bytes;
    o->unroll = b->unroll;
    o->grid_pct = b->grid_pct;
    o->blocks_per_sm = b->blocks_per_sm;
    o->last_launches = b->last_launches;
    return COLA_SUCCESS;
}

cola_status cola_batch_set_params(cola_batch *b, int32_t unroll, int32_t grid_pct, int32_t blocks_per_sm)
{
    COLA_REQUIRE(b && (unroll == 2 || unroll == 4) && grid_pct >= 10 && grid_pct <= 100 &&
                     (blocks_per_sm == 3 || blocks_per_sm == 4),
                 COLA_ERROR_INVALID_ARGUMENT,
                 "cola_batch_set_params: unroll 2 or 4, grid_pct 10..100, blocks_per_sm 3 or 4");
    b->unroll = unroll;
    b->grid_pct = grid_pct;
    b->blocks_per_sm = blocks_per_sm;
    return COLA_SUCCESS;
}

cola_status cola_batch_autotune(cola_batch *b, int32_t reps, cola_stream_t stream, float *best_ms)
{
    COLA_REQUIRE(b && b->bound, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_autotune: bind the dense operands first");
    cudaStream_t st = (cudaStream_t)stream;
    reps = std::max(reps, 1);
    cudaEvent_t e0, e1;
    COLA_CUDA(cudaEventCreate(&e0));
    COLA_CUDA(cudaEventCreate(&e1));
    const int32_t unrolls[] = {2, 4};
    const int32_t grids[] = {50, 75, 100};
    const int32_t occ[] = {3, 4};
    float best = 1e30f;
    int32_t bu = b->unroll, bg = b->grid_pct, bo = b->blocks_per_sm;
    cola_status s = COLA_SUCCESS;
    for (int32_t ob : occ)
    for (int32_t u : unrolls)
        for (int32_t gp : grids) {
            b->unroll = u;
            b->grid_pct = gp;
            b->blocks_per_sm = ob;
            if ((s = batch_run(b, nullptr, st)) != COLA_SUCCESS)  // warm-up
                goto done;
            cudaEventRecord(e0, st);
            for (int32_t r = 0; r < reps; r++)
                if ((s = batch_run(b, nullptr, st)) != COLA_SUCCESS)
                    goto done;
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                s = fail(COLA_ERROR_CUDA, "cola_batch_autotune: %s", cudaGetErrorString(cudaGetLastError()));
                goto done;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
            if (ms < best) {
                best = ms;
                bu = u;
                bg = gp;
                bo = ob;
            }
        }
done:
    b->unroll = bu;
    b->grid_pct = bg;
    b->blocks_per_sm = bo;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s == COLA_SUCCESS && best_ms)
        *best_ms = best;
    return s;
}

cola_status cola_batch_autotune_cached(cola_batch *b, int32_t reps, const char *cache_path, cola_stream_t stream,
                                       float *best_ms, int32_t *from_cache)
{
    COLA_REQUIRE(b && b->bound, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_batch_autotune_cached: bind the dense operands first");
    COLA_REQUIRE(cache_path, COLA_ERROR_INVALID_ARGUMENT, "cola_batch_autotune_cached: cache path is NULL");
    const std::string key = cola::tune_key(b);
    TuneEntry e;
    if (tune_cache_find(cache_path, key, e)) {
        b->unroll = e.unroll;
        b->grid_pct = e.grid_pct;
        b->blocks_per_sm = e.blocks_per_sm;
        if (best_ms)
            *best_ms = e.ms;
        if (from_cache)
            *from_cache = 1;
        return COLA_SUCCESS;
    }
    float ms = 0.f;
    COLA_TRY(cola_batch_autotune(b, reps, stream, &ms));
    e.unroll = b->unroll;
    e.grid_pct = b->grid_pct;
    e.blocks_per_sm = b->blocks_per_sm;
    e.ms = ms;
    COLA_REQUIRE(tune_cache_append(cache_path, key, e), COLA_ERROR_IO,
                 "cola_batch_autotune_cached: cannot append to %s", cache_path);
    if (best_ms)
        *best_ms = ms;
    if (from_cache)
        *from_cache = 0;
    return COLA_SUCCESS;
}

}  // extern "C"
