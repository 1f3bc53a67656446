// Serving loop: graphs registered once stay resident on the device; requests
// (host X in, host Y out) are admitted by a device-memory budget, grouped by
// feature width and dtype into one batched launch across graphs, and run on
// several streams at once, so requests that arrive while others are on the GPU
// start as soon as a slot and memory free up (continuous batching).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "batch.h"
#include "common.h"
#include "graph.h"
#include "server_policy.h"

using cola::dev::BatchGraph;

namespace {

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

using cola::kCancelled;
using cola::kDone;
using cola::kFailed;
using cola::kPending;
using cola::kRunning;

struct Request {
    uint64_t id = 0;
    int32_t graph = 0;
    const void *X_host = nullptr;
    void *Y_host = nullptr;
    cola_dtype xdt = COLA_FLOAT32, ydt = COLA_FLOAT32;
    int32_t K = 0;
    int64_t rows = 0;
    int64_t bytes = 0;  // device bytes while in flight: X + Y + hub workspace
    int64_t copy_bytes = 0;  // host<->device bytes: X in + Y out
    double t_submit = 0, t_launch = 0, t_done = 0;
    int state = kPending;
    cola_status status = COLA_SUCCESS;
    void *dX = nullptr, *dY = nullptr;
    float *dws = nullptr;
};

struct Request;
using Group = cola::SchedGroup<Request>;

struct Slot {
    cudaStream_t stream = nullptr;
    Group *busy = nullptr;
    BatchGraph *d_desc = nullptr;  // descriptor table (device)
    BatchGraph *h_desc = nullptr;  // staging (pinned)
    int cap = 0;
    cudaEvent_t ev[4] = {};  // group start, X copied in, launch done, Y copied out
};

}  // namespace

struct cola_server {
    int device = 0;
    int64_t budget = 0, used = 0, peak_used = 0, graph_bytes = 0;
    int32_t max_group = 16;
    int64_t group_bytes = 32 << 20;
    int64_t small_bytes = 16 << 20;  // size classes (server_policy.h); 0 = off
    int32_t small_slots = 1;
    int64_t copy_chunk = 32 << 20;
    bool sm_copies = true;  // small groups copy with the SMs (copy_by_sms_kernel)
    std::vector<cola_graph *> graphs;
    std::vector<Slot> slots;
    // request buffers come from a pool of the server's own that keeps freed
    // memory mapped (release threshold = budget): after warm-up an admitted
    // request costs no device mapping work
    cudaMemPool_t pool = nullptr;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<Request *> pending;
    std::unordered_map<uint64_t, Request *> reqs;
    std::vector<Group *> finished;  // groups whose stream work is complete
    uint64_t next_id = 1;
    bool stop = false;
    std::thread th;
    // statistics
    int64_t submitted = 0, completed = 0, rejected = 0, cancelled = 0, failed = 0;
    int32_t inflight = 0, max_inflight = 0, groups_launched = 0, max_group_seen = 0;
    std::vector<double> lat_ms;
    double queue_ms_sum = 0, copy_in_ms_sum = 0, kernel_ms_sum = 0, copy_out_ms_sum = 0;
    int64_t timed_groups = 0;
    double t_first = 0, t_last = 0, t_window = 0;  // statistics cover requests submitted from t_window on
};

namespace cola {

static void CUDART_CB group_done_cb(void *arg);

struct HostCbArg {
    cola_server *s;
    Group *g;
};

// One cudaMemcpyAsync per piece of at most `chunk` bytes: the copy engine
// takes other streams' copies between the pieces, so a small request's copy
// does not wait for the whole of a long one.
static cola_status copy_chunked(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, int64_t chunk,
                                cudaStream_t st)
{
    const size_t c = chunk > 0 ? (size_t)chunk : bytes;
    for (size_t off = 0; off < bytes; off += c)
        COLA_CUDA(cudaMemcpyAsync(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off,
                                  std::min(c, bytes - off), kind, st));
    return COLA_SUCCESS;
}

// Copies by the SMs instead of the copy engines, for small groups: the copy
// engines take copies in the order they were queued, so a small request's
// copy queued behind another slot's gigabyte would wait for all of it.  Pinned
// host memory is addressable from the device (unified addressing), so a
// kernel moves the bytes itself; writes to host memory are fenced system-wide
// before the kernel ends.  n16: 16-byte units; both pointers 16-byte aligned.
__global__ void __launch_bounds__(256) copy_by_sms_kernel(uint4 *__restrict__ dst, const uint4 *__restrict__ src,
                                                           int64_t n16, int to_host)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n16; i += 4 * stride) {  // four loads in flight per thread
        const uint4 a = src[i], b = src[i + stride], c = src[i + 2 * stride], d = src[i + 3 * stride];
        dst[i] = a;
        dst[i + stride] = b;
        dst[i + 2 * stride] = c;
        dst[i + 3 * stride] = d;
    }
    for (; i < n16; i += stride)
        dst[i] = src[i];
    if (to_host)
        __threadfence_system();
}

// Whether the SMs can copy `bytes` between these pointers: the host side
// pinned and addressable from the device, both 16-byte aligned.
static bool sm_copy_ok(const void *host, const void *dev, size_t bytes)
{
    if (((uintptr_t)host | (uintptr_t)dev | bytes) & 15u)
        return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, host) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost && at.devicePointer == host;
}

static cola_status copy_by_sms(void *dst, const void *src, size_t bytes, bool to_host, cudaStream_t st)
{
    const int64_t n16 = (int64_t)(bytes / 16);
    if (n16 == 0)
        return COLA_SUCCESS;
    const int blocks = (int)std::min<int64_t>((n16 + 1023) / 1024, 128);
    copy_by_sms_kernel<<<blocks, 256, 0, st>>>(static_cast<uint4 *>(dst), static_cast<const uint4 *>(src), n16,
                                               to_host ? 1 : 0);
    COLA_CUDA(cudaGetLastError());
    return COLA_SUCCESS;
}

// Launch one admitted group on its slot: copy every X in, run one batched
// launch over the group's graphs, copy every Y out, then signal completion.
static cola_status launch_group(cola_server *S, Group *G)
{
    Slot &sl = S->slots[(size_t)G->slot];
    cudaStream_t st = sl.stream;
    const int n = (int)G->reqs.size();
    COLA_REQUIRE(n <= sl.cap, COLA_ERROR_INVALID_ARGUMENT, "server: group of %d exceeds the slot's %d", n, sl.cap);
    const Request *r0 = G->reqs[0];
    const size_t xs = r0->xdt == COLA_FLOAT32 ? 4 : 2, ys = r0->ydt == COLA_FLOAT32 ? 4 : 2;
    int64_t items = 0, hub = 0;
    // a small group moves its bytes with the SMs when every host buffer allows it
    bool by_sms = G->small && S->sm_copies && sm_copy_ok(sl.h_desc, sl.d_desc, 16);
    for (const Request *r : G->reqs)
        by_sms = by_sms && ((r->rows * r->K * (int64_t)xs) % 16) == 0 && ((r->rows * r->K * (int64_t)ys) % 16) == 0 &&
                 sm_copy_ok(r->X_host, r->X_host, 16) && sm_copy_ok(r->Y_host, r->Y_host, 16);
    G->by_sms = by_sms;
    COLA_CUDA(cudaEventRecord(sl.ev[0], st));
    for (int i = 0; i < n; i++) {
        Request *r = G->reqs[(size_t)i];
        const cola_graph *g = S->graphs[(size_t)r->graph];
        COLA_CUDA(cudaMallocFromPoolAsync(&r->dX, (size_t)r->rows * r->K * xs, S->pool, st));
        COLA_CUDA(cudaMallocFromPoolAsync(&r->dY, (size_t)r->rows * r->K * ys, S->pool, st));
        if (g->nseg > 0)
            COLA_CUDA(cudaMallocFromPoolAsync((void **)&r->dws, (size_t)g->nseg * r->K * sizeof(float), S->pool, st));
        if (by_sms)
            COLA_TRY(copy_by_sms(r->dX, r->X_host, (size_t)r->rows * r->K * xs, false, st));
        else
            COLA_TRY(copy_chunked(r->dX, r->X_host, (size_t)r->rows * r->K * xs, cudaMemcpyHostToDevice,
                                  S->copy_chunk, st));
        BatchGraph &d = sl.h_desc[i];
        fill_batch_graph(d, g, r->dX, r->K, r->dY, r->K, r->K, r->xdt, r->dws);
        d.item0 = items;
        d.hub0 = hub;
        items += g->nseg + g->ntask;
        hub += g->nhub * ((r->K + 127) / 128);
    }
    COLA_CUDA(cudaEventRecord(sl.ev[1], st));
    if (by_sms && ((size_t)n * sizeof(BatchGraph)) % 16 == 0)
        COLA_TRY(copy_by_sms(sl.d_desc, sl.h_desc, (size_t)n * sizeof(BatchGraph), false, st));
    else
        COLA_CUDA(cudaMemcpyAsync(sl.d_desc, sl.h_desc, (size_t)n * sizeof(BatchGraph), cudaMemcpyHostToDevice, st));
    BatchLaunch L;
    L.desc = sl.d_desc;
    L.ngraphs = n;
    L.total_items = items;
    L.total_hub = hub;
    L.xdt = r0->xdt;
    L.ydt = r0->ydt;
    L.unroll = 4;
    L.grid_pct = 100;
    L.blocks_per_sm = 4;
    L.accumulate = 0;
    L.queue = reinterpret_cast<unsigned int *>(reinterpret_cast<char *>(sl.d_desc) +
                                               batch_queue_offset((size_t)S->max_group * sizeof(BatchGraph)));
    COLA_TRY(launch_batch(L, st));
    COLA_CUDA(cudaEventRecord(sl.ev[2], st));
    for (Request *r : G->reqs) {
        if (by_sms)
            COLA_TRY(copy_by_sms(r->Y_host, r->dY, (size_t)r->rows * r->K * ys, true, st));
        else
            COLA_TRY(copy_chunked(r->Y_host, r->dY, (size_t)r->rows * r->K * ys, cudaMemcpyDeviceToHost,
                                  S->copy_chunk, st));
    }
    COLA_CUDA(cudaEventRecord(sl.ev[3], st));
    for (Request *r : G->reqs) {
        COLA_CUDA(cudaFreeAsync(r->dX, st));
        COLA_CUDA(cudaFreeAsync(r->dY, st));
        if (r->dws)
            COLA_CUDA(cudaFreeAsync(r->dws, st));
        r->dX = r->dY = nullptr;
        r->dws = nullptr;
    }
    HostCbArg *arg = new HostCbArg{S, G};
    const cudaError_t e = cudaLaunchHostFunc(st, group_done_cb, arg);
    if (e != cudaSuccess) {
        delete arg;
        return fail(COLA_ERROR_CUDA, "server: cudaLaunchHostFunc: %s", cudaGetErrorString(e));
    }
    return COLA_SUCCESS;
}

// Runs on a CUDA driver thread once the group's stream work is done: no CUDA
// calls here, only hand the group back to the scheduler.
static void CUDART_CB group_done_cb(void *p)
{
    HostCbArg *a = static_cast<HostCbArg *>(p);
    group_finished(a->s, a->g, now_s());
    delete a;
}

// The device hooks of the scheduler loop (run_scheduler in server_policy.h).
struct CudaSched {
    static cola_status launch(cola_server *S, Group *G) { return launch_group(S, G); }
    // phase timings from the slot's events (the slot stays busy until the
    // group is retired, so they are not recorded again meanwhile)
    static void read_timings(cola_server *S, Group *G)
    {
        Slot &sl = S->slots[(size_t)G->slot];
        G->timed = true;
        for (int k = 0; k < 3; k++)
            G->timed = G->timed && cudaEventElapsedTime(&G->ms[k], sl.ev[k], sl.ev[k + 1]) == cudaSuccess;
    }
    static void release_failed(cola_server *S, Group *G)
    {
        cudaStream_t st = S->slots[(size_t)G->slot].stream;
        for (Request *r : G->reqs) {
            if (r->dX)
                cudaFreeAsync(r->dX, st);
            if (r->dY)
                cudaFreeAsync(r->dY, st);
            if (r->dws)
                cudaFreeAsync(r->dws, st);
            r->dX = r->dY = nullptr;
            r->dws = nullptr;
        }
    }
    static double now() { return now_s(); }
};

// Scheduler: retire finished groups (return their memory to the budget, wake
// waiters), then admit pending requests into free slots, a group at a time as
// pick_group (server_policy.h) chooses: FIFO, the head opening a group of its
// (K, dtypes) key that later requests of the key join while the request count,
// the copy bytes and the budget allow; a head that does not fit waits for
// memory to free up.  The copy-byte cap keeps large requests in groups of
// their own, so one slot's copy-in overlaps another's launch and copy-out.
static void scheduler(cola_server *S)
{
    cudaSetDevice(S->device);
    run_scheduler<cola_server, CudaSched>(S);
}

}  // namespace cola

using namespace cola;

extern "C" {

// Device resources of a server whose scheduler is not running (never started
// or joined): streams after their work, descriptors, events, graphs, the
// memory pool, leftover requests; then the server itself.
static void server_release(cola_server *S)
{
    if (!S)
        return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(S->device);
    for (Slot &sl : S->slots) {
        if (sl.stream) {
            cudaStreamSynchronize(sl.stream);
            cudaStreamDestroy(sl.stream);
        }
        cudaFree(sl.d_desc);
        cudaFreeHost(sl.h_desc);
        for (cudaEvent_t e : sl.ev)
            if (e)
                cudaEventDestroy(e);
    }
    for (cola_graph *g : S->graphs)
        graph_release(g);
    if (S->pool)
        cudaMemPoolDestroy(S->pool);
    for (auto &kv : S->reqs)
        delete kv.second;
    cudaSetDevice(cur);
    delete S;
}

cola_status cola_server_create(const cola_server_opts *opts, cola_server **out)
{
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "cola_server_create: out is NULL");
    *out = nullptr;
    std::unique_ptr<cola_server, void (*)(cola_server *)> S(new (std::nothrow) cola_server(), server_release);
    COLA_REQUIRE(S, COLA_ERROR_OUT_OF_MEMORY, "cola_server_create: host allocation failed");
    COLA_CUDA(cudaGetDevice(&S->device));
    S->budget = opts && opts->memory_budget > 0 ? opts->memory_budget : (int64_t)120 << 30;
    const int nslots = opts && opts->slots > 0 ? opts->slots : 4;
    S->max_group = opts && opts->max_group > 0 ? opts->max_group : 16;
    S->group_bytes = (int64_t)(opts && opts->group_mib > 0 ? opts->group_mib : 32) << 20;
    S->small_bytes = opts && opts->small_mib < 0 ? 0 : (int64_t)(opts && opts->small_mib > 0 ? opts->small_mib : 16) << 20;
    S->copy_chunk = (int64_t)(opts && opts->copy_chunk_mib > 0 ? opts->copy_chunk_mib : 32) << 20;
    S->sm_copies = !(opts && opts->copy_engines_only);
    cudaMemPoolProps pp;
    std::memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = S->device;
    COLA_CUDA(cudaMemPoolCreate(&S->pool, &pp));
    uint64_t keep = (uint64_t)S->budget;
    COLA_CUDA(cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    try {
        S->slots.resize((size_t)nslots);
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_server_create: host allocation failed");
    }
    for (Slot &sl : S->slots) {
        COLA_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
        // the descriptor table, then the slot's work-item counters (zero between launches;
        // a slot's launches are ordered on its stream)
        const size_t qoff = batch_queue_offset((size_t)S->max_group * sizeof(BatchGraph));
        COLA_CUDA(cudaMalloc(&sl.d_desc, qoff + kBatchQueueBytes));
        COLA_CUDA(cudaMemset(reinterpret_cast<char *>(sl.d_desc) + qoff, 0, kBatchQueueBytes));
        COLA_CUDA(cudaMallocHost(&sl.h_desc, (size_t)S->max_group * sizeof(BatchGraph)));
        sl.cap = S->max_group;
        for (cudaEvent_t &e : sl.ev)
            COLA_CUDA(cudaEventCreate(&e));
    }
    try {
        S->th = std::thread(scheduler, S.get());
    } catch (const std::system_error &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_server_create: cannot start the scheduler thread");
    }
    *out = S.release();
    return COLA_SUCCESS;
}

cola_status cola_server_destroy(cola_server *S)
{
    if (!S)
        return COLA_SUCCESS;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        for (Request *r : S->pending) {  // never admitted: cancel
            r->state = kCancelled;
            r->status = COLA_ERROR_CANCELLED;
        }
        S->pending.clear();
    }
    S->cv_sched.notify_all();
    S->th.join();  // returns once every admitted group has completed
    server_release(S);
    return COLA_SUCCESS;
}

cola_status cola_server_register(cola_server *S, const cola_partition_set *parts, const cola_upload_opts *opts,
                                 int32_t *graph_id)
{
    COLA_REQUIRE(S && parts && graph_id, COLA_ERROR_INVALID_ARGUMENT, "cola_server_register: null argument");
    COLA_REQUIRE(!(opts && opts->no_row_view), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_server_register: the server runs on the row view");
    int cur = 0;
    COLA_CUDA(cudaGetDevice(&cur));
    COLA_REQUIRE(cur == S->device, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_server_register: server lives on device %d, current device is %d", S->device, cur);
    cola_graph *g = nullptr;
    COLA_TRY(graph_upload(parts, opts, g, nullptr));
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->used + (int64_t)g->dbytes > S->budget) {
        const long long used = (long long)S->used, budget = (long long)S->budget;
        lk.unlock();  // no CUDA call under the lock
        const size_t need = g->dbytes;
        graph_release(g);
        return fail(COLA_ERROR_BUDGET, "cola_server_register: graph needs %zu bytes, %lld of %lld bytes in use",
                    need, used, budget);
    }
    S->used += (int64_t)g->dbytes;
    S->graph_bytes += (int64_t)g->dbytes;
    S->peak_used = std::max(S->peak_used, S->used);
    S->graphs.push_back(g);
    *graph_id = (int32_t)S->graphs.size() - 1;
    return COLA_SUCCESS;
}

cola_status cola_server_register_graph(cola_server *S, cola_graph *g, int32_t *graph_id)
{
    if (!(S && g && graph_id)) {
        graph_release(g);  // ownership was passed: never leak it
        return fail(COLA_ERROR_INVALID_ARGUMENT, "cola_server_register_graph: null argument");
    }
    if (!g->has_rows || g->device != S->device) {
        const int dev = g->device;
        graph_release(g);
        return fail(COLA_ERROR_INVALID_ARGUMENT,
                    "cola_server_register_graph: the graph needs its row view and the server's device %d (it "
                    "lives on %d)", S->device, dev);
    }
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->used + (int64_t)g->dbytes > S->budget) {
        const long long used = (long long)S->used, budget = (long long)S->budget;
        lk.unlock();  // no CUDA call under the lock
        const size_t need = g->dbytes;
        graph_release(g);
        return fail(COLA_ERROR_BUDGET, "cola_server_register_graph: graph needs %zu bytes, %lld of %lld bytes in use",
                    need, used, budget);
    }
    S->used += (int64_t)g->dbytes;
    S->graph_bytes += (int64_t)g->dbytes;
    S->peak_used = std::max(S->peak_used, S->used);
    S->graphs.push_back(g);
    *graph_id = (int32_t)S->graphs.size() - 1;
    return COLA_SUCCESS;
}

cola_status cola_server_submit(cola_server *S, int32_t graph_id, const void *X_host, cola_dtype x_dtype,
                               int32_t K, void *Y_host, cola_dtype y_dtype, uint64_t *request_id)
{
    COLA_REQUIRE(S && request_id, COLA_ERROR_INVALID_ARGUMENT, "cola_server_submit: null argument");
    COLA_REQUIRE((x_dtype == COLA_FLOAT32 || x_dtype == COLA_BFLOAT16) &&
                     (y_dtype == COLA_FLOAT32 || y_dtype == COLA_BFLOAT16),
                 COLA_ERROR_INVALID_ARGUMENT, "cola_server_submit: unknown dtype");
    const int E = x_dtype == COLA_FLOAT32 ? 4 : 8;
    COLA_REQUIRE(K >= 1 && K % E == 0, COLA_ERROR_UNSUPPORTED,
                 "cola_server_submit: K=%d must be a multiple of %d for this dtype", K, E);
    std::unique_ptr<Request> r(new (std::nothrow) Request());
    COLA_REQUIRE(r, COLA_ERROR_OUT_OF_MEMORY, "cola_server_submit: host allocation failed");
    std::lock_guard<std::mutex> lk(S->mu);
    COLA_REQUIRE(!S->stop, COLA_ERROR_CANCELLED, "cola_server_submit: server is shutting down");
    COLA_REQUIRE(graph_id >= 0 && graph_id < (int32_t)S->graphs.size(), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_server_submit: unknown graph %d", graph_id);
    const cola_graph *g = S->graphs[(size_t)graph_id];
    COLA_REQUIRE(g->N == 0 || (X_host && Y_host), COLA_ERROR_INVALID_ARGUMENT, "cola_server_submit: null X or Y");
    r->graph = graph_id;
    r->X_host = X_host;
    r->Y_host = Y_host;
    r->xdt = x_dtype;
    r->ydt = y_dtype;
    r->K = K;
    r->rows = g->N;
    r->copy_bytes = (int64_t)g->N * K * ((x_dtype == COLA_FLOAT32 ? 4 : 2) + (y_dtype == COLA_FLOAT32 ? 4 : 2));
    r->bytes = r->copy_bytes + g->nseg * K * 4;
    if (S->graph_bytes + r->bytes > S->budget) {
        S->rejected++;
        return fail(COLA_ERROR_BUDGET,
                    "cola_server_submit: the request needs %lld device bytes; the budget leaves %lld beside the "
                    "registered graphs",
                    (long long)r->bytes, (long long)(S->budget - S->graph_bytes));
    }
    r->id = S->next_id++;
    r->t_submit = now_s();
    if (S->submitted == 0)
        S->t_first = r->t_submit;
    S->submitted++;
    *request_id = r->id;
    Request *raw = r.release();
    S->pending.push_back(raw);
    S->reqs[raw->id] = raw;
    S->cv_sched.notify_all();
    return COLA_SUCCESS;
}

cola_status cola_server_wait(cola_server *S, uint64_t request_id, int32_t timeout_ms)
{
    COLA_REQUIRE(S, COLA_ERROR_INVALID_ARGUMENT, "cola_server_wait: server is NULL");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(request_id);
    COLA_REQUIRE(it != S->reqs.end(), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_server_wait: unknown request %llu (or already collected)", (unsigned long long)request_id);
    Request *r = it->second;
    auto finished = [&] { return r->state >= kDone; };
    if (timeout_ms < 0)
        S->cv_done.wait(lk, finished);
    else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished))
        return fail(COLA_ERROR_TIMEOUT, "cola_server_wait: request %llu not finished after %d ms",
                    (unsigned long long)request_id, timeout_ms);
    const cola_status st = r->state == kDone ? COLA_SUCCESS : r->status;
    S->reqs.erase(it);
    delete r;
    if (st != COLA_SUCCESS)
        return fail(st, "cola_server_wait: request %llu %s", (unsigned long long)request_id,
                    st == COLA_ERROR_CANCELLED ? "was cancelled" : "failed");
    return COLA_SUCCESS;
}

cola_status cola_server_cancel(cola_server *S, uint64_t request_id)
{
    COLA_REQUIRE(S, COLA_ERROR_INVALID_ARGUMENT, "cola_server_cancel: server is NULL");
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(request_id);
    COLA_REQUIRE(it != S->reqs.end(), COLA_ERROR_INVALID_ARGUMENT, "cola_server_cancel: unknown request %llu",
                 (unsigned long long)request_id);
    Request *r = it->second;
    COLA_REQUIRE(r->state == kPending, COLA_ERROR_NOT_READY,
                 "cola_server_cancel: request %llu is already on the GPU or finished", (unsigned long long)request_id);
    S->pending.erase(std::find(S->pending.begin(), S->pending.end(), r));
    r->state = kCancelled;
    r->status = COLA_ERROR_CANCELLED;
    S->cancelled++;
    S->cv_done.notify_all();
    S->cv_sched.notify_all();  // a new head may fit where the cancelled one did not
    return COLA_SUCCESS;
}

cola_status cola_server_reset_stats(cola_server *S)
{
    COLA_REQUIRE(S, COLA_ERROR_INVALID_ARGUMENT, "cola_server_reset_stats: server is NULL");
    std::lock_guard<std::mutex> lk(S->mu);
    S->submitted = S->completed = S->rejected = S->cancelled = S->failed = 0;
    S->max_inflight = S->inflight;
    S->groups_launched = S->max_group_seen = 0;
    S->peak_used = S->used;
    S->lat_ms.clear();
    S->queue_ms_sum = S->copy_in_ms_sum = S->kernel_ms_sum = S->copy_out_ms_sum = 0;
    S->timed_groups = 0;
    S->t_first = S->t_last = 0;
    S->t_window = now_s();
    return COLA_SUCCESS;
}

cola_status cola_server_get_stats(cola_server *S, cola_server_stats *o)
{
    COLA_REQUIRE(S && o, COLA_ERROR_INVALID_ARGUMENT, "cola_server_get_stats: null argument");
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(o, 0, sizeof *o);
    o->submitted = S->submitted;
    o->completed = S->completed;
    o->rejected = S->rejected;
    o->cancelled = S->cancelled;
    o->failed = S->failed;
    o->pending = (int64_t)S->pending.size();
    o->inflight = S->inflight;
    o->max_inflight = S->max_inflight;
    o->groups_launched = S->groups_launched;
    o->max_group = S->max_group_seen;
    o->bytes_in_use = S->used;
    o->peak_bytes = S->peak_used;
    o->budget = S->budget;
    if (!S->lat_ms.empty()) {
        std::vector<double> v = S->lat_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) {
            return v[(size_t)std::min<double>((double)v.size() - 1, q * (double)(v.size() - 1) + 0.5)];
        };
        o->p50_ms = pct(0.50);
        o->p99_ms = pct(0.99);
        o->max_ms = v.back();
        double sum = 0;
        for (double x : v)
            sum += x;
        o->mean_ms = sum / (double)v.size();
        if (S->t_last > S->t_first)
            o->req_per_s = (double)S->completed / (S->t_last - S->t_first);
        o->queue_ms_mean = S->queue_ms_sum / (double)v.size();
    }
    if (S->timed_groups > 0) {
        o->copy_in_ms_mean = S->copy_in_ms_sum / (double)S->timed_groups;
        o->kernel_ms_mean = S->kernel_ms_sum / (double)S->timed_groups;
        o->copy_out_ms_mean = S->copy_out_ms_sum / (double)S->timed_groups;
    }
    return COLA_SUCCESS;
}

}  // extern "C"
