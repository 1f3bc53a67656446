// Y = A X with the dense operands in host memory (cola_spmm_host): the
// feature matrix is copied in, multiplied on the device and the result copied
// out, with consecutive calls pipelined.  The graph keeps two staging sets
// (device X and Y) and two copy streams of its own: call i + 1's upload runs
// while call i's result is downloading, and each call's SpMM waits only for
// its own upload and for the staging set it reuses, so both directions of the
// host link stay busy.  cola_spmm_host_sync waits for every call made so far.
#include <algorithm>
#include <new>

#include <cuda_runtime.h>

#include "common.h"
#include "graph.h"

namespace cola {

struct HostStage {
    void *dX = nullptr, *dY = nullptr;
    size_t x_bytes = 0, y_bytes = 0;
    cudaEvent_t x_ready = nullptr, x_free = nullptr, y_ready = nullptr, y_free = nullptr;
};

struct HostPipe {
    int device = 0;
    cudaStream_t up = nullptr, down = nullptr;
    HostStage st[2];
    int next = 0;
};

void host_pipe_release(HostPipe *p)
{
    if (!p)
        return;
    cudaStreamSynchronize(p->up);
    cudaStreamSynchronize(p->down);
    for (HostStage &s : p->st) {
        cudaFree(s.dX);
        cudaFree(s.dY);
        for (cudaEvent_t e : {s.x_ready, s.x_free, s.y_ready, s.y_free})
            if (e)
                cudaEventDestroy(e);
    }
    if (p->up)
        cudaStreamDestroy(p->up);
    if (p->down)
        cudaStreamDestroy(p->down);
    delete p;
}

static cola_status host_pipe_get(cola_graph *g, HostPipe *&out)
{
    if (!g->host_pipe) {
        HostPipe *p = new (std::nothrow) HostPipe();
        COLA_REQUIRE(p, COLA_ERROR_OUT_OF_MEMORY, "cola_spmm_host: host allocation failed");
        p->device = g->device;
        g->host_pipe = p;  // released with the graph, whatever fails below
        COLA_CUDA(cudaStreamCreateWithFlags(&p->up, cudaStreamNonBlocking));
        COLA_CUDA(cudaStreamCreateWithFlags(&p->down, cudaStreamNonBlocking));
        for (HostStage &s : p->st)
            for (cudaEvent_t *e : {&s.x_ready, &s.x_free, &s.y_ready, &s.y_free})
                COLA_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    out = g->host_pipe;
    return COLA_SUCCESS;
}

}  // namespace cola

using namespace cola;

extern "C" cola_status cola_spmm_host(cola_graph *g, const void *X_host, cola_dtype x_dtype, int64_t ldx,
                                      void *Y_host, cola_dtype y_dtype, int64_t ldy, int32_t K,
                                      const cola_spmm_opts *opts, cola_stream_t stream)
{
    const char *who = "cola_spmm_host";
    COLA_REQUIRE(g, COLA_ERROR_INVALID_ARGUMENT, "%s: graph is NULL", who);
    COLA_REQUIRE(K >= 1 && ldx >= K && ldy >= K, COLA_ERROR_INVALID_ARGUMENT, "%s: K=%d ldx=%lld ldy=%lld", who, K,
                 (long long)ldx, (long long)ldy);
    COLA_REQUIRE((x_dtype == COLA_FLOAT32 || x_dtype == COLA_BFLOAT16) &&
                     (y_dtype == COLA_FLOAT32 || y_dtype == COLA_BFLOAT16),
                 COLA_ERROR_INVALID_ARGUMENT, "%s: unknown dtype", who);
    COLA_REQUIRE(!(opts && opts->accumulate), COLA_ERROR_UNSUPPORTED,
                 "%s: accumulate needs Y on the device (use cola_spmm)", who);
    COLA_REQUIRE(g->N == 0 || (X_host && Y_host), COLA_ERROR_INVALID_ARGUMENT, "%s: null X or Y", who);
    if (g->N == 0)
        return COLA_SUCCESS;
    int cur = 0;
    COLA_CUDA(cudaGetDevice(&cur));
    COLA_REQUIRE(cur == g->device, COLA_ERROR_INVALID_ARGUMENT, "%s: graph lives on device %d, current device is %d",
                 who, g->device, cur);
    HostPipe *p = nullptr;
    COLA_TRY(host_pipe_get(g, p));
    HostStage &s = p->st[p->next];
    const size_t xs = x_dtype == COLA_FLOAT32 ? 4 : 2, ys = y_dtype == COLA_FLOAT32 ? 4 : 2;
    // the staging set is dense (ld = K); the host rows may be strided
    const size_t xb = (size_t)g->N * K * xs, yb = (size_t)g->N * K * ys;
    if (s.x_bytes < xb || s.y_bytes < yb) {
        // a set grows only after the work that used it has finished
        COLA_CUDA(cudaEventSynchronize(s.x_free));
        COLA_CUDA(cudaEventSynchronize(s.y_free));
        if (s.x_bytes < xb) {
            cudaFree(s.dX);
            s.dX = nullptr;
            s.x_bytes = 0;
            COLA_CUDA(cudaMalloc(&s.dX, xb));
            s.x_bytes = xb;
        }
        if (s.y_bytes < yb) {
            cudaFree(s.dY);
            s.dY = nullptr;
            s.y_bytes = 0;
            COLA_CUDA(cudaMalloc(&s.dY, yb));
            s.y_bytes = yb;
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    // upload, once the SpMM that last read this set's X is done (X_host must
    // hold the features when the call is made: the copy does not wait for
    // earlier work on `stream`)
    COLA_CUDA(cudaStreamWaitEvent(p->up, s.x_free, 0));
    if (ldx == K)
        COLA_CUDA(cudaMemcpyAsync(s.dX, X_host, xb, cudaMemcpyHostToDevice, p->up));
    else
        COLA_CUDA(cudaMemcpy2DAsync(s.dX, (size_t)K * xs, X_host, (size_t)ldx * xs, (size_t)K * xs, (size_t)g->N,
                                    cudaMemcpyHostToDevice, p->up));
    COLA_CUDA(cudaEventRecord(s.x_ready, p->up));
    // multiply on the caller's stream, once X is in and this set's Y is downloaded
    COLA_CUDA(cudaStreamWaitEvent(st, s.x_ready, 0));
    COLA_CUDA(cudaStreamWaitEvent(st, s.y_free, 0));
    cola_spmm_opts o = opts ? *opts : cola_spmm_opts{};
    o.accumulate = 0;
    COLA_TRY(cola_spmm(g, s.dX, x_dtype, K, s.dY, y_dtype, K, K, &o, stream));
    COLA_CUDA(cudaEventRecord(s.x_free, st));
    COLA_CUDA(cudaEventRecord(s.y_ready, st));
    // download
    COLA_CUDA(cudaStreamWaitEvent(p->down, s.y_ready, 0));
    if (ldy == K)
        COLA_CUDA(cudaMemcpyAsync(Y_host, s.dY, yb, cudaMemcpyDeviceToHost, p->down));
    else
        COLA_CUDA(cudaMemcpy2DAsync(Y_host, (size_t)ldy * ys, s.dY, (size_t)K * ys, (size_t)K * ys, (size_t)g->N,
                                    cudaMemcpyDeviceToHost, p->down));
    COLA_CUDA(cudaEventRecord(s.y_free, p->down));
    p->next ^= 1;
    return COLA_SUCCESS;
}

extern "C" cola_status cola_spmm_host_join(cola_graph *g, cola_stream_t stream)
{
    COLA_REQUIRE(g, COLA_ERROR_INVALID_ARGUMENT, "cola_spmm_host_join: graph is NULL");
    if (!g->host_pipe)
        return COLA_SUCCESS;
    for (const HostStage &s : g->host_pipe->st)
        COLA_CUDA(cudaStreamWaitEvent((cudaStream_t)stream, s.y_free, 0));
    return COLA_SUCCESS;
}

extern "C" cola_status cola_spmm_host_sync(cola_graph *g)
{
    COLA_REQUIRE(g, COLA_ERROR_INVALID_ARGUMENT, "cola_spmm_host_sync: graph is NULL");
    if (!g->host_pipe)
        return COLA_SUCCESS;
    COLA_CUDA(cudaStreamSynchronize(g->host_pipe->up));
    COLA_CUDA(cudaStreamSynchronize(g->host_pipe->down));
    for (const HostStage &s : g->host_pipe->st)
        COLA_CUDA(cudaEventSynchronize(s.x_free));  // the SpMMs on the caller's stream
    return COLA_SUCCESS;
}
