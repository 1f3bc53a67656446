// Ceilings of the row gather the SpMM kernels are made of, measured on the
// device they run on (cola_probe_gather): warps read whole rows of a table
// (16-byte vector loads across the warp, 4 rows in flight per warp as in the
// SpMM, a persistent grid of one full wave) at pseudo-random row indices read
// from an index array, 32 at a time, as the SpMM reads its entries.  With a table
// that fits in L2 the rows come from L2 (the ceiling of the SpMM's gathers,
// most of which hit L2); with a table several times larger than L2 they come
// from DRAM.  The sums are kept (one value per warp) so that no load is dead.
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "common.h"
#include "graph.h"

namespace cola {
namespace probe {

__device__ __forceinline__ uint32_t mix32(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (uint32_t)x;
}

__global__ void make_indices_kernel(int32_t *__restrict__ idx, int64_t n, int64_t rows, uint64_t seed)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        idx[i] = (int32_t)(mix32(seed + (uint64_t)i) % (uint64_t)rows);
}

// The SpMM's gather loop without the arithmetic: a warp reads 32 row indices
// with one coalesced load, then the rows they name, UNROLL rows in flight
// (16-byte vectors across the warp).
template <int UNROLL>
__global__ void __launch_bounds__(256) gather_probe_kernel(const uint4 *__restrict__ table, const int32_t *__restrict__ idx,
                                                           int row_vecs, int64_t gathers, float *__restrict__ sink)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int64_t nwarps = (int64_t)gridDim.x * 8;
    uint32_t acc = 0;
    for (int64_t g0 = warp * 32; g0 < gathers; g0 += nwarps * 32) {
        const int n = (int)min((int64_t)32, gathers - g0);
        const int32_t mine = lane < n ? __ldcs(idx + g0 + lane) : 0;
        for (int j = 0; j < n; j += UNROLL) {
            uint4 v[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; u++) {
                const int k = j + u;
                const int32_t r = __shfl_sync(0xffffffffu, mine, k & 31);
                v[u] = (k < n && lane < row_vecs) ? __ldg(table + (int64_t)r * row_vecs + lane) : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
                acc += v[u].x ^ v[u].y ^ v[u].z ^ v[u].w;
        }
    }
    if (acc == 0x9e3779b9u)  // practically never: keeps the loads alive
        sink[warp] = (float)acc;
}

// The graph's own access pattern without the arithmetic: warps walk the row
// view's entries in order, 32 at a time (as the streaming kernel's tasks do,
// the next 32 indices loading while these are used), and read the X row each
// entry names -- VECS 16-byte vectors per lane, 4 rows in flight -- keeping
// only an XOR of the data.  Its time is the
// memory system's time for exactly the SpMM's gathers.
template <int VECS>
__global__ void __launch_bounds__(256) graph_gather_kernel(const char *__restrict__ X, int64_t ld_bytes,
                                                           const int32_t *__restrict__ col, int64_t nnz,
                                                           int row_vecs, float *__restrict__ sink)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int64_t nwarps = (int64_t)gridDim.x * 8;
    uint32_t acc = 0;
    // the next batch of indices is loaded while this one's rows are read
    int32_t next = warp * 32 + lane < nnz ? __ldcs(col + warp * 32 + lane) : 0;
    for (int64_t e0 = warp * 32; e0 < nnz; e0 += nwarps * 32) {
        const int n = (int)min((int64_t)32, nnz - e0);
        const int32_t mine = next;
        const int64_t e1 = e0 + nwarps * 32 + lane;
        next = e1 < nnz ? __ldcs(col + e1) : 0;
        for (int j = 0; j < n; j += 4) {
            uint4 v[4][VECS];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int32_t r = __shfl_sync(0xffffffffu, mine, (j + u) & 31);
                const uint4 *p = reinterpret_cast<const uint4 *>(X + (int64_t)r * ld_bytes);
#pragma unroll
                for (int q = 0; q < VECS; q++)
                    v[u][q] = (j + u < n && lane + 32 * q < row_vecs) ? __ldg(p + lane + 32 * q)
                                                                      : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int q = 0; q < VECS; q++)
                    acc += v[u][q].x ^ v[u][q].y ^ v[u][q].z ^ v[u][q].w;
        }
    }
    if (acc == 0x9e3779b9u)  // practically never: keeps the loads alive
        sink[warp] = (float)acc;
}

}  // namespace probe
}  // namespace cola

using namespace cola;

extern "C" cola_status cola_probe_gather(int64_t table_bytes, int32_t row_bytes, int64_t gathers, int32_t reps,
                                         cola_stream_t stream, double *gbps)
{
    COLA_REQUIRE(gbps && table_bytes >= row_bytes && row_bytes >= 16 && row_bytes <= 512 && row_bytes % 16 == 0 &&
                     gathers >= 1 && reps >= 1,
                 COLA_ERROR_INVALID_ARGUMENT,
                 "cola_probe_gather: table %lld bytes, rows of %d bytes (16..512, a multiple of 16), %lld gathers",
                 (long long)table_bytes, row_bytes, (long long)gathers);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t rows = table_bytes / row_bytes;
    void *table = nullptr;
    int32_t *idx = nullptr;
    float *sink = nullptr;
    const int blocks = sm_count() * blocks_per_sm((const void *)probe::gather_probe_kernel<4>, 256);
    COLA_CUDA(cudaMallocAsync(&table, (size_t)(rows * row_bytes), st));
    cudaError_t e = cudaMallocAsync((void **)&sink, (size_t)blocks * 8 * sizeof(float), st);
    if (e == cudaSuccess)
        e = cudaMallocAsync((void **)&idx, (size_t)gathers * sizeof(int32_t), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(table, 0x5a, (size_t)(rows * row_bytes), st);
    if (e == cudaSuccess) {
        probe::make_indices_kernel<<<sm_count() * 8, 256, 0, st>>>(idx, gathers, rows, 0x1234567ull);
        e = cudaGetLastError();
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess)
        e = cudaEventCreate(&e0);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e1);
    float ms = 0.f;
    for (int pass = 0; pass < 2 && e == cudaSuccess; pass++) {  // pass 0 warms the cache
        e = cudaEventRecord(e0, st);
        for (int r = 0; r < (pass ? reps : 1) && e == cudaSuccess; r++) {
            probe::gather_probe_kernel<4><<<blocks, 256, 0, st>>>(static_cast<const uint4 *>(table), idx,
                                                                  row_bytes / 16, gathers, sink);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaEventRecord(e1, st);
        if (e == cudaSuccess)
            e = cudaEventSynchronize(e1);
        if (e == cudaSuccess && pass)
            e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    cudaFreeAsync(idx, st);
    cudaFreeAsync(sink, st);
    cudaFreeAsync(table, st);
    COLA_CUDA(e);
    COLA_CUDA(cudaStreamSynchronize(st));
    *gbps = (double)gathers * row_bytes * reps / (ms * 1e-3) / 1e9;
    return COLA_SUCCESS;
}

extern "C" cola_status cola_probe_graph_gather(const cola_graph *g, const void *X, int64_t ld_bytes,
                                               int32_t row_bytes, int32_t reps, cola_stream_t stream, double *gbps,
                                               float *ms_per_pass)
{
    COLA_REQUIRE(g && g->has_rows && X && gbps && row_bytes >= 16 && row_bytes <= 2048 && row_bytes % 16 == 0 &&
                     ld_bytes >= row_bytes && ld_bytes % 16 == 0 && ((uintptr_t)X & 15u) == 0 && reps >= 1,
                 COLA_ERROR_INVALID_ARGUMENT,
                 "cola_probe_graph_gather: a graph with its row view, X 16-byte aligned, rows of 16..2048 bytes "
                 "(a multiple of 16) at a stride of at least that many");
    cudaStream_t st = (cudaStream_t)stream;
    int64_t nnz = 0;
    COLA_CUDA(cudaMemcpyAsync(&nnz, g->rv_ptr + g->N, sizeof nnz, cudaMemcpyDeviceToHost, st));
    COLA_CUDA(cudaStreamSynchronize(st));
    const int row_vecs = row_bytes / 16, vecs = (row_vecs + 31) / 32;
    auto fn = vecs == 1 ? probe::graph_gather_kernel<1> : vecs == 2 ? probe::graph_gather_kernel<2>
                                                                    : probe::graph_gather_kernel<4>;
    const int blocks = sm_count() * blocks_per_sm((const void *)fn, 256);
    float *sink = nullptr;
    COLA_CUDA(cudaMallocAsync((void **)&sink, (size_t)blocks * 8 * sizeof(float), st));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess)
        e = cudaEventCreate(&e1);
    float ms = 0.f;
    for (int pass = 0; pass < 2 && e == cudaSuccess; pass++) {  // pass 0 warms the cache
        e = cudaEventRecord(e0, st);
        for (int r = 0; r < (pass ? reps : 1) && e == cudaSuccess; r++) {
            fn<<<blocks, 256, 0, st>>>(static_cast<const char *>(X), ld_bytes, g->rv_col, nnz, row_vecs, sink);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaEventRecord(e1, st);
        if (e == cudaSuccess)
            e = cudaEventSynchronize(e1);
        if (e == cudaSuccess && pass)
            e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    cudaFreeAsync(sink, st);
    COLA_CUDA(e);
    COLA_CUDA(cudaStreamSynchronize(st));
    ms /= reps;
    *gbps = (double)nnz * row_bytes / (ms * 1e-3) / 1e9;
    if (ms_per_pass)
        *ms_per_pass = ms;
    return COLA_SUCCESS;
}
