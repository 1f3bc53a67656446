// The project's autotuner for one graph's SpMM (cola_spmm_autotune): times the
// launch options of a schedule on the caller's operands with CUDA events and
// keeps the fastest, optionally through the cache file of tune_cache.h.
//
// Row-major schedule: the feature tile of one pass (k_tile), the row loads in
// flight (unroll) and the resident blocks per SM (min_blocks).  Where a full
// warp covers a feature tile (K >= 128 FP32 X, K >= 256 BF16 X) every
// candidate sums each element in the same order, so the tuned result is the
// same bits as the untuned one.  Narrower K has one geometry: nothing to tune.
// Buffer and pipelined schedules: the remote-row gather batch
// (gather_batch_rows), the reference's staging granularity.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "graph.h"
#include "tune_cache.h"

namespace cola {
namespace {

struct Cand {
    int k_tile, unroll, min_blocks, gather;
};

std::vector<Cand> rows_candidates(cola_dtype xdt, int K)
{
    std::vector<Cand> c;
    const int e16 = xdt == COLA_FLOAT32 ? 4 : 8;
    if (K < 32 * e16) {
        c.push_back({0, 0, 0, 0});
        return c;
    }
    const int tiles[] = {64, 128, 256, 512, 1024};
    for (int kt : tiles) {
        if (xdt == COLA_FLOAT32 && kt == 1024)
            continue;
        if (kt > 64 && kt / 2 >= K)  // wider than K needs
            continue;
        const bool narrow = kt * (xdt == COLA_FLOAT32 ? 4 : 2) < 512;
        const int V = kt / e16;
        // (resident blocks beyond 4 per SM spill registers: measured 1.5-3x slower, not searched)
        if (narrow) {
            c.push_back({kt, 4, 4, 0});
            c.push_back({kt, 8, 4, 0});
        } else if (V == 32) {
            c.push_back({kt, 2, 0, 0});
            for (int mb : {3, 4})
                c.push_back({kt, 4, mb, 0});
            c.push_back({kt, 6, 0, 0});
            c.push_back({kt, 8, 0, 0});
        } else if (V == 64) {
            c.push_back({kt, 2, 0, 0});
            c.push_back({kt, 4, 0, 0});
        } else {
            c.push_back({kt, 0, 0, 0});
        }
    }
    return c;
}

std::string spmm_tune_key(const cola_graph *g, cola_dtype xdt, cola_dtype ydt, int K, int schedule)
{
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, g->device) != cudaSuccess)
        std::strcpy(prop.name, "unknown");
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int i = 0; i < 8; i++) {
            h ^= (v >> (8 * i)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    for (uint64_t v : {(uint64_t)xdt, (uint64_t)ydt, (uint64_t)K, (uint64_t)schedule, (uint64_t)g->N,
                       (uint64_t)(g->nnz_l + g->nnz_r), (uint64_t)g->ntask, (uint64_t)g->nseg, (uint64_t)g->P,
                       (uint64_t)g->rchunks})
        mix(v);
    std::string name = prop.name;
    for (char &ch : name)
        if (ch == ' ' || ch == '|')
            ch = '_';
    char buf[96];
    std::snprintf(buf, sizeof buf, "|%d|%016llx", prop.multiProcessorCount, (unsigned long long)h);
    return "spmm|" + name + buf;
}

}  // namespace
}  // namespace cola

using namespace cola;

extern "C" cola_status cola_spmm_autotune(cola_graph *g, const void *X, cola_dtype x_dtype, int64_t ldx, void *Y,
                                          cola_dtype y_dtype, int64_t ldy, int32_t K, int32_t schedule, int32_t reps,
                                          const char *cache_path, cola_stream_t stream, cola_spmm_opts *best,
                                          float *best_ms, int32_t *from_cache)
{
    const char *who = "cola_spmm_autotune";
    COLA_REQUIRE(g && best, COLA_ERROR_INVALID_ARGUMENT, "%s: null graph or result", who);
    if (schedule == COLA_SCHEDULE_AUTO)
        schedule = g->has_rows ? COLA_SCHEDULE_ROWS : (g->nstages > 1 ? COLA_SCHEDULE_PIPELINE : COLA_SCHEDULE_FUSED);
    std::memset(best, 0, sizeof *best);
    best->schedule = schedule;
    std::vector<Cand> cands;
    if (schedule == COLA_SCHEDULE_ROWS) {
        cands = rows_candidates(x_dtype, K);
    } else if (schedule == COLA_SCHEDULE_BUFFER || schedule == COLA_SCHEDULE_PIPELINE) {
        for (int b : {1024, 2048, 4096, 8192, 16384})
            cands.push_back({0, 0, 0, b});
    } else {
        cands.push_back({0, 0, 0, 0});
    }
    const std::string key = spmm_tune_key(g, x_dtype, y_dtype, K, schedule);
    if (cache_path) {
        SpmmTuneEntry e;
        if (spmm_tune_cache_find(cache_path, key, e)) {
            best->k_tile = e.k_tile;
            best->unroll = e.unroll;
            best->min_blocks = e.min_blocks;
            best->gather_batch_rows = e.gather_batch_rows;
            if (best_ms)
                *best_ms = e.ms;
            if (from_cache)
                *from_cache = 1;
            return COLA_SUCCESS;
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    reps = std::max(reps, 1);
    cudaEvent_t e0, e1;
    COLA_CUDA(cudaEventCreate(&e0));
    COLA_CUDA(cudaEventCreate(&e1));
    float top = 1e30f;
    Cand pick = cands.front();
    cola_status s = COLA_SUCCESS;
    for (const Cand &c : cands) {
        cola_spmm_opts o = {};
        o.schedule = schedule;
        o.k_tile = c.k_tile;
        o.unroll = c.unroll;
        o.min_blocks = c.min_blocks;
        o.gather_batch_rows = c.gather;
        if ((s = cola_spmm(g, X, x_dtype, ldx, Y, y_dtype, ldy, K, &o, stream)) != COLA_SUCCESS)  // warm-up
            break;
        cudaEventRecord(e0, st);
        for (int32_t r = 0; r < reps && s == COLA_SUCCESS; r++)
            s = cola_spmm(g, X, x_dtype, ldx, Y, y_dtype, ldy, K, &o, stream);
        cudaEventRecord(e1, st);
        if (s != COLA_SUCCESS)
            break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            s = fail(COLA_ERROR_CUDA, "%s: %s", who, cudaGetErrorString(cudaGetLastError()));
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= reps;
        if (ms < top) {
            top = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != COLA_SUCCESS)
        return s;
    best->k_tile = pick.k_tile;
    best->unroll = pick.unroll;
    best->min_blocks = pick.min_blocks;
    best->gather_batch_rows = pick.gather;
    if (best_ms)
        *best_ms = top;
    if (from_cache)
        *from_cache = 0;
    if (cache_path) {
        SpmmTuneEntry e;
        e.k_tile = pick.k_tile;
        e.unroll = pick.unroll;
        e.min_blocks = pick.min_blocks;
        e.gather_batch_rows = pick.gather;
        e.ms = top;
        COLA_REQUIRE(spmm_tune_cache_append(cache_path, key, e), COLA_ERROR_IO, "%s: cannot append to %s", who,
                     cache_path);
    }
    return COLA_SUCCESS;
}
