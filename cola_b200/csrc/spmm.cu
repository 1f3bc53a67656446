// Launchers, kernel-level C ABI and the device-resident graph of the
// partitioned SpMM (sm_100a).
#include <algorithm>
#include <climits>
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include <cuda.h>  // CUcontext and CUresult, for the context id read through the runtime
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.h"
#include "prep.h"
#include "graph.h"
#include "spmm_kernels.cuh"
#include "spmm_rows.cuh"

using cola::dev::GatherSeg;
using cola::dev::PartDesc;

namespace cola {


// Kernel launches issued by this thread (cola_spmm reports the count of its last call).
thread_local int64_t t_launches = 0;

int sm_count()
{
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64)
        dev = 0;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

// Resident blocks per SM for a kernel (cached by function address).
int blocks_per_sm(const void *fn, int threads)
{
    static std::mutex mu;
    static std::unordered_map<const void *, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(fn);
    if (it != cache.end())
        return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, 0) != cudaSuccess || n <= 0)
        n = 1;
    cache[fn] = n;
    return n;
}

int64_t grid_for(const void *fn, int64_t items)
{
    const int64_t need = (items + dev::kWarpsPerBlock - 1) / dev::kWarpsPerBlock;
    const int64_t full = (int64_t)sm_count() * blocks_per_sm(fn, dev::kThreads);
    return std::max<int64_t>(1, std::min(need, full));
}



// ---------------------------------------------------------------------------
// fused kernel dispatch
// ---------------------------------------------------------------------------
struct FusedArgs {
    const PartDesc *parts;  // device table, or nullptr to use `single`
    PartDesc single;
    int nparts;
    int64_t total;
    const void *X;
    int64_t ldx;
    float *Y;
    int64_t ldy;
    int K;
    cola_dtype xdt;
    bool vec;  // 16-byte vector path allowed
};

template <typename TR, int LG, int NV, int UNROLL, bool VEC_Y, int MINB = 1>
static cola_status launch_fused_t(const FusedArgs &a, cudaStream_t st)
{
    using T = typename dev::ElemOf<TR>::T;
    constexpr int W = LG * NV * TR::E;
    auto fn = dev::fused_spmm_kernel<TR, LG, NV, UNROLL, VEC_Y, MINB>;
    // one warp per chunk (as many blocks as the chunks need): measured 11 %
    // faster than a persistent grid for this kernel, whose items are short
    const int64_t gx = std::max<int64_t>(1, (a.total + dev::kWarpsPerBlock - 1) / dev::kWarpsPerBlock);
    const int gy = (a.K + W - 1) / W;
    t_launches++;
    fn<<<dim3((unsigned)gx, (unsigned)gy), dev::kThreads, 0, st>>>(a.parts, a.single, a.nparts, a.total,
                                                                   static_cast<const T *>(a.X), a.ldx, a.Y, a.ldy,
                                                                   a.K);
    COLA_CUDA(cudaGetLastError());
    return COLA_SUCCESS;
}

template <typename TR, bool VEC_Y>
static cola_status launch_fused_geo(const FusedArgs &a, int V, cudaStream_t st)
{
    // V = vectors (of TR::E elements) per row
    if (V <= 1)
        return launch_fused_t<TR, 1, 1, 4, VEC_Y>(a, st);
    if (V <= 2)
        return launch_fused_t<TR, 2, 1, 4, VEC_Y>(a, st);
    if (V <= 4)
        return launch_fused_t<TR, 4, 1, 4, VEC_Y>(a, st);
    if (V <= 8)
        return launch_fused_t<TR, 8, 1, 4, VEC_Y>(a, st);
    if (V <= 16)
        return launch_fused_t<TR, 16, 1, 4, VEC_Y>(a, st);
    if (V <= 32) {
        // FP32 rows of 65-128 features (K = 128 in the reference's runs): one row in
        // flight per warp and 32 registers, so 8 blocks (64 warps) fit an SM --
        // measured 4 % faster than 2 rows in flight at 6 blocks on the
        // per-partition launches of an R-MAT scale-20 graph at K = 128
        if constexpr (std::is_same<TR, dev::VecTraits<float>>::value)
            return launch_fused_t<TR, 32, 1, 1, VEC_Y, 8>(a, st);
        return launch_fused_t<TR, 32, 1, 2, VEC_Y>(a, st);  // 2 rows in flight: fewer registers, more warps
    }
    if (V <= 64)
        return launch_fused_t<TR, 32, 2, 2, VEC_Y>(a, st);
    return launch_fused_t<TR, 32, 4, 2, VEC_Y>(a, st);
}

static cola_status launch_fused(const FusedArgs &a, cudaStream_t st)
{
    if (a.total <= 0 || a.K <= 0)
        return COLA_SUCCESS;
    if (a.xdt == COLA_FLOAT32) {
        if (a.vec)
            return launch_fused_geo<dev::VecTraits<float>, true>(a, a.K / 4, st);
        return launch_fused_geo<dev::ScalarTraits<float>, false>(a, a.K, st);
    }
    if (a.vec)
        return launch_fused_geo<dev::VecTraits<__nv_bfloat16>, true>(a, a.K / 8, st);
    return launch_fused_geo<dev::ScalarTraits<__nv_bfloat16>, false>(a, a.K, st);
}

// Whether the 16-byte vector path applies to X (and staged rows) / Y.
static bool vec_ok(cola_dtype xdt, const void *X, int64_t ldx, const void *stage, int64_t ld_stage, const float *Y,
                   int64_t ldy, int K)
{
    const int E = xdt == COLA_FLOAT32 ? 4 : 8;
    if (K % E || ldx % E || !aligned16(X))
        return false;
    if (stage && (ld_stage % E || !aligned16(stage)))
        return false;
    if (ldy % 4 || !aligned16(Y))
        return false;
    return true;
}

// ---------------------------------------------------------------------------
// gather dispatch
// ---------------------------------------------------------------------------
// Set by a kernel whose bounded wait ran out (read and cleared by
// cola_device_error_check); one per device.
__device__ int g_dev_error = 0;

static int *device_error_flag()
{
    static std::mutex mu;
    static std::unordered_map<int, int *> by_dev;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    auto it = by_dev.find(dev);
    if (it != by_dev.end())
        return it->second;
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dev_error) != cudaSuccess)
        return nullptr;
    by_dev[dev] = static_cast<int *>(p);
    return static_cast<int *>(p);
}

static std::atomic<int> g_gather_bulk{0};  // off: the vector gather measured as fast or faster
static std::atomic<uint32_t> g_gather_wait_limit{dev::kWaitLimitDefault};

// Bulk-copy (TMA) gather, when switched on, for rows of 1 KB or more (measured
// alone: within 1 % of the vector gather from 1 KB to 4 KB, behind below 1 KB;
// inside the BUFFER schedule's 4,096-row batches 2-7 % behind) when every row and
// address is 16-byte aligned and at least two row slots fit a warp's share of
// shared memory; returns false to leave the rows to the vector gather.
template <typename T>
static bool launch_gather_bulk(const GatherSeg *segs, const GatherSeg &single, int nsegs, int64_t total,
                               const void *src, int64_t ld_src, void *dst, int64_t ld_dst, int K, cudaStream_t st,
                               cola_status &rc)
{
    const int64_t bytes = (int64_t)K * (int64_t)sizeof(T);
    if (!g_gather_bulk.load() || bytes < 1024 || bytes % 16 || (ld_src * (int64_t)sizeof(T)) % 16 ||
        (ld_dst * (int64_t)sizeof(T)) % 16 || !aligned16(src) || !aligned16(dst))
        return false;
    constexpr int kBudget = 200 * 1024;  // dynamic shared memory per block (one block per SM)
    const int slot = (int)((bytes + 127) / 128 * 128);
    const int ns = (int)std::min<int64_t>(dev::kGatherMaxSlots, kBudget / dev::kWarpsPerBlock / std::max(slot, 1));
    if (ns < 2)
        return false;
    int *err = device_error_flag();
    if (!err)
        return false;
    auto fn = dev::gather_rows_bulk_kernel<T>;
    const size_t smem = (size_t)dev::kWarpsPerBlock * ns * (slot + 8);
    {
        static std::mutex mu;
        static std::unordered_map<int, size_t> set_for;  // per device: largest dynamic size allowed so far
        int d = 0;
        cudaGetDevice(&d);
        std::lock_guard<std::mutex> lk(mu);
        size_t &have = set_for[d * 2 + (sizeof(T) == 4 ? 0 : 1)];
        if (have < smem) {
            if (cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                cudaSuccess)
                return false;
            have = smem;
        }
    }
    const int64_t need = (total + dev::kWarpsPerBlock - 1) / dev::kWarpsPerBlock;
    const int64_t gx = std::max<int64_t>(1, std::min<int64_t>(need, sm_count()));
    // rows per chunk: all ns slots when there are rows enough for every warp
    const int64_t per_warp = (total + gx * dev::kWarpsPerBlock - 1) / (gx * dev::kWarpsPerBlock);
    const int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(ns, per_warp));
    t_launches++;
    fn<<<(unsigned)gx, dev::kThreads, smem, st>>>(segs, single, nsegs, total, static_cast<const T *>(src), ld_src,
                                                  static_cast<T *>(dst), ld_dst, K, ns, chunk, slot,
                                                  g_gather_wait_limit.load(), err);
    const cudaError_t e = cudaGetLastError();
    rc = e == cudaSuccess ? COLA_SUCCESS : fail(COLA_ERROR_CUDA, "gather (bulk copies): %s", cudaGetErrorString(e));
    return true;
}

static cola_status launch_gather(const GatherSeg *segs, const GatherSeg &single, int nsegs, int64_t total,
                                 const void *src, int64_t ld_src, void *dst, int64_t ld_dst, int K, cola_dtype dt,
                                 cudaStream_t st)
{
    if (total <= 0 || K <= 0)
        return COLA_SUCCESS;
    {
        cola_status rc = COLA_SUCCESS;
        if (dt == COLA_FLOAT32 ? launch_gather_bulk<float>(segs, single, nsegs, total, src, ld_src, dst, ld_dst, K,
                                                           st, rc)
                               : launch_gather_bulk<__nv_bfloat16>(segs, single, nsegs, total, src, ld_src, dst,
                                                                   ld_dst, K, st, rc))
            return rc;
    }
    const int E = dt == COLA_FLOAT32 ? 4 : 8;
    const bool vec = K % E == 0 && ld_src % E == 0 && ld_dst % E == 0 && aligned16(src) && aligned16(dst);
#define COLA_GATHER(TR)                                                                                        \
    do {                                                                                                       \
        using T = typename dev::ElemOf<TR>::T;                                                                 \
        auto fn = dev::gather_rows_kernel<TR>;                                                                 \
        const int64_t gx = grid_for((const void *)fn, total);                                                 \
        t_launches++;                                                                                          \
        fn<<<(unsigned)gx, dev::kThreads, 0, st>>>(segs, single, nsegs, total, static_cast<const T *>(src),    \
                                                   ld_src, static_cast<T *>(dst), ld_dst, K);                 \
    } while (0)
    if (dt == COLA_FLOAT32) {
        if (vec)
            COLA_GATHER(dev::VecTraits<float>);
        else
            COLA_GATHER(dev::ScalarTraits<float>);
    } else {
        if (vec)
            COLA_GATHER(dev::VecTraits<__nv_bfloat16>);
        else
            COLA_GATHER(dev::ScalarTraits<__nv_bfloat16>);
    }
#undef COLA_GATHER
    COLA_CUDA(cudaGetLastError());
    return COLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// row-major schedule dispatch
// ---------------------------------------------------------------------------
struct RowsLaunch {
    dev::RowsArgs ra;
    const void *X;
    int64_t ldx;
    void *Y;
    int64_t ldy;
    int K;
    cola_dtype xdt, ydt;
    bool vec;
    int accumulate;
    int unroll;
    int min_blocks;
    int k_tile;
};

template <typename TR, typename TY, int LG, int NV, int UNROLL, bool VEC>
static cola_status launch_rows_t(const RowsLaunch &a, cudaStream_t st)
{
    using T = typename dev::ElemOf<TR>::T;
    constexpr int W = LG * NV * TR::E;
    auto fn = dev::rows_spmm_kernel<TR, TY, LG, NV, UNROLL, VEC>;
    const int64_t gx = grid_for((const void *)fn, a.ra.nseg + a.ra.nrows);
    const int gy = (a.K + W - 1) / W;
    t_launches++;
    fn<<<dim3((unsigned)gx, (unsigned)gy), dev::kThreads, 0, st>>>(a.ra, static_cast<const T *>(a.X), a.ldx,
                                                                   static_cast<TY *>(a.Y), a.ldy, a.K, a.accumulate);
    COLA_CUDA(cudaGetLastError());
    return COLA_SUCCESS;
}

template <typename TR, typename TY, bool VEC>
static cola_status launch_rows_geo(const RowsLaunch &a, int V, cudaStream_t st)
{
    if (V <= 1)
        return launch_rows_t<TR, TY, 1, 1, 4, VEC>(a, st);
    if (V <= 2)
        return launch_rows_t<TR, TY, 2, 1, 4, VEC>(a, st);
    if (V <= 4)
        return launch_rows_t<TR, TY, 4, 1, 4, VEC>(a, st);
    if (V <= 8)
        return launch_rows_t<TR, TY, 8, 1, 4, VEC>(a, st);
    if (V <= 16)
        return launch_rows_t<TR, TY, 16, 1, 4, VEC>(a, st);
    if (V <= 32) {
        if (a.unroll == 8)
            return launch_rows_t<TR, TY, 32, 1, 8, VEC>(a, st);
        if (a.unroll == 2)
            return launch_rows_t<TR, TY, 32, 1, 2, VEC>(a, st);
        return launch_rows_t<TR, TY, 32, 1, 4, VEC>(a, st);
    }
    if (V <= 64) {
        if (a.unroll == 4 || a.unroll == 8)
            return launch_rows_t<TR, TY, 32, 2, 4, VEC>(a, st);
        return launch_rows_t<TR, TY, 32, 2, 2, VEC>(a, st);
    }
    return launch_rows_t<TR, TY, 32, 4, 2, VEC>(a, st);
}

static cola_status launch_rows(const RowsLaunch &a, cudaStream_t st)
{
    if (a.ra.nseg + a.ra.nrows <= 0 || a.K <= 0)
        return COLA_SUCCESS;
    using BF = __nv_bfloat16;
    if (a.xdt == COLA_FLOAT32) {
        if (a.ydt == COLA_FLOAT32)
            return a.vec ? launch_rows_geo<dev::VecTraits<float>, float, true>(a, a.K / 4, st)
                         : launch_rows_geo<dev::ScalarTraits<float>, float, false>(a, a.K, st);
        return a.vec ? launch_rows_geo<dev::VecTraits<float>, BF, true>(a, a.K / 4, st)
                     : launch_rows_geo<dev::ScalarTraits<float>, BF, false>(a, a.K, st);
    }
    if (a.ydt == COLA_FLOAT32)
        return a.vec ? launch_rows_geo<dev::VecTraits<BF>, float, true>(a, a.K / 8, st)
                     : launch_rows_geo<dev::ScalarTraits<BF>, float, false>(a, a.K, st);
    return a.vec ? launch_rows_geo<dev::VecTraits<BF>, BF, true>(a, a.K / 8, st)
                 : launch_rows_geo<dev::ScalarTraits<BF>, BF, false>(a, a.K, st);
}

template <typename TR, typename TY, int LG, int NV, int UNROLL, bool VEC, int MINB = 1>
static cola_status launch_block_t(const dev::BlockArgs &ba, const RowsLaunch &a, cudaStream_t st)
{
    using T = typename dev::ElemOf<TR>::T;
    constexpr int W = LG * NV * TR::E;
    const int64_t ntile = (a.K + W - 1) / W;
    if constexpr (LG == 32) {
        if (a.k_tile > 0 && ntile > 1) {
            // a requested tile width: one grid sweeps the tiles one after another
            auto fn = dev::rowblock_tiled_kernel<TR, TY, NV, UNROLL, MINB>;
            const int64_t gx = grid_for((const void *)fn, (ba.nseg + ba.ntask) * ntile);
            t_launches++;
            fn<<<(unsigned)gx, dev::kThreads, 0, st>>>(ba, static_cast<const T *>(a.X), a.ldx,
                                                       static_cast<TY *>(a.Y), a.ldy, a.K, a.accumulate);
            COLA_CUDA(cudaGetLastError());
            return COLA_SUCCESS;
        }
    }
    if (ba.queue && ntile <= dev::kMaxItemQueues) {
        // items drawn from the graph's counters: a warp that met slow items draws fewer
        auto fn = dev::rowblock_spmm_kernel<TR, TY, LG, NV, UNROLL, VEC, MINB, true>;
        const int64_t gx = grid_for((const void *)fn, ba.nseg + ba.ntask);
        t_launches++;
        fn<<<dim3((unsigned)gx, (unsigned)ntile), dev::kThreads, 0, st>>>(ba, static_cast<const T *>(a.X), a.ldx,
                                                                          static_cast<TY *>(a.Y), a.ldy, a.K,
                                                                          a.accumulate);
        COLA_CUDA(cudaGetLastError());
        return COLA_SUCCESS;
    }
    auto fn = dev::rowblock_spmm_kernel<TR, TY, LG, NV, UNROLL, VEC, MINB>;
    const int64_t gx = grid_for((const void *)fn, ba.nseg + ba.ntask);
    t_launches++;
    fn<<<dim3((unsigned)gx, (unsigned)ntile), dev::kThreads, 0, st>>>(ba, static_cast<const T *>(a.X), a.ldx,
                                                                      static_cast<TY *>(a.Y), a.ldy, a.K,
                                                                      a.accumulate);
    COLA_CUDA(cudaGetLastError());
    return COLA_SUCCESS;
}

// Narrow passes (a full warp on a 64- or 128-feature tile, 8 or 4 bytes per
// lane): loads in flight 4 or 8, resident blocks per SM 4, 6 or 8.
template <typename TR, typename TY>
static cola_status launch_block_narrow(const dev::BlockArgs &ba, const RowsLaunch &a, cudaStream_t st)
{
    const int mb = a.min_blocks == 6 || a.min_blocks == 8 ? a.min_blocks : 4;
    if (a.unroll == 8) {
        if (mb == 8)
            return launch_block_t<TR, TY, 32, 1, 8, true, 8>(ba, a, st);
        if (mb == 6)
            return launch_block_t<TR, TY, 32, 1, 8, true, 6>(ba, a, st);
        return launch_block_t<TR, TY, 32, 1, 8, true, 4>(ba, a, st);
    }
    if (mb == 8)
        return launch_block_t<TR, TY, 32, 1, 4, true, 8>(ba, a, st);
    if (mb == 6)
        return launch_block_t<TR, TY, 32, 1, 4, true, 6>(ba, a, st);
    return launch_block_t<TR, TY, 32, 1, 4, true, 4>(ba, a, st);
}

// V = 16-byte vectors per row: LG lanes per row tile, G = 32/LG lane groups.
template <typename TR, typename TY>
static cola_status launch_block_geo(const dev::BlockArgs &ba, const RowsLaunch &a, int V, cudaStream_t st)
{
    if (V <= 1)
        return launch_block_t<TR, TY, 1, 1, 1, true>(ba, a, st);
    if (V <= 2)
        return launch_block_t<TR, TY, 2, 1, 2, true>(ba, a, st);
    if (V <= 4)
        return launch_block_t<TR, TY, 4, 1, 4, true, 4>(ba, a, st);
    if (V <= 8)
        return launch_block_t<TR, TY, 8, 1, 4, true, 4>(ba, a, st);
    if (V <= 16)
        return launch_block_t<TR, TY, 16, 1, 4, true, 4>(ba, a, st);
    if (V <= 32) {
        if (a.unroll == 8)
            return launch_block_t<TR, TY, 32, 1, 8, true>(ba, a, st);
        if (a.unroll == 2)
            return launch_block_t<TR, TY, 32, 1, 2, true>(ba, a, st);
        if (a.unroll == 6)
            return launch_block_t<TR, TY, 32, 1, 6, true>(ba, a, st);
        // resident blocks per SM: measured best 3 for FP32 X (K = 128: 3 % faster
        // than 4) and 4 for BF16 X (5 % faster than 3)
        const int mb = a.min_blocks > 0 ? a.min_blocks : (TR::E == 4 ? 3 : 4);
        if (mb == 3)
            return launch_block_t<TR, TY, 32, 1, 4, true, 3>(ba, a, st);
        if (mb == 5)
            return launch_block_t<TR, TY, 32, 1, 4, true, 5>(ba, a, st);
        if (mb == 6)
            return launch_block_t<TR, TY, 32, 1, 4, true, 6>(ba, a, st);
        return launch_block_t<TR, TY, 32, 1, 4, true, 4>(ba, a, st);
    }
    if (V <= 64) {
        if (a.unroll == 4 || a.unroll == 8)
            return launch_block_t<TR, TY, 32, 2, 4, true>(ba, a, st);
        return launch_block_t<TR, TY, 32, 2, 2, true>(ba, a, st);
    }
    return launch_block_t<TR, TY, 32, 4, 2, true>(ba, a, st);
}

// Feature tile of one pass for the requested k_tile (0 = the library's
// choice), in the regime where a full warp covers one tile (K >= 128 FP32 X,
// K >= 256 BF16 X); 0 where k_tile does not apply.
static int rows_k_tile(cola_dtype xdt, int K, int k_tile)
{
    const int e16 = xdt == COLA_FLOAT32 ? 4 : 8;
    if (K < 32 * e16 || k_tile <= 0)
        return 0;
    if (xdt == COLA_FLOAT32)
        return k_tile == 64 || k_tile == 128 || k_tile == 256 || k_tile == 512 ? k_tile : 0;
    return k_tile == 64 || k_tile == 128 || k_tile == 256 || k_tile == 512 || k_tile == 1024 ? k_tile : 0;
}

// Row-block streaming launch (vector path).
static cola_status launch_block(const dev::BlockArgs &ba, const RowsLaunch &a, cudaStream_t st)
{
    if (ba.nseg + ba.ntask <= 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(ba.nseg + ba.ntask < INT32_MAX, COLA_ERROR_UNSUPPORTED, "cola_spmm: %lld work items (2^31 at most)",
                 (long long)(ba.nseg + ba.ntask));
    using BF = __nv_bfloat16;
    const int kt = rows_k_tile(a.xdt, a.K, a.k_tile);
    if (kt > 0) {
        // every tile width sums each element in the same order (one lane group)
        const int e16 = a.xdt == COLA_FLOAT32 ? 4 : 8;
        if (a.xdt == COLA_FLOAT32 && kt == 64)
            return a.ydt == COLA_FLOAT32 ? launch_block_narrow<dev::NarrowTraits<float, 8>, float>(ba, a, st)
                                         : launch_block_narrow<dev::NarrowTraits<float, 8>, BF>(ba, a, st);
        if (a.xdt == COLA_BFLOAT16 && kt == 128)
            return a.ydt == COLA_FLOAT32 ? launch_block_narrow<dev::NarrowTraits<BF, 8>, float>(ba, a, st)
                                         : launch_block_narrow<dev::NarrowTraits<BF, 8>, BF>(ba, a, st);
        if (a.xdt == COLA_BFLOAT16 && kt == 64)
            return a.ydt == COLA_FLOAT32 ? launch_block_narrow<dev::NarrowTraits<BF, 4>, float>(ba, a, st)
                                         : launch_block_narrow<dev::NarrowTraits<BF, 4>, BF>(ba, a, st);
        // 16-byte vectors, NV per lane: V = kt / e16 selects the geometry below
        const int V = kt / e16;
        if (a.xdt == COLA_FLOAT32)
            return a.ydt == COLA_FLOAT32 ? launch_block_geo<dev::VecTraits<float>, float>(ba, a, V, st)
                                         : launch_block_geo<dev::VecTraits<float>, BF>(ba, a, V, st);
        return a.ydt == COLA_FLOAT32 ? launch_block_geo<dev::VecTraits<BF>, float>(ba, a, V, st)
                                     : launch_block_geo<dev::VecTraits<BF>, BF>(ba, a, V, st);
    }
    if (a.xdt == COLA_FLOAT32)
        return a.ydt == COLA_FLOAT32 ? launch_block_geo<dev::VecTraits<float>, float>(ba, a, a.K / 4, st)
                                     : launch_block_geo<dev::VecTraits<float>, BF>(ba, a, a.K / 4, st);
    return a.ydt == COLA_FLOAT32 ? launch_block_geo<dev::VecTraits<BF>, float>(ba, a, a.K / 8, st)
                                 : launch_block_geo<dev::VecTraits<BF>, BF>(ba, a, a.K / 8, st);
}

// Vector path of the row-major schedule: X rows in 16-byte vectors, Y rows
// written E elements at a time (E*sizeof(TY) bytes, aligned).
bool vec_ok_rows(cola_dtype xdt, const void *X, int64_t ldx, cola_dtype ydt, const void *Y, int64_t ldy, int K)
{
    const int E = xdt == COLA_FLOAT32 ? 4 : 8;
    const int ysz = ydt == COLA_FLOAT32 ? 4 : 2;
    if (K % E || ldx % E || ldx > INT32_MAX || !aligned16(X))
        return false;
    if (ldy % E || ((uintptr_t)Y % (uintptr_t)(E * ysz)) != 0)
        return false;
    return true;
}

static PartDesc part_desc_zero()
{
    PartDesc d;
    std::memset(&d, 0, sizeof d);
    return d;
}

static cola_status check_dim(int32_t dim, int32_t npp)
{
    COLA_REQUIRE(dim >= 1, COLA_ERROR_INVALID_ARGUMENT, "dim must be >= 1 (got %d)", dim);
    COLA_REQUIRE(npp >= 1, COLA_ERROR_INVALID_ARGUMENT, "nodesPerPE must be >= 1 (got %d)", npp);
    return COLA_SUCCESS;
}

}  // namespace cola

using namespace cola;

// ===========================================================================
// Kernel-level C ABI (drop-ins for include/dist_spmm_ppl_batch.cuh launchers)
// ===========================================================================
extern "C" {

cola_status cola_ppl0_batch_spmm(float *output, const float *input, const int32_t *csr_rowPtr_l,
                                 const int32_t *csr_colIdx_l, const int32_t *csr_rowIdx_zip_l,
                                 const float *csr_val_l, const int32_t *csc_colPtr_r, const int32_t *csc_rowIdx_r,
                                 const int32_t *csc_colIdx_zip_r, const float *csc_val_r, int32_t local_row_lb,
                                 int32_t remote_col_lb, int32_t local_row_num, int32_t remote_col_num, int32_t dim,
                                 int32_t nodesPerPE, int32_t peid, cola_stream_t stream)
{
    (void)local_row_lb;  // unused by the reference kernel too (dist_spmm_ppl_batch.cuh:164-167)
    COLA_TRY(check_dim(dim, nodesPerPE));
    COLA_REQUIRE(local_row_num >= 0 && remote_col_num >= 0 && remote_col_lb >= 0 && peid >= 0,
                 COLA_ERROR_INVALID_ARGUMENT, "cola_ppl0_batch_spmm: negative count or offset");
    const int64_t T = (int64_t)local_row_num + remote_col_num;
    if (T == 0)
        return COLA_SUCCESS;  // :232
    COLA_REQUIRE(output && input, COLA_ERROR_INVALID_ARGUMENT, "cola_ppl0_batch_spmm: null dense pointer");
    COLA_REQUIRE(local_row_num == 0 || (csr_rowPtr_l && csr_colIdx_l && csr_rowIdx_zip_l && csr_val_l),
                 COLA_ERROR_INVALID_ARGUMENT, "cola_ppl0_batch_spmm: null local CSR array");
    COLA_REQUIRE(remote_col_num == 0 || (csc_colPtr_r && csc_rowIdx_r && csc_colIdx_zip_r && csc_val_r),
                 COLA_ERROR_INVALID_ARGUMENT, "cola_ppl0_batch_spmm: null remote CSC array");
    PartDesc d = part_desc_zero();
    d.l_ptr = csr_rowPtr_l;
    d.l_col = csr_colIdx_l;
    d.l_row = csr_rowIdx_zip_l;
    d.l_val = csr_val_l;
    d.r_ptr = csc_colPtr_r;
    d.r_row = csc_rowIdx_r;
    d.r_col = csc_colIdx_zip_r;
    d.r_val = csc_val_r;
    d.l_begin = 0;
    d.l_num = local_row_num;
    d.r_begin = remote_col_lb;
    d.r_num = remote_col_num;
    d.x_local0 = 0;
    d.x_remote0 = -(int64_t)peid * nodesPerPE;
    d.r_mode = dev::kRemoteFromX;
    FusedArgs a{nullptr, d, 1, T, input, dim, output, dim, dim, COLA_FLOAT32,
                vec_ok(COLA_FLOAT32, input, dim, nullptr, 0, output, dim, dim)};
    return launch_fused(a, (cudaStream_t)stream);
}

cola_status cola_ppl0_batch_spmm_seq(float *output, const float *input, const int32_t *csr_rowPtr_l,
                                     const int32_t *csr_colIdx_l, const int32_t *csr_rowIdx_zip_l,
                                     const float *csr_val_l, const int32_t *csc_colPtr_r,
                                     const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r,
                                     const float *csc_val_r, int32_t local_row_lb, int32_t remote_col_lb,
                                     int32_t local_row_num, int32_t remote_col_num, int32_t dim,
                                     int32_t nodesPerPE, int32_t peid, cola_stream_t stream)
{
    return cola_ppl0_batch_spmm(output, input, csr_rowPtr_l, csr_colIdx_l, csr_rowIdx_zip_l, csr_val_l,
                                csc_colPtr_r, csc_rowIdx_r, csc_colIdx_zip_r, csc_val_r, local_row_lb,
                                remote_col_lb, local_row_num, remote_col_num, dim, nodesPerPE, peid, stream);
}

cola_status cola_ppl0_batch_buffer_spmm(float *output, const float *input, float *comm_buffer,
                                        const int32_t *csr_rowPtr_l, const int32_t *csr_colIdx_l,
                                        const int32_t *csr_rowIdx_zip_l, const float *csr_val_l,
                                        const int32_t *csc_colPtr_r, const int32_t *csc_rowIdx_r,
                                        const int32_t *csc_colIdx_zip_r, const float *csc_val_r,
                                        int32_t local_row_lb, int32_t remote_col_lb, int32_t local_row_num,
                                        int32_t remote_col_num, int32_t dim, int32_t nodesPerPE, int32_t peid,
                                        cola_stream_t stream)
{
    (void)local_row_lb;
    COLA_TRY(check_dim(dim, nodesPerPE));
    COLA_REQUIRE(local_row_num >= 0 && remote_col_num >= 0 && remote_col_lb >= 0 && peid >= 0,
                 COLA_ERROR_INVALID_ARGUMENT, "cola_ppl0_batch_buffer_spmm: negative count or offset");
    const int64_t T = (int64_t)local_row_num + remote_col_num;
    if (T == 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(output && input && (remote_col_num == 0 || comm_buffer), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_ppl0_batch_buffer_spmm: null dense pointer");
    cudaStream_t st = (cudaStream_t)stream;
    float *stage = comm_buffer ? comm_buffer + (int64_t)remote_col_lb * dim : nullptr;
    if (remote_col_num > 0) {
        GatherSeg s;
        std::memset(&s, 0, sizeof s);
        s.idx = csc_colIdx_zip_r + remote_col_lb;
        s.n = remote_col_num;
        s.src_row0 = -(int64_t)peid * nodesPerPE;
        s.dst_row0 = 0;
        COLA_TRY(launch_gather(nullptr, s, 1, remote_col_num, input, dim, stage, dim, dim, COLA_FLOAT32, st));
    }
    PartDesc d = part_desc_zero();
    d.l_ptr = csr_rowPtr_l;
    d.l_col = csr_colIdx_l;
    d.l_row = csr_rowIdx_zip_l;
    d.l_val = csr_val_l;
    d.r_ptr = csc_colPtr_r;
    d.r_row = csc_rowIdx_r;
    d.r_col = csc_colIdx_zip_r;
    d.r_val = csc_val_r;
    d.l_num = local_row_num;
    d.r_begin = remote_col_lb;
    d.r_num = remote_col_num;
    d.r_mode = dev::kRemoteStagedChunk;
    d.stage = stage;
    d.ld_stage = dim;
    FusedArgs a{nullptr, d, 1, T, input, dim, output, dim, dim, COLA_FLOAT32,
                vec_ok(COLA_FLOAT32, input, dim, stage, dim, output, dim, dim)};
    return launch_fused(a, st);
}

cola_status cola_ppl_batch_spmm(float *output, const float *input, const int32_t *csc_colPtr_r,
                                const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r,
                                const float *csc_val_r, int32_t local_col_lb, int32_t local_col_ub,
                                int32_t remote_col_lb, int32_t remote_col_ub, int32_t stage, const int32_t *idx_ppl,
                                int32_t dim, int32_t nodesPerPE, int32_t group_size, int32_t group_offset,
                                int32_t peid, cola_stream_t stream)
{
    (void)stage;
    COLA_TRY(check_dim(dim, nodesPerPE));
    COLA_REQUIRE(group_size >= 1 && remote_col_lb >= 0 && peid >= 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_ppl_batch_spmm: bad group_size/offset");
    const int64_t T = (int64_t)remote_col_ub - remote_col_lb;
    if (T <= 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(output && input && idx_ppl && csc_colPtr_r && csc_rowIdx_r && csc_colIdx_zip_r && csc_val_r,
                 COLA_ERROR_INVALID_ARGUMENT, "cola_ppl_batch_spmm: null pointer");
    PartDesc d = part_desc_zero();
    d.r_ptr = csc_colPtr_r;
    d.r_row = csc_rowIdx_r;
    d.r_col = csc_colIdx_zip_r;
    d.r_val = csc_val_r;
    d.r_begin = remote_col_lb;
    d.r_num = (int32_t)T;
    d.r_mode = dev::kRemoteStageBuffer;
    d.stage = input;
    d.ld_stage = dim;
    d.pe_stride = (int64_t)nodesPerPE * dim;
    d.idx_ppl = idx_ppl;
    d.npp = nodesPerPE;
    d.gs = group_size;
    d.group_offset = group_offset;
    d.peid = peid;
    d.local_col_lb = local_col_lb;
    d.local_col_ub = local_col_ub;
    FusedArgs a{nullptr, d, 1, T, input, dim, output, dim, dim, COLA_FLOAT32,
                vec_ok(COLA_FLOAT32, input, dim, input, dim, output, dim, dim)};
    return launch_fused(a, (cudaStream_t)stream);
}

cola_status cola_batching_data_ppl(const float *input, float *send, const int32_t *put_colIdx, int32_t nemb,
                                   int32_t dim, int32_t nodesPerPE, int32_t group_size, cola_stream_t stream)
{
    (void)group_size;
    COLA_TRY(check_dim(dim, nodesPerPE));
    if (nemb <= 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(input && send && put_colIdx, COLA_ERROR_INVALID_ARGUMENT, "cola_batching_data_ppl: null pointer");
    GatherSeg s;
    std::memset(&s, 0, sizeof s);
    s.idx = put_colIdx;
    s.n = nemb;
    s.mod = nodesPerPE;
    return launch_gather(nullptr, s, 1, nemb, input, dim, send, dim, dim, COLA_FLOAT32, (cudaStream_t)stream);
}

}  // extern "C"

// ===========================================================================
// Device-resident graph
// ===========================================================================

namespace cola {

cola_status ensure(void *&p, size_t &have, size_t need)
{
    if (have >= need)
        return COLA_SUCCESS;
    if (p)
        COLA_CUDA(cudaFree(p));
    p = nullptr;
    have = 0;
    COLA_CUDA(cudaMalloc(&p, need));
    have = need;
    return COLA_SUCCESS;
}

RowViewParams row_view_params(int64_t nnz, const cola_upload_opts *opts)
{
    const int64_t warps = (int64_t)sm_count() * 32;
    int64_t t = 256;
    if (nnz < 128 * 4 * warps)
        t = 128;
    while (t >= 256 && t < 512 && 2 * t * 16 * warps <= nnz)
        t *= 2;
    RowViewParams p;
    p.hub_threshold = opts && opts->hub_threshold > 0 ? opts->hub_threshold : (int32_t)t;
    p.hub_segment = opts && opts->hub_segment > 0 ? opts->hub_segment : (int32_t)t;
    p.task_entries = opts && opts->task_entries > 0 ? opts->task_entries : (int32_t)(t / 2);
    return p;
}

void graph_release(cola_graph *g)
{
    if (!g)
        return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(g->device);
    cudaFree(g->dmem);
    cudaFree(g->ppl_buf);
    cudaFree(g->stage_buf);
    cudaFree(g->ws);
    cudaFree(g->ws_hub);
    host_pipe_release(g->host_pipe);
    cudaSetDevice(cur);
    delete g;
}

// Arena: sub-allocations of one device allocation, 256-byte aligned.
struct Arena {
    std::vector<std::pair<const void *, size_t>> items;  // host src, bytes
    std::vector<size_t> offs;
    size_t total = 0;
    size_t add(const void *src, size_t bytes)
    {
        size_t o = total;
        items.push_back({src, bytes});
        offs.push_back(o);
        total += (bytes + 255) & ~(size_t)255;
        return o;
    }
};

cola_status graph_upload(const cola_partition_set *ps, const cola_upload_opts *opts, cola_graph *&out,
                                cudaStream_t st)
{
    COLA_REQUIRE(ps, COLA_ERROR_INVALID_ARGUMENT, "cola_graph_upload: partition set is NULL");
    const int32_t P = ps->nparts;
    int32_t gs = opts && opts->group_size > 0 ? opts->group_size : P;
    const int32_t if_split = opts ? opts->if_split : 1;
    COLA_REQUIRE(gs >= 1 && gs <= P && P % gs == 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_graph_upload: group_size %d must divide nparts %d", gs, P);
    for (const PartHost &ph : ps->parts)
        COLA_TRY(validate_partition(*ps, ph));
    std::unique_ptr<cola_graph, void (*)(cola_graph *)> g(new cola_graph(), graph_release);
    COLA_CUDA(cudaGetDevice(&g->device));
    g->N = ps->num_nodes;
    g->P = P;
    g->npp = ps->npp;
    g->gs = gs;
    g->nstages = P / gs;
    g->if_split = if_split;

    // split every partition (src/distSpMM_ppl_batch.cu:79-99)
    struct Split {
        std::vector<int32_t> l_row, l_ptr, r_col, r_ptr;
    };
    std::vector<Split> sp((size_t)P);
    for (int32_t p = 0; p < P; p++) {
        const PartHost &ph = ps->parts[(size_t)p];
        COLA_TRY(nnz_split(ph.l_rowIdx.data(), (int64_t)ph.l_rowIdx.size(), ph.l_rowPtr.data(),
                           (int64_t)ph.l_colIdx.size(), sp[(size_t)p].l_row, sp[(size_t)p].l_ptr));
        if (if_split) {
            COLA_TRY(nnz_split(ph.r_colIdx.data(), (int64_t)ph.r_colIdx.size(), ph.r_colPtr.data(),
                               (int64_t)ph.r_rowIdx.size(), sp[(size_t)p].r_col, sp[(size_t)p].r_ptr));
        } else {
            sp[(size_t)p].r_col.assign(ph.r_colIdx.begin(), ph.r_colIdx.end());
            if (ph.r_colIdx.empty())
                sp[(size_t)p].r_ptr.clear();
            else
                sp[(size_t)p].r_ptr.assign(ph.r_colPtr.begin(), ph.r_colPtr.end());
        }
    }
    // stage tables (pipelined schedule only): work-group column lists are the
    // sorted unique columns of the group's partitions (= prep_torch_ppl.py:24-49)
    std::vector<int32_t> wg_cols;
    std::vector<int64_t> wg_off(1, 0);
    if (g->nstages > 1) {
        for (int32_t s = 0; s < g->nstages; s++) {
            std::vector<int32_t> cols;
            for (int32_t p = s * gs; p < (s + 1) * gs; p++) {
                const PartHost &ph = ps->parts[(size_t)p];
                for (int32_t c : ph.l_colIdx)
                    cols.push_back((int32_t)((int64_t)p * ps->npp + c));
                cols.insert(cols.end(), ph.r_colIdx.begin(), ph.r_colIdx.end());
            }
            std::sort(cols.begin(), cols.end());
            cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
            wg_cols.insert(wg_cols.end(), cols.begin(), cols.end());
            wg_off.push_back((int64_t)wg_cols.size());
        }
        g->tables.resize((size_t)P);
        for (int32_t p = 0; p < P; p++)
            COLA_TRY(stage_tables(p, P, gs, g->N, sp[(size_t)p].r_col.data(), (int64_t)sp[(size_t)p].r_col.size(),
                                  (int64_t)sp[(size_t)p].l_row.size(), wg_cols.data(), wg_off.data(),
                                  g->tables[(size_t)p]));
    }

    // row-major view (build_row_view in prep.cpp): per output row its
    // entries in ascending global column order, hub segments, row tasks
    const bool rows = !(opts && opts->no_row_view);
    RowView rv;
    if (rows) {
        int64_t nnz_all = 0;
        for (const PartHost &ph : ps->parts)
            nnz_all += (int64_t)ph.l_colIdx.size() + (int64_t)ph.r_rowIdx.size();
        const RowViewParams rp = row_view_params(nnz_all, opts);
        g->hub_threshold = rp.hub_threshold;
        g->hub_segment = rp.hub_segment;
        g->task_entries = rp.task_entries;
        COLA_TRY(build_row_view(*ps, g->hub_threshold, g->hub_segment, g->task_entries, rv));
        g->nseg = (int64_t)rv.seg_row.size();
        g->nhub = (int64_t)rv.hub_row.size();
        g->ntask = (int64_t)rv.task_rb.size();
    }

    // one device allocation for everything
    Arena ar;
    struct Offs {
        size_t l_ptr, l_col, l_val, l_row, r_ptr, r_row, r_val, r_col;
    };
    std::vector<Offs> offs((size_t)P);
    for (int32_t p = 0; p < P; p++) {
        const PartHost &ph = ps->parts[(size_t)p];
        const Split &s = sp[(size_t)p];
        Offs &o = offs[(size_t)p];
        o.l_ptr = ar.add(s.l_ptr.data(), s.l_ptr.size() * 4);
        o.l_col = ar.add(ph.l_colIdx.data(), ph.l_colIdx.size() * 4);
        o.l_val = ar.add(ph.l_val.data(), ph.l_val.size() * 4);
        o.l_row = ar.add(s.l_row.data(), s.l_row.size() * 4);
        o.r_ptr = ar.add(s.r_ptr.data(), s.r_ptr.size() * 4);
        o.r_row = ar.add(ph.r_rowIdx.data(), ph.r_rowIdx.size() * 4);
        o.r_val = ar.add(ph.r_val.data(), ph.r_val.size() * 4);
        o.r_col = ar.add(s.r_col.data(), s.r_col.size() * 4);
        g->nnz_l += (int64_t)ph.l_colIdx.size();
        g->nnz_r += (int64_t)ph.r_rowIdx.size();
        g->lchunks += (int64_t)s.l_row.size();
        g->rchunks += (int64_t)s.r_col.size();
        g->rcols += (int64_t)ph.r_colIdx.size();
    }
    std::vector<size_t> idx_offs, put_offs;
    if (g->nstages > 1) {
        for (int32_t p = 0; p < P; p++) {
            const StageTables &t = g->tables[(size_t)p];
            for (const auto &l : t.idx_ppl)
                idx_offs.push_back(ar.add(l.data(), l.size() * 4));
            for (const auto &l : t.put_colIdx)
                put_offs.push_back(ar.add(l.data(), l.size() * 4));
        }
    }
    const size_t desc_fused = ar.add(nullptr, (size_t)P * sizeof(PartDesc));
    size_t desc_stage0 = 0;
    std::vector<size_t> desc_stage, desc_put;
    if (g->nstages > 1) {
        desc_stage0 = ar.add(nullptr, (size_t)P * sizeof(PartDesc));
        for (int32_t s = 1; s < g->nstages; s++) {
            desc_stage.push_back(ar.add(nullptr, (size_t)P * sizeof(PartDesc)));
            desc_put.push_back(ar.add(nullptr, (size_t)P * sizeof(GatherSeg)));
        }
    }
    const size_t desc_buf = ar.add(nullptr, (size_t)P * sizeof(GatherSeg));
    size_t o_rv_ptr = 0, o_rv_col = 0, o_rv_val = 0, o_seg_row = 0, o_seg_beg = 0, o_hub_row = 0, o_hub_seg = 0;
    size_t o_task_rb = 0, o_task_re = 0, o_queue = 0;
    if (rows) {
        o_rv_ptr = ar.add(rv.ptr.data(), rv.ptr.size() * 8);
        o_rv_col = ar.add(rv.col.data(), rv.col.size() * 4);
        o_rv_val = ar.add(rv.val.data(), rv.val.size() * 4);
        o_seg_row = ar.add(rv.seg_row.data(), rv.seg_row.size() * 4);
        o_seg_beg = ar.add(rv.seg_beg.data(), rv.seg_beg.size() * 8);
        o_hub_row = ar.add(rv.hub_row.data(), rv.hub_row.size() * 4);
        o_hub_seg = ar.add(rv.hub_seg.data(), rv.hub_seg.size() * 8);
        o_task_rb = ar.add(rv.task_rb.data(), rv.task_rb.size() * 4);
        o_task_re = ar.add(rv.task_re.data(), rv.task_re.size() * 4);
        o_queue = ar.add(nullptr, (dev::kMaxItemQueues + 1) * sizeof(unsigned int));  // zero in the image
    }
    ar.total = std::max<size_t>(ar.total, 256);
    COLA_CUDA(cudaMalloc(&g->dmem, ar.total));
    g->dbytes = ar.total;
    char *base = static_cast<char *>(g->dmem);
    auto at = [&](size_t o) { return reinterpret_cast<const int32_t *>(base + o); };
    if (rows) {
        g->has_rows = true;
        g->rv_ptr = reinterpret_cast<const int64_t *>(base + o_rv_ptr);
        g->rv_col = at(o_rv_col);
        g->rv_val = reinterpret_cast<const float *>(base + o_rv_val);
        g->seg_row = at(o_seg_row);
        g->seg_beg = reinterpret_cast<const int64_t *>(base + o_seg_beg);
        g->hub_row = at(o_hub_row);
        g->hub_seg = reinterpret_cast<const int64_t *>(base + o_hub_seg);
        g->task_rb = at(o_task_rb);
        g->task_re = at(o_task_re);
        g->item_queue = reinterpret_cast<unsigned int *>(base + o_queue);
    }

    // descriptors
    g->zips.resize((size_t)P);
    g->h_fused.resize((size_t)P);
    int64_t item = 0;
    for (int32_t p = 0; p < P; p++) {
        const Offs &o = offs[(size_t)p];
        const Split &s = sp[(size_t)p];
        cola_zip_view &z = g->zips[(size_t)p];
        z.csr_rowPtr = at(o.l_ptr);
        z.csr_colIdx = at(o.l_col);
        z.csr_val = reinterpret_cast<const float *>(base + o.l_val);
        z.csr_rowIdx_zip = at(o.l_row);
        z.csc_colPtr = at(o.r_ptr);
        z.csc_rowIdx = at(o.r_row);
        z.csc_val = reinterpret_cast<const float *>(base + o.r_val);
        z.csc_colIdx_zip = at(o.r_col);
        z.local_chunks = (int32_t)s.l_row.size();
        z.remote_chunks = (int32_t)s.r_col.size();
        z.nnz_l = (int64_t)ps->parts[(size_t)p].l_colIdx.size();
        z.nnz_r = (int64_t)ps->parts[(size_t)p].r_rowIdx.size();
        PartDesc d = part_desc_zero();
        d.l_ptr = z.csr_rowPtr;
        d.l_col = z.csr_colIdx;
        d.l_row = z.csr_rowIdx_zip;
        d.l_val = z.csr_val;
        d.r_ptr = z.csc_colPtr;
        d.r_row = z.csc_rowIdx;
        d.r_col = z.csc_colIdx_zip;
        d.r_val = z.csc_val;
        d.l_num = z.local_chunks;
        d.r_num = z.remote_chunks;
        d.x_local0 = (int64_t)p * g->npp;
        d.x_remote0 = 0;
        d.y_row0 = (int64_t)p * g->npp;
        d.item0 = item;
        d.r_mode = dev::kRemoteFromX;
        item += (int64_t)d.l_num + d.r_num;
        g->h_fused[(size_t)p] = d;
    }
    g->fused_total = item;
    g->d_fused = reinterpret_cast<PartDesc *>(base + desc_fused);
    g->h_bufsegs.assign((size_t)P, GatherSeg{});
    g->d_bufsegs = reinterpret_cast<GatherSeg *>(base + desc_buf);

    std::vector<std::pair<size_t, std::vector<char>>> extra;  // descriptor tables to upload
    auto push_tbl = [&](size_t off, const void *src, size_t bytes) {
        extra.push_back({off, std::vector<char>((const char *)src, (const char *)src + bytes)});
    };
    push_tbl(desc_fused, g->h_fused.data(), (size_t)P * sizeof(PartDesc));

    if (g->nstages > 1) {
        // stage 0: local chunks + intra-group remote chunks of every PE
        std::vector<PartDesc> s0((size_t)P);
        item = 0;
        for (int32_t p = 0; p < P; p++) {
            const StageTables &t = g->tables[(size_t)p];
            PartDesc d = g->h_fused[(size_t)p];
            d.l_begin = t.local_offset[0];
            d.l_num = t.local_offset[1] - t.local_offset[0];
            d.r_begin = t.remote_offset[0];
            d.r_num = t.remote_offset[1] - t.remote_offset[0];
            d.item0 = item;
            item += (int64_t)d.l_num + d.r_num;
            s0[(size_t)p] = d;
        }
        g->stage0_total = item;
        g->d_stage0 = reinterpret_cast<PartDesc *>(base + desc_stage0);
        push_tbl(desc_stage0, s0.data(), s0.size() * sizeof(PartDesc));
        g->h_stage.assign((size_t)g->nstages - 1, std::vector<PartDesc>((size_t)P));
        g->h_put.assign((size_t)g->nstages - 1, std::vector<GatherSeg>((size_t)P));
        for (int32_t s = 1; s < g->nstages; s++) {
            int64_t it = 0, pit = 0;
            for (int32_t p = 0; p < P; p++) {
                const StageTables &t = g->tables[(size_t)p];
                const size_t io = idx_offs[(size_t)p * (g->nstages - 1) + (s - 1)];
                PartDesc d = g->h_fused[(size_t)p];
                d.l_num = 0;
                d.r_begin = t.remote_offset[2 * s];
                d.r_num = t.remote_offset[2 * s + 1] - t.remote_offset[2 * s];
                d.r_mode = dev::kRemoteStageBuffer;
                d.idx_ppl = at(io);
                d.npp = g->npp;
                d.gs = gs;
                d.group_offset = p / gs * gs;
                d.peid = p;
                d.local_col_lb = t.local_offset[2 * s];
                d.local_col_ub = t.local_offset[2 * s + 1];
                d.item0 = it;
                it += d.r_num;
                g->h_stage[(size_t)s - 1][(size_t)p] = d;
                // the put that fills stage s's buffer: PE p sends its list
                // s-1 to target (p - s*gs) mod P  (dist_spmm_ppl_batch.cuh:788-793, 811-816)
                const size_t po = put_offs[(size_t)p * (g->nstages - 1) + (s - 1)];
                GatherSeg q;
                std::memset(&q, 0, sizeof q);
                q.idx = at(po);
                q.n = (int64_t)t.put_colIdx[(size_t)s - 1].size();
                q.src_row0 = 0;  // put lists hold global columns; X is global
                const int32_t target = ((p - s * gs) % P + P) % P;
                q.dst_row0 = (int64_t)target * g->npp;
                q.item0 = pit;
                pit += q.n;
                g->h_put[(size_t)s - 1][(size_t)p] = q;
            }
            g->stage_total.push_back(it);
            g->put_total.push_back(pit);
            g->d_stage.push_back(reinterpret_cast<PartDesc *>(base + desc_stage[(size_t)s - 1]));
            g->d_put.push_back(reinterpret_cast<GatherSeg *>(base + desc_put[(size_t)s - 1]));
            push_tbl(desc_stage[(size_t)s - 1], g->h_stage[(size_t)s - 1].data(), (size_t)P * sizeof(PartDesc));
            push_tbl(desc_put[(size_t)s - 1], g->h_put[(size_t)s - 1].data(), (size_t)P * sizeof(GatherSeg));
        }
    }

    // upload: pack into one pinned-free host image and copy once
    std::vector<char> img(ar.total, 0);
    for (size_t i = 0; i < ar.items.size(); i++)
        if (ar.items[i].first && ar.items[i].second)
            std::memcpy(img.data() + ar.offs[i], ar.items[i].first, ar.items[i].second);
    for (auto &e : extra)
        std::memcpy(img.data() + e.first, e.second.data(), e.second.size());
    COLA_CUDA(cudaMemcpyAsync(g->dmem, img.data(), ar.total, cudaMemcpyHostToDevice, st));
    COLA_CUDA(cudaStreamSynchronize(st));
    out = g.release();
    return COLA_SUCCESS;
}

}  // namespace cola

extern "C" {

cola_status cola_graph_upload(const cola_partition_set *parts, const cola_upload_opts *opts, cola_graph **out,
                              cola_stream_t stream)
{
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "cola_graph_upload: out is NULL");
    *out = nullptr;
    try {
        return graph_upload(parts, opts, *out, (cudaStream_t)stream);
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_graph_upload: host allocation failed");
    }
}

cola_status cola_graph_free(cola_graph *g)
{
    graph_release(g);
    return COLA_SUCCESS;
}

cola_status cola_graph_get_info(const cola_graph *g, cola_graph_info *o)
{
    COLA_REQUIRE(g && o, COLA_ERROR_INVALID_ARGUMENT, "cola_graph_get_info: null argument");
    o->num_nodes = g->N;
    o->nparts = g->P;
    o->nodes_per_part = g->npp;
    o->group_size = g->gs;
    o->nnz_local = g->nnz_l;
    o->nnz_remote = g->nnz_r;
    o->nnz = g->nnz_l + g->nnz_r;
    o->local_chunks = g->lchunks;
    o->remote_chunks = g->rchunks;
    o->remote_cols = g->rcols;
    o->device_bytes = (int64_t)(g->dbytes + g->ppl_bytes + g->stage_bytes + g->ws_bytes + g->ws_hub_bytes);
    o->hub_rows = g->nhub;
    o->hub_segments = g->nseg;
    o->row_tasks = g->ntask;
    o->last_launches = g->last_launches;
    return COLA_SUCCESS;
}

cola_status cola_device_error_check(int32_t *code)
{
    COLA_REQUIRE(code, COLA_ERROR_INVALID_ARGUMENT, "cola_device_error_check: code is NULL");
    *code = 0;
    COLA_CUDA(cudaDeviceSynchronize());
    int v = 0;
    COLA_CUDA(cudaMemcpyFromSymbol(&v, g_dev_error, sizeof(int)));
    if (v) {
        const int zero = 0;
        COLA_CUDA(cudaMemcpyToSymbol(g_dev_error, &zero, sizeof(int)));
    }
    *code = v;
    return COLA_SUCCESS;
}

cola_status cola_set_gather_bulk(int32_t enable)
{
    g_gather_bulk.store(enable ? 1 : 0);
    return COLA_SUCCESS;
}

cola_status cola_set_gather_wait_limit(int64_t polls)
{
    COLA_REQUIRE(polls >= 0 && polls <= (int64_t)dev::kWaitLimitDefault * 64, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_set_gather_wait_limit: polls=%lld (0 .. %lld)", (long long)polls,
                 (long long)dev::kWaitLimitDefault * 64);
    g_gather_wait_limit.store(polls == 0 ? dev::kWaitLimitDefault : (uint32_t)polls);
    return COLA_SUCCESS;
}

cola_status cola_graph_zip_view(const cola_graph *g, int32_t part, cola_zip_view *o)
{
    COLA_REQUIRE(g && o && part >= 0 && part < g->P, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_graph_zip_view: bad argument (part %d)", part);
    COLA_REQUIRE(g->has_split, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_graph_zip_view: a graph built on the device has no split blocks");
    *o = g->zips[(size_t)part];
    return COLA_SUCCESS;
}

static cola_status spmm_impl(cola_graph *g, const void *X, cola_dtype xdt, int64_t ldx, void *Y, cola_dtype ydt,
                             int64_t ldy, int32_t K, const cola_spmm_opts *opts, cola_stream_t stream);

cola_status cola_spmm(cola_graph *g, const void *X, cola_dtype xdt, int64_t ldx, void *Y, cola_dtype ydt,
                      int64_t ldy, int32_t K, const cola_spmm_opts *opts, cola_stream_t stream)
{
    const int64_t before = t_launches;
    const cola_status s = spmm_impl(g, X, xdt, ldx, Y, ydt, ldy, K, opts, stream);
    if (g)
        g->last_launches = t_launches - before;
    return s;
}

static cola_status spmm_impl(cola_graph *g, const void *X, cola_dtype xdt, int64_t ldx, void *Y, cola_dtype ydt,
                             int64_t ldy, int32_t K, const cola_spmm_opts *opts, cola_stream_t stream)
{
    COLA_REQUIRE(g, COLA_ERROR_INVALID_ARGUMENT, "cola_spmm: graph is NULL");
    COLA_REQUIRE(K >= 1 && ldx >= K && ldy >= K, COLA_ERROR_INVALID_ARGUMENT, "cola_spmm: K=%d ldx=%lld ldy=%lld",
                 K, (long long)ldx, (long long)ldy);
    COLA_REQUIRE((xdt == COLA_FLOAT32 || xdt == COLA_BFLOAT16) && (ydt == COLA_FLOAT32 || ydt == COLA_BFLOAT16),
                 COLA_ERROR_INVALID_ARGUMENT, "cola_spmm: unknown dtype");
    COLA_REQUIRE(g->N == 0 || (X && Y), COLA_ERROR_INVALID_ARGUMENT, "cola_spmm: null X or Y");
    const int accumulate = opts ? opts->accumulate : 0;
    int schedule = opts ? opts->schedule : COLA_SCHEDULE_AUTO;
    const int batch_rows = opts && opts->gather_batch_rows > 0 ? opts->gather_batch_rows : 4096;
    COLA_REQUIRE(!(accumulate && ydt != COLA_FLOAT32), COLA_ERROR_UNSUPPORTED,
                 "cola_spmm: accumulate needs an FP32 Y");
    if (schedule == COLA_SCHEDULE_AUTO)
        schedule = g->has_rows ? COLA_SCHEDULE_ROWS : (g->nstages > 1 ? COLA_SCHEDULE_PIPELINE : COLA_SCHEDULE_FUSED);
    COLA_REQUIRE(schedule != COLA_SCHEDULE_ROWS || g->has_rows, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_spmm: the row-major schedule needs a graph uploaded with its row view");
    COLA_REQUIRE(schedule == COLA_SCHEDULE_ROWS || g->has_split, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_spmm: a graph built on the device has the row-major schedule only");
    COLA_REQUIRE(schedule >= COLA_SCHEDULE_FUSED && schedule <= COLA_SCHEDULE_ROWS, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_spmm: unknown schedule %d", schedule);
    COLA_REQUIRE(schedule != COLA_SCHEDULE_PIPELINE || g->nstages > 1, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_spmm: the pipelined schedule needs a graph uploaded with group_size < nparts");
    int cur = 0;
    COLA_CUDA(cudaGetDevice(&cur));
    COLA_REQUIRE(cur == g->device, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_spmm: graph lives on device %d, current device is %d", g->device, cur);
    cudaStream_t st = (cudaStream_t)stream;
    if (g->N == 0)
        return COLA_SUCCESS;

    if (schedule == COLA_SCHEDULE_ROWS) {
        // one writer per output row: Y written directly in its own dtype
        if (g->nseg > 0)
            COLA_TRY(ensure(reinterpret_cast<void *&>(g->ws_hub), g->ws_hub_bytes, (size_t)g->nseg * K * sizeof(float)));
        RowsLaunch a;
        a.ra.rowptr = g->rv_ptr;
        a.ra.col = g->rv_col;
        a.ra.val = g->rv_val;
        a.ra.nrows = g->N;
        a.ra.hub_threshold = g->hub_threshold;
        a.ra.seg_row = g->seg_row;
        a.ra.seg_beg = g->seg_beg;
        a.ra.nseg = g->nseg;
        a.ra.seg_len = g->hub_segment;
        a.ra.ws = g->ws_hub;
        a.ra.ld_ws = K;
        a.X = X;
        a.ldx = ldx;
        a.Y = Y;
        a.ldy = ldy;
        a.K = K;
        a.xdt = xdt;
        a.ydt = ydt;
        a.vec = vec_ok_rows(xdt, X, ldx, ydt, Y, ldy, K);
        a.accumulate = accumulate;
        a.unroll = opts ? opts->unroll : 0;
        a.min_blocks = opts ? opts->min_blocks : 0;
        a.k_tile = opts ? opts->k_tile : 0;
        if (a.vec) {
            dev::BlockArgs ba;
            ba.rowptr = g->rv_ptr;
            ba.col = g->rv_col;
            ba.val = g->rv_val;
            ba.task_rb = g->task_rb;
            ba.task_re = g->task_re;
            ba.ntask = g->ntask;
            ba.seg_row = g->seg_row;
            ba.seg_beg = g->seg_beg;
            ba.nseg = g->nseg;
            ba.seg_len = g->hub_segment;
            ba.ws = g->ws_hub;
            ba.ld_ws = K;
            ba.queue = g->item_queue;
            COLA_TRY(launch_block(ba, a, st));
        } else {
            COLA_TRY(launch_rows(a, st));
        }
        if (g->nhub > 0 && a.vec && K % 4 == 0 && ldy % 4 == 0 &&
            aligned16(g->ws_hub) && ((uintptr_t)Y % (ydt == COLA_FLOAT32 ? 16 : 8)) == 0) {
            const int64_t items = g->nhub * ((K + 127) / 128);
            const int64_t blocks = std::min<int64_t>((items + dev::kWarpsPerBlock - 1) / dev::kWarpsPerBlock,
                                                     (int64_t)sm_count() * 16);
            t_launches++;
            if (ydt == COLA_FLOAT32)
                dev::hub_combine_vec_kernel<float, 4><<<(unsigned)blocks, dev::kThreads, 0, st>>>(
                    g->hub_row, g->hub_seg, g->nhub, g->ws_hub, K, static_cast<float *>(Y), ldy, K, accumulate);
            else
                dev::hub_combine_vec_kernel<__nv_bfloat16, 4><<<(unsigned)blocks, dev::kThreads, 0, st>>>(
                    g->hub_row, g->hub_seg, g->nhub, g->ws_hub, K, static_cast<__nv_bfloat16 *>(Y), ldy, K,
                    accumulate);
            COLA_CUDA(cudaGetLastError());
        } else if (g->nhub > 0) {
            const int64_t blocks = (g->nhub + dev::kWarpsPerBlock - 1) / dev::kWarpsPerBlock;
            t_launches++;
            if (ydt == COLA_FLOAT32)
                dev::hub_combine_kernel<float><<<(unsigned)blocks, dev::kThreads, 0, st>>>(
                    g->hub_row, g->hub_seg, g->nhub, g->ws_hub, K, static_cast<float *>(Y), ldy, K, accumulate);
            else
                dev::hub_combine_kernel<__nv_bfloat16><<<(unsigned)blocks, dev::kThreads, 0, st>>>(
                    g->hub_row, g->hub_seg, g->nhub, g->ws_hub, K, static_cast<__nv_bfloat16 *>(Y), ldy, K,
                    accumulate);
            COLA_CUDA(cudaGetLastError());
        }
        return COLA_SUCCESS;
    }

    // accumulation target
    float *acc = nullptr;
    int64_t ldacc = 0;
    if (ydt == COLA_FLOAT32) {
        acc = static_cast<float *>(Y);
        ldacc = ldy;
    } else {
        COLA_TRY(ensure(reinterpret_cast<void *&>(g->ws), g->ws_bytes, (size_t)g->N * K * sizeof(float)));
        acc = g->ws;
        ldacc = K;
    }
    if (!accumulate) {
        if (ldacc == K)
            COLA_CUDA(cudaMemsetAsync(acc, 0, (size_t)g->N * K * sizeof(float), st));
        else
            COLA_CUDA(cudaMemset2DAsync(acc, (size_t)ldacc * sizeof(float), 0, (size_t)K * sizeof(float),
                                        (size_t)g->N, st));
    }
    const size_t esz = xdt == COLA_FLOAT32 ? 4 : 2;
    const int P = g->P;

    if (schedule == COLA_SCHEDULE_FUSED) {
        FusedArgs a{g->d_fused, part_desc_zero(), P, g->fused_total, X, ldx, acc, ldacc, K, xdt,
                    vec_ok(xdt, X, ldx, nullptr, 0, acc, ldacc, K)};
        COLA_TRY(launch_fused(a, st));
    } else if (schedule == COLA_SCHEDULE_BUFFER) {
        // local chunks of every partition, then per partition the remote rows in
        // batches: gather into the HBM staging buffer, scatter from it.
        const int64_t ldst = (K + 7) / 8 * 8;
        COLA_TRY(ensure(g->stage_buf, g->stage_bytes, (size_t)2 * batch_rows * ldst * esz));
        // one launch for the local parts: r_num = 0 via a host copy of the table
        {
            FusedArgs a{nullptr, part_desc_zero(), 1, 0, X, ldx, acc, ldacc, K, xdt,
                        vec_ok(xdt, X, ldx, nullptr, 0, acc, ldacc, K)};
            for (int32_t p = 0; p < P; p++) {
                PartDesc d = g->h_fused[(size_t)p];
                d.r_num = 0;
                d.item0 = 0;
                a.single = d;
                a.total = d.l_num;
                COLA_TRY(launch_fused(a, st));
            }
        }
        int pp = 0;
        for (int32_t p = 0; p < P; p++) {
            const PartDesc &full = g->h_fused[(size_t)p];
            for (int32_t b0 = 0; b0 < full.r_num; b0 += batch_rows) {
                const int32_t nb = std::min(batch_rows, full.r_num - b0);
                char *sb = static_cast<char *>(g->stage_buf) + (size_t)(pp & 1) * batch_rows * ldst * esz;
                pp++;
                GatherSeg s;
                std::memset(&s, 0, sizeof s);
                s.idx = full.r_col + b0;
                s.n = nb;
                COLA_TRY(launch_gather(nullptr, s, 1, nb, X, ldx, sb, ldst, K, xdt, st));
                PartDesc d = full;
                d.l_num = 0;
                d.r_begin = b0;
                d.r_num = nb;
                d.item0 = 0;
                d.r_mode = dev::kRemoteStagedChunk;
                d.stage = sb;
                d.ld_stage = ldst;
                FusedArgs a{nullptr, d, 1, nb, X, ldx, acc, ldacc, K, xdt,
                            vec_ok(xdt, X, ldx, sb, ldst, acc, ldacc, K)};
                COLA_TRY(launch_fused(a, st));
            }
        }
    } else {  // PIPELINE
        const int64_t ld = ldx;
        const size_t per_pe = (size_t)g->npp * ld * esz;
        COLA_TRY(ensure(g->ppl_buf, g->ppl_bytes, 2 * (size_t)P * per_pe));
        // stage 0: local + intra-group remote of every PE (.cuh:797-805)
        {
            FusedArgs a{g->d_stage0, part_desc_zero(), P, g->stage0_total, X, ldx, acc, ldacc, K, xdt,
                        vec_ok(xdt, X, ldx, nullptr, 0, acc, ldacc, K)};
            COLA_TRY(launch_fused(a, st));
        }
        for (int32_t s = 1; s < g->nstages; s++) {
            char *buf = static_cast<char *>(g->ppl_buf) + (size_t)((s - 1) % 2) * P * per_pe;
            // every PE's put for stage s (batching_data_ppl + put_nbi, .cuh:788-793/811-816)
            COLA_TRY(launch_gather(g->d_put[(size_t)s - 1], GatherSeg{}, P, g->put_total[(size_t)s - 1], X, ldx,
                                   buf, ld, K, xdt, st));
            // stage s compute of every PE (.cuh:822-835)
            // each PE reads its own copy of the buffer (PE p's copy at p * npp rows)
            std::vector<PartDesc> &hs = g->h_stage[(size_t)s - 1];
            bool stage_ok = true;
            for (int32_t p = 0; p < P; p++) {
                const PartDesc &d = hs[(size_t)p];
                if (d.stage != buf + (size_t)p * per_pe || d.ld_stage != ld || d.pe_stride != (int64_t)g->npp * ld) {
                    stage_ok = false;
                    break;
                }
            }
            if (!stage_ok) {
                for (int32_t p = 0; p < P; p++) {
                    PartDesc &d = hs[(size_t)p];
                    d.stage = buf + (size_t)p * per_pe;
                    d.ld_stage = ld;
                    d.pe_stride = (int64_t)g->npp * ld;
                }
                COLA_CUDA(cudaMemcpyAsync(g->d_stage[(size_t)s - 1], hs.data(), hs.size() * sizeof(PartDesc),
                                          cudaMemcpyHostToDevice, st));
                COLA_CUDA(cudaStreamSynchronize(st));
            }
            FusedArgs a{g->d_stage[(size_t)s - 1], part_desc_zero(), P, g->stage_total[(size_t)s - 1], X, ldx, acc,
                        ldacc, K, xdt, vec_ok(xdt, X, ldx, buf, ld, acc, ldacc, K)};
            COLA_TRY(launch_fused(a, st));
        }
    }

    if (ydt == COLA_BFLOAT16) {
        const int64_t n = (int64_t)g->N * K;
        const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
        t_launches++;
        dev::f32_to_bf16_kernel<<<(unsigned)std::max<int64_t>(blocks, 1), dev::kThreads, 0, st>>>(
            acc, ldacc, static_cast<__nv_bfloat16 *>(Y), ldy, g->N, K);
        COLA_CUDA(cudaGetLastError());
    }
    return COLA_SUCCESS;
}

}  // extern "C"

// ===========================================================================
// Buffer-staged launcher that allocates nothing: the remote rows are staged in
// a fixed array compiled into the library instead of a caller buffer.
// ===========================================================================
static __device__ __align__(256) float g_noalloc_stage[COLA_NOALLOC_STAGE_FLOATS];

namespace cola {

// Unique id of the calling thread's current CUDA context (cuCtxGetId, reached
// through the runtime's driver entry points, so the library does not link the
// driver library itself); 0 if it cannot be read.
static unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of g_noalloc_stage on the current device.  In host code the
// array's name only stands in for the symbol, so the address is looked up with
// cudaGetSymbolAddress on the first call on each device, and again whenever
// that device's context is no longer the one the address was taken in (after
// cudaDeviceReset the array lives in a new context, at a new address).
static cola_status noalloc_stage(float **out)
{
    static std::mutex mu;
    static float *addr[64] = {nullptr};
    static unsigned long long ctx_of[64] = {0};
    int dev = 0;
    COLA_CUDA(cudaGetDevice(&dev));
    COLA_REQUIRE(dev >= 0 && dev < 64, COLA_ERROR_UNSUPPORTED, "noalloc staging: device %d out of range", dev);
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev] || ctx == 0 || ctx != ctx_of[dev]) {
        void *p = nullptr;
        COLA_CUDA(cudaGetSymbolAddress(&p, g_noalloc_stage));  // also makes the device's context current
        addr[dev] = static_cast<float *>(p);
        ctx_of[dev] = current_context_id();
    }
    *out = addr[dev];
    return COLA_SUCCESS;
}

}  // namespace cola

extern "C" cola_status cola_ppl0_batch_buffer_spmm_noalloc(
    float *output, const float *input, const int32_t *csr_rowPtr_l, const int32_t *csr_colIdx_l,
    const int32_t *csr_rowIdx_zip_l, const float *csr_val_l, const int32_t *csc_colPtr_r, const int32_t *csc_rowIdx_r,
    const int32_t *csc_colIdx_zip_r, const float *csc_val_r, int32_t local_row_lb, int32_t remote_col_lb,
    int32_t local_row_num, int32_t remote_col_num, int32_t dim, int32_t nodesPerPE, int32_t peid,
    cola_stream_t stream)
{
    (void)local_row_lb;
    COLA_TRY(check_dim(dim, nodesPerPE));
    COLA_REQUIRE(local_row_num >= 0 && remote_col_num >= 0 && remote_col_lb >= 0 && peid >= 0,
                 COLA_ERROR_INVALID_ARGUMENT, "cola_ppl0_batch_buffer_spmm_noalloc: negative count or offset");
    const int64_t need = (int64_t)remote_col_num * dim;
    COLA_REQUIRE(need <= (int64_t)COLA_NOALLOC_STAGE_FLOATS, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_ppl0_batch_buffer_spmm_noalloc: %d remote rows x dim %d need %lld staging floats, the "
                 "library's fixed array holds %u (use cola_ppl0_batch_buffer_spmm with a caller buffer)",
                 remote_col_num, dim, (long long)need, (unsigned)COLA_NOALLOC_STAGE_FLOATS);
    const int64_t T = (int64_t)local_row_num + remote_col_num;
    if (T == 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(output && input, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_ppl0_batch_buffer_spmm_noalloc: null dense pointer");
    float *stage = nullptr;
    COLA_TRY(noalloc_stage(&stage));
    cudaStream_t st = (cudaStream_t)stream;
    if (remote_col_num > 0) {
        // every staged row read below is written here first
        GatherSeg s;
        std::memset(&s, 0, sizeof s);
        s.idx = csc_colIdx_zip_r + remote_col_lb;
        s.n = remote_col_num;
        s.src_row0 = -(int64_t)peid * nodesPerPE;
        s.dst_row0 = 0;
        COLA_TRY(launch_gather(nullptr, s, 1, remote_col_num, input, dim, stage, dim, dim, COLA_FLOAT32, st));
    }
    PartDesc d = part_desc_zero();
    d.l_ptr = csr_rowPtr_l;
    d.l_col = csr_colIdx_l;
    d.l_row = csr_rowIdx_zip_l;
    d.l_val = csr_val_l;
    d.r_ptr = csc_colPtr_r;
    d.r_row = csc_rowIdx_r;
    d.r_col = csc_colIdx_zip_r;
    d.r_val = csc_val_r;
    d.l_num = local_row_num;
    d.r_begin = remote_col_lb;
    d.r_num = remote_col_num;
    d.r_mode = dev::kRemoteStagedChunk;
    d.stage = stage;
    d.ld_stage = dim;
    FusedArgs a{nullptr, d, 1, T, input, dim, output, dim, dim, COLA_FLOAT32,
                vec_ok(COLA_FLOAT32, input, dim, stage, dim, output, dim, dim)};
    return launch_fused(a, st);
}
