// Row-major ("one writer per output row") schedule of the partitioned SpMM.
//
// At upload every partition's remote CSC block is transposed and merged with
// its local CSR, giving for each output row its entries in column order.  One
// warp owns one row: it gathers the rows of X its entries name (16-byte
// vectors, UNROLL loads in flight per lane group), accumulates in FP32
// registers and writes the output row once with plain stores — no atomics, no
// zeroing pass, the same summation order on every run, and BF16 output is
// rounded straight from the registers.  Rows longer than a threshold ("hubs")
// are cut into fixed-length segments processed by separate warps into an FP32
// workspace; a second kernel adds each hub's segment partials pairwise (a
// binary tree in fixed order) and writes the row.
#pragma once
#include "spmm_kernels.cuh"

namespace cola {
namespace dev {

// Store E accumulated values to Y (FP32 or BF16), optionally adding the old
// contents (single writer, so a plain read-modify-write).
template <typename TY, int E, bool VEC_Y>
__device__ __forceinline__ void store_out(TY *p, const float (&a)[E], bool accumulate);

template <>
__device__ __forceinline__ void store_out<float, 4, true>(float *p, const float (&a)[4], bool accumulate)
{
    float4 v = make_float4(a[0], a[1], a[2], a[3]);
    if (accumulate) {
        const float4 o = *reinterpret_cast<const float4 *>(p);
        v.x += o.x;
        v.y += o.y;
        v.z += o.z;
        v.w += o.w;
    }
    __stcs(reinterpret_cast<float4 *>(p), v);  // Y is written once: evict-first in L2, X rows stay
}

template <>
__device__ __forceinline__ void store_out<float, 8, true>(float *p, const float (&a)[8], bool accumulate)
{
    const float lo[4] = {a[0], a[1], a[2], a[3]};
    const float hi[4] = {a[4], a[5], a[6], a[7]};
    store_out<float, 4, true>(p, lo, accumulate);
    store_out<float, 4, true>(p + 4, hi, accumulate);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // RNE; .x = a (low half)
    return *reinterpret_cast<uint32_t *>(&h);
}

template <>
__device__ __forceinline__ void store_out<__nv_bfloat16, 8, true>(__nv_bfloat16 *p, const float (&a)[8], bool)
{
    __stcs(reinterpret_cast<uint4 *>(p),
           make_uint4(pack_bf16x2(a[0], a[1]), pack_bf16x2(a[2], a[3]), pack_bf16x2(a[4], a[5]), pack_bf16x2(a[6], a[7])));
}

template <>
__device__ __forceinline__ void store_out<__nv_bfloat16, 4, true>(__nv_bfloat16 *p, const float (&a)[4], bool)
{
    *reinterpret_cast<uint2 *>(p) = make_uint2(pack_bf16x2(a[0], a[1]), pack_bf16x2(a[2], a[3]));
}

template <>
__device__ __forceinline__ void store_out<float, 2, true>(float *p, const float (&a)[2], bool accumulate)
{
    float2 v = make_float2(a[0], a[1]);
    if (accumulate) {
        const float2 o = *reinterpret_cast<const float2 *>(p);
        v.x += o.x;
        v.y += o.y;
    }
    __stcs(reinterpret_cast<float2 *>(p), v);
}

template <>
__device__ __forceinline__ void store_out<__nv_bfloat16, 2, true>(__nv_bfloat16 *p, const float (&a)[2], bool)
{
    *reinterpret_cast<uint32_t *>(p) = pack_bf16x2(a[0], a[1]);
}

template <>
__device__ __forceinline__ void store_out<float, 1, false>(float *p, const float (&a)[1], bool accumulate)
{
    *p = accumulate ? *p + a[0] : a[0];
}

template <>
__device__ __forceinline__ void store_out<__nv_bfloat16, 1, false>(__nv_bfloat16 *p, const float (&a)[1], bool)
{
    *p = __float2bfloat16_rn(a[0]);
}

// Hub segment table: segment s covers entries [beg[s], min(beg[s]+seg_len,
// rowptr[row[s]+1])) and writes its partial to ws row s.
struct RowsArgs {
    const int64_t *rowptr;  // N+1
    const int32_t *col;     // global column ids
    const float *val;
    int32_t nrows;
    int32_t hub_threshold;  // rows with more entries are handled by segments
    const int32_t *seg_row;
    const int64_t *seg_beg;
    int64_t nseg;
    int32_t seg_len;
    float *ws;              // nseg x K FP32 partials
    int64_t ld_ws;
};

template <typename TR, typename TY, int LG, int NV, int UNROLL, bool VEC_Y>
__global__ void __launch_bounds__(kThreads) rows_spmm_kernel(const __grid_constant__ RowsArgs ra,
                                                             const typename ElemOf<TR>::T *__restrict__ X,
                                                             int64_t ldx, TY *__restrict__ Y, int64_t ldy, int K,
                                                             int accumulate)
{
    using T = typename ElemOf<TR>::T;
    using raw_t = typename TR::raw_t;
    constexpr int E = TR::E;
    constexpr int G = 32 / LG;
    constexpr int W = LG * NV * E;
    const int lane = threadIdx.x & 31;
    const int g = lane / LG;
    const int gl = lane % LG;
    const int k0 = blockIdx.y * W;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int64_t total = ra.nseg + ra.nrows;
    bool kok[NV];
#pragma unroll
    for (int j = 0; j < NV; j++)
        kok[j] = (k0 + (gl + j * LG) * E) < K;
    const T *xk = X + k0;

    for (int64_t it = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); it < total; it += nwarps) {
        int64_t b, e;
        bool to_ws;
        int64_t out_row;
        if (it < ra.nseg) {
            const int32_t r = __ldg(ra.seg_row + it);
            b = __ldg(ra.seg_beg + it);
            e = min(b + (int64_t)ra.seg_len, __ldg(ra.rowptr + r + 1));
            to_ws = true;
            out_row = it;
        } else {
            const int64_t r = it - ra.nseg;
            b = __ldg(ra.rowptr + r);
            e = __ldg(ra.rowptr + r + 1);
            if (e - b > ra.hub_threshold)
                continue;  // written by the hub combine
            to_ws = false;
            out_row = r;
        }
        float acc[NV][E];
#pragma unroll
        for (int j = 0; j < NV; j++)
#pragma unroll
            for (int q = 0; q < E; q++)
                acc[j][q] = 0.f;
        for (int64_t base = b; base < e; base += 32) {
            const int n = (int)min((int64_t)32, e - base);
            int mc = 0;
            float mv = 0.f;
            if (lane < n) {
                mc = __ldg(ra.col + base + lane);
                mv = __ldg(ra.val + base + lane);
            }
            for (int jj = 0; jj < n; jj += G * UNROLL) {
                raw_t xr[UNROLL][NV];
                float vv[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; u++) {
                    const int k = jj + u * G + g;
                    const int cc = __shfl_sync(kFull, mc, k & 31);
                    const float v = __shfl_sync(kFull, mv, k & 31);
                    const bool ok = k < n;
                    vv[u] = ok ? v : 0.f;
                    const T *xp = xk + (int64_t)cc * ldx;
#pragma unroll
                    for (int j = 0; j < NV; j++)
                        xr[u][j] = (ok && kok[j]) ? TR::load(xp + (gl + j * LG) * E) : TR::zero();
                }
#pragma unroll
                for (int u = 0; u < UNROLL; u++)
#pragma unroll
                    for (int j = 0; j < NV; j++) {
                        float f[E];
                        TR::unpack(xr[u][j], f);
#pragma unroll
                        for (int q = 0; q < E; q++)
                            acc[j][q] = fmaf(vv[u], f[q], acc[j][q]);
                    }
            }
        }
#pragma unroll
        for (int off = LG; off < 32; off <<= 1)
#pragma unroll
            for (int j = 0; j < NV; j++)
#pragma unroll
                for (int q = 0; q < E; q++)
                    acc[j][q] += __shfl_xor_sync(kFull, acc[j][q], off);
        if (g == 0) {
            if (to_ws) {
                float *wp = ra.ws + out_row * ra.ld_ws + k0;
#pragma unroll
                for (int j = 0; j < NV; j++)
                    if (kok[j]) {
                        float *p = wp + (gl + j * LG) * E;
#pragma unroll
                        for (int q = 0; q < E; q++)
                            p[q] = acc[j][q];
                    }
            } else {
                TY *yp = Y + out_row * ldy + k0;
#pragma unroll
                for (int j = 0; j < NV; j++)
                    if (kok[j])
                        store_out<TY, E, VEC_Y>(yp + (gl + j * LG) * E, acc[j], accumulate != 0);
            }
        }
    }
}

// Row-block streaming form of the same schedule, for rows one warp wide
// (LG = 32).  A task is a contiguous block of rows holding about the same
// number of entries as every other task (hub rows excluded: they come as
// segments).  The warp streams the block's entries as one flat list -- index
// batch b+1 is loaded while batch b is consumed, UNROLL rows of X are in flight
// -- and flushes the running sums to the output row whenever the stream
// crosses a row end, writing empty rows as zeros.  Loads therefore keep flowing
// across row boundaries instead of restarting a dependent chain per row.
struct BlockArgs {
    const int64_t *rowptr;
    const int32_t *col;
    const float *val;
    const int32_t *task_rb, *task_re;  // task t: rows [task_rb[t], task_re[t])
    int64_t ntask;
    const int32_t *seg_row;
    const int64_t *seg_beg;
    int64_t nseg;
    int32_t seg_len;
    float *ws;
    int64_t ld_ws;
    // Work-item counters for the dynamic schedule (kMaxItemQueues per-tile
    // counters, then the count of warps that have finished); all zero between
    // launches: the last warp of a launch resets them.  NULL: static
    // grid-stride assignment.
    unsigned int *queue;
};

// acc[q] += v * x[2q .. 2q+1] for one 16-byte vector of X, with the packed
// FP32x2 fused multiply-add of sm_100 (two products per instruction).
template <typename TR>
__device__ __forceinline__ void fma_vec2(float2 (&acc)[TR::E / 2], float v, const typename TR::raw_t &r)
{
    float f[TR::E];
    TR::unpack(r, f);
    const float2 vv = make_float2(v, v);
#pragma unroll
    for (int q = 0; q < TR::E / 2; q++)
        acc[q] = __ffma2_rn(vv, make_float2(f[2 * q], f[2 * q + 1]), acc[q]);
}

// LG lanes cover one row tile of X (NV vectors each); G = 32 / LG lane groups
// of the warp take interleaved entries of the same stream (group g takes
// entries g, g + G, ...), so narrow rows still keep 32 lanes busy.  A round is
// G * UNROLL consecutive entries: when it lies inside the current output row
// every group just accumulates; otherwise it is cut at the row ends, and at
// every row end the groups' partial sums are added with __shfl_xor_sync and
// group 0 writes the row.
// Work items it0, it0 + stride, ... (< total) of the streaming schedule, each a
// row-block task (rows [task_rb, task_re) of ba) or a hub segment (its partial
// goes to ws row `it`); items count segments first, then tasks.  k0 is the
// first feature of this call's tile; ent is the warp's 32-entry shared-memory
// index batch.
// LG > 0 fixes the lane-group width at compile time; LG == 0 takes it from
// lg_rt at run time (8, 16 or 32), as the batched form does per graph.
// BARef is `const BlockArgs` (the single-graph kernel: arguments read straight
// from the kernel's parameter space) or `const BlockArgs &` (the batched form:
// a descriptor in global memory).
template <typename TR, typename TY, int LG, int NV, int UNROLL, bool VEC_Y, typename BARef = const BlockArgs,
          bool DYN = false>
__device__ __forceinline__ void rowblock_items(BARef ba, const int64_t it0, const int64_t stride,
                                               const int64_t total,
                                              const typename ElemOf<TR>::T *__restrict__ X, const int64_t ldx,
                                              TY *__restrict__ Y, const int64_t ldy, const int K, const int accumulate,
                                              const int k0, int2 *ent, const int lg_rt = 0,
                                              unsigned int *queue = nullptr)
{
    using T = typename ElemOf<TR>::T;
    using raw_t = typename TR::raw_t;
    constexpr int E = TR::E;
    static_assert(LG == 0 || (32 / (LG > 0 ? LG : 1)) * UNROLL <= 32, "a round must fit in the 32-entry index batch");
    const int lg = LG > 0 ? LG : lg_rt;
    const int G = 32 / lg;
    const int R = G * UNROLL;  // entries per round
    const int lane = threadIdx.x & 31;
    const int g = lane / lg;
    const int gl = lane % lg;
    bool kok[NV];
#pragma unroll
    for (int j = 0; j < NV; j++)
        kok[j] = (k0 + (gl + j * lg) * E) < K;
    const T *xk = X + k0 + gl * E;
    const int32_t ldx32 = (int32_t)ldx;  // the vector path's row stride fits 32 bits (one multiply-add per entry)

    // DYN: items are drawn from a counter (lane 0, one item ahead, so the
    // atomic's latency hides behind the current item); a warp that drew a
    // slow item simply draws fewer.  Otherwise: it0, it0 + stride, ...
    // Item numbers fit 32 bits (the launchers check nseg + ntask < 2^31): one
    // register each, which keeps the 4-blocks-per-SM build within its 64.
    const int32_t total32 = (int32_t)total;
    int32_t it = (int32_t)it0;
    if constexpr (DYN) {
        unsigned int t = 0;
        if (lane == 0)
            t = atomicAdd(queue, 1u);
        it = (int32_t)__shfl_sync(kFull, t, 0);
    }
    while (it < total32) {
        unsigned int next_it = 0;
        if constexpr (DYN) {
            if (lane == 0)
                next_it = atomicAdd(queue, 1u);
        }
        const bool seg = it < ba.nseg;
        int32_t rb, re;
        int64_t e_beg;
        int32_t n_ent;  // entries of this item; indices below are relative to e_beg
        if (seg) {
            rb = __ldg(ba.seg_row + it);
            re = rb + 1;
            e_beg = __ldg(ba.seg_beg + it);
            n_ent = (int32_t)min((int64_t)ba.seg_len, __ldg(ba.rowptr + rb + 1) - e_beg);
        } else {
            const int64_t t = it - ba.nseg;
            rb = __ldg(ba.task_rb + t);
            re = __ldg(ba.task_re + t);
            e_beg = __ldg(ba.rowptr + rb);
            n_ent = (int32_t)(__ldg(ba.rowptr + re) - e_beg);
        }
        const int32_t *colp = ba.col + e_beg;
        const float *valp = ba.val + e_beg;
        // ends of rows q0 .. q0+31, relative to e_beg (lane l: row q0 + l)
        int32_t q0 = rb;
        int32_t my_end = seg ? n_ent : (rb + lane < re ? (int32_t)(__ldg(ba.rowptr + rb + lane + 1) - e_beg) : n_ent);
        int32_t cur = rb;
        int32_t row_end = __shfl_sync(kFull, my_end, 0);

        float2 acc[NV][E / 2];
    #pragma unroll
        for (int j = 0; j < NV; j++)
    #pragma unroll
            for (int q = 0; q < E / 2; q++)
                acc[j][q] = make_float2(0.f, 0.f);

        auto flush = [&]() {
    #pragma unroll
            for (int off = lg; off < 32; off <<= 1)
    #pragma unroll
                for (int j = 0; j < NV; j++)
    #pragma unroll
                    for (int q = 0; q < E / 2; q++) {
                        acc[j][q].x += __shfl_xor_sync(kFull, acc[j][q].x, off);
                        acc[j][q].y += __shfl_xor_sync(kFull, acc[j][q].y, off);
                    }
            if (g == 0) {
                if (seg) {
                    // the segment's FP32 partial, read once by the combine kernel
                    float *wp = ba.ws + (int64_t)it * ba.ld_ws + k0 + gl * E;
    #pragma unroll
                    for (int j = 0; j < NV; j++)
                        if (kok[j]) {
                            float a[E];
    #pragma unroll
                            for (int q = 0; q < E / 2; q++) {
                                a[2 * q] = acc[j][q].x;
                                a[2 * q + 1] = acc[j][q].y;
                            }
                            store_out<float, E, true>(wp + j * lg * E, a, false);
                        }
                } else {
                    TY *yp = Y + (int64_t)cur * ldy + k0 + gl * E;
    #pragma unroll
                    for (int j = 0; j < NV; j++)
                        if (kok[j]) {
                            float a[E];
    #pragma unroll
                            for (int q = 0; q < E / 2; q++) {
                                a[2 * q] = acc[j][q].x;
                                a[2 * q + 1] = acc[j][q].y;
                            }
                            store_out<TY, E, VEC_Y>(yp + j * lg * E, a, accumulate != 0);
                        }
                }
            }
    #pragma unroll
            for (int j = 0; j < NV; j++)
    #pragma unroll
                for (int q = 0; q < E / 2; q++)
                    acc[j][q] = make_float2(0.f, 0.f);
            cur++;
            if (!seg && cur < re) {
                if (cur - q0 >= 32) {
                    q0 += 32;
                    my_end = q0 + lane < re ? (int32_t)(__ldg(ba.rowptr + q0 + lane + 1) - e_beg) : n_ent;
                }
                row_end = __shfl_sync(kFull, my_end, cur - q0);
            }
        };

        int mc = 0;
        float mv = 0.f;
        if (lane < n_ent) {
            // the entry stream is read once: evict-first, so it does not push X rows out of L2
            mc = __ldcs(colp + lane);
            mv = __ldcs(valp + lane);
        }
        for (int32_t base = 0; base < n_ent; base += 32) {
            const int n = min(32, n_ent - base);
            __syncwarp();
            ent[lane] = make_int2(mc, __float_as_int(mv));
            __syncwarp();
            // prefetch the next index batch while this one is consumed
            if (base + 32 + lane < n_ent) {
                mc = __ldcs(colp + base + 32 + lane);
                mv = __ldcs(valp + base + 32 + lane);
            }
            for (int jj = 0; jj < n; jj += R) {
                // the values are read from shared memory when the rows have
                // arrived, not held in registers while the loads are in flight
                raw_t xr[UNROLL][NV];
                if (jj + R <= n && base + jj + R <= row_end) {
                    // the whole round inside the current row: no boundary checks
    #pragma unroll
                    for (int u = 0; u < UNROLL; u++) {
                        const T *xp = xk + (int64_t)ent[jj + u * G + g].x * ldx32;
    #pragma unroll
                        for (int j = 0; j < NV; j++)
                            if (kok[j])
                                xr[u][j] = TR::load(xp + j * lg * E);
                    }
    #pragma unroll
                    for (int u = 0; u < UNROLL; u++) {
                        const float v = __int_as_float(ent[jj + u * G + g].y);
    #pragma unroll
                        for (int j = 0; j < NV; j++)
                            fma_vec2<TR>(acc[j], v, xr[u][j]);
                    }
                } else {
    #pragma unroll
                    for (int u = 0; u < UNROLL; u++) {
                        const int idx = jj + u * G + g;
                        if (idx < n) {
                            const T *xp = xk + (int64_t)ent[idx].x * ldx32;
    #pragma unroll
                            for (int j = 0; j < NV; j++)
                                if (kok[j])
                                    xr[u][j] = TR::load(xp + j * lg * E);
                        }
                    }
                    // cut the round [lo, hi) at the row ends it contains
                    int32_t lo = base + jj;
                    const int32_t hi = base + jj + min(R, n - jj);
                    while (true) {
                        while (lo >= row_end)
                            flush();
                        const int32_t sh = min(row_end, hi);
    #pragma unroll
                        for (int u = 0; u < UNROLL; u++) {
                            const int32_t e = base + jj + u * G + g;
                            if (e >= lo && e < sh) {
                                const float v = __int_as_float(ent[jj + u * G + g].y);
    #pragma unroll
                                for (int j = 0; j < NV; j++)
                                    fma_vec2<TR>(acc[j], v, xr[u][j]);
                            }
                        }
                        lo = sh;
                        if (lo >= hi)
                            break;
                    }
                }
            }
        }
        while (cur < re)
            flush();
        if constexpr (DYN)
            it = (int32_t)__shfl_sync(kFull, next_it, 0);
        else
            it += (int32_t)stride;
    }
}

// End of a launch with the dynamic schedule: the last warp to finish puts the
// item counters back to zero for the next launch (every warp has drawn its
// final item before it counts itself finished).
__device__ __forceinline__ void item_queue_release(unsigned int *queue)
{
    if ((threadIdx.x & 31) == 0) {
        const unsigned int warps = gridDim.x * gridDim.y * kWarpsPerBlock;
        if (atomicAdd(queue + kMaxItemQueues, 1u) == warps - 1) {
            for (unsigned t = 0; t < gridDim.y; t++)
                atomicExch(queue + t, 0u);
            atomicExch(queue + kMaxItemQueues, 0u);
        }
    }
}

template <typename TR, typename TY, int LG, int NV, int UNROLL, bool VEC_Y, int MINB = 1, bool DYN = false>
__global__ void __launch_bounds__(kThreads, MINB) rowblock_spmm_kernel(const __grid_constant__ BlockArgs ba,
                                                                       const typename ElemOf<TR>::T *__restrict__ X,
                                                                       int64_t ldx, TY *__restrict__ Y, int64_t ldy,
                                                                       int K, int accumulate)
{
    // the current batch of 32 (col, val) pairs of each warp, read back with
    // one 8-byte shared-memory load per entry and lane group
    __shared__ int2 s_ent[kWarpsPerBlock][32];
    int2 *ent = s_ent[threadIdx.x >> 5];
    constexpr int W = LG * NV * TR::E;
    const int k0 = blockIdx.y * W;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int64_t total = ba.nseg + ba.ntask;
    rowblock_items<TR, TY, LG, NV, UNROLL, VEC_Y, const BlockArgs, DYN>(
        ba, (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5), nwarps, total, X, ldx, Y, ldy, K, accumulate,
        k0, ent, 0, DYN ? ba.queue + blockIdx.y : nullptr);
    if constexpr (DYN)
        item_queue_release(ba.queue);
}

// The same schedule with the feature tiles one after another instead of side
// by side (blockIdx.y): the grid sweeps every item of tile 0, then of tile 1,
// ..., so the X columns being gathered at any moment are one tile wide.  Every
// element's sum is the same chain of FMAs whichever tile width computes it
// (one lane group per row: LG = 32).  A separate kernel, so that the default
// one keeps its own register allocation.
template <typename TR, typename TY, int NV, int UNROLL, int MINB = 1>
__global__ void __launch_bounds__(kThreads, MINB) rowblock_tiled_kernel(const __grid_constant__ BlockArgs ba,
                                                                        const typename ElemOf<TR>::T *__restrict__ X,
                                                                        int64_t ldx, TY *__restrict__ Y, int64_t ldy,
                                                                        int K, int accumulate)
{
    __shared__ int2 s_ent[kWarpsPerBlock][32];
    int2 *ent = s_ent[threadIdx.x >> 5];
    constexpr int W = 32 * NV * TR::E;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int64_t total = ba.nseg + ba.ntask;
    const int ntile = (K + W - 1) / W;
    for (int64_t w = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); w < total * ntile; w += nwarps) {
        const int tile = (int)(w / total);
        const int64_t it = w - (int64_t)tile * total;
        rowblock_items<TR, TY, 32, NV, UNROLL, true>(ba, it, 1, it + 1, X, ldx, Y, ldy, K, accumulate, tile * W,
                                                     ent);
    }
}

// Hub rows: sum the segment partials ws[s0 .. s1) pairwise — a binary tree in
// fixed order, computed in place in the workspace by the owning lane — and
// write the row.  One warp per hub row; lane l owns features l, l+32, ...
template <typename TY>
__global__ void __launch_bounds__(kThreads) hub_combine_kernel(const int32_t *__restrict__ hub_row,
                                                              const int64_t *__restrict__ hub_seg, int64_t nhub,
                                                              float *__restrict__ ws, int64_t ld_ws, TY *__restrict__ Y,
                                                              int64_t ldy, int K, int accumulate)
{
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    for (int64_t h = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); h < nhub; h += nwarps) {
        const int64_t s0 = hub_seg[h], m = hub_seg[h + 1] - s0;
        float *w0 = ws + s0 * ld_ws;
        for (int64_t stride = 1; stride < m; stride <<= 1)
            for (int64_t i = 0; i + stride < m; i += 2 * stride) {
                float *a = w0 + i * ld_ws;
                const float *c = w0 + (i + stride) * ld_ws;
                for (int k = lane; k < K; k += 32)
                    a[k] += c[k];
            }
        TY *yp = Y + (int64_t)hub_row[h] * ldy;
        for (int k = lane; k < K; k += 32) {
            const float v = w0[k];
            if constexpr (sizeof(TY) == 4)
                yp[k] = accumulate ? (float)yp[k] + v : v;
            else
                yp[k] = __float2bfloat16_rn(v);
        }
    }
}

// Hub rows, 16-byte vector form (K a multiple of 4, ws rows 16-byte aligned):
// one warp per (hub, 128-feature tile); every partial is read exactly once,
// UNROLL partials in flight, and summed pairwise by a binary counter: partial
// i is added to the running block sums of sizes 1, 2, 4, ... that its index's
// trailing one bits close, so the sum is the same fixed binary tree for every
// run.  The stack has one slot per tree level (at most 32).
// One (hub, 128-feature tile) of the combine: partials ws[hub_seg[h] ..
// hub_seg[h+1]) summed pairwise and written to output row hub_row[h].
template <typename TY, int UNROLL>
__device__ __forceinline__ void hub_combine_item(const int32_t *__restrict__ hub_row,
                                                 const int64_t *__restrict__ hub_seg, const int64_t h, const int tile,
                                                 const float *__restrict__ ws, const int64_t ld_ws, TY *__restrict__ Y,
                                                 const int64_t ldy, const int K, const int accumulate)
{
    const int lane = threadIdx.x & 31;
    const int k = tile * 128 + lane * 4;
    const bool kok = k < K;
    const int64_t s0 = __ldg(hub_seg + h), m = __ldg(hub_seg + h + 1) - s0;
    const float *wp = ws + s0 * ld_ws + k;
    float4 stk[32];
    for (int64_t i0 = 0; i0 < m; i0 += UNROLL) {
        float4 v[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; u++)
            if (kok && i0 + u < m)
                v[u] = __ldcg(reinterpret_cast<const float4 *>(wp + (i0 + u) * ld_ws));
#pragma unroll
        for (int u = 0; u < UNROLL; u++) {
            const int64_t i = i0 + u;
            if (i < m) {
                float4 c = v[u];
                int l = 0;
                while ((i >> l) & 1) {
                    const float4 a = stk[l];
                    c = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w + c.w);
                    l++;
                }
                stk[l] = c;
            }
        }
    }
    // fold the open block sums, larger (earlier) blocks first
    float4 tot = make_float4(0.f, 0.f, 0.f, 0.f);
    bool first = true;
    for (int l = 31; l >= 0; l--)
        if ((m >> l) & 1) {
            const float4 a = stk[l];
            tot = first ? a : make_float4(tot.x + a.x, tot.y + a.y, tot.z + a.z, tot.w + a.w);
            first = false;
        }
    if (kok) {
        const float r[4] = {tot.x, tot.y, tot.z, tot.w};
        store_out<TY, 4, true>(Y + (int64_t)__ldg(hub_row + h) * ldy + k, r, accumulate != 0);
    }
}

// Hub rows, 16-byte vector form (K a multiple of 4, ws rows 16-byte aligned):
// one warp per (hub, 128-feature tile); every partial is read exactly once,
// UNROLL partials in flight, and summed pairwise by a binary counter: partial
// i is added to the running block sums of sizes 1, 2, 4, ... that its index's
// trailing one bits close, so the sum is the same fixed binary tree for every
// run.  The stack has one slot per tree level (at most 32).
template <typename TY, int UNROLL>
__global__ void __launch_bounds__(kThreads) hub_combine_vec_kernel(const int32_t *__restrict__ hub_row,
                                                                  const int64_t *__restrict__ hub_seg, int64_t nhub,
                                                                  const float *__restrict__ ws, int64_t ld_ws,
                                                                  TY *__restrict__ Y, int64_t ldy, int K,
                                                                  int accumulate)
{
    const int tiles = (K + 127) / 128;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    for (int64_t w = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); w < nhub * tiles; w += nwarps)
        hub_combine_item<TY, UNROLL>(hub_row, hub_seg, w / tiles, (int)(w % tiles), ws, ld_ws, Y, ldy, K, accumulate);
}

}  // namespace dev
}  // namespace cola
