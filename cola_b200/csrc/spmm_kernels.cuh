// Device code of the partitioned SpMM (sm_100a).
//
// One warp owns one work item: a local CSR chunk (gather-FMA over its
// entries, include/dist_spmm_ppl_batch.cuh:164-197) or a remote CSC chunk
// (one staged dense row scattered to every row of the chunk, :112-160).
// Feature rows move as 16-byte vectors: a lane owns NV vectors of E elements
// (E = 4 FP32 or 8 BF16), LG lanes cover one row tile and G = 32/LG groups of a
// warp work on different entries of the same chunk at once (narrow K), their
// partial sums combined with warp shuffles before the single write.
// Accumulation is FP32 in registers; writes into Y are 16-byte vector
// reductions (red.global.add.v4.f32 via atomicAdd(float4*)).
#pragma once
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cola {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarpsPerBlock = 8;
constexpr int kThreads = kWarpsPerBlock * 32;
// Row-major schedule: feature tiles (gridDim.y) that can draw work items from
// counters of their own; a graph holds kMaxItemQueues + 1 counters.
constexpr int kMaxItemQueues = 64;

// Where a remote chunk's dense row comes from.
enum RemoteMode : int32_t {
    kRemoteFromX = 0,       // X[x_remote0 + global col]           (on-chip staging)
    kRemoteStagedChunk = 1, // stage[c - r_begin]                  (HBM staging buffer)
    kRemoteStageBuffer = 2  // pipeline buffer row idx_ppl[w] of this PE or a group peer
};

// One virtual partition's slice of a launch.
struct PartDesc {
    const int32_t *l_ptr, *l_col, *l_row;
    const float *l_val;
    const int32_t *r_ptr, *r_row, *r_col;
    const float *r_val;
    int32_t l_begin, l_num, r_begin, r_num;
    int64_t x_local0;   // X row holding local column 0
    int64_t x_remote0;  // X row holding global column 0
    int64_t y_row0;     // Y row holding partition row 0
    int64_t item0;      // first launch item of this partition (prefix over parts)
    int32_t r_mode;
    int32_t npp, gs, group_offset, peid, local_col_lb, local_col_ub, pad_;
    const void *stage;  // staged rows (modes 1, 2)
    int64_t ld_stage;   // elements between staged rows
    int64_t pe_stride;  // elements between PEs' copies of the stage buffer (mode 2)
    const int32_t *idx_ppl;
};

template <typename T>
struct VecTraits;

template <>
struct VecTraits<float> {
    static constexpr int E = 4;
    using raw_t = float4;
    __device__ __forceinline__ static raw_t load(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
    __device__ __forceinline__ static raw_t zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ __forceinline__ static void unpack(const raw_t &r, float (&f)[E])
    {
        f[0] = r.x;
        f[1] = r.y;
        f[2] = r.z;
        f[3] = r.w;
    }
};

template <>
struct VecTraits<__nv_bfloat16> {
    static constexpr int E = 8;
    using raw_t = uint4;
    __device__ __forceinline__ static raw_t load(const __nv_bfloat16 *p)
    {
        return __ldg(reinterpret_cast<const uint4 *>(p));
    }
    __device__ __forceinline__ static raw_t zero() { return make_uint4(0u, 0u, 0u, 0u); }
    // BF16 -> FP32 is exact: the 16 bits become the high half of the float.
    __device__ __forceinline__ static void unpack(const raw_t &r, float (&f)[E])
    {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            f[2 * i] = __uint_as_float(w[i] << 16);
            f[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
        }
    }
};

// Narrower vectors (BYTES = 8 or 4 per lane) for feature tiles a full warp
// reads 256 or 128 bytes of: the row-major schedule's narrow passes.
template <typename T, int BYTES>
struct NarrowTraits;

template <>
struct NarrowTraits<float, 8> {
    static constexpr int E = 2;
    using raw_t = float2;
    __device__ __forceinline__ static raw_t load(const float *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }
    __device__ __forceinline__ static raw_t zero() { return make_float2(0.f, 0.f); }
    __device__ __forceinline__ static void unpack(const raw_t &r, float (&f)[E])
    {
        f[0] = r.x;
        f[1] = r.y;
    }
};

template <>
struct NarrowTraits<__nv_bfloat16, 8> {
    static constexpr int E = 4;
    using raw_t = uint2;
    __device__ __forceinline__ static raw_t load(const __nv_bfloat16 *p)
    {
        return __ldg(reinterpret_cast<const uint2 *>(p));
    }
    __device__ __forceinline__ static raw_t zero() { return make_uint2(0u, 0u); }
    __device__ __forceinline__ static void unpack(const raw_t &r, float (&f)[E])
    {
        f[0] = __uint_as_float(r.x << 16);
        f[1] = __uint_as_float(r.x & 0xffff0000u);
        f[2] = __uint_as_float(r.y << 16);
        f[3] = __uint_as_float(r.y & 0xffff0000u);
    }
};

template <>
struct NarrowTraits<__nv_bfloat16, 4> {
    static constexpr int E = 2;
    using raw_t = uint32_t;
    __device__ __forceinline__ static raw_t load(const __nv_bfloat16 *p)
    {
        return __ldg(reinterpret_cast<const unsigned int *>(p));
    }
    __device__ __forceinline__ static raw_t zero() { return 0u; }
    __device__ __forceinline__ static void unpack(const raw_t &r, float (&f)[E])
    {
        f[0] = __uint_as_float(r << 16);
        f[1] = __uint_as_float(r & 0xffff0000u);
    }
};

// Scalar fallback (rows not 16-byte aligned or K not a multiple of E).
template <typename T>
struct ScalarTraits {
    static constexpr int E = 1;
    using raw_t = T;
    __device__ __forceinline__ static raw_t load(const T *p) { return *p; }
    __device__ __forceinline__ static raw_t zero() { return T(0.f); }
    __device__ __forceinline__ static void unpack(const raw_t &r, float (&f)[1]) { f[0] = (float)r; }
};

template <typename TR>
struct ElemOf;
template <>
struct ElemOf<VecTraits<float>> {
    using T = float;
};
template <>
struct ElemOf<VecTraits<__nv_bfloat16>> {
    using T = __nv_bfloat16;
};
template <typename U>
struct ElemOf<ScalarTraits<U>> {
    using T = U;
};
template <typename U, int B>
struct ElemOf<NarrowTraits<U, B>> {
    using T = U;
};

// Y[p..p+E) += a[0..E): 16-byte vector reductions when E is a multiple of 4.
template <int E, bool VEC_Y>
__device__ __forceinline__ void red_add(float *p, const float (&a)[E])
{
    if constexpr (VEC_Y && (E % 4) == 0) {
#pragma unroll
        for (int q = 0; q < E / 4; q++)
            atomicAdd(reinterpret_cast<float4 *>(p + 4 * q), make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]));
    } else {
#pragma unroll
        for (int q = 0; q < E; q++)
            atomicAdd(p + q, a[q]);
    }
}

// Locate the partition of launch item `it`, moving forward from *p.
__device__ __forceinline__ const PartDesc *find_part(const PartDesc *parts, int nparts, int64_t it, int &p)
{
    while (p + 1 < nparts && it >= parts[p + 1].item0)
        p++;
    return parts + p;
}

// The fused partitioned SpMM: items [0, total) over all parts; item i of part
// d is local chunk d.l_begin + i when i < d.l_num, else remote chunk
// d.r_begin + (i - d.l_num).  blockIdx.y selects the feature tile.  MINB is
// the number of blocks per SM the registers must allow.
template <typename TR, int LG, int NV, int UNROLL, bool VEC_Y, int MINB = 1>
__global__ void __launch_bounds__(kThreads, MINB) fused_spmm_kernel(const PartDesc *__restrict__ parts,
                                                              const __grid_constant__ PartDesc single, int nparts,
                                                              int64_t total,
                                                              const typename ElemOf<TR>::T *__restrict__ X,
                                                              int64_t ldx, float *__restrict__ Y, int64_t ldy, int K)
{
    using T = typename ElemOf<TR>::T;
    using raw_t = typename TR::raw_t;
    constexpr int E = TR::E;
    constexpr int G = 32 / LG;
    constexpr int W = LG * NV * E;  // features per tile
    const int lane = threadIdx.x & 31;
    const int g = lane / LG;
    const int gl = lane % LG;
    const int k0 = blockIdx.y * W;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int64_t w0 = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    int pidx = 0;

    // features owned by this lane: k0 + (gl + j*LG)*E + e, j < NV
    bool kok[NV];
#pragma unroll
    for (int j = 0; j < NV; j++)
        kok[j] = (k0 + (gl + j * LG) * E) < K;

    for (int64_t it = w0; it < total; it += nwarps) {
        const PartDesc &d = parts ? *find_part(parts, nparts, it, pidx) : single;
        const int64_t li = it - d.item0;
        if (li < d.l_num) {
            // ---------------- local CSR chunk ----------------
            const int64_t c = d.l_begin + li;
            const int lb = __ldg(d.l_ptr + c), hb = __ldg(d.l_ptr + c + 1);
            const int row = __ldg(d.l_row + c);
            float acc[NV][E];
#pragma unroll
            for (int j = 0; j < NV; j++)
#pragma unroll
                for (int e = 0; e < E; e++)
                    acc[j][e] = 0.f;
            const T *xl = X + d.x_local0 * ldx + k0;
            for (int base = lb; base < hb; base += 32) {
                const int n = min(32, hb - base);
                int mc = 0;
                float mv = 0.f;
                if (lane < n) {
                    mc = __ldg(d.l_col + base + lane);
                    mv = __ldg(d.l_val + base + lane);
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
                        const T *xp = xl + (int64_t)cc * ldx;
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
                            for (int e = 0; e < E; e++)
                                acc[j][e] = fmaf(vv[u], f[e], acc[j][e]);
                        }
                }
            }
#pragma unroll
            for (int off = LG; off < 32; off <<= 1)
#pragma unroll
                for (int j = 0; j < NV; j++)
#pragma unroll
                    for (int e = 0; e < E; e++)
                        acc[j][e] += __shfl_xor_sync(kFull, acc[j][e], off);
            if (g == 0) {
                float *yp = Y + (d.y_row0 + row) * ldy + k0;
#pragma unroll
                for (int j = 0; j < NV; j++)
                    if (kok[j])
                        red_add<E, VEC_Y>(yp + (gl + j * LG) * E, acc[j]);
            }
        } else {
            // ---------------- remote CSC chunk ----------------
            const int64_t w = li - d.l_num;
            const int64_t c = d.r_begin + w;
            const int lb = __ldg(d.r_ptr + c), hb = __ldg(d.r_ptr + c + 1);
            const T *src;
            if (d.r_mode == kRemoteFromX) {
                src = X + (d.x_remote0 + __ldg(d.r_col + c)) * ldx;
            } else if (d.r_mode == kRemoteStagedChunk) {
                src = static_cast<const T *>(d.stage) + w * d.ld_stage;
            } else {
                const int32_t col = __ldg(d.r_col + c);
                const int64_t ix = __ldg(d.idx_ppl + w);
                int64_t peer_off = 0;
                if (!(c >= d.local_col_lb && c < d.local_col_ub)) {
                    const int peer = (col / d.npp) % d.gs + d.group_offset;
                    peer_off = (int64_t)(peer - d.peid) * d.pe_stride;
                }
                src = static_cast<const T *>(d.stage) + peer_off + ix * d.ld_stage;
            }
            src += k0;
            // stage the dense row on chip (registers)
            float xs[NV][E];
#pragma unroll
            for (int j = 0; j < NV; j++) {
                raw_t r = kok[j] ? TR::load(src + (gl + j * LG) * E) : TR::zero();
                TR::unpack(r, xs[j]);
            }
            for (int base = lb; base < hb; base += 32) {
                const int n = min(32, hb - base);
                int mr = 0;
                float mv = 0.f;
                if (lane < n) {
                    mr = __ldg(d.r_row + base + lane);
                    mv = __ldg(d.r_val + base + lane);
                }
                for (int jj = 0; jj < n; jj += G) {
                    const int k = jj + g;
                    const int r = __shfl_sync(kFull, mr, k & 31);
                    const float v = __shfl_sync(kFull, mv, k & 31);
                    if (k < n) {
                        float *yp = Y + (d.y_row0 + r) * ldy + k0;
#pragma unroll
                        for (int j = 0; j < NV; j++)
                            if (kok[j]) {
                                float a[E];
#pragma unroll
                                for (int e = 0; e < E; e++)
                                    a[e] = v * xs[j][e];
                                red_add<E, VEC_Y>(yp + (gl + j * LG) * E, a);
                            }
                    }
                }
            }
        }
    }
}

// A segment of a row gather: dst[dst_row0 + b] = src[src_row0 + idx[b] (% mod)].
struct GatherSeg {
    const int32_t *idx;
    int64_t n;
    int64_t src_row0;
    int64_t dst_row0;
    int64_t item0;
    int32_t mod;  // 0: no modulo
    int32_t pad_;
};

// ---------------------------------------------------------------------------
// Staged row gather through the Tensor Memory Accelerator: each row moves
// global -> shared -> global with bulk asynchronous copies (cp.async.bulk of
// one CTA, no tensor map), so no register touches the row data.  A warp takes
// chunks of `chunk` consecutive rows (at most its ns row slots of the block's
// dynamic shared memory, at most 32; fewer when a launch has few rows, so that
// every warp gets some): the lanes resolve the chunk's source and
// destination rows together (one coalesced index load), then one elected lane
// issues every row's load at once, stores each row as its load lands on the
// slot's mbarrier, and waits for the stores to finish reading before the next
// chunk reuses the slots.  Rows are K elements of 16-byte granularity, every
// address 16-byte aligned (checked by the host).  Every wait is bounded.  A
// row's wait gives up after `wait_limit` polls (a kernel argument); the kernel
// then records error 1 in *err, stops issuing copies and drains every load it
// has issued, each with the separate, much larger kDrainLimit, before the CTA
// exits (its bulk stores are waited for by cp.async.bulk.wait_group, which
// always ends).  Only if a drain wait also runs out is error 2 recorded: a load
// may then still be writing this CTA's shared memory after it exits.
// ---------------------------------------------------------------------------
constexpr int kGatherMaxSlots = 32;
constexpr uint32_t kWaitLimitDefault = 1u << 22;  // polls: at least 0.25 s
constexpr uint32_t kDrainLimit = 1u << 25;        // polls: at least 2 s

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Polls the mbarrier's phase `parity` up to `limit` times (non-blocking
// test_wait, a short sleep between polls); true once the phase completed.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done)
            return true;
        __nanosleep(64);
    }
    return false;
}

// Source and destination row of gather item `it`; sidx walks the segments
// forward (each lane visits its items in increasing order).
template <typename T>
__device__ __forceinline__ void gather_row(const GatherSeg *segs, const GatherSeg &single, int nsegs, int &sidx,
                                           int64_t it, const T *src, int64_t ld_src, T *dst, int64_t ld_dst,
                                           const T *&sp, T *&dp)
{
    const GatherSeg *sg = &single;
    if (segs) {
        while (sidx + 1 < nsegs && it >= segs[sidx + 1].item0)
            sidx++;
        sg = segs + sidx;
    }
    const int64_t b = it - sg->item0;
    int32_t r = __ldg(sg->idx + b);
    if (sg->mod)
        r %= sg->mod;
    sp = src + (sg->src_row0 + r) * ld_src;
    dp = dst + (sg->dst_row0 + b) * ld_dst;
}

// Dynamic shared memory: kWarpsPerBlock x ns slots of slot_bytes, then
// kWarpsPerBlock x ns mbarriers.
template <typename T>
__global__ void __launch_bounds__(kThreads) gather_rows_bulk_kernel(const GatherSeg *__restrict__ segs,
                                                                    const __grid_constant__ GatherSeg single,
                                                                    int nsegs, int64_t total,
                                                                    const T *__restrict__ src, int64_t ld_src,
                                                                    T *__restrict__ dst, int64_t ld_dst, int K,
                                                                    int ns, int chunk, int slot_bytes,
                                                                    uint32_t wait_limit, int *err)
{
    extern __shared__ __align__(128) unsigned char s_dyn[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int64_t wg = (int64_t)blockIdx.x * kWarpsPerBlock + w;
    const uint32_t bytes = (uint32_t)K * (uint32_t)sizeof(T);
    const uint32_t buf0 = smem_addr(s_dyn) + (uint32_t)(w * ns * slot_bytes);
    const uint32_t bar0 = smem_addr(s_dyn) + (uint32_t)(kWarpsPerBlock * ns * slot_bytes) + (uint32_t)(w * ns * 8);
    if (lane == 0) {
        for (int q = 0; q < ns; q++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0 + 8u * q) : "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // barriers visible to the copy engine
    }
    __syncwarp();
    const int64_t nchunks = (total + chunk - 1) / chunk;
    uint32_t phase = 0;  // bit q: parity of slot q's next completion (lane 0)
    int sidx = 0, ok = 1, pending_from = 0, pending_to = 0;
    for (int64_t c = wg; c < nchunks; c += nwarps) {
        const int64_t b0 = c * chunk;
        const int cnt = (int)min((int64_t)chunk, total - b0);
        const T *sp = nullptr;
        T *dp = nullptr;
        if (lane < cnt)
            gather_row(segs, single, nsegs, sidx, b0 + lane, src, ld_src, dst, ld_dst, sp, dp);
        for (int j = 0; j < cnt; j++) {  // every row's load at once
            const T *s_j = reinterpret_cast<const T *>(__shfl_sync(kFull, reinterpret_cast<uintptr_t>(sp), j));
            if (lane == 0) {
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar0 + 8u * j),
                             "r"(bytes)
                             : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                        buf0 + (uint32_t)j * (uint32_t)slot_bytes),
                    "l"(s_j), "r"(bytes), "r"(bar0 + 8u * j)
                    : "memory");
            }
        }
        for (int j = 0; j < cnt; j++) {  // each row's store as its load lands
            T *d_j = reinterpret_cast<T *>(__shfl_sync(kFull, reinterpret_cast<uintptr_t>(dp), j));
            if (lane == 0 && ok) {
                if (!mbar_wait(bar0 + 8u * j, (phase >> j) & 1u, wait_limit)) {
                    ok = 0;
                    pending_from = j;
                    pending_to = cnt;
                } else {
                    phase ^= 1u << j;
                    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(d_j),
                                 "r"(buf0 + (uint32_t)j * (uint32_t)slot_bytes), "r"(bytes)
                                 : "memory");
                }
            }
        }
        if (lane == 0) {
            asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
            asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");  // slots free for the next chunk
        }
        if (!__shfl_sync(kFull, ok, 0))
            break;
    }
    if (lane == 0) {
        if (!ok) {
            // every load issued for rows pending_from .. pending_to-1 lands
            // before the CTA exits (no store is issued for them)
            int code = 1;
            for (int j = pending_from; j < pending_to; j++)
                if (!mbar_wait(bar0 + 8u * j, (phase >> j) & 1u, kDrainLimit))
                    code = 2;
            atomicMax(err, code);
        }
        asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    }
}

// Staged row gather (include/dist_spmm_ppl_batch.cuh:59-73 generalised): one
// warp per row, 16-byte vectors, rows of all segments in one launch.
template <typename TR>
__global__ void __launch_bounds__(kThreads) gather_rows_kernel(const GatherSeg *__restrict__ segs,
                                                               const __grid_constant__ GatherSeg single, int nsegs,
                                                               int64_t total,
                                                               const typename ElemOf<TR>::T *__restrict__ src,
                                                               int64_t ld_src, typename ElemOf<TR>::T *__restrict__ dst,
                                                               int64_t ld_dst, int K)
{
    using T = typename ElemOf<TR>::T;
    using raw_t = typename TR::raw_t;
    constexpr int E = TR::E;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    int sidx = 0;
    for (int64_t it = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); it < total; it += nwarps) {
        const GatherSeg *s = &single;
        if (segs) {
            while (sidx + 1 < nsegs && it >= segs[sidx + 1].item0)
                sidx++;
            s = segs + sidx;
        }
        const int64_t b = it - s->item0;
        int32_t r = __ldg(s->idx + b);
        if (s->mod)
            r %= s->mod;
        const T *sp = src + (s->src_row0 + r) * ld_src;
        T *dp = dst + (s->dst_row0 + b) * ld_dst;
        for (int k = lane * E; k < K; k += 32 * E) {
            raw_t v = TR::load(sp + k);
            *reinterpret_cast<raw_t *>(dp + k) = v;
        }
    }
}

// FP32 -> BF16 (round to nearest even) of an n x K block, row strides ld_in/ld_out.
static __global__ void __launch_bounds__(kThreads) f32_to_bf16_kernel(const float *__restrict__ in, int64_t ld_in,
                                                              __nv_bfloat16 *__restrict__ out, int64_t ld_out,
                                                              int64_t rows, int K)
{
    const int64_t total = rows * (int64_t)K;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / K, k = i % K;
        out[r * ld_out + k] = __float2bfloat16_rn(in[r * ld_in + k]);
    }
}

}  // namespace dev
}  // namespace cola
