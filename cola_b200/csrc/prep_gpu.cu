// Device preprocessing: the row partitioning of prep_torch_par.py:24-79
// (row_partition), nnz_split (include/dist_spmm_ppl_batch.cuh:29-56) and the
// vertex relabelling of rabbit_module/src/reorder.cpp:283-288, run on the GPU
// with outputs bit-identical to the host build in prep.cpp.
//
// Partitioning is one stable LSD radix sort of every COO entry by
//     key = group << (pb + sb) | primary << sb | secondary
// with group = 2 * part + (entry is remote), and
//     local  entry: primary = row - lb (CSR row),    secondary = col - clb
//     remote entry: primary = col (global CSC col),  secondary = row - lb
// (lb = clb = part * npp).  Sorting by that key is the order tocsr() gives the
// local block and tocsc() the remote block; entries with equal keys (duplicate
// (row, col) pairs) keep input order, so summing each run of equal keys left
// to right sums duplicate values in input order, as the host build and scipy
// do.  The unique keys then are the index arrays: the secondary is the stored
// index (csr_colIdx_l / csc_rowIdx_r), a change of primary opens a row
// (column), the primaries at those points are csr_rowIdx_l / csc_colIdx_r and
// their positions are the row (column) pointers.  All of it is integer work
// bound by HBM: the sort moves 12 bytes per entry per 8-bit digit.
#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "graph.h"
#include "prep.h"

namespace cola {
namespace pg {

constexpr int kThreads = 256;
constexpr int kItems = 16;                     // radix tile: kThreads * kItems entries
constexpr int kTile = kThreads * kItems;
constexpr int kDigitBits = 8;
constexpr int kBins = 1 << kDigitBits;         // == kThreads: one bin per thread
constexpr int kWarps = kThreads / 32;
constexpr int kScanItems = 8;                  // scan tile: kThreads * kScanItems values
constexpr int kScanTile = kThreads * kScanItems;
static_assert(kBins == kThreads, "one radix bin per thread");

__device__ __forceinline__ uint32_t lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// ---------------------------------------------------------------------------
// exclusive scan of n uint32 values given by a functor (three launches)
// ---------------------------------------------------------------------------

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t &excl)
{
    __shared__ uint32_t wsum[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
            inc += y;
    }
    if (lane == 31)
        wsum[w] = inc;
    __syncthreads();
    uint32_t wbase = 0, total = 0;
#pragma unroll
    for (int k = 0; k < kWarps; k++) {
        const uint32_t s = wsum[k];
        wbase += k < w ? s : 0u;
        total += s;
    }
    __syncthreads();  // wsum reusable by the next call
    excl = wbase + inc - v;
    return total;
}

template <class F>
__global__ void __launch_bounds__(kThreads) scan_reduce_kernel(F f, int64_t n, uint32_t *partial)
{
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++)
        s += base + j < n ? f(base + j) : 0u;
    uint32_t excl;
    const uint32_t total = block_exclusive_scan(s, excl);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = total;
}

// One block: partial[] becomes its exclusive scan; *total = the sum.
__global__ void __launch_bounds__(kThreads) scan_partials_kernel(uint32_t *partial, int64_t nb, uint32_t *total)
{
    __shared__ uint32_t carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (int64_t b0 = 0; b0 < nb; b0 += kThreads) {
        const int64_t b = b0 + threadIdx.x;
        const uint32_t v = b < nb ? partial[b] : 0u;
        uint32_t excl;
        const uint32_t t = block_exclusive_scan(v, excl);
        const uint32_t c = carry;
        if (b < nb)
            partial[b] = c + excl;
        __syncthreads();
        if (threadIdx.x == 0)
            carry = c + t;
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *total = carry;
}

template <class F>
__global__ void __launch_bounds__(kThreads) scan_write_kernel(F f, int64_t n, const uint32_t *partial, uint32_t *out)
{
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems], s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        v[j] = base + j < n ? f(base + j) : 0u;
        s += v[j];
    }
    uint32_t excl;
    block_exclusive_scan(s, excl);
    uint32_t run = partial[blockIdx.x] + excl;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        if (base + j < n)
            out[base + j] = run;
        run += v[j];
    }
}

struct ArrayF {
    const uint32_t *a;
    __device__ uint32_t operator()(int64_t i) const { return a[i]; }
};
// 1 where a new key starts in the sorted keys
struct KeyStartF {
    const uint64_t *k;
    int shift;
    __device__ uint32_t operator()(int64_t i) const { return i == 0 || (k[i] >> shift) != (k[i - 1] >> shift); }
};
// nnz_split chunks of row i: ceil(len / gran)
struct ChunksF {
    const int32_t *ptr;
    int64_t gran;
    __device__ uint32_t operator()(int64_t i) const
    {
        const int64_t len = (int64_t)ptr[i + 1] - ptr[i];
        return len > 0 ? (uint32_t)((len + gran - 1) / gran) : 0u;
    }
};

// ---------------------------------------------------------------------------
// partitioning kernels
// ---------------------------------------------------------------------------

__global__ void check_coo_kernel(const int32_t *row, const int32_t *col, int64_t n, int32_t N,
                                 unsigned long long *first_bad)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = row[i], c = col[i];
        if (r < 0 || r >= N || c < 0 || c >= N)
            atomicMin(first_bad, (unsigned long long)i);
    }
}

__global__ void make_keys_kernel(const int32_t *row, const int32_t *col, int64_t n, uint32_t npp, int sb, int gshift,
                                 uint64_t *key, uint32_t *idx)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)row[i], c = (uint32_t)col[i];
        const uint32_t p = r / npp, lb = p * npp;
        const bool local = c / npp == p;
        const uint64_t g = 2ull * p + (local ? 0u : 1u);
        const uint64_t prim = local ? r - lb : c;
        const uint64_t sec = local ? c - lb : r - lb;
        key[i] = g << gshift | prim << sb | sec;
        idx[i] = (uint32_t)i;
    }
}

// Per tile digit counts, stored bin-major (hist[bin * ntiles + tile]) so one
// exclusive scan gives every (bin, tile) its first output position.
__global__ void __launch_bounds__(kThreads) radix_hist_kernel(const uint64_t *key, int64_t n, int shift,
                                                              int64_t ntiles, uint32_t *hist)
{
    __shared__ uint32_t h[kBins];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t tile0 = (int64_t)blockIdx.x * kTile;
    for (int r = 0; r < kItems; r++) {
        const int64_t i = tile0 + r * kThreads + threadIdx.x;
        const uint32_t d = i < n ? (uint32_t)(key[i] >> shift) & (kBins - 1) : (uint32_t)kBins;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (d < kBins && (peers & lanemask_lt()) == 0)
            atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: entries keep their order within each digit.
// Rounds of kThreads consecutive entries; inside a round a warp ranks its
// lanes per digit (match_any), warps are ranked per digit in shared memory,
// and rounds follow one another per digit through base[].
__global__ void __launch_bounds__(kThreads) radix_scatter_kernel(const uint64_t *kin, const uint32_t *vin,
                                                                 uint64_t *kout, uint32_t *vout, int64_t n, int shift,
                                                                 int64_t ntiles, const uint32_t *hist_scan)
{
    __shared__ uint32_t base[kBins];
    __shared__ uint32_t wcnt[kWarps][kBins];
    __shared__ uint32_t wpos[kWarps][kBins];
    const int t = threadIdx.x, w = t >> 5;
    base[t] = hist_scan[(int64_t)t * ntiles + blockIdx.x];
#pragma unroll
    for (int k = 0; k < kWarps; k++)
        wcnt[k][t] = 0;
    __syncthreads();
    const int64_t tile0 = (int64_t)blockIdx.x * kTile;
    for (int r = 0; r < kItems; r++) {
        if (tile0 + (int64_t)r * kThreads >= n)
            break;  // uniform across the block
        const int64_t i = tile0 + r * kThreads + t;
        const bool valid = i < n;
        const uint64_t k = valid ? kin[i] : 0ull;
        const uint32_t v = valid ? vin[i] : 0u;
        const uint32_t d = valid ? (uint32_t)(k >> shift) & (kBins - 1) : (uint32_t)kBins;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & lanemask_lt());
        if (valid && rank == 0)
            wcnt[w][d] = __popc(peers);
        __syncthreads();
        uint32_t run = base[t];
#pragma unroll
        for (int q = 0; q < kWarps; q++) {
            const uint32_t c = wcnt[q][t];
            wpos[q][t] = run;
            run += c;
            wcnt[q][t] = 0;
        }
        base[t] = run;
        __syncthreads();
        if (valid) {
            const uint32_t pos = wpos[w][d] + rank;
            kout[pos] = k;
            vout[pos] = v;
        }
    }
}

// One thread per run of equal keys: the unique key and its values summed in
// input order (1.0 each without values).
__global__ void dedupe_kernel(const uint64_t *key, const uint32_t *idx, const float *val, int64_t n,
                              const uint32_t *upos, uint64_t *ukey, float *uval)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[i];
        if (i > 0 && key[i - 1] == k)
            continue;
        float v = val ? val[idx[i]] : 1.0f;
        for (int64_t j = i + 1; j < n && key[j] == k; j++)
            v += val ? val[idx[j]] : 1.0f;
        const uint32_t u = upos[i];
        ukey[u] = k;
        uval[u] = v;
    }
}

__global__ void seg_start_kernel(const uint64_t *ukey, int64_t U, const uint32_t *spos, int sb, uint32_t *seg_start)
{
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x)
        if (u == 0 || (ukey[u] >> sb) != (ukey[u - 1] >> sb))
            seg_start[spos[u]] = (uint32_t)u;
}

// u_off[g] / s_off[g]: first unique entry / segment of group g (g = 0..G).
__global__ void group_bounds_kernel(const uint64_t *ukey, int64_t U, const uint32_t *seg_start, int64_t S, int G,
                                    int gshift, int64_t *u_off, int64_t *s_off)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g > G)
        return;
    if (g == G) {
        u_off[g] = U;
        s_off[g] = S;
        return;
    }
    const uint64_t kb = (uint64_t)g << gshift;
    int64_t lo = 0, hi = U;
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (ukey[m] < kb)
            lo = m + 1;
        else
            hi = m;
    }
    u_off[g] = lo;
    int64_t a = 0, b = S;
    while (a < b) {
        const int64_t m = (a + b) >> 1;
        if (ukey[seg_start[m]] < kb)
            a = m + 1;
        else
            b = m;
    }
    s_off[g] = a;
}

__global__ void out_entries_kernel(const uint64_t *ukey, int64_t U, uint64_t smask, int32_t *sec)
{
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x)
        sec[u] = (int32_t)(ukey[u] & smask);
}

// Segment s of group g: its primary, and ptr[s + g] = its first entry
// relative to the group (group g's pointer array is ptr[s_off[g] + g ...]).
__global__ void out_segments_kernel(const uint64_t *ukey, const uint32_t *seg_start, int64_t S, int sb,
                                    uint64_t pmask, int gshift, const int64_t *u_off, int32_t *prim, int32_t *ptr)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < S; s += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t u = seg_start[s];
        const uint64_t k = ukey[u];
        const int g = (int)(k >> gshift);
        prim[s] = (int32_t)((k >> sb) & pmask);
        ptr[s + g] = (int32_t)(u - u_off[g]);
    }
}

__global__ void out_group_ends_kernel(const int64_t *u_off, const int64_t *s_off, int G, int32_t *ptr)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G)
        ptr[s_off[g + 1] + g] = (int32_t)(u_off[g + 1] - u_off[g]);
}

// nnz_split: one thread per chunk; its row is the last row whose first chunk
// is at or before it.
__global__ void split_write_kernel(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, const uint32_t *coff,
                                   int64_t nchunks, int64_t gran, int32_t *target, int32_t *ptr)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nchunks;
         c += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = nrows;  // first row with coff > c
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (coff[m] <= (uint64_t)c)
                lo = m + 1;
            else
                hi = m;
        }
        const int64_t r = lo - 1;
        const int64_t k = c - coff[r];
        const int64_t hb = rowPtr[r + 1];
        const int64_t e = (int64_t)rowPtr[r] + (k + 1) * gran;
        target[c] = rowIdx[r];
        ptr[c + 1] = (int32_t)(e > hb ? hb : e);
        if (c == 0)
            ptr[0] = 0;
    }
}

__global__ void relabel_kernel(const int32_t *row, const int32_t *col, int64_t n, const int32_t *map, int32_t N,
                               int32_t *out_row, int32_t *out_col, unsigned long long *first_bad)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = row[i], c = col[i];
        if (r < 0 || r >= N || c < 0 || c >= N) {
            atomicMin(first_bad, (unsigned long long)i);
            continue;
        }
        const int32_t mr = map[r], mc = map[c];
        if (mr < 0 || mr >= N || mc < 0 || mc >= N) {
            atomicMin(first_bad, (unsigned long long)i);
            continue;
        }
        out_row[i] = mr;
        out_col[i] = mc;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

inline int bits_for(uint64_t v)  // bits to hold values 0..v
{
    int b = 0;
    while (b < 64 && (v >> b) != 0)
        b++;
    return b;
}

inline unsigned grid_stride_blocks(int64_t n)
{
    const int64_t cap = (int64_t)sm_count() * 8;
    const int64_t need = (n + 255) / 256;
    return (unsigned)(need < 1 ? 1 : need < cap ? need : cap);
}

// Scratch device memory for one call, released on every exit path: carved
// from one arena when the caller reserves one (a single mapping per call, kept
// for the whole call), else one stream-ordered allocation per request.
struct Scratch {
    cudaStream_t st;
    std::vector<void *> ptrs;
    char *arena = nullptr;
    size_t used = 0, cap = 0;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch()
    {
        for (void *p : ptrs)
            cudaFreeAsync(p, st);
    }
    cola_status alloc(void *&q, size_t bytes)
    {
        const cudaError_t e = cudaMallocAsync(&q, bytes, st);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? COLA_ERROR_OUT_OF_MEMORY : COLA_ERROR_CUDA,
                        "device preprocessing: cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
        ptrs.push_back(q);
        return COLA_SUCCESS;
    }
    cola_status reserve(size_t bytes)
    {
        void *q = nullptr;
        COLA_TRY(alloc(q, bytes));
        arena = static_cast<char *>(q);
        cap = bytes;
        used = 0;
        return COLA_SUCCESS;
    }
    template <class T>
    cola_status get(T *&p, int64_t count)
    {
        const size_t bytes = ((size_t)(count > 0 ? count : 1) * sizeof(T) + 255) & ~(size_t)255;
        if (arena && used + bytes <= cap) {
            p = reinterpret_cast<T *>(arena + used);
            used += bytes;
            return COLA_SUCCESS;
        }
        void *q = nullptr;
        COLA_TRY(alloc(q, bytes));
        p = static_cast<T *>(q);
        return COLA_SUCCESS;
    }
};

// Device -> host copies through a pinned double buffer: chunk i + 1 crosses
// PCIe while host threads spread chunk i into its destinations, so large
// results reach pageable host memory near link speed.  One staging area per
// process, grown on demand, used by one call at a time.
struct HostCopy {
    void *dst;
    const void *src;
    size_t bytes;
};

static std::mutex g_stage_mu;
static char *g_stage[2] = {nullptr, nullptr};
static cudaEvent_t g_stage_ev[2] = {nullptr, nullptr};
constexpr size_t kStageBytes = 16u << 20;

static cola_status copy_to_host(const std::vector<HostCopy> &jobs, cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(g_stage_mu);
    for (int b = 0; b < 2; b++) {
        if (!g_stage[b])
            COLA_CUDA(cudaMallocHost((void **)&g_stage[b], kStageBytes));
        if (!g_stage_ev[b])
            COLA_CUDA(cudaEventCreateWithFlags(&g_stage_ev[b], cudaEventDisableTiming));
    }
    // pieces of at most one chunk, packed into chunks in order
    struct Piece {
        char *dst;
        const char *src;
        size_t bytes, off;  // off: position in its chunk
    };
    std::vector<std::vector<Piece>> chunks(1);
    size_t fill = 0;
    for (const HostCopy &j : jobs) {
        size_t done = 0;
        while (done < j.bytes) {
            if (fill == kStageBytes) {
                chunks.emplace_back();
                fill = 0;
            }
            const size_t n = std::min(j.bytes - done, kStageBytes - fill);
            chunks.back().push_back(
                {static_cast<char *>(j.dst) + done, static_cast<const char *>(j.src) + done, n, fill});
            fill += n;
            done += n;
        }
    }
    auto issue = [&](size_t c) -> cola_status {
        char *buf = g_stage[c & 1];
        for (const Piece &p : chunks[c])
            COLA_CUDA(cudaMemcpyAsync(buf + p.off, p.src, p.bytes, cudaMemcpyDeviceToHost, st));
        COLA_CUDA(cudaEventRecord(g_stage_ev[c & 1], st));
        return COLA_SUCCESS;
    };
    if (chunks[0].empty())
        return COLA_SUCCESS;
    COLA_TRY(issue(0));
    for (size_t c = 0; c < chunks.size(); c++) {
        if (c + 1 < chunks.size())
            COLA_TRY(issue(c + 1));  // the other buffer: its previous chunk was spread already
        COLA_CUDA(cudaEventSynchronize(g_stage_ev[c & 1]));
        const char *buf = g_stage[c & 1];
        const std::vector<Piece> &ps = chunks[c];
        // spread in 256 KiB slices over the host threads
        constexpr size_t kSlice = 256u << 10;
        std::vector<std::pair<size_t, size_t>> work;  // (piece, slice start)
        for (size_t i = 0; i < ps.size(); i++)
            for (size_t o = 0; o < ps[i].bytes; o += kSlice)
                work.emplace_back(i, o);
#pragma omp parallel for schedule(dynamic, 4)
        for (int64_t w = 0; w < (int64_t)work.size(); w++) {
            const Piece &p = ps[work[(size_t)w].first];
            const size_t o = work[(size_t)w].second;
            std::memcpy(p.dst + o, buf + p.off + o, std::min(kSlice, p.bytes - o));
        }
    }
    return COLA_SUCCESS;
}

// out[i] = exclusive prefix sum of f(0..i-1) for i < n; *total (host) = sum.
template <class F>
static cola_status exclusive_scan(F f, int64_t n, uint32_t *out, uint32_t *d_total, uint32_t *total, Scratch &sc)
{
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    uint32_t *partial = nullptr;
    COLA_TRY(sc.get(partial, nb));
    if (n > 0) {
        scan_reduce_kernel<F><<<(unsigned)nb, kThreads, 0, sc.st>>>(f, n, partial);
        t_launches++;
    }
    scan_partials_kernel<<<1, kThreads, 0, sc.st>>>(partial, nb, d_total);
    t_launches++;
    if (n > 0) {
        scan_write_kernel<F><<<(unsigned)nb, kThreads, 0, sc.st>>>(f, n, partial, out);
        t_launches++;
    }
    COLA_CUDA(cudaGetLastError());
    if (total) {
        COLA_CUDA(cudaMemcpyAsync(total, d_total, sizeof(uint32_t), cudaMemcpyDeviceToHost, sc.st));
        COLA_CUDA(cudaStreamSynchronize(sc.st));
    }
    return COLA_SUCCESS;
}

static cola_status check_range(const int32_t *row, const int32_t *col, int64_t n, int32_t N, Scratch &sc,
                               const char *who)
{
    unsigned long long *bad = nullptr, h_bad = 0;
    COLA_TRY(sc.get(bad, 1));
    COLA_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(*bad), sc.st));
    check_coo_kernel<<<grid_stride_blocks(n), 256, 0, sc.st>>>(row, col, n, N, bad);
    t_launches++;
    COLA_CUDA(cudaGetLastError());
    COLA_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(h_bad), cudaMemcpyDeviceToHost, sc.st));
    COLA_CUDA(cudaStreamSynchronize(sc.st));
    if (h_bad != ULLONG_MAX) {
        int32_t r = 0, c = 0;
        cudaMemcpy(&r, row + h_bad, 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(&c, col + h_bad, 4, cudaMemcpyDeviceToHost);
        return fail(COLA_ERROR_INVALID_ARGUMENT, "%s: entry %llu (%d, %d) outside %d x %d", who, h_bad, r, c, N, N);
    }
    return COLA_SUCCESS;
}

static cola_status partition_build_device(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col,
                                          const float *val, int32_t nparts, cudaStream_t st, cola_partition_set *&out)
{
    const char *who = "cola_partition_build_device";
    COLA_REQUIRE(N >= 0 && nnz >= 0 && nparts >= 1, COLA_ERROR_INVALID_ARGUMENT, "%s: N=%d nnz=%lld nparts=%d", who,
                 N, (long long)nnz, nparts);
    COLA_REQUIRE(nnz == 0 || (row && col), COLA_ERROR_INVALID_ARGUMENT, "%s: null COO arrays", who);
    COLA_REQUIRE(nnz < (int64_t)UINT32_MAX, COLA_ERROR_UNSUPPORTED, "%s: nnz >= 2^32", who);
    const int64_t npp = ((int64_t)N + nparts - 1) / nparts;  // prep_torch_par.py:31
    const int G = 2 * nparts;
    const int sb = bits_for(npp > 0 ? (uint64_t)npp - 1 : 0);
    const int pb = bits_for(N > 0 ? (uint64_t)N - 1 : 0);
    const int gshift = sb + pb;
    COLA_REQUIRE(gshift + bits_for((uint64_t)G - 1) <= 64, COLA_ERROR_UNSUPPORTED,
                 "%s: %d nodes in %d partitions need a sort key wider than 64 bits", who, N, nparts);
    const int key_bits = gshift + bits_for((uint64_t)G - 1);

    std::unique_ptr<cola_partition_set> s(new (std::nothrow) cola_partition_set());
    COLA_REQUIRE(s, COLA_ERROR_OUT_OF_MEMORY, "%s: host allocation failed", who);
    s->num_nodes = N;
    s->nparts = nparts;
    s->npp = (int32_t)npp;
    s->parts.resize((size_t)nparts);
    for (int32_t r = 0; r < nparts; r++) {
        PartHost &P = s->parts[(size_t)r];
        P.part = r;
        P.row_lb = (int32_t)std::min<int64_t>((int64_t)r * npp, N);
        P.row_ub = (int32_t)std::min<int64_t>((int64_t)(r + 1) * npp, N);
        P.l_rowPtr.assign(1, 0);
        P.r_colPtr.assign(1, 0);
    }
    if (nnz == 0) {
        out = s.release();
        return COLA_SUCCESS;
    }
    Scratch sc(st);
    const int64_t ntiles = (nnz + kTile - 1) / kTile;
    {
        // every buffer below, each rounded to 256 bytes, plus the scans' block sums
        const size_t n = (size_t)nnz, a = 256;
        const size_t scan_blocks = (size_t)((std::max<int64_t>(ntiles * kBins, nnz) + kScanTile - 1) / kScanTile) + 1;
        const size_t bytes = 2 * (8 * n + a) + 2 * (4 * n + a) + (4 * (size_t)ntiles * kBins + a) + 4 * (4 * n + a) +
                             (4 * (n + (size_t)G) + a) + 2 * (8 * ((size_t)G + 1) + a) + 2 * a +
                             (2 * 6 + 16) * (4 * scan_blocks + a);
        COLA_TRY(sc.reserve(bytes));
    }
    COLA_TRY(check_range(row, col, nnz, N, sc, who));

    // sort
    uint64_t *k0 = nullptr, *k1 = nullptr;
    uint32_t *v0 = nullptr, *v1 = nullptr, *hist = nullptr, *d_total = nullptr;
    COLA_TRY(sc.get(k0, nnz));
    COLA_TRY(sc.get(k1, nnz));
    COLA_TRY(sc.get(v0, nnz));
    COLA_TRY(sc.get(v1, nnz));
    COLA_TRY(sc.get(hist, ntiles * kBins));
    COLA_TRY(sc.get(d_total, 1));
    make_keys_kernel<<<grid_stride_blocks(nnz), 256, 0, st>>>(row, col, nnz, (uint32_t)(npp > 0 ? npp : 1), sb,
                                                              gshift, k0, v0);
    t_launches++;
    COLA_CUDA(cudaGetLastError());
    for (int shift = 0; shift < key_bits; shift += kDigitBits) {
        radix_hist_kernel<<<(unsigned)ntiles, kThreads, 0, st>>>(k0, nnz, shift, ntiles, hist);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
        COLA_TRY(exclusive_scan(ArrayF{hist}, ntiles * kBins, hist, d_total, nullptr, sc));
        radix_scatter_kernel<<<(unsigned)ntiles, kThreads, 0, st>>>(k0, v0, k1, v1, nnz, shift, ntiles, hist);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
        std::swap(k0, k1);
        std::swap(v0, v1);
    }
    // merge duplicates: unique keys into k1, summed values
    uint32_t *upos = nullptr;
    float *uval = nullptr;
    uint32_t U = 0;
    COLA_TRY(sc.get(upos, nnz));
    COLA_TRY(exclusive_scan(KeyStartF{k0, 0}, nnz, upos, d_total, &U, sc));
    COLA_TRY(sc.get(uval, U));
    uint64_t *ukey = k1;
    dedupe_kernel<<<grid_stride_blocks(nnz), 256, 0, st>>>(k0, v0, val, nnz, upos, ukey, uval);
    t_launches++;
    COLA_CUDA(cudaGetLastError());
    // rows (local) / columns (remote): runs of equal primary within a group
    uint32_t *spos = upos, *seg_start = v1;  // both free again (U <= nnz)
    uint32_t S = 0;
    COLA_TRY(exclusive_scan(KeyStartF{ukey, sb}, U, spos, d_total, &S, sc));
    seg_start_kernel<<<grid_stride_blocks(U), 256, 0, st>>>(ukey, U, spos, sb, seg_start);
    t_launches++;
    int64_t *u_off = nullptr, *s_off = nullptr;
    COLA_TRY(sc.get(u_off, G + 1));
    COLA_TRY(sc.get(s_off, G + 1));
    group_bounds_kernel<<<(G + 1 + 127) / 128, 128, 0, st>>>(ukey, U, seg_start, S, G, gshift, u_off, s_off);
    t_launches++;
    int32_t *sec = nullptr, *prim = nullptr, *ptr = nullptr;
    COLA_TRY(sc.get(sec, U));
    COLA_TRY(sc.get(prim, S));
    COLA_TRY(sc.get(ptr, (int64_t)S + G));
    const uint64_t smask = sb >= 64 ? ~0ull : (1ull << sb) - 1, pmask = pb >= 64 ? ~0ull : (1ull << pb) - 1;
    out_entries_kernel<<<grid_stride_blocks(U), 256, 0, st>>>(ukey, U, smask, sec);
    out_segments_kernel<<<grid_stride_blocks(S), 256, 0, st>>>(ukey, seg_start, S, sb, pmask, gshift, u_off, prim,
                                                               ptr);
    out_group_ends_kernel<<<(G + 127) / 128, 128, 0, st>>>(u_off, s_off, G, ptr);
    t_launches += 3;
    COLA_CUDA(cudaGetLastError());
    std::vector<int64_t> hu((size_t)G + 1), hs((size_t)G + 1);
    COLA_CUDA(cudaMemcpyAsync(hu.data(), u_off, hu.size() * 8, cudaMemcpyDeviceToHost, st));
    COLA_CUDA(cudaMemcpyAsync(hs.data(), s_off, hs.size() * 8, cudaMemcpyDeviceToHost, st));
    COLA_CUDA(cudaStreamSynchronize(st));
    std::vector<HostCopy> jobs;
    try {
        for (int32_t r = 0; r < nparts; r++) {
            PartHost &P = s->parts[(size_t)r];
            for (int rem = 0; rem < 2; rem++) {
                const int g = 2 * r + rem;
                const int64_t u0 = hu[(size_t)g], nu = hu[(size_t)g + 1] - u0;
                const int64_t s0 = hs[(size_t)g], ns = hs[(size_t)g + 1] - s0;
                ivec &ent = rem ? P.r_rowIdx : P.l_colIdx;
                fvec &v = rem ? P.r_val : P.l_val;
                ivec &ids = rem ? P.r_colIdx : P.l_rowIdx;
                ivec &ptrs = rem ? P.r_colPtr : P.l_rowPtr;
                ent.resize((size_t)nu);
                v.resize((size_t)nu);
                ids.resize((size_t)ns);
                ptrs.resize((size_t)ns + 1);
                if (nu > 0) {
                    jobs.push_back({ent.data(), sec + u0, (size_t)nu * 4});
                    jobs.push_back({v.data(), uval + u0, (size_t)nu * 4});
                    jobs.push_back({ids.data(), prim + s0, (size_t)ns * 4});
                    jobs.push_back({ptrs.data(), ptr + s0 + g, (size_t)(ns + 1) * 4});
                } else {
                    ptrs[0] = 0;
                }
            }
        }
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "%s: host allocation failed", who);
    }
    COLA_TRY(copy_to_host(jobs, st));
    out = s.release();
    return COLA_SUCCESS;
}

}  // namespace pg
}  // namespace cola

using namespace cola;

extern "C" {

cola_status cola_partition_build_device(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                        const float *val, int32_t nparts, cudaStream_t stream,
                                        cola_partition_set **out)
{
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "cola_partition_build_device: out is NULL");
    *out = nullptr;
    clear_error();
    cola_partition_set *s = nullptr;
    COLA_TRY(pg::partition_build_device(num_nodes, nnz, row, col, val, nparts, stream, s));
    *out = s;
    return COLA_SUCCESS;
}

cola_status cola_nnz_split_device(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                                  int32_t *target, int32_t *ptr, int64_t capacity, int64_t *nchunks,
                                  cudaStream_t stream)
{
    COLA_REQUIRE(nchunks && nrows >= 0 && nnz >= 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_nnz_split_device: bad arguments");
    *nchunks = 0;
    if (nrows == 0)
        return COLA_SUCCESS;  // include/dist_spmm_ppl_batch.cuh:32-33: both outputs stay empty
    COLA_REQUIRE(rowIdx && rowPtr, COLA_ERROR_INVALID_ARGUMENT, "cola_nnz_split_device: null arrays");
    const int64_t avg = nnz / nrows;            // :34
    const int64_t gran = (avg + 31) / 32 * 32;  // :35
    COLA_REQUIRE(gran > 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_nnz_split_device: %lld entries over %lld rows gives a zero chunk size", (long long)nnz,
                 (long long)nrows);
    COLA_REQUIRE(nrows < (int64_t)UINT32_MAX, COLA_ERROR_UNSUPPORTED, "cola_nnz_split_device: too many rows");
    pg::Scratch sc(stream);
    uint32_t *coff = nullptr, *d_total = nullptr, total = 0;
    COLA_TRY(sc.get(coff, nrows));
    COLA_TRY(sc.get(d_total, 1));
    COLA_TRY(pg::exclusive_scan(pg::ChunksF{rowPtr, gran}, nrows, coff, d_total, &total, sc));
    *nchunks = total;
    if (!target)
        return COLA_SUCCESS;
    COLA_REQUIRE(ptr && capacity >= (int64_t)total, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_nnz_split_device: capacity %lld < %u chunks", (long long)capacity, total);
    if (total == 0) {
        COLA_CUDA(cudaMemsetAsync(ptr, 0, 4, stream));
    } else {
        pg::split_write_kernel<<<pg::grid_stride_blocks(total), 256, 0, stream>>>(rowIdx, nrows, rowPtr, coff, total,
                                                                                   gran, target, ptr);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
    }
    COLA_CUDA(cudaStreamSynchronize(stream));
    return COLA_SUCCESS;
}

cola_status cola_relabel_edges_device(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                      const int32_t *mapping, int32_t *out_row, int32_t *out_col, cudaStream_t stream)
{
    COLA_REQUIRE(num_nodes >= 0 && nnz >= 0, COLA_ERROR_INVALID_ARGUMENT, "cola_relabel_edges_device: bad sizes");
    if (nnz == 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(row && col && mapping && out_row && out_col, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_relabel_edges_device: null arrays");
    pg::Scratch sc(stream);
    unsigned long long *bad = nullptr, h_bad = 0;
    COLA_TRY(sc.get(bad, 1));
    COLA_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(*bad), stream));
    pg::relabel_kernel<<<pg::grid_stride_blocks(nnz), 256, 0, stream>>>(row, col, nnz, mapping, num_nodes, out_row,
                                                                         out_col, bad);
    t_launches++;
    COLA_CUDA(cudaGetLastError());
    COLA_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(h_bad), cudaMemcpyDeviceToHost, stream));
    COLA_CUDA(cudaStreamSynchronize(stream));
    COLA_REQUIRE(h_bad == ULLONG_MAX, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_relabel_edges_device: entry %llu or its relabelled ids outside 0..%d", h_bad, num_nodes - 1);
    return COLA_SUCCESS;
}

}  // extern "C"
