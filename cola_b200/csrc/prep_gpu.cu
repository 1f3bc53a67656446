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
#include <array>
#include <climits>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
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

__global__ void check_coo_kernel(const int32_t *row, const int32_t *col, int64_t n, int32_t NR, int32_t NC,
                                 unsigned long long *first_bad)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = row[i], c = col[i];
        if (r < 0 || r >= NR || c < 0 || c >= NC)
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
// row view of a graph built on the device: the global CSR (row, col) order of
// the unique entries, hub segments and row-block tasks, the same arrays the
// host upload derives from the partitions (spmm.cu graph_upload)
// ---------------------------------------------------------------------------

__global__ void make_row_keys_kernel(const int32_t *row, const int32_t *col, int64_t n, int cb, uint64_t *key,
                                     uint32_t *idx)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        key[i] = (uint64_t)(uint32_t)row[i] << cb | (uint32_t)col[i];
        idx[i] = (uint32_t)i;
    }
}

// rv_ptr[r] = first unique entry of row >= r (r = 0..N); rv_col = the columns
__global__ void row_ptr_kernel(const uint64_t *ukey, int64_t U, int cb, int64_t N, int64_t *rv_ptr)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= N; r += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t kb = (uint64_t)r << cb;
        int64_t lo = 0, hi = U;
        while (lo < hi) {
            const int64_t m = (lo + hi) >> 1;
            if (ukey[m] < kb)
                lo = m + 1;
            else
                hi = m;
        }
        rv_ptr[r] = lo;
    }
}

__global__ void row_cols_kernel(const uint64_t *ukey, int64_t U, uint64_t cmask, int32_t *rv_col)
{
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x)
        rv_col[u] = (int32_t)(ukey[u] & cmask);
}

// 1 per hub row (more than thr entries)
struct HubF {
    const int64_t *ptr;
    int64_t thr;
    __device__ uint32_t operator()(int64_t r) const { return ptr[r + 1] - ptr[r] > thr; }
};
// segments of row r: ceil(len / seg) for a hub row, else 0
struct SegCountF {
    const int64_t *ptr;
    int64_t thr, seg;
    __device__ uint32_t operator()(int64_t r) const
    {
        const int64_t len = ptr[r + 1] - ptr[r];
        return len > thr ? (uint32_t)((len + seg - 1) / seg) : 0u;
    }
};
// 1 where a run of non-hub rows starts
struct RunStartF {
    const int64_t *ptr;
    int64_t thr;
    __device__ uint32_t operator()(int64_t r) const
    {
        const bool hub = ptr[r + 1] - ptr[r] > thr;
        return !hub && (r == 0 || ptr[r] - ptr[r - 1] > thr);
    }
};

__global__ void hub_segments_kernel(const int64_t *ptr, int64_t N, int64_t thr, int64_t seg, const uint32_t *hubpos,
                                    const uint32_t *segoff, int64_t nhub, int64_t nseg, int32_t *hub_row,
                                    int64_t *hub_seg, int32_t *seg_row, int64_t *seg_beg)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = ptr[r], e = ptr[r + 1];
        if (e - b <= thr)
            continue;
        const int64_t h = hubpos[r], s0 = segoff[r];
        hub_row[h] = (int32_t)r;
        hub_seg[h] = s0;
        int64_t s = s0;
        for (int64_t q = b; q < e; q += seg, s++) {
            seg_row[s] = (int32_t)r;
            seg_beg[s] = q;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        hub_seg[nhub] = nseg;
}

// The host's greedy packing of rows into tasks (a row costs its entries plus
// 2; a task closes once its cost reaches te; hub rows close a task and belong
// to none), run independently on every run of non-hub rows, which is exactly
// where the greedy state is reset.  Pass 1 (rb == nullptr) counts each run's
// tasks into cnt; pass 2 writes them from off[run] on.
__global__ void run_tasks_kernel(const int64_t *ptr, int64_t N, int64_t thr, int64_t te, const uint32_t *runpos,
                                 uint32_t *cnt, const uint32_t *off, int32_t *rb, int32_t *re)
{
    for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < N; a += (int64_t)gridDim.x * blockDim.x) {
        const bool hub_a = ptr[a + 1] - ptr[a] > thr;
        if (hub_a || (a > 0 && !(ptr[a] - ptr[a - 1] > thr)))
            continue;  // not the first row of a run
        const uint32_t run = runpos[a];
        uint32_t t = rb ? off[run] : 0u, k = 0;
        int64_t start = -1, cost = 0, r = a;
        for (; r < N; r++) {
            const int64_t len = ptr[r + 1] - ptr[r];
            if (len > thr)
                break;
            if (start < 0)
                start = r;
            cost += len + 2;
            if (cost >= te) {
                if (rb) {
                    rb[t + k] = (int32_t)start;
                    re[t + k] = (int32_t)(r + 1);
                }
                k++;
                start = -1;
                cost = 0;
            }
        }
        if (start >= 0) {
            if (rb) {
                rb[t + k] = (int32_t)start;
                re[t + k] = (int32_t)r;
            }
            k++;
        }
        if (!rb)
            cnt[run] = k;
    }
}

// entries whose column lies in the row's own partition (the local block)
__global__ void count_local_kernel(const uint64_t *ukey, int64_t U, int cb, uint32_t npp,
                                   unsigned long long *local)
{
    unsigned long long c = 0;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(ukey[u] >> cb), k = (uint32_t)(ukey[u] & ((1ull << cb) - 1));
        c += r / npp == k / npp;
    }
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(local, c);
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
static char *g_stage[2] = {nullptr, nullptr};  // pinned: reachable from every device
static std::unordered_map<int, std::array<cudaEvent_t, 2>> g_stage_ev;  // events belong to one device
constexpr size_t kStageBytes = 16u << 20;

static cola_status copy_to_host(const std::vector<HostCopy> &jobs, cudaStream_t st)
{
    std::lock_guard<std::mutex> lk(g_stage_mu);
    int dev = 0;
    COLA_CUDA(cudaGetDevice(&dev));
    for (int b = 0; b < 2; b++)
        if (!g_stage[b])
            COLA_CUDA(cudaMallocHost((void **)&g_stage[b], kStageBytes));
    auto it = g_stage_ev.find(dev);
    if (it == g_stage_ev.end()) {
        std::array<cudaEvent_t, 2> ev{};
        for (cudaEvent_t &e : ev)
            COLA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        it = g_stage_ev.emplace(dev, ev).first;
    }
    const std::array<cudaEvent_t, 2> &stage_ev = it->second;
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
        COLA_CUDA(cudaEventRecord(stage_ev[c & 1], st));
        return COLA_SUCCESS;
    };
    if (chunks[0].empty())
        return COLA_SUCCESS;
    COLA_TRY(issue(0));
    for (size_t c = 0; c < chunks.size(); c++) {
        if (c + 1 < chunks.size())
            COLA_TRY(issue(c + 1));  // the other buffer: its previous chunk was spread already
        COLA_CUDA(cudaEventSynchronize(stage_ev[c & 1]));
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

// Every entry inside NR rows x NC columns (NC < 0: NC = NR).
static cola_status check_range(const int32_t *row, const int32_t *col, int64_t n, int32_t N, Scratch &sc,
                               const char *who, int32_t NC = -1)
{
    if (NC < 0)
        NC = N;
    unsigned long long *bad = nullptr, h_bad = 0;
    COLA_TRY(sc.get(bad, 1));
    COLA_CUDA(cudaMemsetAsync(bad, 0xff, sizeof(*bad), sc.st));
    check_coo_kernel<<<grid_stride_blocks(n), 256, 0, sc.st>>>(row, col, n, N, NC, bad);
    t_launches++;
    COLA_CUDA(cudaGetLastError());
    COLA_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(h_bad), cudaMemcpyDeviceToHost, sc.st));
    COLA_CUDA(cudaStreamSynchronize(sc.st));
    if (h_bad != ULLONG_MAX) {
        int32_t r = 0, c = 0;
        cudaMemcpy(&r, row + h_bad, 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(&c, col + h_bad, 4, cudaMemcpyDeviceToHost);
        return fail(COLA_ERROR_INVALID_ARGUMENT, "%s: entry %llu (%d, %d) outside %d x %d", who, h_bad, r, c, N, NC);
    }
    return COLA_SUCCESS;
}

// Stable LSD radix sort of (key, id) pairs by the low key_bits bits of the
// keys: on return k0/v0 point at the sorted pairs, k1/v1 at the other buffers.
static cola_status radix_sort_pairs(uint64_t *&k0, uint32_t *&v0, uint64_t *&k1, uint32_t *&v1, int64_t n,
                                    int key_bits, uint32_t *hist, uint32_t *d_total, Scratch &sc)
{
    const int64_t ntiles = (n + kTile - 1) / kTile;
    for (int shift = 0; shift < key_bits; shift += kDigitBits) {
        radix_hist_kernel<<<(unsigned)ntiles, kThreads, 0, sc.st>>>(k0, n, shift, ntiles, hist);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
        COLA_TRY(exclusive_scan(ArrayF{hist}, ntiles * kBins, hist, d_total, nullptr, sc));
        radix_scatter_kernel<<<(unsigned)ntiles, kThreads, 0, sc.st>>>(k0, v0, k1, v1, n, shift, ntiles, hist);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
        std::swap(k0, k1);
        std::swap(v0, v1);
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
    COLA_TRY(radix_sort_pairs(k0, v0, k1, v1, nnz, key_bits, hist, d_total, sc));
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

// The row view of cola_graph_upload, built from a device COO without the
// host: entries sorted by (row, col) with duplicates merged (values summed in
// input order), row pointers, hub segments and row-block tasks.  The result is
// identical to the upload of the same COO's partitions, array for array.
// NC > 0: a rectangular N x NC matrix (rows N, columns NC >= N), as one
// partition's rows over the global columns are.
static cola_status graph_build_device(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col,
                                      const float *val, int32_t nparts, const cola_upload_opts *opts, cudaStream_t st,
                                      cola_graph *&out, int32_t NC = -1, const char *who = "cola_graph_build_device")
{
    if (NC < 0)
        NC = N;
    COLA_REQUIRE(NC >= N, COLA_ERROR_INVALID_ARGUMENT, "%s: %d columns < %d rows", who, NC, N);
    COLA_REQUIRE(N >= 0 && nnz >= 0 && nparts >= 1, COLA_ERROR_INVALID_ARGUMENT, "%s: N=%d nnz=%lld nparts=%d", who,
                 N, (long long)nnz, nparts);
    COLA_REQUIRE(nnz == 0 || (row && col), COLA_ERROR_INVALID_ARGUMENT, "%s: null COO arrays", who);
    COLA_REQUIRE(nnz < (int64_t)UINT32_MAX, COLA_ERROR_UNSUPPORTED, "%s: nnz >= 2^32", who);
    COLA_REQUIRE(!(opts && opts->no_row_view), COLA_ERROR_INVALID_ARGUMENT,
                 "%s: a graph built on the device is its row view", who);
    COLA_REQUIRE(!(opts && opts->group_size > 0 && opts->group_size != nparts), COLA_ERROR_UNSUPPORTED,
                 "%s: the pipelined schedule needs the split blocks (cola_graph_upload)", who);
    const RowViewParams rp = row_view_params(nnz, opts);
    const int64_t thr = rp.hub_threshold, seg = rp.hub_segment, te = rp.task_entries;
    const int64_t npp = ((int64_t)N + nparts - 1) / nparts;
    const int cb = bits_for(NC > 0 ? (uint64_t)NC - 1 : 0);  // column bits; rows (< N <= NC) fit in as many

    std::unique_ptr<cola_graph, void (*)(cola_graph *)> g(new (std::nothrow) cola_graph(), graph_release);
    COLA_REQUIRE(g, COLA_ERROR_OUT_OF_MEMORY, "%s: host allocation failed", who);
    COLA_CUDA(cudaGetDevice(&g->device));
    g->N = N;
    g->P = nparts;
    g->npp = (int32_t)npp;
    g->gs = nparts;
    g->nstages = 1;
    g->has_split = false;
    g->hub_threshold = (int32_t)thr;
    g->hub_segment = (int32_t)seg;
    g->task_entries = (int32_t)te;

    Scratch sc(st);
    {
        const size_t n = (size_t)nnz, a = 256;
        const int64_t ntiles = (nnz + kTile - 1) / kTile;
        const size_t rows = (size_t)N + 1;
        const size_t scan_blocks = (size_t)((std::max<int64_t>(std::max<int64_t>(ntiles * kBins, nnz), N + 1) +
                                             kScanTile - 1) / kScanTile) + 1;
        // sort keys and ids (x2), digit counts, unique positions, values and
        // columns, row pointers, hub / segment / run positions, run task
        // counts and offsets, small values, the scans' block sums
        const size_t bytes = 2 * (8 * n + a) + 2 * (4 * n + a) + (4 * (size_t)ntiles * kBins + a) + 3 * (4 * n + a) +
                             (8 * rows + a) + 5 * (4 * rows + a) + 4 * a + 24 * (4 * scan_blocks + a);
        COLA_TRY(sc.reserve(bytes));
    }
    if (nnz > 0)
        COLA_TRY(check_range(row, col, nnz, N, sc, who, NC));
    uint32_t *d_total = nullptr;
    COLA_TRY(sc.get(d_total, 1));
    uint64_t *ukey = nullptr;
    float *uval = nullptr;
    uint32_t U = 0;
    if (nnz > 0) {
        uint64_t *k0 = nullptr, *k1 = nullptr;
        uint32_t *v0 = nullptr, *v1 = nullptr, *hist = nullptr, *upos = nullptr;
        const int64_t ntiles = (nnz + kTile - 1) / kTile;
        COLA_TRY(sc.get(k0, nnz));
        COLA_TRY(sc.get(k1, nnz));
        COLA_TRY(sc.get(v0, nnz));
        COLA_TRY(sc.get(v1, nnz));
        COLA_TRY(sc.get(hist, ntiles * kBins));
        make_row_keys_kernel<<<grid_stride_blocks(nnz), 256, 0, st>>>(row, col, nnz, cb, k0, v0);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
        COLA_TRY(radix_sort_pairs(k0, v0, k1, v1, nnz, 2 * cb, hist, d_total, sc));
        COLA_TRY(sc.get(upos, nnz));
        COLA_TRY(exclusive_scan(KeyStartF{k0, 0}, nnz, upos, d_total, &U, sc));
        COLA_TRY(sc.get(uval, U));
        ukey = k1;
        dedupe_kernel<<<grid_stride_blocks(nnz), 256, 0, st>>>(k0, v0, val, nnz, upos, ukey, uval);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
    }
    // row pointers and columns
    int64_t *rv_ptr = nullptr;
    int32_t *rv_col = nullptr;
    COLA_TRY(sc.get(rv_ptr, (int64_t)N + 1));
    COLA_TRY(sc.get(rv_col, U));
    if (U > 0) {
        row_ptr_kernel<<<grid_stride_blocks((int64_t)N + 1), 256, 0, st>>>(ukey, U, cb, N, rv_ptr);
        row_cols_kernel<<<grid_stride_blocks(U), 256, 0, st>>>(ukey, U, cb >= 64 ? ~0ull : (1ull << cb) - 1, rv_col);
        t_launches += 2;
    } else {
        COLA_CUDA(cudaMemsetAsync(rv_ptr, 0, ((size_t)N + 1) * 8, st));
    }
    COLA_CUDA(cudaGetLastError());
    // hub rows and their segments; runs of non-hub rows and their tasks
    uint32_t nhub = 0, nseg = 0, nrun = 0, ntask = 0;
    uint32_t *hubpos = nullptr, *segoff = nullptr, *runpos = nullptr, *cnt = nullptr, *toff = nullptr;
    COLA_TRY(sc.get(hubpos, N));
    COLA_TRY(sc.get(segoff, N));
    COLA_TRY(sc.get(runpos, N));
    COLA_TRY(exclusive_scan(HubF{rv_ptr, thr}, N, hubpos, d_total, &nhub, sc));
    COLA_TRY(exclusive_scan(SegCountF{rv_ptr, thr, seg}, N, segoff, d_total, &nseg, sc));
    COLA_TRY(exclusive_scan(RunStartF{rv_ptr, thr}, N, runpos, d_total, &nrun, sc));
    COLA_TRY(sc.get(cnt, nrun));
    COLA_TRY(sc.get(toff, nrun));
    if (nrun > 0) {
        run_tasks_kernel<<<grid_stride_blocks(N), 256, 0, st>>>(rv_ptr, N, thr, te, runpos, cnt, nullptr, nullptr,
                                                                nullptr);
        t_launches++;
        COLA_CUDA(cudaGetLastError());
        COLA_TRY(exclusive_scan(ArrayF{cnt}, nrun, toff, d_total, &ntask, sc));
    }
    // nnz in the partitions' local blocks
    unsigned long long *d_local = nullptr, h_local = 0;
    COLA_TRY(sc.get(d_local, 1));
    COLA_CUDA(cudaMemsetAsync(d_local, 0, sizeof(*d_local), st));
    if (U > 0) {
        count_local_kernel<<<grid_stride_blocks(U), 256, 0, st>>>(ukey, U, cb, (uint32_t)std::max<int64_t>(npp, 1),
                                                                  d_local);
        t_launches++;
    }
    COLA_CUDA(cudaMemcpyAsync(&h_local, d_local, sizeof(h_local), cudaMemcpyDeviceToHost, st));

    // the graph's own arena, in the order and alignment of the host upload
    size_t total = 0;
    auto place = [&](size_t bytes) {
        const size_t o = total;
        total += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_ptr = place(((size_t)N + 1) * 8), o_col = place((size_t)U * 4), o_val = place((size_t)U * 4);
    const size_t o_srow = place((size_t)nseg * 4), o_sbeg = place((size_t)nseg * 8);
    const size_t o_hrow = place((size_t)nhub * 4), o_hseg = place(((size_t)nhub + 1) * 8);
    const size_t o_trb = place((size_t)ntask * 4), o_tre = place((size_t)ntask * 4);
    const size_t qbytes = (dev::kMaxItemQueues + 1) * sizeof(unsigned int), o_q = place(qbytes);
    total = std::max<size_t>(total, 256);
    COLA_CUDA(cudaMalloc(&g->dmem, total));
    g->dbytes = total;
    char *base = static_cast<char *>(g->dmem);
    COLA_CUDA(cudaMemcpyAsync(base + o_ptr, rv_ptr, ((size_t)N + 1) * 8, cudaMemcpyDeviceToDevice, st));
    COLA_CUDA(cudaMemsetAsync(base + o_q, 0, qbytes, st));
    if (U > 0) {
        COLA_CUDA(cudaMemcpyAsync(base + o_col, rv_col, (size_t)U * 4, cudaMemcpyDeviceToDevice, st));
        COLA_CUDA(cudaMemcpyAsync(base + o_val, uval, (size_t)U * 4, cudaMemcpyDeviceToDevice, st));
    }
    const int64_t *ptr_final = reinterpret_cast<const int64_t *>(base + o_ptr);
    if (N > 0) {
        hub_segments_kernel<<<grid_stride_blocks(N), 256, 0, st>>>(
            ptr_final, N, thr, seg, hubpos, segoff, nhub, nseg, reinterpret_cast<int32_t *>(base + o_hrow),
            reinterpret_cast<int64_t *>(base + o_hseg), reinterpret_cast<int32_t *>(base + o_srow),
            reinterpret_cast<int64_t *>(base + o_sbeg));
        t_launches++;
        if (nrun > 0) {
            run_tasks_kernel<<<grid_stride_blocks(N), 256, 0, st>>>(ptr_final, N, thr, te, runpos, nullptr, toff,
                                                                    reinterpret_cast<int32_t *>(base + o_trb),
                                                                    reinterpret_cast<int32_t *>(base + o_tre));
            t_launches++;
        }
        COLA_CUDA(cudaGetLastError());
    } else {
        const int64_t zero = 0;
        COLA_CUDA(cudaMemcpyAsync(base + o_hseg, &zero, 8, cudaMemcpyHostToDevice, st));
    }
    COLA_CUDA(cudaStreamSynchronize(st));
    g->has_rows = true;
    g->rv_ptr = ptr_final;
    g->rv_col = reinterpret_cast<const int32_t *>(base + o_col);
    g->rv_val = reinterpret_cast<const float *>(base + o_val);
    g->seg_row = reinterpret_cast<const int32_t *>(base + o_srow);
    g->seg_beg = reinterpret_cast<const int64_t *>(base + o_sbeg);
    g->hub_row = reinterpret_cast<const int32_t *>(base + o_hrow);
    g->hub_seg = reinterpret_cast<const int64_t *>(base + o_hseg);
    g->task_rb = reinterpret_cast<const int32_t *>(base + o_trb);
    g->task_re = reinterpret_cast<const int32_t *>(base + o_tre);
    g->item_queue = reinterpret_cast<unsigned int *>(base + o_q);
    g->nseg = nseg;
    g->nhub = nhub;
    g->ntask = ntask;
    g->nnz_l = (int64_t)h_local;
    g->nnz_r = (int64_t)U - (int64_t)h_local;
    out = g.release();
    return COLA_SUCCESS;
}

}  // namespace pg

cola_status graph_build_device_rect(int32_t nrows, int32_t ncols, int64_t nnz, const int32_t *row, const int32_t *col,
                                    const float *val, const cola_upload_opts *opts, cudaStream_t st, cola_graph *&out,
                                    const char *who)
{
    return pg::graph_build_device(nrows, nnz, row, col, val, 1, opts, st, out, ncols, who);
}

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

cola_status cola_graph_build_device(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                    const float *val, int32_t nparts, const cola_upload_opts *opts,
                                    cudaStream_t stream, cola_graph **out)
{
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "cola_graph_build_device: out is NULL");
    *out = nullptr;
    clear_error();
    cola_graph *g = nullptr;
    COLA_TRY(pg::graph_build_device(num_nodes, nnz, row, col, val, nparts, opts, stream, g));
    *out = g;
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
