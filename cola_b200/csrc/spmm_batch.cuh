// Batched form: many graphs, each with its own X, Y and feature width, in one
// persistent launch.  Work items of all graphs are concatenated (graph g owns
// items [item0, item0 + nseg + ntask)); a warp finds its graph by advancing
// through the descriptor table (its items only increase) and runs the item with
// the lane geometry of that graph's width.  With DYN the items are drawn from a
// counter (one ahead, as in the single-graph kernel): items of a K = 512 graph
// cost 30 times those of a K = 16 one, so a static share leaves warps idle.
#pragma once
#include "spmm_rows.cuh"

namespace cola {
namespace dev {

struct BatchGraph {
    BlockArgs ba;  // row view, tasks, hub segments, workspace of this graph
    const void *X;
    int64_t ldx;
    void *Y;
    int64_t ldy;
    int32_t K;
    int32_t lg;    // lanes per row tile (8, 16 or 32): batch_lane_width(K, E)
    int64_t item0; // first work item of this graph in the launch
    int64_t hub0;  // first combine item (hub x 128-feature tile) of this graph
    const int32_t *hub_row;
    const int64_t *hub_seg;
    int64_t nhub;
};

// The lane-group width is a per-graph value read at run time (one kernel
// instantiation for all graphs): lg = 8, 16 or 32 lanes cover one row tile of
// lg 16-byte vectors, the warp's 32/lg groups take interleaved entries, and
// rows wider than one tile are walked tile by tile.
inline int batch_lane_width(int K, int E)
{
    int lg = 8;
    while (lg < 32 && lg * E < K)
        lg <<= 1;
    return lg;
}

template <typename TR, typename TY, int UNROLL, int MINB, bool DYN = false>
__global__ void __launch_bounds__(kThreads, MINB) batch_rowblock_kernel(const BatchGraph *__restrict__ gs, int ng,
                                                                     int64_t total, int accumulate,
                                                                     unsigned int *queue)
{
    using T = typename ElemOf<TR>::T;
    __shared__ int2 s_ent[kWarpsPerBlock][32];
    int2 *ent = s_ent[threadIdx.x >> 5];
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    const int lane = threadIdx.x & 31;
    int gi = 0;
    int64_t it = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if constexpr (DYN) {
        unsigned int t = 0;
        if (lane == 0)
            t = atomicAdd(queue, 1u);
        it = (int64_t)__shfl_sync(kFull, t, 0);
    }
    while (it < total) {
        unsigned int next_it = 0;
        if constexpr (DYN) {
            if (lane == 0)
                next_it = atomicAdd(queue, 1u);
        }
        while (gi + 1 < ng && it >= gs[gi + 1].item0)
            gi++;
        const BatchGraph &bg = gs[gi];
        const int64_t li = it - bg.item0;
        const int W = bg.lg * TR::E;  // features per tile
        for (int k0 = 0; k0 < bg.K; k0 += W)
            rowblock_items<TR, TY, 0, 1, UNROLL, true, const BlockArgs &>(
                bg.ba, li, 1, li + 1, static_cast<const T *>(bg.X), bg.ldx, static_cast<TY *>(bg.Y), bg.ldy, bg.K,
                accumulate, k0, ent, bg.lg);
        if constexpr (DYN)
            it = (int64_t)__shfl_sync(kFull, next_it, 0);
        else
            it += nwarps;
    }
    if constexpr (DYN)
        item_queue_release(queue);
}

template <typename TY, int UNROLL>
__global__ void __launch_bounds__(kThreads) batch_hub_combine_kernel(const BatchGraph *__restrict__ gs, int ng,
                                                                    int64_t total, int accumulate)
{
    const int64_t nwarps = (int64_t)gridDim.x * kWarpsPerBlock;
    int gi = 0;
    for (int64_t w = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); w < total; w += nwarps) {
        while (gi + 1 < ng && w >= gs[gi + 1].hub0)
            gi++;
        const BatchGraph &bg = gs[gi];
        const int tiles = (bg.K + 127) / 128;
        const int64_t lw = w - bg.hub0;
        hub_combine_item<TY, UNROLL>(bg.hub_row, bg.hub_seg, lw / tiles, (int)(lw % tiles), bg.ba.ws, bg.ba.ld_ws,
                                     static_cast<TY *>(bg.Y), bg.ldy, bg.K, accumulate);
    }
}

}  // namespace dev
}  // namespace cola
