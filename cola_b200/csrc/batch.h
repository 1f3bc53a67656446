// Internal: the batched launch shared by the batched form and the server.
#pragma once
#include "graph.h"
#include "spmm_batch.cuh"

namespace cola {

// One batched launch over a device table of graph descriptors (item0 / hub0
// prefixes filled in by the caller).
struct BatchLaunch {
    const dev::BatchGraph *desc;
    int ngraphs;
    int64_t total_items, total_hub;
    cola_dtype xdt, ydt;
    int unroll, grid_pct, accumulate;
    int blocks_per_sm;  // resident blocks per SM the streaming kernel is compiled for: 3 or 4
    // dev::kMaxItemQueues + 1 counters, zero between launches (kBatchQueueBytes
    // at the end of the descriptor table's allocation), or NULL for the static
    // assignment; launches that share counters must not overlap
    unsigned int *queue;
};

// Bytes of work-item counters a descriptor table's allocation carries after
// the descriptors (at a 256-byte aligned offset: batch_queue_offset).
constexpr size_t kBatchQueueBytes = 512;
inline size_t batch_queue_offset(size_t desc_bytes) { return (desc_bytes + 255) & ~(size_t)255; }

cola_status launch_batch(const BatchLaunch &L, cudaStream_t st);

// Descriptor of graph g with these operands and hub workspace (item0 / hub0
// left zero).
void fill_batch_graph(dev::BatchGraph &d, const cola_graph *g, const void *X, int64_t ldx, void *Y, int64_t ldy,
                      int32_t K, cola_dtype xdt, float *ws);

}  // namespace cola
