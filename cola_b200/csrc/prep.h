// Host-side partition structures and preprocessing steps (see prep.cpp).
#pragma once
#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "cola_spmm.h"

namespace cola {

// Allocator whose resize() leaves new elements uninitialised: partition
// arrays are always written in full after sizing, so large ones are not
// zero-filled first.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept
    {
    }
    template <class U>
    void construct(U *p) noexcept
    {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...a)
    {
        ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
    }
};
using ivec = std::vector<int32_t, NoInitAlloc<int32_t>>;
using fvec = std::vector<float, NoInitAlloc<float>>;

// One virtual partition as prep_torch_par.py:24-79 writes it, plus values.
struct PartHost {
    int32_t part = 0, row_lb = 0, row_ub = 0;
    ivec l_rowPtr, l_colIdx, l_rowIdx;  // local CSR (col % npp), non-empty rows
    fvec l_val;
    ivec r_colPtr, r_rowIdx, r_colIdx;  // remote CSC (global cols), non-empty cols
    fvec r_val;
};

// Tables of src/distSpMM_ppl_batch.cu:101-193 for one PE.
struct StageTables {
    int32_t nstages = 1;
    std::vector<int32_t> local_offset, remote_offset, put_offset;  // 2*nstages each
    std::vector<std::vector<int32_t>> idx_ppl;                      // stages 1..nstages-1
    std::vector<std::vector<int32_t>> put_colIdx;                   // stages 0..nstages-2
};

cola_status partition_build(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col, const float *val,
                            int32_t nparts, cola_partition_set *&out);
cola_status nnz_split(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                      std::vector<int32_t> &target, std::vector<int32_t> &ptr);
cola_status stage_tables(int32_t me, int32_t nranks, int32_t gs, int32_t N, const int32_t *zr, int64_t nrc,
                         int64_t nchunks_l, const int32_t *wg_cols, const int64_t *wg_off, StageTables &t);
cola_status workgroup_cols(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col, int32_t nparts,
                           int32_t gs, int32_t stage, std::vector<int32_t> &out);
cola_status validate_partition(const cola_partition_set &s, const PartHost &P);

// The row-major view the default schedule runs on: for every output row its
// entries in ascending global column order (the partition's remote columns
// left of its own block, its local entries, the remote columns right of it),
// rows longer than hub_threshold cut into hub_segment-entry segments, and the
// other rows packed greedily into tasks of about task_entries (a row costs its
// entries + 2; a task never spans a hub row).
struct RowView {
    std::vector<int64_t> ptr;  // N + 1
    std::vector<int32_t> col;
    std::vector<float> val;
    std::vector<int32_t> seg_row, hub_row;  // segment -> its row; hub -> its row
    std::vector<int64_t> seg_beg, hub_seg;  // segment -> first entry; hub -> first segment (nhub + 1)
    std::vector<int32_t> task_rb, task_re;  // task -> rows [rb, re)
};
cola_status build_row_view(const cola_partition_set &s, int64_t hub_threshold, int64_t hub_segment,
                           int64_t task_entries, RowView &rv);

}  // namespace cola

struct cola_partition_set {
    int32_t num_nodes = 0, nparts = 0, npp = 0;
    std::vector<cola::PartHost> parts;
};
