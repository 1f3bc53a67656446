// Builds the row-major view (build_row_view in cola_b200/csrc/prep.cpp, the
// function cola_graph_upload runs) from a COO on the CPU, for
// tests/test_row_view.py.
//
//   row_view_main <in> <out>
//
// in:  int32 N, int32 P, int64 nnz, int64 hub_threshold, int64 hub_segment,
//      int64 task_entries, then int32 row[nnz], int32 col[nnz], float val[nnz].
// out: per array (ptr, col, val, seg_row, seg_beg, hub_row, hub_seg, task_rb,
//      task_re) an int64 element count followed by the elements.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "prep.h"

template <typename T>
static bool read_n(FILE *f, T *p, size_t n)
{
    return std::fread(p, sizeof(T), n, f) == n;
}

template <typename V>
static void write_vec(FILE *f, const V &v)
{
    const int64_t n = (int64_t)v.size();
    std::fwrite(&n, 8, 1, f);
    if (n)
        std::fwrite(v.data(), sizeof(v[0]), (size_t)n, f);
}

int main(int argc, char **argv)
{
    if (argc < 3)
        return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f)
        return 2;
    int32_t N = 0, P = 0;
    int64_t nnz = 0, thr = 0, seg = 0, te = 0;
    if (!read_n(f, &N, 1) || !read_n(f, &P, 1) || !read_n(f, &nnz, 1) || !read_n(f, &thr, 1) ||
        !read_n(f, &seg, 1) || !read_n(f, &te, 1))
        return 2;
    std::vector<int32_t> row((size_t)nnz), col((size_t)nnz);
    std::vector<float> val((size_t)nnz);
    if (!read_n(f, row.data(), (size_t)nnz) || !read_n(f, col.data(), (size_t)nnz) ||
        !read_n(f, val.data(), (size_t)nnz))
        return 2;
    std::fclose(f);
    cola_partition_set *ps = nullptr;
    if (cola::partition_build(N, nnz, row.data(), col.data(), val.data(), P, ps) != COLA_SUCCESS)
        return 3;
    cola::RowView rv;
    const cola_status st = cola::build_row_view(*ps, thr, seg, te, rv);
    delete ps;
    if (st != COLA_SUCCESS)
        return 4;
    FILE *o = std::fopen(argv[2], "wb");
    if (!o)
        return 2;
    write_vec(o, rv.ptr);
    write_vec(o, rv.col);
    write_vec(o, rv.val);
    write_vec(o, rv.seg_row);
    write_vec(o, rv.seg_beg);
    write_vec(o, rv.hub_row);
    write_vec(o, rv.hub_seg);
    write_vec(o, rv.task_rb);
    write_vec(o, rv.task_re);
    return std::fclose(o) == 0 ? 0 : 2;
}
