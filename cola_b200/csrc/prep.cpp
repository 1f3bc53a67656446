// Host preprocessing of the partitioned SpMM: row partitioning into local CSR
// + compacted remote CSC blocks, nnz_split chunking, the pipelined schedule's
// stage tables, the reference's .bin on-disk format and a seeded R-MAT
// generator.  Outputs are bit-identical to the reference's preprocessing
// (prep_torch_par.py, prep_torch_ppl.py, include/dist_spmm_ppl_batch.cuh:29-56,
// src/distSpMM_ppl_batch.cu:101-193).
#include <parallel/algorithm>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <omp.h>
#include <sys/stat.h>

#include "common.h"
#include "prep.h"

namespace cola {

static thread_local std::string g_last_error;

cola_status fail(cola_status s, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

void clear_error() { g_last_error.clear(); }

// Stable counting sort of `idx` by key(idx) in [0, range).
template <typename KeyFn>
static void counting_sort(std::vector<uint32_t> &idx, std::vector<uint32_t> &tmp, int64_t range, KeyFn key)
{
    std::vector<int64_t> cnt((size_t)range + 1, 0);
    for (uint32_t i : idx)
        cnt[(size_t)key(i) + 1]++;
    for (int64_t k = 0; k < range; k++)
        cnt[(size_t)k + 1] += cnt[(size_t)k];
    tmp.resize(idx.size());
    for (uint32_t i : idx)
        tmp[(size_t)cnt[(size_t)key(i)]++] = i;
    idx.swap(tmp);
}

// One partition of prep_torch_par.py:24-79 (row_partition).
//  rows [lb, ub) with lb = r*npp, ub = min((r+1)*npp, N)      (:34-36)
//  local: cols in [r*npp, (r+1)*npp), CSR over (row-lb, col%npp),
//         sorted + merged by tocsr() (:40-47); rowPtr = unique(indptr) (:51-52);
//         rowIdx = unique(local rows) (:48)
//  remote: other cols, CSC over global cols (:60-66); colPtr = unique(indptr)
//         (:72-73); colIdx = unique(remote cols) (:67-68)
// Duplicate entries merge into one, values summed in input order.
static void build_partition(PartHost &P, int32_t N, int64_t npp, int64_t nnz, const int32_t *row,
                            const int32_t *col, const float *val)
{
    const int64_t lb = P.row_lb, ub = P.row_ub;
    const int64_t clb = (int64_t)P.part * npp, cub = clb + npp;
    std::vector<uint32_t> li, ri, tmp;
    for (int64_t i = 0; i < nnz; i++) {
        int64_t r = row[i];
        if (r < lb || r >= ub)
            continue;
        int64_t c = col[i];
        if (c >= clb && c < cub)
            li.push_back((uint32_t)i);
        else
            ri.push_back((uint32_t)i);
    }
    // local: sort by (row, col%npp): LSD = col then row
    counting_sort(li, tmp, npp, [&](uint32_t i) { return (int64_t)col[i] - clb; });
    counting_sort(li, tmp, std::max<int64_t>(ub - lb, 1), [&](uint32_t i) { return (int64_t)row[i] - lb; });
    P.l_rowPtr.assign(1, 0);
    for (size_t k = 0; k < li.size(); k++) {
        uint32_t i = li[k];
        float v = val ? val[i] : 1.0f;
        int32_t lr = (int32_t)(row[i] - lb), lc = (int32_t)(col[i] - clb);
        if (k > 0) {
            uint32_t j = li[k - 1];
            if (row[j] == row[i] && col[j] == col[i]) {
                P.l_val.back() += v;
                continue;
            }
            if (row[j] != row[i])
                P.l_rowPtr.push_back((int32_t)P.l_colIdx.size());
        }
        if (k == 0 || row[li[k - 1]] != row[i])
            P.l_rowIdx.push_back(lr);
        P.l_colIdx.push_back(lc);
        P.l_val.push_back(v);
    }
    if (!li.empty())
        P.l_rowPtr.push_back((int32_t)P.l_colIdx.size());
    // remote: sort by (col, row): LSD = row then col
    counting_sort(ri, tmp, std::max<int64_t>(ub - lb, 1), [&](uint32_t i) { return (int64_t)row[i] - lb; });
    counting_sort(ri, tmp, std::max<int64_t>(N, 1), [&](uint32_t i) { return (int64_t)col[i]; });
    P.r_colPtr.assign(1, 0);
    for (size_t k = 0; k < ri.size(); k++) {
        uint32_t i = ri[k];
        float v = val ? val[i] : 1.0f;
        if (k > 0) {
            uint32_t j = ri[k - 1];
            if (row[j] == row[i] && col[j] == col[i]) {
                P.r_val.back() += v;
                continue;
            }
            if (col[j] != col[i])
                P.r_colPtr.push_back((int32_t)P.r_rowIdx.size());
        }
        if (k == 0 || col[ri[k - 1]] != col[i])
            P.r_colIdx.push_back(col[i]);
        P.r_rowIdx.push_back((int32_t)(row[i] - lb));
        P.r_val.push_back(v);
    }
    if (!ri.empty())
        P.r_colPtr.push_back((int32_t)P.r_rowIdx.size());
}

cola_status partition_build(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col, const float *val,
                            int32_t nparts, cola_partition_set *&out)
{
    COLA_REQUIRE(N >= 0 && nnz >= 0 && nparts >= 1, COLA_ERROR_INVALID_ARGUMENT,
                 "partition_build: N=%d nnz=%lld nparts=%d", N, (long long)nnz, nparts);
    COLA_REQUIRE(nnz == 0 || (row && col), COLA_ERROR_INVALID_ARGUMENT, "partition_build: null COO arrays");
    COLA_REQUIRE(nnz < (int64_t)UINT32_MAX, COLA_ERROR_UNSUPPORTED, "partition_build: nnz >= 2^32");
    for (int64_t i = 0; i < nnz; i++)
        COLA_REQUIRE(row[i] >= 0 && row[i] < N && col[i] >= 0 && col[i] < N, COLA_ERROR_INVALID_ARGUMENT,
                     "partition_build: entry %lld (%d, %d) outside %d x %d", (long long)i, row[i], col[i], N, N);
    std::unique_ptr<cola_partition_set> s(new (std::nothrow) cola_partition_set());
    COLA_REQUIRE(s, COLA_ERROR_OUT_OF_MEMORY, "partition_build: host allocation failed");
    s->num_nodes = N;
    s->nparts = nparts;
    const int64_t npp = ((int64_t)N + nparts - 1) / nparts;  // prep_torch_par.py:31
    s->npp = (int32_t)npp;
    s->parts.resize((size_t)nparts);
    for (int32_t r = 0; r < nparts; r++) {
        PartHost &P = s->parts[(size_t)r];
        P.part = r;
        P.row_lb = (int32_t)std::min<int64_t>((int64_t)r * npp, N);
        P.row_ub = (int32_t)std::min<int64_t>((int64_t)(r + 1) * npp, N);
    }
    bool oom = false;
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t r = 0; r < nparts; r++) {
        try {
            build_partition(s->parts[(size_t)r], N, npp, nnz, row, col, val);
        } catch (const std::bad_alloc &) {
#pragma omp atomic write
            oom = true;
        }
    }
    COLA_REQUIRE(!oom, COLA_ERROR_OUT_OF_MEMORY, "partition_build: host allocation failed");
    out = s.release();
    return COLA_SUCCESS;
}

// include/dist_spmm_ppl_batch.cuh:29-56 (nnz_split).
cola_status nnz_split(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                      std::vector<int32_t> &target, std::vector<int32_t> &ptr)
{
    target.clear();
    ptr.clear();
    if (nrows == 0)
        return COLA_SUCCESS;  // :32-33, both outputs stay empty
    const int avg = (int)((uint64_t)nnz / (uint64_t)nrows);  // :34
    const int gran = (avg + 32 - 1) / 32 * 32;                // :35
    COLA_REQUIRE(gran > 0, COLA_ERROR_INVALID_ARGUMENT,
                 "nnz_split: %lld entries over %lld rows gives a zero chunk size", (long long)nnz, (long long)nrows);
    ptr.push_back(0);
    for (int64_t i = 0; i < nrows; i++) {
        int64_t lb = rowPtr[i], hb = rowPtr[i + 1];
        for (; lb < hb; lb += gran) {
            target.push_back(rowIdx[i]);
            ptr.push_back((int32_t)(lb + gran > hb ? hb : lb + gran));
        }
    }
    return COLA_SUCCESS;
}

static int64_t lower_bound_i32(const int32_t *a, int64_t n, int64_t v)
{
    return std::lower_bound(a, a + n, v, [](int32_t x, int64_t y) { return (int64_t)x < y; }) - a;
}

// src/distSpMM_ppl_batch.cu:101-193.
cola_status stage_tables(int32_t me, int32_t nranks, int32_t gs, int32_t N, const int32_t *zr, int64_t nrc,
                         int64_t nchunks_l, const int32_t *wg_cols, const int64_t *wg_off, StageTables &t)
{
    COLA_REQUIRE(nranks >= 1 && gs >= 1 && nranks % gs == 0 && me >= 0 && me < nranks,
                 COLA_ERROR_INVALID_ARGUMENT, "stage_tables: me=%d nranks=%d group_size=%d", me, nranks, gs);
    const int32_t nstages = nranks / gs;
    COLA_REQUIRE(nstages == 1 || (wg_cols && wg_off), COLA_ERROR_INVALID_ARGUMENT,
                 "stage_tables: work-group column lists are required when group_size < nranks");
    const int64_t npp = ((int64_t)N + nranks - 1) / nranks;  // .cu:74
    t.nstages = nstages;
    t.local_offset.assign((size_t)2 * nstages, 0);
    t.remote_offset.assign((size_t)2 * nstages, 0);
    t.put_offset.assign((size_t)2 * nstages, 0);
    t.idx_ppl.assign((size_t)std::max(nstages - 1, 0), {});
    t.put_colIdx.assign((size_t)std::max(nstages - 1, 0), {});
    const int32_t *mywg = nstages > 1 ? wg_cols + wg_off[me / gs] : nullptr;
    const int64_t mywg_n = nstages > 1 ? wg_off[me / gs + 1] - wg_off[me / gs] : 0;
    for (int32_t i = 0; i < nstages; i++) {
        const int32_t next_pos = (me + gs * i) % nranks;  // :109
        const int32_t group_id = next_pos / gs;
        const int64_t local_lb = (int64_t)next_pos * npp;
        const int64_t local_ub = std::min<int64_t>(N, local_lb + npp);
        const int64_t remote_lb = (int64_t)group_id * gs * npp;
        const int64_t remote_ub = std::min<int64_t>(N, remote_lb + (int64_t)gs * npp);
        if (i == 0) {  // :117-122
            t.local_offset[0] = 0;
            t.local_offset[1] = (int32_t)nchunks_l;
        } else {  // :124-130
            t.local_offset[2 * i] = (int32_t)lower_bound_i32(zr, nrc, local_lb);
            t.local_offset[2 * i + 1] = (int32_t)lower_bound_i32(zr, nrc, local_ub);
        }
        t.remote_offset[2 * i] = (int32_t)lower_bound_i32(zr, nrc, remote_lb);  // :132-135
        t.remote_offset[2 * i + 1] = (int32_t)lower_bound_i32(zr, nrc, remote_ub);
        if (i != 0) {  // :137-169
            std::vector<int64_t> slb((size_t)gs), sub((size_t)gs), pos((size_t)gs, 0);
            for (int32_t j = 0; j < gs; j++) {
                const int64_t src_pe = j + (int64_t)group_id * gs;
                const int64_t lb = src_pe * npp, ub = std::min<int64_t>(N, lb + npp);
                slb[(size_t)j] = lower_bound_i32(mywg, mywg_n, lb);
                sub[(size_t)j] = lower_bound_i32(mywg, mywg_n, ub);
            }
            auto &lst = t.idx_ppl[(size_t)i - 1];
            for (int64_t j = t.remote_offset[2 * i]; j < t.remote_offset[2 * i + 1]; j++) {
                const int32_t cur_col = zr[j];
                const int32_t rg = (int32_t)((cur_col / npp) % gs);
                int64_t k = pos[(size_t)rg];
                const int64_t n = sub[(size_t)rg] - slb[(size_t)rg];
                while (k < n) {
                    if (mywg[slb[(size_t)rg] + k] == cur_col) {
                        lst.push_back((int32_t)k);
                        pos[(size_t)rg] = k;
                        break;
                    }
                    k++;
                }
            }
        }
    }
    for (int32_t i = 0; i < nstages - 1; i++) {  // :173-193
        int32_t target_pe = (me - (i + 1) * gs) % nranks;
        target_pe = (target_pe + nranks) % nranks;
        const int32_t tw = target_pe / gs;
        const int32_t *tl = wg_cols + wg_off[tw];
        const int64_t tn = wg_off[tw + 1] - wg_off[tw];
        const int64_t plb = (int64_t)me * npp, pub = std::min<int64_t>(N, plb + npp);
        const int64_t a = lower_bound_i32(tl, tn, plb), b = lower_bound_i32(tl, tn, pub);
        t.put_offset[2 * i] = (int32_t)a;
        t.put_offset[2 * i + 1] = (int32_t)b;
        t.put_colIdx[(size_t)i].assign(tl + a, tl + b);
    }
    return COLA_SUCCESS;
}

// prep_torch_ppl.py:24-49.
cola_status workgroup_cols(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col, int32_t nparts,
                           int32_t gs, int32_t stage, std::vector<int32_t> &out)
{
    COLA_REQUIRE(nparts >= 1 && gs >= 1 && stage >= 0, COLA_ERROR_INVALID_ARGUMENT,
                 "workgroup_cols: nparts=%d group_size=%d stage=%d", nparts, gs, stage);
    const int64_t npp = ((int64_t)N + nparts - 1) / nparts;
    const int64_t lb = (int64_t)stage * gs * npp;
    const int64_t ub = std::min<int64_t>((int64_t)(stage + 1) * gs * npp, N);
    std::vector<uint8_t> seen((size_t)N + 1, 0);
    for (int64_t i = 0; i < nnz; i++)
        if (row[i] >= lb && row[i] < ub)
            seen[(size_t)col[i]] = 1;
    out.clear();
    for (int64_t j = 0; j < N; j++)
        if (seen[(size_t)j])
            out.push_back((int32_t)j);
    return COLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// R-MAT generator
// ---------------------------------------------------------------------------
static inline uint64_t splitmix64(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

cola_status rmat_generate(int32_t scale, double deg, double a, double b, double c, uint64_t seed, int self_loops,
                          int value_kind, std::vector<int32_t> &row, std::vector<int32_t> &col,
                          std::vector<float> &val)
{
    COLA_REQUIRE(scale >= 1 && scale <= 30 && deg > 0 && a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0,
                 COLA_ERROR_INVALID_ARGUMENT, "rmat_generate: scale=%d deg=%g a=%g b=%g c=%g", scale, deg, a, b, c);
    const int64_t n = (int64_t)1 << scale;
    const int64_t m = (int64_t)std::ceil(deg * (double)n / 2.0);
    std::vector<uint64_t> keys((size_t)(2 * m));
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) {
        uint64_t st = seed * 0xD1B54A32D192ED03ull + (uint64_t)e * 0x9E3779B97F4A7C15ull;
        uint64_t u = 0, v = 0, bits = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 1) == 0)
                bits = splitmix64(st);
            const double p = (double)((bits >> ((l & 1) * 32)) & 0xFFFFFFFFull) * (1.0 / 4294967296.0);
            const uint64_t rb = p >= ab ? 1 : 0;
            const uint64_t cb = ((p >= a && p < ab) || p >= abc) ? 1 : 0;
            u = (u << 1) | rb;
            v = (v << 1) | cb;
        }
        if (u == v) {  // self-loops dropped; marked so they sort last
            keys[(size_t)(2 * e)] = keys[(size_t)(2 * e + 1)] = ~0ull;
        } else {
            keys[(size_t)(2 * e)] = (u << 32) | v;
            keys[(size_t)(2 * e + 1)] = (v << 32) | u;
        }
    }
    if (self_loops) {
        keys.reserve(keys.size() + (size_t)n);
        for (int64_t i = 0; i < n; i++)
            keys.push_back(((uint64_t)i << 32) | (uint64_t)i);
    }
    __gnu_parallel::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if (!keys.empty() && keys.back() == ~0ull)
        keys.pop_back();
    const size_t nnz = keys.size();
    row.resize(nnz);
    col.resize(nnz);
    std::vector<int32_t> degv((size_t)n, 0);
    for (size_t i = 0; i < nnz; i++) {
        row[i] = (int32_t)(keys[i] >> 32);
        col[i] = (int32_t)(keys[i] & 0xFFFFFFFFull);
        degv[(size_t)row[i]]++;
    }
    val.assign(nnz, 1.0f);
    if (value_kind == 1) {
        for (size_t i = 0; i < nnz; i++)
            val[i] = (float)(1.0 / (double)degv[(size_t)row[i]]);
    } else if (value_kind == 2) {
        for (size_t i = 0; i < nnz; i++)
            val[i] = (float)(1.0 / std::sqrt((double)degv[(size_t)row[i]] * (double)degv[(size_t)col[i]]));
    }
    return COLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// .bin files (include/dist_spmm_ppl_batch.cuh:7-27 with 64-bit sizes)
// ---------------------------------------------------------------------------
cola_status bin_read(const char *path, void *out, size_t elem, int64_t capacity, int64_t *count)
{
    COLA_REQUIRE(path && count, COLA_ERROR_INVALID_ARGUMENT, "bin_read: null argument");
    FILE *f = fopen(path, "rb");
    COLA_REQUIRE(f, COLA_ERROR_IO, "bin_read: cannot open %s", path);
    if (fseeko(f, 0, SEEK_END) != 0) {
        fclose(f);
        return fail(COLA_ERROR_IO, "bin_read: cannot seek %s", path);
    }
    const int64_t bytes = (int64_t)ftello(f);
    fseeko(f, 0, SEEK_SET);
    const int64_t n = bytes / (int64_t)elem;
    *count = n;
    if (!out) {
        fclose(f);
        return COLA_SUCCESS;
    }
    if (n > capacity) {
        fclose(f);
        return fail(COLA_ERROR_INVALID_ARGUMENT, "bin_read: %s holds %lld elements, capacity %lld", path,
                    (long long)n, (long long)capacity);
    }
    const size_t got = fread(out, elem, (size_t)n, f);
    fclose(f);
    COLA_REQUIRE((int64_t)got == n, COLA_ERROR_IO, "bin_read: short read of %s", path);
    return COLA_SUCCESS;
}

cola_status bin_write(const char *path, const void *data, size_t elem, int64_t n)
{
    COLA_REQUIRE(path && (n == 0 || data), COLA_ERROR_INVALID_ARGUMENT, "bin_write: null argument");
    FILE *f = fopen(path, "wb");
    COLA_REQUIRE(f, COLA_ERROR_IO, "bin_write: cannot create %s", path);
    const size_t put = n ? fwrite(data, elem, (size_t)n, f) : 0;
    const int rc = fclose(f);
    COLA_REQUIRE((int64_t)put == n && rc == 0, COLA_ERROR_IO, "bin_write: short write of %s", path);
    return COLA_SUCCESS;
}

static std::string part_file(const std::string &dir, const char *name, int P, int r)
{
    return dir + "/GPU" + std::to_string(P) + "/" + name + "_" + std::to_string(P) + "_" + std::to_string(r) +
           ".bin";
}

cola_status partition_write_bin(const cola_partition_set *s, const char *dir)
{
    COLA_REQUIRE(s && dir, COLA_ERROR_INVALID_ARGUMENT, "partition_write_bin: null argument");
    std::string d = dir;
    mkdir(d.c_str(), 0755);
    std::string g = d + "/GPU" + std::to_string(s->nparts);
    mkdir(g.c_str(), 0755);
    for (const PartHost &P : s->parts) {
        const int np = s->nparts, r = P.part;
        COLA_TRY(bin_write(part_file(d, "csr_rowPtr_l", np, r).c_str(), P.l_rowPtr.data(), 4, (int64_t)P.l_rowPtr.size()));
        COLA_TRY(bin_write(part_file(d, "csr_colIdx_l", np, r).c_str(), P.l_colIdx.data(), 4, (int64_t)P.l_colIdx.size()));
        COLA_TRY(bin_write(part_file(d, "csr_rowIdx_l", np, r).c_str(), P.l_rowIdx.data(), 4, (int64_t)P.l_rowIdx.size()));
        COLA_TRY(bin_write(part_file(d, "csc_rowIdx_r", np, r).c_str(), P.r_rowIdx.data(), 4, (int64_t)P.r_rowIdx.size()));
        COLA_TRY(bin_write(part_file(d, "csc_colPtr_r", np, r).c_str(), P.r_colPtr.data(), 4, (int64_t)P.r_colPtr.size()));
        COLA_TRY(bin_write(part_file(d, "csc_colIdx_r", np, r).c_str(), P.r_colIdx.data(), 4, (int64_t)P.r_colIdx.size()));
        COLA_TRY(bin_write(part_file(d, "csr_val_l", np, r).c_str(), P.l_val.data(), 4, (int64_t)P.l_val.size()));
        COLA_TRY(bin_write(part_file(d, "csc_val_r", np, r).c_str(), P.r_val.data(), 4, (int64_t)P.r_val.size()));
    }
    return COLA_SUCCESS;
}

template <typename T, typename A>
static cola_status read_vec(const std::string &path, std::vector<T, A> &v, bool optional, bool *present)
{
    struct stat st;
    if (stat(path.c_str(), &st) != 0) {
        if (present)
            *present = false;
        if (optional)
            return COLA_SUCCESS;
        return fail(COLA_ERROR_IO, "partition_read_bin: missing %s", path.c_str());
    }
    if (present)
        *present = true;
    int64_t n = 0;
    COLA_TRY(bin_read(path.c_str(), nullptr, sizeof(T), 0, &n));
    v.resize((size_t)n);
    return bin_read(path.c_str(), v.data(), sizeof(T), n, &n);
}

cola_status partition_read_bin(const char *dir, int32_t N, int32_t nparts, cola_partition_set *&out)
{
    COLA_REQUIRE(dir && N >= 0 && nparts >= 1, COLA_ERROR_INVALID_ARGUMENT, "partition_read_bin: bad argument");
    std::unique_ptr<cola_partition_set> s(new cola_partition_set());
    s->num_nodes = N;
    s->nparts = nparts;
    const int64_t npp = ((int64_t)N + nparts - 1) / nparts;
    s->npp = (int32_t)npp;
    s->parts.resize((size_t)nparts);
    const std::string d = dir;
    for (int32_t r = 0; r < nparts; r++) {
        PartHost &P = s->parts[(size_t)r];
        P.part = r;
        P.row_lb = (int32_t)std::min<int64_t>((int64_t)r * npp, N);
        P.row_ub = (int32_t)std::min<int64_t>((int64_t)(r + 1) * npp, N);
        COLA_TRY(read_vec(part_file(d, "csr_rowPtr_l", nparts, r), P.l_rowPtr, false, nullptr));
        COLA_TRY(read_vec(part_file(d, "csr_colIdx_l", nparts, r), P.l_colIdx, false, nullptr));
        COLA_TRY(read_vec(part_file(d, "csr_rowIdx_l", nparts, r), P.l_rowIdx, false, nullptr));
        COLA_TRY(read_vec(part_file(d, "csc_colPtr_r", nparts, r), P.r_colPtr, false, nullptr));
        COLA_TRY(read_vec(part_file(d, "csc_rowIdx_r", nparts, r), P.r_rowIdx, false, nullptr));
        COLA_TRY(read_vec(part_file(d, "csc_colIdx_r", nparts, r), P.r_colIdx, false, nullptr));
        bool has = false;
        COLA_TRY(read_vec(part_file(d, "csr_val_l", nparts, r), P.l_val, true, &has));
        if (!has)
            P.l_val.assign(P.l_colIdx.size(), 1.0f);
        COLA_TRY(read_vec(part_file(d, "csc_val_r", nparts, r), P.r_val, true, &has));
        if (!has)
            P.r_val.assign(P.r_rowIdx.size(), 1.0f);
        COLA_TRY(validate_partition(*s, P));
    }
    out = s.release();
    return COLA_SUCCESS;
}

// Structural checks of one partition (everything a kernel indexes with).
cola_status validate_partition(const cola_partition_set &s, const PartHost &P)
{
    const int64_t npp = s.npp, rows = (int64_t)P.row_ub - P.row_lb;
    const int64_t nl = (int64_t)P.l_rowIdx.size(), nzl = (int64_t)P.l_colIdx.size();
    const int64_t nc = (int64_t)P.r_colIdx.size(), nzr = (int64_t)P.r_rowIdx.size();
    COLA_REQUIRE((int64_t)P.l_rowPtr.size() == nl + 1 || (nl == 0 && P.l_rowPtr.size() <= 1),
                 COLA_ERROR_INVALID_ARGUMENT, "partition %d: local rowPtr length %zu vs %lld rows", P.part,
                 P.l_rowPtr.size(), (long long)nl);
    COLA_REQUIRE((int64_t)P.r_colPtr.size() == nc + 1 || (nc == 0 && P.r_colPtr.size() <= 1),
                 COLA_ERROR_INVALID_ARGUMENT, "partition %d: remote colPtr length %zu vs %lld cols", P.part,
                 P.r_colPtr.size(), (long long)nc);
    COLA_REQUIRE(P.l_val.size() == P.l_colIdx.size() && P.r_val.size() == P.r_rowIdx.size(),
                 COLA_ERROR_INVALID_ARGUMENT, "partition %d: value arrays do not match index arrays", P.part);
    if (nl > 0) {
        COLA_REQUIRE(P.l_rowPtr[0] == 0 && P.l_rowPtr[(size_t)nl] == nzl, COLA_ERROR_INVALID_ARGUMENT,
                     "partition %d: local rowPtr ends", P.part);
        for (int64_t i = 0; i < nl; i++) {
            COLA_REQUIRE(P.l_rowPtr[(size_t)i] <= P.l_rowPtr[(size_t)i + 1], COLA_ERROR_INVALID_ARGUMENT,
                         "partition %d: local rowPtr not monotone at %lld", P.part, (long long)i);
            COLA_REQUIRE(P.l_rowIdx[(size_t)i] >= 0 && P.l_rowIdx[(size_t)i] < rows, COLA_ERROR_INVALID_ARGUMENT,
                         "partition %d: local row id %d out of range", P.part, P.l_rowIdx[(size_t)i]);
        }
    } else {
        COLA_REQUIRE(nzl == 0, COLA_ERROR_INVALID_ARGUMENT, "partition %d: local entries without rows", P.part);
    }
    for (int64_t i = 0; i < nzl; i++)
        COLA_REQUIRE(P.l_colIdx[(size_t)i] >= 0 && P.l_colIdx[(size_t)i] < npp, COLA_ERROR_INVALID_ARGUMENT,
                     "partition %d: local col id %d out of range", P.part, P.l_colIdx[(size_t)i]);
    if (nc > 0) {
        COLA_REQUIRE(P.r_colPtr[0] == 0 && P.r_colPtr[(size_t)nc] == nzr, COLA_ERROR_INVALID_ARGUMENT,
                     "partition %d: remote colPtr ends", P.part);
        for (int64_t i = 0; i < nc; i++) {
            COLA_REQUIRE(P.r_colPtr[(size_t)i] <= P.r_colPtr[(size_t)i + 1], COLA_ERROR_INVALID_ARGUMENT,
                         "partition %d: remote colPtr not monotone at %lld", P.part, (long long)i);
            COLA_REQUIRE(P.r_colIdx[(size_t)i] >= 0 && P.r_colIdx[(size_t)i] < s.num_nodes &&
                             (i == 0 || P.r_colIdx[(size_t)i] > P.r_colIdx[(size_t)i - 1]),
                         COLA_ERROR_INVALID_ARGUMENT, "partition %d: remote col ids not ascending in range",
                         P.part);
        }
    } else {
        COLA_REQUIRE(nzr == 0, COLA_ERROR_INVALID_ARGUMENT, "partition %d: remote entries without cols", P.part);
    }
    for (int64_t i = 0; i < nzr; i++)
        COLA_REQUIRE(P.r_rowIdx[(size_t)i] >= 0 && P.r_rowIdx[(size_t)i] < rows, COLA_ERROR_INVALID_ARGUMENT,
                     "partition %d: remote row id %d out of range", P.part, P.r_rowIdx[(size_t)i]);
    return COLA_SUCCESS;
}

cola_status build_row_view(const cola_partition_set &s, int64_t hub_threshold, int64_t hub_segment,
                           int64_t task_entries, RowView &rv)
{
    COLA_REQUIRE(hub_threshold >= 1 && hub_segment >= 1 && task_entries >= 1, COLA_ERROR_INVALID_ARGUMENT,
                 "row view: hub_threshold, hub_segment and task_entries must be >= 1");
    const int64_t N = s.num_nodes;
    const int32_t P = s.nparts;
    rv = RowView();
    rv.ptr.assign((size_t)N + 1, 0);
    for (const PartHost &ph : s.parts) {
        for (size_t i = 0; i < ph.l_rowIdx.size(); i++)
            rv.ptr[(size_t)(ph.row_lb + ph.l_rowIdx[i]) + 1] += ph.l_rowPtr[i + 1] - ph.l_rowPtr[i];
        for (int32_t r : ph.r_rowIdx)
            rv.ptr[(size_t)(ph.row_lb + r) + 1] += 1;
    }
    for (int64_t r = 0; r < N; r++)
        rv.ptr[(size_t)r + 1] += rv.ptr[(size_t)r];
    rv.col.resize((size_t)rv.ptr[(size_t)N]);
    rv.val.resize((size_t)rv.ptr[(size_t)N]);
    std::vector<int64_t> cur(rv.ptr.begin(), rv.ptr.end() - 1);
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t p = 0; p < P; p++) {
        const PartHost &ph = s.parts[(size_t)p];
        const int64_t clb = (int64_t)p * s.npp;
        size_t ci = 0;
        // the remote columns below `limit`, column by column (each column's
        // rows are distinct, so every row receives its entries in column order)
        auto remote_cols_below = [&](int64_t limit) {
            for (; ci < ph.r_colIdx.size() && ph.r_colIdx[ci] < limit; ci++)
                for (int32_t q = ph.r_colPtr[ci]; q < ph.r_colPtr[ci + 1]; q++) {
                    const int64_t row = ph.row_lb + ph.r_rowIdx[(size_t)q];
                    const int64_t at = cur[(size_t)row]++;
                    rv.col[(size_t)at] = ph.r_colIdx[ci];
                    rv.val[(size_t)at] = ph.r_val[(size_t)q];
                }
        };
        remote_cols_below(clb);
        for (size_t i = 0; i < ph.l_rowIdx.size(); i++) {
            const int64_t row = ph.row_lb + ph.l_rowIdx[i];
            for (int32_t q = ph.l_rowPtr[i]; q < ph.l_rowPtr[i + 1]; q++) {
                const int64_t at = cur[(size_t)row]++;
                rv.col[(size_t)at] = (int32_t)(clb + ph.l_colIdx[(size_t)q]);
                rv.val[(size_t)at] = ph.l_val[(size_t)q];
            }
        }
        remote_cols_below(INT64_MAX);
    }
    // hub rows -> fixed-length segments
    for (int64_t r = 0; r < N; r++) {
        const int64_t b = rv.ptr[(size_t)r], e = rv.ptr[(size_t)r + 1];
        if (e - b <= hub_threshold)
            continue;
        rv.hub_row.push_back((int32_t)r);
        rv.hub_seg.push_back((int64_t)rv.seg_row.size());
        for (int64_t q = b; q < e; q += hub_segment) {
            rv.seg_row.push_back((int32_t)r);
            rv.seg_beg.push_back(q);
        }
    }
    rv.hub_seg.push_back((int64_t)rv.seg_row.size());
    // row blocks of about task_entries entries, never containing a hub row
    int64_t start = -1, cost = 0;
    for (int64_t r = 0; r < N; r++) {
        const int64_t len = rv.ptr[(size_t)r + 1] - rv.ptr[(size_t)r];
        if (len > hub_threshold) {
            if (start >= 0) {
                rv.task_rb.push_back((int32_t)start);
                rv.task_re.push_back((int32_t)r);
            }
            start = -1;
            cost = 0;
            continue;
        }
        if (start < 0)
            start = r;
        cost += len + 2;
        if (cost >= task_entries) {
            rv.task_rb.push_back((int32_t)start);
            rv.task_re.push_back((int32_t)(r + 1));
            start = -1;
            cost = 0;
        }
    }
    if (start >= 0) {
        rv.task_rb.push_back((int32_t)start);
        rv.task_re.push_back((int32_t)N);
    }
    return COLA_SUCCESS;
}

}  // namespace cola

// ===========================================================================
// C ABI (host part)
// ===========================================================================
using namespace cola;

extern "C" {

const char *cola_status_string(cola_status s)
{
    switch (s) {
    case COLA_SUCCESS: return "success";
    case COLA_ERROR_INVALID_ARGUMENT: return "invalid argument";
    case COLA_ERROR_CUDA: return "CUDA error";
    case COLA_ERROR_OUT_OF_MEMORY: return "out of memory";
    case COLA_ERROR_UNSUPPORTED: return "unsupported";
    case COLA_ERROR_IO: return "I/O error";
    case COLA_ERROR_BUDGET: return "over memory budget";
    case COLA_ERROR_TIMEOUT: return "timed out";
    case COLA_ERROR_NOT_READY: return "not ready";
    case COLA_ERROR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char *cola_last_error(void) { return g_last_error.c_str(); }

const char *cola_version(void) { return "cola_b200 0.1.0 (sm_100a)"; }

cola_status cola_partition_build(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                 const float *val, int32_t nparts, cola_partition_set **out)
{
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "cola_partition_build: out is NULL");
    *out = nullptr;
    try {
        return partition_build(num_nodes, nnz, row, col, val, nparts, *out);
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_partition_build: host allocation failed");
    }
}

void cola_partition_set_free(cola_partition_set *s) { delete s; }

cola_status cola_partition_get(const cola_partition_set *s, int32_t part, cola_partition_view *o)
{
    COLA_REQUIRE(s && o && part >= 0 && part < s->nparts, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_partition_get: bad argument (part %d)", part);
    const PartHost &P = s->parts[(size_t)part];
    o->part = part;
    o->nparts = s->nparts;
    o->num_nodes = s->num_nodes;
    o->nodes_per_part = s->npp;
    o->row_lb = P.row_lb;
    o->row_ub = P.row_ub;
    o->csr_rowPtr_l = P.l_rowPtr.data();
    o->csr_colIdx_l = P.l_colIdx.data();
    o->csr_val_l = P.l_val.data();
    o->csr_rowIdx_l = P.l_rowIdx.data();
    o->csc_colPtr_r = P.r_colPtr.data();
    o->csc_rowIdx_r = P.r_rowIdx.data();
    o->csc_val_r = P.r_val.data();
    o->csc_colIdx_r = P.r_colIdx.data();
    o->n_rowPtr_l = (int64_t)P.l_rowPtr.size();
    o->nnz_l = (int64_t)P.l_colIdx.size();
    o->n_rows_l = (int64_t)P.l_rowIdx.size();
    o->n_colPtr_r = (int64_t)P.r_colPtr.size();
    o->nnz_r = (int64_t)P.r_rowIdx.size();
    o->n_cols_r = (int64_t)P.r_colIdx.size();
    return COLA_SUCCESS;
}

cola_status cola_nnz_split(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                           int32_t *target, int32_t *ptr, int64_t capacity, int64_t *nchunks)
{
    COLA_REQUIRE(nchunks && nrows >= 0 && nnz >= 0 && (nrows == 0 || (rowIdx && rowPtr)),
                 COLA_ERROR_INVALID_ARGUMENT, "cola_nnz_split: bad argument");
    std::vector<int32_t> t, p;
    try {
        COLA_TRY(cola::nnz_split(rowIdx, nrows, rowPtr, nnz, t, p));
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_nnz_split: host allocation failed");
    }
    *nchunks = (int64_t)t.size();
    if (!target)
        return COLA_SUCCESS;
    COLA_REQUIRE((int64_t)t.size() <= capacity && ptr, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_nnz_split: %zu chunks exceed capacity %lld", t.size(), (long long)capacity);
    std::copy(t.begin(), t.end(), target);
    std::copy(p.begin(), p.end(), ptr);
    return COLA_SUCCESS;
}

// rabbit_module/src/reorder.cpp:283-288: edges relabelled by an old -> new map.
cola_status cola_relabel_edges(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                               const int32_t *mapping, int32_t *out_row, int32_t *out_col)
{
    clear_error();
    COLA_REQUIRE(num_nodes >= 0 && nnz >= 0, COLA_ERROR_INVALID_ARGUMENT, "cola_relabel_edges: bad sizes");
    if (nnz == 0)
        return COLA_SUCCESS;
    COLA_REQUIRE(row && col && mapping && out_row && out_col, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_relabel_edges: null arrays");
    for (int64_t i = 0; i < nnz; i++) {
        const int32_t r = row[i], c = col[i];
        COLA_REQUIRE(r >= 0 && r < num_nodes && c >= 0 && c < num_nodes, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_relabel_edges: entry %lld (%d, %d) outside %d x %d", (long long)i, r, c, num_nodes,
                     num_nodes);
        const int32_t mr = mapping[r], mc = mapping[c];
        COLA_REQUIRE(mr >= 0 && mr < num_nodes && mc >= 0 && mc < num_nodes, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_relabel_edges: entry %lld or its relabelled ids outside 0..%d", (long long)i,
                     num_nodes - 1);
        out_row[i] = mr;
        out_col[i] = mc;
    }
    return COLA_SUCCESS;
}

cola_status cola_global_csr(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col, const float *val_in,
                            int32_t *rowPtr, int32_t *colIdx, float *val_out, int64_t *nnz_out)
{
    COLA_REQUIRE(rowPtr && colIdx && nnz_out && N >= 0 && nnz >= 0, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_global_csr: bad argument");
    // The global CSR is partition 0 of a one-partition split (all columns local).
    cola_partition_set *s = nullptr;
    COLA_TRY(cola_partition_build(N, nnz, row, col, val_in, 1, &s));
    std::unique_ptr<cola_partition_set> hold(s);
    const PartHost &P = s->parts[0];
    std::fill(rowPtr, rowPtr + (int64_t)N + 1, 0);
    for (size_t i = 0; i < P.l_rowIdx.size(); i++)
        rowPtr[P.l_rowIdx[i] + 1] = P.l_rowPtr[i + 1] - P.l_rowPtr[i];
    for (int64_t r = 0; r < N; r++)
        rowPtr[r + 1] += rowPtr[r];
    std::copy(P.l_colIdx.begin(), P.l_colIdx.end(), colIdx);
    if (val_out)
        std::copy(P.l_val.begin(), P.l_val.end(), val_out);
    *nnz_out = (int64_t)P.l_colIdx.size();
    return COLA_SUCCESS;
}

cola_status cola_workgroup_cols(int32_t N, int64_t nnz, const int32_t *row, const int32_t *col, int32_t nparts,
                                int32_t gs, int32_t stage, int32_t *out, int64_t *count)
{
    COLA_REQUIRE(out && count, COLA_ERROR_INVALID_ARGUMENT, "cola_workgroup_cols: bad argument");
    std::vector<int32_t> v;
    COLA_TRY(workgroup_cols(N, nnz, row, col, nparts, gs, stage, v));
    std::copy(v.begin(), v.end(), out);
    *count = (int64_t)v.size();
    return COLA_SUCCESS;
}

cola_status cola_stage_tables(int32_t me, int32_t nranks, int32_t gs, int32_t N, const int32_t *zr, int64_t nrc,
                              int64_t nchunks_l, const int32_t *wg_cols, const int64_t *wg_off, int32_t *lo,
                              int32_t *ro, int32_t *po, int32_t *idx_ppl, int64_t *idx_off, int64_t idx_cap,
                              int32_t *put_colIdx, int64_t *put_lst_off, int64_t put_cap)
{
    COLA_REQUIRE(lo && ro && po && idx_off && put_lst_off && (nrc == 0 || zr), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_stage_tables: null argument");
    StageTables t;
    COLA_TRY(stage_tables(me, nranks, gs, N, zr, nrc, nchunks_l, wg_cols, wg_off, t));
    std::copy(t.local_offset.begin(), t.local_offset.end(), lo);
    std::copy(t.remote_offset.begin(), t.remote_offset.end(), ro);
    std::copy(t.put_offset.begin(), t.put_offset.end(), po);
    int64_t n = 0;
    idx_off[0] = 0;
    for (int32_t i = 1; i < t.nstages; i++) {
        const auto &l = t.idx_ppl[(size_t)i - 1];
        COLA_REQUIRE(n + (int64_t)l.size() <= idx_cap && idx_ppl, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_stage_tables: idx_ppl capacity %lld too small", (long long)idx_cap);
        std::copy(l.begin(), l.end(), idx_ppl + n);
        n += (int64_t)l.size();
        idx_off[i] = n;
    }
    n = 0;
    put_lst_off[0] = 0;
    for (int32_t i = 0; i + 1 < t.nstages; i++) {
        const auto &l = t.put_colIdx[(size_t)i];
        COLA_REQUIRE(n + (int64_t)l.size() <= put_cap && put_colIdx, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_stage_tables: put list capacity %lld too small", (long long)put_cap);
        std::copy(l.begin(), l.end(), put_colIdx + n);
        n += (int64_t)l.size();
        put_lst_off[i + 1] = n;
    }
    return COLA_SUCCESS;
}

cola_status cola_bin_read_i32(const char *path, int32_t *out, int64_t cap, int64_t *count)
{
    return bin_read(path, out, 4, cap, count);
}
cola_status cola_bin_write_i32(const char *path, const int32_t *data, int64_t n) { return bin_write(path, data, 4, n); }
cola_status cola_bin_read_f32(const char *path, float *out, int64_t cap, int64_t *count)
{
    return bin_read(path, out, 4, cap, count);
}
cola_status cola_bin_write_f32(const char *path, const float *data, int64_t n) { return bin_write(path, data, 4, n); }

cola_status cola_partition_write_bin(const cola_partition_set *s, const char *dir)
{
    return partition_write_bin(s, dir);
}

cola_status cola_partition_read_bin(const char *dir, int32_t N, int32_t nparts, cola_partition_set **out)
{
    COLA_REQUIRE(out, COLA_ERROR_INVALID_ARGUMENT, "cola_partition_read_bin: out is NULL");
    *out = nullptr;
    try {
        return partition_read_bin(dir, N, nparts, *out);
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_partition_read_bin: host allocation failed");
    }
}

cola_status cola_rmat_generate(int32_t scale, double deg, double a, double b, double c, uint64_t seed,
                               int32_t self_loops, int32_t value_kind, int32_t *row, int32_t *col, float *val,
                               int64_t capacity, int64_t *nnz)
{
    COLA_REQUIRE(nnz, COLA_ERROR_INVALID_ARGUMENT, "cola_rmat_generate: nnz is NULL");
    std::vector<int32_t> r, cc;
    std::vector<float> v;
    try {
        COLA_TRY(rmat_generate(scale, deg, a, b, c, seed, self_loops, value_kind, r, cc, v));
    } catch (const std::bad_alloc &) {
        return fail(COLA_ERROR_OUT_OF_MEMORY, "cola_rmat_generate: host allocation failed");
    }
    *nnz = (int64_t)r.size();
    if (!row)
        return COLA_SUCCESS;
    COLA_REQUIRE((int64_t)r.size() <= capacity && col, COLA_ERROR_INVALID_ARGUMENT,
                 "cola_rmat_generate: %zu entries exceed capacity %lld", r.size(), (long long)capacity);
    std::copy(r.begin(), r.end(), row);
    std::copy(cc.begin(), cc.end(), col);
    if (val)
        std::copy(v.begin(), v.end(), val);
    return COLA_SUCCESS;
}

}  // extern "C"
