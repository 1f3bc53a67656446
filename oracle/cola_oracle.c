/*
 * cola_oracle.c -- CPU oracle for CoLa's partitioned SpMM path.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline / reference legs of bench.py load this library, and only
 * as the checker or as the timed CPU baseline.  The cola_b200 package never
 * links, loads or calls it.
 *
 * Every function restates one step of the reference (zzzlxhhh/CoLa) in plain
 * C; its comment names the reference file:line it follows.  The preprocessing
 * restatements are pinned against golden vectors written by the reference's own
 * Python preprocessing (tests/golden/make_golden.py imports prep_torch_par.py
 * and prep_torch_ppl.py and runs them on seeded COO inputs).
 *
 * Conventions: int32 indices as in the reference's .bin files, int64 sizes,
 * caller-provided output buffers whose capacities come from the *_count helpers.
 * Duplicate (row, col) entries are merged as scipy's tocsr()/tocsc() merge them;
 * their values are summed in input order (the reference keeps no values, so the
 * order is this project's definition, shared with the product).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR 1

/* ---------------------------------------------------------------------------
 * Stable LSD radix sort of 64-bit keys carrying an int64 payload.
 * ------------------------------------------------------------------------- */
static int radix_sort_u64(uint64_t *key, int64_t *idx, int64_t n, int key_bits)
{
    if (n <= 1)
        return ORC_OK;
    uint64_t *k2 = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    int64_t *i2 = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    if (!k2 || !i2) {
        free(k2);
        free(i2);
        return ORC_ERR;
    }
    int64_t *cnt = (int64_t *)malloc(65536 * sizeof(int64_t));
    if (!cnt) {
        free(k2);
        free(i2);
        return ORC_ERR;
    }
    uint64_t *ks = key, *kd = k2;
    int64_t *is = idx, *id = i2;
    for (int shift = 0; shift < key_bits; shift += 16) {
        memset(cnt, 0, 65536 * sizeof(int64_t));
        for (int64_t i = 0; i < n; i++)
            cnt[(ks[i] >> shift) & 0xFFFF]++;
        int64_t s = 0;
        for (int d = 0; d < 65536; d++) {
            int64_t c = cnt[d];
            cnt[d] = s;
            s += c;
        }
        for (int64_t i = 0; i < n; i++) {
            int64_t p = cnt[(ks[i] >> shift) & 0xFFFF]++;
            kd[p] = ks[i];
            id[p] = is[i];
        }
        uint64_t *tk = ks;
        ks = kd;
        kd = tk;
        int64_t *ti = is;
        is = id;
        id = ti;
    }
    if (ks != key) {
        memcpy(key, ks, (size_t)n * sizeof(uint64_t));
        memcpy(idx, is, (size_t)n * sizeof(int64_t));
    }
    free(k2);
    free(i2);
    free(cnt);
    return ORC_OK;
}

/* Number of COO entries whose row lies in partition r (the capacity every
 * per-partition output array of orc_row_partition needs at most). */
int64_t orc_partition_count(int32_t num_nodes, int64_t nnz, const int32_t *row,
                            int32_t nparts, int32_t r)
{
    int64_t npp = ((int64_t)num_nodes + nparts - 1) / nparts;
    int64_t lb = (int64_t)r * npp;
    int64_t ub = lb + npp < num_nodes ? lb + npp : num_nodes;
    int64_t c = 0;
    for (int64_t i = 0; i < nnz; i++)
        if (row[i] >= lb && row[i] < ub)
            c++;
    return c;
}

/*
 * prep_torch_par.py:24-79 (row_partition), one partition r.
 *   nodesPerGPU = ceil(N/P) (:31); rows [r*npp, min((r+1)*npp, N)) (:34-36).
 *   Local = cols in [r*npp, (r+1)*npp) (:40); CSR over (row-lb, col%npp) with
 *   sorted, merged columns (:44-47); rowPtr = unique(indptr) drops empty rows
 *   (:51-52); rowIdx = sorted unique local rows (:48).
 *   Remote = the other cols (:60); CSC over global cols (:63-66);
 *   colPtr = unique(indptr) drops empty cols (:72-73); colIdx = sorted unique
 *   remote cols (:67-68); rowIdx = partition-local row ids (:75).
 * counts[0..5] = len(l_rowPtr), len(l_colIdx), len(l_rowIdx),
 *                len(r_colPtr), len(r_rowIdx), len(r_colIdx).
 * Output capacity: cap = orc_partition_count(); *_Ptr arrays need cap+1.
 * val may be NULL (all ones).
 */
int orc_row_partition(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                      const float *val, int32_t nparts, int32_t r,
                      int32_t *l_rowPtr, int32_t *l_colIdx, float *l_val, int32_t *l_rowIdx,
                      int32_t *r_colPtr, int32_t *r_rowIdx, float *r_val, int32_t *r_colIdx,
                      int64_t *counts)
{
    int64_t npp = ((int64_t)num_nodes + nparts - 1) / nparts;
    int64_t lb = (int64_t)r * npp;
    int64_t ub = lb + npp < num_nodes ? lb + npp : num_nodes;
    int64_t cap = orc_partition_count(num_nodes, nnz, row, nparts, r);
    uint64_t *lk = (uint64_t *)malloc((size_t)(cap + 1) * sizeof(uint64_t));
    int64_t *li = (int64_t *)malloc((size_t)(cap + 1) * sizeof(int64_t));
    uint64_t *rk = (uint64_t *)malloc((size_t)(cap + 1) * sizeof(uint64_t));
    int64_t *ri = (int64_t *)malloc((size_t)(cap + 1) * sizeof(int64_t));
    if (!lk || !li || !rk || !ri) {
        free(lk);
        free(li);
        free(rk);
        free(ri);
        return ORC_ERR;
    }
    int64_t nl = 0, nr = 0;
    for (int64_t i = 0; i < nnz; i++) {
        if (row[i] < lb || row[i] >= ub)
            continue;
        uint64_t lrow = (uint64_t)(row[i] - lb);
        int64_t c = col[i];
        if (c >= (int64_t)r * npp && c < (int64_t)(r + 1) * npp) {
            lk[nl] = (lrow << 32) | (uint64_t)(c % npp);
            li[nl++] = i;
        } else {
            rk[nr] = ((uint64_t)c << 32) | lrow;
            ri[nr++] = i;
        }
    }
    if (radix_sort_u64(lk, li, nl, 64) || radix_sort_u64(rk, ri, nr, 64)) {
        free(lk);
        free(li);
        free(rk);
        free(ri);
        return ORC_ERR;
    }
    /* local CSR, merged duplicates, empty rows dropped */
    int64_t nzl = 0, nrows = 0;
    l_rowPtr[0] = 0;
    for (int64_t i = 0; i < nl; i++) {
        float v = val ? val[li[i]] : 1.0f;
        if (i > 0 && lk[i] == lk[i - 1]) {
            l_val[nzl - 1] += v;
            continue;
        }
        uint32_t rr = (uint32_t)(lk[i] >> 32);
        if (i == 0 || rr != (uint32_t)(lk[i - 1] >> 32)) {
            if (nrows > 0)
                l_rowPtr[nrows] = (int32_t)nzl;
            l_rowIdx[nrows++] = (int32_t)rr;
        }
        l_colIdx[nzl] = (int32_t)(lk[i] & 0xFFFFFFFFu);
        l_val[nzl++] = v;
    }
    if (nrows > 0)
        l_rowPtr[nrows] = (int32_t)nzl;
    /* remote CSC, merged duplicates, empty cols dropped */
    int64_t nzr = 0, ncols = 0;
    r_colPtr[0] = 0;
    for (int64_t i = 0; i < nr; i++) {
        float v = val ? val[ri[i]] : 1.0f;
        if (i > 0 && rk[i] == rk[i - 1]) {
            r_val[nzr - 1] += v;
            continue;
        }
        uint32_t cc = (uint32_t)(rk[i] >> 32);
        if (i == 0 || cc != (uint32_t)(rk[i - 1] >> 32)) {
            if (ncols > 0)
                r_colPtr[ncols] = (int32_t)nzr;
            r_colIdx[ncols++] = (int32_t)cc;
        }
        r_rowIdx[nzr] = (int32_t)(rk[i] & 0xFFFFFFFFu);
        r_val[nzr++] = v;
    }
    if (ncols > 0)
        r_colPtr[ncols] = (int32_t)nzr;
    counts[0] = nrows + 1;
    counts[1] = nzl;
    counts[2] = nrows;
    counts[3] = ncols + 1;
    counts[4] = nzr;
    counts[5] = ncols;
    free(lk);
    free(li);
    free(rk);
    free(ri);
    return ORC_OK;
}

/*
 * prep_torch_par.py:93-101 (serialize): global CSR = A.tocsr() with merged,
 * sorted columns.  rowPtr has N+1 entries; colIdx/val capacity nnz.
 */
int orc_global_csr(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                   const float *val, int32_t *rowPtr, int32_t *colIdx, float *val_out,
                   int64_t *nnz_out)
{
    uint64_t *k = (uint64_t *)malloc((size_t)(nnz + 1) * sizeof(uint64_t));
    int64_t *ix = (int64_t *)malloc((size_t)(nnz + 1) * sizeof(int64_t));
    if (!k || !ix) {
        free(k);
        free(ix);
        return ORC_ERR;
    }
    for (int64_t i = 0; i < nnz; i++) {
        k[i] = ((uint64_t)(uint32_t)row[i] << 32) | (uint32_t)col[i];
        ix[i] = i;
    }
    if (radix_sort_u64(k, ix, nnz, 64)) {
        free(k);
        free(ix);
        return ORC_ERR;
    }
    int64_t m = 0;
    for (int32_t r = 0; r <= num_nodes; r++)
        rowPtr[r] = 0;
    for (int64_t i = 0; i < nnz; i++) {
        float v = val ? val[ix[i]] : 1.0f;
        if (i > 0 && k[i] == k[i - 1]) {
            val_out[m - 1] += v;
            continue;
        }
        colIdx[m] = (int32_t)(k[i] & 0xFFFFFFFFu);
        val_out[m] = v;
        rowPtr[(k[i] >> 32) + 1]++;
        m++;
    }
    for (int32_t r = 0; r < num_nodes; r++)
        rowPtr[r + 1] += rowPtr[r];
    *nnz_out = m;
    free(k);
    free(ix);
    return ORC_OK;
}

/*
 * prep_torch_ppl.py:24-49 (row_partition of the pipelined path): work-group
 * `stage` covers rows [stage*gs*npp, min((stage+1)*gs*npp, N)) (:182-184); its
 * list is the sorted unique set of columns those rows reference (:190-195).
 * out capacity: nnz (or N).  *count receives the list length.
 */
int orc_workgroup_cols(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                       int32_t nparts, int32_t gs, int32_t stage, int32_t *out, int64_t *count)
{
    int64_t npp = ((int64_t)num_nodes + nparts - 1) / nparts;
    int64_t lb = (int64_t)stage * gs * npp;
    int64_t ub = (int64_t)(stage + 1) * gs * npp;
    if (ub > num_nodes)
        ub = num_nodes;
    unsigned char *seen = (unsigned char *)calloc((size_t)num_nodes + 1, 1);
    if (!seen)
        return ORC_ERR;
    for (int64_t i = 0; i < nnz; i++)
        if (row[i] >= lb && row[i] < ub)
            seen[col[i]] = 1;
    int64_t c = 0;
    for (int64_t j = 0; j < num_nodes; j++)
        if (seen[j])
            out[c++] = (int32_t)j;
    *count = c;
    free(seen);
    return ORC_OK;
}

/*
 * include/dist_spmm_ppl_batch.cuh:29-56 (nnz_split).  gran = the average
 * entries per listed row, rounded up to a multiple of 32 (:34-35); every row
 * becomes chunks of at most gran entries; target[c] = the row id of chunk c,
 * ptr[c+1] = its end (ptr[0] = 0).  An empty row list leaves both outputs
 * empty (:32-33), so *ptr_len is 0 then, else nchunks+1.
 * Capacity: nnz/32 + nrows chunks always suffice.
 */
int orc_nnz_split(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                  int32_t *target, int32_t *ptr, int64_t cap, int64_t *nchunks, int64_t *ptr_len)
{
    *nchunks = 0;
    *ptr_len = 0;
    if (nrows == 0)
        return ORC_OK;
    int avg = (int)((uint64_t)nnz / (uint64_t)nrows);
    int gran = (avg + 32 - 1) / 32 * 32;
    if (gran <= 0)
        return ORC_ERR; /* the reference would loop forever here */
    int64_t c = 0;
    ptr[0] = 0;
    for (int64_t i = 0; i < nrows; i++) {
        int32_t lb = rowPtr[i], hb = rowPtr[i + 1];
        for (; lb < hb; lb += gran) {
            if (c >= cap)
                return ORC_ERR;
            target[c] = rowIdx[i];
            ptr[c + 1] = (lb + gran > hb) ? hb : lb + gran;
            c++;
        }
    }
    *nchunks = c;
    *ptr_len = c + 1;
    return ORC_OK;
}

static int64_t lower_bound_i32(const int32_t *a, int64_t n, int64_t v)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/*
 * src/distSpMM_ppl_batch.cu:101-193 (stage offset and index tables of PE `me`).
 * Inputs: the split remote chunk column ids csc_colIdx_zip_r (ascending), the
 * local chunk count, and every work group's column list (prep_torch_ppl.py
 * output) concatenated in wg_cols with wg_off[g]..wg_off[g+1].
 * Outputs (nstages = nranks/gs):
 *   local_off[2*nstages], remote_off[2*nstages], put_off[2*nstages]   (:69-72)
 *   idx_ppl lists for stages 1..nstages-1, concatenated, idx_off[nstages]
 *   put_colIdx lists for stages 0..nstages-2, concatenated, put_lst_off[nstages]
 * idx_cap/put_cap: capacities of idx_ppl/put_colIdx.
 */
int orc_stage_tables(int32_t me, int32_t nranks, int32_t gs, int32_t num_nodes,
                     const int32_t *csc_colIdx_zip_r, int64_t nrc, int64_t nchunks_l,
                     const int32_t *wg_cols, const int64_t *wg_off,
                     int32_t *local_off, int32_t *remote_off, int32_t *put_off,
                     int32_t *idx_ppl, int64_t *idx_off, int64_t idx_cap,
                     int32_t *put_colIdx, int64_t *put_lst_off, int64_t put_cap)
{
    int32_t nstages = nranks / gs;
    int64_t npp = ((int64_t)num_nodes + nranks - 1) / nranks; /* .cu:74 */
    for (int32_t i = 0; i < 2 * nstages; i++)
        local_off[i] = remote_off[i] = put_off[i] = 0;
    idx_off[0] = 0;
    int64_t ni = 0;
    const int32_t *mywg = wg_cols ? wg_cols + wg_off[me / gs] : NULL;
    int64_t mywg_n = wg_cols ? wg_off[me / gs + 1] - wg_off[me / gs] : 0;
    for (int32_t i = 0; i < nstages; i++) {
        int32_t next_pos = (me + gs * i) % nranks;
        int32_t group_id = next_pos / gs;
        int64_t local_lb = (int64_t)next_pos * npp;
        int64_t local_ub = local_lb + npp < num_nodes ? local_lb + npp : num_nodes;
        int64_t remote_lb = (int64_t)group_id * gs * npp;
        int64_t remote_ub = remote_lb + (int64_t)gs * npp < num_nodes ? remote_lb + (int64_t)gs * npp : num_nodes;
        if (i == 0) {
            local_off[0] = 0;
            local_off[1] = (int32_t)nchunks_l;
        } else {
            local_off[2 * i] = (int32_t)lower_bound_i32(csc_colIdx_zip_r, nrc, local_lb);
            local_off[2 * i + 1] = (int32_t)lower_bound_i32(csc_colIdx_zip_r, nrc, local_ub);
        }
        remote_off[2 * i] = (int32_t)lower_bound_i32(csc_colIdx_zip_r, nrc, remote_lb);
        remote_off[2 * i + 1] = (int32_t)lower_bound_i32(csc_colIdx_zip_r, nrc, remote_ub);
        if (i != 0) {
            /* :139-151  my work group's columns that live on each source PE */
            int64_t *slb = (int64_t *)malloc((size_t)gs * sizeof(int64_t));
            int64_t *sub = (int64_t *)malloc((size_t)gs * sizeof(int64_t));
            int64_t *pos = (int64_t *)calloc((size_t)gs, sizeof(int64_t));
            if (!slb || !sub || !pos) {
                free(slb);
                free(sub);
                free(pos);
                return ORC_ERR;
            }
            for (int32_t j = 0; j < gs; j++) {
                int64_t src_pe = j + (int64_t)group_id * gs;
                int64_t lb = src_pe * npp;
                int64_t ub = lb + npp < num_nodes ? lb + npp : num_nodes;
                slb[j] = lower_bound_i32(mywg, mywg_n, lb);
                sub[j] = lower_bound_i32(mywg, mywg_n, ub);
            }
            /* :153-168  forward search from the last match, per source PE */
            for (int64_t j = remote_off[2 * i]; j < remote_off[2 * i + 1]; j++) {
                int32_t cur_col = csc_colIdx_zip_r[j];
                int32_t rg = (int32_t)((cur_col / npp) % gs);
                int64_t k = pos[rg];
                while (k < sub[rg] - slb[rg]) {
                    if (mywg[slb[rg] + k] == cur_col) {
                        if (ni >= idx_cap) {
                            free(slb);
                            free(sub);
                            free(pos);
                            return ORC_ERR;
                        }
                        idx_ppl[ni++] = (int32_t)k;
                        pos[rg] = k;
                        break;
                    }
                    k++;
                }
            }
            free(slb);
            free(sub);
            free(pos);
            idx_off[i] = ni;
        }
    }
    /* :172-193  rows this PE sends at each stage */
    int64_t np = 0;
    put_lst_off[0] = 0;
    for (int32_t i = 0; i < nstages - 1; i++) {
        int32_t target_pe = (me - (i + 1) * gs) % nranks;
        target_pe = (target_pe + nranks) % nranks;
        int32_t tw = target_pe / gs;
        const int32_t *tl = wg_cols + wg_off[tw];
        int64_t tn = wg_off[tw + 1] - wg_off[tw];
        int64_t plb = (int64_t)me * npp;
        int64_t pub = plb + npp < num_nodes ? plb + npp : num_nodes;
        int64_t a = lower_bound_i32(tl, tn, plb);
        int64_t b = lower_bound_i32(tl, tn, pub);
        put_off[2 * i] = (int32_t)a;
        put_off[2 * i + 1] = (int32_t)b;
        for (int64_t q = a; q < b; q++) {
            if (np >= put_cap)
                return ORC_ERR;
            put_colIdx[np++] = tl[q];
        }
        put_lst_off[i + 1] = np;
    }
    return ORC_OK;
}

/*
 * FP64 SpMM over a CSR (the oracle of the product's output):
 * Y[i,:] = sum_p val[p] * X[colIdx[p], :], accumulated in double.
 * The reference's own check (include/utils.cuh:45-69, SAG_reference_host)
 * is the same loop in FP32 without values.
 */
void orc_spmm_csr_f64(int64_t nrows, const int32_t *rowPtr, const int32_t *colIdx,
                      const float *val, const float *X, int64_t ldx, int32_t K,
                      double *Y, int64_t ldy)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nrows; i++) {
        double *y = Y + i * ldy;
        for (int32_t k = 0; k < K; k++)
            y[k] = 0.0;
        for (int32_t p = rowPtr[i]; p < rowPtr[i + 1]; p++) {
            double v = val ? (double)val[p] : 1.0;
            const float *x = X + (int64_t)colIdx[p] * ldx;
            for (int32_t k = 0; k < K; k++)
                y[k] += v * (double)x[k];
        }
    }
}

/*
 * FP32 SpMM in one fixed order, to be matched bit for bit: row by row,
 * entries in CSR order, one fused multiply-add (fmaf, correctly rounded) per
 * product into an accumulator that starts at +0.  A row with more than
 * hub_threshold entries is summed as segments of hub_segment entries (each
 * from +0); the segment partials are then added by a binary counter -- partial
 * s is added onto the open block sums of sizes 1, 2, 4, ... that the trailing
 * one bits of s close -- and the open sums are folded largest first.  This is
 * the summation order of cola_b200's row-major schedule for row tiles of one
 * warp (32 lanes x 16 bytes: K a multiple of 128 with FP32 X); the math is the
 * reference's SpMM (include/utils.cuh:45-69, SAG_reference_host) with values.
 */
int orc_spmm_rows_f32_ordered(int64_t nrows, const int64_t *rowPtr, const int32_t *colIdx, const float *val,
                              const float *X, int64_t ldx, int32_t K, int64_t hub_threshold, int64_t hub_segment,
                              float *Y, int64_t ldy)
{
    if (hub_threshold < 1 || hub_segment < 1 || K < 1)
        return ORC_ERR;
    int bad = 0;
#pragma omp parallel
    {
        float *stk = (float *)malloc((size_t)65 * K * sizeof(float));  /* levels 0..63, then a partial */
        if (!stk) {
#pragma omp atomic write
            bad = 1;
        }
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < nrows; i++) {
            if (!stk)
                continue;
            float *y = Y + i * ldy;
            const int64_t b = rowPtr[i], e = rowPtr[i + 1];
            if (e - b <= hub_threshold) {
                for (int32_t k = 0; k < K; k++)
                    y[k] = 0.0f;
                for (int64_t p = b; p < e; p++) {
                    const float v = val[p];
                    const float *x = X + (int64_t)colIdx[p] * ldx;
                    for (int32_t k = 0; k < K; k++)
                        y[k] = fmaf(v, x[k], y[k]);
                }
                continue;
            }
            const int64_t m = (e - b + hub_segment - 1) / hub_segment;
            float *c = stk + (size_t)64 * K;
            for (int64_t sgi = 0; sgi < m; sgi++) {
                const int64_t q1 = b + (sgi + 1) * hub_segment < e ? b + (sgi + 1) * hub_segment : e;
                for (int32_t k = 0; k < K; k++)
                    c[k] = 0.0f;
                for (int64_t p = b + sgi * hub_segment; p < q1; p++) {
                    const float v = val[p];
                    const float *x = X + (int64_t)colIdx[p] * ldx;
                    for (int32_t k = 0; k < K; k++)
                        c[k] = fmaf(v, x[k], c[k]);
                }
                int l = 0;
                while ((sgi >> l) & 1) {
                    const float *a = stk + (size_t)l * K;
                    for (int32_t k = 0; k < K; k++)
                        c[k] = a[k] + c[k];
                    l++;
                }
                memcpy(stk + (size_t)l * K, c, (size_t)K * sizeof(float));
            }
            int first = 1;
            for (int l = 63; l >= 0; l--)
                if ((m >> l) & 1) {
                    const float *a = stk + (size_t)l * K;
                    for (int32_t k = 0; k < K; k++)
                        y[k] = first ? a[k] : y[k] + a[k];
                    first = 0;
                }
        }
        free(stk);
    }
    return bad ? ORC_ERR : ORC_OK;
}

/* Same with BF16 X (raw uint16 bit patterns, widened exactly to FP32). */
void orc_spmm_csr_f64_bf16x(int64_t nrows, const int32_t *rowPtr, const int32_t *colIdx,
                            const float *val, const uint16_t *X, int64_t ldx, int32_t K,
                            double *Y, int64_t ldy)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < nrows; i++) {
        double *y = Y + i * ldy;
        for (int32_t k = 0; k < K; k++)
            y[k] = 0.0;
        for (int32_t p = rowPtr[i]; p < rowPtr[i + 1]; p++) {
            double v = val ? (double)val[p] : 1.0;
            const uint16_t *x = X + (int64_t)colIdx[p] * ldx;
            for (int32_t k = 0; k < K; k++) {
                uint32_t bits = (uint32_t)x[k] << 16;
                float f;
                memcpy(&f, &bits, 4);
                y[k] += v * (double)f;
            }
        }
    }
}

/*
 * One partition's SpMM from its split ("zip") arrays, in FP64:
 * include/dist_spmm_ppl_batch.cuh:76-200 (ppl0_batch_SpMM_kernel) restated
 * without atomics.  Local chunk c adds sum_p val*X_p[colIdx[p]] to row
 * rowIdx_zip[c] (:164-197); remote chunk c adds val*X[colIdx_zip[c]] to every
 * row in its range (:112-160).  X_p = X + part*npp*ldx; remote columns are
 * global ids into X.  Y (npp x ldy) is overwritten.
 */
void orc_spmm_partition_f64(int32_t part, int32_t npp,
                            const int32_t *l_ptr, const int32_t *l_colIdx, const int32_t *l_rowIdx_zip,
                            const float *l_val, int64_t l_nchunks,
                            const int32_t *r_ptr, const int32_t *r_rowIdx, const int32_t *r_colIdx_zip,
                            const float *r_val, int64_t r_nchunks,
                            const float *X, int64_t ldx, int32_t K, double *Y, int64_t ldy)
{
    for (int64_t i = 0; i < (int64_t)npp; i++)
        for (int32_t k = 0; k < K; k++)
            Y[i * ldy + k] = 0.0;
    const float *Xp = X + (int64_t)part * npp * ldx;
    for (int64_t c = 0; c < l_nchunks; c++) {
        double *y = Y + (int64_t)l_rowIdx_zip[c] * ldy;
        for (int32_t p = l_ptr[c]; p < l_ptr[c + 1]; p++) {
            double v = l_val ? l_val[p] : 1.0;
            const float *x = Xp + (int64_t)l_colIdx[p] * ldx;
            for (int32_t k = 0; k < K; k++)
                y[k] += v * (double)x[k];
        }
    }
    for (int64_t c = 0; c < r_nchunks; c++) {
        const float *x = X + (int64_t)r_colIdx_zip[c] * ldx;
        for (int32_t p = r_ptr[c]; p < r_ptr[c + 1]; p++) {
            double v = r_val ? r_val[p] : 1.0;
            double *y = Y + (int64_t)r_rowIdx[p] * ldy;
            for (int32_t k = 0; k < K; k++)
                y[k] += v * (double)x[k];
        }
    }
}

/*
 * OpenMP FP32 loop over P partitions (local CSR chunks + remote CSC chunks),
 * the CPU baseline of the partitioned matrix: one thread owns one partition's
 * output block, so no two threads write the same row.  Arrays of all
 * partitions are concatenated; partition p's arrays start at the offsets
 * l_ptr_off[p], l_nz_off[p], l_ch_off[p] (and r_*), Y is (P*npp) x ldy.
 */
void orc_spmm_partitions_f32_omp(int32_t nparts, int32_t npp,
                                 const int32_t *l_ptr, const int64_t *l_ptr_off,
                                 const int32_t *l_colIdx, const float *l_val, const int64_t *l_nz_off,
                                 const int32_t *l_rowIdx_zip, const int64_t *l_ch_off,
                                 const int32_t *r_ptr, const int64_t *r_ptr_off,
                                 const int32_t *r_rowIdx, const float *r_val, const int64_t *r_nz_off,
                                 const int32_t *r_colIdx_zip, const int64_t *r_ch_off,
                                 const float *X, int64_t ldx, int32_t K, float *Y, int64_t ldy,
                                 int32_t nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t p = 0; p < nparts; p++) {
        float *Yp = Y + (int64_t)p * npp * ldy;
        const float *Xp = X + (int64_t)p * npp * ldx;
        for (int64_t i = 0; i < (int64_t)npp; i++)
            memset(Yp + i * ldy, 0, (size_t)K * sizeof(float));
        const int32_t *lp = l_ptr + l_ptr_off[p];
        const int32_t *lc = l_colIdx + l_nz_off[p];
        const float *lv = l_val + l_nz_off[p];
        const int32_t *lr = l_rowIdx_zip + l_ch_off[p];
        int64_t nlc = l_ch_off[p + 1] - l_ch_off[p];
        for (int64_t c = 0; c < nlc; c++) {
            float *y = Yp + (int64_t)lr[c] * ldy;
            for (int32_t q = lp[c]; q < lp[c + 1]; q++) {
                const float *x = Xp + (int64_t)lc[q] * ldx;
                float v = lv[q];
                for (int32_t k = 0; k < K; k++)
                    y[k] += v * x[k];
            }
        }
        const int32_t *rp = r_ptr + r_ptr_off[p];
        const int32_t *rr = r_rowIdx + r_nz_off[p];
        const float *rv = r_val + r_nz_off[p];
        const int32_t *rc = r_colIdx_zip + r_ch_off[p];
        int64_t nrc = r_ch_off[p + 1] - r_ch_off[p];
        for (int64_t c = 0; c < nrc; c++) {
            const float *x = X + (int64_t)rc[c] * ldx;
            for (int32_t q = rp[c]; q < rp[c + 1]; q++) {
                float *y = Yp + (int64_t)rr[q] * ldy;
                float v = rv[q];
                for (int32_t k = 0; k < K; k++)
                    y[k] += v * x[k];
            }
        }
    }
}

/* Largest OpenMP team this process may use. */
int32_t orc_max_threads(void)
{
#ifdef _OPENMP
    return (int32_t)omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------------------
 * Seeded R-MAT graph: the synthetic stand-in for the reference's dataset, as
 * the library's cola_rmat_generate defines it (the reference ships no
 * generator; its dataset is a file).  Edge e draws `scale` quadrant choices
 * from its own splitmix64 stream (seed * 0xD1B54A32D192ED03 + e * golden
 * ratio), 32 bits per level; self-loops are dropped, every edge is stored
 * both ways, optional self-loops are added for every vertex, and the list is
 * sorted by (row, col) with duplicates removed.  Values: 0 -> 1.0,
 * 1 -> 1/deg(row), 2 -> 1/sqrt(deg(row) deg(col)).  Two-call protocol: row ==
 * NULL returns the entry count in *nnz.  The bench's reference leg uses this
 * restatement so that it loads nothing of the product.
 * ------------------------------------------------------------------------- */
static uint64_t orc_splitmix64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* LSD radix sort of keys only (16-bit digits over key_bits). */
static int radix_sort_keys(uint64_t *key, int64_t n, int key_bits)
{
    if (n <= 1)
        return ORC_OK;
    uint64_t *tmp = (uint64_t *)malloc((size_t)n * sizeof(uint64_t));
    int64_t *cnt = (int64_t *)malloc(65536 * sizeof(int64_t));
    if (!tmp || !cnt) {
        free(tmp);
        free(cnt);
        return ORC_ERR;
    }
    uint64_t *src = key, *dst = tmp;
    for (int shift = 0; shift < key_bits; shift += 16) {
        memset(cnt, 0, 65536 * sizeof(int64_t));
        for (int64_t i = 0; i < n; i++)
            cnt[(src[i] >> shift) & 0xFFFF]++;
        int64_t s = 0;
        for (int d = 0; d < 65536; d++) {
            int64_t c = cnt[d];
            cnt[d] = s;
            s += c;
        }
        for (int64_t i = 0; i < n; i++)
            dst[cnt[(src[i] >> shift) & 0xFFFF]++] = src[i];
        uint64_t *t = src;
        src = dst;
        dst = t;
    }
    if (src != key)
        memcpy(key, src, (size_t)n * sizeof(uint64_t));
    free(tmp);
    free(cnt);
    return ORC_OK;
}

int orc_rmat_generate(int32_t scale, double deg, double a, double b, double c, uint64_t seed,
                      int32_t self_loops, int32_t value_kind, int32_t *row, int32_t *col, float *val,
                      int64_t capacity, int64_t *nnz)
{
    if (scale < 1 || scale > 30 || !(deg > 0) || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 || !nnz)
        return ORC_ERR;
    const int64_t n = (int64_t)1 << scale;
    const int64_t m = (int64_t)ceil(deg * (double)n / 2.0);
    const int64_t cap = 2 * m + (self_loops ? n : 0);
    uint64_t *keys = (uint64_t *)malloc((size_t)cap * sizeof(uint64_t));
    unsigned char *keep = (unsigned char *)malloc((size_t)m);
    if (!keys || !keep) {
        free(keys);
        free(keep);
        return ORC_ERR;
    }
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++) {
        uint64_t st = seed * 0xD1B54A32D192ED03ull + (uint64_t)e * 0x9E3779B97F4A7C15ull;
        uint64_t u = 0, v = 0, bits = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 1) == 0)
                bits = orc_splitmix64(&st);
            const double p = (double)((bits >> ((l & 1) * 32)) & 0xFFFFFFFFull) * (1.0 / 4294967296.0);
            const uint64_t rb = p >= ab ? 1 : 0;
            const uint64_t cb = ((p >= a && p < ab) || p >= abc) ? 1 : 0;
            u = (u << 1) | rb;
            v = (v << 1) | cb;
        }
        keep[e] = u != v;
        keys[2 * e] = (u << scale) | v;
        keys[2 * e + 1] = (v << scale) | u;
    }
    int64_t k = 0;
    for (int64_t e = 0; e < m; e++)
        if (keep[e]) {
            keys[k++] = keys[2 * e];
            keys[k++] = keys[2 * e + 1];
        }
    free(keep);
    if (self_loops)
        for (int64_t i = 0; i < n; i++)
            keys[k++] = ((uint64_t)i << scale) | (uint64_t)i;
    if (radix_sort_keys(keys, k, 2 * scale) != ORC_OK) {
        free(keys);
        return ORC_ERR;
    }
    int64_t u = 0;
    for (int64_t i = 0; i < k; i++)
        if (i == 0 || keys[i] != keys[i - 1])
            keys[u++] = keys[i];
    *nnz = u;
    if (!row) {
        free(keys);
        return ORC_OK;
    }
    if (u > capacity || !col || !val) {
        free(keys);
        return ORC_ERR;
    }
    int32_t *dg = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    if (!dg) {
        free(keys);
        return ORC_ERR;
    }
    const uint64_t mask = ((uint64_t)1 << scale) - 1;
    for (int64_t i = 0; i < u; i++) {
        row[i] = (int32_t)(keys[i] >> scale);
        col[i] = (int32_t)(keys[i] & mask);
        dg[row[i]]++;
    }
    for (int64_t i = 0; i < u; i++) {
        if (value_kind == 1)
            val[i] = (float)(1.0 / (double)dg[row[i]]);
        else if (value_kind == 2)
            val[i] = (float)(1.0 / sqrt((double)dg[row[i]] * (double)dg[col[i]]));
        else
            val[i] = 1.0f;
    }
    free(dg);
    free(keys);
    return ORC_OK;
}
