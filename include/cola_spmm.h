/*
 * cola_spmm.h -- C ABI of cola_b200, a single-GPU B200 (sm_100a) implementation
 * of CoLa's partitioned SpMM (zzzlxhhh/CoLa).
 *
 * The matrix is split into P virtual row partitions ("PEs").  Partition p owns
 * rows [p*npp, min((p+1)*npp, N)), npp = ceil(N/P), and holds
 *   - a local CSR block over the columns it owns (column ids are col % npp),
 *   - a remote CSC block over the other columns (global ids), compacted so that
 *     only non-empty columns appear,
 * both optionally chunked by nnz_split.  Dense matrices are row-major.
 *
 * Symmetric-buffer convention (replaces the NVSHMEM symmetric heap on one GPU):
 * the P copies of a per-PE dense buffer (the input X slices, the pipeline
 * buffers) are laid out back to back, nodesPerPE*dim elements apart, so PE q's
 * copy of a buffer that PE me addresses as `a` is a + (q - me)*nodesPerPE*dim.
 * For X this means: the whole X is one (P*npp) x dim array and PE me's `input`
 * points at row me*npp of it.
 *
 * Errors: every entry point returns a cola_status and never exits the process
 * (the reference exits on error: include/utils.cuh:10-22).
 * cola_last_error() returns a thread-local message for the last failure.
 * Launch entry points are asynchronous on the given stream, like the
 * reference's launchers.
 */
#ifndef COLA_SPMM_H
#define COLA_SPMM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Binary-compatible with cudaStream_t. */
typedef struct CUstream_st *cola_stream_t;

typedef enum cola_status {
    COLA_SUCCESS = 0,
    COLA_ERROR_INVALID_ARGUMENT = 1,
    COLA_ERROR_CUDA = 2,
    COLA_ERROR_OUT_OF_MEMORY = 3,
    COLA_ERROR_UNSUPPORTED = 4,
    COLA_ERROR_IO = 5,
    COLA_ERROR_BUDGET = 6,
    COLA_ERROR_TIMEOUT = 7,
    COLA_ERROR_NOT_READY = 8,
    COLA_ERROR_CANCELLED = 9
} cola_status;

typedef enum cola_dtype {
    COLA_FLOAT32 = 0,
    COLA_BFLOAT16 = 1
} cola_dtype;

const char *cola_status_string(cola_status s);
/* Thread-local description of the last failure in this thread ("" if none). */
const char *cola_last_error(void);
/* Library version string. */
const char *cola_version(void);

/* ========================================================================
 * Preprocessing (host).  Replaces prep_torch_par.py, prep_torch_ppl.py,
 * nnz_split and the stage tables of src/distSpMM_ppl_batch.cu; outputs are
 * bit-identical to the reference's.
 * ====================================================================== */

typedef struct cola_partition_set cola_partition_set;

/* prep_torch_par.py:24-79 (row_partition) for all nparts partitions, from a
 * COO list (duplicates allowed; merged as scipy's tocsr()/tocsc() merge them,
 * their values summed in input order).  val may be NULL (all ones, which is
 * what the reference uses: src/distSpMM_ppl_batch.cu:83,99). */
cola_status cola_partition_build(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                 const float *val, int32_t nparts, cola_partition_set **out);
void cola_partition_set_free(cola_partition_set *s);

/* Read-only view of one partition.  Array lengths follow the reference's .bin
 * files: n_rowPtr_l = n_rows_l + 1 (1 if no local entries), n_colPtr_r =
 * n_cols_r + 1 (1 if no remote entries). */
typedef struct cola_partition_view {
    int32_t part, nparts, num_nodes, nodes_per_part, row_lb, row_ub;
    const int32_t *csr_rowPtr_l;  /* n_rowPtr_l */
    const int32_t *csr_colIdx_l;  /* nnz_l, local column ids (col % npp) */
    const float *csr_val_l;       /* nnz_l */
    const int32_t *csr_rowIdx_l;  /* n_rows_l, partition-local row ids */
    const int32_t *csc_colPtr_r;  /* n_colPtr_r */
    const int32_t *csc_rowIdx_r;  /* nnz_r, partition-local row ids */
    const float *csc_val_r;       /* nnz_r */
    const int32_t *csc_colIdx_r;  /* n_cols_r, global column ids */
    int64_t n_rowPtr_l, nnz_l, n_rows_l, n_colPtr_r, nnz_r, n_cols_r;
} cola_partition_view;

cola_status cola_partition_get(const cola_partition_set *s, int32_t part, cola_partition_view *out);

/* include/dist_spmm_ppl_batch.cuh:29-56 (nnz_split).  Chunk granularity is the
 * average entries per listed row rounded up to a multiple of 32.  Pass
 * target == NULL to only count (*nchunks).  ptr receives nchunks+1 entries, or
 * none when nrows == 0 (as the reference leaves it empty). */
cola_status cola_nnz_split(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                           int32_t *target, int32_t *ptr, int64_t capacity, int64_t *nchunks);

/* ------------------------------------------------------------------------
 * Preprocessing on the device (same outputs, bit for bit, as the host calls
 * above).  Inputs are device arrays; the calls run on `stream` and return once
 * their results are complete.
 * ---------------------------------------------------------------------- */

/* cola_partition_build with the COO (row, col, optional val) in device memory:
 * the partitions are built by a radix sort on the device and returned as a
 * host partition set, identical to what cola_partition_build gives for the
 * same COO.  Needs about 40 bytes of device memory per entry while it runs. */
cola_status cola_partition_build_device(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                        const float *val, int32_t nparts, cola_stream_t stream,
                                        cola_partition_set **out);

/* cola_nnz_split on device arrays (rowIdx: nrows, rowPtr: nrows+1; target and
 * ptr device arrays of capacity / capacity+1 entries).  target == NULL only
 * counts (*nchunks). */
cola_status cola_nnz_split_device(const int32_t *rowIdx, int64_t nrows, const int32_t *rowPtr, int64_t nnz,
                                  int32_t *target, int32_t *ptr, int64_t capacity, int64_t *nchunks,
                                  cola_stream_t stream);

/* Vertex relabelling of a COO edge list, as rabbit_module/src/reorder.cpp:
 * 283-288 applies its old -> new id mapping: out_row[i] = mapping[row[i]],
 * out_col[i] = mapping[col[i]].  The mapping itself (community ordering) is
 * computed elsewhere; any permutation of 0..num_nodes-1 is accepted.  Host and
 * device forms; the outputs may alias the inputs. */
cola_status cola_relabel_edges(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                               const int32_t *mapping, int32_t *out_row, int32_t *out_col);
cola_status cola_relabel_edges_device(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                      const int32_t *mapping, int32_t *out_row, int32_t *out_col,
                                      cola_stream_t stream);

/* The reordering step the reference runs before partitioning
 * (rabbit_order_write.py:48-55 calls its Rabbit Order module,
 * rabbit_module/src/reorder.cpp:260-288), written from the published method:
 * communities found by incremental aggregation (vertices visited by increasing
 * degree, each merged into the neighbouring community of largest positive
 * modularity gain), then numbered community by community, each community's
 * merge tree depth first, so that its vertices get consecutive ids.  The COO is
 * read as an undirected graph (self-loops ignored, duplicates adding up).
 * mapping[old] = new (a permutation of 0..num_nodes-1, for
 * cola_relabel_edges); *communities (may be NULL) receives the number of
 * top-level communities.  Deterministic; host only. */
cola_status cola_community_order(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                 int32_t *mapping, int64_t *communities);

/* prep_torch_par.py:93-101 (serialize: global CSR).  rowPtr: num_nodes+1;
 * colIdx/val: capacity nnz (val may be NULL). */
cola_status cola_global_csr(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                            const float *val_in, int32_t *rowPtr, int32_t *colIdx, float *val_out,
                            int64_t *nnz_out);

/* prep_torch_ppl.py:24-49: sorted unique columns referenced by work group
 * `stage` (rows [stage*gs*npp, min((stage+1)*gs*npp, N))).  out capacity:
 * num_nodes. */
cola_status cola_workgroup_cols(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                int32_t nparts, int32_t group_size, int32_t stage, int32_t *out,
                                int64_t *count);

/* src/distSpMM_ppl_batch.cu:101-193: stage offset and index tables of PE `me`.
 * wg_cols/wg_off: all work groups' column lists concatenated (wg_off has
 * nranks/group_size + 1 entries; may be NULL when group_size == nranks).
 * Outputs: local/remote/put offsets (2*nstages each), idx_ppl lists of stages
 * 1..nstages-1 concatenated with idx_off (nstages entries, idx_off[0] = 0,
 * stage i list = [idx_off[i-1], idx_off[i])), put lists of stages
 * 0..nstages-2 concatenated with put_lst_off (nstages entries). */
cola_status cola_stage_tables(int32_t me, int32_t nranks, int32_t group_size, int32_t num_nodes,
                              const int32_t *csc_colIdx_zip_r, int64_t n_remote_chunks, int64_t n_local_chunks,
                              const int32_t *wg_cols, const int64_t *wg_off, int32_t *local_offset_ppl,
                              int32_t *remote_offset_ppl, int32_t *put_offset_ppl, int32_t *idx_ppl,
                              int64_t *idx_off, int64_t idx_capacity, int32_t *put_colIdx_ppl,
                              int64_t *put_lst_off, int64_t put_capacity);

/* include/dist_spmm_ppl_batch.cuh:7-27 (bin2vec) without its 2 GiB int
 * overflow: raw little-endian int32 files, no header.  Pass out == NULL to
 * size (*count = file bytes / 4). */
cola_status cola_bin_read_i32(const char *path, int32_t *out, int64_t capacity, int64_t *count);
cola_status cola_bin_write_i32(const char *path, const int32_t *data, int64_t n);
cola_status cola_bin_read_f32(const char *path, float *out, int64_t capacity, int64_t *count);
cola_status cola_bin_write_f32(const char *path, const float *data, int64_t n);

/* Write the reference's on-disk layout for this partition set
 * (prep_torch_par.py:56-58,77-79): <dir>/GPU<P>/{csr_rowPtr_l,csr_colIdx_l,
 * csr_rowIdx_l,csc_colPtr_r,csc_rowIdx_r,csc_colIdx_r}_<P>_<r>.bin, plus
 * csr_val_l_/csc_val_r_ FP32 files (the reference writes no values). */
cola_status cola_partition_write_bin(const cola_partition_set *s, const char *dir);
/* Load a partition set from that layout.  Value files are optional (missing
 * values load as 1.0, the reference's choice). */
cola_status cola_partition_read_bin(const char *dir, int32_t num_nodes, int32_t nparts, cola_partition_set **out);

/* Seeded R-MAT graph (a, b, c, 1-a-b-c), scale s -> 2^s nodes.  Draws
 * undirected non-self-loop edges until avg_degree*N/2 distinct ones exist,
 * then symmetrises (each edge both ways), optionally adds self-loops, and
 * sorts by (row, col).  Values: 0 none(1.0), 1 = 1/deg(row), 2 =
 * 1/sqrt(deg(row)*deg(col)).  Two-call protocol: row == NULL returns *nnz. */
cola_status cola_rmat_generate(int32_t scale, double avg_degree, double a, double b, double c, uint64_t seed,
                               int32_t self_loops, int32_t value_kind, int32_t *row, int32_t *col, float *val,
                               int64_t capacity, int64_t *nnz);

/* ========================================================================
 * Kernel-level launchers: drop-ins for the reference's launchers in
 * include/dist_spmm_ppl_batch.cuh, same argument meaning.  FP32, any dim >= 1.
 * `output` is accumulated into (the caller zeroes it, as the reference's
 * caller does: src/distSpMM_ppl_batch.cu:225-226).
 * ====================================================================== */

/* ppl0_batch_SpMM (include/dist_spmm_ppl_batch.cuh:202-245): local CSR chunks
 * [local_row_lb, +local_row_num) and remote CSC chunks [remote_col_lb,
 * +remote_col_num) of PE peid.  input = PE peid's X slice (symmetric
 * convention above); remote rows are staged on chip by the kernel. */
cola_status cola_ppl0_batch_spmm(float *output, const float *input, const int32_t *csr_rowPtr_l,
                                 const int32_t *csr_colIdx_l, const int32_t *csr_rowIdx_zip_l,
                                 const float *csr_val_l, const int32_t *csc_colPtr_r, const int32_t *csc_rowIdx_r,
                                 const int32_t *csc_colIdx_zip_r, const float *csc_val_r, int32_t local_row_lb,
                                 int32_t remote_col_lb, int32_t local_row_num, int32_t remote_col_num,
                                 int32_t dim, int32_t nodesPerPE, int32_t peid, cola_stream_t stream);

/* ppl0_batch_SpMM_seq (include/dist_spmm_ppl_batch.cuh:543-587): same result
 * as cola_ppl0_batch_spmm (the reference's variant only orders work
 * differently). */
cola_status cola_ppl0_batch_spmm_seq(float *output, const float *input, const int32_t *csr_rowPtr_l,
                                     const int32_t *csr_colIdx_l, const int32_t *csr_rowIdx_zip_l,
                                     const float *csr_val_l, const int32_t *csc_colPtr_r,
                                     const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r,
                                     const float *csc_val_r, int32_t local_row_lb, int32_t remote_col_lb,
                                     int32_t local_row_num, int32_t remote_col_num, int32_t dim,
                                     int32_t nodesPerPE, int32_t peid, cola_stream_t stream);

/* ppl0_batch_buffer_SpMM (include/dist_spmm_ppl_batch.cuh:373-417): remote
 * rows are first gathered into comm_buffer (row j of comm_buffer = remote
 * chunk j's column; it must hold remote_col_lb + remote_col_num rows of dim
 * floats), in batches, then consumed from there. */
cola_status cola_ppl0_batch_buffer_spmm(float *output, const float *input, float *comm_buffer,
                                        const int32_t *csr_rowPtr_l, const int32_t *csr_colIdx_l,
                                        const int32_t *csr_rowIdx_zip_l, const float *csr_val_l,
                                        const int32_t *csc_colPtr_r, const int32_t *csc_rowIdx_r,
                                        const int32_t *csc_colIdx_zip_r, const float *csc_val_r,
                                        int32_t local_row_lb, int32_t remote_col_lb, int32_t local_row_num,
                                        int32_t remote_col_num, int32_t dim, int32_t nodesPerPE, int32_t peid,
                                        cola_stream_t stream);

/* Capacity, in floats, of the library's own staging array used by
 * cola_ppl0_batch_buffer_spmm_noalloc (8 MiB; every GPU that loads the library
 * holds it until the process exits). */
#define COLA_NOALLOC_STAGE_FLOATS (2u * 1024u * 1024u)

/* No counterpart in the reference.  The same computation as
 * cola_ppl0_batch_buffer_spmm for callers that cannot allocate device memory
 * and have none to lend: code running under a host framework that owns every
 * device allocation, or a latency-bound loop that must not call cudaMalloc
 * (it synchronises the device and can fail under memory pressure).  Instead of
 * a caller-provided comm_buffer, the remote rows are staged in a fixed array
 * inside the library, so this call allocates nothing.
 * Limit: remote_col_num * dim must not exceed COLA_NOALLOC_STAGE_FLOATS;
 * larger requests return COLA_ERROR_INVALID_ARGUMENT and launch nothing.
 * The first call on a device looks up the array's device address (once per
 * device, and again after that device's context was reset, e.g. by
 * cudaDeviceReset); make that first call before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (on different streams, or from
 * different threads) race on it and must be serialised by the caller.  The
 * array keeps whatever the last call left in it; every call overwrites the
 * rows it reads before reading them. */
cola_status cola_ppl0_batch_buffer_spmm_noalloc(float *output, const float *input, const int32_t *csr_rowPtr_l,
                                                const int32_t *csr_colIdx_l, const int32_t *csr_rowIdx_zip_l,
                                                const float *csr_val_l, const int32_t *csc_colPtr_r,
                                                const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r,
                                                const float *csc_val_r, int32_t local_row_lb, int32_t remote_col_lb,
                                                int32_t local_row_num, int32_t remote_col_num, int32_t dim,
                                                int32_t nodesPerPE, int32_t peid, cola_stream_t stream);

/* The row view of the chunks one ppl0_batch_SpMM call covers
 * (include/dist_spmm_ppl_batch.cuh:202-245, the arguments of
 * cola_ppl0_batch_spmm without the dense ones): the local CSR chunks
 * [local_row_lb, +local_row_num) and remote CSC chunks [remote_col_lb,
 * +remote_col_num) of PE peid, merged per output row in column order on the
 * device (long rows split into segments, as cola_graph_upload does).  Built once
 * (synchronises `stream`; needs about 12 bytes of device memory per entry
 * while it runs and keeps about 8 per entry); the zip arrays are not read
 * again.  cola_zip_rows_spmm then adds the same product as
 * cola_ppl0_batch_spmm to `output` with the row-major schedule: one writer
 * per row, no atomics, the same bits on every call.  compat.h's
 * ppl0_batch_SpMM builds and keeps one for every d_csr_zip / d_csc_zip pair
 * it is called with. */
typedef struct cola_zip_rows cola_zip_rows;
cola_status cola_zip_rows_create(const int32_t *csr_rowPtr_l, const int32_t *csr_colIdx_l,
                                 const int32_t *csr_rowIdx_zip_l, const float *csr_val_l, const int32_t *csc_colPtr_r,
                                 const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r, const float *csc_val_r,
                                 int32_t local_row_lb, int32_t remote_col_lb, int32_t local_row_num,
                                 int32_t remote_col_num, int32_t nodesPerPE, int32_t peid, cola_stream_t stream,
                                 cola_zip_rows **out);
/* One PE's arguments for cola_zip_rows_create_all: its zip arrays and the
 * chunk ranges its ppl0_batch_SpMM call covers. */
typedef struct cola_zip_part {
    const int32_t *csr_rowPtr_l, *csr_colIdx_l, *csr_rowIdx_zip_l;
    const float *csr_val_l;
    const int32_t *csc_colPtr_r, *csc_rowIdx_r, *csc_colIdx_zip_r;
    const float *csc_val_r;
    int32_t local_row_lb, remote_col_lb, local_row_num, remote_col_num;
} cola_zip_part;
/* The row view of every PE's call at once (PE p = parts[p], its output rows
 * starting at row p*nodesPerPE of the symmetric output): one
 * cola_zip_rows_spmm(h, output, input, dim) with output and input at PE 0's
 * slices then adds what the nparts per-PE calls add, in one launch (plus one
 * for hub rows) instead of one per PE. */
cola_status cola_zip_rows_create_all(const cola_zip_part *parts, int32_t nparts, int32_t nodesPerPE,
                                     cola_stream_t stream, cola_zip_rows **out);
/* output[r] += sum of the covered entries of row r times input rows (input =
 * PE peid's slice of the symmetric X, as for cola_ppl0_batch_spmm); FP32,
 * any dim >= 1.  Asynchronous on `stream`. */
cola_status cola_zip_rows_spmm(cola_zip_rows *h, float *output, const float *input, int32_t dim,
                               cola_stream_t stream);
cola_status cola_zip_rows_free(cola_zip_rows *h);
/* Rows spanned (up to the last with an entry), entries, hub rows, device bytes held. */
cola_status cola_zip_rows_get_info(const cola_zip_rows *h, int64_t *rows, int64_t *nnz, int64_t *hub_rows,
                                   int64_t *device_bytes);

/* ppl_batch_SpMM (include/dist_spmm_ppl_batch.cuh:709-760): stage-i CSC
 * scatter over remote chunks [remote_col_lb, remote_col_ub).  Chunks in
 * [local_col_lb, local_col_ub) read row idx_ppl[w] of `input` (this PE's
 * received pipeline buffer); the others read row idx_ppl[w] of group peer
 * (col/npp) % group_size + group_offset's buffer (symmetric convention). */
cola_status cola_ppl_batch_spmm(float *output, const float *input, const int32_t *csc_colPtr_r,
                                const int32_t *csc_rowIdx_r, const int32_t *csc_colIdx_zip_r,
                                const float *csc_val_r, int32_t local_col_lb, int32_t local_col_ub,
                                int32_t remote_col_lb, int32_t remote_col_ub, int32_t stage,
                                const int32_t *idx_ppl, int32_t dim, int32_t nodesPerPE, int32_t group_size,
                                int32_t group_offset, int32_t peid, cola_stream_t stream);

/* batching_data_ppl (include/dist_spmm_ppl_batch.cuh:59-73): the staged
 * gather send[b,:] = input[put_colIdx[b] % nodesPerPE, :], b < nemb. */
cola_status cola_batching_data_ppl(const float *input, float *send, const int32_t *put_colIdx, int32_t nemb,
                                   int32_t dim, int32_t nodesPerPE, int32_t group_size, cola_stream_t stream);

/* ========================================================================
 * Graph-level API: device-resident partitions, all P virtual PEs in one call.
 * Replaces distSpMM_ppl_batch / distSpMM_ppl_batch_wrapper
 * (include/dist_spmm_ppl_batch.cuh:762-918) on one GPU.
 * ====================================================================== */

typedef struct cola_graph cola_graph;

typedef struct cola_upload_opts {
    int32_t if_split;       /* nnz_split the remote CSC too (src/distSpMM_ppl_batch.cu:86-98); 1 = yes */
    int32_t group_size;     /* work-group size for the pipelined schedule; 0 or nparts = single stage */
    int32_t no_row_view;    /* 1: skip the row-major view (COLA_SCHEDULE_ROWS unavailable, less memory) */
    int32_t hub_threshold;  /* ROWS: rows with more entries are split into segments; 0 = T */
    int32_t hub_segment;    /* ROWS: entries per hub segment; 0 = T */
    int32_t task_entries;   /* ROWS: entries per row-block task (one warp each); 0 = T / 2.
                               T = 512 if nnz >= 512 x 16 x 32 x SMs (16 or more 512-entry items
                               per warp of a full wave), 128 if nnz < 128 x 4 x 32 x SMs, else 256 */
    int32_t reserved[2];
} cola_upload_opts;

/* Splits, builds stage tables and uploads every partition to the current
 * device.  opts may be NULL (if_split = 1, group_size = nparts). */
cola_status cola_graph_upload(const cola_partition_set *parts, const cola_upload_opts *opts, cola_graph **out,
                              cola_stream_t stream);
cola_status cola_graph_free(cola_graph *g);

/* A graph for the row-major schedule (COLA_SCHEDULE_ROWS, what AUTO picks)
 * built straight from the COO in device memory: entries sorted by (row, col)
 * with duplicates merged, row pointers, hub segments and row-block tasks, all
 * on the device, identical to what cola_graph_upload derives from the
 * partitions of the same COO (so every SpMM gives the same bits).  It has no
 * split blocks: the FUSED, BUFFER and PIPELINE schedules and
 * cola_graph_zip_view refuse it.  opts: hub_threshold, hub_segment and
 * task_entries as for cola_graph_upload (may be NULL).  Free with
 * cola_graph_free. */
cola_status cola_graph_build_device(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                    const float *val, int32_t nparts, const cola_upload_opts *opts,
                                    cola_stream_t stream, cola_graph **out);


typedef struct cola_graph_info {
    int32_t num_nodes, nparts, nodes_per_part, group_size;
    int64_t nnz, nnz_local, nnz_remote;
    int64_t local_chunks, remote_chunks, remote_cols;
    int64_t device_bytes;
    int64_t hub_rows, hub_segments;  /* ROWS schedule */
    int64_t row_tasks;               /* ROWS schedule: row blocks of about task_entries entries */
    int64_t last_launches;           /* kernels the last cola_spmm call on this graph launched */
} cola_graph_info;
cola_status cola_graph_get_info(const cola_graph *g, cola_graph_info *out);

/* Staged row gathers (BUFFER staging, PIPELINE puts, cola_batching_data_ppl)
 * move rows with 16-byte vector loads and stores (enable = 0, the default), or
 * with bulk asynchronous copies through shared memory (enable = 1) for rows of
 * 1 KB or more whose addresses are all 16-byte aligned.  Same results either
 * way; on a B200 the vector gather measured as fast or faster. */
cola_status cola_set_gather_bulk(int32_t enable);

/* How many times the bulk-copy gather polls for one row's load before it gives
 * up (0 = the default, 4,194,304 polls: at least a quarter of a second).  A
 * wait that gives up makes that launch stop early and drain the loads it
 * issued; cola_device_error_check then reports it.  Small values exist to
 * exercise that path. */
cola_status cola_set_gather_wait_limit(int64_t polls);

/* The row-gather ceiling of the current device: warps read whole rows of
 * row_bytes (16..512) from a table of table_bytes at pseudo-random row indices
 * (16-byte loads, 4 rows in flight per warp, one full wave), `gathers` rows per
 * run, `reps` timed runs after one warm-up run; *gbps = row bytes read per
 * second.  A table that fits in L2 measures the L2 ceiling of the SpMM's
 * gathers, a table far larger than L2 the DRAM ceiling.  Allocates the table
 * (stream-ordered) and synchronises `stream`. */
cola_status cola_probe_gather(int64_t table_bytes, int32_t row_bytes, int64_t gathers, int32_t reps,
                              cola_stream_t stream, double *gbps);

/* The same ceiling for one graph's own access pattern: warps walk the row
 * view's entries in order, 32 at a time, and read the row_bytes (16..2048) of X
 * each entry names (rows ld_bytes apart), with no arithmetic and no writes.
 * *gbps = entries x row_bytes per second over `reps` passes after a warm-up
 * pass; *ms_per_pass (may be NULL) the time of one pass.  The SpMM kernel's
 * time against this one is its overhead over the memory system's time for
 * exactly its gathers.  Synchronises `stream`. */
cola_status cola_probe_graph_gather(const cola_graph *g, const void *X, int64_t ld_bytes, int32_t row_bytes,
                                    int32_t reps, cola_stream_t stream, double *gbps, float *ms_per_pass);

/* Waits for the current device, then reports (and clears) the error code a
 * kernel left when one of its bounded waits ran out: 0 = none; 1 = a bulk-copy
 * gather stopped early (it drained every copy it had issued before exiting);
 * 2 = as 1, and a drain also ran out (a copy may have still been in flight when
 * its block exited).  Any nonzero code means that the results of every launch
 * on the device since the previous check must not be used; after code 2 the
 * device should not be trusted for further work in this process. */
cola_status cola_device_error_check(int32_t *code);

/* Device pointers of partition `part`'s split arrays (the d_csr_zip / d_csc_zip
 * members of include/sparse_data.h:28-77) and its chunk counts. */
typedef struct cola_zip_view {
    const int32_t *csr_rowPtr, *csr_colIdx, *csr_rowIdx_zip;
    const float *csr_val;
    const int32_t *csc_colPtr, *csc_rowIdx, *csc_colIdx_zip;
    const float *csc_val;
    int32_t local_chunks, remote_chunks;
    int64_t nnz_l, nnz_r;
} cola_zip_view;
cola_status cola_graph_zip_view(const cola_graph *g, int32_t part, cola_zip_view *out);

enum cola_schedule {
    COLA_SCHEDULE_AUTO = 0,     /* ROWS when the graph has its row view (the fastest measured), else
                                   PIPELINE for group_size < nparts, else FUSED */
    COLA_SCHEDULE_FUSED = 1,    /* one launch: local CSR + remote CSC, rows staged on chip */
    COLA_SCHEDULE_BUFFER = 2,   /* remote rows gathered into an HBM staging buffer in batches first */
    COLA_SCHEDULE_PIPELINE = 3, /* the reference's multi-stage work-group schedule */
    COLA_SCHEDULE_ROWS = 4      /* row-major view (remote CSC transposed at upload, merged with the
                                   local CSR): one writer per output row, no atomics, deterministic;
                                   hub rows split into segments combined pairwise */
};

typedef struct cola_spmm_opts {
    int32_t accumulate;         /* 0: Y is overwritten; 1: Y += A X (Y must be FP32) */
    int32_t schedule;           /* enum cola_schedule */
    int32_t gather_batch_rows;  /* staging batch (rows) for BUFFER/PIPELINE; 0 = 4096 */
    int32_t unroll;             /* ROWS: row loads in flight per lane group (2, 4, 6 or 8; 0 = 4) */
    int32_t min_blocks;         /* ROWS: resident blocks per SM the kernel is compiled for (3, 4, 5, 6;
                                   0 = 3 for FP32 X, 4 for BF16 X) */
    int32_t k_tile;             /* ROWS, K >= 128 (FP32 X) or >= 256 (BF16 X): features per pass over the
                                   graph (64, 128, 256, 512, 1024; 0 = chosen by the library).  The passes
                                   run one after another so the X columns in use are one tile wide; every
                                   choice gives the same bits.  Ignored for narrower K. */
    int32_t reserved[2];
} cola_spmm_opts;

/* Y = A X (or Y += A X) for all partitions.  X: >= P*npp rows (rows past N are
 * read only if the caller's X has them; padding rows are never referenced),
 * ldx >= K elements; Y: N rows, ldy >= K.  x_dtype FP32 or BF16 (BF16 is
 * widened exactly and accumulated in FP32); y_dtype FP32 or BF16 (rounded
 * once, at the end).  opts may be NULL.  The ROWS schedule hands its work
 * items (hub segments, row blocks) to warps from counters kept in the graph,
 * and hub rows' partial sums go to a workspace of the graph: calls on one
 * graph that overlap on the GPU (different streams or threads) race on both
 * and must be serialised by the caller; calls on one stream are. */
cola_status cola_spmm(cola_graph *g, const void *X, cola_dtype x_dtype, int64_t ldx, void *Y, cola_dtype y_dtype,
                      int64_t ldy, int32_t K, const cola_spmm_opts *opts, cola_stream_t stream);

/* The project's autotuner for one graph: times every candidate launch option
 * of `schedule` (AUTO picks as cola_spmm does) on these operands with CUDA
 * events, `reps` runs each after a warm-up, and returns the fastest in *best
 * (schedule, k_tile, unroll, min_blocks, gather_batch_rows; accumulate 0).
 * Row-major schedule: feature tile per pass x loads in flight x resident
 * blocks per SM; for K >= 128 (FP32 X) or >= 256 (BF16 X) every candidate
 * gives the same bits, narrower K has a single geometry.  Buffer and pipelined
 * schedules: the remote-row gather batch (1,024 to 16,384 rows).  Y is
 * overwritten; synchronises `stream`.  cache_path (may be NULL): a text file
 * of tuned results keyed by device model, SM count, graph shape, K, dtypes and
 * schedule; a hit returns its line without timing anything (*from_cache = 1),
 * a miss appends one. */
cola_status cola_spmm_autotune(cola_graph *g, const void *X, cola_dtype x_dtype, int64_t ldx, void *Y,
                               cola_dtype y_dtype, int64_t ldy, int32_t K, int32_t schedule, int32_t reps,
                               const char *cache_path, cola_stream_t stream, cola_spmm_opts *best, float *best_ms,
                               int32_t *from_cache);

/* Y = A X with X and Y in host memory (pinned memory lets the copies run
 * asynchronously): X is copied in, multiplied as cola_spmm does (opts as
 * there; accumulate is not supported) and Y copied out, asynchronously.  The
 * graph keeps two device staging sets and two copy streams of its own, so
 * consecutive calls overlap: call i + 1's upload runs while call i's result
 * downloads, and the SpMMs run on `stream`.  X_host must hold the features
 * when the call is made and stay unchanged, and Y_host untouched, until the
 * call's work is complete: cola_spmm_host_sync(g) waits for every call made
 * on the graph so far.  The staging sets (N x K elements of each dtype, twice)
 * are allocated by the first calls and kept with the graph. */
cola_status cola_spmm_host(cola_graph *g, const void *X_host, cola_dtype x_dtype, int64_t ldx, void *Y_host,
                           cola_dtype y_dtype, int64_t ldy, int32_t K, const cola_spmm_opts *opts,
                           cola_stream_t stream);
cola_status cola_spmm_host_sync(cola_graph *g);
/* Makes `stream` wait (without blocking the host) for every cola_spmm_host
 * call made on the graph so far, Y downloads included. */
cola_status cola_spmm_host_join(cola_graph *g, cola_stream_t stream);

/* ========================================================================
 * Batched form: many graphs of uneven size, each with its own X, Y and
 * feature width, in one persistent launch (plus one for hub rows).
 * ====================================================================== */

typedef struct cola_batch cola_batch;

/* Upload ngraphs partition sets (each split and given its row view, as
 * cola_graph_upload does); opts applies to all of them and may be NULL. */
cola_status cola_batch_create(const cola_partition_set *const *parts, int32_t ngraphs, const cola_upload_opts *opts,
                              cola_batch **out, cola_stream_t stream);
/* A batch over graphs that already exist (cola_graph_upload with the row
 * view, or cola_graph_build_device).  The batch borrows them (free the batch
 * first, then the graphs) and uses each graph's hub workspace, so a graph of
 * the batch must not run elsewhere while the batch runs. */
cola_status cola_batch_create_from_graphs(cola_graph *const *graphs, int32_t ngraphs, cola_batch **out);
cola_status cola_batch_free(cola_batch *b);

/* Bind graph g's dense operands: X[g] (>= N_g rows, ldx[g]), Y[g] (N_g rows,
 * ldy[g]), width K[g]; every X in x_dtype, every Y in y_dtype.  Sizes the
 * workspaces and uploads the launch descriptors (synchronises `stream`); call
 * it again when a pointer changes.  Graphs whose operands are not 16-byte
 * vectors (K not a multiple of 4 FP32 / 8 BF16, unaligned rows) run through
 * cola_spmm inside cola_batch_run instead of the batched launch. */
cola_status cola_batch_bind(cola_batch *b, const void *const *X, const int64_t *ldx, void *const *Y,
                            const int64_t *ldy, const int32_t *K, cola_dtype x_dtype, cola_dtype y_dtype,
                            cola_stream_t stream);

/* Y[g] = A_g X[g] (or +=, opts->accumulate) for every bound graph.  Only
 * kernel launches on `stream`: no allocation, no synchronisation. */
cola_status cola_batch_run(cola_batch *b, const cola_spmm_opts *opts, cola_stream_t stream);

/* Record cola_batch_run into a CUDA graph kept by the batch (replaced by the
 * next capture or bind), and launch it. */
cola_status cola_batch_capture(cola_batch *b, const cola_spmm_opts *opts, cola_stream_t stream);
cola_status cola_batch_replay(cola_batch *b, cola_stream_t stream);

/* Launch parameters of the batched kernel: loads in flight per lane group (2
 * or 4), the persistent grid as a percentage of one full wave and the resident
 * blocks per SM it is compiled for (3 or 4). */
cola_status cola_batch_set_params(cola_batch *b, int32_t unroll, int32_t grid_pct, int32_t blocks_per_sm);

/* The project's autotuner for the batched launch: times every candidate
 * (blocks per SM x unroll x grid size) on the bound operands with CUDA events, `reps` runs
 * each, and keeps the fastest (synchronises `stream`). */
cola_status cola_batch_autotune(cola_batch *b, int32_t reps, cola_stream_t stream, float *best_ms);

/* cola_batch_autotune with a cache file: when cache_path holds a line for this
 * batch (same device model and SM count, same graph sizes, widths and dtypes)
 * its parameters are applied without timing anything (*from_cache = 1);
 * otherwise the batch is tuned and a line appended (*from_cache = 0).  Text,
 * one line per batch: "<key> <unroll> <grid_pct> <blocks_per_sm> <best_ms>";
 * lines that do not parse or hold invalid values are ignored. */
cola_status cola_batch_autotune_cached(cola_batch *b, int32_t reps, const char *cache_path, cola_stream_t stream,
                                       float *best_ms, int32_t *from_cache);

typedef struct cola_batch_info {
    int32_t ngraphs, batched_graphs;
    int64_t work_items, hub_items, nnz, device_bytes;
    int32_t unroll, grid_pct, blocks_per_sm;
    int64_t last_launches;
} cola_batch_info;
cola_status cola_batch_get_info(const cola_batch *b, cola_batch_info *out);

/* ========================================================================
 * Serving loop: resident graphs, requests admitted by a device-memory
 * budget, grouped by feature width and dtype into one batched launch across
 * graphs, several groups in flight on separate streams.
 * ====================================================================== */

typedef struct cola_server cola_server;

typedef struct cola_server_opts {
    int64_t memory_budget;  /* device bytes for registered graphs + in-flight requests; 0 = 120 GiB */
    int32_t slots;          /* groups in flight at once (one CUDA stream each); 0 = 4 */
    int32_t max_group;      /* requests of one (K, dtypes) launched together; 0 = 16 */
    int32_t group_mib;      /* host<->device MiB (X in + Y out) past which a group takes no more
                               requests, so large requests pipeline copies against other groups'
                               launches instead of waiting for one long copy phase; 0 = 32 */
    int32_t small_mib;      /* size classes: a request with at most this many MiB of host<->device
                               copies is small; one slot is kept for small requests, and a small
                               request may be admitted ahead of a large one that waits for a slot
                               or memory (the memory the waiting one needs stays reserved for it).
                               0 = 16; -1 = no size classes (plain FIFO) */
    int32_t copy_chunk_mib; /* copies move in pieces of at most this many MiB, so that another
                               slot's copies can run between the pieces of a long one; 0 = 32 */
    int32_t copy_engines_only; /* 0: a small group's copies (and its launch descriptors) are made by
                                  a kernel reading and writing the pinned host buffers directly, so
                                  they do not queue behind other slots' copies in the copy engines
                                  (used when every host buffer is pinned, device-addressable and
                                  16-byte aligned); 1: every copy by the copy engines */
} cola_server_opts;

/* Create a server on the current device (opts may be NULL).  A scheduler
 * thread admits requests as slots and memory free up. */
cola_status cola_server_create(const cola_server_opts *opts, cola_server **out);
/* Cancel what is still pending, wait for what is on the GPU, free everything. */
cola_status cola_server_destroy(cola_server *s);

/* Upload a partition set (split + row view) and keep it resident; its device
 * bytes count against the budget (COLA_ERROR_BUDGET if they do not fit). */
cola_status cola_server_register(cola_server *s, const cola_partition_set *parts, const cola_upload_opts *opts,
                                 int32_t *graph_id);

/* Register a graph that already exists (cola_graph_upload with the row view,
 * or cola_graph_build_device).  The server takes ownership of g in every case
 * (it is freed on failure and at cola_server_destroy). */
cola_status cola_server_register_graph(cola_server *s, cola_graph *g, int32_t *graph_id);

/* Queue Y = A_graph X.  X_host: N x K row-major host memory in x_dtype (pinned
 * memory lets the copies overlap); Y_host: N x K in y_dtype, written when the
 * request completes.  Both must stay valid until cola_server_wait returns.
 * K must be a multiple of 4 (FP32 X) or 8 (BF16 X).  Returns at once with the
 * request id; COLA_ERROR_BUDGET if the request could never fit the budget
 * beside the registered graphs. */
cola_status cola_server_submit(cola_server *s, int32_t graph_id, const void *X_host, cola_dtype x_dtype, int32_t K,
                               void *Y_host, cola_dtype y_dtype, uint64_t *request_id);

/* Wait for a request (timeout_ms < 0: no limit).  COLA_SUCCESS: Y_host holds
 * the result; COLA_ERROR_TIMEOUT: still pending or running (call again);
 * COLA_ERROR_CANCELLED / other: the request did not run.  A finished request
 * is forgotten after its wait returns. */
cola_status cola_server_wait(cola_server *s, uint64_t request_id, int32_t timeout_ms);

/* Cancel a request that has not been admitted yet (COLA_ERROR_NOT_READY if it
 * is already on the GPU or finished). */
cola_status cola_server_cancel(cola_server *s, uint64_t request_id);

typedef struct cola_server_stats {
    int64_t submitted, completed, rejected, cancelled, failed, pending;
    int32_t inflight, max_inflight, groups_launched, max_group;
    int64_t bytes_in_use, peak_bytes, budget;
    double p50_ms, p99_ms, max_ms, mean_ms;  /* submit -> result in host memory */
    double req_per_s;                        /* completed / (last completion - first submission) */
    double queue_ms_mean;                    /* submit -> the group's launch, per request */
    /* per group, from CUDA events on the slot's stream: */
    double copy_in_ms_mean, kernel_ms_mean, copy_out_ms_mean;
} cola_server_stats;
cola_status cola_server_get_stats(cola_server *s, cola_server_stats *out);
/* Start a new measurement window: counts, latencies and peaks restart from
 * the requests submitted after this call (in-flight work is unaffected). */
cola_status cola_server_reset_stats(cola_server *s);

#ifdef __cplusplus
}
#endif
#endif /* COLA_SPMM_H */
