/*
 * abhsf_gpu.h -- C ABI of the B200 (sm_100a) ABHSF builder and SpMV.
 *
 * Drop-in for the reference's per-format call surface
 *   from_elements(elements_t&, const matrix_properties&)   build
 *   spmv(const real_type* x, real_type* y)                  y += A x
 *   release()                                               free
 * (spmv/unified/spmv.cpp:74-127,140-159,210-226; spmv/bottlenecks/spmv.cpp:43-64,
 * 125-133; spmv/orig/88.cpp:150-236) and for the block-statistics tools
 * (block_statistics/block_stats.cpp:69-100, block_statistics/mmf.cpp:53-138,
 * include/abhsf/msmf.h:9-63).
 *
 * Conventions: every call returns abhsf_status and never throws; the reason
 * for the last failure on the calling thread is abhsf_last_error_string().
 * Indices are 0-based (matrix_market_reader.h:135-136).  A handle owns all of
 * its device memory.  Calls taking a stream are ordered on it; a NULL stream
 * is the legacy default stream.  abhsf_stats_get may be called from several
 * threads at once.  abhsf_spmv keeps a work counter in the handle: SpMVs on
 * one handle must not overlap on the GPU (queue them on one stream, or order
 * the streams).  abhsf_spmv_host, abhsf_export_host and abhsf_release need
 * exclusive use of the handle.
 *
 * Format (device arrays, s = block size, M = ceil(m/s), T = nonzero tiles):
 *   brow_ptr[M+1]  int64  tiles of block row I are [brow_ptr[I], brow_ptr[I+1])
 *   tile_col[T]    uint32 block column J, ascending within a block row
 *   tile_nnz[T]    uint32 nonzeros of the tile
 *   tile_scheme[T] uint8  ABHSF_SCHEME_*
 *   tile_val_off[T+1] int64  first stored value of the tile
 *   tile_idx_off[T+1] int64  first payload byte of the tile (16-byte aligned)
 *   payload: COO    uint16 (lrow << log2 s) | lcol per nonzero
 *            CSR    uint16 row_end[s] (nonzeros in rows <= r), uint8 lcol[nnz]
 *            bitmap uint64 words; bit lrow*s + lcol, LSB first
 *            dense  none
 *            each tile's payload zero-padded to a multiple of 16 bytes
 *   values: nonzeros in row-major order inside the tile; dense tiles store
 *           all s*s entries, zeros included.
 */
#ifndef ABHSF_GPU_H
#define ABHSF_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ABHSF_ABI_VERSION 1

#if defined(__GNUC__)
#define ABHSF_API __attribute__((visibility("default")))
#else
#define ABHSF_API
#endif

/* Same object as cudaStream_t / CUstream. */
typedef struct CUstream_st* abhsf_stream_t;

typedef enum abhsf_status {
    ABHSF_SUCCESS = 0,
    ABHSF_ERROR_INVALID_VALUE = 1,      /* bad argument or option */
    ABHSF_ERROR_INDEX_OUT_OF_RANGE = 2, /* an element outside m x n */
    ABHSF_ERROR_DUPLICATE_ENTRY = 3,    /* two elements at one (row, col) */
    ABHSF_ERROR_OUT_OF_MEMORY = 4,
    ABHSF_ERROR_UNSUPPORTED = 5,        /* valid request this build does not handle */
    ABHSF_ERROR_CUDA = 6                /* CUDA runtime error, see the error string */
} abhsf_status;

typedef enum abhsf_scheme {
    ABHSF_SCHEME_COO = 0,
    ABHSF_SCHEME_CSR = 1,
    ABHSF_SCHEME_BITMAP = 2,
    ABHSF_SCHEME_DENSE = 3
} abhsf_scheme;

typedef enum abhsf_value_type {
    ABHSF_VALUE_F64 = 0,
    ABHSF_VALUE_F32 = 1, /* RN(f64) */
    ABHSF_VALUE_BF16 = 2 /* RNE(RN_f32(f64)) */
} abhsf_value_type;

/* Summation order of y += A x.  REFERENCE adds each row's products one at a
 * time, columns ascending, onto y (each product rounded first): bitwise the
 * result of the reference's CSR spmv_naive (spmv/bottlenecks/spmv.cpp:58-64).
 * TREE sums each row with warp-level reduction trees (error within the usual
 * n u (|A||x|) bound, bitwise reproducible run to run). */
typedef enum abhsf_sum_order {
    ABHSF_SUM_REFERENCE = 0,
    ABHSF_SUM_TREE = 1
} abhsf_sum_order;

/* Bits of the per-matrix device status word (abhsf_device_status). */
#define ABHSF_DEVSTAT_WAIT_TIMEOUT 1 /* a bounded copy wait gave up; that SpMV's y is incomplete */

/* include/abhsf/utils/matrix_properties.h:8-14 */
typedef enum abhsf_matrix_type {
    ABHSF_MATRIX_BINARY = 0,
    ABHSF_MATRIX_INTEGER = 1,
    ABHSF_MATRIX_REAL = 2,
    ABHSF_MATRIX_COMPLEX = 3
} abhsf_matrix_type;

/* How abhsf_build picks the block size when opts.block_size is 0.  MINBSS
 * builds the block histograms of all five sizes and takes the one of least
 * ABHSF storage, ties to the smaller (block_statistics/min-bss.cpp:14-58).
 * LEARNED computes ABHSF_FEATURES features in one pass and lets a small MLP
 * predict that size.  LEARNED_TIME does the same with the MLP trained on the
 * library's measured SpMV time at each size: it predicts the fastest size,
 * not the smallest.  AUTOTUNE builds the matrix at every size and keeps the
 * one whose SpMV (abhsf_spmv, or abhsf_spmv_f32 for f32 / bf16 values) ran
 * fastest on the stream (abhsf_autotune, 10 timed calls each).  Whichever
 * selector, only the block size is chosen: every tile's scheme, indices and
 * values follow from it exactly. */
typedef enum abhsf_selector {
    ABHSF_SELECT_MINBSS = 0,
    ABHSF_SELECT_LEARNED = 1,
    ABHSF_SELECT_AUTOTUNE = 2,
    ABHSF_SELECT_LEARNED_TIME = 3
} abhsf_selector;

/* The learned selector's MLP: ABHSF_FEATURES inputs, two hidden layers of
 * ABHSF_MLP_HIDDEN ReLU units, ABHSF_MLP_CLASSES outputs (block size 16 << k),
 * FP32.  A model is ABHSF_MLP_PARAMS floats laid out as
 *   W1[F][H] b1[H] W2[H][H] b2[H] W3[H][C] b3[C] mean[F] inv_std[F]
 * (row-major, h = relu(x W + b)); the network's input is
 * (features - mean) * inv_std. */
#define ABHSF_FEATURES 12
#define ABHSF_MLP_HIDDEN 64
#define ABHSF_MLP_CLASSES 5
#define ABHSF_MLP_PARAMS (ABHSF_FEATURES * ABHSF_MLP_HIDDEN + ABHSF_MLP_HIDDEN + \
                          ABHSF_MLP_HIDDEN * ABHSF_MLP_HIDDEN + ABHSF_MLP_HIDDEN + \
                          ABHSF_MLP_HIDDEN * ABHSF_MLP_CLASSES + ABHSF_MLP_CLASSES + 2 * ABHSF_FEATURES)

typedef struct abhsf_build_opts {
    int32_t block_size;       /* s: 16, 32, 64, 128 or 256; 0 = chosen by `selector` */
    int32_t value_type;       /* abhsf_value_type of the stored values */
    int32_t allow_csr;        /* 1: block_min_msmf (msmf.h:35-48); 0: block_min_msmf_wocsr (msmf.h:50-63) */
    int32_t matrix_type;      /* abhsf_matrix_type; BINARY never selects dense and stores 1.0 values */
    int32_t forced_scheme;    /* -1: minimum storage; 0..3: this scheme for every tile */
    int32_t inputs_on_device; /* rows / cols / vals are device pointers */
    int32_t sum_order;        /* abhsf_sum_order of abhsf_spmv / abhsf_spmv_host */
    int64_t bits_per_value;   /* dense-cost element width; 0 = width of value_type */
    int32_t selector;         /* abhsf_selector, used when block_size is 0 */
    int32_t slice_tile_nnz;   /* reference-order SpMV: block rows without a dense tile that have no bitmap
                                 tile, whose tiles hold at most this many elements on average, or that
                                 have more than 256 tiles, are summed from delta-coded row slices;
                                 0 = the library's default (32), -1 = none */
    const float* selector_model; /* host, ABHSF_MLP_PARAMS floats; NULL = the model built into the library */
} abhsf_build_opts;

/* include/abhsf/utils/matrix_properties.h:17-23 (kept apart from abhsf_matrix_type) */
typedef enum abhsf_symmetry {
    ABHSF_SYMMETRY_SYMMETRIC = 0,
    ABHSF_SYMMETRY_HERMITIAN = 1,
    ABHSF_SYMMETRY_SKEW = 2,
    ABHSF_SYMMETRY_GENERAL = 3
} abhsf_symmetry;

/* A matrix read from a file into host memory (abhsf_read_mtx): 0-based COO
 * arrays of nnz elements, allocated by the library, freed by
 * abhsf_coo_host_free. */
typedef struct abhsf_coo_host {
    int64_t m, n, nnz;
    int32_t matrix_type;     /* ABHSF_MATRIX_REAL or ABHSF_MATRIX_BINARY (values 1.0) */
    int32_t symmetry;        /* abhsf_symmetry of the file */
    int32_t stored_triangle; /* symmetric files: 1 lower, 2 upper (the part stored, not expanded); else 0 */
    int32_t reserved;
    int64_t* rows;
    int64_t* cols;
    double* vals;
} abhsf_coo_host;

/* A matrix read from a file into device memory (abhsf_read_mtx_device): the
 * fields of abhsf_coo_host, with rows, cols and vals in device memory
 * (allocated by the library on the current device, freed by
 * abhsf_coo_device_free), and how many entries the host parsed instead of the
 * device (spellings other than plain decimal numbers). */
typedef struct abhsf_coo_device {
    int64_t m, n, nnz;
    int32_t matrix_type;
    int32_t symmetry;
    int32_t stored_triangle;
    int32_t reserved;
    int64_t* rows;
    int64_t* cols;
    double* vals;
    int64_t host_parsed;
} abhsf_coo_device;

typedef struct abhsf_matrix abhsf_matrix;
typedef struct abhsf_batch abhsf_batch;

/* Outcome of abhsf_cg / abhsf_cg_mixed. */
typedef struct abhsf_cg_info {
    int32_t iterations;       /* CG iterations (for the mixed solver: its f32 iterations) */
    int32_t outer_iterations; /* residual replacements of the mixed solver (1 for plain CG) */
    int32_t converged;        /* rel_residual <= rtol */
    int32_t reserved;
    double rel_residual;      /* ||b - A x|| / ||b|| in FP64 with the FP64 matrix, at return */
} abhsf_cg_info;

typedef struct abhsf_stats {
    int64_t m, n, nnz;
    int32_t block_size, value_type;
    int64_t block_rows, block_cols, tiles;
    int64_t tiles_per_scheme[4];
    int64_t nnz_per_scheme[4];
    int64_t stored_values;
    int64_t payload_bytes;
    int64_t format_bytes;   /* all device arrays of the format (B_fmt) */
    uint64_t msmf_bits[8];  /* this block size's mmf line at the dense-cost width:
                               coo32 csr32 coo csr bitmap dense abhsf abhsf134,
                               values included (block_statistics/mmf.cpp:122-138) */
    int64_t spmv_bytes;     /* what one reference-order SpMV reads of the matrix (x and y excluded): the
                               format bytes of the block rows the tile kernel sums, and for the block
                               rows in row slices their words, values, lane records and slice records
                               (format_bytes when no block row is in slices) */
} abhsf_stats;

/* Fills the defaults: s = 64, f64, CSR allowed, REAL, minimum storage, host
 * inputs, reference summation order. */
ABHSF_API void abhsf_build_opts_default(abhsf_build_opts* opts);

/* Builds the format on the GPU from COO triplets (any order, no duplicates).
 * vals may be NULL for BINARY matrices (values 1.0).  Synchronises stream.
 * Replaces from_elements/assemble (spmv/unified/spmv.cpp:74-127,
 * spmv/bottlenecks/spmv.cpp:43-49, spmv/orig/88.cpp:150-202); unlike the
 * reference it leaves the caller's arrays untouched. */
ABHSF_API abhsf_status abhsf_build(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz,
                         int64_t m, int64_t n, const abhsf_build_opts* opts, abhsf_stream_t stream,
                         abhsf_matrix** out);

/* How many kernels one abhsf_spmv of this matrix launches (the tile kernel
 * or the streaming kernel for the block rows it serves, the row-slice kernel
 * and the chain kernel for those in slices).  No counterpart in the
 * reference. */
ABHSF_API abhsf_status abhsf_spmv_kernels(const abhsf_matrix* a, int32_t* kernels);

/* y += A x, x[n] and y[m] float64 in device memory; matrix stored as f64.
 * Replaces spmv(x, y) (spmv/bottlenecks/spmv.cpp:58-64, spmv/orig/88.cpp:204-236). */
ABHSF_API abhsf_status abhsf_spmv(const abhsf_matrix* a, const double* x, double* y, abhsf_stream_t stream);

/* y += A x in f32 for a matrix stored as f32 or bf16: x[n], y[m] float in
 * device memory, values widened to f32, each product and each sum rounded to
 * f32, per row in the reference's column order, at every block size.
 * The reference's f32 kernels (spmv/orig/88.cpp:204-236, value type float)
 * are the counterpart. */
ABHSF_API abhsf_status abhsf_spmv_f32(const abhsf_matrix* a, const float* x, float* y, abhsf_stream_t stream);

/* Solves A x = b by conjugate gradients in FP64 (A symmetric positive
 * definite, stored as f64): b[n] and x[n] in device memory, x holding the
 * initial guess on entry.  Stops when the recurrence residual reaches
 * rtol * ||b|| or after max_iters iterations; info gets the true residual.
 * Ordered after the work queued on stream; returns when the solve is done.
 * No reference counterpart (the reference has SpMV only); this is the
 * solver its SpMV serves. */
ABHSF_API abhsf_status abhsf_cg(const abhsf_matrix* a, const double* b, double* x, double rtol, int32_t max_iters,
                                abhsf_cg_info* info, abhsf_stream_t stream);

/* The same system solved in mixed precision: CG runs in f32 on a_lo (the
 * same matrix stored as f32 or bf16, any block size) with f32 vectors;
 * its solution is folded into x in FP64, and each time its residual has
 * fallen by update_factor (in (0, 1), e.g. 0.1) it is replaced by the FP64
 * residual b - A x of the f64 matrix a64 (a reliable update), the search
 * direction kept.  Stops when ||b - A x|| <= rtol ||b|| at an update, after
 * max_iters iterations, or after max_updates updates.  info.iterations counts
 * f32 iterations, info.outer_iterations the updates. */
ABHSF_API abhsf_status abhsf_cg_mixed(const abhsf_matrix* a64, const abhsf_matrix* a_lo, const double* b, double* x,
                                      double rtol, int32_t max_iters, double update_factor, int32_t max_updates,
                                      abhsf_cg_info* info, abhsf_stream_t stream);

/* A batch: count f64 matrices of one block size, at most 4096 (at block
 * sizes 32 and 64 each with fewer than 2^20 block columns), whose SpMVs run
 * as one launch: the ring kernel at 32 and 64, the streaming kernel at 16,
 * 128 and 256.
 * The matrices stay owned by the caller and must outlive the batch.  The
 * non-empty block rows of all of them are dealt over one grid at creation.
 * No reference counterpart (the reference multiplies one matrix per call). */
ABHSF_API abhsf_status abhsf_batch_create(const abhsf_matrix* const* mats, int32_t count, abhsf_stream_t stream,
                                          abhsf_batch** out);

/* y_i += A_i x_i for every matrix of the batch in one call: one launch of
 * each kernel the matrices need (the tile kernel, the row-slice kernel, and
 * the chain kernel on a side stream forked from `stream` and joined back;
 * abhsf_batch_kernels), in the reference's summation order (each y_i bitwise
 * what abhsf_spmv gives).  xs and ys are DEVICE arrays of count device
 * pointers (x_i of n_i doubles, y_i of m_i), so the call can be captured in
 * a CUDA graph.  Calls on one batch must not overlap on the GPU. */
ABHSF_API abhsf_status abhsf_batch_spmv(const abhsf_batch* b, const double* const* xs, double* const* ys,
                                        abhsf_stream_t stream);

/* How many kernels one abhsf_batch_spmv launches: the tile kernel (when some
 * block row is its: ring or streaming kernel), the row-slice kernel and the
 * chain kernel (when some block row is in slices), 0 to 3.  No counterpart in the reference. */
ABHSF_API abhsf_status abhsf_batch_kernels(const abhsf_batch* b, int32_t* kernels);

/* The batch's device status word (ABHSF_DEVSTAT_* bits), as abhsf_device_status. */
ABHSF_API abhsf_status abhsf_batch_status(abhsf_batch* b, abhsf_stream_t stream, int32_t clear, int32_t* out);

ABHSF_API abhsf_status abhsf_batch_release(abhsf_batch* b);

/* Y += A X for k right-hand sides, X (n x k) and Y (m x k) float64 row-major
 * in device memory: element (i, j) of X at X[i * ldx + j], ldx >= k, and the
 * same for Y with ldy.  Column j of Y gets exactly what abhsf_spmv gives for
 * column j.  In the reference order the matrix is read once per pass of 16
 * or 32 columns when k is a multiple of 16, X and Y are 16-byte aligned and
 * ldx, ldy are even (block sizes 16, 32, 64), else once per pass of up to 8
 * columns (block sizes 32 and 64); otherwise the columns go through
 * abhsf_spmv one at a time.  No reference counterpart: the reference has single-vector
 * SpMV only (spmv/bottlenecks/spmv.cpp:58-64); this is its multi-vector form. */
ABHSF_API abhsf_status abhsf_spmm(const abhsf_matrix* a, int32_t k, const double* X, int64_t ldx, double* Y,
                                  int64_t ldy, abhsf_stream_t stream);

/* The same with x and y in host memory: copies x and y in, runs, copies y
 * back and synchronises.  The drop-in for callers of the reference's
 * host-memory spmv(x, y).  Device staging buffers are allocated on first use
 * and kept by the handle. */
ABHSF_API abhsf_status abhsf_spmv_host(abhsf_matrix* a, const double* x, double* y, abhsf_stream_t stream);

/* Frees the handle and its device memory (release(), spmv/bottlenecks/spmv.cpp:125-133). */
ABHSF_API abhsf_status abhsf_release(abhsf_matrix* a);

/* Format statistics, including the reference's per-scheme storage totals. */
ABHSF_API abhsf_status abhsf_stats_get(const abhsf_matrix* a, abhsf_stats* out);

/* Copies the format arrays (layout above) to host buffers sized from
 * abhsf_stats_get (tiles, stored_values, payload_bytes); NULL skips one. */
ABHSF_API abhsf_status abhsf_export_host(const abhsf_matrix* a, int64_t* brow_ptr, uint32_t* tile_col,
                               uint32_t* tile_nnz, uint8_t* tile_scheme, int64_t* tile_val_off,
                               int64_t* tile_idx_off, uint8_t* payload, void* values);

/* Block histogram for block size r x s (powers of two, 2..256) computed on
 * the GPU: hist[z] = number of r x s blocks holding z nonzeros, for
 * z < hist_len (hist_len >= r*s + 1).  *blocks = nonzero blocks.
 * Replaces process_block_size_powers (block_statistics/block_stats.cpp:69-100). */
ABHSF_API abhsf_status abhsf_block_histogram(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m,
                                   int64_t n, int32_t r, int32_t s, int32_t inputs_on_device,
                                   abhsf_stream_t stream, uint64_t* hist, int64_t hist_len,
                                   int64_t* blocks);

/* Counters abhsf_block_histogram_all writes: the sum over r, s = 2..256 of r*s + 1. */
#define ABHSF_BSTATS_ALL_LEN 260164

/* The block histograms of all 64 block sizes r x s = 2^k x 2^l (k, l = 1..8)
 * in one call, as block_statistics/block_stats.cpp:144-170 writes its 64
 * RxS.bstats files: size p = (k - 1) * 8 + (l - 1) occupies
 * hist[off_p .. off_p + r*s], off_p = the sum of r'*s' + 1 over the sizes
 * before it, and hist[off_p + z] = blocks holding z nonzeros.  blocks[64]
 * (NULL allowed): nonzero blocks of each size.  The reference sorts the
 * elements once per size; here elements sorted by (column >> l, row) put the
 * blocks of all eight heights in runs, so one sort per width serves eight
 * sizes.  Synchronises stream. */
ABHSF_API abhsf_status abhsf_block_histogram_all(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m,
                                                 int64_t n, int32_t inputs_on_device, abhsf_stream_t stream,
                                                 uint64_t* hist, int64_t* blocks);

/* Largest nnz abhsf_block_histogram_noalloc accepts. */
#define ABHSF_NOALLOC_MAX_NNZ 1048576

/* abhsf_block_histogram for callers that may not allocate device memory: no
 * cudaMalloc, cudaFree or allocating library call is made.  Such callers are,
 * for example, programs whose device memory is handed out by their own
 * allocator or pool, code paths where a cudaMalloc (which can synchronise the
 * device) is not acceptable, and processes already at their memory limit.
 * No counterpart in the reference (its block_stats runs on the host).
 * rows and cols are device pointers; nnz <= ABHSF_NOALLOC_MAX_NNZ.  The
 * scratch is one 64 MiB array inside the library's device image, held by
 * every GPU that loads the library until the process exits.  The first call
 * on a device looks up that array's device address, so make it before any
 * stream capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset of that device the kept address is stale, so do not call
 * this entry point again in that process.  All calls share the array: calls
 * whose GPU work overlaps (other streams, other host threads) race on it.
 * Synchronises stream. */
ABHSF_API abhsf_status abhsf_block_histogram_noalloc(const int64_t* rows, const int64_t* cols, int64_t nnz,
                                                     int64_t m, int64_t n, int32_t r, int32_t s,
                                                     abhsf_stream_t stream, uint64_t* hist, int64_t hist_len,
                                                     int64_t* blocks);

/* The delta-coded row slices through which the reference-order SpMV sums the
 * matrix's hypersparse block rows (abhsf_build_opts.slice_tile_nnz): slices,
 * slots (words and values, padding included), lane records, elements and
 * block rows.  The encoding follows the reference's delta COO
 * (spmv/orig/delta.cpp:118-219, spmv/unified/spmv.cpp:815-1032: row by row,
 * each column the difference to the row's previous one).  The block rows go
 * in segments: the quarters [M c / 4, M (c + 1) / 4) that abhsf_spmv_host
 * works through one after another, each cut into pieces of at most 2^24 rows.
 * Per segment, first, block row by block row, every row of more than 256
 * elements as a chain slice (longest first, then ascending row; brow = its
 * block row, meta = the row within it, its elements at slots
 * base .. base + length - 1, each word the absolute column); then the
 * segment's other non-empty rows, ordered by length (longest first, then
 * ascending row), in slices of up to 32 rows, one per lane: brow = the
 * segment's first block row, element k of lane l at slot base + 32 k + l,
 * each word the column minus the row's previous column (the first absolute),
 * lane record l = (row - brow s) << 8 | (length - 1) at meta + l (0 past the
 * slice's rows), steps = the longest row's length.  Values: a copy in slot
 * order; padding slots hold 0. */
ABHSF_API abhsf_status abhsf_slices_info(const abhsf_matrix* a, int64_t* slices, int64_t* slots,
                                         int64_t* lane_records, int64_t* elements, int64_t* block_rows);

/* The slices into host arrays (any may be NULL), in slice order: base, meta
 * (the first lane record, or a chain's row within its block row), block row
 * (a chain's own; a sliced slice's segment's first),
 * steps, lanes, chain flag; the lane records; the words and values of every
 * slot.  No counterpart in the reference (its delta COO lives in host
 * memory). */
ABHSF_API abhsf_status abhsf_slices_export(const abhsf_matrix* a, int64_t* base, int64_t* meta, uint32_t* brow,
                                           uint32_t* steps, uint32_t* lanes, uint8_t* chain,
                                           uint32_t* lane_records, uint32_t* words, void* values);

/* One line of the reference's mmf-single / mmf-double (block_statistics/mmf.cpp:53-138)
 * from props and a block histogram; out_* = coo32 csr32 coo csr bitmap dense abhsf abhsf134. */
ABHSF_API abhsf_status abhsf_mmf_line(int64_t m, int64_t n, int64_t nnz, int32_t matrix_type, int32_t r, int32_t s,
                            const uint64_t* hist, int64_t hist_len, uint64_t out_single[8],
                            uint64_t out_double[8]);

/* Bits of one r x s block with nnz nonzeros under `scheme` (msmf.h:9-33), and
 * the scheme minimum storage selects (msmf.h:35-63, ties COO > CSR > bitmap > dense). */
ABHSF_API uint64_t abhsf_block_scheme_bits(int32_t scheme, int64_t r, int64_t s, int64_t nnz, int64_t bits_per_value);
ABHSF_API int32_t abhsf_block_select_scheme(int64_t r, int64_t s, int64_t nnz, int64_t bits_per_value, int32_t is_binary,
                                  int32_t allow_csr);

/* ABHSF storage in bits (the mmf line's abhsf column, or abhsf134 when
 * opts->allow_csr is 0, at opts' value width) of the square block sizes 16,
 * 32, 64, 128, 256 (bits[k]: size 16 << k), from five block histograms on the
 * GPU, and in *best the size of least storage, ties to the smaller: the
 * exhaustive block-size sweep of block_statistics/min-bss.cpp:14-58 over
 * square sizes.  Uses opts' value_type, allow_csr, matrix_type,
 * inputs_on_device and bits_per_value; NULL opts = defaults.  best may be
 * NULL.  Synchronises stream. */
ABHSF_API abhsf_status abhsf_block_size_storage(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m,
                                                int64_t n, const abhsf_build_opts* opts, abhsf_stream_t stream,
                                                uint64_t bits[5], int32_t* best);

/* Block size by measured time: builds the matrix at each candidate size
 * (bit k of candidates: size 16 << k; 0 = all five), runs one untimed and
 * then reps timed SpMVs of it on stream (x = 0, y = 0 device scratch; the
 * kernels' speed does not depend on the values) and writes the mean time per
 * SpMV in milliseconds to ms[k] (-1 for sizes not timed; abhsf_spmv_f32 for
 * f32 / bf16 values).  *best = the fastest size;
 * out (NULL allowed) receives that size's matrix, which the caller releases.
 * Uses opts as abhsf_build does (block_size ignored).  No counterpart in the
 * reference, which chooses by storage only (block_statistics/min-bss.cpp:14-58).
 * Synchronises stream. */
ABHSF_API abhsf_status abhsf_autotune(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz,
                                      int64_t m, int64_t n, const abhsf_build_opts* opts, int32_t candidates,
                                      int32_t reps, abhsf_stream_t stream, float ms[5], int32_t* best,
                                      abhsf_matrix** out);

/* The learned selector's features of a matrix, computed on the GPU
 * (inputs_on_device: rows / cols are device pointers).  out[12] =
 *   log2 m, log2 n, log2(nnz/m + 1),
 *   log2(population stdev of row nnz + 1) (block_statistics/rows-nnz-stdev.cpp:11-30),
 *   max |i - j| / max(m, n), mean |i - j| / max(m, n),
 *   shares of the nonzeros lying in 64 x 64 tiles with 1-4, 5-32, 33-256,
 *   257-1024 and 1025-4096 nonzeros (the tile density histogram),
 *   log2(nonzero 64 x 64 tiles per block row + 1).
 * No counterpart in the reference.  Synchronises stream. */
ABHSF_API abhsf_status abhsf_selector_features(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m,
                                               int64_t n, int32_t inputs_on_device, abhsf_stream_t stream,
                                               float out[12]);

/* Block size the MLP `model` (host, ABHSF_MLP_PARAMS floats; NULL = the
 * built-in model) predicts for features[12]: 16 << argmax of its outputs.
 * Runs the forward kernel on the current device.  No counterpart in the
 * reference. */
ABHSF_API abhsf_status abhsf_selector_predict(const float* model, const float features[12], abhsf_stream_t stream,
                                              int32_t* block_size);

/* The built-in model (ABHSF_MLP_PARAMS floats) into out. */
ABHSF_API abhsf_status abhsf_selector_builtin_model(float* out);

/* The built-in model trained on measured SpMV times (ABHSF_SELECT_LEARNED_TIME)
 * into out.  No counterpart in the reference. */
ABHSF_API abhsf_status abhsf_selector_builtin_time_model(float* out);

/* Training kernels of the MLP, all pointers device memory, ordered on stream.
 * forward: probs[batch][C] = softmax of the network at x[batch][F]; act
 * (NULL, or batch * 2 * H floats) keeps the hidden activations for backward.
 * backward: grad[P] = gradient of the mean cross-entropy against targets
 * (batch x C probabilities, rows summing to 1; a one-hot row is a label) with
 * respect to the trainable parameters (all but mean / inv_std, whose entries
 * of grad are left alone), from forward's probs and act; delta
 * is scratch of batch * (C + 2 H) floats; loss (NULL allowed) gets the mean
 * cross-entropy.  The sums over the batch run in sample order, so gradients
 * are bitwise reproducible.  adam: one Adam step (beta 0.9 / 0.999, eps 1e-8,
 * bias-corrected by step >= 1) of the trainable parameters with moment
 * buffers m, v (P floats each, zero at step 1).  No counterpart in the
 * reference. */
ABHSF_API abhsf_status abhsf_mlp_forward(const float* params, const float* x, int32_t batch, float* probs,
                                         float* act, abhsf_stream_t stream);
ABHSF_API abhsf_status abhsf_mlp_backward(const float* params, const float* x, const float* targets, int32_t batch,
                                          const float* probs, const float* act, float* delta, float* grad,
                                          float* loss, abhsf_stream_t stream);
ABHSF_API abhsf_status abhsf_mlp_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr,
                                      abhsf_stream_t stream);

/* Reads a Matrix Market coordinate file as read_mtx_real_or_binary does
 * (include/abhsf/utils/matrix_market_reader.h:146-200): real or pattern
 * (values 1.0), indices made 0-based, explicit zeros of a real matrix
 * dropped, a symmetric / skew / hermitian file's stored triangle kept as
 * stored (ABHSF_ERROR_INVALID_VALUE when both triangles appear), the first nnz
 * entries read.  Integer and complex files are ABHSF_ERROR_UNSUPPORTED (the
 * reference reader throws for them); indices outside m x n are
 * ABHSF_ERROR_INDEX_OUT_OF_RANGE (the reference does not check).  The entry
 * lines are parsed by `threads` host threads (0: all).  The arrays go to
 * abhsf_build as they are. */
ABHSF_API abhsf_status abhsf_read_mtx(const char* path, int32_t threads, abhsf_coo_host* out);
ABHSF_API abhsf_status abhsf_coo_host_free(abhsf_coo_host* coo);

/* The same read with the parse on the GPU: the file is read into host memory
 * and copied to the device, where one thread per line reads the entry (line
 * ends found by a scan), rounds its value to the nearest double exactly as
 * strtod does (a 64-bit significand times a 128-bit power of five; values of
 * more than 19 significant digits, other spellings and the rare result that
 * product cannot decide go to the host's parser, line by line), and the
 * checks, the zero drop and the compaction of the first nnz entries run as
 * kernels.  The elements equal abhsf_read_mtx's, in the same order, and the
 * errors are its errors (a file whose entries span lines is read by the
 * host's parser).  Ordered on stream; the arrays are ready when it returns. */
ABHSF_API abhsf_status abhsf_read_mtx_device(const char* path, abhsf_stream_t stream, abhsf_coo_device* out);
ABHSF_API abhsf_status abhsf_coo_device_free(abhsf_coo_device* coo);
/* Copies the arrays of coo into the caller's device arrays of nnz elements
 * each (any may be NULL), ordered on stream: for callers whose memory comes
 * from their own allocator. */
ABHSF_API abhsf_status abhsf_coo_device_copy(const abhsf_coo_device* coo, int64_t* rows, int64_t* cols,
                                             double* vals, abhsf_stream_t stream);

/* The reference's binary matrix file (".mm", written by
 * utils/mtx2mm/mtx2mm.cpp:102-135): u64 m, n, nnz, type (0 pattern, 2 real),
 * symmetry flag (0 general; 1 symmetric, 2 hermitian, 3 skew; the reference
 * writes a bool), then u32 rows[nnz], u32 cols[nnz] (0-based) and, for a real
 * matrix, f64 vals[nnz].  abhsf_read_mm returns what abhsf_read_mtx returns for
 * the text file the .mm was made from: explicit zeros dropped, the stored
 * triangle found (ABHSF_ERROR_INVALID_VALUE when a non-general file holds both),
 * indices checked against m x n; integer and complex files are
 * ABHSF_ERROR_UNSUPPORTED, a file whose size differs from its header's arrays
 * ABHSF_ERROR_INVALID_VALUE.  abhsf_write_mm writes coo (real or pattern, m and
 * n at most 2^32) in that layout. */
ABHSF_API abhsf_status abhsf_read_mm(const char* path, abhsf_coo_host* out);
ABHSF_API abhsf_status abhsf_write_mm(const char* path, const abhsf_coo_host* coo);

/* Waits for the work queued on stream, then returns the matrix's device
 * status word (ABHSF_DEVSTAT_* bits; 0 = every SpMV so far completed) and,
 * if clear != 0, resets it.  No reference counterpart (the reference has no
 * device code). */
ABHSF_API abhsf_status abhsf_device_status(abhsf_matrix* a, abhsf_stream_t stream, int32_t clear, int32_t* out);

/* Reason for the last non-success status returned on this thread. */
ABHSF_API const char* abhsf_last_error_string(void);

ABHSF_API int32_t abhsf_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ABHSF_GPU_H */
