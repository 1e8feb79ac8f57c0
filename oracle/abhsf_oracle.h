/*
 * abhsf_oracle.h -- CPU restatement of the reference's ABHSF hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (abhsf_b200/, include/)
 * links or calls this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py use it, always as the checker.
 *
 * Every function cites the reference file:line it restates (paths relative
 * to the DanielLangr/abhsf project root).  The restatement is pinned against
 * outputs of the reference's own block_stats / mmf / CSR spmv_naive, built
 * from source by oracle/Makefile into oracle/_ref and recorded as golden
 * fixtures under tests/golden/.
 */
#ifndef ABHSF_ORACLE_H
#define ABHSF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_COO = 0, ORC_CSR = 1, ORC_BITMAP = 2, ORC_DENSE = 3 };
enum { ORC_TYPE_BINARY = 0, ORC_TYPE_INTEGER = 1, ORC_TYPE_REAL = 2, ORC_TYPE_COMPLEX = 3 };
enum { ORC_VAL_F64 = 0, ORC_VAL_F32 = 1, ORC_VAL_BF16 = 2 };

enum {
    ORC_OK = 0,
    ORC_ERR_INVALID = 1,
    ORC_ERR_RANGE = 2,
    ORC_ERR_DUPLICATE = 3,
    ORC_ERR_NOMEM = 4,
    ORC_ERR_UNSUPPORTED = 5
};

/* include/abhsf/utils/math.h:18-31 (ceil_log2, loop form, ceil_log2(1) == 0) */
uint64_t orc_ceil_log2(uint64_t n);
/* include/abhsf/msmf.h:9-33 */
uint64_t orc_block_coo_bits(uint64_t m, uint64_t n, uint64_t nnz);
uint64_t orc_block_csr_bits(uint64_t m, uint64_t n, uint64_t nnz);
uint64_t orc_block_bitmap_bits(uint64_t m, uint64_t n);
uint64_t orc_block_dense_bits(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits_per_element);
/* include/abhsf/msmf.h:35-63 -- the minimum (value only) */
uint64_t orc_block_min_bits(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits, int is_binary);
uint64_t orc_block_min_bits_wocsr(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits, int is_binary);
/* Scheme implied by msmf.h's std::min nesting (ties keep the first argument,
 * msmf.h:42,46,57,61): COO > CSR > bitmap > dense. */
int orc_select_scheme(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits, int is_binary, int allow_csr);

/* block_statistics/block_stats.cpp:69-100: sort elements by the block key
 * ((row >> k) << 32) + (col >> l) and count the nonzeros of every nonzero
 * block.  hist must hold (1 << k) * (1 << l) + 1 zeroed counters; hist[z] +=
 * number of blocks with z nonzeros.  Returns the number of nonzero blocks, or
 * a negative ORC_ERR_* code. */
int64_t orc_block_histogram(const int64_t* rows, const int64_t* cols, int64_t nnz,
                            int k, int l, uint64_t* hist);

/* block_statistics/mmf.cpp:53-138: one line of mmf-single and mmf-double for
 * block size r x s, from the props (m, n, stored nnz, type) and the block
 * histogram (hist[z] blocks with z nonzeros, z in [0, hist_len)).
 * out[8] = coo32 csr32 coo csr bitmap dense abhsf abhsf134, values included. */
void orc_mmf_line(uint64_t m, uint64_t n, uint64_t nnz, int type, uint64_t r, uint64_t s,
                  const uint64_t* hist, uint64_t hist_len,
                  uint64_t out_single[8], uint64_t out_double[8]);

/* ---------------------------------------------------------------------------
 * CPU builder restatement that emits the declared ABHSF device arrays
 * (block-row CSR of tiles, per-tile scheme, payloads, values).  Block
 * partition follows block_stats.cpp:69-100, scheme choice msmf.h:35-63, in-tile
 * row-major order and LSB-first bitmaps spmv/orig/88.cpp:112-130.
 * ------------------------------------------------------------------------ */
typedef struct orc_matrix {
    int64_t m, n, nnz;
    int32_t s, log2s;
    int64_t M, N, T;            /* block rows, block cols, nonzero tiles */
    int32_t value_type;         /* ORC_VAL_* */
    int64_t n_values;           /* stored values (dense tiles include zeros) */
    int64_t idx_bytes;          /* payload bytes (each tile padded to 16) */
    int64_t* brow_ptr;          /* [M+1] */
    uint32_t* tile_col;         /* [T] */
    uint32_t* tile_nnz;         /* [T] */
    uint8_t* tile_scheme;       /* [T] */
    int64_t* tile_val_off;      /* [T+1] */
    int64_t* tile_idx_off;      /* [T+1] bytes */
    uint8_t* idx;               /* [idx_bytes] */
    void* values;               /* [n_values] of value_type */
} orc_matrix;

/* Builds; returns ORC_OK and fills *out (free with orc_free), or an error.
 * bits_per_value feeds the dense cost (64 for mmf-double, 32 for mmf-single).
 * forced_scheme < 0 selects by minimum storage. */
int orc_build(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz,
              int64_t m, int64_t n, int32_t s, int32_t value_type, uint64_t bits_per_value,
              int32_t is_binary, int32_t allow_csr, int32_t forced_scheme, orc_matrix** out);
void orc_free(orc_matrix* a);

/* y += A x over the built arrays, decoding every scheme (CPU restatement of
 * spmv/orig/88.cpp:204-236 (COO), 88_bitmap.cpp:183-207 (bitmap), 88.cpp:579-605
 * (dense), generalised to s x s and FP64).  Values of f32/bf16 matrices are
 * widened to double. */
void orc_spmv_abhsf(const orc_matrix* a, const double* x, double* y);
/* The same on all host threads (OpenMP over block rows), bit for bit. */
void orc_spmv_abhsf_omp(const orc_matrix* a, const double* x, double* y);
int orc_omp_threads(void);

/* The reference's verification loop, spmv/unified/spmv.cpp:1195-1201 and
 * spmv/bottlenecks/spmv.cpp:307-313: y[row] += val * x[col] in element order. */
void orc_spmv_elements(const int64_t* rows, const int64_t* cols, const double* vals,
                       int64_t nnz, const double* x, double* y);
/* (|A| |x|)_i, the scale used for the per-element error bound. */
void orc_abs_spmv_elements(const int64_t* rows, const int64_t* cols, const double* vals,
                           int64_t nnz, const double* x, double* out);

/* Value conversions the format declares: f32 = RN(f64); bf16 = RNE(f32). */
float orc_f64_to_f32(double v);
/* Values as stored in an f32 (vt 1) or bf16 (vt 2) matrix, widened to f32. */
void orc_values_as_f32(const double* v, int64_t n, int vt, float* out);
/* y += A x in f32, element order, product and sum each rounded to f32. */
void orc_spmv_elements_f32(const int64_t* rows, const int64_t* cols, const float* vals,
                           int64_t nnz, const float* x, float* y);
uint16_t orc_f64_to_bf16(double v);
double orc_bf16_to_f64(uint16_t b);

/* Delta-coded row slices of the hypersparse block rows (the encoding the
 * library's SpMV reads for them; spmv/orig/delta.cpp:118-219 is the
 * reference's row-by-row delta COO it follows).  Block rows: non-empty, no
 * dense tile, and no bitmap tile, at most avg elements per tile on average or
 * more than 256 tiles; none when n > 2^32 or the elements reach 2^31.
 * Segments of block rows: the quarters [M c / 4, M (c + 1) / 4), each cut
 * into pieces of at most 2^24 rows.  Per segment: first, per block row
 * (ascending), its rows of more than 256 elements by length (longest first,
 * then row), each a chain slice (lanes 1, brow = its block row, meta = the
 * row within it, steps = its length, its elements at slots base + k with
 * absolute columns); then the segment's other non-empty rows by length
 * (longest first, then ascending row) in slices of up to 32 (brow = the
 * segment's first block row, steps = the first row's length, lane record
 * l = (row - brow s) << 8 | (length - 1) at lane[meta + l], element k of lane
 * l at slot base + 32 k + l, each word the column minus the row's previous
 * column, the first absolute).  vidx: each slot's index in the format's
 * values (-1 for padding, whose word is 0). */
typedef struct orc_slices {
    int64_t n, slots, lane_records, E, block_rows;
    int64_t* base;
    int64_t* meta;
    uint32_t* brow;
    uint32_t* steps;
    uint32_t* lanes;
    uint8_t* chain;
    uint32_t* lane;
    uint32_t* words;
    int64_t* vidx;
} orc_slices;
int orc_slices_build(const orc_matrix* a, double avg, orc_slices** out);
void orc_slices_free(orc_slices* p);
/* y += A x over the slice rows only, each row's words decoded in order. */
void orc_spmv_slices(const orc_matrix* a, const orc_slices* p, const double* x, double* y);

#ifdef __cplusplus
}
#endif
#endif
