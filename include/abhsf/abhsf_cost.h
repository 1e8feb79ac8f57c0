/*
 * abhsf_cost.h -- minimum-storage cost model of one block and the scheme it
 * selects, usable from host and device code.
 *
 * Restates include/abhsf/msmf.h:9-63 and include/abhsf/utils/math.h:18-31 of
 * DanielLangr/abhsf (bits, not bytes; values are counted outside the scheme
 * cost, block_statistics/mmf.cpp:119-120):
 *   COO    = ceil_log2(m n) + nnz (ceil_log2 m + ceil_log2 n)
 *   CSR    = m ceil_log2(m n) + nnz ceil_log2 n
 *   bitmap = m n
 *   dense  = (m n - nnz) bits_per_element           (never for binary matrices)
 * The block's scheme is the argmin in the order the reference's std::min
 * nesting implies (msmf.h:42,46,57,61: ties keep the first argument), i.e.
 * COO > CSR > bitmap > dense.
 */
#ifndef ABHSF_COST_H
#define ABHSF_COST_H

#include <stdint.h>

#if defined(__CUDACC__)
#define ABHSF_HD __host__ __device__ __forceinline__
#else
#define ABHSF_HD static inline
#endif

enum { ABHSF_COST_COO = 0, ABHSF_COST_CSR = 1, ABHSF_COST_BITMAP = 2, ABHSF_COST_DENSE = 3 };

/* Smallest k with 2^k >= v (0 for v <= 1). */
ABHSF_HD uint64_t abhsf_ceil_log2(uint64_t v)
{
    uint64_t k = 0;
    while (k < 64 && ((uint64_t)1 << k) < v)
        ++k;
    return k;
}

ABHSF_HD uint64_t abhsf_coo_bits(uint64_t m, uint64_t n, uint64_t nnz)
{
    return abhsf_ceil_log2(m * n) + nnz * (abhsf_ceil_log2(m) + abhsf_ceil_log2(n));
}

ABHSF_HD uint64_t abhsf_csr_bits(uint64_t m, uint64_t n, uint64_t nnz)
{
    return m * abhsf_ceil_log2(m * n) + nnz * abhsf_ceil_log2(n);
}

ABHSF_HD uint64_t abhsf_bitmap_bits(uint64_t m, uint64_t n) { return m * n; }

ABHSF_HD uint64_t abhsf_dense_bits(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits)
{
    return (m * n - nnz) * bits;
}

/* Scheme of an m x n block with nnz nonzeros; *min_bits (optional) receives
 * its cost.  allow_csr = 0 is the reference's block_min_msmf_wocsr. */
ABHSF_HD int abhsf_select_scheme(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits,
                                 int is_binary, int allow_csr, uint64_t* min_bits)
{
    const uint64_t coo = abhsf_coo_bits(m, n, nnz);
    int best = ABHSF_COST_COO;
    uint64_t best_v = coo;
    if (allow_csr) {
        const uint64_t csr = abhsf_csr_bits(m, n, nnz);
        if (csr < best_v) {
            best = ABHSF_COST_CSR;
            best_v = csr;
        }
    }
    /* right-hand side of the nesting: min(bitmap, dense), then compared */
    int right = ABHSF_COST_BITMAP;
    uint64_t right_v = abhsf_bitmap_bits(m, n);
    if (!is_binary) {
        const uint64_t dense = abhsf_dense_bits(m, n, nnz, bits);
        if (dense < right_v) {
            right = ABHSF_COST_DENSE;
            right_v = dense;
        }
    }
    if (right_v < best_v) {
        best = right;
        best_v = right_v;
    }
    if (min_bits)
        *min_bits = best_v;
    return best;
}

#endif /* ABHSF_COST_H */
