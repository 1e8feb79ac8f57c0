/*
 * abhsf_test.h -- test hooks of libabhsf_b200.so.  Not for production use.
 *
 * abhsf_test_set_hooks makes the reference-order SpMV (block sizes 32 and 64)
 * skip the bulk copies of one tile -- the drop_desc-th entry of the matrix's
 * tile schedule -- and poll each wait at most spin_limit times, so a test can
 * check that a wait that runs out ends the kernel with
 * ABHSF_DEVSTAT_WAIT_TIMEOUT in the matrix's status word (abhsf_device_status)
 * instead of hanging.  No copy is left in flight and the CUDA context stays
 * usable.  drop_desc < 0 and spin_limit == 0 restore normal operation.
 * Process-wide, not thread-safe.  No reference counterpart (the reference has
 * no device code).
 */
#ifndef ABHSF_TEST_H
#define ABHSF_TEST_H

#include "abhsf_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

ABHSF_API void abhsf_test_set_hooks(int64_t drop_desc, uint32_t spin_limit);

/* The launch variant the build chose for a matrix's single-right-hand-side
 * ring kernel, and a way to force one, so that a test can check that every
 * variant gives the same y and a benchmark can time each.  layout: the
 * consumers' arrangement, 0 = one team of s/32 warps (a row per lane),
 * 1 = two such teams, 2 = four teams of one warp (s/32 rows per lane),
 * 3 = two teams of one warp; bulk: x / y blocks as bulk copies (1) or element
 * copies (0).  layout = -1 on a matrix the ring kernel does not serve.  Not
 * thread-safe with SpMVs of the same matrix. */
ABHSF_API abhsf_status abhsf_test_ring_variant(abhsf_matrix* a, int32_t set, int32_t* layout, int32_t* bulk);

/* Device allocations (cudaMalloc) the library has made since it was loaded,
 * so that a test can check that an entry point which promises to allocate
 * nothing keeps that promise. */
ABHSF_API int64_t abhsf_test_device_allocations(void);

/* The device Matrix Market parser's decimal conversion, run on the host on
 * the len bytes at text: 0 = converted (*value, *used bytes read), 1 = left to
 * the host's parser (not a plain decimal, more than 19 significant digits, a
 * result the 128-bit product cannot round, or outside the normal range).  So
 * that tests can compare it with strtod over many numbers without a GPU. */
ABHSF_API int32_t abhsf_test_parse_decimal(const char* text, int64_t len, double* value, int64_t* used);

#ifdef __cplusplus
}
#endif
#endif
