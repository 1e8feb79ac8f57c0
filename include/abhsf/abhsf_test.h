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

#ifdef __cplusplus
}
#endif
#endif
