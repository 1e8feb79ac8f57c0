/* c_consumer.c -- the C ABI used from plain C99 (the header compiles as C,
 * the library links from a C program).  Calls only host-side entry points,
 * so it runs on a machine without a GPU: the ABI version, the default
 * options, the cost model, one mmf line, the Matrix Market and .mm readers,
 * and the status / message of a refused build.  Built and run by
 * tests/test_c_consumer.py. */
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "abhsf/abhsf_gpu.h"

int main(int argc, char** argv)
{
    if (abhsf_abi_version() != ABHSF_ABI_VERSION) {
        printf("FAIL abi\n");
        return 1;
    }
    abhsf_build_opts o;
    abhsf_build_opts_default(&o);
    if (o.block_size != 64 || o.value_type != ABHSF_VALUE_F64 || o.allow_csr != 1) {
        printf("FAIL defaults\n");
        return 1;
    }
    /* s = 64, 64-bit values: COO up to 126 nonzeros, CSR from 127 */
    if (abhsf_block_select_scheme(64, 64, 126, 64, 0, 1) != ABHSF_SCHEME_COO ||
        abhsf_block_select_scheme(64, 64, 127, 64, 0, 1) != ABHSF_SCHEME_CSR) {
        printf("FAIL scheme\n");
        return 1;
    }
    printf("coo_bits %llu\n", (unsigned long long)abhsf_block_scheme_bits(ABHSF_SCHEME_COO, 64, 64, 64, 64));
    /* the 512 x 512 2D Laplacian's 64 x 64 line: {1: 7168, 64: 8176, 190: 4096} */
    uint64_t hist[191];
    memset(hist, 0, sizeof(hist));
    hist[1] = 7168;
    hist[64] = 8176;
    hist[190] = 4096;
    uint64_t single[8], dbl[8];
    if (abhsf_mmf_line(262144, 262144, 1308672, ABHSF_MATRIX_REAL, 64, 64, hist, 191, single, dbl) != ABHSF_SUCCESS) {
        printf("FAIL mmf %s\n", abhsf_last_error_string());
        return 1;
    }
    printf("abhsf_bits %llu\n", (unsigned long long)dbl[6]);
    /* a refused build: block size 48 */
    abhsf_matrix* A = NULL;
    int64_t r = 0, c = 0;
    double v = 1.0;
    o.block_size = 48;
    if (abhsf_build(&r, &c, &v, 1, 1, 1, &o, NULL, &A) != ABHSF_ERROR_INVALID_VALUE || A != NULL) {
        printf("FAIL refused build\n");
        return 1;
    }
    printf("refused: %s\n", abhsf_last_error_string());
    /* readers */
    if (argc > 2) {
        abhsf_coo_host t, b;
        if (abhsf_read_mtx(argv[1], 2, &t) != ABHSF_SUCCESS || abhsf_write_mm(argv[2], &t) != ABHSF_SUCCESS ||
            abhsf_read_mm(argv[2], &b) != ABHSF_SUCCESS) {
            printf("FAIL readers %s\n", abhsf_last_error_string());
            return 1;
        }
        int same = t.nnz == b.nnz && t.m == b.m && t.n == b.n;
        for (int64_t k = 0; same && k < t.nnz; ++k)
            same = t.rows[k] == b.rows[k] && t.cols[k] == b.cols[k] &&
                   memcmp(&t.vals[k], &b.vals[k], sizeof(double)) == 0;
        printf("read %lld %lld %lld same %d\n", (long long)t.m, (long long)t.n, (long long)t.nnz, same);
        abhsf_coo_host_free(&t);
        abhsf_coo_host_free(&b);
        if (!same)
            return 1;
    }
    printf("OK\n");
    return 0;
}
