/*
 * abhsf_oracle.c -- CPU restatement of the reference's ABHSF hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see abhsf_oracle.h).  Plain C99, single thread,
 * written for clarity, not speed, except for the LSD radix sort that keeps the
 * full-size workloads within seconds.
 */
#include "abhsf_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------- cost model */

uint64_t orc_ceil_log2(uint64_t n)
{
    /* include/abhsf/utils/math.h:18-31: smallest k with 2^k >= n. */
    uint64_t k = 0;
    while (k < 64 && ((uint64_t)1 << k) < n)
        k++;
    return k;
}

uint64_t orc_block_coo_bits(uint64_t m, uint64_t n, uint64_t nnz)
{
    /* include/abhsf/msmf.h:9-14 */
    return orc_ceil_log2(m * n) + nnz * (orc_ceil_log2(m) + orc_ceil_log2(n));
}

uint64_t orc_block_csr_bits(uint64_t m, uint64_t n, uint64_t nnz)
{
    /* include/abhsf/msmf.h:16-21 */
    return m * orc_ceil_log2(m * n) + nnz * orc_ceil_log2(n);
}

uint64_t orc_block_bitmap_bits(uint64_t m, uint64_t n)
{
    /* include/abhsf/msmf.h:23-26 */
    return m * n;
}

uint64_t orc_block_dense_bits(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits)
{
    /* include/abhsf/msmf.h:28-33 (zero padding only; values counted outside) */
    return (m * n - nnz) * bits;
}

static uint64_t min_u64(uint64_t a, uint64_t b)
{
    /* std::min(a, b): returns a unless b < a. */
    return (b < a) ? b : a;
}

uint64_t orc_block_min_bits(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits, int is_binary)
{
    /* include/abhsf/msmf.h:35-48 */
    uint64_t coo = orc_block_coo_bits(m, n, nnz);
    uint64_t csr = orc_block_csr_bits(m, n, nnz);
    uint64_t bmp = orc_block_bitmap_bits(m, n);
    if (is_binary)
        return min_u64(min_u64(coo, csr), bmp);
    return min_u64(min_u64(coo, csr), min_u64(bmp, orc_block_dense_bits(m, n, nnz, bits)));
}

uint64_t orc_block_min_bits_wocsr(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits, int is_binary)
{
    /* include/abhsf/msmf.h:50-63 */
    uint64_t coo = orc_block_coo_bits(m, n, nnz);
    uint64_t bmp = orc_block_bitmap_bits(m, n);
    if (is_binary)
        return min_u64(coo, bmp);
    return min_u64(coo, min_u64(bmp, orc_block_dense_bits(m, n, nnz, bits)));
}

int orc_select_scheme(uint64_t m, uint64_t n, uint64_t nnz, uint64_t bits, int is_binary, int allow_csr)
{
    /* The argmin that msmf.h's nesting implies.  With CSR:
     *   min(min(coo, csr), min(bitmap, dense))  (msmf.h:46), binary: msmf.h:42
     * without CSR:
     *   min(coo, min(bitmap, dense))            (msmf.h:61), binary: msmf.h:57
     * std::min keeps its first argument on ties. */
    uint64_t coo = orc_block_coo_bits(m, n, nnz);
    uint64_t csr = orc_block_csr_bits(m, n, nnz);
    uint64_t bmp = orc_block_bitmap_bits(m, n);
    uint64_t dns = is_binary ? 0 : orc_block_dense_bits(m, n, nnz, bits);

    int left;
    uint64_t left_v;
    if (allow_csr) {
        left = (csr < coo) ? ORC_CSR : ORC_COO;
        left_v = (csr < coo) ? csr : coo;
    } else {
        left = ORC_COO;
        left_v = coo;
    }
    int right;
    uint64_t right_v;
    if (is_binary) {
        right = ORC_BITMAP;
        right_v = bmp;
    } else {
        right = (dns < bmp) ? ORC_DENSE : ORC_BITMAP;
        right_v = (dns < bmp) ? dns : bmp;
    }
    return (right_v < left_v) ? right : left;
}

/* ---------------------------------------------------------------- radix sort */

/* Stable LSD radix sort of (key, payload) pairs on the low `bits` bits. */
static int radix_sort_pairs(uint64_t* key, uint64_t* val, int64_t n, int bits)
{
    if (n <= 1 || bits <= 0)
        return ORC_OK;
    uint64_t* k2 = (uint64_t*)malloc((size_t)n * sizeof(uint64_t));
    uint64_t* v2 = val ? (uint64_t*)malloc((size_t)n * sizeof(uint64_t)) : NULL;
    size_t* cnt = (size_t*)malloc(65536 * sizeof(size_t));
    if (!k2 || (val && !v2) || !cnt) {
        free(k2); free(v2); free(cnt);
        return ORC_ERR_NOMEM;
    }
    uint64_t *ks = key, *vs = val, *kd = k2, *vd = v2;
    int passes = (bits + 15) / 16;
    for (int p = 0; p < passes; ++p) {
        int shift = 16 * p;
        memset(cnt, 0, 65536 * sizeof(size_t));
        for (int64_t i = 0; i < n; ++i)
            cnt[(ks[i] >> shift) & 0xFFFF]++;
        size_t sum = 0;
        for (int d = 0; d < 65536; ++d) {
            size_t c = cnt[d];
            cnt[d] = sum;
            sum += c;
        }
        for (int64_t i = 0; i < n; ++i) {
            size_t pos = cnt[(ks[i] >> shift) & 0xFFFF]++;
            kd[pos] = ks[i];
            if (vs)
                vd[pos] = vs[i];
        }
        uint64_t* t = ks; ks = kd; kd = t;
        t = vs; vs = vd; vd = t;
    }
    if (ks != key) {
        memcpy(key, ks, (size_t)n * sizeof(uint64_t));
        if (val)
            memcpy(val, vs, (size_t)n * sizeof(uint64_t));
    }
    /* k2 / v2 are always the scratch pair; the result now sits in key / val. */
    free(cnt);
    free(k2);
    free(v2);
    return ORC_OK;
}

static int bits_for(uint64_t v)
{
    int b = 0;
    while (b < 64 && (v >> b) != 0)
        b++;
    return b;
}

/* ---------------------------------------------------------------- histogram */

int64_t orc_block_histogram(const int64_t* rows, const int64_t* cols, int64_t nnz,
                            int k, int l, uint64_t* hist)
{
    /* block_statistics/block_stats.cpp:69-74 (key), 78-100 (sort + runs). */
    if (nnz <= 0)
        return 0;
    uint64_t* key = (uint64_t*)malloc((size_t)nnz * sizeof(uint64_t));
    if (!key)
        return -ORC_ERR_NOMEM;
    uint64_t maxk = 0;
    for (int64_t i = 0; i < nnz; ++i) {
        if (rows[i] < 0 || cols[i] < 0 || rows[i] >= ((int64_t)1 << 32) || cols[i] >= ((int64_t)1 << 32)) {
            free(key);
            return -ORC_ERR_RANGE;
        }
        uint64_t br = (uint64_t)rows[i] >> k;
        uint64_t bc = (uint64_t)cols[i] >> l;
        key[i] = (br << 32) + bc;
        if (key[i] > maxk)
            maxk = key[i];
    }
    int rc = radix_sort_pairs(key, NULL, nnz, bits_for(maxk));
    if (rc != ORC_OK) {
        free(key);
        return -rc;
    }
    int64_t blocks = 0;
    uint64_t run = 1;
    for (int64_t i = 1; i < nnz; ++i) {
        if (key[i] != key[i - 1]) {
            hist[run]++;
            blocks++;
            run = 0;
        }
        run++;
    }
    hist[run]++;
    blocks++;
    free(key);
    return blocks;
}

/* ---------------------------------------------------------------- mmf line */

static uint64_t ceil_div_u64(uint64_t a, uint64_t b)
{
    /* include/abhsf/utils/math.h:6-16 */
    return (a % b) ? a / b + 1 : a / b;
}

void orc_mmf_line(uint64_t m, uint64_t n, uint64_t nnz, int type, uint64_t r, uint64_t s,
                  const uint64_t* hist, uint64_t hist_len,
                  uint64_t out_single[8], uint64_t out_double[8])
{
    /* block_statistics/mmf.cpp:31-47 (type -> bits), 53-138 (totals). */
    const int is_binary = (type == ORC_TYPE_BINARY);
    uint64_t bits1;
    switch (type) {
    case ORC_TYPE_INTEGER:
    case ORC_TYPE_REAL: bits1 = 32; break;
    case ORC_TYPE_COMPLEX: bits1 = 64; break;
    default: bits1 = 0;
    }
    const uint64_t coo32 = nnz * 32 * 2;
    const uint64_t csr32 = (m + 1 + nnz) * 32;
    const uint64_t M = ceil_div_u64(m, r);
    const uint64_t N = ceil_div_u64(n, s);
    uint64_t NNZ = 0;
    for (uint64_t z = 0; z < hist_len; ++z)
        NNZ += hist[z];
    const uint64_t csr0 = M * orc_ceil_log2(N + 1) + NNZ * orc_ceil_log2(N);

    uint64_t coo = csr0, csr = csr0, bmp = csr0, d1 = csr0, d2 = csr0;
    uint64_t a1 = csr0, a2 = csr0, w1 = csr0, w2 = csr0;
    if (is_binary) {
        d1 = UINT64_MAX;
        d2 = UINT64_MAX;
    }
    for (uint64_t z = 0; z < hist_len; ++z) {
        uint64_t c = hist[z];
        if (!c)
            continue;
        coo += orc_block_coo_bits(r, s, z) * c;
        csr += orc_block_csr_bits(r, s, z) * c;
        bmp += orc_block_bitmap_bits(r, s) * c;
        if (!is_binary) {
            d1 += orc_block_dense_bits(r, s, z, bits1) * c;
            d2 += orc_block_dense_bits(r, s, z, bits1 * 2) * c;
        }
        a1 += (orc_block_min_bits(r, s, z, bits1, is_binary) + 2) * c;
        a2 += (orc_block_min_bits(r, s, z, bits1 * 2, is_binary) + 2) * c;
        w1 += (orc_block_min_bits_wocsr(r, s, z, bits1, is_binary) + 2) * c;
        w2 += (orc_block_min_bits_wocsr(r, s, z, bits1 * 2, is_binary) + 2) * c;
    }
    const uint64_t v1 = nnz * bits1;
    const uint64_t v2 = v1 * 2;
    uint64_t o1[8] = {coo32 + v1, csr32 + v1, coo + v1, csr + v1, bmp + v1, d1 + v1, a1 + v1, w1 + v1};
    uint64_t o2[8] = {coo32 + v2, csr32 + v2, coo + v2, csr + v2, bmp + v2, d2 + v2, a2 + v2, w2 + v2};
    memcpy(out_single, o1, sizeof(o1));
    memcpy(out_double, o2, sizeof(o2));
}

/* ---------------------------------------------------------------- values */

float orc_f64_to_f32(double v)
{
    return (float)v; /* IEEE round-to-nearest-even */
}

uint16_t orc_f64_to_bf16(double v)
{
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) /* NaN: keep quiet NaN */
        return (uint16_t)((u >> 16) | 0x0040u);
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7FFFu + lsb;
    return (uint16_t)(u >> 16);
}

double orc_bf16_to_f64(uint16_t b)
{
    uint32_t u = (uint32_t)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return (double)f;
}

/* ---------------------------------------------------------------- builder */

static int64_t pad16(int64_t b) { return (b + 15) & ~(int64_t)15; }

static int64_t payload_bytes(int scheme, int64_t s, int64_t nnz)
{
    switch (scheme) {
    case ORC_COO: return pad16(2 * nnz);            /* u16 (lrow << log2 s) | lcol */
    case ORC_CSR: return pad16(2 * s + nnz);        /* u16 row_end[s] + u8 col[nnz] */
    case ORC_BITMAP: return pad16(s * s / 8);       /* u64 words, bit lrow*s + lcol */
    default: return 0;                              /* dense: values only */
    }
}

void orc_free(orc_matrix* a)
{
    if (!a)
        return;
    free(a->brow_ptr); free(a->tile_col); free(a->tile_nnz); free(a->tile_scheme);
    free(a->tile_val_off); free(a->tile_idx_off); free(a->idx); free(a->values);
    free(a);
}

int orc_build(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz,
              int64_t m, int64_t n, int32_t s, int32_t value_type, uint64_t bits_per_value,
              int32_t is_binary, int32_t allow_csr, int32_t forced_scheme, orc_matrix** out)
{
    *out = NULL;
    if (m <= 0 || n <= 0 || nnz < 0 || s < 2 || s > 256 || (s & (s - 1)) ||
        value_type < 0 || value_type > 2 || forced_scheme > 3)
        return ORC_ERR_INVALID;
    if (forced_scheme == ORC_DENSE && is_binary)
        return ORC_ERR_INVALID;
    int lg = 0;
    while ((1 << lg) < s)
        lg++;
    const int64_t M = (m + s - 1) / s, N = (n + s - 1) / s;

    orc_matrix* a = (orc_matrix*)calloc(1, sizeof(orc_matrix));
    if (!a)
        return ORC_ERR_NOMEM;
    a->m = m; a->n = n; a->nnz = nnz; a->s = s; a->log2s = lg; a->M = M; a->N = N;
    a->value_type = value_type;

    uint64_t* key = (uint64_t*)malloc((size_t)(nnz ? nnz : 1) * sizeof(uint64_t));
    uint64_t* perm = (uint64_t*)malloc((size_t)(nnz ? nnz : 1) * sizeof(uint64_t));
    if (!key || !perm) {
        free(key); free(perm); orc_free(a);
        return ORC_ERR_NOMEM;
    }
    /* Key = (I * N + J) * s^2 + lrow * s + lcol: tiles in (block row, block col)
     * order (block_stats.cpp:69-74 with the rows of a tile kept together), and
     * the elements of a tile row-major (spmv/orig/88.cpp:112-130). */
    uint64_t maxk = 0;
    for (int64_t i = 0; i < nnz; ++i) {
        if (rows[i] < 0 || rows[i] >= m || cols[i] < 0 || cols[i] >= n) {
            free(key); free(perm); orc_free(a);
            return ORC_ERR_RANGE;
        }
        uint64_t I = (uint64_t)rows[i] >> lg, J = (uint64_t)cols[i] >> lg;
        uint64_t lr = (uint64_t)rows[i] & (s - 1), lc = (uint64_t)cols[i] & (s - 1);
        key[i] = ((I * (uint64_t)N + J) << (2 * lg)) | (lr << lg) | lc;
        perm[i] = (uint64_t)i;
        if (key[i] > maxk)
            maxk = key[i];
    }
    int rc = radix_sort_pairs(key, perm, nnz, bits_for(maxk));
    if (rc != ORC_OK) {
        free(key); free(perm); orc_free(a);
        return rc;
    }
    for (int64_t i = 1; i < nnz; ++i)
        if (key[i] == key[i - 1]) {
            free(key); free(perm); orc_free(a);
            return ORC_ERR_DUPLICATE;
        }

    /* tiles */
    int64_t T = 0;
    for (int64_t i = 0; i < nnz; ++i)
        if (i == 0 || (key[i] >> (2 * lg)) != (key[i - 1] >> (2 * lg)))
            T++;
    a->T = T;
    a->brow_ptr = (int64_t*)calloc((size_t)(M + 1), sizeof(int64_t));
    a->tile_col = (uint32_t*)calloc((size_t)(T ? T : 1), sizeof(uint32_t));
    a->tile_nnz = (uint32_t*)calloc((size_t)(T ? T : 1), sizeof(uint32_t));
    a->tile_scheme = (uint8_t*)calloc((size_t)(T ? T : 1), 1);
    a->tile_val_off = (int64_t*)calloc((size_t)(T + 1), sizeof(int64_t));
    a->tile_idx_off = (int64_t*)calloc((size_t)(T + 1), sizeof(int64_t));
    int64_t* tile_start = (int64_t*)calloc((size_t)(T + 1), sizeof(int64_t));
    int64_t* tile_row = (int64_t*)calloc((size_t)(T ? T : 1), sizeof(int64_t));
    if (!a->brow_ptr || !a->tile_col || !a->tile_nnz || !a->tile_scheme || !a->tile_val_off ||
        !a->tile_idx_off || !tile_start || !tile_row) {
        free(key); free(perm); free(tile_start); free(tile_row); orc_free(a);
        return ORC_ERR_NOMEM;
    }
    int64_t t = -1;
    for (int64_t i = 0; i < nnz; ++i) {
        if (i == 0 || (key[i] >> (2 * lg)) != (key[i - 1] >> (2 * lg))) {
            t++;
            uint64_t tk = key[i] >> (2 * lg);
            tile_start[t] = i;
            tile_row[t] = (int64_t)(tk / (uint64_t)N);
            a->tile_col[t] = (uint32_t)(tk % (uint64_t)N);
        }
    }
    tile_start[T] = nnz;
    const int64_t ss = (int64_t)s * s;
    for (t = 0; t < T; ++t) {
        int64_t z = tile_start[t + 1] - tile_start[t];
        int sch = forced_scheme >= 0
                      ? forced_scheme
                      : orc_select_scheme((uint64_t)s, (uint64_t)s, (uint64_t)z, bits_per_value, is_binary, allow_csr);
        if (sch == ORC_CSR && z > 65535) {
            free(key); free(perm); free(tile_start); free(tile_row); orc_free(a);
            return ORC_ERR_UNSUPPORTED;
        }
        a->tile_nnz[t] = (uint32_t)z;
        a->tile_scheme[t] = (uint8_t)sch;
        a->tile_val_off[t + 1] = a->tile_val_off[t] + (sch == ORC_DENSE ? ss : z);
        a->tile_idx_off[t + 1] = a->tile_idx_off[t] + payload_bytes(sch, s, z);
    }
    a->n_values = a->tile_val_off[T];
    a->idx_bytes = a->tile_idx_off[T];
    /* brow_ptr[i] = first tile whose block row is >= i */
    {
        int64_t tt = 0;
        for (int64_t i = 0; i <= M; ++i) {
            while (tt < T && tile_row[tt] < i)
                tt++;
            a->brow_ptr[i] = tt;
        }
    }
    const size_t vsz = value_type == ORC_VAL_F64 ? 8 : value_type == ORC_VAL_F32 ? 4 : 2;
    a->idx = (uint8_t*)calloc((size_t)(a->idx_bytes ? a->idx_bytes : 1), 1);
    a->values = calloc((size_t)(a->n_values ? a->n_values : 1), vsz);
    if (!a->idx || !a->values) {
        free(key); free(perm); free(tile_start); free(tile_row); orc_free(a);
        return ORC_ERR_NOMEM;
    }

    for (t = 0; t < T; ++t) {
        const int sch = a->tile_scheme[t];
        uint8_t* pay = a->idx + a->tile_idx_off[t];
        const int64_t z = a->tile_nnz[t];
        for (int64_t p = 0; p < z; ++p) {
            const int64_t i = tile_start[t] + p;
            const uint64_t local = key[i] & ((uint64_t)ss - 1);
            const uint32_t lr = (uint32_t)(local >> lg), lc = (uint32_t)(local & (s - 1));
            const double v = vals ? vals[perm[i]] : 1.0;
            int64_t vpos = a->tile_val_off[t] + (sch == ORC_DENSE ? (int64_t)local : p);
            switch (value_type) {
            case ORC_VAL_F64: ((double*)a->values)[vpos] = v; break;
            case ORC_VAL_F32: ((float*)a->values)[vpos] = orc_f64_to_f32(v); break;
            default: ((uint16_t*)a->values)[vpos] = orc_f64_to_bf16(v); break;
            }
            if (sch == ORC_COO) {
                uint16_t packed = (uint16_t)((lr << lg) | lc);
                memcpy(pay + 2 * p, &packed, 2);
            } else if (sch == ORC_CSR) {
                pay[2 * s + p] = (uint8_t)lc;
            } else if (sch == ORC_BITMAP) {
                uint64_t w;
                memcpy(&w, pay + 8 * (local >> 6), 8);
                w |= (uint64_t)1 << (local & 63);
                memcpy(pay + 8 * (local >> 6), &w, 8);
            }
        }
        if (sch == ORC_CSR) {
            /* row_end[r] = number of tile elements in rows <= r */
            int64_t p = 0;
            for (int r = 0; r < s; ++r) {
                while (p < z && (int64_t)(((key[tile_start[t] + p] & ((uint64_t)ss - 1)) >> lg)) <= r)
                    p++;
                uint16_t e = (uint16_t)p;
                memcpy(pay + 2 * r, &e, 2);
            }
        }
    }
    free(key); free(perm); free(tile_start); free(tile_row);
    *out = a;
    return ORC_OK;
}

/* ---------------------------------------------------------------- SpMV */

static double value_at(const orc_matrix* a, int64_t i)
{
    switch (a->value_type) {
    case ORC_VAL_F64: return ((const double*)a->values)[i];
    case ORC_VAL_F32: return (double)((const float*)a->values)[i];
    default: return orc_bf16_to_f64(((const uint16_t*)a->values)[i]);
    }
}

/* y += A x over block row I: its tiles in column order, each tile's
 * elements in stored order (row-major), so every row adds its products
 * columns ascending. */
static void spmv_block_row(const orc_matrix* a, int64_t I, const double* x, double* y)
{
    const int s = a->s, lg = a->log2s;
    for (int64_t t = a->brow_ptr[I]; t < a->brow_ptr[I + 1]; ++t) {
        const int64_t J = a->tile_col[t];
        const int64_t z = a->tile_nnz[t];
        const int64_t vo = a->tile_val_off[t];
        const uint8_t* pay = a->idx + a->tile_idx_off[t];
        const int64_t r0 = I * s, c0 = J * s;
        switch (a->tile_scheme[t]) {
        case ORC_COO:
            for (int64_t p = 0; p < z; ++p) {
                uint16_t k;
                memcpy(&k, pay + 2 * p, 2);
                y[r0 + (k >> lg)] += value_at(a, vo + p) * x[c0 + (k & (s - 1))];
            }
            break;
        case ORC_CSR: {
            int64_t p = 0;
            for (int r = 0; r < s; ++r) {
                uint16_t e;
                memcpy(&e, pay + 2 * r, 2);
                for (; p < e; ++p)
                    y[r0 + r] += value_at(a, vo + p) * x[c0 + pay[2 * s + p]];
            }
            break;
        }
        case ORC_BITMAP: {
            int64_t p = 0;
            for (int64_t b = 0; b < (int64_t)s * s; ++b) {
                uint64_t w;
                memcpy(&w, pay + 8 * (b >> 6), 8);
                if ((w >> (b & 63)) & 1) {
                    y[r0 + (b >> lg)] += value_at(a, vo + p) * x[c0 + (b & (s - 1))];
                    p++;
                }
            }
            break;
        }
        default:
            for (int64_t b = 0; b < (int64_t)s * s; ++b) {
                int64_t r = r0 + (b >> lg), c = c0 + (b & (s - 1));
                if (r < a->m && c < a->n)
                    y[r] += value_at(a, vo + b) * x[c];
            }
        }
    }
}

void orc_spmv_abhsf(const orc_matrix* a, const double* x, double* y)
{
    for (int64_t I = 0; I < a->M; ++I)
        spmv_block_row(a, I, x, y);
}

/* The same over the host's threads (OpenMP, block rows dealt dynamically):
 * block rows write disjoint rows of y, so y is the serial one bit for bit.
 * A CPU ABHSF SpMV to time beside the reference's CSR kernel. */
void orc_spmv_abhsf_omp(const orc_matrix* a, const double* x, double* y)
{
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t I = 0; I < a->M; ++I)
        spmv_block_row(a, I, x, y);
}

int orc_omp_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_spmv_elements(const int64_t* rows, const int64_t* cols, const double* vals,
                       int64_t nnz, const double* x, double* y)
{
    for (int64_t k = 0; k < nnz; ++k)
        y[rows[k]] += vals[k] * x[cols[k]];
}

/* Values as a matrix stored as f32 (vt 1) or bf16 (vt 2) holds them, widened
 * to f32: what an f32 SpMV multiplies. */
void orc_values_as_f32(const double* v, int64_t n, int vt, float* out)
{
    for (int64_t k = 0; k < n; ++k)
        out[k] = vt == ORC_VAL_F32 ? orc_f64_to_f32(v[k]) : (float)orc_bf16_to_f64(orc_f64_to_bf16(v[k]));
}

/* The same loop in f32 for matrices stored as f32 or bf16 (vals already
 * converted to f32): each product and each sum rounded to f32, the order of
 * the reference's loop (spmv/unified/spmv.cpp:1195-1201) kept. */
void orc_spmv_elements_f32(const int64_t* rows, const int64_t* cols, const float* vals,
                           int64_t nnz, const float* x, float* y)
{
    for (int64_t k = 0; k < nnz; ++k) {
        const float p = vals[k] * x[cols[k]];
        y[rows[k]] = y[rows[k]] + p;
    }
}

void orc_abs_spmv_elements(const int64_t* rows, const int64_t* cols, const double* vals,
                           int64_t nnz, const double* x, double* out)
{
    for (int64_t k = 0; k < nnz; ++k) {
        double p = vals[k] * x[cols[k]];
        out[rows[k]] += p < 0 ? -p : p;
    }
}

/* ---------------------------------------------------------------------------
 * Delta-coded row slices of the hypersparse block rows: the encoding the
 * library's SpMV reads for those block rows, restated element by element.
 * The reference's delta COO (spmv/orig/delta.cpp:118-219,
 * spmv/unified/spmv.cpp:815-1032) keeps the elements row by row and each
 * column as the difference to the previous one; here a row of more than
 * ORC_CHAIN_MIN elements is a chain with absolute columns, and the other
 * rows of a segment of block rows go to slices of up to 32 (one per lane,
 * stored column-major) by length.  Segments: the ORC_HOST_CHUNKS parts
 * [M c / 4, M (c + 1) / 4), each cut into pieces of at most 2^24 rows.
 * ------------------------------------------------------------------------ */
#define ORC_CHAIN_MIN 256
#define ORC_RING_TILES_MAX 256
#define ORC_HOST_CHUNKS 4
#define ORC_LEN_BITS 8

/* Elements of tile t in the format's order: local row / column of each. */
static int64_t tile_elements(const orc_matrix* a, int64_t t, int* lr, int* lc)
{
    const int s = a->s, lg = a->log2s;
    const uint8_t* pay = a->idx + a->tile_idx_off[t];
    const int64_t z = a->tile_val_off[t + 1] - a->tile_val_off[t];
    int64_t e = 0;
    switch (a->tile_scheme[t]) {
    case ORC_COO:
        for (e = 0; e < z; ++e) {
            const uint16_t k = ((const uint16_t*)pay)[e];
            lr[e] = k >> lg;
            lc[e] = k & (s - 1);
        }
        break;
    case ORC_CSR: {
        const uint16_t* re = (const uint16_t*)pay;
        for (int r = 0; r < s; ++r)
            for (int64_t q = r ? re[r - 1] : 0; q < re[r]; ++q) {
                lr[e] = r;
                lc[e] = pay[2 * s + q];
                ++e;
            }
        break;
    }
    case ORC_BITMAP: {
        const uint64_t* bm = (const uint64_t*)pay;
        for (int64_t bit = 0; bit < (int64_t)s * s; ++bit)
            if ((bm[bit >> 6] >> (bit & 63)) & 1u) {
                lr[e] = (int)(bit >> lg);
                lc[e] = (int)(bit & (s - 1));
                ++e;
            }
        break;
    }
    default:
        return -1;
    }
    return e;
}

static const int64_t* g_len_cmp;  /* row lengths for the comparator below */
static int by_length(const void* p, const void* q)
{
    const int a = *(const int*)p, b = *(const int*)q;
    if (g_len_cmp[a] != g_len_cmp[b])
        return g_len_cmp[a] > g_len_cmp[b] ? -1 : 1;
    return a < b ? -1 : a > b;
}

/* Row lengths of block row I (len[r], r < s). */
static void row_lengths(const orc_matrix* a, int64_t I, int* lr, int* lc, int64_t* len)
{
    for (int r = 0; r < a->s; ++r)
        len[r] = 0;
    for (int64_t t = a->brow_ptr[I]; t < a->brow_ptr[I + 1]; ++t) {
        const int64_t z = tile_elements(a, t, lr, lc);
        for (int64_t e = 0; e < z; ++e)
            len[lr[e]]++;
    }
}

/* The non-empty rows of a block row by length (longest first, then row). */
static int rows_by_length(int s, const int64_t* len, int* order)
{
    int live = 0;
    for (int r = 0; r < s; ++r)
        if (len[r])
            order[live++] = r;
    g_len_cmp = len;
    qsort(order, (size_t)live, sizeof(int), by_length);
    return live;
}

/* ascending (length desc, index asc) over rows q of the segment, lengths in g_seg_len */
static const int64_t* g_seg_len;
static int seg_by_length(const void* p, const void* q)
{
    const int64_t a = *(const int64_t*)p, b = *(const int64_t*)q;
    if (g_seg_len[a] != g_seg_len[b])
        return g_seg_len[a] > g_seg_len[b] ? -1 : 1;
    return a < b ? -1 : a > b;
}

/* Segment boundaries (block rows): nb + 1 values in b (room for M + 5). */
static int64_t slice_segments(int64_t M, int s, int64_t* b)
{
    int64_t piece = ((int64_t)1 << (32 - ORC_LEN_BITS)) / s, nb = 0;
    if (piece < 1)
        piece = 1;
    b[0] = 0;
    for (int c = 1; c <= ORC_HOST_CHUNKS; ++c) {
        const int64_t e = M * c / ORC_HOST_CHUNKS;
        while (e - b[nb] > piece) {
            b[nb + 1] = b[nb] + piece;
            ++nb;
        }
        if (e > b[nb])
            b[++nb] = e;
    }
    return nb;
}

int orc_slices_build(const orc_matrix* a, double avg, orc_slices** out)
{
    *out = (orc_slices*)calloc(1, sizeof(orc_slices));
    orc_slices* P = *out;
    if (!P)
        return ORC_ERR_NOMEM;
    const int s = a->s;
    if (avg <= 0 || (uint64_t)a->n > ((uint64_t)1 << 32))
        return ORC_OK;
    /* the block rows: non-empty, no dense tile, and no bitmap tile, at most
     * avg elements per tile on average or more than ORC_RING_TILES_MAX tiles */
    int64_t* sidx = (int64_t*)malloc(((size_t)a->M + 1) * sizeof(int64_t));
    int64_t E = 0, ns = 0;
    for (int64_t I = 0; I < a->M; ++I) {
        sidx[I] = -1;
        const int64_t t0 = a->brow_ptr[I], t1 = a->brow_ptr[I + 1];
        if (t1 == t0)
            continue;
        int ok = 1, bitmap = 0;
        for (int64_t t = t0; t < t1; ++t) {
            ok = ok && a->tile_scheme[t] != ORC_DENSE;
            bitmap = bitmap || a->tile_scheme[t] == ORC_BITMAP;
        }
        const int64_t e = a->tile_val_off[t1] - a->tile_val_off[t0];
        if (ok && ((double)e <= avg * (double)(t1 - t0) || t1 - t0 > ORC_RING_TILES_MAX || !bitmap)) {
            sidx[I] = ns++;
            E += e;
        }
    }
    if (ns == 0 || E == 0 || E >= ((int64_t)1 << 31) || ns * (int64_t)s >= ((int64_t)1 << 32)) {
        free(sidx);
        return ORC_OK;
    }
    int* lr = (int*)malloc((size_t)s * s * sizeof(int));
    int* lc = (int*)malloc((size_t)s * s * sizeof(int));
    int* order = (int*)malloc(s * sizeof(int));
    int64_t* len = (int64_t*)calloc((size_t)ns * s, sizeof(int64_t)); /* row q = k s + r */
    int64_t* browk = (int64_t*)malloc(ns * sizeof(int64_t));          /* block row of slice row k */
    for (int64_t I = 0; I < a->M; ++I)
        if (sidx[I] >= 0) {
            browk[sidx[I]] = I;
            row_lengths(a, I, lr, lc, len + sidx[I] * s);
        }
    int64_t* seg = (int64_t*)malloc(((size_t)a->M + 8) * sizeof(int64_t));
    const int64_t nseg = slice_segments(a->M, s, seg);
    int64_t* rest = (int64_t*)malloc(((size_t)ns * s + 1) * sizeof(int64_t));
    int64_t* slot0 = (int64_t*)malloc(((size_t)ns * s + 1) * sizeof(int64_t));
    uint8_t* chain = (uint8_t*)calloc((size_t)ns * s + 1, 1);
    /* the slices (two passes: count, then fill) */
    for (int pass = 0; pass < 2; ++pass) {
        int64_t nsl = 0, slots = 0, nlr = 0, k = 0;
        for (int64_t g = 0; g < nseg; ++g) {
            int64_t nrest = 0;
            for (; k < ns && browk[k] < seg[g + 1]; ++k) {
                const int live = rows_by_length(s, len + k * s, order);
                int i = 0;
                for (; i < live && len[k * s + order[i]] > ORC_CHAIN_MIN; ++i) {
                    const int64_t q = k * s + order[i];
                    if (pass) {
                        P->base[nsl] = slots;
                        P->meta[nsl] = order[i];
                        P->brow[nsl] = (uint32_t)browk[k];
                        P->steps[nsl] = (uint32_t)len[q];
                        P->lanes[nsl] = 1;
                        P->chain[nsl] = 1;
                        slot0[q] = slots;
                        chain[q] = 1;
                    }
                    ++nsl;
                    slots += len[q];
                }
                for (int r = 0; r < s; ++r) /* the others, ascending row */
                    if (len[k * s + r] && len[k * s + r] <= ORC_CHAIN_MIN)
                        rest[nrest++] = k * s + r;
            }
            g_seg_len = len;
            qsort(rest, (size_t)nrest, sizeof(int64_t), seg_by_length);
            for (int64_t i = 0; i < nrest; i += 32) {
                const int n32 = nrest - i < 32 ? (int)(nrest - i) : 32;
                if (pass) {
                    P->base[nsl] = slots;
                    P->meta[nsl] = nlr;
                    P->brow[nsl] = (uint32_t)seg[g];
                    P->steps[nsl] = (uint32_t)len[rest[i]];
                    P->lanes[nsl] = (uint32_t)n32;
                    P->chain[nsl] = 0;
                    for (int l = 0; l < n32; ++l) {
                        const int64_t q = rest[i + l];
                        const int64_t off = browk[q / s] * s + q % s - seg[g] * s;
                        P->lane[nlr + l] = (uint32_t)off << ORC_LEN_BITS | (uint32_t)(len[q] - 1);
                        slot0[q] = slots + l;
                    }
                }
                ++nsl;
                nlr += 32;
                slots += 32 * len[rest[i]];
            }
        }
        if (!pass) {
            P->base = (int64_t*)malloc((nsl + 1) * sizeof(int64_t));
            P->meta = (int64_t*)malloc((nsl + 1) * sizeof(int64_t));
            P->brow = (uint32_t*)malloc((nsl + 1) * sizeof(uint32_t));
            P->steps = (uint32_t*)malloc((nsl + 1) * sizeof(uint32_t));
            P->lanes = (uint32_t*)malloc((nsl + 1) * sizeof(uint32_t));
            P->chain = (uint8_t*)malloc(nsl + 1);
            P->lane = (uint32_t*)calloc(nlr + 1, sizeof(uint32_t));
            P->words = (uint32_t*)calloc(slots + 1, sizeof(uint32_t));
            P->vidx = (int64_t*)malloc((slots + 1) * sizeof(int64_t));
            for (int64_t q = 0; q < slots; ++q)
                P->vidx[q] = -1;
        } else {
            P->n = nsl;
            P->slots = slots;
            P->lane_records = nlr;
        }
    }
    /* every element at its slot: the k-th element of row q (format order
     * keeps a row's columns ascending) at slot0[q] + k (chain) or
     * slot0[q] + 32 k (sliced) */
    int64_t* fill = (int64_t*)malloc(s * sizeof(int64_t));
    int64_t* prev = (int64_t*)malloc(s * sizeof(int64_t));
    for (int64_t k = 0; k < ns; ++k) {
        const int64_t I = browk[k];
        for (int r = 0; r < s; ++r) {
            fill[r] = 0;
            prev[r] = 0;
        }
        for (int64_t t = a->brow_ptr[I]; t < a->brow_ptr[I + 1]; ++t) {
            const int64_t z = tile_elements(a, t, lr, lc);
            const int64_t c0 = (int64_t)a->tile_col[t] * s;
            for (int64_t e = 0; e < z; ++e) {
                const int r = lr[e];
                const int64_t q = k * s + r;
                const int64_t col = c0 + lc[e];
                const int64_t kk = fill[r]++;
                const int64_t slot = slot0[q] + (chain[q] ? kk : 32 * kk);
                P->words[slot] = (uint32_t)((chain[q] || kk == 0) ? col : col - prev[r]);
                P->vidx[slot] = a->tile_val_off[t] + e;
                prev[r] = col;
            }
        }
    }
    P->E = E;
    P->block_rows = ns;
    free(sidx);
    free(lr);
    free(lc);
    free(order);
    free(len);
    free(browk);
    free(seg);
    free(rest);
    free(slot0);
    free(chain);
    free(fill);
    free(prev);
    return ORC_OK;
}

void orc_slices_free(orc_slices* p)
{
    if (!p)
        return;
    free(p->base);
    free(p->meta);
    free(p->brow);
    free(p->steps);
    free(p->lanes);
    free(p->chain);
    free(p->lane);
    free(p->words);
    free(p->vidx);
    free(p);
}

/* y += A x over the slice rows: every row's words decoded in order (a
 * running column), each product added onto its row from y (f64 values). */
void orc_spmv_slices(const orc_matrix* a, const orc_slices* P, const double* x, double* y)
{
    const int s = a->s;
    const double* v = (const double*)a->values;
    for (int64_t q = 0; q < P->n; ++q) {
        const int nl = P->chain[q] ? 1 : (int)P->lanes[q];
        for (int l = 0; l < nl; ++l) {
            const uint32_t rec = P->chain[q] ? 0 : P->lane[P->meta[q] + l];
            const int64_t r = P->chain[q] ? P->meta[q] : (int64_t)(rec >> ORC_LEN_BITS);
            const int64_t n = P->chain[q] ? (int64_t)P->steps[q] : (int64_t)(rec & ((1u << ORC_LEN_BITS) - 1u)) + 1;
            const int64_t row = (int64_t)P->brow[q] * s + r;
            uint64_t col = 0;
            for (int64_t k = 0; k < n; ++k) {
                const int64_t slot = P->base[q] + (P->chain[q] ? k : 32 * k + l);
                const uint32_t w = P->words[slot];
                col = P->chain[q] ? w : (uint32_t)(col + w);
                y[row] += v[P->vidx[slot]] * x[col];
            }
        }
    }
}
