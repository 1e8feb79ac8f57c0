// builder.cu -- GPU construction of the ABHSF format and GPU block histograms.
//
// The reference builds nothing on a device: it partitions elements into
// blocks by sorting on the block key (block_statistics/block_stats.cpp:69-100,
// preprocessing/test.cpp:237-368) and evaluates the per-block cost model
// (include/abhsf/msmf.h:9-63).  Here the same partition is one radix sort of a
// 64-bit key on the device (CUB), and every other step -- key build, tile
// segmentation, per-tile scheme, offsets, payload scatter -- is a kernel of
// this file.  Results are deterministic: the only atomics are integer ORs /
// adds whose result does not depend on their order.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n)
{
    int64_t b = (n + kThreads - 1) / kThreads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32));
}

#define GRID_STRIDE(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

enum : int { kErrRange = 1, kErrDuplicate = 2, kErrCsrTooLong = 4, kErrHistOverflow = 8 };

// key = ((I * N + J) << 2 lg) | (lrow << lg) | lcol: tiles in (block row,
// block column) order, elements of a tile in row-major order.
__global__ void k_make_keys(const int64_t* __restrict__ rows, const int64_t* __restrict__ cols,
                            const double* __restrict__ vals, int64_t nnz, int64_t m, int64_t n, int lg,
                            uint64_t N, uint64_t* __restrict__ keys, double* __restrict__ vout,
                            int* __restrict__ err)
{
    const uint64_t lmask = (uint64_t(1) << lg) - 1;
    GRID_STRIDE(i, nnz)
    {
        const int64_t r = rows[i], c = cols[i];
        if (r < 0 || r >= m || c < 0 || c >= n) {
            atomicOr(err, kErrRange);
            keys[i] = 0;
            vout[i] = 0.0;
            continue;
        }
        const uint64_t I = uint64_t(r) >> lg, J = uint64_t(c) >> lg;
        keys[i] = ((I * N + J) << (2 * lg)) | ((uint64_t(r) & lmask) << lg) | (uint64_t(c) & lmask);
        vout[i] = vals ? vals[i] : 1.0;
    }
}

// head[i] = 1 where a new block starts (key >> shift changes); flags
// duplicate (row, col) pairs when check_dup.
__global__ void k_heads(const uint64_t* __restrict__ keys, int64_t nnz, int shift, int check_dup,
                        int64_t* __restrict__ head, int* __restrict__ err)
{
    GRID_STRIDE(i, nnz)
    {
        const uint64_t k = keys[i];
        int64_t h = 1;
        if (i > 0) {
            const uint64_t p = keys[i - 1];
            if (check_dup && p == k)
                atomicOr(err, kErrDuplicate);
            h = ((p >> shift) != (k >> shift)) ? 1 : 0;
        }
        head[i] = h;
    }
}

// After an inclusive scan of the head flags, tile_of[i] is 1 + the tile of i.
__global__ void k_tile_starts(const uint64_t* __restrict__ keys, const int64_t* __restrict__ tile_of,
                              int64_t nnz, int shift, int64_t* __restrict__ tile_start,
                              uint64_t* __restrict__ tile_key)
{
    GRID_STRIDE(i, nnz)
    {
        const int64_t t = tile_of[i] - 1;
        if (i == 0 || tile_of[i - 1] != tile_of[i]) {
            tile_start[t] = i;
            if (tile_key)
                tile_key[t] = keys[i] >> shift;
        }
        if (i == nnz - 1)
            tile_start[t + 1] = nnz;
    }
}

struct scheme_params {
    int64_t s;
    uint64_t bits;
    int is_binary, allow_csr, forced;
};

__global__ void k_tile_meta(int64_t T, const int64_t* __restrict__ tile_start, const uint64_t* __restrict__ tile_key,
                            uint64_t N, scheme_params sp, int64_t* __restrict__ tile_row,
                            uint32_t* __restrict__ tile_col, uint32_t* __restrict__ tile_nnz,
                            uint8_t* __restrict__ tile_scheme, int64_t* __restrict__ stored,
                            int64_t* __restrict__ pay, int* __restrict__ err)
{
    GRID_STRIDE(t, T + 1)
    {
        if (t == T) {  // the scans run over T + 1 entries; the last yields the totals
            stored[T] = 0;
            pay[T] = 0;
            continue;
        }
        const int64_t z = tile_start[t + 1] - tile_start[t];
        const uint64_t tk = tile_key[t];
        int sch = sp.forced;
        if (sch < 0)
            sch = abhsf_select_scheme(sp.s, sp.s, (uint64_t)z, sp.bits, sp.is_binary, sp.allow_csr, nullptr);
        if (sch == ABHSF_SCHEME_CSR && z > 65535)
            atomicOr(err, kErrCsrTooLong);
        tile_row[t] = (int64_t)(tk / N);
        tile_col[t] = (uint32_t)(tk % N);
        tile_nnz[t] = (uint32_t)z;
        tile_scheme[t] = (uint8_t)sch;
        stored[t] = (sch == ABHSF_SCHEME_DENSE) ? sp.s * sp.s : z;
        pay[t] = tile_payload_bytes(sch, sp.s, z);
    }
}

// brow_ptr[i] = first tile whose block row is >= i.
__global__ void k_brow_ptr(int64_t M, int64_t T, const int64_t* __restrict__ tile_row, int64_t* __restrict__ brow_ptr)
{
    GRID_STRIDE(i, M + 1)
    {
        int64_t lo = 0, hi = T;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (tile_row[mid] < i)
                lo = mid + 1;
            else
                hi = mid;
        }
        brow_ptr[i] = lo;
    }
}

__device__ __forceinline__ uint16_t f64_to_bf16_bits(double v)
{
    const float f = __double2float_rn(v);
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu))
        return (uint16_t)((u >> 16) | 0x0040u);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

__global__ void k_scatter(const uint64_t* __restrict__ keys, const double* __restrict__ vals,
                          const int64_t* __restrict__ tile_of, int64_t nnz, int lg,
                          const int64_t* __restrict__ tile_start, const uint8_t* __restrict__ tile_scheme,
                          const int64_t* __restrict__ tile_val_off, const int64_t* __restrict__ tile_idx_off,
                          int value_type, uint8_t* __restrict__ payload, void* __restrict__ values)
{
    const int64_t s = int64_t(1) << lg;
    const uint64_t lmask = (uint64_t(1) << (2 * lg)) - 1;
    GRID_STRIDE(i, nnz)
    {
        const int64_t t = tile_of[i] - 1;
        const int64_t p = i - tile_start[t];
        const uint64_t local = keys[i] & lmask;
        const uint32_t lr = (uint32_t)(local >> lg), lc = (uint32_t)(local & (s - 1));
        const int sch = tile_scheme[t];
        const int64_t vpos = tile_val_off[t] + (sch == ABHSF_SCHEME_DENSE ? (int64_t)local : p);
        const double v = vals[i];
        if (value_type == ABHSF_VALUE_F64)
            static_cast<double*>(values)[vpos] = v;
        else if (value_type == ABHSF_VALUE_F32)
            static_cast<float*>(values)[vpos] = __double2float_rn(v);
        else
            static_cast<uint16_t*>(values)[vpos] = f64_to_bf16_bits(v);
        uint8_t* pay = payload + tile_idx_off[t];
        if (sch == ABHSF_SCHEME_COO) {
            reinterpret_cast<uint16_t*>(pay)[p] = (uint16_t)((lr << lg) | lc);
        } else if (sch == ABHSF_SCHEME_CSR) {
            pay[2 * s + p] = (uint8_t)lc;
            // The last element of each row writes row_end for its row and the
            // empty rows that follow it (rows before the first element stay 0).
            const int64_t tend = tile_start[t + 1];
            uint32_t next_lr = (uint32_t)s;
            if (i + 1 < tend)
                next_lr = (uint32_t)((keys[i + 1] & lmask) >> lg);
            if (next_lr != lr) {
                uint16_t* row_end = reinterpret_cast<uint16_t*>(pay);
                for (uint32_t r = lr; r < next_lr; ++r)
                    row_end[r] = (uint16_t)(p + 1);
            }
        } else if (sch == ABHSF_SCHEME_BITMAP) {
            atomicOr(reinterpret_cast<unsigned long long*>(pay) + (local >> 6), 1ull << (local & 63));
        }
    }
}

// Duplicate elements are counted like distinct ones (as block_stats.cpp does),
// so a run may exceed r * s: such runs are reported, never written past hist.
__global__ void k_len_hist(int64_t B, const int64_t* __restrict__ start, unsigned long long* __restrict__ hist,
                           int64_t hist_len, int* __restrict__ err)
{
    GRID_STRIDE(b, B)
    {
        const int64_t len = start[b + 1] - start[b];
        if (len < hist_len)
            atomicAdd(hist + len, 1ull);
        else
            atomicOr(err, kErrHistOverflow);
    }
}

__global__ void k_block_keys(const int64_t* __restrict__ rows, const int64_t* __restrict__ cols, int64_t nnz,
                             int64_t m, int64_t n, int k, int l, uint64_t* __restrict__ keys, int* __restrict__ err)
{
    GRID_STRIDE(i, nnz)
    {
        const int64_t r = rows[i], c = cols[i];
        if (r < 0 || r >= m || c < 0 || c >= n) {
            atomicOr(err, kErrRange);
            keys[i] = 0;
            continue;
        }
        // block_statistics/block_stats.cpp:69-74
        keys[i] = ((uint64_t(r) >> k) << 32) + (uint64_t(c) >> l);
    }
}

// All 64 block sizes: elements sorted by (column >> l, row) put every block
// of 2^k x 2^l (k = 1..8) in one run, so one sort per column width l serves
// eight block heights.
__global__ void k_col_row_keys(const int64_t* __restrict__ rows, const int64_t* __restrict__ cols, int64_t nnz,
                               int64_t m, int64_t n, int l, uint64_t* __restrict__ keys, int* __restrict__ err)
{
    GRID_STRIDE(i, nnz)
    {
        const int64_t r = rows[i], c = cols[i];
        if (r < 0 || r >= m || c < 0 || c >= n) {
            atomicOr(err, kErrRange);
            keys[i] = 0;
            continue;
        }
        keys[i] = ((uint64_t(c) >> l) << 32) | uint64_t(r);
    }
}

// Bit k - 1 of heads[e]: element e starts a 2^k x 2^l block in the sorted order.
__global__ void k_block_heads_all(const uint64_t* __restrict__ keys, int64_t nnz, uint8_t* __restrict__ heads)
{
    GRID_STRIDE(e, nnz)
    {
        uint8_t h = 0xff;
        if (e > 0) {
            const uint64_t a = keys[e - 1], b = keys[e];
            if ((a >> 32) == (b >> 32)) {
                const uint32_t ra = (uint32_t)a, rb = (uint32_t)b;
                h = 0;
#pragma unroll
                for (int k = 1; k <= 8; ++k)
                    h |= (uint8_t)(((ra >> k) != (rb >> k)) << (k - 1));
            }
        }
        heads[e] = h;
    }
}

__global__ void k_head_bit(const uint8_t* __restrict__ heads, int64_t nnz, int bit, uint8_t* __restrict__ flag)
{
    GRID_STRIDE(e, nnz)
    flag[e] = (heads[e] >> bit) & 1u;
}

__global__ void k_iota(int64_t nnz, int64_t* __restrict__ out)
{
    GRID_STRIDE(e, nnz)
    out[e] = e;
}

// Block lengths into a histogram held in shared memory (hist_len <= 8192),
// then added to the global one.
__global__ void k_len_hist_shared(int64_t B, const int64_t* __restrict__ start, int64_t nnz,
                                  unsigned long long* __restrict__ hist, int hist_len, int* __restrict__ err)
{
    extern __shared__ unsigned int sh[];
    for (int i = threadIdx.x; i < hist_len; i += blockDim.x)
        sh[i] = 0;
    __syncthreads();
    GRID_STRIDE(b, B)
    {
        const int64_t len = (b + 1 < B ? start[b + 1] : nnz) - start[b];
        if (len < hist_len)
            atomicAdd(&sh[len], 1u);
        else
            atomicOr(err, kErrHistOverflow);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < hist_len; i += blockDim.x)
        if (sh[i])
            atomicAdd(hist + i, (unsigned long long)sh[i]);
}

__global__ void k_len_hist_global(int64_t B, const int64_t* __restrict__ start, int64_t nnz,
                                  unsigned long long* __restrict__ hist, int64_t hist_len, int* __restrict__ err)
{
    GRID_STRIDE(b, B)
    {
        const int64_t len = (b + 1 < B ? start[b + 1] : nnz) - start[b];
        if (len < hist_len)
            atomicAdd(hist + len, 1ull);
        else
            atomicOr(err, kErrHistOverflow);
    }
}

void check_launch(const char* what) { ABHSF_CUDA(cudaGetLastError()); (void)what; }

template <typename T>
T read_scalar(const T* dptr, cudaStream_t st)
{
    T v{};
    ABHSF_CUDA(cudaMemcpyAsync(&v, dptr, sizeof(T), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    return v;
}

// Copies host inputs to the device (or wraps device inputs).
struct coo_inputs {
    dbuf<int64_t> rows_d, cols_d;
    dbuf<double> vals_d;
    const int64_t* rows = nullptr;
    const int64_t* cols = nullptr;
    const double* vals = nullptr;

    coo_inputs(const int64_t* r, const int64_t* c, const double* v, int64_t nnz, bool on_device, cudaStream_t st)
    {
        if (on_device) {
            rows = r; cols = c; vals = v;
            return;
        }
        rows_d.alloc(nnz);
        cols_d.alloc(nnz);
        ABHSF_CUDA(cudaMemcpyAsync(rows_d.get(), r, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(cols_d.get(), c, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        rows = rows_d.get();
        cols = cols_d.get();
        if (v) {
            vals_d.alloc(nnz);
            ABHSF_CUDA(cudaMemcpyAsync(vals_d.get(), v, nnz * sizeof(double), cudaMemcpyHostToDevice, st));
            vals = vals_d.get();
        }
    }
};

// Segments sorted keys into runs of equal (key >> shift); returns the run
// count and fills start[0..runs] (start[runs] = nnz) and optionally run keys.
int64_t segment_runs(const uint64_t* keys, int64_t nnz, int shift, bool check_dup, cudaStream_t st,
                     dbuf<int64_t>& tile_of, dbuf<int64_t>& start, dbuf<uint64_t>* run_key, int* err)
{
    dbuf<int64_t> head(nnz);
    tile_of.alloc(nnz);
    k_heads<<<grid_for(nnz), kThreads, 0, st>>>(keys, nnz, shift, check_dup ? 1 : 0, head.get(), err);
    check_launch("k_heads");
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, head.get(), tile_of.get(), nnz, st));
    dbuf<uint8_t> tmp(tmp_bytes);
    ABHSF_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tmp_bytes, head.get(), tile_of.get(), nnz, st));
    const int64_t runs = read_scalar(tile_of.get() + nnz - 1, st);
    start.alloc(runs + 1);
    if (run_key)
        run_key->alloc(runs);
    k_tile_starts<<<grid_for(nnz), kThreads, 0, st>>>(keys, tile_of.get(), nnz, shift, start.get(),
                                                       run_key ? run_key->get() : nullptr);
    check_launch("k_tile_starts");
    return runs;
}

void sort_pairs(dbuf<uint64_t>& keys, dbuf<double>& vals, int64_t nnz, int end_bit, cudaStream_t st)
{
    dbuf<uint64_t> keys_out(nnz);
    dbuf<double> vals_out(nnz);
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.get(), keys_out.get(), vals.get(),
                                               vals_out.get(), nnz, 0, end_bit, st));
    dbuf<uint8_t> tmp(tmp_bytes);
    ABHSF_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, keys.get(), keys_out.get(), vals.get(),
                                               vals_out.get(), nnz, 0, end_bit, st));
    keys = std::move(keys_out);
    vals = std::move(vals_out);
}

void exclusive_scan(int64_t* in, int64_t* out, int64_t count, cudaStream_t st)
{
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, count, st));
    dbuf<uint8_t> tmp(tmp_bytes);
    ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmp_bytes, in, out, count, st));
}

void raise_err(int e)
{
    if (e & kErrRange)
        fail(ABHSF_ERROR_INDEX_OUT_OF_RANGE, "an element lies outside the m x n matrix");
    if (e & kErrDuplicate)
        fail(ABHSF_ERROR_DUPLICATE_ENTRY, "two elements share one (row, col) position");
    if (e & kErrCsrTooLong)
        fail(ABHSF_ERROR_UNSUPPORTED, "forced CSR tile with more than 65535 nonzeros (uint16 row_end)");
    if (e & kErrHistOverflow)
        fail(ABHSF_ERROR_INVALID_VALUE, "a block holds more elements than hist_len - 1 (duplicate elements)");
}

}  // namespace

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t count, cudaStream_t st)
{
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, count, st));
    dbuf<uint8_t> tmp(tmp_bytes);
    ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmp_bytes, in, out, count, st));
}

void inclusive_scan_i64(const int64_t* in, int64_t* out, int64_t count, cudaStream_t st)
{
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, in, out, count, st));
    dbuf<uint8_t> tmp(tmp_bytes);
    ABHSF_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), tmp_bytes, in, out, count, st));
}

// Host computation of one mmf line (block_statistics/mmf.cpp:53-138) for a
// given single-precision element width bits1 (32 for INTEGER / REAL, 64 for
// COMPLEX, 0 for BINARY: mmf.cpp:34-47); the double line uses 2 * bits1.
void mmf_line_from_hist(int64_t m, int64_t n, int64_t nnz, int type, int64_t r, int64_t s,
                        const std::map<uint64_t, uint64_t>& hist, uint64_t bits1, uint64_t o1[8], uint64_t o2[8])
{
    const bool is_binary = (type == ABHSF_MATRIX_BINARY);
    const uint64_t M = (uint64_t)((m + r - 1) / r), N = (uint64_t)((n + s - 1) / s);
    uint64_t blocks = 0;
    for (const auto& kv : hist)
        blocks += kv.second;
    const uint64_t csr0 = M * abhsf_ceil_log2(N + 1) + blocks * abhsf_ceil_log2(N);
    uint64_t coo = csr0, csr = csr0, bmp = csr0, d1 = csr0, d2 = csr0, a1 = csr0, a2 = csr0, w1 = csr0, w2 = csr0;
    if (is_binary)
        d1 = d2 = UINT64_MAX;
    const uint64_t R = (uint64_t)r, S = (uint64_t)s;
    for (const auto& kv : hist) {
        const uint64_t z = kv.first, c = kv.second;
        if (!c)
            continue;
        coo += abhsf_coo_bits(R, S, z) * c;
        csr += abhsf_csr_bits(R, S, z) * c;
        bmp += abhsf_bitmap_bits(R, S) * c;
        if (!is_binary) {
            d1 += abhsf_dense_bits(R, S, z, bits1) * c;
            d2 += abhsf_dense_bits(R, S, z, 2 * bits1) * c;
        }
        uint64_t b;
        abhsf_select_scheme(R, S, z, bits1, is_binary, 1, &b);
        a1 += (b + 2) * c;
        abhsf_select_scheme(R, S, z, 2 * bits1, is_binary, 1, &b);
        a2 += (b + 2) * c;
        abhsf_select_scheme(R, S, z, bits1, is_binary, 0, &b);
        w1 += (b + 2) * c;
        abhsf_select_scheme(R, S, z, 2 * bits1, is_binary, 0, &b);
        w2 += (b + 2) * c;
    }
    const uint64_t coo32 = (uint64_t)nnz * 64, csr32 = ((uint64_t)m + 1 + (uint64_t)nnz) * 32;
    const uint64_t v1 = (uint64_t)nnz * bits1, v2 = 2 * v1;
    const uint64_t s1[8] = {coo32 + v1, csr32 + v1, coo + v1, csr + v1, bmp + v1, d1 + v1, a1 + v1, w1 + v1};
    const uint64_t s2[8] = {coo32 + v2, csr32 + v2, coo + v2, csr + v2, bmp + v2, d2 + v2, a2 + v2, w2 + v2};
    std::copy(s1, s1 + 8, o1);
    std::copy(s2, s2 + 8, o2);
}

// ABHSF storage (bits, the mmf line's abhsf column at the stored value width,
// CSR as the options allow) of square block sizes 16, 32, 64, 128, 256: the
// quantity the reference's min-bss tool minimises (block_statistics/min-bss.cpp:14-58).
void block_size_storage(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n,
                        const abhsf_build_opts& o, cudaStream_t st, uint64_t bits[kNumBlockSizes])
{
    if (o.value_type < 0 || o.value_type > 2)
        fail(ABHSF_ERROR_INVALID_VALUE, "value_type out of range");
    if (o.matrix_type < 0 || o.matrix_type > 3)
        fail(ABHSF_ERROR_INVALID_VALUE, "matrix_type out of range");
    const uint64_t dense_bits = o.bits_per_value > 0 ? (uint64_t)o.bits_per_value : 8 * value_size(o.value_type);
    const uint64_t bits1 = (o.matrix_type == ABHSF_MATRIX_BINARY) ? 0 : dense_bits / 2;
    if (nnz > 0 && (!rows || !cols))
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL");
    coo_inputs in(rows, cols, nullptr, nnz, o.inputs_on_device != 0, st);  // host inputs cross once
    for (int k = 0; k < kNumBlockSizes; ++k) {
        const int s = 16 << k;
        std::vector<uint64_t> h((size_t)s * s + 1);
        int64_t blocks = 0;
        block_histogram(in.rows, in.cols, nnz, m, n, s, s, true, st, h.data(), (int64_t)h.size(), &blocks);
        std::map<uint64_t, uint64_t> hist;
        for (size_t z = 1; z < h.size(); ++z)
            if (h[z])
                hist[z] = h[z];
        uint64_t o1[8], o2[8];
        mmf_line_from_hist(m, n, nnz, o.matrix_type, s, s, hist, bits1, o1, o2);
        bits[k] = o.allow_csr ? o2[6] : o2[7];
    }
}

int select_block_size(const uint64_t bits[kNumBlockSizes])
{
    int best = 0;
    for (int k = 1; k < kNumBlockSizes; ++k)
        if (bits[k] < bits[best])
            best = k;
    return 16 << best;
}

namespace {

void finish_stats(abhsf_matrix& a, uint64_t dense_bits, cudaStream_t st)
{
    std::vector<uint32_t> nz(a.T);
    std::vector<uint8_t> sch(a.T);
    if (a.T) {
        ABHSF_CUDA(cudaMemcpyAsync(nz.data(), a.tile_nnz.get(), a.T * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(sch.data(), a.tile_scheme.get(), a.T, cudaMemcpyDeviceToHost, st));
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));
    abhsf_stats& s = a.stats;
    s = abhsf_stats{};
    s.m = a.m; s.n = a.n; s.nnz = a.nnz;
    s.block_size = a.s; s.value_type = a.value_type;
    s.block_rows = a.M; s.block_cols = a.N; s.tiles = a.T;
    std::map<uint64_t, uint64_t> hist;
    for (int64_t t = 0; t < a.T; ++t) {
        s.tiles_per_scheme[sch[t]]++;
        s.nnz_per_scheme[sch[t]] += nz[t];
        hist[nz[t]]++;
    }
    s.stored_values = a.n_values;
    s.payload_bytes = a.payload_bytes;
    s.format_bytes = (a.M + 1) * 8 + a.T * (4 + 4 + 1) + (a.T + 1) * 16 + a.payload_bytes +
                     a.n_values * (int64_t)value_size(a.value_type);
    s.spmv_bytes = s.format_bytes;  // the row slices, where prepared, replace their block rows' part
    // mmf line at this block size whose "double" column has the dense-cost
    // width; binary matrices carry no value bits (mmf.cpp:45-46).
    uint64_t o1[8], o2[8];
    const uint64_t bits1 = (a.matrix_type == ABHSF_MATRIX_BINARY) ? 0 : dense_bits / 2;
    mmf_line_from_hist(a.m, a.n, a.nnz, a.matrix_type, a.s, a.s, hist, bits1, o1, o2);
    std::copy(o2, o2 + 8, s.msmf_bits);
}

}  // namespace

void build_matrix(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m, int64_t n,
                  const abhsf_build_opts& o, cudaStream_t st, abhsf_matrix& a)
{
    const int lg = log2_exact(o.block_size);
    if (lg < 4 || lg > 8)
        fail(ABHSF_ERROR_INVALID_VALUE, "block_size must be 16, 32, 64, 128 or 256");
    if (o.value_type < 0 || o.value_type > 2)
        fail(ABHSF_ERROR_INVALID_VALUE, "value_type out of range");
    if (o.matrix_type < 0 || o.matrix_type > 3)
        fail(ABHSF_ERROR_INVALID_VALUE, "matrix_type out of range");
    if (o.matrix_type == ABHSF_MATRIX_COMPLEX)
        fail(ABHSF_ERROR_UNSUPPORTED, "complex values are not stored by this build");
    if (o.forced_scheme < -1 || o.forced_scheme > 3)
        fail(ABHSF_ERROR_INVALID_VALUE, "forced_scheme must be -1 or 0..3");
    if (o.sum_order != ABHSF_SUM_REFERENCE && o.sum_order != ABHSF_SUM_TREE)
        fail(ABHSF_ERROR_INVALID_VALUE, "sum_order must be ABHSF_SUM_REFERENCE or ABHSF_SUM_TREE");
    if (o.slice_tile_nnz < -1)
        fail(ABHSF_ERROR_INVALID_VALUE, "slice_tile_nnz must be -1, 0 or positive");
    const bool binary = (o.matrix_type == ABHSF_MATRIX_BINARY);
    if (binary && o.forced_scheme == ABHSF_SCHEME_DENSE)
        fail(ABHSF_ERROR_INVALID_VALUE, "dense scheme is never used for binary matrices");
    if (m <= 0 || n <= 0 || nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
    if (nnz > 0 && (!rows || !cols))
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL");
    if (!vals && !binary && nnz > 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "vals may be NULL only for binary matrices");
    const int64_t s = o.block_size;
    const int64_t M = (m + s - 1) / s, N = (n + s - 1) / s;
    if (M > int64_t(UINT32_MAX) || N > int64_t(UINT32_MAX))
        fail(ABHSF_ERROR_UNSUPPORTED, "more than 2^32 block rows or columns");
    const int key_bits = bit_length((uint64_t)(M * N - 1)) + 2 * lg;
    if (key_bits > 64)
        fail(ABHSF_ERROR_UNSUPPORTED, "matrix too large for a 64-bit block key");
    const uint64_t dense_bits = o.bits_per_value > 0 ? (uint64_t)o.bits_per_value : 8 * value_size(o.value_type);

    a.m = m; a.n = n; a.nnz = nnz; a.s = (int32_t)s; a.lg = lg;
    a.value_type = o.value_type; a.matrix_type = o.matrix_type;
    a.sum_order = o.sum_order;
    a.dc_avg = o.slice_tile_nnz < 0 ? 0.f : o.slice_tile_nnz == 0 ? kSliceTileNnzDefault : (float)o.slice_tile_nnz;
    a.M = M; a.N = N;
    ABHSF_CUDA(cudaGetDevice(&a.device));

    dbuf<int> err(1);
    ABHSF_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    dbuf<int64_t> tile_of, tile_start, tile_row, stored, pay;
    dbuf<uint64_t> keys, tile_key;
    dbuf<double> svals;
    int64_t T = 0;
    if (nnz > 0) {
        coo_inputs in(rows, cols, binary ? nullptr : vals, nnz, o.inputs_on_device != 0, st);
        keys.alloc(nnz);
        svals.alloc(nnz);
        k_make_keys<<<grid_for(nnz), kThreads, 0, st>>>(in.rows, in.cols, in.vals, nnz, m, n, lg, (uint64_t)N,
                                                         keys.get(), svals.get(), err.get());
        check_launch("k_make_keys");
        raise_err(read_scalar(err.get(), st));
    }
    if (nnz > 0) {
        sort_pairs(keys, svals, nnz, key_bits, st);
        T = segment_runs(keys.get(), nnz, 2 * lg, true, st, tile_of, tile_start, &tile_key, err.get());
        raise_err(read_scalar(err.get(), st));
    }
    a.T = T;
    a.brow_ptr.alloc(M + 1);
    a.tile_col.alloc(T);
    a.tile_nnz.alloc(T);
    a.tile_scheme.alloc(T);
    a.tile_val_off.alloc(T + 1);
    a.tile_idx_off.alloc(T + 1);
    tile_row.alloc(T);
    stored.alloc(T + 1);
    pay.alloc(T + 1);
    scheme_params sp{s, dense_bits, binary ? 1 : 0, o.allow_csr ? 1 : 0, o.forced_scheme};
    k_tile_meta<<<grid_for(T + 1), kThreads, 0, st>>>(T, tile_start.get(), tile_key.get(), (uint64_t)N, sp,
                                                       tile_row.get(), a.tile_col.get(), a.tile_nnz.get(),
                                                       a.tile_scheme.get(), stored.get(), pay.get(), err.get());
    check_launch("k_tile_meta");
    exclusive_scan(stored.get(), a.tile_val_off.get(), T + 1, st);
    exclusive_scan(pay.get(), a.tile_idx_off.get(), T + 1, st);
    k_brow_ptr<<<grid_for(M + 1), kThreads, 0, st>>>(M, T, tile_row.get(), a.brow_ptr.get());
    check_launch("k_brow_ptr");
    raise_err(read_scalar(err.get(), st));
    a.n_values = read_scalar(a.tile_val_off.get() + T, st);
    a.payload_bytes = read_scalar(a.tile_idx_off.get() + T, st);
    a.payload.alloc(a.payload_bytes);
    // 16 bytes of padding: pipelined kernels copy 16-byte-aligned supersets of value ranges
    a.values.alloc(a.n_values * value_size(a.value_type) + 16);
    ABHSF_CUDA(cudaMemsetAsync(a.payload.get(), 0, a.payload.size(), st));
    ABHSF_CUDA(cudaMemsetAsync(a.values.get(), 0, a.values.size(), st));
    if (nnz > 0) {
        k_scatter<<<grid_for(nnz), kThreads, 0, st>>>(keys.get(), svals.get(), tile_of.get(), nnz, lg,
                                                       tile_start.get(), a.tile_scheme.get(), a.tile_val_off.get(),
                                                       a.tile_idx_off.get(), a.value_type, a.payload.get(),
                                                       a.values.get());
        check_launch("k_scatter");
    }
    a.dev_status.alloc(1);
    ABHSF_CUDA(cudaMemsetAsync(a.dev_status.get(), 0, sizeof(int), st));
    finish_stats(a, dense_bits, st);
    prepare_tree(a, st);
    prepare_ring(a, st);
}

void block_histogram(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, int r, int s,
                     bool on_device, cudaStream_t st, uint64_t* hist, int64_t hist_len, int64_t* blocks)
{
    const int k = log2_exact(r), l = log2_exact(s);
    if (k < 1 || k > 8 || l < 1 || l > 8)
        fail(ABHSF_ERROR_INVALID_VALUE, "r and s must be powers of two in 2..256");
    if (m <= 0 || n <= 0 || nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
    if (!hist || hist_len < (int64_t)r * s + 1)
        fail(ABHSF_ERROR_INVALID_VALUE, "hist must hold r*s + 1 counters");
    if (((uint64_t)(m - 1) >> k) >= (uint64_t(1) << 32) || ((uint64_t)(n - 1) >> l) >= (uint64_t(1) << 32))
        fail(ABHSF_ERROR_UNSUPPORTED, "block row or column index beyond 32 bits");
    std::fill(hist, hist + hist_len, 0);
    if (blocks)
        *blocks = 0;
    if (nnz == 0)
        return;
    if (!rows || !cols)
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL");
    coo_inputs in(rows, cols, nullptr, nnz, on_device, st);
    dbuf<int> err(1);
    ABHSF_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    dbuf<uint64_t> keys(nnz), keys_out(nnz);
    k_block_keys<<<grid_for(nnz), kThreads, 0, st>>>(in.rows, in.cols, nnz, m, n, k, l, keys.get(), err.get());
    check_launch("k_block_keys");
    raise_err(read_scalar(err.get(), st));
    const int end_bit = 32 + bit_length((uint64_t)(m - 1) >> k);
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, keys.get(), keys_out.get(), nnz, 0, end_bit, st));
    {
        dbuf<uint8_t> tmp(tmp_bytes);
        ABHSF_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(), tmp_bytes, keys.get(), keys_out.get(), nnz, 0, end_bit,
                                                  st));
    }
    dbuf<int64_t> run_of, start;
    const int64_t B = segment_runs(keys_out.get(), nnz, 0, false, st, run_of, start, nullptr, err.get());
    dbuf<unsigned long long> dh(hist_len);
    ABHSF_CUDA(cudaMemsetAsync(dh.get(), 0, hist_len * sizeof(unsigned long long), st));
    k_len_hist<<<grid_for(B), kThreads, 0, st>>>(B, start.get(), dh.get(), hist_len, err.get());
    check_launch("k_len_hist");
    ABHSF_CUDA(cudaMemcpyAsync(hist, dh.get(), hist_len * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    raise_err(read_scalar(err.get(), st));
    if (blocks)
        *blocks = B;
}

// ---------------------------------------------------------------------------
// Block histogram that allocates nothing (abhsf_block_histogram_noalloc).
//
// For callers that may not call cudaMalloc: processes whose device memory is
// handed out by their own allocator or pool, paths where a cudaMalloc (which
// can synchronise the device) is not acceptable, and processes already at
// their device-memory limit.  All scratch lives in the array below, which is
// part of the library's device image: every GPU that loads the library holds
// it until the process exits.  Every call reuses it; a call clears what must
// start at zero, and calls that overlap on the GPU race on it.
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device.  Looked up once
// per device with that device current; host code may not use the symbol
// itself as an address.
unsigned char* noalloc_scratch()
{
    int dev = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        fail(ABHSF_ERROR_UNSUPPORTED, "device index beyond the no-allocation table");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        ABHSF_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_noalloc_ptr[dev];
}

// Hands out 256-byte-aligned pieces of the scratch array.
struct scratch_arena {
    unsigned char* base;
    size_t cap, used = 0;
    template <typename T>
    T* take(size_t count)
    {
        const size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
        if (used + bytes > cap)
            fail(ABHSF_ERROR_INVALID_VALUE, "input too large for the no-allocation scratch");
        T* p = reinterpret_cast<T*>(base + used);
        used += bytes;
        return p;
    }
};

}  // namespace

void block_histogram_all(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, bool on_device,
                         cudaStream_t st, uint64_t* hist, int64_t* blocks)
{
    if (m <= 0 || n <= 0 || nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
    if (!hist)
        fail(ABHSF_ERROR_INVALID_VALUE, "hist must hold ABHSF_BSTATS_ALL_LEN counters");
    if ((uint64_t)(m - 1) >= (uint64_t(1) << 32) || ((uint64_t)(n - 1) >> 1) >= (uint64_t(1) << 32))
        fail(ABHSF_ERROR_UNSUPPORTED, "row index or block column index beyond 32 bits");
    std::fill(hist, hist + ABHSF_BSTATS_ALL_LEN, 0);
    if (blocks)
        std::fill(blocks, blocks + 64, 0);
    if (nnz == 0)
        return;
    if (!rows || !cols)
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL");
    coo_inputs in(rows, cols, nullptr, nnz, on_device, st);
    dbuf<int> err(1);
    ABHSF_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), st));
    dbuf<unsigned long long> dh(ABHSF_BSTATS_ALL_LEN);
    ABHSF_CUDA(cudaMemsetAsync(dh.get(), 0, ABHSF_BSTATS_ALL_LEN * sizeof(unsigned long long), st));
    dbuf<uint64_t> keys(nnz), sorted(nnz);
    dbuf<uint8_t> heads(nnz), flag(nnz);
    dbuf<int64_t> iota(nnz), starts(nnz);
    dbuf<int64_t> nsel(1);
    k_iota<<<grid_for(nnz), kThreads, 0, st>>>(nnz, iota.get());
    check_launch("k_iota");
    size_t sort_bytes = 0, sel_bytes = 0;
    ABHSF_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, keys.get(), sorted.get(), nnz, 0, 64, st));
    ABHSF_CUDA(cub::DeviceSelect::Flagged(nullptr, sel_bytes, iota.get(), flag.get(), starts.get(), nsel.get(), nnz,
                                          st));
    dbuf<uint8_t> tmp(std::max(sort_bytes, sel_bytes));
    std::vector<int64_t> count(64, 0);
    int64_t off[64];
    for (int p = 0, o = 0; p < 64; ++p) {
        off[p] = o;
        o += (1 << (p / 8 + 1)) * (1 << (p % 8 + 1)) + 1;
    }
    for (int l = 1; l <= 8; ++l) {
        k_col_row_keys<<<grid_for(nnz), kThreads, 0, st>>>(in.rows, in.cols, nnz, m, n, l, keys.get(), err.get());
        check_launch("k_col_row_keys");
        if (l == 1)
            raise_err(read_scalar(err.get(), st));
        const int end_bit = 32 + bit_length((uint64_t)(n - 1) >> l);
        size_t b1 = sort_bytes;
        ABHSF_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(), b1, keys.get(), sorted.get(), nnz, 0, end_bit, st));
        k_block_heads_all<<<grid_for(nnz), kThreads, 0, st>>>(sorted.get(), nnz, heads.get());
        check_launch("k_block_heads_all");
        for (int k = 1; k <= 8; ++k) {
            const int p = (k - 1) * 8 + (l - 1);
            const int64_t hl = (int64_t(1) << k) * (int64_t(1) << l) + 1;
            k_head_bit<<<grid_for(nnz), kThreads, 0, st>>>(heads.get(), nnz, k - 1, flag.get());
            check_launch("k_head_bit");
            size_t b2 = sel_bytes;
            ABHSF_CUDA(cub::DeviceSelect::Flagged(tmp.get(), b2, iota.get(), flag.get(), starts.get(), nsel.get(), nnz,
                                                  st));
            const int64_t B = read_scalar(nsel.get(), st);
            count[p] = B;
            if (hl <= 8192)
                k_len_hist_shared<<<grid_for(B), kThreads, hl * sizeof(unsigned int), st>>>(
                    B, starts.get(), nnz, dh.get() + off[p], (int)hl, err.get());
            else
                k_len_hist_global<<<grid_for(B), kThreads, 0, st>>>(B, starts.get(), nnz, dh.get() + off[p], hl,
                                                                     err.get());
            check_launch("k_len_hist");
        }
    }
    raise_err(read_scalar(err.get(), st));
    ABHSF_CUDA(cudaMemcpyAsync(hist, dh.get(), ABHSF_BSTATS_ALL_LEN * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    if (blocks)
        std::copy(count.begin(), count.end(), blocks);
}

void block_histogram_noalloc(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, int r,
                             int s, cudaStream_t st, uint64_t* hist, int64_t hist_len, int64_t* blocks)
{
    const int k = log2_exact(r), l = log2_exact(s);
    if (k < 1 || k > 8 || l < 1 || l > 8)
        fail(ABHSF_ERROR_INVALID_VALUE, "r and s must be powers of two in 2..256");
    if (m <= 0 || n <= 0 || nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
    if (nnz > ABHSF_NOALLOC_MAX_NNZ)
        fail(ABHSF_ERROR_INVALID_VALUE, "nnz exceeds ABHSF_NOALLOC_MAX_NNZ, the no-allocation limit");
    if (!hist || hist_len < (int64_t)r * s + 1)
        fail(ABHSF_ERROR_INVALID_VALUE, "hist must hold r*s + 1 counters");
    if (((uint64_t)(m - 1) >> k) >= (uint64_t(1) << 32) || ((uint64_t)(n - 1) >> l) >= (uint64_t(1) << 32))
        fail(ABHSF_ERROR_UNSUPPORTED, "block row or column index beyond 32 bits");
    if (nnz > 0 && (!rows || !cols))
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL device pointers");
    unsigned char* base = noalloc_scratch();  // before any early return: the set-up is per device
    std::fill(hist, hist + hist_len, 0);
    if (blocks)
        *blocks = 0;
    if (nnz == 0)
        return;
    const int64_t hl = (int64_t)r * s + 1;  // counters the device fills
    scratch_arena ar{base, kNoAllocScratchBytes};
    int* err = ar.take<int>(1);
    uint64_t* keys = ar.take<uint64_t>(nnz);
    uint64_t* keys_out = ar.take<uint64_t>(nnz);
    int64_t* head = ar.take<int64_t>(nnz);
    int64_t* run_of = ar.take<int64_t>(nnz);
    int64_t* start = ar.take<int64_t>(nnz + 1);
    unsigned long long* dh = ar.take<unsigned long long>(hl);
    const int end_bit = 32 + bit_length((uint64_t)(m - 1) >> k);
    size_t sort_bytes = 0, scan_bytes = 0;
    ABHSF_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, keys, keys_out, nnz, 0, end_bit, st));
    ABHSF_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, head, run_of, nnz, st));
    unsigned char* sort_tmp = ar.take<unsigned char>(sort_bytes);
    unsigned char* scan_tmp = ar.take<unsigned char>(scan_bytes);
    // the scratch keeps the previous call's contents: clear what must start at zero
    ABHSF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    ABHSF_CUDA(cudaMemsetAsync(dh, 0, hl * sizeof(unsigned long long), st));
    k_block_keys<<<grid_for(nnz), kThreads, 0, st>>>(rows, cols, nnz, m, n, k, l, keys, err);
    check_launch("k_block_keys");
    raise_err(read_scalar(err, st));
    ABHSF_CUDA(cub::DeviceRadixSort::SortKeys(sort_tmp, sort_bytes, keys, keys_out, nnz, 0, end_bit, st));
    k_heads<<<grid_for(nnz), kThreads, 0, st>>>(keys_out, nnz, 0, 0, head, err);
    check_launch("k_heads");
    ABHSF_CUDA(cub::DeviceScan::InclusiveSum(scan_tmp, scan_bytes, head, run_of, nnz, st));
    const int64_t B = read_scalar(run_of + nnz - 1, st);
    k_tile_starts<<<grid_for(nnz), kThreads, 0, st>>>(keys_out, run_of, nnz, 0, start, nullptr);
    check_launch("k_tile_starts");
    k_len_hist<<<grid_for(B), kThreads, 0, st>>>(B, start, dh, hl, err);
    check_launch("k_len_hist");
    ABHSF_CUDA(cudaMemcpyAsync(hist, dh, hl * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    raise_err(read_scalar(err, st));
    if (blocks)
        *blocks = B;
}

}  // namespace abhsf
