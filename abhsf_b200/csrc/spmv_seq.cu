// spmv_seq.cu -- y += A x over the ABHSF format in the reference's summation
// order, sm_100a, streaming through registers: FP64, and f32 / bf16 values
// widened to f32 with f32 x, y and sums (the same order in f32).
//
// The reference's CSR SpMV (csr_matrix::spmv_naive,
// spmv/bottlenecks/spmv.cpp:58-64) adds a row's products one at a time,
// columns ascending, onto y[row], each product rounded before its add.  Here
// persistent warps take non-empty block rows one at a time, heaviest first
// (the order prepare_tree lists them in), from a work counter; a warp keeps
// its block row's y segment in shared memory (starting from y0) and walks the
// tiles in column order.  For a group of rows of a bitmap or dense
// tile the lanes load the values with coalesced, predicated loads (lane l
// owns columns l, l+32, ...; a set bit's value sits at the row start plus the
// popcount of the lower bits), form value * x, and store the products
// compactly -- row-major, columns ascending -- in a small per-warp buffer.
// Then one lane per row adds its row's products, a contiguous run, one at a
// time onto the row's y entry (dadd_rn(acc, p), p = dmul_rn(v, x)): exactly
// the reference's order, so y is bitwise the reference CSR's.  The next
// group's loads are issued before these add chains so that they overlap.
// COO / CSR tiles stream 32 elements at a time: each lane forms one product,
// and the first lane of each row segment adds the segment in order.  A dense
// tile's stored zeros become -0.0, which leaves a sum bitwise unchanged (the
// reference's CSR has no such elements).
#include <algorithm>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

constexpr int kWarps = 4;
#ifndef ABHSF_SEQ_MINB
#define ABHSF_SEQ_MINB 6
#endif
constexpr int kMinCtasPerSm = ABHSF_SEQ_MINB;
constexpr unsigned kFull = 0xffffffffu;

template <int S>
struct sg {
    static constexpr int CPL = S >= 32 ? S / 32 : 1;       // columns per lane
    static constexpr int RB = S >= 64 ? 64 : S;            // bitmap rows staged at once
    static constexpr int WPB = RB * CPL;                   // u32 words of a staged bitmap block
#ifndef ABHSF_SEQ_VALS
#define ABHSF_SEQ_VALS 16
#endif
    // rows per load group: ABHSF_SEQ_VALS values per lane in flight
    // (s >= 128 keeps 16 so that four warps' buffers fit the static shared-memory limit)
    static constexpr int RG = S <= 16 ? 16 : S >= 128 ? 16 / CPL : (ABHSF_SEQ_VALS / CPL > 32 ? 32 : ABHSF_SEQ_VALS / CPL);
    static constexpr int BUF = RG * S;                     // product buffer (doubles)
    static constexpr int AUX = WPB > 8 ? WPB : 8;
};

// Stored value type V and arithmetic type T of a value type.
template <int VT>
struct seq_t {
    using V = double;
    using T = double;
};
template <>
struct seq_t<ABHSF_VALUE_F32> {
    using V = float;
    using T = float;
};
template <>
struct seq_t<ABHSF_VALUE_BF16> {
    using V = uint16_t;
    using T = float;
};

template <int S, typename T>
struct seq_smem {
    alignas(16) uint32_t aux[sg<S>::AUX];  // a staged bitmap block, or CSR row_end
    T ys[S];                               // the block row's y segment
    T xs[S];                               // x segment (element streams)
    int32_t rowstart[sg<S>::RB + 1];       // staged rows' first values (tile-relative), + end
    T buf[sg<S>::BUF];                     // a group's products, row-major
};

struct seq_args {
    tiles_view A;
    const uint32_t* rows;  // non-empty block rows, ascending
    int64_t nrows;
    unsigned int* counter;
    const void* x;  // T
    void* y;        // T
    // a batch: work item k is block row items[k].y of matrix items[k].x,
    // whose arrays are mats[i] and whose x and y are xs[i], ys[i]
    const tiles_view* mats;
    const uint2* items;
    const void* const* xs;
    void* const* ys;
};

__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ uint16_t ld_stream(const uint16_t* p)
{
    return __ldcs(reinterpret_cast<const unsigned short*>(p));
}
__device__ __forceinline__ double wide(double v) { return v; }
__device__ __forceinline__ float wide(float v) { return v; }
__device__ __forceinline__ float wide(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }
__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }

// acc + p[0] + p[1] + ... + p[n-1], one at a time, left to right.
template <typename T>
__device__ __forceinline__ T chain(T acc, const T* p, int n)
{
    int i = 0;
    for (; i + 8 <= n; i += 8) {
        T t[8];
#pragma unroll
        for (int v = 0; v < 8; ++v)
            t[v] = p[i + v];
#pragma unroll
        for (int v = 0; v < 8; ++v)
            acc = fadd(acc, t[v]);
    }
    for (; i < n; ++i)
        acc = fadd(acc, p[i]);
    return acc;
}

// Bitmap tile, s >= 32: row r's columns 32j..32j+31 are bitmap word r*CPL + j.
template <int S, int VT>
__device__ __forceinline__ void seq_bitmap(const uint32_t* __restrict__ bm32,
                                           const typename seq_t<VT>::V* __restrict__ vals,
                                           const typename seq_t<VT>::T (&xr)[sg<S>::CPL],
                                           seq_smem<S, typename seq_t<VT>::T>& sm, int lane)
{
    using T = typename seq_t<VT>::T;
    constexpr int CPL = sg<S>::CPL, RB = sg<S>::RB, WPB = sg<S>::WPB, RG = sg<S>::RG;
    constexpr int NG = RB / RG;
    const uint32_t lt = (1u << lane) - 1u;
    int running = 0;
#pragma unroll 1
    for (int blk = 0; blk < S / RB; ++blk) {
        const uint4* src = reinterpret_cast<const uint4*>(bm32 + blk * WPB);
        uint4* dst = reinterpret_cast<uint4*>(sm.aux);
        for (int i = lane; i < WPB / 4; i += 32)
            dst[i] = __ldcs(src + i);
        __syncwarp();
        int pc0 = 0, pc1 = 0;  // rows lane and lane + 32 of the block
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            if (lane < RB)
                pc0 += __popc(sm.aux[lane * CPL + j]);
            if (RB == 64)
                pc1 += __popc(sm.aux[(lane + 32) * CPL + j]);
        }
        int inc0 = pc0, inc1 = pc1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t0 = __shfl_up_sync(kFull, inc0, d);
            const int t1 = __shfl_up_sync(kFull, inc1, d);
            if (lane >= d) {
                inc0 += t0;
                inc1 += t1;
            }
        }
        const int tot0 = __shfl_sync(kFull, inc0, 31);
        const int tot1 = __shfl_sync(kFull, inc1, 31);
        if (lane < RB)
            sm.rowstart[lane] = running + inc0 - pc0;
        if (RB == 64)
            sm.rowstart[lane + 32] = running + tot0 + inc1 - pc1;
        running += tot0 + tot1;
        if (lane == 0)
            sm.rowstart[RB] = running;
        __syncwarp();

        // a group's value indices (tile-relative; -1: bit clear) and values
        int idx[RG][CPL];
        T v[RG][CPL];
        auto load_group = [&](int g) {
#pragma unroll
            for (int i = 0; i < RG; ++i) {
                const int row = g * RG + i;
                int run = sm.rowstart[row];
#pragma unroll
                for (int j = 0; j < CPL; ++j) {
                    const uint32_t w = sm.aux[row * CPL + j];
                    idx[i][j] = ((w >> lane) & 1u) ? run + __popc(w & lt) : -1;
                    v[i][j] = idx[i][j] >= 0 ? wide(ld_stream(vals + idx[i][j])) : T(0);
                    run += __popc(w);
                }
            }
        };
        load_group(0);
#pragma unroll 1
        for (int g = 0; g < NG; ++g) {
            const int base = sm.rowstart[g * RG];
#pragma unroll
            for (int i = 0; i < RG; ++i)
#pragma unroll
                for (int j = 0; j < CPL; ++j)
                    if (idx[i][j] >= 0)
                        sm.buf[idx[i][j] - base] = fmul(v[i][j], xr[j]);
            __syncwarp();
            if (g + 1 < NG)
                load_group(g + 1);  // in flight during the add chains below
            if (lane < RG) {
                const int row = g * RG + lane;
                const int lo = sm.rowstart[row] - base, hi = sm.rowstart[row + 1] - base;
                T& yr = sm.ys[blk * RB + row];
                yr = chain(yr, sm.buf + lo, hi - lo);
            }
            __syncwarp();
        }
    }
}

// Dense tile, s >= 32: all s*s values, row-major.
template <int S, int VT>
__device__ __forceinline__ void seq_dense(const typename seq_t<VT>::V* __restrict__ vals,
                                          const typename seq_t<VT>::T (&xr)[sg<S>::CPL], int64_t c0, int64_t n,
                                          seq_smem<S, typename seq_t<VT>::T>& sm, int lane)
{
    using T = typename seq_t<VT>::T;
    constexpr int CPL = sg<S>::CPL, RG = sg<S>::RG, NG = S / RG;
    T v[RG][CPL];
    auto load_group = [&](int g) {
#pragma unroll
        for (int i = 0; i < RG; ++i)
#pragma unroll
            for (int j = 0; j < CPL; ++j)
                v[i][j] = wide(ld_stream(vals + (size_t)(g * RG + i) * S + lane + 32 * j));
    };
    load_group(0);
#pragma unroll 1
    for (int g = 0; g < NG; ++g) {
#pragma unroll
        for (int i = 0; i < RG; ++i)
#pragma unroll
            for (int j = 0; j < CPL; ++j) {
                const int c = lane + 32 * j;
                // stored zeros become -0.0, a no-op in the sums
                sm.buf[i * S + c] = (v[i][j] != T(0) && c0 + c < n) ? fmul(v[i][j], xr[j]) : T(-0.0);
            }
        __syncwarp();
        if (g + 1 < NG)
            load_group(g + 1);
        if (lane < RG) {
            T& yr = sm.ys[g * RG + lane];
            yr = chain(yr, sm.buf + lane * S, S);
        }
        __syncwarp();
    }
}

// s = 16 bitmap or dense: the whole tile (256 positions) at once.
template <bool DENSE, int VT>
__device__ __forceinline__ void seq_16(const uint32_t* __restrict__ bm32, const typename seq_t<VT>::V* __restrict__ vals,
                                       typename seq_t<VT>::T xl, int64_t c0, int64_t n,
                                       seq_smem<16, typename seq_t<VT>::T>& sm, int lane)
{
    using T = typename seq_t<VT>::T;
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t w[8];
    T v[8];
    int running = 0;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        w[it] = DENSE ? 0xffffffffu : __ldcs(bm32 + it);
        v[it] = T(0);
        if ((w[it] >> lane) & 1u)
            v[it] = wide(ld_stream(vals + (DENSE ? it * 32 + lane : running + __popc(w[it] & lt))));
        running += __popc(w[it]);
    }
    running = 0;
    const bool col_ok = c0 + (lane & 15) < n;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        if ((w[it] >> lane) & 1u)
            sm.buf[running + __popc(w[it] & lt)] =
                DENSE && !(v[it] != T(0) && col_ok) ? T(-0.0) : fmul(v[it], xl);
        running += __popc(w[it]);
    }
    // row r's bits: half (r & 1) of word r >> 1
    int pc = 0;
    if (lane < 16) {
        uint32_t wr = 0;
#pragma unroll
        for (int it = 0; it < 8; ++it)
            if (it == (lane >> 1))
                wr = w[it];
        pc = __popc((wr >> ((lane & 1) * 16)) & 0xffffu);
    }
    int inc = pc;
#pragma unroll
    for (int d = 1; d < 16; d <<= 1) {
        const int t = __shfl_up_sync(kFull, inc, d);
        if (lane >= d)
            inc += t;
    }
    __syncwarp();
    if (lane < 16)
        sm.ys[lane] = chain(sm.ys[lane], sm.buf + inc - pc, pc);
    __syncwarp();
}

// COO / CSR tile: 32 stored elements at a time; the first lane of each row
// segment adds the segment's products onto the row, in element order.
template <int S, bool CSR, int VT>
__device__ __forceinline__ void seq_stream(const uint8_t* __restrict__ pay,
                                           const typename seq_t<VT>::V* __restrict__ vals, int z,
                                           seq_smem<S, typename seq_t<VT>::T>& sm, int lane)
{
    constexpr int LG = S == 16 ? 4 : S == 32 ? 5 : S == 64 ? 6 : S == 128 ? 7 : 8;
    const uint16_t* key16 = reinterpret_cast<const uint16_t*>(pay);
    const uint8_t* col8 = pay + 2 * S;
    uint16_t* row_end = reinterpret_cast<uint16_t*>(sm.aux);
    if (CSR) {
        for (int r = lane; r < S; r += 32)
            row_end[r] = __ldcs(key16 + r);
        __syncwarp();
    }
#pragma unroll 1
    for (int base = 0; base < z; base += 32) {
        const int k = base + lane;
        int lr = S;  // idle lanes: no row
        if (k < z) {
            int lc;
            if (CSR) {
                lc = __ldcs(col8 + k);
                int lo = 0, hi = S;  // first r with row_end[r] > k
#pragma unroll
                for (int step = 0; step <= LG; ++step) {
                    if (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (row_end[mid] > k)
                            hi = mid;
                        else
                            lo = mid + 1;
                    }
                }
                lr = lo;
            } else {
                const uint32_t key = __ldcs(key16 + k);
                lr = (int)(key >> LG);
                lc = (int)(key & (S - 1));
            }
            sm.buf[lane] = fmul(wide(ld_stream(vals + k)), sm.xs[lc]);
        }
        const int plr = __shfl_up_sync(kFull, lr, 1);
        const bool head = k < z && (lane == 0 || plr != lr);
        const unsigned heads = __ballot_sync(kFull, head);
        __syncwarp();
        if (head) {
            const unsigned later = heads & ~((2u << lane) - 1u);  // heads after this lane (lane 31: none)
            const int cnt = min(z - base, 32);
            const int end = later ? __ffs(later) - 1 : cnt;
            sm.ys[lr] = chain(sm.ys[lr], sm.buf + lane, end - lane);
        }
        __syncwarp();
    }
}

template <int S, int VT>
__device__ __forceinline__ void seq_block_row(const tiles_view& A, const void* x, void* y, int64_t I,
                                              seq_smem<S, typename seq_t<VT>::T>& sm, int lane)
{
    using T = typename seq_t<VT>::T;
    using V = typename seq_t<VT>::V;
    constexpr int CPL = sg<S>::CPL;
    const V* __restrict__ values = static_cast<const V*>(A.values);
    const T* __restrict__ X = static_cast<const T*>(x);
    T* __restrict__ Y = static_cast<T*>(y);
    const int64_t t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
    const int64_t r0 = I * S;
    for (int r = lane; r < S; r += 32)
        sm.ys[r] = (r0 + r < A.m) ? Y[r0 + r] : T(0);
    __syncwarp();
    uint32_t n_col = A.tile_col[t0], n_z = A.tile_nnz[t0];
    uint8_t n_sch = A.tile_scheme[t0];
    int64_t n_vo = A.tile_val_off[t0], n_io = A.tile_idx_off[t0];
#pragma unroll 1
    for (int64_t t = t0; t < t1; ++t) {
        const int64_t c0 = (int64_t)n_col * S;
        const int z = (int)n_z;
        const int sch = n_sch;
        const V* vals = values + n_vo;
        const uint8_t* pay = A.payload + n_io;
        if (t + 1 < t1) {
            n_col = A.tile_col[t + 1];
            n_z = A.tile_nnz[t + 1];
            n_sch = A.tile_scheme[t + 1];
            n_vo = A.tile_val_off[t + 1];
            n_io = A.tile_idx_off[t + 1];
        }
        T xr[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int64_t c = c0 + (S >= 32 ? 32 * j + lane : (lane & (S - 1)));
            xr[j] = c < A.n ? __ldg(X + c) : T(0);
        }
        if (S >= 32 && sch == ABHSF_SCHEME_BITMAP) {
            if constexpr (S >= 32)
                seq_bitmap<S, VT>(reinterpret_cast<const uint32_t*>(pay), vals, xr, sm, lane);
        } else if (S >= 32 && sch == ABHSF_SCHEME_DENSE) {
            if constexpr (S >= 32)
                seq_dense<S, VT>(vals, xr, c0, A.n, sm, lane);
        } else if (S == 16 && sch == ABHSF_SCHEME_BITMAP) {
            if constexpr (S == 16)
                seq_16<false, VT>(reinterpret_cast<const uint32_t*>(pay), vals, xr[0], c0, A.n, sm, lane);
        } else if (S == 16 && sch == ABHSF_SCHEME_DENSE) {
            if constexpr (S == 16)
                seq_16<true, VT>(nullptr, vals, xr[0], c0, A.n, sm, lane);
        } else {
#pragma unroll
            for (int j = 0; j < CPL; ++j)
                if (S >= 32 || lane < S)
                    sm.xs[S >= 32 ? 32 * j + lane : lane] = xr[j];
            __syncwarp();
            if (sch == ABHSF_SCHEME_CSR)
                seq_stream<S, true, VT>(pay, vals, z, sm, lane);
            else
                seq_stream<S, false, VT>(pay, vals, z, sm, lane);
        }
    }
    __syncwarp();
    for (int r = lane; r < S; r += 32)
        if (r0 + r < A.m)
            Y[r0 + r] = sm.ys[r];
    __syncwarp();
}

template <int S, int VT, bool B = false>
__global__ void __launch_bounds__(kWarps * 32, kMinCtasPerSm) k_spmv_seq(seq_args P)
{
    using T = typename seq_t<VT>::T;
    __shared__ seq_smem<S, T> smem[kWarps];
    const int lane = threadIdx.x & 31;
    seq_smem<S, T>& sm = smem[threadIdx.x >> 5];
    const unsigned int nw = gridDim.x * kWarps;
    unsigned int k = blockIdx.x * kWarps + (threadIdx.x >> 5);
    while ((int64_t)k < P.nrows) {
        unsigned int next = 0;
        if (lane == 0)
            next = atomicAdd(P.counter, 1u) + nw;  // in flight during this block row
        if constexpr (B) {
            const uint2 it = P.items[k];
            const tiles_view A = P.mats[it.x];
            seq_block_row<S, VT>(A, P.xs[it.x], P.ys[it.x], (int64_t)it.y, sm, lane);
        } else {
            seq_block_row<S, VT>(P.A, P.x, P.y, (int64_t)P.rows[k], sm, lane);
        }
        k = __shfl_sync(kFull, next, 0);
    }
}

template <int S, int VT>
void launch_seq(const abhsf_matrix& a, const uint32_t* rows, int64_t nrows, const void* x, void* y, cudaStream_t st)
{
    if (nrows == 0)
        return;
    int dev = 0, nsm = 0, per_sm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv_seq<S, VT>, kWarps * 32, 0));
    seq_args P{a.view(), rows, nrows, a.tree_counter.get(), x, y, nullptr, nullptr, nullptr, nullptr};
    ABHSF_CUDA(cudaMemsetAsync(a.tree_counter.get(), 0, sizeof(unsigned int), st));
    const int64_t ctas = (nrows + kWarps - 1) / kWarps;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ctas, (int64_t)nsm * std::max(per_sm, 1)));
    k_spmv_seq<S, VT><<<grid, kWarps * 32, 0, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

template <int VT>
void launch_seq_vt(const abhsf_matrix& a, const uint32_t* rows, int64_t nrows, const void* x, void* y,
                   cudaStream_t st)
{
    switch (a.s) {
    case 16: launch_seq<16, VT>(a, rows, nrows, x, y, st); break;
    case 32: launch_seq<32, VT>(a, rows, nrows, x, y, st); break;
    case 64: launch_seq<64, VT>(a, rows, nrows, x, y, st); break;
    case 128: launch_seq<128, VT>(a, rows, nrows, x, y, st); break;
    case 256: launch_seq<256, VT>(a, rows, nrows, x, y, st); break;
    default: fail(ABHSF_ERROR_UNSUPPORTED, "block size without an SpMV kernel");
    }
}

// The streaming kernel over the block rows it serves: all of them, or those
// the row slices leave (block sizes 16 / 128 / 256), the slices beside it.
void seq_any(const abhsf_matrix& a, const void* x, void* y, cudaStream_t st)
{
    if (a.M == 0 || a.T == 0)
        return;
    const bool slices = a.dc_rows > 0 && a.sum_order == ABHSF_SUM_REFERENCE && a.s != 32 && a.s != 64;
    std::unique_lock<std::mutex> lock(a.dc_mu, std::defer_lock);
    dc_plan p;
    const uint32_t* rows = a.tree_rows.get();
    int64_t nrows = a.tree_nrows;
    if (slices) {
        lock.lock();
        p = plan_of(a);
        slices_begin(a, p, x, 1, y, 1, st);
        rows = a.seq_rows.get();
        nrows = a.seq_nrows;
    }
    if (a.value_type == ABHSF_VALUE_F64)
        launch_seq_vt<ABHSF_VALUE_F64>(a, rows, nrows, x, y, st);
    else if (a.value_type == ABHSF_VALUE_F32)
        launch_seq_vt<ABHSF_VALUE_F32>(a, rows, nrows, x, y, st);
    else
        launch_seq_vt<ABHSF_VALUE_BF16>(a, rows, nrows, x, y, st);
    if (slices)
        slices_end(a, p, x, 1, y, 1, st);
}

}  // namespace

void spmv_f64_seq(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (a.value_type != ABHSF_VALUE_F64)
        fail(ABHSF_ERROR_INVALID_VALUE, "the f64 streaming SpMV needs a matrix stored as f64");
    seq_any(a, x, y, st);
}

// A batch of block sizes 16 / 128 / 256: matrix i's block rows outside the
// slices (heaviest first within a matrix) are interleaved by rank -- every
// matrix's heaviest, then every matrix's second, ... -- so that the work
// counter hands out the heavy block rows of all matrices first.
void prepare_batch_seq(abhsf_batch& b, cudaStream_t st)
{
    std::vector<tiles_view> views;
    std::vector<std::vector<uint32_t>> rows(b.mats.size());
    size_t longest = 0;
    for (size_t i = 0; i < b.mats.size(); ++i) {
        const abhsf_matrix& a = *b.mats[i];
        views.push_back(a.view());
        const bool sliced = a.dc_rows > 0;
        const int64_t nr = sliced ? a.seq_nrows : a.tree_nrows;
        rows[i].resize((size_t)nr);
        if (nr > 0 && a.T > 0)
            ABHSF_CUDA(cudaMemcpyAsync(rows[i].data(), sliced ? a.seq_rows.get() : a.tree_rows.get(),
                                       nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        else
            rows[i].clear();
        longest = std::max(longest, rows[i].size());
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));
    std::vector<uint2> items;
    for (size_t r = 0; r < longest; ++r)
        for (size_t i = 0; i < rows.size(); ++i)
            if (r < rows[i].size())
                items.push_back(make_uint2((unsigned)i, rows[i][r]));
    b.seq_mats.alloc(views.size() * sizeof(tiles_view));
    ABHSF_CUDA(cudaMemcpyAsync(b.seq_mats.get(), views.data(), views.size() * sizeof(tiles_view),
                               cudaMemcpyHostToDevice, st));
    b.seq_nitems = (int64_t)items.size();
    b.seq_items.alloc(std::max<size_t>(items.size(), 1));
    if (!items.empty())
        ABHSF_CUDA(cudaMemcpyAsync(b.seq_items.get(), items.data(), items.size() * sizeof(uint2),
                                   cudaMemcpyHostToDevice, st));
    b.seq_counter.alloc(1);
    b.dev_status.alloc(1);
    ABHSF_CUDA(cudaMemsetAsync(b.dev_status.get(), 0, sizeof(int), st));
    b.ctas = 0;
    prepare_batch_stream(b, st);
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

namespace {

template <int S>
void launch_batch_seq(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st)
{
    int dev = 0, nsm = 0, per_sm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    auto kern = k_spmv_seq<S, ABHSF_VALUE_F64, true>;
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarps * 32, 0));
    seq_args P{};
    P.nrows = b.seq_nitems;
    P.counter = b.seq_counter.get();
    P.mats = reinterpret_cast<const tiles_view*>(b.seq_mats.get());
    P.items = b.seq_items.get();
    P.xs = reinterpret_cast<const void* const*>(xs);
    P.ys = reinterpret_cast<void* const*>(ys);
    ABHSF_CUDA(cudaMemsetAsync(b.seq_counter.get(), 0, sizeof(unsigned int), st));
    const int64_t ctas = (b.seq_nitems + kWarps - 1) / kWarps;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ctas, (int64_t)nsm * std::max(per_sm, 1)));
    kern<<<grid, kWarps * 32, 0, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

}  // namespace

void batch_seq_spmv(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st)
{
    std::lock_guard<std::mutex> lock(b.dc_mu);
    batch_stream_begin(b, xs, ys, st);  // the chains, beside the rest
    if (b.seq_nitems > 0) {
        switch (b.s) {
        case 16: launch_batch_seq<16>(b, xs, ys, st); break;
        case 128: launch_batch_seq<128>(b, xs, ys, st); break;
        case 256: launch_batch_seq<256>(b, xs, ys, st); break;
        default: fail(ABHSF_ERROR_UNSUPPORTED, "the batched streaming kernel serves block sizes 16, 128, 256");
        }
    }
    batch_stream_end(b, xs, ys, st);
}

void spmv_f32_seq(const abhsf_matrix& a, const float* x, float* y, cudaStream_t st)
{
    if (a.value_type == ABHSF_VALUE_F64)
        fail(ABHSF_ERROR_INVALID_VALUE, "the f32 streaming SpMV needs a matrix stored as f32 or bf16");
    seq_any(a, x, y, st);
}

}  // namespace abhsf
