// spmv_f64.cu -- y += A x over the ABHSF format, FP64 values, sm_100a.
//
// Persistent warps take non-empty block rows from a work counter, a few at a
// time; one warp owns a block row (s rows of y) and walks its tiles in column
// order.  Per tile it dispatches on the scheme:
//
//  * bitmap / dense, s >= 32: lane l owns columns l, l+32, ... of the tile and
//    keeps those x values in registers.  Rows are taken kRG (8) at a time; for
//    each row a lane loads its value when its bit is set, at the row start plus
//    the popcount of the lower bits (so the set lanes read one contiguous run:
//    coalesced), and accumulates value * x.  The per-lane row partials are
//    reduced by a butterfly reduce-scatter that leaves row r's sum on lane r.  Replaces the bit-by-bit decode loops of
//    spmv/orig/88_bitmap.cpp:183-354 and 44_bitmap.cpp:187-396, and the dense
//    loop of spmv/orig/88.cpp:579-605.
//  * COO / CSR (and every scheme at s = 16): the tile's stored elements are
//    streamed 32 at a time with coalesced loads of values and local indices;
//    row indices come from the packed COO key or a binary search of the CSR
//    row_end array; products are summed per row by a segmented warp reduction
//    on the (sorted) row index.  Replaces spmv/orig/88.cpp:204-236.
//
// Row sums collect in a per-warp shared-memory copy of the block row's y
// segment and are added to y once per block row: no atomics, so the result is
// bitwise reproducible run to run.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

// Persistent warps: warp w first takes the w-th non-empty block row, then
// takes the next untaken one from a work counter, heaviest block rows first,
// so empty rows cost nothing and the warps finish close together.
constexpr int kWarps = 4;
#ifndef ABHSF_TREE_MINB
#define ABHSF_TREE_MINB 6
#endif
constexpr int kMinCtasPerSm = ABHSF_TREE_MINB;  // resident CTAs per SM the register budget must allow
#ifndef ABHSF_TREE_RG
#define ABHSF_TREE_RG 8
#endif
constexpr int kRG = ABHSF_TREE_RG;  // rows reduced together in bitmap / dense tiles
constexpr unsigned kFull = 0xffffffffu;

template <int S>
struct geom {
    static constexpr int CPL = S >= 32 ? S / 32 : 1;  // x values per lane
    static constexpr int RB = S >= 64 ? 64 : S;       // bitmap rows staged at once
    static constexpr int WPB = RB * CPL;              // u32 words of a staged bitmap block
    static constexpr int AUX = WPB > S / 2 ? (WPB > 8 ? WPB : 8) : (S / 2 > 8 ? S / 2 : 8);
};

template <int S>
struct warp_smem {
    alignas(16) uint32_t aux[geom<S>::AUX];  // a staged bitmap block, or CSR row_end
    double ys[S];                            // y segment of the block row
    double xs[S];                            // x segment of the current tile (element streams)
    int32_t rowstart[64];
};

__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t* p) { return __ldcs(p); }

// acc[0..RG-1] per lane -> lane l holds the sum over all lanes of acc[l % RG]
// (a reduce-scatter: RG-1 shuffles, then log2(32/RG) to finish).
template <int RG>
__device__ __forceinline__ double butterfly(double (&acc)[RG], int lane)
{
#pragma unroll
    for (int half = RG / 2; half >= 1; half >>= 1) {
        const bool upper = (lane & half) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const double send = upper ? acc[i] : acc[i + half];
            const double keep = upper ? acc[i + half] : acc[i];
            acc[i] = keep + __shfl_xor_sync(kFull, send, half);
        }
    }
    double r = acc[0];
#pragma unroll
    for (int d = RG; d < 32; d <<= 1)
        r += __shfl_xor_sync(kFull, r, d);
    return r;
}

// Bitmap tile, s >= 32.  bm32 = tile bitmap as little-endian u32 words: row
// r's columns 32j..32j+31 are word r * CPL + j.  Up to 64 rows of bitmap are
// staged in shared memory with one vector load per lane, their row starts
// found by one popcount scan; rows are then summed kRG at a time.
template <int S>
__device__ __forceinline__ void tile_bitmap(const uint32_t* __restrict__ bm32, const double* __restrict__ vals,
                                            const double (&xr)[geom<S>::CPL], warp_smem<S>& sm, int lane)
{
    constexpr int CPL = geom<S>::CPL;
    constexpr int RB = geom<S>::RB;
    constexpr int WPB = geom<S>::WPB;
    const uint32_t lt = (1u << lane) - 1u;
    int running = 0;
#pragma unroll 1
    for (int blk = 0; blk < S / RB; ++blk) {
        const uint4* src = reinterpret_cast<const uint4*>(bm32 + blk * WPB);
        uint4* dst = reinterpret_cast<uint4*>(sm.aux);
        for (int i = lane; i < WPB / 4; i += 32)
            dst[i] = __ldcs(src + i);
        __syncwarp();
        // rows lane and lane + 32 of the block
        int pc0 = 0, pc1 = 0;
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
        __syncwarp();
#pragma unroll 1
        for (int g = 0; g < RB / kRG; ++g) {
            double acc[kRG];
            if constexpr (CPL <= 2) {
                // all of the group's value loads are issued before any is used,
                // so kRG * CPL loads per lane are in flight at once
                double v[kRG][CPL];
#pragma unroll
                for (int i = 0; i < kRG; ++i) {
                    const int row = g * kRG + i;
                    const double* rv = vals + sm.rowstart[row];
                    int run = 0;
#pragma unroll
                    for (int j = 0; j < CPL; ++j) {
                        const uint32_t w = sm.aux[row * CPL + j];
                        v[i][j] = 0.0;
                        if ((w >> lane) & 1u)
                            v[i][j] = ld_stream(rv + run + __popc(w & lt));
                        run += __popc(w);
                    }
                }
#pragma unroll
                for (int i = 0; i < kRG; ++i) {
                    double a = 0.0;
#pragma unroll
                    for (int j = 0; j < CPL; ++j)
                        a = fma(v[i][j], xr[j], a);
                    acc[i] = a;
                }
            } else {  // wide tiles: loads and FMAs interleaved (registers)
#pragma unroll
                for (int i = 0; i < kRG; ++i) {
                    const int row = g * kRG + i;
                    const double* rv = vals + sm.rowstart[row];
                    int run = 0;
                    double a = 0.0;
#pragma unroll
                    for (int j = 0; j < CPL; ++j) {
                        const uint32_t w = sm.aux[row * CPL + j];
                        double v = 0.0;
                        if ((w >> lane) & 1u)
                            v = ld_stream(rv + run + __popc(w & lt));
                        a = fma(v, xr[j], a);
                        run += __popc(w);
                    }
                    acc[i] = a;
                }
            }
            const double r = butterfly<kRG>(acc, lane);
            if (lane < kRG)
                sm.ys[blk * RB + g * kRG + lane] += r;
        }
        __syncwarp();
    }
}

// Dense tile, s >= 32: all s*s values, row-major.
template <int S>
__device__ __forceinline__ void tile_dense(const double* __restrict__ vals, const double (&xr)[geom<S>::CPL],
                                           warp_smem<S>& sm, int lane)
{
    constexpr int CPL = geom<S>::CPL;
#pragma unroll 1
    for (int g = 0; g < S / kRG; ++g) {
        double acc[kRG];
        if constexpr (CPL <= 2) {
            double v[kRG][CPL];
#pragma unroll
            for (int i = 0; i < kRG; ++i)
#pragma unroll
                for (int j = 0; j < CPL; ++j)
                    v[i][j] = ld_stream(vals + (size_t)(g * kRG + i) * S + lane + 32 * j);
#pragma unroll
            for (int i = 0; i < kRG; ++i) {
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < CPL; ++j)
                    a = fma(v[i][j], xr[j], a);
                acc[i] = a;
            }
        } else {
#pragma unroll
            for (int i = 0; i < kRG; ++i) {
                const double* rv = vals + (size_t)(g * kRG + i) * S + lane;
                double a = 0.0;
#pragma unroll
                for (int j = 0; j < CPL; ++j)
                    a = fma(ld_stream(rv + 32 * j), xr[j], a);
                acc[i] = a;
            }
        }
        const double r = butterfly<kRG>(acc, lane);
        if (lane < kRG)
            sm.ys[g * kRG + lane] += r;
    }
    __syncwarp();
}

// s = 16 bitmap or dense: 32 bit positions (two rows) per step; lanes 0-15
// take row 2i, lanes 16-31 row 2i+1.
template <bool DENSE>
__device__ __forceinline__ void tile_16(const uint32_t* __restrict__ bm32, const double* __restrict__ vals, double xl,
                                        warp_smem<16>& sm, int lane)
{
    const uint32_t lt = (1u << lane) - 1u;
    int running = 0;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        double v = 0.0;
        if (DENSE) {
            v = ld_stream(vals + it * 32 + lane);
        } else {
            const uint32_t w = ld_stream_u32(bm32 + it);
            if ((w >> lane) & 1u)
                v = ld_stream(vals + running + __popc(w & lt));
            running += __popc(w);
        }
        double p = v * xl;
        p += __shfl_xor_sync(kFull, p, 8);
        p += __shfl_xor_sync(kFull, p, 4);
        p += __shfl_xor_sync(kFull, p, 2);
        p += __shfl_xor_sync(kFull, p, 1);
        if ((lane & 15) == 0)
            sm.ys[2 * it + (lane >> 4)] += p;
    }
    __syncwarp();
}

// COO / CSR tile: stream the z stored elements.
template <int S, bool CSR>
__device__ __forceinline__ void tile_stream(const uint8_t* __restrict__ pay, const double* __restrict__ vals, int z,
                                            warp_smem<S>& sm, int lane)
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
        int lr = S;  // sentinel for idle lanes: matches no real row
        double prod = 0.0;
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
            prod = ld_stream(vals + k) * sm.xs[lc];
        }
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double o = __shfl_down_sync(kFull, prod, d);
            const int olr = __shfl_down_sync(kFull, lr, d);
            if (lane + d < 32 && olr == lr)
                prod += o;
        }
        const int plr = __shfl_up_sync(kFull, lr, 1);
        if (k < z && (lane == 0 || plr != lr))
            sm.ys[lr] += prod;
        __syncwarp();
    }
}

struct tree_args {
    tiles_view A;
    const uint32_t* rows;  // non-empty block rows, ascending
    int64_t nrows;
    unsigned int* counter;  // next entry of rows to hand out (zeroed before each launch)
    const double* x;
    double* y;
};

template <int S>
__device__ __forceinline__ void block_row(const tree_args& P, int64_t I, warp_smem<S>& sm, int lane)
{
    constexpr int CPL = geom<S>::CPL;
    const tiles_view& A = P.A;
    const double* __restrict__ values = static_cast<const double*>(A.values);
    const double* __restrict__ x = P.x;
    const int64_t t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
    for (int r = lane; r < S; r += 32)
        sm.ys[r] = 0.0;
    __syncwarp();
    // the next tile's header is loaded while the current tile is summed
    uint32_t n_col = A.tile_col[t0], n_z = A.tile_nnz[t0];
    uint8_t n_sch = A.tile_scheme[t0];
    int64_t n_vo = A.tile_val_off[t0], n_io = A.tile_idx_off[t0];
#pragma unroll 1
    for (int64_t t = t0; t < t1; ++t) {
        const int64_t c0 = (int64_t)n_col * S;
        const int z = (int)n_z;
        const int sch = n_sch;
        const double* vals = values + n_vo;
        const uint8_t* pay = A.payload + n_io;
        if (t + 1 < t1) {
            n_col = A.tile_col[t + 1];
            n_z = A.tile_nnz[t + 1];
            n_sch = A.tile_scheme[t + 1];
            n_vo = A.tile_val_off[t + 1];
            n_io = A.tile_idx_off[t + 1];
        }
        double xr[CPL];
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
            const int64_t c = c0 + (S >= 32 ? 32 * j + lane : (lane & (S - 1)));
            xr[j] = c < A.n ? __ldg(x + c) : 0.0;
        }
        if (S >= 32 && sch == ABHSF_SCHEME_BITMAP) {
            if constexpr (S >= 32)
                tile_bitmap<S>(reinterpret_cast<const uint32_t*>(pay), vals, xr, sm, lane);
        } else if (S >= 32 && sch == ABHSF_SCHEME_DENSE) {
            if constexpr (S >= 32)
                tile_dense<S>(vals, xr, sm, lane);
        } else if (S == 16 && sch == ABHSF_SCHEME_BITMAP) {
            if constexpr (S == 16)
                tile_16<false>(reinterpret_cast<const uint32_t*>(pay), vals, xr[0], sm, lane);
        } else if (S == 16 && sch == ABHSF_SCHEME_DENSE) {
            if constexpr (S == 16)
                tile_16<true>(nullptr, vals, xr[0], sm, lane);
        } else {
#pragma unroll
            for (int j = 0; j < CPL; ++j)
                if (S >= 32 || lane < S)
                    sm.xs[S >= 32 ? 32 * j + lane : lane] = xr[j];
            __syncwarp();
            if (sch == ABHSF_SCHEME_CSR)
                tile_stream<S, true>(pay, vals, z, sm, lane);
            else
                tile_stream<S, false>(pay, vals, z, sm, lane);
        }
    }
    const int64_t r0 = I * S;
    for (int r = lane; r < S; r += 32)
        if (r0 + r < A.m)
            P.y[r0 + r] += sm.ys[r];
    __syncwarp();
}

template <int S>
__global__ void __launch_bounds__(kWarps * 32, kMinCtasPerSm) k_spmv_f64(tree_args P)
{
    __shared__ warp_smem<S> smem[kWarps];
    const int lane = threadIdx.x & 31;
    warp_smem<S>& sm = smem[threadIdx.x >> 5];
    const unsigned int nw = gridDim.x * kWarps;
    unsigned int k = blockIdx.x * kWarps + (threadIdx.x >> 5);
    while ((int64_t)k < P.nrows) {
        unsigned int next = 0;
        if (lane == 0)
            next = atomicAdd(P.counter, 1u) + nw;  // in flight during this block row
        block_row<S>(P, (int64_t)P.rows[k], sm, lane);
        k = __shfl_sync(kFull, next, 0);
    }
}

// Lists the non-empty block rows (the work items of k_spmv_f64).
__global__ void k_nonempty_flags(int64_t M, const int64_t* __restrict__ brow_ptr, int64_t* __restrict__ flag)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = brow_ptr[i + 1] > brow_ptr[i] ? 1 : 0;
}

__global__ void k_nonempty_scatter(int64_t M, const int64_t* __restrict__ brow_ptr, const int64_t* __restrict__ pos,
                                   uint32_t* __restrict__ rows)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x)
        if (brow_ptr[i + 1] > brow_ptr[i])
            rows[pos[i]] = (uint32_t)i;
}

// A block row's weight: the bytes an SpMV reads for it (values, index payload,
// and per tile its x segment and header).
__global__ void k_row_weight(int64_t nr, const uint32_t* __restrict__ rows, tiles_view A, int vsize, int s,
                             uint64_t* __restrict__ weight)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nr; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = rows[k], t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        weight[k] = (uint64_t)((A.tile_val_off[t1] - A.tile_val_off[t0]) * vsize +
                               (A.tile_idx_off[t1] - A.tile_idx_off[t0]) + (t1 - t0) * (8 * (int64_t)s + 32));
    }
}

template <int S>
int tree_ctas_per_sm()
{
    int nb = 0;
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spmv_f64<S>, kWarps * 32, 0));
    return std::max(nb, 1);
}

template <int S>
void launch(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (a.tree_nrows == 0)
        return;
    tree_args P{a.view(), a.tree_rows.get(), a.tree_nrows, a.tree_counter.get(), x, y};
    ABHSF_CUDA(cudaMemsetAsync(a.tree_counter.get(), 0, sizeof(unsigned int), st));
    // every resident warp takes part unless there are fewer block rows than warps
    const int64_t ctas = (a.tree_nrows + kWarps - 1) / kWarps;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ctas, (int64_t)a.tree_ctas));
    k_spmv_f64<S><<<grid, kWarps * 32, 0, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

}  // namespace

void prepare_tree(abhsf_matrix& a, cudaStream_t st)
{
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int per_sm = 1;
    switch (a.s) {
    case 16: per_sm = tree_ctas_per_sm<16>(); break;
    case 32: per_sm = tree_ctas_per_sm<32>(); break;
    case 64: per_sm = tree_ctas_per_sm<64>(); break;
    case 128: per_sm = tree_ctas_per_sm<128>(); break;
    case 256: per_sm = tree_ctas_per_sm<256>(); break;
    default: fail(ABHSF_ERROR_UNSUPPORTED, "block size without an SpMV kernel");
    }
    a.tree_ctas = nsm * per_sm;
    a.tree_counter.alloc(1);
    dbuf<int64_t> flag(a.M + 1), pos(a.M + 1);
    ABHSF_CUDA(cudaMemsetAsync(flag.get() + a.M, 0, sizeof(int64_t), st));
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((a.M + 255) / 256, 4096));
    k_nonempty_flags<<<g, 256, 0, st>>>(a.M, a.brow_ptr.get(), flag.get());
    ABHSF_CUDA(cudaGetLastError());
    exclusive_scan_i64(flag.get(), pos.get(), a.M + 1, st);
    int64_t nr = 0;
    ABHSF_CUDA(cudaMemcpyAsync(&nr, pos.get() + a.M, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    if (nr > int64_t(UINT32_MAX))
        fail(ABHSF_ERROR_UNSUPPORTED, "more than 2^32 non-empty block rows");
    a.tree_rows.alloc(nr);
    a.tree_nrows = nr;
    if (nr == 0)
        return;
    // Heaviest block rows first: the SpMV kernels hand out one block row at a
    // time in this order, so the last ones to start are the shortest and all
    // warps finish close together.  The sort is stable (ties keep ascending
    // row order), so the order is deterministic; it does not affect results,
    // since each block row is summed by one warp on its own.
    dbuf<uint32_t> asc(nr);
    dbuf<uint64_t> w(nr), w_sorted(nr);
    k_nonempty_scatter<<<g, 256, 0, st>>>(a.M, a.brow_ptr.get(), pos.get(), asc.get());
    ABHSF_CUDA(cudaGetLastError());
    const unsigned gw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nr + 255) / 256, 4096));
    k_row_weight<<<gw, 256, 0, st>>>(nr, asc.get(), a.view(), (int)value_size(a.value_type), (int)a.s, w.get());
    ABHSF_CUDA(cudaGetLastError());
    size_t tmp_bytes = 0;
    ABHSF_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_bytes, w.get(), w_sorted.get(), asc.get(),
                                                         a.tree_rows.get(), nr, 0, 64, st));
    dbuf<uint8_t> tmp(std::max<size_t>(tmp_bytes, 1));
    ABHSF_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tmp_bytes, w.get(), w_sorted.get(), asc.get(),
                                                         a.tree_rows.get(), nr, 0, 64, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

void spmv_f64(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (a.M == 0 || a.T == 0)
        return;
    switch (a.s) {
    case 16: launch<16>(a, x, y, st); break;
    case 32: launch<32>(a, x, y, st); break;
    case 64: launch<64>(a, x, y, st); break;
    case 128: launch<128>(a, x, y, st); break;
    case 256: launch<256>(a, x, y, st); break;
    default: fail(ABHSF_ERROR_UNSUPPORTED, "block size without an SpMV kernel");
    }
}

}  // namespace abhsf
