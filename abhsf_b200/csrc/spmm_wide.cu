// spmm_wide.cu -- Y += A X with 16 or 32 right-hand sides a pass over A,
// FP64, in the reference's summation order (every column bitwise its SpMV):
// the host side for every block size it serves (16, 32, 64), and the kernel
// of block size 16.  Block sizes 32 and 64 run k_spmm_staged (spmv_ring.cu),
// a row a lane with the ring's per-scheme sums; measured on the tiled
// mixture (4M rows, 59.8M elements), block size 64: 32 columns 1.06 ms and
// 16 columns 0.76 ms, against 1.99 and 0.98 ms for the ring's passes of 8.
//
// At block size 16 a warp's 32 lanes hold only 16 rows, so here the lanes
// are the columns: lane h keeps column h of the rows its warp owns, every
// element of a row is applied by the whole warp in the row's column order
// (the element's value and column are the same for all lanes, so the control
// flow is uniform), and X's block for a tile is staged in shared memory once
// for all rows.
//
// A CTA of 4 warps takes the block rows dealt to it (the non-empty block rows
// outside the slices, heaviest first, dealt round robin) tile by tile, two
// stages deep: while the warps sum tile t, cp.async brings tile t + 1's X
// block (S rows of K values), payload and values (spmm_stage.cuh).  Warp w
// owns rows w, w + 4, ..., whose sums stay in registers from the block row's
// first tile to its last.  Rows in the slices go through the slice SpMM
// kernels (spmv_stream.cu).  No wait in this file spins: the stages are
// guarded by cp.async.wait_group and __syncthreads.
//
// Reference summation order: spmv/bottlenecks/spmv.cpp:58-64 (csr spmv_naive,
// per row, columns ascending, y = y + v x); the per-scheme tile layouts are
// those the builder writes (payload of COO keys, CSR row ends + columns,
// bitmap rows; dense values row-major), spmv/orig/88.cpp:43-141.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "internal.cuh"
#include "spmm_stage.cuh"

namespace abhsf {
namespace {

constexpr int kWideWarps = 4;
constexpr int kWideThreads = 32 * kWideWarps;

// Resident CTAs an SM the register bound is set for (the shared memory
// decides in the end).
template <int S>
constexpr int wide_min_ctas()
{
    return S >= 64 ? 2 : 4;
}

using stage::x_block_bytes;

// Marks of a COO tile's row runs: each warp's rows' first and end element.
template <int S>
constexpr int mark_bytes()
{
    return kWideWarps * 2 * (S / kWideWarps) * 2;
}

struct wide_args {
    tiles_view A;
    const uint32_t* rows;  // block rows, heaviest first
    int64_t nrows;
    const double* X;  // row-major, X(i, j) at X[i * ldx + j]
    double* Y;
    int64_t ldx, ldy;
    int stage_bytes;  // X block + payload and values of the largest tile, 16-byte multiple
};

__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }

// Bits of row r of a bitmap tile (row-major bits, column c at bit c).
template <int S>
__device__ __forceinline__ uint64_t row_bits(const uint8_t* pay, int r)
{
    if constexpr (S == 64)
        return reinterpret_cast<const uint64_t*>(pay)[r];
    else if constexpr (S == 32)
        return reinterpret_cast<const uint32_t*>(pay)[r];
    else
        return reinterpret_cast<const uint16_t*>(pay)[r];
}


// Row r of a staged tile onto a (column h of the lanes): its elements in
// column order, each as a = a + v x.  vs: the tile's values; xs: X's block.
template <int S, int K>
__device__ __forceinline__ double row_bitmap(double a, uint64_t bits, int q, const double* vs, const double* xs,
                                             int h)
{
    const int cnt = __popcll(bits);
#pragma unroll 4
    for (int e = 0; e < cnt; ++e) {
        const int c = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        a = fadd(a, fmul(vs[q + e], xs[c * K + h]));
    }
    return a;
}

template <int S, int K>
__device__ __forceinline__ double row_dense(double a, const double* vr, const double* xs, int h)
{
#pragma unroll 8
    for (int c = 0; c < S; ++c) {
        const double v = vr[c];
        if (v != 0.0)  // stored zeros and the padding past n, as the SpMV kernels skip them
            a = fadd(a, fmul(v, xs[c * K + h]));
    }
    return a;
}

// CSR (columns as bytes) and COO (keys row << lg | column): elements lo .. hi - 1.
template <int S, int K, bool CSR>
__device__ __forceinline__ double row_run(double a, int lo, int hi, const uint8_t* pay, const double* vs,
                                          const double* xs, int h)
{
    const uint8_t* col8 = pay + 2 * S;
    const uint16_t* key16 = reinterpret_cast<const uint16_t*>(pay);
#pragma unroll 4
    for (int k = lo; k < hi; ++k) {
        const int c = CSR ? (int)col8[k] : (int)(key16[k] & (S - 1));
        a = fadd(a, fmul(vs[k], xs[c * K + h]));
    }
    return a;
}

// Adds a staged tile onto the warp's rows (w + 4 i).
template <int S, int K>
__device__ __forceinline__ void sum_tile(int sch, int nv, int pb, int lead, const uint8_t* stage,
                                         double (&acc)[S / kWideWarps], uint16_t* marks, int warp, int lane)
{
    constexpr int RPW = S / kWideWarps, LG = S == 16 ? 4 : S == 32 ? 5 : 6;
    const int h = lane & (K - 1);
    const double* xs = reinterpret_cast<const double*>(stage);
    const uint8_t* pay = stage + x_block_bytes<S, K>();
    const double* vs = reinterpret_cast<const double*>(pay + pb) + lead;
    if (sch == ABHSF_SCHEME_BITMAP) {
        // value index of each row's first element: set bits of the rows above
        // (lane l counts rows l and l + 32)
        const int c0 = lane < S ? __popcll(row_bits<S>(pay, lane)) : 0;
        const int c1 = S == 64 ? __popcll(row_bits<S>(pay, (lane + 32) & (S - 1))) : 0;
        int i0 = c0, i1 = c1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t0 = __shfl_up_sync(0xffffffffu, i0, d), t1 = __shfl_up_sync(0xffffffffu, i1, d);
            if (lane >= d) {
                i0 += t0;
                i1 += t1;
            }
        }
        const int lower = __shfl_sync(0xffffffffu, i0, 31);
        const int e0 = i0 - c0, e1 = lower + i1 - c1;  // first value of rows lane, lane + 32
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
            const int r = warp + kWideWarps * i;
            const int q = r < 32 ? __shfl_sync(0xffffffffu, e0, r & 31) : __shfl_sync(0xffffffffu, e1, r & 31);
            acc[i] = row_bitmap<S, K>(acc[i], row_bits<S>(pay, r), q, vs, xs, h);
        }
    } else if (sch == ABHSF_SCHEME_DENSE) {
#pragma unroll
        for (int i = 0; i < RPW; ++i)
            acc[i] = row_dense<S, K>(acc[i], vs + (warp + kWideWarps * i) * S, xs, h);
    } else if (sch == ABHSF_SCHEME_CSR) {
        const uint16_t* row_end = reinterpret_cast<const uint16_t*>(pay);
#pragma unroll
        for (int i = 0; i < RPW; ++i) {
            const int r = warp + kWideWarps * i;
            acc[i] = row_run<S, K, true>(acc[i], r > 0 ? row_end[r - 1] : 0, row_end[r], pay, vs, xs, h);
        }
    } else {
        // COO: the keys are sorted, so a row's elements are a run; mark where
        // this warp's rows start and end
        const uint16_t* key16 = reinterpret_cast<const uint16_t*>(pay);
        uint16_t* lo = marks + warp * 2 * RPW;
        uint16_t* hi = lo + RPW;
        for (int i = lane; i < RPW; i += 32) {
            lo[i] = 0;
            hi[i] = 0;
        }
        __syncwarp();
        for (int k = lane; k < nv; k += 32) {
            const int rk = key16[k] >> LG;
            if ((rk & (kWideWarps - 1)) == warp) {
                if (k == 0 || (key16[k - 1] >> LG) != rk)
                    lo[rk / kWideWarps] = (uint16_t)k;
                if (k + 1 == nv || (key16[k + 1] >> LG) != rk)
                    hi[rk / kWideWarps] = (uint16_t)(k + 1);
            }
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < RPW; ++i)
            acc[i] = row_run<S, K, false>(acc[i], lo[i], hi[i], pay, vs, xs, h);
    }
}

template <int S, int K>
__global__ void __launch_bounds__(kWideThreads, wide_min_ctas<S>()) k_spmm_wide(wide_args P)
{
    constexpr int RPW = S / kWideWarps;
    extern __shared__ __align__(16) uint8_t wide_smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, h = lane & (K - 1);
    const tiles_view& A = P.A;
    uint16_t* marks = reinterpret_cast<uint16_t*>(wide_smem + 2 * P.stage_bytes);
    int64_t k = blockIdx.x;
    if (k >= P.nrows)
        return;
    int64_t I = P.rows[k], t = A.brow_ptr[I], tend = A.brow_ptr[I + 1];
    stage::tile<S, K, kWideThreads>(A, P.X, P.ldx, t, wide_smem, tid);
    stage::commit();
    double acc[RPW];
    int cur = 0;
    bool first = true;
#pragma unroll 1
    for (;;) {
        // the next tile: the block row's next, or the first of the CTA's next block row
        int64_t kn = k, In = I, tn = t + 1, tne = tend;
        bool more = true;
        const bool next_row = tn >= tend;
        if (next_row) {
            kn = k + gridDim.x;
            more = kn < P.nrows;
            if (more) {
                In = P.rows[kn];
                tn = A.brow_ptr[In];
                tne = A.brow_ptr[In + 1];
            }
        }
        if (more)
            stage::tile<S, K, kWideThreads>(A, P.X, P.ldx, tn, wide_smem + (cur ^ 1) * P.stage_bytes, tid);
        stage::commit();  // (an empty group at the end keeps the wait below uniform)
        const int64_t r0 = I * S;
        if (first) {
#pragma unroll
            for (int i = 0; i < RPW; ++i) {
                const int64_t r = r0 + warp + kWideWarps * i;
                acc[i] = r < A.m ? P.Y[r * P.ldy + h] : 0.0;
            }
        }
        const int sch = A.tile_scheme[t];
        const int64_t vo = A.tile_val_off[t];
        const int nv = (int)(A.tile_val_off[t + 1] - vo);
        const int pb = (int)(A.tile_idx_off[t + 1] - A.tile_idx_off[t]);
        stage::wait_all_but_one();
        __syncthreads();  // tile t has landed
        sum_tile<S, K>(sch, nv, pb, (int)(vo & 1), wide_smem + cur * P.stage_bytes, acc, marks, warp, lane);
        if (t + 1 == tend && lane < K) {
#pragma unroll
            for (int i = 0; i < RPW; ++i) {
                const int64_t r = r0 + warp + kWideWarps * i;
                if (r < A.m)
                    P.Y[r * P.ldy + h] = acc[i];
            }
        }
        __syncthreads();  // everyone is done with this stage before it is refilled
        if (!more)
            break;
        first = next_row;
        k = kn;
        I = In;
        t = tn;
        tend = tne;
        cur ^= 1;
    }
}

// Largest payload + value bytes of one tile.
__global__ void k_tile_bytes_max(int64_t T, const int64_t* __restrict__ idx_off, const int64_t* __restrict__ val_off,
                                 unsigned long long* __restrict__ out)
{
    unsigned long long most = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x)
        most = max(most, (unsigned long long)((idx_off[t + 1] - idx_off[t]) + 8 * (val_off[t + 1] - val_off[t])));
    atomicMax(out, most);
}

template <int S, int K>
int wide_smem_bytes(const abhsf_matrix& a)
{
    return 2 * (x_block_bytes<S, K>() + (int)a.wide_cap) + mark_bytes<S>();
}

template <int S, int K>
void launch_wide(const abhsf_matrix& a, const uint32_t* rows, int64_t nrows, const double* X, int64_t ldx, double* Y,
                 int64_t ldy, cudaStream_t st)
{
    const int smem = wide_smem_bytes<S, K>(a);
    auto kern = k_spmm_wide<S, K>;
    ABHSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ABHSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
    int dev = 0, nsm = 0, per_sm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWideThreads, smem));
    if (per_sm < 1)
        fail(ABHSF_ERROR_UNSUPPORTED, "wide SpMM: the stages do not fit shared memory");
    const unsigned grid = (unsigned)std::min<int64_t>(nrows, (int64_t)nsm * per_sm);
    wide_args P{a.view(), rows, nrows, X, Y, ldx, ldy, x_block_bytes<S, K>() + (int)a.wide_cap};
    kern<<<grid, kWideThreads, smem, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

}  // namespace

void prepare_wide(abhsf_matrix& a, cudaStream_t st)
{
    a.wide_cap = 0;
    if (a.value_type != ABHSF_VALUE_F64 || a.sum_order != ABHSF_SUM_REFERENCE ||
        (a.s != 16 && a.s != 32 && a.s != 64) || a.T == 0 || a.tree_nrows == 0)
        return;
    dbuf<unsigned long long> most(1);
    ABHSF_CUDA(cudaMemsetAsync(most.get(), 0, sizeof(unsigned long long), st));
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((a.T + 255) / 256, 1024));
    k_tile_bytes_max<<<g, 256, 0, st>>>(a.T, a.tile_idx_off.get(), a.tile_val_off.get(), most.get());
    ABHSF_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    ABHSF_CUDA(cudaMemcpyAsync(&h, most.get(), sizeof(h), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    // the values start up to 8 bytes into their first granule and end on a whole one
    const int64_t cap = (int64_t)((h + 15) & ~15ull) + 16;
    const int64_t x32 = (int64_t)a.s * 32 * 8;
    // two stages and each warp's COO marks (at most 8 warps of 2 s marks of 2 bytes) in 227 KiB
    if (2 * (x32 + cap) + 8 * 2 * a.s * 2 > 232448)
        return;
    a.wide_cap = cap;
}

bool spmm_f64_wide(const abhsf_matrix& a, int k, const double* X, int64_t ldx, double* Y, int64_t ldy,
                   cudaStream_t st)
{
    if (a.wide_cap == 0 || k <= 0 || k % 16 != 0 || (ldx & 1) || (ldy & 1) ||
        ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 15))
        return false;
    const bool sliced = a.dc_rows > 0;
    const uint32_t* rows = sliced ? a.seq_rows.get() : a.tree_rows.get();
    const int64_t nrows = sliced ? a.seq_nrows : a.tree_nrows;
    std::lock_guard<std::mutex> lock(a.dc_mu);
    const dc_plan p = plan_of(a);
    for (int j = 0; j < k;) {
        const int cols = k - j >= 32 ? 32 : 16;
        if (nrows > 0 && (a.s == 32 || a.s == 64))
            spmm_staged(a, cols, rows, nrows, X + j, ldx, Y + j, ldy, st);
        else if (nrows > 0 && cols == 32)
            launch_wide<16, 32>(a, rows, nrows, X + j, ldx, Y + j, ldy, st);
        else if (nrows > 0)
            launch_wide<16, 16>(a, rows, nrows, X + j, ldx, Y + j, ldy, st);
        if (sliced) {
            slices_begin(a, p, X + j, ldx, Y + j, ldy, st, cols);
            slices_end(a, p, X + j, ldx, Y + j, ldy, st, cols);
        }
        j += cols;
    }
    return true;
}

}  // namespace abhsf
