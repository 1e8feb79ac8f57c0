// spmv_stream.cu -- y += A x over hypersparse block rows through delta-coded
// row slices, in the reference's summation order, sm_100a.
//
// A block row whose tiles hold one or a few elements each costs the ring
// kernel (spmv_ring.cu) a descriptor, an x block and a tile walk per tile for
// a few multiply-adds.  Such block rows are re-encoded once, when the matrix
// is prepared, the way the reference's delta COO keeps a matrix
// (spmv/orig/delta.cpp:118-219, spmv/unified/spmv.cpp:815-1032: elements row
// by row, columns ascending, each column stored as the difference to the
// previous one), laid out for a warp:
//
// * The non-empty rows of a range of block rows (slice_segments) are ordered
//   by length (longest first, then ascending row) and dealt to slices of up
//   to 32 rows, one row per lane, so that a slice's rows end together.  A
//   slice stores its rows' elements column-major -- element k of lane l at
//   slot base + 32 k + l -- as one 32-bit word each, the column minus the
//   row's previous column (the first one absolute), and a copy of the value.
//   A lane record (offset << 8 | length - 1, the offset from the range's
//   first row) says which row a lane sums.
// * A row longer than kChainMin is a slice of its own (a chain): its elements
//   stored in order, each word the absolute column.
//
// A warp sums one slice at a time.  Sliced rows: every lane walks its row,
// kUnroll elements per step -- coalesced word and value loads (the active
// lanes are always a prefix, rows being ordered by length), the column by a
// running sum of the deltas, x gathered through L2 -- and adds each product
// onto its row's sum in column order, starting from y: the order of the
// reference CSR's spmv_naive (spmv/bottlenecks/spmv.cpp:58-64), so y is
// bitwise the same.  A chain (its own kernel, on a side stream forked from
// the caller's so that it runs beside the others): the lanes form 32
// products at a time, kChainAhead steps ahead, and every lane adds them in
// order.  Slices and chains are dealt to warps at
// preparation time, longest first.  No waits: nothing here can stall on
// another warp.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <queue>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {

namespace {

constexpr int kWarpsPerCta = 8;
constexpr int kCtasPerSm = 4;     // CTAs per SM in the grid (64 registers a thread)
constexpr int kUnroll = 4;        // elements a lane loads per step of a sliced row
constexpr int kChainWarps = 4;    // warps per CTA of the chain kernel
constexpr int kChainCtasPerSm = 4;  // register bound of the chain kernel (128 a thread)
constexpr int kChainGridPerSm = 1;  // chain CTAs per SM in the grid: the rest of the SM is left to the others
constexpr int kChainAhead = 8;    // chain: steps of 32 products in flight ahead of the sums
constexpr uint32_t kChain = 1u;   // dc_slice::geo: a one-row chain
constexpr int kMidShift = 20;     // dc_slice::geo: matrix index of a batch
constexpr int kLenBits = 8;       // lane record: row offset << kLenBits | (length - 1)
constexpr uint32_t kLenMask = (1u << kLenBits) - 1u;
constexpr int kChainMin = 256;   // rows longer than this are summed alone, as a chain
static_assert(kChainMin <= (1 << kLenBits), "a sliced row's length - 1 fits the lane record");
constexpr int kRingTilesMax = 256;  // block rows of more tiles go to the slices whatever their density

// What the kernel needs of one slice (32 bytes, in schedule order).
struct __align__(16) dc_slice {
    int64_t base;    // first slot of its words and values
    int64_t meta;    // sliced: first of its 32 lane records; chain: the row within the block row
    uint32_t brow;   // block row
    uint32_t steps;  // sliced: elements of its longest row; chain: the row's elements
    uint32_t lanes;  // rows (1 for a chain)
    uint32_t geo;    // kChain | matrix index << kMidShift
};
static_assert(sizeof(dc_slice) == 32, "dc_slice is 32 bytes");

template <int VT>
struct vt_of {
    using V = double;
    using T = double;
};
template <>
struct vt_of<ABHSF_VALUE_F32> {
    using V = float;
    using T = float;
};
template <>
struct vt_of<ABHSF_VALUE_BF16> {
    using V = uint16_t;
    using T = float;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float dmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double wide(double v) { return v; }
__device__ __forceinline__ float wide(float v) { return v; }
__device__ __forceinline__ float wide(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// Streamed once: loaded with the evict-first hint so that x stays in L2.
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ uint16_t ld_stream(const uint16_t* p)
{
    return __ldcs(reinterpret_cast<const unsigned short*>(p));
}

// One matrix of a launch.
struct dc_mat {
    const uint32_t* words;
    const void* vals;        // values in slot order
    const uint32_t* lane;    // lane records
    int64_t m;
};

struct dc_args {
    const dc_slice* slices;  // every warp's slices, warp after warp
    const int64_t* wbeg;     // [warps + 1]
    int warps;
    dc_mat A;                // the matrix (B = false)
    const void* x;
    void* y;
    int64_t ldx, ldy;        // x[i * ldx], y[i * ldy]
    const dc_mat* mats;      // a batch (B = true): matrix i's arrays, x and y
    const void* const* xs;
    void* const* ys;
};

// Eight consecutive products from shared memory (every lane the same
// address: a broadcast), in two or four 16-byte loads.
__device__ __forceinline__ void load8(const double* q, double (&t)[8])
{
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double2 u = reinterpret_cast<const double2*>(q)[k];
        t[2 * k] = u.x;
        t[2 * k + 1] = u.y;
    }
}
__device__ __forceinline__ void load8(const float* q, float (&t)[8])
{
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float4 u = reinterpret_cast<const float4*>(q)[k];
        t[4 * k] = u.x;
        t[4 * k + 1] = u.y;
        t[4 * k + 2] = u.z;
        t[4 * k + 3] = u.w;
    }
}

// Adds the first nv products of q (shared memory, 16-byte aligned) onto run
// in order.  The loads of the next eight are issued before the adds of the
// current eight, so that nothing but the adds themselves lies on the chain.
template <int N, typename T>
__device__ __forceinline__ T add_products(T run, const T* q, int nv)
{
    T t[2][8];
    load8(q, t[0]);
#pragma unroll
    for (int b = 0; b < N / 8; ++b) {
        if (8 * b >= nv)
            break;
        if (b + 1 < N / 8)
            load8(q + 8 * (b + 1), t[(b + 1) & 1]);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (8 * b + k < nv)
                run = dadd(run, t[b & 1][k]);
    }
    return run;
}

// All N products, no tests in the chain.
template <int N, typename T>
__device__ __forceinline__ T add_products_full(T run, const T* q)
{
    T t[2][8];
    load8(q, t[0]);
#pragma unroll
    for (int b = 0; b < N / 8; ++b) {
        if (b + 1 < N / 8)
            load8(q + 8 * (b + 1), t[(b + 1) & 1]);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            run = dadd(run, t[b & 1][k]);
    }
    return run;
}

// Sliced rows.  A warp sums its dealt slices one after another, each lane
// one row.  The next slice's descriptor and lane record, and the next step's
// words and values, are loaded while the current ones are summed, so that a
// step waits only on its x gathers.
template <int S, int VT, bool B>
__global__ void __launch_bounds__(32 * kWarpsPerCta, kCtasPerSm) k_spmv_slices(dc_args P)
{
    using T = typename vt_of<VT>::T;
    using V = typename vt_of<VT>::V;
    // f32 / bf16 values leave room in 64 registers for twice the steps in flight
    constexpr int U = VT == ABHSF_VALUE_F64 ? kUnroll : 2 * kUnroll;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kWarpsPerCta + warp;
    if (gw >= P.warps)
        return;
    int64_t si = P.wbeg[gw];
    const int64_t s1 = P.wbeg[gw + 1];
    if (si >= s1)
        return;
    auto mat = [&](const dc_slice& q) -> const dc_mat& { return B ? P.mats[q.geo >> kMidShift] : P.A; };
    auto record = [&](const dc_slice& q) -> uint32_t {
        return lane < (int)q.lanes ? mat(q).lane[q.meta + lane] : 0u;
    };
    dc_slice sl = P.slices[si];
    dc_slice nx = si + 1 < s1 ? P.slices[si + 1] : sl;
    uint32_t rec = record(sl);
#pragma unroll 1
    for (; si < s1; ++si) {
        const bool more = si + 1 < s1;
        const dc_slice nn = si + 2 < s1 ? P.slices[si + 2] : nx;
        const uint32_t rec_n = more ? record(nx) : 0u;
        const int mid = (int)(sl.geo >> kMidShift);
        const dc_mat& M = mat(sl);
        const T* X = static_cast<const T*>(B ? P.xs[mid] : P.x);
        T* Y = static_cast<T*>(B ? P.ys[mid] : P.y);
        const int64_t ldx = B ? 1 : P.ldx, ldy = B ? 1 : P.ldy;
        const uint32_t* W = M.words + sl.base + lane;
        const V* Vv = static_cast<const V*>(M.vals) + sl.base + lane;
        // one row per lane, element k of the lane's row at slot 32 k + lane
        const int len = lane < (int)sl.lanes ? (int)(rec & kLenMask) + 1 : 0;
        const int64_t row = (int64_t)sl.brow * S + (int64_t)(rec >> kLenBits);
        T acc = len ? Y[row * ldy] : T(0);
        uint32_t col = 0;
        // values stay in their stored type until their product: a widening
        // at the load would wait for the prefetch it belongs to
        uint32_t w[U];
        V v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            w[u] = u < len ? ld_stream(W + 32 * u) : 0u;
            v[u] = u < len ? ld_stream(Vv + 32 * u) : V(0);
        }
#pragma unroll 1
        for (int k0 = 0; k0 < (int)sl.steps; k0 += U) {
            uint32_t wn[U];
            V vn[U];
            T x[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {  // the next step's words and values
                const int k = k0 + U + u;
                wn[u] = k < len ? ld_stream(W + 32 * k) : 0u;
                vn[u] = k < len ? ld_stream(Vv + 32 * k) : V(0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                col += w[u];
                x[u] = k0 + u < len ? __ldg(X + (int64_t)col * ldx) : T(0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (k0 + u < len)
                    acc = dadd(acc, dmul(wide(v[u]), x[u]));
#pragma unroll
            for (int u = 0; u < U; ++u) {
                w[u] = wn[u];
                v[u] = vn[u];
            }
        }
        if (len)
            Y[row * ldy] = acc;
        sl = nx;
        nx = nn;
        rec = rec_n;
    }
}

// The chains: one warp per row, the row's elements in order (each word the
// absolute column).  Lane l forms the product of element 32 j + l of a group
// of kChainAhead x 32 and stores it in the warp's shared buffer; every lane
// then adds the group's products in order, read back by broadcast loads (a
// shuffle per product would cost more issue slots than the add it feeds).
// The values and gathered x of the next group are in flight meanwhile, so
// that the chain of adds -- the one thing that must run in sequence -- does
// not wait on memory.
template <int S, int VT, bool B>
__global__ void __launch_bounds__(32 * kChainWarps, kChainCtasPerSm) k_spmv_chains(dc_args P)
{
    using T = typename vt_of<VT>::T;
    using V = typename vt_of<VT>::V;
    constexpr int AH = kChainAhead, G = 32 * AH;
    __shared__ __align__(16) T sbuf[kChainWarps][G];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kChainWarps + warp;
    if (gw >= P.warps)
        return;
    T* buf = sbuf[warp];
    const int64_t s1 = P.wbeg[gw + 1];
#pragma unroll 1
    for (int64_t si = P.wbeg[gw]; si < s1; ++si) {
        const dc_slice sl = P.slices[si];
        const int mid = (int)(sl.geo >> kMidShift);
        const dc_mat& M = B ? P.mats[mid] : P.A;
        const T* X = static_cast<const T*>(B ? P.xs[mid] : P.x);
        T* Y = static_cast<T*>(B ? P.ys[mid] : P.y);
        const int64_t ldx = B ? 1 : P.ldx, ldy = B ? 1 : P.ldy;
        const uint32_t* W = M.words + sl.base;
        const V* Vv = static_cast<const V*>(M.vals) + sl.base;
        const int64_t row = (int64_t)sl.brow * S + sl.meta;
        const int len = (int)sl.steps;
        // slot j: the value and x of element 32 j + lane of the current
        // group; the word of the same element of the next group
        uint32_t wq[AH];
        V vq[AH];  // widened at the product (see k_spmv_slices)
        T xq[AH];
#pragma unroll
        for (int j = 0; j < AH; ++j) {
            const int e = 32 * j + lane;
            wq[j] = e < len ? ld_stream(W + e) : 0u;
        }
#pragma unroll
        for (int j = 0; j < AH; ++j) {
            const int e = 32 * j + lane;
            vq[j] = e < len ? ld_stream(Vv + e) : V(0);
            xq[j] = e < len ? __ldg(X + (int64_t)wq[j] * ldx) : T(0);
            wq[j] = e + G < len ? ld_stream(W + e + G) : 0u;
        }
        T run = Y[row * ldy];
        // whole groups: the refills clamped to the row (what they fetch past
        // its end is never used)
        int b0 = 0;
#pragma unroll 1
        for (; b0 + G <= len; b0 += G) {
            __syncwarp();  // the previous group's products are read
#pragma unroll
            for (int j = 0; j < AH; ++j) {
                buf[32 * j + lane] = dmul(wide(vq[j]), xq[j]);
                const int e = b0 + G + 32 * j + lane;  // the same element of the next group
                vq[j] = ld_stream(Vv + min(e, len - 1));
                xq[j] = __ldg(X + (int64_t)wq[j] * ldx);
                wq[j] = ld_stream(W + min(e + G, len - 1));
            }
            __syncwarp();
            run = add_products_full<G>(run, buf);
        }
        // the last, partial group
        const int rem = len - b0;
        if (rem > 0) {
            __syncwarp();
#pragma unroll
            for (int j = 0; j < AH; ++j)
                buf[32 * j + lane] = 32 * j + lane < rem ? dmul(wide(vq[j]), xq[j]) : T(0);
            __syncwarp();
            run = add_products<G>(run, buf, rem);
        }
        if (lane == 0)
            Y[row * ldy] = run;
    }
}

// Y += A X over K columns of X and Y (FP64, K = 2 .. 32), sliced rows.  Lane
// (g, h) = (lane / K, lane % K) keeps the sums of column h for rows g, g + G,
// ... of the slice (G = 32 / K): the group of K lanes reads one row of X, K
// contiguous values, per product.  Each step loads the slice's 32 words and
// values as the SpMV does (lane r: row r); lane r keeps row r's running
// column, and the groups take column and value by shuffles.  Every (row,
// column) sum adds its products in the row's column order from Y's value:
// column j of Y is bitwise the SpMV of column j of X.
template <int K>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_spmm_slices(dc_args P, int S)
{
    constexpr int G = 32 / K;
    constexpr int CH = K < 8 ? K : 8;  // rows whose gathers are in flight together
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / K, h = lane % K;
    const int gw = blockIdx.x * kWarpsPerCta + warp;
    if (gw >= P.warps)
        return;
    const double* X = static_cast<const double*>(P.x) + h;
    double* Y = static_cast<double*>(P.y) + h;
    const int64_t s1 = P.wbeg[gw + 1];
#pragma unroll 1
    for (int64_t si = P.wbeg[gw]; si < s1; ++si) {
        const dc_slice sl = P.slices[si];
        const uint32_t* W = P.A.words + sl.base;
        const double* Vv = static_cast<const double*>(P.A.vals) + sl.base;
        const uint32_t rec = lane < (int)sl.lanes ? P.A.lane[sl.meta + lane] : 0u;
        const int len = lane < (int)sl.lanes ? (int)(rec & kLenMask) + 1 : 0;
        const uint32_t off = rec >> kLenBits;  // lane r: row r's offset from the slice's first row
        const int64_t row0 = (int64_t)sl.brow * S;
        double acc[K];
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = g + G * i;
            const uint32_t oi = __shfl_sync(0xffffffffu, off, r);
            acc[i] = r < (int)sl.lanes ? Y[(row0 + oi) * P.ldy] : 0.0;
        }
        uint32_t col = 0;  // lane r: row r's column
#pragma unroll 1
        for (int k = 0; k < (int)sl.steps; ++k) {
            const bool on = k < len;
            const int64_t slot = (int64_t)k * 32 + lane;
            col += on ? ld_stream(W + slot) : 0u;
            const double v = on ? ld_stream(Vv + slot) : 0.0;
            const uint32_t act = __ballot_sync(0xffffffffu, on);
#pragma unroll
            for (int i0 = 0; i0 < K; i0 += CH) {
                double x[CH], vv[CH];
#pragma unroll
                for (int i = 0; i < CH; ++i) {
                    const int r = g + G * (i0 + i);
                    const uint32_t c = __shfl_sync(0xffffffffu, col, r);
                    vv[i] = __shfl_sync(0xffffffffu, v, r);
                    x[i] = (act >> r) & 1u ? __ldg(X + (int64_t)c * P.ldx) : 0.0;
                }
#pragma unroll
                for (int i = 0; i < CH; ++i)
                    if ((act >> (g + G * (i0 + i))) & 1u)
                        acc[i0 + i] = dadd(acc[i0 + i], dmul(vv[i], x[i]));
            }
        }
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const int r = g + G * i;
            const uint32_t oi = __shfl_sync(0xffffffffu, off, r);
            if (r < (int)sl.lanes)
                Y[(row0 + oi) * P.ldy] = acc[i];
        }
    }
}

// Y += A X over K columns, the chains: one row per warp, lane h (of the first
// K; the others repeat them and store nothing) keeps column h's sum and adds
// the row's products one after another, 32 elements' words and values loaded
// at a time (the next 32 in flight meanwhile) and taken by shuffles.
template <int K>
__global__ void __launch_bounds__(32 * kChainWarps, kChainCtasPerSm) k_spmm_chains(dc_args P, int S)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int h = lane % K;
    const int gw = blockIdx.x * kChainWarps + warp;
    if (gw >= P.warps)
        return;
    const double* X = static_cast<const double*>(P.x) + h;
    double* Y = static_cast<double*>(P.y) + h;
    const int64_t s1 = P.wbeg[gw + 1];
#pragma unroll 1
    for (int64_t si = P.wbeg[gw]; si < s1; ++si) {
        const dc_slice sl = P.slices[si];
        const uint32_t* W = P.A.words + sl.base;
        const double* Vv = static_cast<const double*>(P.A.vals) + sl.base;
        const int64_t row = (int64_t)sl.brow * S + sl.meta;
        const int len = (int)sl.steps;
        double acc = Y[row * P.ldy];
        uint32_t c = lane < len ? ld_stream(W + lane) : 0u;
        double v = lane < len ? ld_stream(Vv + lane) : 0.0;
#pragma unroll 1
        for (int e0 = 0; e0 < len; e0 += 32) {
            const int n = min(32, len - e0);
            const int en = e0 + 32 + lane;
            const uint32_t cn = en < len ? ld_stream(W + en) : 0u;
            const double vn = en < len ? ld_stream(Vv + en) : 0.0;
#pragma unroll
            for (int j0 = 0; j0 < 32; j0 += 8) {
                double x[8], vv[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const uint32_t cj = __shfl_sync(0xffffffffu, c, j0 + j);
                    vv[j] = __shfl_sync(0xffffffffu, v, j0 + j);
                    x[j] = j0 + j < n ? __ldg(X + (int64_t)cj * P.ldx) : 0.0;
                }
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (j0 + j < n)
                        acc = dadd(acc, dmul(vv[j], x[j]));
            }
            c = cn;
            v = vn;
        }
        if (lane < K)
            Y[row * P.ldy] = acc;
    }
}

// --------------------------------------------------------------- preparation

// Block rows the slices serve: no dense tile (its stored zeros would need
// words too), and no bitmap tile (the ring kernel's bitmap walk reads a bit
// per position where a slice reads a word per element), at most `avg`
// elements per tile on average, or more than kRingTilesMax tiles (one CTA of
// the ring kernel sums a whole block row, so a block row of very many tiles
// would keep one SM busy long after the rest).
// fbytes[k]: the block row's share of the format bytes (its brow_ptr entry,
// its tiles' headers, payloads and values).
__global__ void k_dc_classify(int64_t nr, const uint32_t* __restrict__ rows, tiles_view A, float avg, int vsize,
                              uint8_t* __restrict__ ok, int64_t* __restrict__ elems, int64_t* __restrict__ fbytes)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nr; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = rows[k], t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        bool sparse = true, bitmap = false;
        for (int64_t t = t0; t < t1 && sparse; ++t) {
            sparse = A.tile_scheme[t] != ABHSF_SCHEME_DENSE;
            bitmap = bitmap || A.tile_scheme[t] == ABHSF_SCHEME_BITMAP;
        }
        const int64_t e = A.tile_val_off[t1] - A.tile_val_off[t0];
        ok[k] = sparse && ((double)e <= (double)avg * (double)(t1 - t0) || t1 - t0 > kRingTilesMax || !bitmap) ? 1 : 0;
        elems[k] = e;
        fbytes[k] = 8 + (t1 - t0) * (4 + 4 + 1 + 8 + 8) + (A.tile_idx_off[t1] - A.tile_idx_off[t0]) + vsize * e;
    }
}

__device__ __forceinline__ int64_t brow_of_tile(const int64_t* brow_ptr, int64_t M, int64_t t)
{
    int64_t lo = 0, hi = M;  // largest I with brow_ptr[I] <= t
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) / 2;
        if (brow_ptr[mid] <= t)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Elements per row of the slice block rows (sidx[I] >= 0): cnt[sidx * s + lrow].
__global__ void k_dc_row_counts(int64_t T, tiles_view A, int s, int lg, const int32_t* __restrict__ sidx,
                                unsigned int* __restrict__ cnt)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = brow_of_tile(A.brow_ptr, A.M, t);
        const int k = sidx[I];
        if (k < 0)
            continue;
        unsigned int* c = cnt + (int64_t)k * s;
        const uint8_t* pay = A.payload + A.tile_idx_off[t];
        const int64_t z = A.tile_val_off[t + 1] - A.tile_val_off[t];
        if (A.tile_scheme[t] == ABHSF_SCHEME_CSR) {
            const uint16_t* re = reinterpret_cast<const uint16_t*>(pay);
            for (int r = 0; r < s; ++r) {
                const unsigned int d = re[r] - (r ? re[r - 1] : 0);
                if (d)
                    atomicAdd(c + r, d);
            }
        } else if (A.tile_scheme[t] == ABHSF_SCHEME_BITMAP) {
            const uint64_t* bm = reinterpret_cast<const uint64_t*>(pay);
            for (int i = 0; i < s * s / 64; ++i)
                for (uint64_t b = bm[i]; b; b &= b - 1)
                    atomicAdd(c + ((i * 64 + __ffsll((long long)b) - 1) >> lg), 1u);
        } else {
            const uint16_t* key = reinterpret_cast<const uint16_t*>(pay);
            for (int64_t e = 0; e < z; ++e)
                atomicAdd(c + (key[e] >> lg), 1u);
        }
    }
}

// Every element of the slice block rows at its place in element order (the
// block rows ascending, each in format order): its key (slice block row * s
// + row), its column and its value index.
__global__ void k_dc_expand(int64_t T, tiles_view A, int s, int lg, const int32_t* __restrict__ sidx,
                            const int64_t* __restrict__ ebase, uint32_t* __restrict__ key, uint32_t* __restrict__ pos,
                            uint32_t* __restrict__ colv, int64_t* __restrict__ vidx)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = brow_of_tile(A.brow_ptr, A.M, t);
        const int k = sidx[I];
        if (k < 0)
            continue;
        const int64_t v0 = A.tile_val_off[t], z = A.tile_val_off[t + 1] - v0;
        const int64_t e0 = ebase[k] + (v0 - A.tile_val_off[A.brow_ptr[I]]);
        const uint8_t* pay = A.payload + A.tile_idx_off[t];
        const uint64_t c0 = (uint64_t)A.tile_col[t] * (uint64_t)s;
        const uint16_t* w16 = reinterpret_cast<const uint16_t*>(pay);
        const uint64_t* bm = reinterpret_cast<const uint64_t*>(pay);
        const int sch = A.tile_scheme[t];
        int r = 0;          // CSR: the element's row
        int wi = 0;         // bitmap: the word holding the next set bit
        uint64_t bits = 0;  // bitmap: that word's bits not yet taken
        if (sch == ABHSF_SCHEME_BITMAP)
            bits = bm[0];
        for (int64_t e = 0; e < z; ++e) {
            int lr, lc;
            if (sch == ABHSF_SCHEME_CSR) {
                while (w16[r] <= e)
                    ++r;
                lr = r;
                lc = pay[2 * s + e];
            } else if (sch == ABHSF_SCHEME_BITMAP) {
                while (bits == 0)
                    bits = bm[++wi];
                const int bit = wi * 64 + __ffsll((long long)bits) - 1;
                bits &= bits - 1;
                lr = bit >> lg;
                lc = bit & (s - 1);
            } else {
                lr = w16[e] >> lg;
                lc = w16[e] & (s - 1);
            }
            const int64_t q = e0 + e;
            key[q] = (uint32_t)((int64_t)k * s + lr);
            pos[q] = (uint32_t)q;
            colv[q] = (uint32_t)(c0 + (uint64_t)lc);
            vidx[q] = v0 + e;
        }
    }
}

// Words and values at their slots, from the elements sorted row by row (each
// row's elements in column order): the q-th sorted element is element
// q - rstart[key] of its row.
template <typename V>
__global__ void k_dc_emit(int64_t E, const uint32_t* __restrict__ key, const uint32_t* __restrict__ pos,
                          const uint32_t* __restrict__ colv, const int64_t* __restrict__ vidx,
                          const int64_t* __restrict__ rstart, const int64_t* __restrict__ slot0,
                          const uint8_t* __restrict__ chain, const V* __restrict__ values,
                          uint32_t* __restrict__ words, V* __restrict__ vals)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < E; q += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t kr = key[q];
        const int64_t rank = q - rstart[kr];
        const uint32_t c = colv[pos[q]];
        const bool ch = chain[kr] != 0;
        const int64_t slot = slot0[kr] + (ch ? rank : 32 * rank);
        words[slot] = (ch || rank == 0) ? c : c - colv[pos[q - 1]];
        vals[slot] = values[vidx[pos[q]]];
    }
}

inline unsigned grid_of(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8192)); }

// Warps of a launch: the chains one CTA per SM; the sliced rows every
// resident CTA, less one per SM when chains run beside them (their CTA needs
// the registers), or one CTA per SM when they run beside the ring kernel
// (which leaves an SM the registers and warps of one such CTA).
int stream_grid_warps(int64_t items, bool chains, bool beside_chains, bool beside_ring)
{
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int ctas = beside_ring ? 1 : kCtasPerSm - (beside_chains ? 1 : 0);
    const int64_t full = chains ? (int64_t)nsm * kChainGridPerSm * kChainWarps : (int64_t)nsm * ctas * kWarpsPerCta;
    return (int)std::max<int64_t>(1, std::min<int64_t>(full, items));
}

// The side stream and the fork / join events of a handle with chains.
void make_side(cudaStream_t& side, cudaEvent_t& fork, cudaEvent_t& join)
{
    if (!side) {
        // the highest priority: the chains' CTAs are placed before the others
        // when both wait for SMs (the longest chain bounds the launch)
        int least = 0, greatest = 0;
        ABHSF_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        ABHSF_CUDA(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, greatest));
    }
    if (!fork)
        ABHSF_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    if (!join)
        ABHSF_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
}

// Time a slice takes, for the deal: a sliced one walks its longest row, a
// chain adds its products one after another.
inline uint64_t slice_weight(const abhsf_matrix::dc_slice_host& p)
{
    return p.chain ? 8ull * p.steps + 64u : 32ull * p.steps + 64u;
}

}  // namespace

// Longest-processing-time deal of the sliced rows (or the chains) of several
// matrices (block rows in [brow_lo, brow_hi) only) over the warps of one
// launch.
void deal_slices(const std::vector<const abhsf_matrix*>& mats, dbuf<uint8_t>& sched, dbuf<int64_t>& wbeg_d,
                 int& warps_out, cudaStream_t st, int64_t brow_lo, int64_t brow_hi, int kind, bool beside_ring)
{
    const bool chains = kind != kDealSliced;
    struct item {
        uint64_t w;
        uint32_t mid;
        uint32_t k;
    };
    std::vector<item> items;
    bool other = false;  // a slice of the other kind in the range
    for (size_t i = 0; i < mats.size(); ++i) {
        const auto& ps = mats[i]->dc_host;
        for (size_t k = 0; k < ps.size(); ++k)
            if ((int64_t)ps[k].brow >= brow_lo && (int64_t)ps[k].brow < brow_hi) {
                if (ps[k].chain != chains)
                    other = true;
                else
                    items.push_back(item{slice_weight(ps[k]), (uint32_t)i, (uint32_t)k});
            }
    }
    warps_out = 0;
    if (items.empty())
        return;
    const int W = stream_grid_warps((int64_t)items.size(), chains, !chains && other, beside_ring);
    std::stable_sort(items.begin(), items.end(), [](const item& a, const item& b) { return a.w > b.w; });
    using load_t = std::pair<uint64_t, int>;
    std::priority_queue<load_t, std::vector<load_t>, std::greater<load_t>> heap;
    for (int w = 0; w < W; ++w)
        heap.push({0, w});
    std::vector<std::vector<uint32_t>> per(W);
    for (uint32_t j = 0; j < items.size(); ++j) {
        load_t top = heap.top();
        heap.pop();
        per[top.second].push_back(j);
        heap.push({top.first + items[j].w, top.second});
    }
    std::vector<dc_slice> out;
    out.reserve(items.size());
    std::vector<int64_t> wbeg(W + 1, 0);
    for (int w = 0; w < W; ++w) {
        wbeg[w] = (int64_t)out.size();
        for (uint32_t j : per[w]) {  // heaviest first within the warp, too
            const auto& h = mats[items[j].mid]->dc_host[items[j].k];
            dc_slice p;
            p.base = h.base;
            p.meta = h.meta;
            p.brow = h.brow;
            p.steps = h.steps;
            p.lanes = h.lanes;
            p.geo = (h.chain ? kChain : 0u) | items[j].mid << kMidShift;
            out.push_back(p);
        }
    }
    wbeg[W] = (int64_t)out.size();
    sched.alloc(out.size() * sizeof(dc_slice));
    wbeg_d.alloc(W + 1);
    ABHSF_CUDA(cudaMemcpyAsync(sched.get(), out.data(), out.size() * sizeof(dc_slice), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemcpyAsync(wbeg_d.get(), wbeg.data(), (W + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    warps_out = W;
}

// Block-row boundaries of the ranges whose sliced rows may share a slice:
// the kHostChunks parts the host-memory SpMV copies and sums one after
// another (a part's slices must not reach into the next), each cut into
// pieces of at most 2^24 rows (the row offset a lane record holds).
std::vector<int64_t> slice_segments(int64_t M, int s)
{
    const int64_t piece = std::max<int64_t>(1, (int64_t(1) << (32 - kLenBits)) / s);
    std::vector<int64_t> b{0};
    for (int c = 1; c <= kHostChunks; ++c) {
        const int64_t e = M * c / kHostChunks;
        while (e - b.back() > piece)
            b.push_back(b.back() + piece);
        if (e > b.back())
            b.push_back(e);
    }
    return b;
}

// The slices of a prepared matrix: which non-empty block rows they serve
// (dc_tree_flag, by tree-row position), their words, values and lane
// records, and the matrix's own schedule.  avg <= 0 leaves every block row
// to the ring.
void prepare_stream(abhsf_matrix& a, float avg, cudaStream_t st)
{
    a.dc_host.clear();
    a.dc_tree_flag.assign((size_t)a.tree_nrows, 0);
    a.dc_warps = a.dc_cwarps = 0;
    a.dc_beside_ring = false;
    a.dc_elements = a.dc_rows = a.dc_slots = a.dc_lane_records = 0;
    const int s = a.s, lg = a.lg;
    if (avg <= 0.f || a.tree_nrows == 0 || a.sum_order != ABHSF_SUM_REFERENCE || (uint64_t)a.n > (uint64_t(1) << 32))
        return;
    const int64_t nr = a.tree_nrows;
    dbuf<uint8_t> ok(nr);
    dbuf<int64_t> elems(nr), fbytes(nr);
    const int vsize = (int)value_size(a.value_type);
    k_dc_classify<<<grid_of(nr), 256, 0, st>>>(nr, a.tree_rows.get(), a.view(), avg, vsize, ok.get(), elems.get(),
                                                fbytes.get());
    ABHSF_CUDA(cudaGetLastError());
    std::vector<uint8_t> okh(nr);
    std::vector<int64_t> eh(nr), fh(nr);
    std::vector<uint32_t> rows(nr);
    ABHSF_CUDA(cudaMemcpyAsync(okh.data(), ok.get(), nr, cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaMemcpyAsync(eh.data(), elems.get(), nr * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaMemcpyAsync(fh.data(), fbytes.get(), nr * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaMemcpyAsync(rows.data(), a.tree_rows.get(), nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    // slice block rows in ascending block-row order
    std::vector<std::pair<uint32_t, int64_t>> sel;  // (block row, tree position)
    for (int64_t k = 0; k < nr; ++k)
        if (okh[k])
            sel.push_back({rows[k], k});
    std::sort(sel.begin(), sel.end());
    const int64_t ns = (int64_t)sel.size();
    int64_t E = 0;
    for (auto& p : sel)
        E += eh[p.second];
    if (ns == 0 || E == 0 || E >= (int64_t(1) << 31) || ns * s >= (int64_t(1) << 32))
        return;
    std::vector<int32_t> sidx_h(a.M, -1);
    std::vector<int64_t> ebase(ns + 1, 0);
    for (int64_t k = 0; k < ns; ++k) {
        sidx_h[sel[k].first] = (int32_t)k;
        ebase[k + 1] = ebase[k] + eh[sel[k].second];
    }
    dbuf<int32_t> sidx(a.M);
    dbuf<unsigned int> cnt(ns * s);
    ABHSF_CUDA(cudaMemcpyAsync(sidx.get(), sidx_h.data(), a.M * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemsetAsync(cnt.get(), 0, ns * s * sizeof(unsigned int), st));
    k_dc_row_counts<<<grid_of(a.T), 256, 0, st>>>(a.T, a.view(), s, lg, sidx.get(), cnt.get());
    ABHSF_CUDA(cudaGetLastError());
    std::vector<unsigned int> ch(ns * s);
    ABHSF_CUDA(cudaMemcpyAsync(ch.data(), cnt.get(), ns * s * sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    // chains: per block row, its rows longer than kChainMin, longest first
    // (then ascending row).  Sliced rows: per segment (slice_segments), the
    // other non-empty rows of its block rows by length, longest first, then
    // ascending row, in groups of 32 -- rows of one length class share a
    // slice whatever their block row, so that its lanes run out together.
    std::vector<int64_t> rstart(ns * s + 1, 0), slot0(ns * s, 0);
    std::vector<uint8_t> chain(ns * s, 0);
    for (int64_t q = 0; q < ns * s; ++q)
        rstart[q + 1] = rstart[q] + ch[q];
    std::vector<uint32_t> lane_rec;
    auto& SL = a.dc_host;
    int64_t slots = 0;
    std::vector<int> order(s);
    std::vector<int64_t> rest;  // sliced rows of a segment: k s + r
    const std::vector<int64_t> seg = slice_segments(a.M, s);
    int64_t k = 0;
    for (size_t g = 0; g + 1 < seg.size(); ++g) {
        const int64_t b0 = seg[g], b1 = seg[g + 1];
        rest.clear();
        for (; k < ns && (int64_t)sel[k].first < b1; ++k) {
            const unsigned int* c = ch.data() + k * s;
            int live = 0;
            for (int r = 0; r < s; ++r)
                if (c[r])
                    order[live++] = r;
            std::stable_sort(order.begin(), order.begin() + live, [&](int p, int q) { return c[p] > c[q]; });
            int i = 0;
            for (; i < live && c[order[i]] > (unsigned int)kChainMin; ++i) {
                abhsf_matrix::dc_slice_host h;
                h.base = slots;
                h.meta = order[i];
                h.brow = sel[k].first;
                h.steps = c[order[i]];
                h.lanes = 1;
                h.chain = true;
                slot0[k * s + order[i]] = slots;
                chain[k * s + order[i]] = 1;
                slots += c[order[i]];
                SL.push_back(h);
            }
            std::sort(order.begin() + i, order.begin() + live);
            for (; i < live; ++i)
                rest.push_back(k * s + order[i]);
        }
        std::stable_sort(rest.begin(), rest.end(), [&](int64_t p, int64_t q) { return ch[p] > ch[q]; });
        for (size_t i = 0; i < rest.size(); i += 32) {
            const int n32 = (int)std::min<size_t>(32, rest.size() - i);
            abhsf_matrix::dc_slice_host h;
            h.base = slots;
            h.meta = (int64_t)lane_rec.size();
            h.brow = (uint32_t)b0;
            h.steps = ch[rest[i]];
            h.lanes = n32;
            h.chain = false;
            for (int l = 0; l < 32; ++l) {
                if (l < n32) {
                    const int64_t q = rest[i + l];
                    const int64_t off = (int64_t)sel[q / s].first * s + q % s - b0 * s;
                    lane_rec.push_back((uint32_t)off << kLenBits | (ch[q] - 1u));
                    slot0[q] = slots + l;
                } else {
                    lane_rec.push_back(0u);
                }
            }
            slots += 32 * (int64_t)h.steps;
            SL.push_back(h);
        }
    }
    // the elements row by row: sort by (block row, row), stable in format order
    dbuf<uint32_t> key(E), pos(E), key2(E), pos2(E), colv(E);
    dbuf<int64_t> vidx(E), ebase_d(ns + 1), rstart_d(ns * s + 1), slot0_d(ns * s);
    dbuf<uint8_t> chain_d(ns * s);
    ABHSF_CUDA(cudaMemcpyAsync(ebase_d.get(), ebase.data(), (ns + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemcpyAsync(rstart_d.get(), rstart.data(), (ns * s + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                               st));
    ABHSF_CUDA(cudaMemcpyAsync(slot0_d.get(), slot0.data(), ns * s * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemcpyAsync(chain_d.get(), chain.data(), ns * s, cudaMemcpyHostToDevice, st));
    k_dc_expand<<<grid_of(a.T), 256, 0, st>>>(a.T, a.view(), s, lg, sidx.get(), ebase_d.get(), key.get(), pos.get(),
                                              colv.get(), vidx.get());
    ABHSF_CUDA(cudaGetLastError());
    int bits = 1;
    while (bits < 32 && (int64_t(1) << bits) < ns * s)
        ++bits;
    size_t tb = 0;
    ABHSF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.get(), key2.get(), pos.get(), pos2.get(), (int)E, 0,
                                               bits, st));
    {
        dbuf<uint8_t> tmp(tb);
        ABHSF_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, key.get(), key2.get(), pos.get(), pos2.get(),
                                                   (int)E, 0, bits, st));
        ABHSF_CUDA(cudaStreamSynchronize(st));  // before tmp goes
    }
    const size_t vs = value_size(a.value_type);
    a.dc_words.alloc(slots);
    a.dc_vals.alloc(slots * vs);
    a.dc_lane.alloc(std::max<size_t>(lane_rec.size(), 1));
    ABHSF_CUDA(cudaMemsetAsync(a.dc_words.get(), 0, slots * sizeof(uint32_t), st));
    ABHSF_CUDA(cudaMemsetAsync(a.dc_vals.get(), 0, slots * vs, st));
    if (!lane_rec.empty())
        ABHSF_CUDA(cudaMemcpyAsync(a.dc_lane.get(), lane_rec.data(), lane_rec.size() * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, st));
    auto emit = [&](auto tag) {
        using V = decltype(tag);
        k_dc_emit<V><<<grid_of(E), 256, 0, st>>>(E, key2.get(), pos2.get(), colv.get(), vidx.get(), rstart_d.get(),
                                                  slot0_d.get(), chain_d.get(),
                                                  reinterpret_cast<const V*>(a.values.get()), a.dc_words.get(),
                                                  reinterpret_cast<V*>(a.dc_vals.get()));
    };
    if (vs == 8)
        emit(double{});
    else if (vs == 4)
        emit(float{});
    else
        emit(uint16_t{});
    ABHSF_CUDA(cudaGetLastError());
    ABHSF_CUDA(cudaStreamSynchronize(st));
    int64_t moved = 0;  // format bytes of the block rows the slices take over
    for (int64_t k = 0; k < ns; ++k) {
        a.dc_tree_flag[sel[k].second] = 1;
        moved += fh[sel[k].second];
    }
    int64_t live_lanes = 0;
    for (const auto& h : SL)
        live_lanes += h.chain ? 0 : h.lanes;
    a.stats.spmv_bytes = a.stats.format_bytes - moved + E * (int64_t)(sizeof(uint32_t) + vs) +
                         (int64_t)SL.size() * (int64_t)sizeof(dc_slice) + live_lanes * (int64_t)sizeof(uint32_t);
    a.dc_elements = E;
    a.dc_rows = ns;
    a.dc_slots = slots;
    a.dc_lane_records = (int64_t)lane_rec.size();
    deal_slices({&a}, a.dc_sched, a.dc_wbeg, a.dc_warps, st, 0, INT64_MAX, kDealSliced);
    deal_slices({&a}, a.dc_csched, a.dc_cwbeg, a.dc_cwarps, st, 0, INT64_MAX, kDealChains);
    if (a.dc_cwarps)
        make_side(a.dc_side, a.dc_fork, a.dc_join);
}

namespace {

// The chain kernel keeps its products in shared memory, the sliced-row
// kernels use none.  An SM set up for a kernel without shared memory (all of
// it L1) takes no CTA that needs some until it drains, so the chains would
// wait for the sliced rows instead of running beside them: every kernel here
// asks for the same split of L1 and shared memory.
constexpr int kCarveoutPct = 25;

// Sets the split for kernel Kern once per device (the attribute belongs to
// the device's context).
template <auto Kern>
void same_carveout()
{
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = uint64_t(1) << (dev & 63);
    if (done.load(std::memory_order_relaxed) & bit)
        return;
    ABHSF_CUDA(cudaFuncSetAttribute(Kern, cudaFuncAttributePreferredSharedMemoryCarveout, kCarveoutPct));
    done.fetch_or(bit, std::memory_order_relaxed);
}

template <int S, int VT, bool B>
void launch_kind(bool chains, const dc_args& P, cudaStream_t st)
{
    if (chains) {
        same_carveout<k_spmv_chains<S, VT, B>>();
        const unsigned grid = (unsigned)((P.warps + kChainWarps - 1) / kChainWarps);
        k_spmv_chains<S, VT, B><<<grid, 32 * kChainWarps, 0, st>>>(P);
    } else {
        same_carveout<k_spmv_slices<S, VT, B>>();
        const unsigned grid = (unsigned)((P.warps + kWarpsPerCta - 1) / kWarpsPerCta);
        k_spmv_slices<S, VT, B><<<grid, 32 * kWarpsPerCta, 0, st>>>(P);
    }
    ABHSF_CUDA(cudaGetLastError());
}

template <int VT, bool B>
void launch_vt(int s, bool chains, const dc_args& P, cudaStream_t st)
{
    switch (s) {
    case 16: launch_kind<16, VT, B>(chains, P, st); break;
    case 32: launch_kind<32, VT, B>(chains, P, st); break;
    case 64: launch_kind<64, VT, B>(chains, P, st); break;
    case 128: launch_kind<128, VT, B>(chains, P, st); break;
    default: launch_kind<256, VT, B>(chains, P, st); break;
    }
}

void launch(int s, int vt, bool batch, bool chains, const dc_args& P, cudaStream_t st)
{
    if (P.warps == 0)
        return;
    if (vt == ABHSF_VALUE_F64)
        batch ? launch_vt<ABHSF_VALUE_F64, true>(s, chains, P, st) : launch_vt<ABHSF_VALUE_F64, false>(s, chains, P, st);
    else if (vt == ABHSF_VALUE_F32)
        batch ? launch_vt<ABHSF_VALUE_F32, true>(s, chains, P, st) : launch_vt<ABHSF_VALUE_F32, false>(s, chains, P, st);
    else
        batch ? launch_vt<ABHSF_VALUE_BF16, true>(s, chains, P, st)
              : launch_vt<ABHSF_VALUE_BF16, false>(s, chains, P, st);
}

dc_mat mat_of(const abhsf_matrix& a) { return dc_mat{a.dc_words.get(), a.dc_vals.get(), a.dc_lane.get(), a.m}; }

dc_args args_of(const abhsf_matrix& a, const uint8_t* sched, const int64_t* wbeg, int warps, const void* x,
                int64_t ldx, void* y, int64_t ldy)
{
    dc_args P{};
    P.slices = reinterpret_cast<const dc_slice*>(sched);
    P.wbeg = wbeg;
    P.warps = warps;
    P.A = mat_of(a);
    P.x = x;
    P.y = y;
    P.ldx = ldx;
    P.ldy = ldy;
    return P;
}

dc_args batch_args(const abhsf_batch& b, const uint8_t* sched, const int64_t* wbeg, int warps,
                   const double* const* xs, double* const* ys)
{
    dc_args P{};
    P.slices = reinterpret_cast<const dc_slice*>(sched);
    P.wbeg = wbeg;
    P.warps = warps;
    P.mats = reinterpret_cast<const dc_mat*>(b.dc_table.get());
    P.xs = reinterpret_cast<const void* const*>(xs);
    P.ys = reinterpret_cast<void* const*>(ys);
    P.ldx = P.ldy = 1;
    return P;
}

template <int K>
void launch_mm_k(bool chains, int s, const dc_args& P, cudaStream_t st)
{
    same_carveout<k_spmm_chains<K>>();
    same_carveout<k_spmm_slices<K>>();
    if (chains)
        k_spmm_chains<K><<<(unsigned)((P.warps + kChainWarps - 1) / kChainWarps), 32 * kChainWarps, 0, st>>>(P, s);
    else
        k_spmm_slices<K><<<(unsigned)((P.warps + kWarpsPerCta - 1) / kWarpsPerCta), 32 * kWarpsPerCta, 0, st>>>(P, s);
    ABHSF_CUDA(cudaGetLastError());
}

// One pass over `cols` columns: the SpMV kernels for one, the K-column ones
// (FP64) otherwise.
void launch_cols(int cols, int s, int vt, bool chains, const dc_args& P, cudaStream_t st)
{
    if (P.warps == 0)
        return;
    switch (cols) {
    case 1: launch(s, vt, false, chains, P, st); break;
    case 2: launch_mm_k<2>(chains, s, P, st); break;
    case 4: launch_mm_k<4>(chains, s, P, st); break;
    case 8: launch_mm_k<8>(chains, s, P, st); break;
    case 16: launch_mm_k<16>(chains, s, P, st); break;
    case 32: launch_mm_k<32>(chains, s, P, st); break;
    default: fail(ABHSF_ERROR_UNSUPPORTED, "slices: a pass of 1, 2, 4, 8, 16 or 32 columns");
    }
}

// Chains on the side stream, after everything queued on st so far.
void fork_chains(cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, int s, int vt, bool batch,
                 const dc_args& P, int cols = 1)
{
    ABHSF_CUDA(cudaEventRecord(fork, st));
    ABHSF_CUDA(cudaStreamWaitEvent(side, fork, 0));
    if (batch)
        launch(s, vt, batch, true, P, side);
    else
        launch_cols(cols, s, vt, true, P, side);
    ABHSF_CUDA(cudaEventRecord(join, side));
}

}  // namespace

dc_plan plan_of(const abhsf_matrix& a)
{
    dc_plan p;
    p.sched = a.dc_sched.get();
    p.wbeg = a.dc_wbeg.get();
    p.warps = a.dc_warps;
    p.csched = a.dc_csched.get();
    p.cwbeg = a.dc_cwbeg.get();
    p.cwarps = a.dc_cwarps;
    return p;
}

// Whether this launch runs the sliced rows on the side stream, beside the ring
// kernel queued on st after slices_begin (single right-hand sides only).
inline bool sliced_beside(const abhsf_matrix& a, const dc_plan& p, int cols)
{
    return a.dc_beside_ring && cols == 1 && p.warps > 0 && p.sched == a.dc_sched.get();
}

void slices_begin(const abhsf_matrix& a, const dc_plan& p, const void* x, int64_t ldx, void* y, int64_t ldy,
                  cudaStream_t st, int cols)
{
    const bool beside = sliced_beside(a, p, cols);
    if (p.cwarps == 0 && !beside)
        return;
    if (!a.dc_side)
        fail(ABHSF_ERROR_CUDA, "matrix has chains but no side stream");
    ABHSF_CUDA(cudaEventRecord(a.dc_fork, st));
    ABHSF_CUDA(cudaStreamWaitEvent(a.dc_side, a.dc_fork, 0));
    if (beside)  // first, so that its CTAs take their place before the ring's fill the SMs
        launch(a.s, a.value_type, false, false, args_of(a, p.sched, p.wbeg, p.warps, x, ldx, y, ldy), a.dc_side);
    if (p.cwarps)
        launch_cols(cols, a.s, a.value_type, true, args_of(a, p.csched, p.cwbeg, p.cwarps, x, ldx, y, ldy),
                    a.dc_side);
    ABHSF_CUDA(cudaEventRecord(a.dc_join, a.dc_side));
}

void slices_end(const abhsf_matrix& a, const dc_plan& p, const void* x, int64_t ldx, void* y, int64_t ldy,
                cudaStream_t st, int cols)
{
    const bool beside = sliced_beside(a, p, cols);
    if (p.warps && !beside)
        launch_cols(cols, a.s, a.value_type, false, args_of(a, p.sched, p.wbeg, p.warps, x, ldx, y, ldy), st);
    if (p.cwarps || beside)
        ABHSF_CUDA(cudaStreamWaitEvent(st, a.dc_join, 0));
}

// The ring kernel serves some block rows: the sliced rows go beside it, dealt
// over one CTA an SM.
void slices_beside_ring(abhsf_matrix& a, cudaStream_t st)
{
    if (a.dc_warps == 0)
        return;
    deal_slices({&a}, a.dc_sched, a.dc_wbeg, a.dc_warps, st, 0, INT64_MAX, kDealSliced, true);
    make_side(a.dc_side, a.dc_fork, a.dc_join);
    a.dc_beside_ring = true;
}

// The slices of every matrix of a batch in one launch (and its chains in one more).
void prepare_batch_stream(abhsf_batch& b, cudaStream_t st)
{
    b.dc_warps = b.dc_cwarps = 0;
    std::vector<dc_mat> t;
    bool any = false;
    for (const abhsf_matrix* a : b.mats) {
        t.push_back(mat_of(*a));
        any = any || !a->dc_host.empty();
    }
    if (!any)
        return;
    b.dc_table.alloc(t.size() * sizeof(dc_mat));
    ABHSF_CUDA(cudaMemcpyAsync(b.dc_table.get(), t.data(), t.size() * sizeof(dc_mat), cudaMemcpyHostToDevice, st));
    deal_slices(b.mats, b.dc_sched, b.dc_wbeg, b.dc_warps, st, 0, INT64_MAX, kDealSliced);
    deal_slices(b.mats, b.dc_csched, b.dc_cwbeg, b.dc_cwarps, st, 0, INT64_MAX, kDealChains);
    if (b.dc_cwarps)
        make_side(b.dc_side, b.dc_fork, b.dc_join);
}

void batch_stream_begin(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st)
{
    if (b.dc_cwarps)
        fork_chains(st, b.dc_side, b.dc_fork, b.dc_join, b.s, ABHSF_VALUE_F64, true,
                    batch_args(b, b.dc_csched.get(), b.dc_cwbeg.get(), b.dc_cwarps, xs, ys));
}

void batch_stream_end(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st)
{
    if (b.dc_warps)
        launch(b.s, ABHSF_VALUE_F64, true, false, batch_args(b, b.dc_sched.get(), b.dc_wbeg.get(), b.dc_warps, xs, ys),
               st);
    if (b.dc_cwarps)
        ABHSF_CUDA(cudaStreamWaitEvent(st, b.dc_join, 0));
}

}  // namespace abhsf

extern "C" abhsf_status abhsf_slices_info(const abhsf_matrix* a, int64_t* slices, int64_t* slots,
                                          int64_t* lane_records, int64_t* elements, int64_t* block_rows)
{
    return abhsf::guarded([&] {
        if (!a)
            abhsf::fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        if (slices)
            *slices = (int64_t)a->dc_host.size();
        if (slots)
            *slots = a->dc_slots;
        if (lane_records)
            *lane_records = a->dc_lane_records;
        if (elements)
            *elements = a->dc_elements;
        if (block_rows)
            *block_rows = a->dc_rows;
    });
}

extern "C" abhsf_status abhsf_slices_export(const abhsf_matrix* a, int64_t* base, int64_t* meta, uint32_t* brow,
                                            uint32_t* steps, uint32_t* lanes, uint8_t* chain, uint32_t* lane_records,
                                            uint32_t* words, void* values)
{
    return abhsf::guarded([&] {
        if (!a)
            abhsf::fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        const auto& P = a->dc_host;
        for (size_t k = 0; k < P.size(); ++k) {
            if (base)
                base[k] = P[k].base;
            if (meta)
                meta[k] = P[k].meta;
            if (brow)
                brow[k] = P[k].brow;
            if (steps)
                steps[k] = P[k].steps;
            if (lanes)
                lanes[k] = P[k].lanes;
            if (chain)
                chain[k] = P[k].chain ? 1 : 0;
        }
        if (lane_records && a->dc_lane_records)
            ABHSF_CUDA(cudaMemcpy(lane_records, a->dc_lane.get(), a->dc_lane_records * sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost));
        if (a->dc_slots > 0) {
            if (words)
                ABHSF_CUDA(cudaMemcpy(words, a->dc_words.get(), a->dc_slots * sizeof(uint32_t), cudaMemcpyDeviceToHost));
            if (values)
                ABHSF_CUDA(cudaMemcpy(values, a->dc_vals.get(), a->dc_slots * abhsf::value_size(a->value_type),
                                      cudaMemcpyDeviceToHost));
        }
    });
}
