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
// * A block row's non-empty rows are ordered by length (longest first) and
//   dealt to slices of up to 32 rows, one row per lane.  A slice stores its
//   rows' elements column-major -- element k of lane l at slot base + 32 k + l
//   -- as one 32-bit word each, the column minus the row's previous column
//   (the first one absolute), and a copy of the value.  A lane record
//   (row << 24 | length) says which row a lane sums.
// * A row longer than kChainMin is a slice of its own (a chain): its elements
//   stored in order, each word the absolute column.
//
// A warp sums one slice at a time.  Sliced rows: every lane walks its row,
// kUnroll elements per step -- coalesced word and value loads (the active
// lanes are always a prefix, rows being ordered by length), the column by a
// running sum of the deltas, x gathered through L2 -- and adds each product
// onto its row's sum in column order, starting from y: the order of the
// reference CSR's spmv_naive (spmv/bottlenecks/spmv.cpp:58-64), so y is
// bitwise the same.  A chain: the lanes form 32 products at a time, kAhead
// steps ahead, and every lane adds them in order from shared memory.  Slices
// are dealt to warps at preparation time, longest first.  No waits: nothing
// here can stall on another warp.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {

namespace {

constexpr int kWarpsPerCta = 8;
constexpr int kCtasPerSm = 4;     // the grid: resident CTAs per SM (64 registers a thread)
constexpr int kUnroll = 4;        // elements a lane loads per step of a sliced row
constexpr int kAhead = 4;         // chain: steps of 32 products formed ahead of the sums
constexpr uint32_t kChain = 1u;   // dc_slice::geo: a one-row chain
constexpr int kMidShift = 20;     // dc_slice::geo: matrix index of a batch
constexpr uint32_t kLenMask = (1u << 24) - 1u;
constexpr int kChainMin = 256;   // rows longer than this are summed alone, as a chain

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

// Adds nv of the 32 products in p (shared memory, in order) onto run.
template <typename T>
__device__ __forceinline__ T add_in_order(T run, const T* p, int nv)
{
    if constexpr (sizeof(T) == 8) {
        const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const double2 t = q[k];
            if (2 * k < nv)
                run = dadd(run, t.x);
            if (2 * k + 1 < nv)
                run = dadd(run, t.y);
        }
    } else {
        const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float4 t = q[k];
            if (4 * k < nv)
                run = dadd(run, t.x);
            if (4 * k + 1 < nv)
                run = dadd(run, t.y);
            if (4 * k + 2 < nv)
                run = dadd(run, t.z);
            if (4 * k + 3 < nv)
                run = dadd(run, t.w);
        }
    }
    return run;
}

template <int S, int VT, bool B>
__global__ void __launch_bounds__(32 * kWarpsPerCta) k_spmv_slices(dc_args P)
{
    using T = typename vt_of<VT>::T;
    using V = typename vt_of<VT>::V;
    __shared__ __align__(16) T pbuf[kWarpsPerCta][32];  // a chain's products of one step
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gw = blockIdx.x * kWarpsPerCta + warp;
    if (gw >= P.warps)
        return;
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
        if (!(sl.geo & kChain)) {
            // one row per lane, element k of the lane's row at slot 32 k + lane
            const uint32_t rec = lane < (int)sl.lanes ? M.lane[sl.meta + lane] : 0u;
            const int len = (int)(rec & kLenMask);
            const int64_t row = (int64_t)sl.brow * S + (int64_t)(rec >> 24);
            T acc = len ? Y[row * ldy] : T(0);
            uint32_t col = 0;
#pragma unroll 1
            for (int k0 = 0; k0 < (int)sl.steps; k0 += kUnroll) {
                uint32_t w[kUnroll];
                T v[kUnroll], x[kUnroll];
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    const bool ok = k0 + u < len;
                    const int64_t slot = (int64_t)(k0 + u) * 32 + lane;
                    w[u] = ok ? ld_stream(W + slot) : 0u;
                    v[u] = ok ? wide(ld_stream(Vv + slot)) : T(0);
                }
#pragma unroll
                for (int u = 0; u < kUnroll; ++u) {
                    col += w[u];
                    x[u] = k0 + u < len ? __ldg(X + (int64_t)col * ldx) : T(0);
                }
#pragma unroll
                for (int u = 0; u < kUnroll; ++u)
                    if (k0 + u < len)
                        acc = dadd(acc, dmul(v[u], x[u]));
            }
            if (len)
                Y[row * ldy] = acc;
            continue;
        }
        // a chain: one row, its elements in order, each word the absolute column
        const int64_t row = (int64_t)sl.brow * S + sl.meta;
        const int len = (int)sl.steps;
        T* pb = pbuf[warp];
        // slot j: the value and x of step c + j; the word of step c + j + kAhead
        uint32_t wq[kAhead];
        T vq[kAhead], xq[kAhead];
#pragma unroll
        for (int j = 0; j < kAhead; ++j) {
            const int e = 32 * j + lane;
            wq[j] = e < len ? ld_stream(W + e) : 0u;
        }
#pragma unroll
        for (int j = 0; j < kAhead; ++j) {
            const int e = 32 * j + lane;
            vq[j] = e < len ? wide(ld_stream(Vv + e)) : T(0);
            xq[j] = e < len ? __ldg(X + (int64_t)wq[j] * ldx) : T(0);
            wq[j] = e + 32 * kAhead < len ? ld_stream(W + e + 32 * kAhead) : 0u;
        }
        T run = Y[row * ldy];
#pragma unroll 1
        for (int b0 = 0; b0 < len; b0 += 32 * kAhead) {
#pragma unroll
            for (int j = 0; j < kAhead; ++j) {
                const int base = b0 + 32 * j;
                if (base >= len)
                    break;
                pb[lane] = base + lane < len ? dmul(vq[j], xq[j]) : T(0);
                const int e = base + 32 * kAhead + lane;  // refill slot j: kAhead steps on
                vq[j] = e < len ? wide(ld_stream(Vv + e)) : T(0);
                xq[j] = e < len ? __ldg(X + (int64_t)wq[j] * ldx) : T(0);
                wq[j] = e + 32 * kAhead < len ? ld_stream(W + e + 32 * kAhead) : 0u;
                __syncwarp();
                run = add_in_order(run, pb, min(32, len - base));
                __syncwarp();
            }
        }
        if (lane == 0)
            Y[row * ldy] = run;
    }
}

// --------------------------------------------------------------- preparation

// Block rows the slices may serve: no dense tile (its stored zeros would
// need words too) and at most `avg` elements per tile on average.
__global__ void k_dc_classify(int64_t nr, const uint32_t* __restrict__ rows, tiles_view A, float avg,
                              uint8_t* __restrict__ ok, int64_t* __restrict__ elems)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nr; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = rows[k], t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        bool sparse = true;
        for (int64_t t = t0; t < t1 && sparse; ++t)
            sparse = A.tile_scheme[t] != ABHSF_SCHEME_DENSE;
        const int64_t e = A.tile_val_off[t1] - A.tile_val_off[t0];
        ok[k] = sparse && (double)e <= (double)avg * (double)(t1 - t0) ? 1 : 0;
        elems[k] = e;
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

int stream_grid_warps(int64_t items)
{
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t full = (int64_t)nsm * kCtasPerSm * kWarpsPerCta;
    return (int)std::max<int64_t>(1, std::min<int64_t>(full, items));
}

// Time a slice takes, for the deal: a sliced one walks its longest row, a
// chain adds its products one after another.
inline uint64_t slice_weight(const abhsf_matrix::dc_slice_host& p)
{
    return p.chain ? 8ull * p.steps + 64u : 32ull * p.steps + 64u;
}

}  // namespace

// Longest-processing-time deal of the slices of several matrices (block rows
// in [brow_lo, brow_hi) only) over the warps of one launch.
void deal_slices(const std::vector<const abhsf_matrix*>& mats, dbuf<uint8_t>& sched, dbuf<int64_t>& wbeg_d,
                 int& warps_out, cudaStream_t st, int64_t brow_lo, int64_t brow_hi)
{
    struct item {
        uint64_t w;
        uint32_t mid;
        uint32_t k;
    };
    std::vector<item> items;
    for (size_t i = 0; i < mats.size(); ++i) {
        const auto& ps = mats[i]->dc_host;
        for (size_t k = 0; k < ps.size(); ++k)
            if ((int64_t)ps[k].brow >= brow_lo && (int64_t)ps[k].brow < brow_hi)
                items.push_back(item{slice_weight(ps[k]), (uint32_t)i, (uint32_t)k});
    }
    warps_out = 0;
    if (items.empty())
        return;
    const int W = stream_grid_warps((int64_t)items.size());
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

// The slices of a prepared matrix: which non-empty block rows they serve
// (dc_tree_flag, by tree-row position), their words, values and lane
// records, and the matrix's own schedule.  avg <= 0 leaves every block row
// to the ring.
void prepare_stream(abhsf_matrix& a, float avg, cudaStream_t st)
{
    a.dc_host.clear();
    a.dc_tree_flag.assign((size_t)a.tree_nrows, 0);
    a.dc_warps = 0;
    a.dc_elements = a.dc_rows = a.dc_slots = a.dc_lane_records = 0;
    const int s = a.s, lg = a.lg;
    if (avg <= 0.f || a.tree_nrows == 0 || a.sum_order != ABHSF_SUM_REFERENCE || (uint64_t)a.n > (uint64_t(1) << 32))
        return;
    const int64_t nr = a.tree_nrows;
    dbuf<uint8_t> ok(nr);
    dbuf<int64_t> elems(nr);
    k_dc_classify<<<grid_of(nr), 256, 0, st>>>(nr, a.tree_rows.get(), a.view(), avg, ok.get(), elems.get());
    ABHSF_CUDA(cudaGetLastError());
    std::vector<uint8_t> okh(nr);
    std::vector<int64_t> eh(nr);
    std::vector<uint32_t> rows(nr);
    ABHSF_CUDA(cudaMemcpyAsync(okh.data(), ok.get(), nr, cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaMemcpyAsync(eh.data(), elems.get(), nr * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
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
    // slices: per block row, the non-empty rows by length (longest first,
    // then ascending row); a row longer than kChainMin alone, the rest in
    // groups of 32
    std::vector<int64_t> rstart(ns * s + 1, 0), slot0(ns * s, 0);
    std::vector<uint8_t> chain(ns * s, 0);
    for (int64_t q = 0; q < ns * s; ++q)
        rstart[q + 1] = rstart[q] + ch[q];
    std::vector<uint32_t> lane_rec;
    auto& SL = a.dc_host;
    int64_t slots = 0;
    std::vector<int> order(s);
    for (int64_t k = 0; k < ns; ++k) {
        const unsigned int* c = ch.data() + k * s;
        int live = 0;
        for (int r = 0; r < s; ++r)
            if (c[r])
                order[live++] = r;
        std::stable_sort(order.begin(), order.begin() + live, [&](int p, int q) { return c[p] > c[q]; });
        int i = 0;
        while (i < live && c[order[i]] > (unsigned int)kChainMin) {
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
            ++i;
        }
        for (; i < live; i += 32) {
            const int n32 = std::min(32, live - i);
            abhsf_matrix::dc_slice_host h;
            h.base = slots;
            h.meta = (int64_t)lane_rec.size();
            h.brow = sel[k].first;
            h.steps = c[order[i]];
            h.lanes = n32;
            h.chain = false;
            for (int l = 0; l < 32; ++l) {
                if (l < n32) {
                    const int r = order[i + l];
                    lane_rec.push_back((uint32_t)r << 24 | c[r]);
                    slot0[k * s + r] = slots + l;
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
    for (int64_t k = 0; k < ns; ++k)
        a.dc_tree_flag[sel[k].second] = 1;
    a.dc_elements = E;
    a.dc_rows = ns;
    a.dc_slots = slots;
    a.dc_lane_records = (int64_t)lane_rec.size();
    deal_slices({&a}, a.dc_sched, a.dc_wbeg, a.dc_warps, st, 0, INT64_MAX);
}

namespace {

template <int S, int VT, bool B>
void launch_slices_s(const dc_args& P, cudaStream_t st)
{
    const unsigned grid = (unsigned)((P.warps + kWarpsPerCta - 1) / kWarpsPerCta);
    k_spmv_slices<S, VT, B><<<grid, 32 * kWarpsPerCta, 0, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

template <int VT, bool B>
void launch_slices_vt(int s, const dc_args& P, cudaStream_t st)
{
    switch (s) {
    case 16: launch_slices_s<16, VT, B>(P, st); break;
    case 32: launch_slices_s<32, VT, B>(P, st); break;
    case 64: launch_slices_s<64, VT, B>(P, st); break;
    case 128: launch_slices_s<128, VT, B>(P, st); break;
    default: launch_slices_s<256, VT, B>(P, st); break;
    }
}

void launch_slices(int s, int vt, bool batch, const dc_args& P, cudaStream_t st)
{
    if (P.warps == 0)
        return;
    if (vt == ABHSF_VALUE_F64)
        batch ? launch_slices_vt<ABHSF_VALUE_F64, true>(s, P, st) : launch_slices_vt<ABHSF_VALUE_F64, false>(s, P, st);
    else if (vt == ABHSF_VALUE_F32)
        batch ? launch_slices_vt<ABHSF_VALUE_F32, true>(s, P, st) : launch_slices_vt<ABHSF_VALUE_F32, false>(s, P, st);
    else
        batch ? launch_slices_vt<ABHSF_VALUE_BF16, true>(s, P, st)
              : launch_slices_vt<ABHSF_VALUE_BF16, false>(s, P, st);
}

dc_mat mat_of(const abhsf_matrix& a) { return dc_mat{a.dc_words.get(), a.dc_vals.get(), a.dc_lane.get(), a.m}; }

}  // namespace

// y += A x over the slice block rows (x[i * ldx], y[i * ldy], elements of
// the matrix's compute type); sched / wbeg / warps default to the matrix's
// own schedule.  Returns false when the matrix has no slices.
bool spmv_stream(const abhsf_matrix& a, const void* x, int64_t ldx, void* y, int64_t ldy, cudaStream_t st,
                 const uint8_t* sched, const int64_t* wbeg, int warps)
{
    if (!sched) {
        sched = a.dc_sched.get();
        wbeg = a.dc_wbeg.get();
        warps = a.dc_warps;
    }
    if (warps == 0)
        return false;
    dc_args P{};
    P.slices = reinterpret_cast<const dc_slice*>(sched);
    P.wbeg = wbeg;
    P.warps = warps;
    P.A = mat_of(a);
    P.x = x;
    P.y = y;
    P.ldx = ldx;
    P.ldy = ldy;
    launch_slices(a.s, a.value_type, false, P, st);
    return true;
}

// The slices of every matrix of a batch in one launch.
void prepare_batch_stream(abhsf_batch& b, cudaStream_t st)
{
    b.dc_warps = 0;
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
    deal_slices(b.mats, b.dc_sched, b.dc_wbeg, b.dc_warps, st, 0, INT64_MAX);
}

void batch_stream(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st)
{
    if (b.dc_warps == 0)
        return;
    dc_args P{};
    P.slices = reinterpret_cast<const dc_slice*>(b.dc_sched.get());
    P.wbeg = b.dc_wbeg.get();
    P.warps = b.dc_warps;
    P.mats = reinterpret_cast<const dc_mat*>(b.dc_table.get());
    P.xs = reinterpret_cast<const void* const*>(xs);
    P.ys = reinterpret_cast<void* const*>(ys);
    P.ldx = P.ldy = 1;
    launch_slices(b.s, ABHSF_VALUE_F64, true, P, st);
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
