// spmv_ring.cu -- y += A x over the ABHSF format in the reference's summation
// order, FP64, block sizes 32 and 64, sm_100a.
//
// The reference's CSR SpMV (csr_matrix::spmv_naive,
// spmv/bottlenecks/spmv.cpp:58-64) adds a row's products one at a time,
// columns ascending, onto y[row], each product rounded before its add.  This
// kernel keeps that order and so returns y bitwise equal to the reference's.
//
// One warp per CTA.  At build time the non-empty block rows are dealt to the
// warps (longest processing time first, by the bytes each block row moves)
// and every warp gets its tiles as a list of 32-byte descriptors, in block-row
// order.  The warp streams its tiles through a private ring in shared memory:
// for each tile, asynchronous copies (cp.async) bring the x segment, the index
// payload, the values and -- for the first tile of a block row -- the y
// segment into one ring slot, several tiles ahead of the one being summed, so
// that HBM latency is covered without holding data in registers.  Waits are
// cp.async.wait_group: the hardware's own completion, never a spin.
//
// Summing a bitmap tile, lane l owns rows l and l + 32: it walks its rows'
// bits in column order and adds v * x onto the row's accumulator, where the
// value sits at the row's first value (a warp scan of the rows' popcounts)
// plus the set bits before it, and x[c] is a broadcast read of the staged x
// segment.  A dense tile is summed the same way with the lanes skewed by one
// column each, so that the row-major values do not meet in one bank; its
// stored zeros are skipped (an exact identity for the sum).  COO and CSR
// tiles go 32 elements at a time: each lane forms one product, and the first
// lane of each row segment adds the segment onto the row in element order.
#include <algorithm>
#include <queue>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

constexpr int kRingBytes = 41 * 1024 + 32;  // per warp; holds any single s = 64 tile slot
constexpr int kMaxQ = 8;               // tiles in flight per warp (cp.async groups)
constexpr int kCtasPerSm = 5;          // resident one-warp CTAs per SM the shared memory allows
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kFirst = 1u << 30, kLast = 1u << 31, kRowMask = kFirst - 1;

// One tile as the kernel needs it; derived from the format arrays at build time.
struct __align__(16) ring_desc {
    int64_t vo;       // first stored value (elements)
    int64_t io;       // payload byte offset (16-byte aligned)
    uint32_t col;     // block column
    uint32_t nv;      // stored values
    uint32_t pb_sch;  // payload bytes | scheme << 24
    uint32_t info;    // block row | kFirst (first tile of its block row) | kLast
};
static_assert(sizeof(ring_desc) == 32, "ring_desc is 32 bytes");

// The largest slot: y and x segments, a COO payload of s * s keys (2 bytes
// each), s * s values and one granule of alignment slack.
template <int S>
constexpr int max_slot_bytes()
{
    return 2 * S * 8 + 2 * S * S + 8 * S * S + 16;
}
static_assert(max_slot_bytes<64>() <= kRingBytes && max_slot_bytes<32>() <= kRingBytes, "ring holds any slot");
static_assert(kRingBytes % 16 == 0, "ring slots are 16-byte aligned");

template <int S>
struct ring_smem {
    alignas(16) uint8_t ring[kRingBytes];
    ring_desc tab[64];  // descriptors of two windows of 32 tiles
    uint32_t slot[64];  // ring offset of each window entry's slot
    double ys[S];       // the block row's y segment
    double buf[32];     // products of a COO / CSR chunk
};

struct ring_args {
    tiles_view A;
    const ring_desc* desc;  // every warp's tiles, warp after warp
    const int64_t* wbeg;    // [warps + 1] each warp's range in desc
    const double* x;
    double* y;
};

// Byte offsets of a slot's parts.  Every part is a multiple of 16 bytes.
struct slot_geo {
    int x, pay, val, size;
};

template <int S>
__device__ __forceinline__ slot_geo geometry(const ring_desc& d)
{
    slot_geo g;
    g.x = (d.info & kFirst) ? S * 8 : 0;  // the y segment comes first
    g.pay = g.x + S * 8;
    g.val = g.pay + (int)(d.pb_sch & 0xffffffu);
    // values are copied in 16-byte granules from the even element at or below vo
    const int nv2 = ((int)d.nv + (int)(d.vo & 1) + 1) & ~1;
    g.size = g.val + nv2 * 8;
    return g;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// 8-byte copy; src_bytes = 0 writes zeros (src must still be a valid address)
__device__ __forceinline__ void cp8(uint32_t dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Waits until at most `newer` of this thread's copy groups are still pending.
__device__ __forceinline__ void cp_wait_newer(int newer)
{
    switch (newer) {
    case 7: cp_wait<7>(); break;
    case 6: cp_wait<6>(); break;
    case 5: cp_wait<5>(); break;
    case 4: cp_wait<4>(); break;
    case 3: cp_wait<3>(); break;
    case 2: cp_wait<2>(); break;
    case 1: cp_wait<1>(); break;
    default: cp_wait<0>(); break;
    }
}

__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }

// Queues the copies of one tile's slot at ring offset off, as one group.
template <int S>
__device__ __forceinline__ void issue(const ring_args& P, const ring_desc& d, const slot_geo& g, uint8_t* slot,
                                      int lane)
{
    const uint32_t base = smem_addr(slot);
    if (d.info & kFirst) {
        const int64_t r0 = (int64_t)(d.info & kRowMask) * S;
#pragma unroll
        for (int r = lane; r < S; r += 32) {
            const bool ok = r0 + r < P.A.m;
            cp8(base + 8 * r, ok ? P.y + r0 + r : P.y, ok ? 8 : 0);
        }
    }
    const int64_t c0 = (int64_t)d.col * S;
#pragma unroll
    for (int c = lane; c < S; c += 32) {
        const bool ok = c0 + c < P.A.n;
        cp8(base + g.x + 8 * c, ok ? P.x + c0 + c : P.x, ok ? 8 : 0);
    }
    const uint8_t* pay = P.A.payload + d.io;
    for (int k = lane; k < (g.val - g.pay) / 16; k += 32)
        cp16(base + g.pay + 16 * k, pay + 16 * k);
    const double* vsrc = static_cast<const double*>(P.A.values) + (d.vo & ~(int64_t)1);
    for (int k = lane; k < (g.size - g.val) / 16; k += 32)
        cp16(base + g.val + 16 * k, vsrc + 2 * k);
    cp_commit();
}

__device__ __forceinline__ int warp_inclusive_sum(int v, int lane)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(kFull, v, d);
        if (lane >= d)
            v += t;
    }
    return v;
}

// Bitmap tile: lane l sums rows l (+ 32).  Row r's bits are u32 words
// r * W .. r * W + W - 1 (W = S / 32), bit b of word j = column 32 j + b.
template <int S>
__device__ __forceinline__ void sum_bitmap(const uint8_t* slot, const slot_geo& g, int parity, double* ys, int lane)
{
    constexpr int R = S / 32, W = S / 32;
    const double* xs = reinterpret_cast<const double*>(slot + g.x);
    const double* vs = reinterpret_cast<const double*>(slot + g.val) + parity;
    uint32_t w[R][W];
    int q[R];
    double acc[R];
    int before = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int row = 32 * i + lane;
        if (W == 2) {
            const uint2 ww = reinterpret_cast<const uint2*>(slot + g.pay)[row];
            w[i][0] = ww.x;
            w[i][W - 1] = ww.y;
        } else {
            w[i][0] = reinterpret_cast<const uint32_t*>(slot + g.pay)[row];
        }
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < W; ++j)
            cnt += __popc(w[i][j]);
        const int inc = warp_inclusive_sum(cnt, lane);
        q[i] = before + inc - cnt;
        before += __shfl_sync(kFull, inc, 31);
        acc[i] = ys[row];
    }
#pragma unroll
    for (int j = 0; j < W; ++j) {
#pragma unroll
        for (int b = 0; b < 32; ++b) {
            const double xv = xs[32 * j + b];
#pragma unroll
            for (int i = 0; i < R; ++i) {
                if ((w[i][j] >> b) & 1u) {
                    acc[i] = fadd(acc[i], fmul(vs[q[i]], xv));
                    ++q[i];
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i)
        ys[32 * i + lane] = acc[i];
}

// Dense tile: all S * S values, row-major.  Lane l runs l columns behind
// lane 0 so that the lanes' values fall in different banks.
template <int S>
__device__ __forceinline__ void sum_dense(const uint8_t* slot, const slot_geo& g, int parity, double* ys, int lane)
{
    constexpr int R = S / 32;
    const double* xs = reinterpret_cast<const double*>(slot + g.x);
    const double* vs = reinterpret_cast<const double*>(slot + g.val) + parity;
    double acc[R];
#pragma unroll
    for (int i = 0; i < R; ++i)
        acc[i] = ys[32 * i + lane];
#pragma unroll 4
    for (int k = 0; k < S + 31; ++k) {
        const int c = k - lane;
        if (c >= 0 && c < S) {
            const double xv = xs[c];
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const double v = vs[(32 * i + lane) * S + c];
                if (v != 0.0)  // stored zeros and the zero padding past n
                    acc[i] = fadd(acc[i], fmul(v, xv));
            }
        }
    }
#pragma unroll
    for (int i = 0; i < R; ++i)
        ys[32 * i + lane] = acc[i];
}

// COO / CSR tile, 32 stored elements at a time.
template <int S, bool CSR>
__device__ __forceinline__ void sum_stream(const uint8_t* slot, const slot_geo& g, int parity, int z, double* ys,
                                           double* buf, int lane)
{
    constexpr int LG = S == 32 ? 5 : 6;
    const double* xs = reinterpret_cast<const double*>(slot + g.x);
    const double* vs = reinterpret_cast<const double*>(slot + g.val) + parity;
    const uint16_t* key16 = reinterpret_cast<const uint16_t*>(slot + g.pay);  // COO keys / CSR row ends
    const uint8_t* col8 = slot + g.pay + 2 * S;                                // CSR local columns
#pragma unroll 1
    for (int base = 0; base < z; base += 32) {
        const int k = base + lane;
        int lr = S;  // idle lanes: no row
        if (k < z) {
            int lc;
            if (CSR) {
                lc = col8[k];
                int lo = 0, hi = S;  // first r with row_end[r] > k
#pragma unroll
                for (int step = 0; step <= LG; ++step) {
                    if (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if ((int)key16[mid] > k)
                            hi = mid;
                        else
                            lo = mid + 1;
                    }
                }
                lr = lo;
            } else {
                const uint32_t key = key16[k];
                lr = (int)(key >> LG);
                lc = (int)(key & (S - 1));
            }
            buf[lane] = fmul(vs[k], xs[lc]);
        }
        const int plr = __shfl_up_sync(kFull, lr, 1);
        const bool head = k < z && (lane == 0 || plr != lr);
        const unsigned heads = __ballot_sync(kFull, head);
        __syncwarp();
        if (head) {
            const unsigned later = heads & ~((2u << lane) - 1u);  // heads after this lane (lane 31: none)
            const int end = later ? __ffs(later) - 1 : min(z - base, 32);
            double acc = ys[lr];
            for (int e = lane; e < end; ++e)
                acc = fadd(acc, buf[e]);
            ys[lr] = acc;
        }
        __syncwarp();
    }
}

template <int S>
__device__ __forceinline__ void sum_tile(const ring_args& P, const ring_desc& d, const uint8_t* slot,
                                         ring_smem<S>& sm, int lane)
{
    const slot_geo g = geometry<S>(d);
    const int parity = (int)(d.vo & 1);
    const int64_t r0 = (int64_t)(d.info & kRowMask) * S;
    if (d.info & kFirst) {
        const double* ysrc = reinterpret_cast<const double*>(slot);
#pragma unroll
        for (int r = lane; r < S; r += 32)
            sm.ys[r] = ysrc[r];
        __syncwarp();
    }
    switch (d.pb_sch >> 24) {
    case ABHSF_SCHEME_BITMAP: sum_bitmap<S>(slot, g, parity, sm.ys, lane); break;
    case ABHSF_SCHEME_DENSE: sum_dense<S>(slot, g, parity, sm.ys, lane); break;
    case ABHSF_SCHEME_CSR: sum_stream<S, true>(slot, g, parity, (int)d.nv, sm.ys, sm.buf, lane); break;
    default: sum_stream<S, false>(slot, g, parity, (int)d.nv, sm.ys, sm.buf, lane); break;
    }
    if (d.info & kLast) {
        __syncwarp();
#pragma unroll
        for (int r = lane; r < S; r += 32)
            if (r0 + r < P.A.m)
                P.y[r0 + r] = sm.ys[r];
    }
}

template <int S>
__global__ void __launch_bounds__(32, kCtasPerSm) k_spmv_f64_ring(ring_args P)
{
    __shared__ ring_smem<S> sm;
    const int lane = threadIdx.x;
    const int64_t eb = P.wbeg[blockIdx.x];
    const int n = (int)(P.wbeg[blockIdx.x + 1] - eb);
    const ring_desc* D = P.desc + eb;
    // descriptors: window 0 into the table, window 1 into registers
    ring_desc nd{};
    if (lane < n)
        sm.tab[lane] = D[lane];
    if (32 + lane < n)
        nd = D[32 + lane];
    __syncwarp();
    int win = 1;                              // next window to move into the table
    int iss = 0, con = 0, head = 0, tail = 0;  // tiles issued / summed; ring in use: [tail, head), maybe wrapped
#pragma unroll 1
    while (con < n) {
#pragma unroll 1
        while (iss < n && iss - con < kMaxQ) {
            if (iss == 32 * win) {
                // window win-2, the table half being replaced, is fully summed (con > iss - kMaxQ)
                if (iss + lane < n)
                    sm.tab[(iss + lane) & 63] = nd;
                if (iss + 32 + lane < n)
                    nd = D[iss + 32 + lane];
                ++win;
                __syncwarp();
            }
            const ring_desc d = sm.tab[iss & 63];
            const slot_geo g = geometry<S>(d);
            int off;
            if (iss == con)
                off = 0;
            else if (head > tail)
                off = head + g.size <= kRingBytes ? head : (g.size <= tail ? 0 : -1);
            else
                off = head + g.size <= tail ? head : -1;
            if (off < 0)
                break;  // no room until the oldest tile is summed
            issue<S>(P, d, g, sm.ring + off, lane);
            if (lane == 0)
                sm.slot[iss & 63] = (uint32_t)off;
            if (iss == con)
                tail = 0;
            head = off + g.size;
            ++iss;
        }
        cp_wait_newer(iss - con - 1);
        __syncwarp();
        sum_tile<S>(P, sm.tab[con & 63], sm.ring + sm.slot[con & 63], sm, lane);
        __syncwarp();
        ++con;
        if (con == iss)
            head = tail = 0;
        else
            tail = (int)sm.slot[con & 63];
    }
}

// Bytes a block row moves through the ring, plus a fixed cost per tile and
// per block row: the weight the build-time deal balances.
__global__ void k_ring_weight(int64_t nr, const uint32_t* __restrict__ rows, tiles_view A, int s,
                              uint64_t* __restrict__ weight, uint32_t* __restrict__ ntiles)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nr; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = rows[k], t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        weight[k] = (uint64_t)(8 * (A.tile_val_off[t1] - A.tile_val_off[t0]) + (A.tile_idx_off[t1] - A.tile_idx_off[t0]) +
                               (t1 - t0) * (8 * (int64_t)s + 1024) + 8 * (int64_t)s + 512);
        ntiles[k] = (uint32_t)(t1 - t0);
    }
}

__global__ void k_ring_fill(int64_t nitems, const uint32_t* __restrict__ rows, const int64_t* __restrict__ base,
                            tiles_view A, ring_desc* __restrict__ out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nitems;
         k += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t I = rows[k];
        const int64_t t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        for (int64_t t = t0; t < t1; ++t) {
            ring_desc d;
            d.vo = A.tile_val_off[t];
            d.io = A.tile_idx_off[t];
            d.col = A.tile_col[t];
            d.nv = (uint32_t)(A.tile_val_off[t + 1] - d.vo);
            d.pb_sch = (uint32_t)(A.tile_idx_off[t + 1] - d.io) | ((uint32_t)A.tile_scheme[t] << 24);
            d.info = I | (t == t0 ? kFirst : 0u) | (t == t1 - 1 ? kLast : 0u);
            out[base[k] + (t - t0)] = d;
        }
    }
}

template <int S>
void launch_ring(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    ring_args P{a.view(), reinterpret_cast<const ring_desc*>(a.ring_desc.get()), a.ring_wbeg.get(), x, y};
    k_spmv_f64_ring<S><<<(unsigned)a.ring_warps, 32, 0, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

template <int S>
int ring_ctas_per_sm()
{
    int nb = 0;
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spmv_f64_ring<S>, 32, 0));
    return std::max(nb, 1);
}

}  // namespace

void prepare_ring(abhsf_matrix& a, cudaStream_t st)
{
    a.ring_warps = 0;
    if ((a.s != 32 && a.s != 64) || a.value_type != ABHSF_VALUE_F64 || a.tree_nrows == 0 || a.M > (int64_t)kRowMask)
        return;
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int per_sm = a.s == 32 ? ring_ctas_per_sm<32>() : ring_ctas_per_sm<64>();
    const int64_t nr = a.tree_nrows;
    const int64_t warps = std::min<int64_t>((int64_t)nsm * per_sm, nr);

    dbuf<uint64_t> w_d(nr);
    dbuf<uint32_t> n_d(nr);
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nr + 255) / 256, 4096));
    k_ring_weight<<<g, 256, 0, st>>>(nr, a.tree_rows.get(), a.view(), (int)a.s, w_d.get(), n_d.get());
    ABHSF_CUDA(cudaGetLastError());
    std::vector<uint32_t> rows(nr), ntiles(nr);
    std::vector<uint64_t> wt(nr);
    ABHSF_CUDA(cudaMemcpyAsync(rows.data(), a.tree_rows.get(), nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaMemcpyAsync(wt.data(), w_d.get(), nr * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaMemcpyAsync(ntiles.data(), n_d.get(), nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));

    // longest processing time first: heaviest block row to the least loaded warp
    std::vector<int64_t> order(nr);
    for (int64_t k = 0; k < nr; ++k)
        order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int64_t p, int64_t q) { return wt[p] > wt[q]; });
    using load_t = std::pair<uint64_t, int64_t>;
    std::priority_queue<load_t, std::vector<load_t>, std::greater<load_t>> heap;
    for (int64_t w = 0; w < warps; ++w)
        heap.push({0, w});
    std::vector<std::vector<int64_t>> items(warps);
    for (int64_t k : order) {
        load_t top = heap.top();
        heap.pop();
        items[top.second].push_back(k);
        heap.push({top.first + wt[k], top.second});
    }
    std::vector<uint32_t> item_rows;
    std::vector<int64_t> item_base, wbeg(warps + 1, 0);
    item_rows.reserve(nr);
    item_base.reserve(nr);
    int64_t tiles = 0;
    for (int64_t w = 0; w < warps; ++w) {
        std::sort(items[w].begin(), items[w].end(), [&](int64_t p, int64_t q) { return rows[p] < rows[q]; });
        wbeg[w] = tiles;
        for (int64_t k : items[w]) {
            item_rows.push_back(rows[k]);
            item_base.push_back(tiles);
            tiles += ntiles[k];
        }
        if (tiles - wbeg[w] > INT32_MAX)
            return;  // too many tiles for one warp's counters: the streaming kernel serves this matrix
    }
    wbeg[warps] = tiles;
    if (tiles != a.T)
        fail(ABHSF_ERROR_CUDA, "reference-order SpMV schedule does not cover every tile");

    dbuf<uint32_t> rows_d(nr);
    dbuf<int64_t> base_d(nr);
    a.ring_desc.alloc(a.T * (int64_t)sizeof(ring_desc));
    a.ring_wbeg.alloc(warps + 1);
    ABHSF_CUDA(cudaMemcpyAsync(rows_d.get(), item_rows.data(), nr * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemcpyAsync(base_d.get(), item_base.data(), nr * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemcpyAsync(a.ring_wbeg.get(), wbeg.data(), (warps + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                               st));
    k_ring_fill<<<g, 256, 0, st>>>(nr, rows_d.get(), base_d.get(), a.view(),
                                   reinterpret_cast<ring_desc*>(a.ring_desc.get()));
    ABHSF_CUDA(cudaGetLastError());
    ABHSF_CUDA(cudaStreamSynchronize(st));
    a.ring_warps = (int)warps;
}

bool spmv_f64_ring(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (a.ring_warps == 0)
        return false;
    if (a.s == 32)
        launch_ring<32>(a, x, y, st);
    else
        launch_ring<64>(a, x, y, st);
    return true;
}

}  // namespace abhsf
