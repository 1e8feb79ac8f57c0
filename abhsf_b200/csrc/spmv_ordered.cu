// spmv_ordered.cu -- y += A x over the ABHSF format with the reference's
// summation order, FP64, sm_100a.
//
// The reference's CSR SpMV (csr_matrix::spmv_naive,
// spmv/bottlenecks/spmv.cpp:58-64) adds the products of a row one at a time,
// columns ascending, onto y[row], each product rounded before its add.  This
// kernel reproduces that order exactly: thread r of a CTA owns row r of the
// current block row, walks the block row's tiles in column order and, inside
// a tile, its row's nonzeros in column order, accumulating
// acc = dadd_rn(acc, dmul_rn(v, x)) from acc = y0.  The result is therefore
// bitwise identical to the reference CSR's y.
//
// The bytes reach shared memory through a TMA bulk-copy pipeline: each tile
// is cut into chunks of at most kVcap stored values; one lane issues
// cp.async.bulk copies of a chunk's values, payload (COO keys / CSR row ends
// and columns / bitmap) and the x and y segments into one of kSlots shared
// memory slots, kSlots - 1 chunks ahead of the chunk being summed, with an
// mbarrier tracking the bytes.  Global reads are therefore whole contiguous
// ranges (no per-lane gathers); the per-row sequential sums read shared
// memory.  Each CTA owns a contiguous, byte-balanced range of block rows
// (computed once per matrix), so no two CTAs touch one y entry.
//
// Every mbarrier wait is bounded: after kSpinLimit failed polls the CTA
// records ABHSF_DEVSTAT_WAIT_TIMEOUT in the matrix's status word and stops.
#include <algorithm>

#include "abhsf/abhsf_test.h"
#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

// Test hooks (include/abhsf/abhsf_test.h); normal operation: {-1, 0}.
int64_t g_drop_item = -1;
uint32_t g_spin_limit = 0;

constexpr int kSlots = 4;         // pipeline depth (chunks resident per CTA)
constexpr int kVcap = 1024;       // stored values per chunk
constexpr int kHdr = 64;          // tile headers cached per refill
constexpr uint32_t kSpinLimit = 1u << 22;

enum : int32_t { F_FIRST_CHUNK = 1, F_ROW_BEGIN = 2, F_ROW_END = 4, F_X_STAGED = 8, F_Y_STAGED = 16, F_NONE = 32 };

template <int S>
struct og {
    static constexpr int NT = S < 32 ? 32 : S;  // threads per CTA; thread r owns row r
    static constexpr int LG = S == 16 ? 4 : S == 32 ? 5 : S == 64 ? 6 : S == 128 ? 7 : 8;
    static constexpr int W64 = S >= 64 ? S / 64 : 1;  // u64 words per bitmap row
    static constexpr int BM_BYTES = S * S / 8;
    static constexpr int c1 = BM_BYTES > 2 * kVcap ? BM_BYTES : 2 * kVcap;
    static constexpr int c2 = 2 * S + kVcap;
    static constexpr int PCAP = ((c1 > c2 ? c1 : c2) + 16 + 15) & ~15;  // payload area
    static constexpr int VBYTES = kVcap * 8 + 16;                       // value area
    static constexpr int SEG = S * 8 < 16 ? 16 : S * 8;                 // x / y segment
    static constexpr int SLOT = 2 * SEG + PCAP + VBYTES;
};

struct item_desc {
    uint32_t row, col;
    int32_t z, k0, k1, scheme, vpre, ppre, flags, pad;
};

struct hdr_cache {
    uint32_t col[kHdr], nnz[kHdr], row[kHdr];
    int64_t val_off[kHdr], idx_off[kHdr];
    uint8_t scheme[kHdr];
};

template <int S>
struct __align__(16) ordered_smem {
    unsigned long long bar[kSlots];
    item_desc desc[kSlots];
    hdr_cache hc;
    int32_t scan[og<S>::NT / 32 + 1];
    alignas(16) unsigned char slot[kSlots][og<S>::SLOT];
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Global -> shared bulk copy (no multicast); completion counted on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Bounded wait; false (and the status word set) on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, int* status, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    atomicOr(status, ABHSF_DEVSTAT_WAIT_TIMEOUT);
    return false;
}

__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }

struct ord_args {
    tiles_view A;
    const uint32_t* tile_row;
    const int64_t* part;  // [gridDim.x + 1] tile ranges
    const double* x;
    double* y;
    int* status;
    int aligned_xy;       // x and y 16-byte aligned: segments may be bulk-copied
    uint32_t spin_limit;  // polls per wait before giving up
    int64_t drop_item;    // test hook: pipeline item whose copies are not issued (-1: none)
};

template <int S>
__global__ void __launch_bounds__(og<S>::NT) k_spmv_f64_ordered(ord_args P)
{
    using G = og<S>;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    ordered_smem<S>& sm = *reinterpret_cast<ordered_smem<S>*>(dyn_smem);
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int64_t t_begin = P.part[blockIdx.x], t_end = P.part[blockIdx.x + 1];
    if (t_begin >= t_end)
        return;
    const tiles_view& A = P.A;
    const double* __restrict__ values = static_cast<const double*>(A.values);

    if (tid == 0) {
        for (int s = 0; s < kSlots; ++s)
            mbar_init(&sm.bar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // ---------------- producer state (warp 0; lane 0 issues) ----------------
    int64_t p_t = t_begin;  // tile of the next chunk to issue
    int32_t p_k0 = 0;       // its first stored value
    int64_t p_item = 0;     // index of the next chunk to issue
    int64_t hc_base = -1;   // tiles cached in sm.hc: [hc_base, hc_base + kHdr)

    // Issues the next chunk into slot s (warp 0 only, uniform control flow).
    auto produce = [&](int s) {
        if (p_t >= t_end) {
            if (lane == 0)
                sm.desc[s].flags = F_NONE;
            return;
        }
        if (hc_base < 0 || p_t + 1 >= hc_base + kHdr) {  // refill: tile p_t and its successors
            hc_base = p_t;
            __syncwarp();
            for (int j = lane; j < kHdr; j += 32) {
                const int64_t t = hc_base + j;
                if (t < t_end) {
                    sm.hc.col[j] = A.tile_col[t];
                    sm.hc.nnz[j] = A.tile_nnz[t];
                    sm.hc.row[j] = P.tile_row[t];
                    sm.hc.val_off[j] = A.tile_val_off[t];
                    sm.hc.idx_off[j] = A.tile_idx_off[t];
                    sm.hc.scheme[j] = A.tile_scheme[t];
                }
            }
            __syncwarp();
        }
        const int h = (int)(p_t - hc_base);
        const int sch = sm.hc.scheme[h];
        const int32_t z = (int32_t)sm.hc.nnz[h];
        const int32_t stored = sch == ABHSF_SCHEME_DENSE ? S * S : z;
        const int32_t k0 = p_k0;
        const int32_t k1 = min(stored, k0 + kVcap);
        const uint32_t row = sm.hc.row[h], col = sm.hc.col[h];
        int32_t flags = 0;
        if (k0 == 0)
            flags |= F_FIRST_CHUNK;
        // the cache holds p_t and p_t + 1; p_t - 1 is read from global memory
        // when it lies before the cache
        if (k0 == 0) {
            bool begin = (p_t == t_begin);
            if (!begin)
                begin = (h > 0 ? sm.hc.row[h - 1] : __ldg(P.tile_row + p_t - 1)) != row;
            if (begin)
                flags |= F_ROW_BEGIN;
        }
        if (k1 == stored) {
            const bool end = (p_t + 1 == t_end) || sm.hc.row[h + 1] != row;
            if (end)
                flags |= F_ROW_END;
        }
        if (lane == 0) {
            unsigned char* base = sm.slot[s];
            unsigned char* ys = base;
            unsigned char* xs = base + G::SEG;
            unsigned char* pay = base + 2 * G::SEG;
            unsigned char* vb = pay + G::PCAP;
            uint32_t bytes = 0;
            // values [k0, k1)
            const uintptr_t vsrc = reinterpret_cast<uintptr_t>(values + sm.hc.val_off[h] + k0);
            const uintptr_t val = vsrc & ~uintptr_t(15);
            const int32_t vpre = (int32_t)(vsrc - val);
            const uint32_t vbytes = (uint32_t)((vpre + (k1 - k0) * 8 + 15) & ~15);
            // payload
            const unsigned char* pbase = A.payload + sm.hc.idx_off[h];
            uintptr_t psrc = 0;
            uint32_t pbytes = 0;
            int32_t ppre = 0;
            if (sch == ABHSF_SCHEME_COO) {
                const uintptr_t a = reinterpret_cast<uintptr_t>(pbase + 2 * k0);
                psrc = a & ~uintptr_t(15);
                ppre = (int32_t)(a - psrc);
                pbytes = (uint32_t)((ppre + 2 * (k1 - k0) + 15) & ~15);
            } else if (sch == ABHSF_SCHEME_CSR) {
                if (k0 == 0) {
                    psrc = reinterpret_cast<uintptr_t>(pbase);
                    pbytes = (uint32_t)((2 * S + k1 + 15) & ~15);
                } else {
                    const uintptr_t a = reinterpret_cast<uintptr_t>(pbase + 2 * S + k0);
                    psrc = a & ~uintptr_t(15);
                    ppre = (int32_t)(a - psrc);
                    pbytes = (uint32_t)((ppre + (k1 - k0) + 15) & ~15);
                }
            } else if (sch == ABHSF_SCHEME_BITMAP && k0 == 0) {
                psrc = reinterpret_cast<uintptr_t>(pbase);
                pbytes = (uint32_t)G::BM_BYTES;
            }
            const bool xst = P.aligned_xy && (int64_t)(col + 1) * S <= A.n && S * 8 >= 16;
            const bool yst = P.aligned_xy && (flags & F_ROW_BEGIN) && (int64_t)(row + 1) * S <= A.m && S * 8 >= 16;
            bytes = vbytes + pbytes + (xst ? S * 8 : 0) + (yst ? S * 8 : 0);
            if (p_item != P.drop_item) {
                mbar_expect_tx(&sm.bar[s], bytes);
                bulk_g2s(vb, reinterpret_cast<const void*>(val), vbytes, &sm.bar[s]);
                if (pbytes)
                    bulk_g2s(pay, reinterpret_cast<const void*>(psrc), pbytes, &sm.bar[s]);
                if (xst)
                    bulk_g2s(xs, P.x + (int64_t)col * S, S * 8, &sm.bar[s]);
                if (yst)
                    bulk_g2s(ys, P.y + (int64_t)row * S, S * 8, &sm.bar[s]);
            }
            item_desc& d = sm.desc[s];
            d.row = row;
            d.col = col;
            d.z = z;
            d.k0 = k0;
            d.k1 = k1;
            d.scheme = sch;
            d.vpre = vpre;
            d.ppre = ppre;
            d.flags = flags | (xst ? F_X_STAGED : 0) | (yst ? F_Y_STAGED : 0);
        }
        ++p_item;
        if (k1 == stored) {
            ++p_t;
            p_k0 = 0;
        } else {
            p_k0 = k1;
        }
    };

    if (tid < 32) {
        for (int s = 0; s < kSlots - 1; ++s)
            produce(s);
    }
    __syncthreads();

    // ---------------- consumer state (thread r = row r) ----------------
    const int r = tid;
    double acc = 0.0;
    // bitmap row still to visit: current word `cur` (index jb) and the rest
    uint64_t bw[G::W64];
    uint64_t cur = 0;
    int jb = G::W64;
    int32_t kr = 0;          // next stored-value index of this row (bitmap)
    int32_t ra = 0, rb = 0;  // this row's element range (CSR)
#pragma unroll
    for (int j = 0; j < G::W64; ++j)
        bw[j] = 0;

    int64_t step = 0;
    bool failed = false;
    for (;; ++step) {
        const int s = (int)(step % kSlots);
        const item_desc d = sm.desc[s];
        if (d.flags & F_NONE)
            break;
        if (tid < 32)
            produce((int)((step + kSlots - 1) % kSlots));
        const bool ok = mbar_wait(&sm.bar[s], (uint32_t)((step / kSlots) & 1), P.status, P.spin_limit);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        const unsigned char* base = sm.slot[s];
        const double* ys = reinterpret_cast<const double*>(base);
        const double* xs = reinterpret_cast<const double*>(base + G::SEG);
        const unsigned char* pay = base + 2 * G::SEG + d.ppre;
        const double* vb = reinterpret_cast<const double*>(base + 2 * G::SEG + G::PCAP + d.vpre);
        const int64_t grow = (int64_t)d.row * S + r;
        const bool row_ok = r < S && grow < A.m;
        const int64_t c0 = (int64_t)d.col * S;
        const bool xst = (d.flags & F_X_STAGED) != 0;
        auto X = [&](int c) -> double { return xst ? xs[c] : __ldg(P.x + c0 + c); };

        if (d.flags & F_ROW_BEGIN)
            acc = row_ok ? ((d.flags & F_Y_STAGED) ? ys[r] : P.y[grow]) : 0.0;

        const int k0 = d.k0, k1 = d.k1;
        if (d.scheme == ABHSF_SCHEME_BITMAP) {
            if (d.flags & F_FIRST_CHUNK) {
                int pc = 0;
                if (r < S) {
#pragma unroll
                    for (int j = 0; j < G::W64; ++j) {
                        uint64_t w;
                        if (S >= 64) {
                            w = reinterpret_cast<const uint64_t*>(pay + r * (S / 8))[j];
                        } else {
                            const uint64_t word = reinterpret_cast<const uint64_t*>(pay)[(r * S) >> 6];
                            w = (word >> ((r * S) & 63)) & ((1ull << (S & 63)) - 1);
                        }
                        bw[j] = w;
                        pc += __popcll(w);
                    }
                }
                cur = bw[0];
                jb = 0;
                // block-wide exclusive scan of the row popcounts -> row starts
                int inc = pc;
#pragma unroll
                for (int dd = 1; dd < 32; dd <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, inc, dd);
                    if (lane >= dd)
                        inc += t;
                }
                if (G::NT > 32) {
                    if (lane == 31)
                        sm.scan[tid >> 5] = inc;
                    __syncthreads();
                    int off = 0;
                    for (int w = 0; w < (tid >> 5); ++w)
                        off += sm.scan[w];
                    inc += off;
                    __syncthreads();
                }
                kr = inc - pc;
            }
            if (r < S) {
                // the row's values with index in [k0, k1), columns ascending
                while (kr < k1) {
                    double p[4];
                    int cnt = 0;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        while (cur == 0 && jb < G::W64 - 1) {
                            ++jb;
#pragma unroll
                            for (int q = 0; q < G::W64; ++q)
                                if (q == jb)
                                    cur = bw[q];
                        }
                        if (cur != 0 && kr + cnt < k1) {
                            const int b = __ffsll((long long)cur) - 1;
                            cur &= cur - 1;
                            p[u] = fmul(vb[kr + cnt - k0], X(jb * 64 + b));
                            ++cnt;
                        }
                    }
                    for (int u = 0; u < cnt; ++u)
                        acc = fadd(acc, p[u]);
                    kr += cnt;
                    if (cnt < 4)
                        break;
                }
            }
        } else if (d.scheme == ABHSF_SCHEME_CSR) {
            const unsigned char* cols;
            if (d.flags & F_FIRST_CHUNK) {
                const uint16_t* re = reinterpret_cast<const uint16_t*>(pay);
                if (r < S) {
                    ra = r == 0 ? 0 : re[r - 1];
                    rb = re[r];
                }
                cols = pay + 2 * S;
            } else {
                cols = pay;
            }
            if (r < S) {
                const int lo = max(ra, k0), hi = min(rb, k1);
                for (int i = lo; i < hi; i += 4) {
                    double p[4];
                    const int cnt = min(4, hi - i);
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (u < cnt)
                            p[u] = fmul(vb[i + u - k0], X(cols[i + u - k0]));
                    for (int u = 0; u < cnt; ++u)
                        acc = fadd(acc, p[u]);
                }
            }
        } else if (d.scheme == ABHSF_SCHEME_COO) {
            if (r < S) {
                const uint16_t* keys = reinterpret_cast<const uint16_t*>(pay);
                const int n = k1 - k0;
                // [lo, e): this row's elements inside the chunk (keys sorted)
                const uint32_t kr0 = (uint32_t)r << G::LG, kr1 = (uint32_t)(r + 1) << G::LG;
                int lo = 0, hi = n;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (keys[mid] < kr0)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                int e = lo;
                hi = n;
                while (e < hi) {
                    const int mid = (e + hi) >> 1;
                    if (keys[mid] < kr1)
                        e = mid + 1;
                    else
                        hi = mid;
                }
                for (int i = lo; i < e; i += 4) {
                    double p[4];
                    const int cnt = min(4, e - i);
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (u < cnt)
                            p[u] = fmul(vb[i + u], X(keys[i + u] & (S - 1)));
                    for (int u = 0; u < cnt; ++u)
                        acc = fadd(acc, p[u]);
                }
            }
        } else {  // dense: the stored zeros are skipped (the reference's CSR has no such elements)
            if (r < S) {
                const int lo = max(r * S, k0), hi = min(r * S + S, k1);
                for (int i = lo; i < hi; i += 4) {
                    double v[4], p[4];
                    const int cnt = min(4, hi - i);
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        v[u] = 0.0;
                        p[u] = 0.0;
                        const int c = i + u - r * S;
                        // columns past n (ragged right edge) hold stored zeros: never read x there
                        if (u < cnt && c0 + c < A.n) {
                            v[u] = vb[i + u - k0];
                            if (v[u] != 0.0)
                                p[u] = fmul(v[u], X(c));
                        }
                    }
                    for (int u = 0; u < cnt; ++u)
                        if (v[u] != 0.0)
                            acc = fadd(acc, p[u]);
                }
            }
        }
        if ((d.flags & F_ROW_END) && row_ok)
            P.y[grow] = acc;
        __syncthreads();
    }
    if (failed && tid == 0) {
        // drain: wait (bounded) for the copies still in flight before exiting;
        // items step .. step + kSlots - 1 were issued
        for (int64_t q = step; q < step + kSlots; ++q) {
            const int s = (int)(q % kSlots);
            if (sm.desc[s].flags & F_NONE)
                break;
            mbar_wait(&sm.bar[s], (uint32_t)((q / kSlots) & 1), P.status, P.spin_limit);
        }
    }
}

template <int S>
size_t ordered_smem_bytes()
{
    return sizeof(ordered_smem<S>);
}

template <int S>
int ordered_ctas_per_sm()
{
    const size_t smem = ordered_smem_bytes<S>();
    ABHSF_CUDA(cudaFuncSetAttribute(k_spmv_f64_ordered<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nb = 0;
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spmv_f64_ordered<S>, og<S>::NT, smem));
    return std::max(nb, 1);
}

// Per-tile work estimate used to balance the CTAs' tile ranges.
__global__ void k_tile_weight(int64_t T, const int64_t* __restrict__ val_off, const int64_t* __restrict__ idx_off,
                              const uint32_t* __restrict__ tile_row, int64_t* __restrict__ w)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t b = (val_off[t + 1] - val_off[t]) * 8 + (idx_off[t + 1] - idx_off[t]) + 512;
        if (t == 0 || tile_row[t - 1] != tile_row[t])
            b += 1024;
        w[t] = b;
    }
}

// part[p] = first tile of CTA p: the start of the block row holding the tile
// where the inclusive weight prefix first reaches p / P of the total.
__global__ void k_partition(int64_t T, int P, const int64_t* __restrict__ incl, const uint32_t* __restrict__ tile_row,
                            const int64_t* __restrict__ brow_ptr, int64_t* __restrict__ part)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= P; p += gridDim.x * blockDim.x) {
        if (p == 0) {
            part[0] = 0;
            continue;
        }
        if (p == P) {
            part[P] = T;
            continue;
        }
        const int64_t total = incl[T - 1];
        const int64_t target = (int64_t)((__int128)total * p / P);
        int64_t lo = 0, hi = T;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (incl[mid] < target)
                lo = mid + 1;
            else
                hi = mid;
        }
        part[p] = lo < T ? brow_ptr[tile_row[lo]] : T;
    }
}

template <int S>
void prepare_ordered_s(abhsf_matrix& a, cudaStream_t st)
{
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int P = nsm * ordered_ctas_per_sm<S>();
    a.ord_ctas = P;
    a.ord_part.alloc(P + 1);
    if (a.T == 0) {
        ABHSF_CUDA(cudaMemsetAsync(a.ord_part.get(), 0, (P + 1) * sizeof(int64_t), st));
        return;
    }
    dbuf<int64_t> w(a.T), incl(a.T);
    k_tile_weight<<<(unsigned)std::min<int64_t>((a.T + 255) / 256, 4096), 256, 0, st>>>(
        a.T, a.tile_val_off.get(), a.tile_idx_off.get(), a.tile_row.get(), w.get());
    ABHSF_CUDA(cudaGetLastError());
    inclusive_scan_i64(w.get(), incl.get(), a.T, st);
    k_partition<<<(P + 1 + 255) / 256, 256, 0, st>>>(a.T, P, incl.get(), a.tile_row.get(), a.brow_ptr.get(),
                                                     a.ord_part.get());
    ABHSF_CUDA(cudaGetLastError());
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

template <int S>
void launch_ordered(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    ord_args P;
    P.A = a.view();
    P.tile_row = a.tile_row.get();
    P.part = a.ord_part.get();
    P.x = x;
    P.y = y;
    P.status = a.dev_status.get();
    P.aligned_xy = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
    P.spin_limit = g_spin_limit ? g_spin_limit : kSpinLimit;
    P.drop_item = g_drop_item;
    k_spmv_f64_ordered<S><<<a.ord_ctas, og<S>::NT, ordered_smem_bytes<S>(), st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

}  // namespace

void prepare_ordered(abhsf_matrix& a, cudaStream_t st)
{
    switch (a.s) {
    case 16: prepare_ordered_s<16>(a, st); break;
    case 32: prepare_ordered_s<32>(a, st); break;
    case 64: prepare_ordered_s<64>(a, st); break;
    case 128: prepare_ordered_s<128>(a, st); break;
    case 256: prepare_ordered_s<256>(a, st); break;
    default: fail(ABHSF_ERROR_UNSUPPORTED, "block size without an SpMV kernel");
    }
}

}  // namespace abhsf

extern "C" void abhsf_test_set_hooks(int64_t drop_item, uint32_t spin_limit)
{
    abhsf::g_drop_item = drop_item < 0 ? -1 : drop_item;
    abhsf::g_spin_limit = spin_limit;
}

namespace abhsf {

void spmv_f64_ordered(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (a.M == 0 || a.T == 0)
        return;
    switch (a.s) {
    case 16: launch_ordered<16>(a, x, y, st); break;
    case 32: launch_ordered<32>(a, x, y, st); break;
    case 64: launch_ordered<64>(a, x, y, st); break;
    case 128: launch_ordered<128>(a, x, y, st); break;
    case 256: launch_ordered<256>(a, x, y, st); break;
    default: fail(ABHSF_ERROR_UNSUPPORTED, "block size without an SpMV kernel");
    }
}

}  // namespace abhsf
