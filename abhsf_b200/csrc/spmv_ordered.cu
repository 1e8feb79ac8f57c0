// spmv_ordered.cu -- y += A x over the ABHSF format with the reference's
// summation order, FP64, sm_100a.
//
// The reference's CSR SpMV (csr_matrix::spmv_naive,
// spmv/bottlenecks/spmv.cpp:58-64) adds the products of a row one at a time,
// columns ascending, onto y[row], each product rounded before its add.  This
// kernel reproduces that order exactly: thread r of a row group owns row r of
// the current block row, walks the block row's tiles in column order and,
// inside a tile, its row's nonzeros in column order, accumulating
// acc = dadd_rn(acc, product) from acc = y0.  The result is bitwise the
// reference CSR's y.
//
// Data movement (persistent, one CTA per SM):
//  * Once per matrix a schedule is built: tiles are cut into chunks of at most
//    VC stored values (fewer for COO / CSR when their index payload would not
//    fit), and the chunk list is split into G * gridDim byte-balanced streams,
//    each a whole number of block rows.  A chunk descriptor holds the
//    16-byte-aligned value and payload ranges to copy.
//  * Warp 0 is the producer: lane g feeds row group g.  For each chunk of its
//    stream it waits until a slot of the group's R-slot ring is free (empty
//    mbarrier), copies the descriptor in, and issues cp.async.bulk copies of
//    the values, payload, x segment and (at a block row's start) y segment,
//    counted on the slot's full mbarrier.  Up to R chunks per group are in
//    flight, so shared memory is mostly bytes in transit.
//  * Row group g (NTG >= S threads, named barrier 1 + g) consumes its chunks
//    in order, up to s = 64 a chunk being a whole tile: (A) a tile's first
//    chunk puts its row starts (bitmap popcount scan / CSR row ends) and
//    bitmap in shared memory; (B) all NTG threads turn values into products
//    in place, the lanes of a warp on consecutive columns of one row (a dense
//    tile's stored zeros become -0.0, which leaves any sum bitwise unchanged);
//    (C) thread r < S adds its row's products -- a contiguous range -- one at
//    a time onto its accumulator.  Thread 0 then releases the slot.
//
// Every wait is bounded.  A wait that gives up records
// ABHSF_DEVSTAT_WAIT_TIMEOUT in the matrix's status word; the producer then
// waits (bounded) for every copy it issued before the CTA exits.
#include <algorithm>

#include "abhsf/abhsf_test.h"
#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

// Test hooks (include/abhsf/abhsf_test.h); normal operation: {-1, 0}.
int64_t g_drop_item = -1;
uint32_t g_spin_limit = 0;

constexpr uint32_t kConsumerPolls = 1u << 21;  // try_wait polls of <= ~1 us each
constexpr uint32_t kProducerPolls = 1u << 27;  // non-blocking test_wait polls

enum : uint32_t { F_FIRST_CHUNK = 1, F_ROW_BEGIN = 2, F_ROW_END = 4, F_X_OK = 8, F_Y_OK = 16, F_X_STAGED = 32, F_Y_STAGED = 64 };

// Geometry per block size.  G row groups of NTG threads, R slots per group.
template <int S>
struct og {
    // NTG threads per row group: all of them form products, the first S sum rows
    static constexpr int NTG = S <= 32 ? 64 : S == 64 ? 128 : 256;
    static constexpr int NWG = NTG / 32;
    // row groups per CTA and slots per group: smem ~ G * R * SLOT <= 225 KB
    static constexpr int G = S == 16 ? 12 : S == 32 ? 7 : S == 64 ? 2 : 1;
    static constexpr int R = S == 16 ? 4 : S == 32 ? 3 : S == 64 ? 3 : S == 128 ? 3 : 4;
    // stored values per chunk: a whole tile up to s = 64
    static constexpr int VC = S <= 64 ? S * S : S == 128 ? 8192 : 4096;
    static constexpr int LG = S == 16 ? 4 : S == 32 ? 5 : S == 64 ? 6 : S == 128 ? 7 : 8;
    static constexpr int CPL = S >= 32 ? S / 32 : 1;         // 32-column groups per row
    static constexpr int LPR = S >= 32 ? 32 : S;             // lanes per row in the product phase
    static constexpr int BM_BYTES = S * S / 8;
    static constexpr int BMW = S * S / 32 < 4 ? 4 : S * S / 32;  // u32 words of a tile bitmap
    static constexpr int PCAP = (BM_BYTES > 1024 ? BM_BYTES : 1024) + 16;  // payload area
    // chunk caps: the values (VC) and the index payload (PCAP) must both fit
    static constexpr int COO_MAX = (PCAP - 16) / 2 < VC ? (PCAP - 16) / 2 : VC;  // COO elements per chunk
    static constexpr int CSR0_MAX = PCAP - 16 - 2 * S < VC ? PCAP - 16 - 2 * S : VC;  // CSR, tile's first chunk
    static constexpr int CSR_MAX = PCAP - 16 < VC ? PCAP - 16 : VC;                 // CSR, later chunks
    static constexpr int SEG = S * 8 < 16 ? 16 : S * 8;      // x / y segment bytes
    static constexpr int VBYTES = VC * 8 + 16;
    static constexpr int DESC = 64;
    static constexpr int SLOT = DESC + 2 * SEG + PCAP + VBYTES;
    static constexpr int NT = 32 + G * NTG;
};

struct __align__(16) item_t {
    uint64_t voff;    // byte offset of the copied (16-byte aligned) value range
    uint64_t poff;    // byte offset of the copied payload range
    uint32_t vbytes;  // bytes copied (multiple of 16)
    uint32_t pbytes;
    uint32_t row, col;
    int32_t k0, k1;   // stored-value range [k0, k1) of the tile in this chunk
    int32_t z;
    int16_t vpre;     // bytes from the copy start to value k0
    int16_t ppre;     // bytes from the copy start to this chunk's payload
    uint8_t scheme, flags;
    uint8_t pad[14];
};
static_assert(sizeof(item_t) == 64, "descriptor is 64 bytes");

// Every bulk copy stays inside its slot area (values <= VC, payload <= PCAP).
template <int S>
struct og_checks {
    using Gm = og<S>;
    static_assert(Gm::COO_MAX <= Gm::VC && Gm::CSR0_MAX <= Gm::VC && Gm::CSR_MAX <= Gm::VC, "chunk values fit");
    static_assert(((2 * Gm::COO_MAX + 15 + 15) & ~15) <= Gm::PCAP, "COO keys fit");
    static_assert(((2 * S + Gm::CSR0_MAX + 15) & ~15) <= Gm::PCAP, "CSR first chunk fits");
    static_assert(((Gm::CSR_MAX + 15 + 15) & ~15) <= Gm::PCAP, "CSR later chunk fits");
    static_assert(Gm::BM_BYTES <= Gm::PCAP, "bitmap fits");
    static_assert(((Gm::VC * 8 + 8 + 15) & ~15) <= Gm::VBYTES, "values fit");
    static constexpr bool ok = true;
};
static_assert(og_checks<16>::ok && og_checks<32>::ok && og_checks<64>::ok && og_checks<128>::ok &&
                  og_checks<256>::ok,
              "slot geometry");
// one CTA per SM: G rings of R slots within the 227 KB a CTA may use
static_assert(og<16>::G * og<16>::R * og<16>::SLOT <= 225 * 1024 && og<32>::G * og<32>::R * og<32>::SLOT <= 225 * 1024 &&
                  og<64>::G * og<64>::R * og<64>::SLOT <= 225 * 1024 &&
                  og<128>::G * og<128>::R * og<128>::SLOT <= 225 * 1024 &&
                  og<256>::G * og<256>::R * og<256>::SLOT <= 225 * 1024,
              "shared memory per CTA");

template <int S>
struct group_smem {
    unsigned long long full[og<S>::R], empty[og<S>::R];
    int32_t scan[og<S>::NWG + 1];
    int32_t failed;
    int32_t rs[S + 1];                         // current tile: first stored value of each row
    int32_t clo[S], chi[S], ctag[S];           // COO chunk: row r's elements [clo, chi) if ctag == item
    alignas(16) uint32_t tbm[og<S>::BMW];      // current tile's bitmap (tiles spanning chunks)
    alignas(16) unsigned char slot[og<S>::R][og<S>::SLOT];
};

template <int S>
struct ordered_smem {
    group_smem<S> g[og<S>::G];
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

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Blocking poll, suspended at most ~1 us per call.
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(1000u)
        : "memory");
    return ok != 0;
}

// Non-blocking probe.
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

// Global -> shared bulk copy (no multicast); completion counted on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void group_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }

// Group-wide OR of pred (named barrier reduction).
__device__ __forceinline__ bool group_any(int id, int n, bool pred)
{
    uint32_t out;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(out)
                 : "r"((uint32_t)pred), "r"(id), "r"(n)
                 : "memory");
    return out != 0;
}

__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }

struct ord_args {
    const item_t* items;
    const int64_t* sb;  // [gridDim.x * G + 1] item range of each stream
    const unsigned char* values;
    const unsigned char* payload;
    const double* x;
    double* y;
    int64_t m, n;
    int* status;
    int aligned_xy;       // x and y 16-byte aligned: segments may be bulk-copied
    uint32_t spin_limit;  // consumer polls per wait (0: default)
    int64_t drop_item;    // test hook: per-stream item whose copies are not issued (-1: none)
};

template <int S>
__device__ void producer(const ord_args& P, ordered_smem<S>& sm, int lane)
{
    using Gm = og<S>;
    if (lane >= Gm::G)
        return;
    group_smem<S>& gs = sm.g[lane];
    const int64_t q = (int64_t)blockIdx.x * Gm::G + lane;
    const int64_t ib = P.sb[q], ie = P.sb[q + 1];
    int64_t it = ib;
    uint32_t polls = 0;
    bool gave_up = false;
    while (it < ie) {
        const int64_t u = it - ib;  // chunk number within the stream
        const int slot = (int)(u % Gm::R);
        const uint32_t use = (uint32_t)(u / Gm::R);
        if (!mbar_test_wait(&gs.empty[slot], (use & 1) ^ 1)) {
            if (++polls > kProducerPolls || *(volatile int32_t*)&gs.failed) {
                gave_up = true;
                break;
            }
            continue;
        }
        item_t d = P.items[it];
        unsigned char* base = gs.slot[slot];
        const bool xst = P.aligned_xy && (d.flags & F_X_OK);
        const bool yst = P.aligned_xy && (d.flags & F_Y_OK) && (d.flags & F_ROW_BEGIN);
        d.flags |= (xst ? F_X_STAGED : 0) | (yst ? F_Y_STAGED : 0);
        *reinterpret_cast<item_t*>(base) = d;
        unsigned char* ys = base + Gm::DESC;
        unsigned char* xs = ys + Gm::SEG;
        unsigned char* pay = xs + Gm::SEG;
        unsigned char* vb = pay + Gm::PCAP;
        const uint32_t bytes = d.vbytes + d.pbytes + (xst ? S * 8 : 0) + (yst ? S * 8 : 0);
        if (u != P.drop_item) {
            mbar_expect_tx(&gs.full[slot], bytes);
            bulk_g2s(vb, P.values + d.voff, d.vbytes, &gs.full[slot]);
            if (d.pbytes)
                bulk_g2s(pay, P.payload + d.poff, d.pbytes, &gs.full[slot]);
            if (xst)
                bulk_g2s(xs, P.x + (int64_t)d.col * S, S * 8, &gs.full[slot]);
            if (yst)
                bulk_g2s(ys, P.y + (int64_t)d.row * S, S * 8, &gs.full[slot]);
        }
        ++it;
    }
    if (gave_up)
        atomicOr(P.status, ABHSF_DEVSTAT_WAIT_TIMEOUT);
    // drain: every chunk this lane issued has landed before the CTA exits
    const int64_t issued = it - ib;
    for (int64_t u = (issued > Gm::R ? issued - Gm::R : 0); u < issued; ++u) {
        if (u == P.drop_item)
            continue;
        if (!mbar_wait(&gs.full[u % Gm::R], (uint32_t)((u / Gm::R) & 1), kConsumerPolls))
            atomicOr(P.status, ABHSF_DEVSTAT_WAIT_TIMEOUT);
    }
}

template <int S>
__device__ void consumer(const ord_args& P, ordered_smem<S>& sm, int gidx, int r)
{
    using Gm = og<S>;
    group_smem<S>& gs = sm.g[gidx];
    const int bar_id = 1 + gidx;
    const int lane = r & 31, warp = r >> 5;
    const int64_t q = (int64_t)blockIdx.x * Gm::G + gidx;
    const int64_t nitems = P.sb[q + 1] - P.sb[q];
    const uint32_t limit = P.spin_limit ? P.spin_limit : kConsumerPolls;
    double acc = 0.0;
    int prev_slot = -1;
    for (int64_t u = 0; u < nitems; ++u) {
        const int slot = (int)(u % Gm::R);
        const bool ok = mbar_wait(&gs.full[slot], (uint32_t)((u / Gm::R) & 1), limit);
        // this barrier also ends the previous chunk: its slot can be refilled
        if (group_any(bar_id, Gm::NTG, !ok)) {
            if (r == 0) {
                *(volatile int32_t*)&gs.failed = 1;
                atomicOr(P.status, ABHSF_DEVSTAT_WAIT_TIMEOUT);
            }
            return;
        }
        if (r == 0 && prev_slot >= 0) {
            // the slot was written in place by the generic proxy; order that
            // before the bulk copies that will refill it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&gs.empty[prev_slot]);
        }
        prev_slot = slot;
        unsigned char* base = gs.slot[slot];
        const item_t d = *reinterpret_cast<const item_t*>(base);
        const double* ys = reinterpret_cast<const double*>(base + Gm::DESC);
        const double* xs = reinterpret_cast<const double*>(base + Gm::DESC + Gm::SEG);
        const unsigned char* pay = base + Gm::DESC + 2 * Gm::SEG + d.ppre;
        double* vb = reinterpret_cast<double*>(base + Gm::DESC + 2 * Gm::SEG + Gm::PCAP + d.vpre);
        const int64_t grow = (int64_t)d.row * S + r;
        const bool row_ok = r < S && grow < P.m;
        const int64_t c0 = (int64_t)d.col * S;
        const bool xst = (d.flags & F_X_STAGED) != 0;
        auto X = [&](int c) -> double { return xst ? xs[c] : __ldg(P.x + c0 + c); };
        const int k0 = d.k0, k1 = d.k1, n = k1 - k0;

        if (d.flags & F_ROW_BEGIN)
            acc = row_ok ? ((d.flags & F_Y_STAGED) ? ys[r] : P.y[grow]) : 0.0;

        // ---- phase A: tile metadata (first chunk of a tile) ----
        if (d.flags & F_FIRST_CHUNK) {
            if (d.scheme == ABHSF_SCHEME_BITMAP) {
                if (Gm::VC < S * S) {  // later chunks of the tile need the bitmap
                    const uint4* src = reinterpret_cast<const uint4*>(pay);
                    uint4* dst = reinterpret_cast<uint4*>(gs.tbm);
                    for (int i = r; i < Gm::BM_BYTES / 16; i += Gm::NTG)
                        dst[i] = src[i];
                }
                int pc = 0;
                if (r < S) {
                    if (S >= 32) {
#pragma unroll
                        for (int j = 0; j < Gm::CPL; ++j)
                            pc += __popc(reinterpret_cast<const uint32_t*>(pay)[r * Gm::CPL + j]);
                    } else {
                        const uint32_t w = reinterpret_cast<const uint32_t*>(pay)[(r * S) >> 5];
                        pc = __popc((w >> ((r * S) & 31)) & ((1u << (S & 31)) - 1));
                    }
                }
                int inc = pc;  // exclusive scan of the row popcounts over the group
#pragma unroll
                for (int dd = 1; dd < 32; dd <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, inc, dd);
                    if (lane >= dd)
                        inc += t;
                }
                if (Gm::NWG > 1) {
                    if (lane == 31)
                        gs.scan[warp] = inc;
                    group_sync(bar_id, Gm::NTG);
                    int off = 0;
                    for (int w = 0; w < warp; ++w)
                        off += gs.scan[w];
                    inc += off;
                }
                if (r < S) {
                    gs.rs[r] = inc - pc;
                    if (r == S - 1)
                        gs.rs[S] = inc;
                }
            } else if (d.scheme == ABHSF_SCHEME_CSR) {
                const uint16_t* re = reinterpret_cast<const uint16_t*>(pay);
                if (r < S)
                    gs.rs[r + 1] = re[r];
                if (r == 0)
                    gs.rs[0] = 0;
            }
            group_sync(bar_id, Gm::NTG);
        }

        // ---- phase B: products in place ----
        if (d.scheme == ABHSF_SCHEME_BITMAP) {
            int r_lo = 0, r_hi = S;
            if (Gm::VC < S * S) {  // a tile may span chunks: rows overlapping [k0, k1)
                int lo = 0, hi = S;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (gs.rs[mid] <= k0)
                        lo = mid;
                    else
                        hi = mid;
                }
                int a = lo, b = S;
                while (a < b) {
                    const int mid = (a + b) >> 1;
                    if (gs.rs[mid] < k1)
                        a = mid + 1;
                    else
                        b = mid;
                }
                r_lo = lo;
                r_hi = a;
            }
            constexpr int RPW = 32 / Gm::LPR;  // rows per warp pass
            constexpr int BATCH = 4;           // rows per batch: loads of a batch precede its stores
            const int sub = lane / Gm::LPR, cl = lane % Gm::LPR;
            const uint32_t lt = (1u << cl) - 1u;
            // x for this lane's columns, once per chunk
            double xr[Gm::CPL];
#pragma unroll
            for (int j = 0; j < Gm::CPL; ++j) {
                const int c = j * 32 + cl;
                xr[j] = (c0 + c < P.n) ? X(c) : 0.0;
            }
            // a whole tile's bitmap is read where it landed; a spanning tile's from its copy
            const uint32_t* __restrict__ tbm =
                Gm::VC < S * S ? gs.tbm : reinterpret_cast<const uint32_t*>(pay);
            const int32_t* __restrict__ rsv = gs.rs;
            double* __restrict__ vv = vb;
            for (int row0 = r_lo + (warp * RPW + sub) * BATCH; row0 < r_hi; row0 += Gm::NWG * RPW * BATCH) {
                int idx[BATCH][Gm::CPL];
                bool on[BATCH][Gm::CPL];
                double v[BATCH][Gm::CPL];
#pragma unroll
                for (int b = 0; b < BATCH; ++b) {
                    const int row = row0 + b;
                    const bool live = row < r_hi;
                    int run = live ? rsv[row] : 0;
#pragma unroll
                    for (int j = 0; j < Gm::CPL; ++j) {
                        uint32_t w = 0;
                        if (live) {
                            if (S >= 32)
                                w = tbm[row * Gm::CPL + j];
                            else
                                w = (tbm[(row * S) >> 5] >> ((row * S) & 31)) & ((1u << (S & 31)) - 1);
                        }
                        idx[b][j] = run + __popc(w & lt);
                        on[b][j] = ((w >> cl) & 1u) && idx[b][j] >= k0 && idx[b][j] < k1;
                        run += __popc(w);
                    }
                }
#pragma unroll
                for (int b = 0; b < BATCH; ++b)
#pragma unroll
                    for (int j = 0; j < Gm::CPL; ++j)
                        v[b][j] = on[b][j] ? vv[idx[b][j] - k0] : 0.0;
#pragma unroll
                for (int b = 0; b < BATCH; ++b)
#pragma unroll
                    for (int j = 0; j < Gm::CPL; ++j)
                        if (on[b][j])
                            vv[idx[b][j] - k0] = fmul(v[b][j], xr[j]);
            }
        } else if (d.scheme == ABHSF_SCHEME_COO) {
            const uint16_t* keys = reinterpret_cast<const uint16_t*>(pay);
            const int tag = (int)(u & 0x7fffffff);
            for (int i = r; i < n; i += Gm::NTG) {
                const uint32_t key = keys[i];
                const int row = (int)(key >> Gm::LG);
                vb[i] = fmul(vb[i], X(key & (S - 1)));
                // keys are sorted: the first and last element of each row mark its range
                if (i == 0 || (keys[i - 1] >> Gm::LG) != (uint32_t)row) {
                    gs.clo[row] = i;
                    gs.ctag[row] = tag;
                }
                if (i == n - 1 || (keys[i + 1] >> Gm::LG) != (uint32_t)row)
                    gs.chi[row] = i + 1;
            }
        } else if (d.scheme == ABHSF_SCHEME_CSR) {
            const unsigned char* cols = (d.flags & F_FIRST_CHUNK) ? pay + 2 * S : pay;
            for (int i = r; i < n; i += Gm::NTG)
                vb[i] = fmul(vb[i], X(cols[i]));
        } else {
            for (int i = r; i < n; i += Gm::NTG) {
                const int c = (k0 + i) & (S - 1);
                const double v = vb[i];
                // stored zeros (absent from the reference's CSR) become -0.0: a + -0.0 == a
                vb[i] = (v != 0.0 && c0 + c < P.n) ? fmul(v, X(c)) : -0.0;
            }
        }
        group_sync(bar_id, Gm::NTG);

        // ---- phase C: this row's products, one at a time, in column order ----
        if (r < S) {
            int lo, hi;
            if (d.scheme == ABHSF_SCHEME_COO) {
                const bool has = gs.ctag[r] == (int)(u & 0x7fffffff);
                lo = has ? gs.clo[r] : 0;
                hi = has ? gs.chi[r] : 0;
            } else {
                const int rs0 = d.scheme == ABHSF_SCHEME_DENSE ? r * S : gs.rs[r];
                const int rs1 = d.scheme == ABHSF_SCHEME_DENSE ? r * S + S : gs.rs[r + 1];
                lo = max(rs0, k0) - k0;
                hi = min(rs1, k1) - k0;
            }
            int i = lo;
            for (; i + 8 <= hi; i += 8) {
                double t[8];
#pragma unroll
                for (int v = 0; v < 8; ++v)
                    t[v] = vb[i + v];
#pragma unroll
                for (int v = 0; v < 8; ++v)
                    acc = fadd(acc, t[v]);
            }
            for (; i < hi; ++i)
                acc = fadd(acc, vb[i]);
        }
        if ((d.flags & F_ROW_END) && row_ok)
            P.y[grow] = acc;
    }
}

template <int S>
__global__ void __launch_bounds__(og<S>::NT, 1) k_spmv_f64_ordered(ord_args P)
{
    using Gm = og<S>;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    ordered_smem<S>& sm = *reinterpret_cast<ordered_smem<S>*>(dyn_smem);
    const int tid = threadIdx.x;
    if (tid < Gm::G) {
        group_smem<S>& gs = sm.g[tid];
        for (int s = 0; s < Gm::R; ++s) {
            mbar_init(&gs.full[s], 1);
            mbar_init(&gs.empty[s], 1);
        }
        gs.failed = 0;
        for (int i = 0; i < S; ++i)
            gs.ctag[i] = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid < 32) {
        producer<S>(P, sm, tid);
        __syncwarp();  // lanes >= G returned at once; reconverge before the CTA barrier
    } else
        consumer<S>(P, sm, (tid - 32) / Gm::NTG, (tid - 32) % Gm::NTG);
    __syncthreads();
}

// ------------------------------------------------------------ schedule build

template <int S>
__device__ __forceinline__ int chunk_cap(int sch, int k0)
{
    using Gm = og<S>;
    if (sch == ABHSF_SCHEME_COO)
        return Gm::COO_MAX;
    if (sch == ABHSF_SCHEME_CSR)
        return k0 == 0 ? Gm::CSR0_MAX : Gm::CSR_MAX;
    return Gm::VC;
}

template <int S>
__device__ __forceinline__ int tile_chunks(int sch, int z)
{
    const int stored = sch == ABHSF_SCHEME_DENSE ? S * S : z;
    int c = 0;
    for (int k0 = 0; k0 < stored; k0 += chunk_cap<S>(sch, k0))
        ++c;
    return c;
}

template <int S>
__global__ void k_count_chunks(int64_t T, const uint32_t* __restrict__ nnz, const uint8_t* __restrict__ sch,
                               const int64_t* __restrict__ val_off, const int64_t* __restrict__ idx_off,
                               const uint32_t* __restrict__ tile_row, int64_t* __restrict__ cnt,
                               int64_t* __restrict__ w)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        const int c = tile_chunks<S>(sch[t], (int)nnz[t]);
        cnt[t] = c;
        // work estimate for stream balancing: bytes moved plus a per-chunk cost
        int64_t b = (val_off[t + 1] - val_off[t]) * 8 + (idx_off[t + 1] - idx_off[t]) + 640 * c;
        if (t == 0 || tile_row[t - 1] != tile_row[t])
            b += 1024;
        w[t] = b;
    }
}

template <int S>
__global__ void k_fill_items(int64_t T, int64_t m, int64_t n, const uint32_t* __restrict__ nnz,
                             const uint8_t* __restrict__ sch, const uint32_t* __restrict__ tcol,
                             const uint32_t* __restrict__ tile_row, const int64_t* __restrict__ val_off,
                             const int64_t* __restrict__ idx_off, const int64_t* __restrict__ item_off,
                             item_t* __restrict__ items)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        const int s = sch[t];
        const int z = (int)nnz[t];
        const int stored = s == ABHSF_SCHEME_DENSE ? S * S : z;
        const uint32_t row = tile_row[t], col = tcol[t];
        const bool rb = (t == 0 || tile_row[t - 1] != row);
        const bool re = (t == T - 1 || tile_row[t + 1] != row);
        int64_t it = item_off[t];
        for (int k0 = 0; k0 < stored; ++it) {
            const int k1 = min(stored, k0 + chunk_cap<S>(s, k0));
            item_t d;
            for (int i = 0; i < 14; ++i)
                d.pad[i] = 0;
            const uint64_t va = (uint64_t)(val_off[t] + k0) * 8;
            const uint64_t va0 = va & ~uint64_t(15);
            d.voff = va0;
            d.vpre = (int16_t)(va - va0);
            d.vbytes = (uint32_t)((d.vpre + (k1 - k0) * 8 + 15) & ~15);
            const uint64_t pb = (uint64_t)idx_off[t];
            uint64_t pa = pb, pe = pb;
            if (s == ABHSF_SCHEME_COO) {
                pa = pb + 2 * (uint64_t)k0;
                pe = pb + 2 * (uint64_t)k1;
            } else if (s == ABHSF_SCHEME_CSR) {
                pa = k0 == 0 ? pb : pb + 2 * S + k0;
                pe = pb + 2 * S + k1;
            } else if (s == ABHSF_SCHEME_BITMAP && k0 == 0) {
                pe = pb + S * S / 8;
            }
            const uint64_t pa0 = pa & ~uint64_t(15);
            d.poff = pa0;
            d.ppre = (int16_t)(pa - pa0);
            d.pbytes = pe > pa ? (uint32_t)((pe - pa0 + 15) & ~uint64_t(15)) : 0;
            d.row = row;
            d.col = col;
            d.k0 = k0;
            d.k1 = k1;
            d.z = z;
            d.scheme = (uint8_t)s;
            uint8_t f = 0;
            if (k0 == 0)
                f |= F_FIRST_CHUNK;
            if (k0 == 0 && rb)
                f |= F_ROW_BEGIN;
            if (k1 == stored && re)
                f |= F_ROW_END;
            if ((int64_t)(col + 1) * S <= n)
                f |= F_X_OK;
            if ((int64_t)(row + 1) * S <= m)
                f |= F_Y_OK;
            d.flags = f;
            items[it] = d;
            k0 = k1;
        }
    }
}

// sb[q] = first chunk of stream q: chunk 0 of the first tile of the block row
// holding the tile where the inclusive work prefix first reaches q / Q of it.
__global__ void k_partition(int64_t T, int64_t Q, const int64_t* __restrict__ incl,
                            const uint32_t* __restrict__ tile_row, const int64_t* __restrict__ brow_ptr,
                            const int64_t* __restrict__ item_off, int64_t* __restrict__ sb)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q <= Q; q += (int64_t)gridDim.x * blockDim.x) {
        int64_t t0;
        if (q == 0) {
            t0 = 0;
        } else if (q == Q) {
            t0 = T;
        } else {
            const int64_t total = incl[T - 1];
            const int64_t target = (int64_t)((__int128)total * q / Q);
            int64_t lo = 0, hi = T;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (incl[mid] < target)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            t0 = lo < T ? brow_ptr[tile_row[lo]] : T;
        }
        sb[q] = item_off[t0];
    }
}

template <int S>
size_t ordered_smem_bytes()
{
    return sizeof(ordered_smem<S>);
}

template <int S>
void prepare_ordered_s(abhsf_matrix& a, cudaStream_t st)
{
    using Gm = og<S>;
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ABHSF_CUDA(cudaFuncSetAttribute(k_spmv_f64_ordered<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ordered_smem_bytes<S>()));
    const int64_t P = nsm;
    const int64_t Q = P * Gm::G;
    a.ord_ctas = (int)P;
    a.ord_streams.alloc(Q + 1);
    if (a.T == 0) {
        ABHSF_CUDA(cudaMemsetAsync(a.ord_streams.get(), 0, (Q + 1) * sizeof(int64_t), st));
        a.ord_items.alloc(1);
        ABHSF_CUDA(cudaStreamSynchronize(st));
        return;
    }
    const int64_t T = a.T;
    const unsigned g = (unsigned)std::min<int64_t>((T + 255) / 256, 4096);
    dbuf<int64_t> cnt(T + 1), item_off(T + 1), w(T), incl(T);
    ABHSF_CUDA(cudaMemsetAsync(cnt.get() + T, 0, sizeof(int64_t), st));
    k_count_chunks<S><<<g, 256, 0, st>>>(T, a.tile_nnz.get(), a.tile_scheme.get(), a.tile_val_off.get(),
                                         a.tile_idx_off.get(), a.tile_row.get(), cnt.get(), w.get());
    ABHSF_CUDA(cudaGetLastError());
    exclusive_scan_i64(cnt.get(), item_off.get(), T + 1, st);
    int64_t nitems = 0;
    ABHSF_CUDA(cudaMemcpyAsync(&nitems, item_off.get() + T, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    a.ord_items.alloc((size_t)nitems * sizeof(item_t));
    k_fill_items<S><<<g, 256, 0, st>>>(T, a.m, a.n, a.tile_nnz.get(), a.tile_scheme.get(), a.tile_col.get(),
                                       a.tile_row.get(), a.tile_val_off.get(), a.tile_idx_off.get(), item_off.get(),
                                       reinterpret_cast<item_t*>(a.ord_items.get()));
    ABHSF_CUDA(cudaGetLastError());
    inclusive_scan_i64(w.get(), incl.get(), T, st);
    k_partition<<<(unsigned)((Q + 1 + 255) / 256), 256, 0, st>>>(T, Q, incl.get(), a.tile_row.get(),
                                                                  a.brow_ptr.get(), item_off.get(),
                                                                  a.ord_streams.get());
    ABHSF_CUDA(cudaGetLastError());
    ABHSF_CUDA(cudaStreamSynchronize(st));
    a.ord_nitems = nitems;
}

template <int S>
void launch_ordered(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    ord_args P;
    P.items = reinterpret_cast<const item_t*>(a.ord_items.get());
    P.sb = a.ord_streams.get();
    P.values = a.values.get();
    P.payload = a.payload.get();
    P.x = x;
    P.y = y;
    P.m = a.m;
    P.n = a.n;
    P.status = a.dev_status.get();
    P.aligned_xy = ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
    P.spin_limit = g_spin_limit;
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
