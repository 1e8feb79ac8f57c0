// spmv_ring.cu -- y += A x and Y += A X (K right-hand sides per pass) over the
// ABHSF format in the reference's summation order, FP64, block sizes 32 and
// 64, sm_100a.
//
// The reference's CSR SpMV (csr_matrix::spmv_naive,
// spmv/bottlenecks/spmv.cpp:58-64) adds a row's products one at a time,
// columns ascending, onto y[row], each product rounded before its add.  This
// kernel keeps that order and so returns y bitwise equal to the reference's.
//
// A CTA is one producer warp and consumer teams (the layout, a template
// parameter: one or two teams of s / 32 warps with one row per lane, or four
// or two teams of one warp with s / 32 rows per lane).  A team keeps its
// rows' accumulators in registers for a whole block row; teams take block
// rows in turn.  At build time the non-empty block rows are dealt to the CTAs
// (longest processing time first, by the bytes each block row moves), every
// CTA gets its tiles as a list of 32-byte descriptors in block-row order, and
// the launch variant (layout, x / y copy mode) is timed on the matrix.  The
// producer streams the tiles through a ring in shared memory several slots
// ahead of the consumers.  A slot carries one tile, or a group of up to
// kGroupMax small tiles that are contiguous in the format arrays, ending with
// the last block row it completes: their descriptors, the y blocks of the
// tiles that start a block row, one x block per tile, and one bulk copy
// (cp.async.bulk) each for the group's index payloads and values -- issued
// first -- all completing on the slot's mbarrier.  x and y blocks travel as
// bulk copies where whole, contiguous and aligned, else as 8- or 4-byte
// cp.async by the producer lanes.  Every wait on an mbarrier is bounded: a
// wait that runs out sets ABHSF_DEVSTAT_WAIT_TIMEOUT in the matrix's status
// word, the CTA waits (again bounded) for the copies it still has in flight,
// and returns.
//
// Summing a bitmap tile, a lane walks its row's bits in column order and adds
// v * x, where the value sits at the row's first value (a warp scan of the
// rows' popcounts) plus the set bits before it, and x[c] is a broadcast read
// of the staged x block.  A dense tile is summed the same way with the lanes
// skewed by one column each, so that the row-major values do not meet in one
// bank; its stored zeros are skipped (an exact identity for the sum).  A CSR
// tile gives each lane its row's range in row_end.  A COO tile of up to 32
// elements hands each element's product to its row's lane by warp shuffles,
// in key order; a larger one whose rows hold one element each finds a row's
// element by a popcount over the occupied rows, and any other first marks
// where each row's run of keys starts and ends.  In every case a row's
// products are added in column order.
//
// With K right-hand sides (X and Y row-major, leading dimensions ldx / ldy)
// a slot holds the tile's S x K block of X (and of Y at a block row's start),
// a lane keeps K accumulators for its row, and each of the K sums follows the
// same order: column j of Y is bitwise what the SpMV of column j gives.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <queue>
#include <vector>

#include "abhsf/abhsf_test.h"
#include "common.cuh"
#include "internal.cuh"
#include "spmm_stage.cuh"

namespace abhsf {
namespace {

#ifndef ABHSF_RING_CTAS
#define ABHSF_RING_CTAS 5
#endif
#ifndef ABHSF_RING_Q
#define ABHSF_RING_Q 16
#endif
constexpr int kCtasPerSm = ABHSF_RING_CTAS;  // resident CTAs per SM
// Consumer layouts (a template parameter L): TM teams of NC warps.  Teams
// take block rows in turn, so while one team's dependent loads wait another
// sums; a team of one warp sums S / 32 rows per lane.  Matrices of few large
// tiles run faster with one team of S / 32 warps, matrices of many small tiles
// with several teams (the layout is timed per matrix when it is prepared).
//   L = 0: 1 team of S/32 warps   L = 1: 2 teams of S/32 warps
//   L = 2: 4 teams of 1 warp      L = 3: 2 teams of 1 warp
constexpr int kLayouts = 4;
constexpr int kMaxConsumerWarps = 4;
template <int S, int L>
struct layout {
    static constexpr int TM = L == 0 ? 1 : L == 2 ? 4 : 2;
    static constexpr int NC = L <= 1 ? S / 32 : 1;
    static constexpr int RPL = S / (32 * NC);
    static_assert(TM * NC <= kMaxConsumerWarps, "consumer warps");
};
constexpr int kMaxQ = ABHSF_RING_Q;          // tiles in flight per CTA (queue slots, one mbarrier each)
static_assert(kMaxQ <= 32, "the producer keeps one queue slot's ring offset per lane");
constexpr uint32_t kWaitPolls = 1u << 21;      // try_wait polls of at most ~1 us each
#ifndef ABHSF_RING_TILE_COST
#define ABHSF_RING_TILE_COST 32768
#endif
constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kFirst = 1u << 30, kLast = 1u << 31, kRowMask = kFirst - 1;
// a COO tile of more than 32 elements whose rows hold one element each
constexpr uint32_t kDistinctRows = 1u << 26;

// test hooks (abhsf_test_set_hooks)
int64_t g_drop_desc = -1;
uint32_t g_spin_limit = 0;

// One tile as the kernel needs it; derived from the format arrays at build time.
struct __align__(16) ring_desc {
    int64_t vo;       // first stored value (elements)
    int64_t io;       // payload byte offset (16-byte aligned)
    uint32_t col;     // block column
    uint32_t nv;      // stored values
    uint32_t pb_sch;  // payload bytes | scheme << 24 | kDistinctRows
    uint32_t info;    // block row | kFirst (first tile of its block row) | kLast
};
static_assert(sizeof(ring_desc) == 32, "ring_desc is 32 bytes");

// Stored value type V and compute type T (x, y, accumulators) of each
// abhsf_value_type: f64 values in f64; f32 and bf16 values in f32.
template <int VT>
struct val_traits {
    using V = double;
    using T = double;
};
template <>
struct val_traits<ABHSF_VALUE_F32> {
    using V = float;
    using T = float;
};
template <>
struct val_traits<ABHSF_VALUE_BF16> {
    using V = uint16_t;
    using T = float;
};

// Bytes of a CTA's shared memory other than the ring (queue records and
// barriers, the y block, the product buffers, the abort flag), rounded up.
template <int S, int K, int VT>
constexpr int ring_overhead()
{
    return kMaxQ * (64 + 16) + kMaxConsumerWarps * 2 * S * 2 + 64;
}

template <int S, int L>
constexpr int ring_threads()
{
    return 32 * layout<S, L>::TM * layout<S, L>::NC + 32;
}

// The ring: the shared memory of an SM (228 KiB, allocated in 1 KiB granules
// with 1 KiB reserved per CTA) split over kCtasPerSm CTAs, less the rest of
// the CTA's shared memory.
template <int S, int K, int VT>
constexpr int ring_bytes()
{
    return (((233472 / kCtasPerSm / 1024 - 1) * 1024 - ring_overhead<S, K, VT>()) / 16) * 16;
}

// Small consecutive tiles travel together: a queue slot carries up to
// kGroupMax tiles whose payloads and values are contiguous in the format
// arrays, while their slot bytes stay within kGroupBytes (a larger tile
// travels alone).
#ifndef ABHSF_RING_GROUP_MAX
#define ABHSF_RING_GROUP_MAX 16
#endif
#ifndef ABHSF_RING_GROUP_BYTES
#define ABHSF_RING_GROUP_BYTES 12288
#endif
constexpr int kGroupMax = ABHSF_RING_GROUP_MAX;
constexpr int kGroupBytes = ABHSF_RING_GROUP_BYTES;
#ifndef ABHSF_RING_SINGLE_BYTES
#define ABHSF_RING_SINGLE_BYTES (ABHSF_RING_GROUP_BYTES / 2)
#endif
constexpr int kSingleBytes = ABHSF_RING_SINGLE_BYTES;  // a first tile above this travels alone

// The largest slot of a single tile in a single-right-hand-side pass: its
// descriptor, y and x segments, a COO payload of s * s keys (2 bytes each),
// s * s values and one granule of alignment slack.  Every matrix can take
// that pass.
template <int S, int VT>
constexpr int max_slot_bytes()
{
    return 32 + 2 * S * (int)sizeof(typename val_traits<VT>::T) + 2 * S * S +
           (int)sizeof(typename val_traits<VT>::V) * S * S + 16;
}
static_assert(max_slot_bytes<64, ABHSF_VALUE_F64>() <= ring_bytes<64, 1, ABHSF_VALUE_F64>() &&
                  max_slot_bytes<32, ABHSF_VALUE_F64>() <= ring_bytes<32, 1, ABHSF_VALUE_F64>() &&
                  max_slot_bytes<64, ABHSF_VALUE_F32>() <= ring_bytes<64, 1, ABHSF_VALUE_F32>() &&
                  max_slot_bytes<64, ABHSF_VALUE_BF16>() <= ring_bytes<64, 1, ABHSF_VALUE_BF16>(),
              "the ring holds any single-right-hand-side slot");

// What the producer tells the consumers about a queued group.  The slot holds
// the group's descriptors, the y blocks of its tiles that start a block row,
// one x block per tile, the payload block and the value block.
struct __align__(16) slot_rec {
    int64_t io0;    // payload offset of the group's first tile
    int64_t vbase;  // value index at the start of the value block
    uint32_t off;   // ring offset of the slot
    int32_t ntiles;
    int32_t y_off, x_off, pay_off, val_off;  // parts, relative to the slot
    void* y;        // the group's matrix: y and its rows
    int64_t m;
    int32_t team;   // the consumer team that sums the group
    int32_t unused;
};
static_assert(sizeof(slot_rec) == 64, "slot_rec is 64 bytes");

template <int S, int K, int VT>
struct ring_smem {
    alignas(16) uint8_t ring[ring_bytes<S, K, VT>()];
    slot_rec rec[kMaxQ];              // queue slot g % kMaxQ
    unsigned long long full[kMaxQ];   // the slot's copies have landed
    unsigned long long empty[kMaxQ];  // the consumers are done with the slot
    uint16_t rng[kMaxConsumerWarps][2 * S];  // each consumer warp's COO row marks: starts, ends
    int abort;                        // a wait ran out: everyone stops
};

// One matrix of a batch: its arrays and shape (x and y come per call).
struct ring_mat {
    const uint8_t* payload;
    const void* values;
    int64_t m, n;
};

struct ring_args {
    tiles_view A;
    const ring_desc* desc;  // every CTA's tiles, CTA after CTA
    const int64_t* wbeg;    // [ctas + 1] each CTA's range in desc
    const void* x;  // X (T), row-major: element (i, j) at x[i * ldx + j]
    void* y;        // Y (T), row-major: element (i, j) at y[i * ldy + j]
    int64_t ldx, ldy;
    // a batch: descriptor column = block column | matrix index << kBatchColBits,
    // and matrix i's arrays, x and y come from mats[i], xs[i], ys[i]
    const ring_mat* mats;
    const void* const* xs;
    void* const* ys;
    int* status;     // ABHSF_DEVSTAT_* bits
    int bulk;        // x and y blocks may travel as bulk copies
    int64_t drop;    // test hook: a descriptor whose group's bulk copies are not issued (-1: none)
    uint32_t polls;  // bound of every mbarrier wait
};

// The matrix a group's tiles belong to, as the producer and consumers use it.
struct mat_view {
    const uint8_t* payload;
    const void* values;
    const void* x;
    void* y;
    int64_t m, n;
};

// B: a batch kernel (the matrix index rides in the descriptor's column)
template <bool B>
__device__ __forceinline__ mat_view view_of(const ring_args& P, int mid)
{
    if constexpr (!B) {
        return mat_view{P.A.payload, P.A.values, P.x, P.y, P.A.m, P.A.n};
    } else {
        const ring_mat& a = P.mats[mid];
        return mat_view{a.payload, a.values, P.xs[mid], P.ys[mid], a.m, a.n};
    }
}

template <bool B>
__device__ __forceinline__ uint32_t col_of(uint32_t col)
{
    return B ? col & ((1u << kBatchColBits) - 1u) : col;
}

template <bool B>
__device__ __forceinline__ int mid_of(uint32_t col)
{
    return B ? (int)(col >> kBatchColBits) : 0;
}

// Values before the tile's first value in its first 16-byte granule.
template <int VT>
__host__ __device__ __forceinline__ int lead(const ring_desc& d)
{
    return (int)(d.vo & (16 / (int)sizeof(typename val_traits<VT>::V) - 1));
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// The mbarrier sees one arrival when this thread's earlier cp.async copies land.
__device__ __forceinline__ void cp_arrive(unsigned long long* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

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

__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

// Global -> shared bulk copy (no multicast); completion counted on bar.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ double fmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }

// x, y and accumulators in T, stored values V widened to T.
__device__ __forceinline__ double widen(double v) { return v; }
__device__ __forceinline__ float widen(float v) { return v; }
__device__ __forceinline__ float widen(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }  // bf16 bits

// 4- or 8-byte copy of one x / y element (src_bytes = 0 writes zeros)
template <typename T>
__device__ __forceinline__ void cp_elem(uint32_t dst, const T* src, int src_bytes)
{
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

// A group the producer warp has formed: lane j < ntiles holds tile j's
// descriptor (d) and the index of its y block (yk).
struct group_geo {
    int ntiles, y_off, x_off, pay_off, val_off, size;
    int64_t io0, vbase;
    uint32_t pay_bytes, val_bytes;
};

// Producer warp: queues the group's slot at ring offset off as queue slot q;
// it completes on full[q].  The payload and value blocks go first: when the
// ring holds one large tile at a time, the time from a freed slot to their
// issue is on the critical path.  (Their bytes may land before the expected
// count is posted; the count only goes negative meanwhile, and the phase
// cannot complete before lane 0's arrival, which posts it.)  Where every x
// block (and y block) of the group lies whole inside x (y), is contiguous
// (one right-hand side per row of X, or ldx = K) and 16-byte aligned, each
// travels as one bulk copy issued by its tile's lane; where the K values of
// each row are 16-byte aligned runs inside wider rows (ldx > K), each row
// travels as a bulk copy; otherwise the warp copies them element by element,
// filling zeros past n (m).
template <int S, int K, int VT, bool B>
__device__ __forceinline__ void issue_group(const ring_args& P, const mat_view& mv, const ring_desc& d, int yk,
                                            const group_geo& gg, uint32_t off, int q, int team,
                                            ring_smem<S, K, VT>& sm, bool drop, int lane)
{
    using T = typename val_traits<VT>::T;
    using V = typename val_traits<VT>::V;
    constexpr int TB = sizeof(T), XB = S * K * TB;
    uint8_t* slot = sm.ring + off;
    const uint32_t base = smem_addr(slot);
    unsigned long long* bar = &sm.full[q];
    const int nt = gg.ntiles;
    if (lane == 0 && !drop) {
        // the slot's bytes were last read through the generic proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (gg.pay_bytes)
            bulk_g2s(base + gg.pay_off, mv.payload + gg.io0, gg.pay_bytes, bar);
        bulk_g2s(base + gg.val_off, static_cast<const V*>(mv.values) + gg.vbase, gg.val_bytes, bar);
    }
    if (lane < nt)
        reinterpret_cast<ring_desc*>(slot)[lane] = d;
    const T* X = static_cast<const T*>(mv.x);
    const T* Y = static_cast<const T*>(mv.y);
    // lane j < nt holds tile j (a single tile: every lane holds it)
    const int64_t c0 = (int64_t)col_of<B>(d.col) * S, r0 = (int64_t)(d.info & kRowMask) * S;
    const bool first = (d.info & kFirst) != 0;
    const bool whole = lane >= nt || (c0 + S <= mv.n && (!first || r0 + S <= mv.m));
    // (a dropped group -- a test hook -- copies x and y element by element, so
    // that cp.async.wait_all covers them when the kernel gives up)
    const bool bulk = P.bulk && !drop && P.ldx == K && P.ldy == K &&
                      ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 15) == 0 &&
                      __all_sync(kFull, whole);
    // several right-hand sides inside wider rows of X and Y (ldx, ldy > K):
    // each of a block's S rows of K values as a bulk copy of its own, where
    // those rows are whole and 16-byte aligned
    constexpr int RB = K * TB;  // bytes of one row of a block
    const bool row_bulk = !bulk && RB % 16 == 0 && P.bulk && !drop && ((P.ldx * TB) & 15) == 0 &&
                          ((P.ldy * TB) & 15) == 0 &&
                          ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 15) == 0 &&
                          __all_sync(kFull, whole);
    uint32_t xy_bytes = 0;
    if (bulk) {
        xy_bytes = (uint32_t)(nt + __popc(__ballot_sync(kFull, lane < nt && first))) * XB;
        if (lane < nt) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_g2s(base + gg.x_off + lane * XB, X + c0 * K, XB, bar);
            if (first)
                bulk_g2s(base + gg.y_off + yk * XB, Y + r0 * K, XB, bar);
        }
    } else if (row_bulk) {
        xy_bytes = (uint32_t)(nt + __popc(__ballot_sync(kFull, lane < nt && first))) * XB;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int j = 0; j < nt; ++j) {
            const int64_t cj = (int64_t)col_of<B>(__shfl_sync(kFull, d.col, j)) * S;
            const uint32_t info = __shfl_sync(kFull, d.info, j);
            const int ykj = __shfl_sync(kFull, yk, j);
            const int64_t rj = (int64_t)(info & kRowMask) * S;
            for (int c = lane; c < S; c += 32) {
                bulk_g2s(base + gg.x_off + j * XB + c * RB, X + (cj + c) * P.ldx, RB, bar);
                if (info & kFirst)
                    bulk_g2s(base + gg.y_off + ykj * XB + c * RB, Y + (rj + c) * P.ldy, RB, bar);
            }
        }
    } else if (nt == 1) {
        const uint32_t col = col_of<B>(__shfl_sync(kFull, d.col, 0)), info = __shfl_sync(kFull, d.info, 0);
        const int64_t c1 = (int64_t)col * S, r1 = (int64_t)(info & kRowMask) * S;
#pragma unroll
        for (int k = lane; k < S * K; k += 32) {
            const int c = k / K, h = k % K;
            const bool okx = c1 + c < mv.n;
            cp_elem(base + gg.x_off + TB * k, okx ? X + (c1 + c) * P.ldx + h : X, okx ? TB : 0);
            if (info & kFirst) {
                const bool oky = r1 + c < mv.m;
                cp_elem(base + gg.y_off + TB * k, oky ? Y + (r1 + c) * P.ldy + h : Y, oky ? TB : 0);
            }
        }
    } else {
        const int total = nt * S * K;
        for (int e0 = 0; e0 < total; e0 += 32) {
            const int e = e0 + lane, jj = (e / (S * K)) & 31, k = e % (S * K);
            const uint32_t col = col_of<B>(__shfl_sync(kFull, d.col, jj));
            const uint32_t info = __shfl_sync(kFull, d.info, jj);
            const int ykk = __shfl_sync(kFull, yk, jj);
            if (e < total) {
                const int c = k / K, h = k % K;
                const int64_t c1 = (int64_t)col * S;
                const bool okx = c1 + c < mv.n;
                cp_elem(base + gg.x_off + jj * XB + TB * k, okx ? X + (c1 + c) * P.ldx + h : X, okx ? TB : 0);
                if (info & kFirst) {
                    const int64_t r1 = (int64_t)(info & kRowMask) * S;
                    const bool oky = r1 + c < mv.m;
                    cp_elem(base + gg.y_off + ykk * XB + TB * k, oky ? Y + (r1 + c) * P.ldy + h : Y, oky ? TB : 0);
                }
            }
        }
    }
    __syncwarp();  // lane 0's arrival below publishes every lane's descriptor
    cp_arrive(bar);
    if (lane == 0) {
        slot_rec& r = sm.rec[q];
        r.io0 = gg.io0;
        r.vbase = gg.vbase;
        r.off = off;
        r.ntiles = nt;
        r.y_off = gg.y_off;
        r.x_off = gg.x_off;
        r.pay_off = gg.pay_off;
        r.val_off = gg.val_off;
        r.y = mv.y;
        r.m = mv.m;
        r.team = team;
        mbar_expect_tx(bar, gg.pay_bytes + gg.val_bytes + xy_bytes);  // also publishes rec[q] and the descriptors
    }
}

__device__ __forceinline__ ring_desc shfl_desc(const ring_desc& v, int src)
{
    ring_desc r;
    const uint32_t* a = reinterpret_cast<const uint32_t*>(&v);
    uint32_t* b = reinterpret_cast<uint32_t*>(&r);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        b[k] = __shfl_sync(kFull, a[k], src);
    return r;
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

// Row c of a staged x block (row stride XS), K values, as 16-byte reads where
// the values are doubles and K is even (x blocks start 16-byte aligned, and
// so do their rows then).
template <int K, int XS, typename T>
__device__ __forceinline__ void x_row(const T* xs, int c, T (&xv)[K])
{
    if constexpr (sizeof(T) == 8 && K % 2 == 0 && XS % 2 == 0) {
        const double2* p = reinterpret_cast<const double2*>(xs + c * XS);
#pragma unroll
        for (int h = 0; h < K / 2; ++h) {
            const double2 u = p[h];
            xv[2 * h] = u.x;
            xv[2 * h + 1] = u.y;
        }
    } else {
#pragma unroll
        for (int h = 0; h < K; ++h)
            xv[h] = xs[c * XS + h];
    }
}

// The rows a consumer lane sums: a team of NC warps covers the S rows of a
// block row, warp wl of the team rows 32 (wl + NC i) + lane for i < RPL
// (RPL = S / (32 NC) rows per lane).  With several rows per lane the lane's
// independent add chains interleave, and a tile's per-tile work (descriptor,
// COO row marks, bitmap offsets) is done once per tile instead of per warp.
template <int S, int NC>
__device__ __forceinline__ int row_of(int wl, int i, int lane)
{
    return 32 * (wl + NC * i) + lane;
}

// Bitmap tile.  Row r's bits are u32 words r * W .. r * W + W - 1 (W = S / 32),
// bit b of word j = column 32 j + b; a row's values start after the set bits
// of all earlier rows.
template <int S, int K, int VT, int NC, int XS = K>
__device__ __forceinline__ void sum_bitmap(const typename val_traits<VT>::T* xs, const uint8_t* pay,
                                           const typename val_traits<VT>::V* vs,
                                           typename val_traits<VT>::T (&acc)[S / (32 * NC)][K], int wl, int lane)
{
    using T = typename val_traits<VT>::T;
    constexpr int W = S / 32, RPL = S / (32 * NC), NB = S / 32;  // NB blocks of 32 rows
    uint32_t w[RPL][W];
    int q[RPL];
    int base = 0;  // set bits of the 32-row blocks before block b
    const int last = wl + NC * (RPL - 1);  // the lane's last block
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        if (b > last)
            break;
        uint32_t wb[W];
        if (W == 2) {
            const uint2 u = reinterpret_cast<const uint2*>(pay)[32 * b + lane];
            wb[0] = u.x;
            wb[W - 1] = u.y;
        } else {
            wb[0] = reinterpret_cast<const uint32_t*>(pay)[32 * b + lane];
        }
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < W; ++j)
            cnt += __popc(wb[j]);
        const int inc = warp_inclusive_sum(cnt, lane);
        if ((b - wl) % NC == 0 && b >= wl) {  // one of the lane's rows
            const int i = (b - wl) / NC;
#pragma unroll
            for (int ii = 0; ii < RPL; ++ii)
                if (ii == i) {
#pragma unroll
                    for (int j = 0; j < W; ++j)
                        w[ii][j] = wb[j];
                    q[ii] = base + inc - cnt;
                }
        }
        base += __shfl_sync(kFull, inc, 31);
    }
    // x of this word's 32 columns in registers, read as 16-byte vectors
    // (every lane reads the same address: a broadcast)
    // (one right-hand side; with several the word's x would not fit registers)
    constexpr int XW = K == 1 ? 32 : 1, XV = 16 / (int)sizeof(T);  // x values of a word; values per 16-byte read
#pragma unroll
    for (int j = 0; j < W; ++j) {
        T xw[XW];
#pragma unroll
        for (int e = 0; K == 1 && e < XW; e += XV) {
            if (XV == 2) {
                const double2 t = reinterpret_cast<const double2*>(xs + 32 * j * K)[e / 2];
                xw[e] = t.x;
                xw[e + 1] = t.y;
            } else {
                const float4 t = reinterpret_cast<const float4*>(xs + 32 * j * K)[e / 4];
                xw[e] = t.x;
                xw[e + 1] = t.y;
                xw[e + 2] = t.z;
                xw[e + 3] = t.w;
            }
        }
#pragma unroll
        for (int b = 0; b < 32; ++b) {
            T xv[K];
            if constexpr (K == 1)
                xv[0] = xw[b % XW];
            else
                x_row<K, XS>(xs, 32 * j + b, xv);
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
                if ((w[i][j] >> b) & 1u) {
                    const T v = widen(vs[q[i]]);
#pragma unroll
                    for (int h = 0; h < K; ++h)
                        acc[i][h] = fadd(acc[i][h], fmul(v, xv[h]));
                    ++q[i];
                }
            }
        }
    }
}

// Dense tile: all S * S values, row-major.  Lane l runs l columns behind
// lane 0 so that the lanes' values fall in different banks.
template <int S, int K, int VT, int NC, int XS = K>
__device__ __forceinline__ void sum_dense(const typename val_traits<VT>::T* xs,
                                          const typename val_traits<VT>::V* vs,
                                          typename val_traits<VT>::T (&acc)[S / (32 * NC)][K], int wl, int lane)
{
    using T = typename val_traits<VT>::T;
    constexpr int RPL = S / (32 * NC);
#pragma unroll 4
    for (int k = 0; k < S + 31; ++k) {
        const int c = k - lane;
        if (c >= 0 && c < S) {
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
                const T v = widen(vs[row_of<S, NC>(wl, i, lane) * S + c]);
                if (v != T(0)) {  // stored zeros and the zero padding past n
                    T xv[K];
                    x_row<K, XS>(xs, c, xv);
#pragma unroll
                    for (int h = 0; h < K; ++h)
                        acc[i][h] = fadd(acc[i][h], fmul(v, xv[h]));
                }
            }
        }
    }
}

// A COO tile of more than 32 elements whose rows hold one element each
// (flagged when the descriptors are built; stencil and band diagonals): the
// warp forms the bit set of occupied rows, and a row's element index is the
// number of occupied rows above it.
template <int S, int K, int VT, int NC, int XS = K>
__device__ __forceinline__ void sum_distinct(const typename val_traits<VT>::T* xs, const uint8_t* pay,
                                             const typename val_traits<VT>::V* vs, int z,
                                             typename val_traits<VT>::T (&acc)[S / (32 * NC)][K], int wl, int lane)
{
    using T = typename val_traits<VT>::T;
    constexpr int LG = S == 32 ? 5 : 6, RPL = S / (32 * NC);
    const uint16_t* key16 = reinterpret_cast<const uint16_t*>(pay);
    uint32_t mlo = 0, mhi = 0;
    for (int k = lane; k < z; k += 32) {  // 32 < z <= S
        const int rk = key16[k] >> LG;
        if (rk < 32)
            mlo |= 1u << rk;
        else
            mhi |= 1u << (rk - 32);
    }
    mlo = __reduce_or_sync(kFull, mlo);
    if (S == 64)
        mhi = __reduce_or_sync(kFull, mhi);
#pragma unroll
    for (int i = 0; i < RPL; ++i) {
        const int row = row_of<S, NC>(wl, i, lane);
        const bool lower = row < 32;
        const uint32_t bits = lower ? mlo : mhi;
        const int rb = lower ? row : row - 32;
        if ((bits >> rb) & 1u) {
            const int k = (lower ? 0 : __popc(mlo)) + __popc(bits & ((1u << rb) - 1u));
            const int c = (int)(key16[k] & (S - 1));
            const T v = widen(vs[k]);
            T xv[K];
            x_row<K, XS>(xs, c, xv);
#pragma unroll
            for (int h = 0; h < K; ++h)
                acc[i][h] = fadd(acc[i][h], fmul(v, xv[h]));
        }
    }
}

// COO / CSR tile: the lane adds each of its rows' elements in stored order
// (columns ascending), the rows' chains interleaved.  A CSR tile gives each
// row's range in its row_end array; a COO tile hands few products to the row
// lanes by shuffles, or marks where each row starts and ends in the sorted
// keys (rng: 2 S marks).
template <int S, int K, int VT, int NC, bool CSR, int XS = K>
__device__ __forceinline__ void sum_sparse(const typename val_traits<VT>::T* xs, const uint8_t* pay,
                                           const typename val_traits<VT>::V* vs, int z,
                                           typename val_traits<VT>::T (&acc)[S / (32 * NC)][K], uint16_t* rng,
                                           int wl, int lane)
{
    using T = typename val_traits<VT>::T;
    constexpr int LG = S == 32 ? 5 : 6, RPL = S / (32 * NC);
    const uint16_t* key16 = reinterpret_cast<const uint16_t*>(pay);  // COO keys / CSR row ends
    const uint8_t* col8 = pay + 2 * S;                                // CSR local columns
    if (!CSR && z <= 32) {
        // few elements: element lane k forms its product, and each row lane
        // takes the products of its rows from the element lanes in key order
        int rk = -1, ck = 0;
        T vk = T(0);
        if (lane < z) {
            const uint32_t key = key16[lane];
            rk = (int)(key >> LG);
            ck = (int)(key & (S - 1));
            vk = widen(vs[lane]);
        }
        T pk[K];
        x_row<K, XS>(xs, ck, pk);
#pragma unroll
        for (int h = 0; h < K; ++h)
            pk[h] = lane < z ? fmul(vk, pk[h]) : T(0);
        for (int k = 0; k < z; ++k) {
            const int r = __shfl_sync(kFull, rk, k);
#pragma unroll
            for (int h = 0; h < K; ++h) {
                const T p = __shfl_sync(kFull, pk[h], k);
#pragma unroll
                for (int i = 0; i < RPL; ++i)
                    if (r == row_of<S, NC>(wl, i, lane))
                        acc[i][h] = fadd(acc[i][h], p);
            }
        }
        return;
    }
    int lo[RPL], len[RPL];
    if (CSR) {
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
            const int row = row_of<S, NC>(wl, i, lane);
            lo[i] = row > 0 ? key16[row - 1] : 0;
            len[i] = key16[row] - lo[i];
        }
    } else {
        // every element whose row is one of this warp's marks where the row
        // starts and ends (keys sorted by row, so a row's elements are a run)
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
            const int row = row_of<S, NC>(wl, i, lane);
            rng[row] = 0;
            rng[S + row] = 0;
        }
        __syncwarp();
        for (int k = lane; k < z; k += 32) {
            const int rk = key16[k] >> LG;
            if (NC == 1 || (rk >> 5) % NC == wl) {
                if (k == 0 || (key16[k - 1] >> LG) != rk)
                    rng[rk] = (uint16_t)k;
                if (k + 1 == z || (key16[k + 1] >> LG) != rk)
                    rng[S + rk] = (uint16_t)(k + 1);
            }
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
            const int row = row_of<S, NC>(wl, i, lane);
            lo[i] = rng[row];
            len[i] = rng[S + row] - lo[i];
        }
        __syncwarp();  // read before the next tile rewrites rng
    }
    int most = len[0];
#pragma unroll
    for (int i = 1; i < RPL; ++i)
        most = max(most, len[i]);
    for (int t = 0; t < most; ++t) {
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
            if (t < len[i]) {
                const int k = lo[i] + t;
                const int c = CSR ? (int)col8[k] : (int)(key16[k] & (S - 1));
                const T v = widen(vs[k]);
                T xv[K];
                x_row<K, XS>(xs, c, xv);
#pragma unroll
                for (int h = 0; h < K; ++h)
                    acc[i][h] = fadd(acc[i][h], fmul(v, xv[h]));
            }
        }
    }
}

// Adds tile j of a queued group onto the lane's row accumulators; the first
// tile of a block row loads them from its y block, the last writes them to y.
template <int S, int K, int VT, bool B, int NC>
__device__ __forceinline__ void sum_tile(const ring_args& P, const uint8_t* slot, const slot_rec& r, int j, int& yk,
                                         uint16_t* rng, typename val_traits<VT>::T (&acc)[S / (32 * NC)][K], int wl,
                                         int lane)
{
    using T = typename val_traits<VT>::T;
    using V = typename val_traits<VT>::V;
    constexpr int XB = S * K * (int)sizeof(T), RPL = S / (32 * NC);
    const ring_desc d = reinterpret_cast<const ring_desc*>(slot)[j];
    if (d.info & kFirst) {
        const T* ys = reinterpret_cast<const T*>(slot + r.y_off + yk * XB);
#pragma unroll
        for (int i = 0; i < RPL; ++i)
#pragma unroll
            for (int h = 0; h < K; ++h)
                acc[i][h] = ys[row_of<S, NC>(wl, i, lane) * K + h];
        ++yk;
    }
    const T* xs = reinterpret_cast<const T*>(slot + r.x_off + j * XB);
    const uint8_t* pay = slot + r.pay_off + (d.io - r.io0);
    const V* vs = reinterpret_cast<const V*>(slot + r.val_off) + (d.vo - r.vbase);
    switch ((d.pb_sch >> 24) & 3u) {
    case ABHSF_SCHEME_BITMAP: sum_bitmap<S, K, VT, NC>(xs, pay, vs, acc, wl, lane); break;
    case ABHSF_SCHEME_DENSE: sum_dense<S, K, VT, NC>(xs, vs, acc, wl, lane); break;
    case ABHSF_SCHEME_CSR: sum_sparse<S, K, VT, NC, true>(xs, pay, vs, (int)d.nv, acc, rng, wl, lane); break;
    default:
        if (d.pb_sch & kDistinctRows)
            sum_distinct<S, K, VT, NC>(xs, pay, vs, (int)d.nv, acc, wl, lane);
        else
            sum_sparse<S, K, VT, NC, false>(xs, pay, vs, (int)d.nv, acc, rng, wl, lane);
        break;
    }
    if (d.info & kLast) {
        const int64_t m = B ? r.m : P.A.m;
        T* y = static_cast<T*>(B ? r.y : P.y);
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
            const int64_t rr = (int64_t)(d.info & kRowMask) * S + row_of<S, NC>(wl, i, lane);
            if (rr < m) {
#pragma unroll
                for (int h = 0; h < K; ++h)
                    y[rr * P.ldy + h] = acc[i][h];
            }
        }
    }
}

// One-pass SpMM with KT = 16 or 32 right-hand sides (FP64).  The ring's K
// accumulators a lane do not fit its slots past K = 8, so here a CTA stages
// whole tiles two deep instead (spmm_stage.cuh: the tile's S x KT block of X,
// payload and values by cp.async while the previous tile is summed) and
// splits the columns: warp w sums rows 32 (w % NC) + lane (NC = S / 32, a row
// a lane, as the ring's one-team layout) for the KW columns KW (w / NC) ..
// KW (w / NC) + KW - 1, with the ring's per-scheme sums over the staged block
// (its row stride KT).  KW = 8: a CTA of 2 KT / 8 warps at s = 64 (measured
// on the tiled mixture, k = 32: KW = 16 1.27 ms, 8 1.19 ms, 4 1.36 ms -- twice
// the warps for the same stages against decoding each tile twice as often).
// A tile's offsets are read a step before it is staged, and a block row's y
// values a step before its first tile is summed.  A block row's sums stay
// in registers from its first tile to its last; the CTA takes the block rows
// dealt to it round robin (the list is heaviest first).  RPL rows a lane
// (the ring's one-warp teams): NC = S / (32 RPL) warps cover the rows.
// Waits: cp.async.wait_group and __syncthreads only.
template <int S, int KT, int KW, int RPL>
struct staged_cfg {
    static constexpr int NC = S / (32 * RPL);  // warps over a block row's rows
    static constexpr int NW = NC * (KT / KW);
    static constexpr int NT = 32 * NW;
};

struct staged_args {
    tiles_view A;
    const uint32_t* rows;  // block rows, heaviest first
    int64_t nrows;
    const double* X;
    double* Y;
    int64_t ldx, ldy;
    int stage_bytes;  // X block + payload and values of the largest tile, 16-byte multiple
};

template <int S, int KT, int KW, int RPL>
__global__ void __launch_bounds__(staged_cfg<S, KT, KW, RPL>::NT) k_spmm_staged(staged_args P)
{
    constexpr int NC = staged_cfg<S, KT, KW, RPL>::NC, NT = staged_cfg<S, KT, KW, RPL>::NT, K = KW;
    extern __shared__ __align__(16) uint8_t st_smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wl = warp % NC, half = warp / NC;
    const tiles_view& A = P.A;
    uint16_t* rng = reinterpret_cast<uint16_t*>(st_smem + 2 * P.stage_bytes) + warp * 2 * S;
    // the CTA's tiles in order: block rows k = blockIdx.x, + gridDim.x, ...,
    // each block row's tiles; a position and the next one
    struct pos {
        int64_t k, I, t, tend;
    };
    auto advance = [&](const pos& p, pos& q) -> bool {  // q = the tile after p; false at the end
        q = p;
        ++q.t;
        if (q.t < p.tend)
            return true;
        q.k = p.k + gridDim.x;
        if (q.k >= P.nrows)
            return false;
        q.I = P.rows[q.k];
        q.t = A.brow_ptr[q.I];
        q.tend = A.brow_ptr[q.I + 1];
        return true;
    };
    if ((int64_t)blockIdx.x >= P.nrows)
        return;
    pos p0;
    p0.k = blockIdx.x;
    p0.I = P.rows[p0.k];
    p0.t = A.brow_ptr[p0.I];
    p0.tend = A.brow_ptr[p0.I + 1];
    stage::tile_meta m0 = stage::meta_of(A, p0.t);
    stage::tile<S, KT, NT>(A, P.X, P.ldx, m0, st_smem, tid);
    stage::commit();
    // the next tile's offsets are read a step ahead, so that staging it waits on nothing
    pos p1;
    bool more1 = advance(p0, p1);
    stage::tile_meta m1 = more1 ? stage::meta_of(A, p1.t) : m0;
    // a block row's y values are loaded while the block row before it is
    // summed (the rows of one block row are the same warps' lanes throughout)
    double acc[RPL][K], ynext[RPL][K];
    auto load_y = [&](int64_t brow) {
#pragma unroll
        for (int i = 0; i < RPL; ++i) {
            const int64_t r = brow * S + row_of<S, NC>(wl, i, lane);
            if (r < A.m) {
                const double2* yr = reinterpret_cast<const double2*>(P.Y + r * P.ldy + K * half);
#pragma unroll
                for (int h = 0; h < K / 2; ++h) {
                    const double2 u = yr[h];
                    ynext[i][2 * h] = u.x;
                    ynext[i][2 * h + 1] = u.y;
                }
            } else {
#pragma unroll
                for (int h = 0; h < K; ++h)
                    ynext[i][h] = 0.0;
            }
        }
    };
    load_y(p0.I);
    int cur = 0;
    bool first = true;
#pragma unroll 1
    for (;;) {
        if (more1)
            stage::tile<S, KT, NT>(A, P.X, P.ldx, m1, st_smem + (cur ^ 1) * P.stage_bytes, tid);
        stage::commit();  // (an empty group at the end keeps the wait below uniform)
        pos p2 = p1;
        const bool more2 = more1 && advance(p1, p2);
        const stage::tile_meta m2 = more2 ? stage::meta_of(A, p2.t) : m1;
        const bool next_row = more1 && p1.k != p0.k;  // the next tile starts a block row
        if (first) {
#pragma unroll
            for (int i = 0; i < RPL; ++i)
#pragma unroll
                for (int h = 0; h < K; ++h)
                    acc[i][h] = ynext[i][h];
        }
        if (next_row)
            load_y(p1.I);
        stage::wait_all_but_one();
        __syncthreads();  // tile p0.t has landed
        {
            const uint8_t* stg = st_smem + cur * P.stage_bytes;
            const double* xs = reinterpret_cast<const double*>(stg) + K * half;
            const uint8_t* pay = stg + stage::x_block_bytes<S, KT>();
            const double* vs = reinterpret_cast<const double*>(pay + m0.pb) + (m0.vo & 1);
            switch (m0.sch) {
            case ABHSF_SCHEME_BITMAP: sum_bitmap<S, K, ABHSF_VALUE_F64, NC, KT>(xs, pay, vs, acc, wl, lane); break;
            case ABHSF_SCHEME_DENSE: sum_dense<S, K, ABHSF_VALUE_F64, NC, KT>(xs, vs, acc, wl, lane); break;
            case ABHSF_SCHEME_CSR:
                sum_sparse<S, K, ABHSF_VALUE_F64, NC, true, KT>(xs, pay, vs, m0.nv, acc, rng, wl, lane);
                break;
            default: sum_sparse<S, K, ABHSF_VALUE_F64, NC, false, KT>(xs, pay, vs, m0.nv, acc, rng, wl, lane); break;
            }
        }
        if (p0.t + 1 == p0.tend) {
#pragma unroll
            for (int i = 0; i < RPL; ++i) {
                const int64_t r = p0.I * S + row_of<S, NC>(wl, i, lane);
                if (r < A.m) {
                    double2* yr = reinterpret_cast<double2*>(P.Y + r * P.ldy + K * half);
#pragma unroll
                    for (int h = 0; h < K / 2; ++h)
                        yr[h] = make_double2(acc[i][2 * h], acc[i][2 * h + 1]);
                }
            }
        }
        __syncthreads();  // everyone is done with this stage before it is refilled
        if (!more1)
            break;
        first = next_row;
        p0 = p1;
        m0 = m1;
        p1 = p2;
        m1 = m2;
        more1 = more2;
        cur ^= 1;
    }
}

template <int S, int KT, int KW, int RPL>
void launch_staged(const abhsf_matrix& a, const uint32_t* rows, int64_t nrows, const double* X, int64_t ldx,
                   double* Y, int64_t ldy, cudaStream_t st)
{
    constexpr int NT = staged_cfg<S, KT, KW, RPL>::NT, NW = staged_cfg<S, KT, KW, RPL>::NW;
    const int stage_bytes = stage::x_block_bytes<S, KT>() + (int)a.wide_cap;
    const int smem = 2 * stage_bytes + NW * 2 * S * 2;
    auto kern = k_spmm_staged<S, KT, KW, RPL>;
    ABHSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ABHSF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared));
    int dev = 0, nsm = 0, per_sm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1)
        fail(ABHSF_ERROR_UNSUPPORTED, "staged SpMM: the stages do not fit shared memory");
    const unsigned grid = (unsigned)std::min<int64_t>(nrows, (int64_t)nsm * per_sm);
    staged_args P{a.view(), rows, nrows, X, Y, ldx, ldy, stage_bytes};
    kern<<<grid, NT, smem, st>>>(P);
    ABHSF_CUDA(cudaGetLastError());
}

// Warps 0 .. TM NC - 1 sum, NC per team; the last warp produces.
template <int S, int K, int VT, bool B, int LY>
__global__ void __launch_bounds__(ring_threads<S, LY>(), kCtasPerSm) k_spmv_f64_ring(ring_args P)
{
    constexpr int TM = layout<S, LY>::TM;    // consumer teams
    constexpr int NC = layout<S, LY>::NC;    // warps of a team
    constexpr int RPL = layout<S, LY>::RPL;  // rows per lane
    constexpr int NW = TM * NC;             // consumer warps
    constexpr int kRingBytes = ring_bytes<S, K, VT>();
    extern __shared__ __align__(16) uint8_t smem_raw[];
    ring_smem<S, K, VT>& sm = *reinterpret_cast<ring_smem<S, K, VT>*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t eb = P.wbeg[blockIdx.x];
    const int n = (int)(P.wbeg[blockIdx.x + 1] - eb);
    const ring_desc* D = P.desc + eb;
    volatile int* abort = &sm.abort;
    if (tid == 0) {
        for (int b = 0; b < kMaxQ; ++b) {
            mbar_init(&sm.full[b], 32 + 1);  // the producer lanes' cp.async arrivals + the expect_tx arrival
            mbar_init(&sm.empty[b], NW);     // one arrival per consumer warp (owner team or not)
        }
        sm.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int issued = 0;  // producer: groups queued
    if (warp == NW) {
        using V = typename val_traits<VT>::V;
        constexpr int XB = S * K * (int)sizeof(typename val_traits<VT>::T), VB = sizeof(V), G = 16 / VB;
        // descriptors of tiles wbase .. wbase + 63, lane j holding tiles wbase + j and wbase + 32 + j
        ring_desc cur{}, nxt{};
        int wbase = 0;
        if (lane < n)
            cur = D[lane];
        if (32 + lane < n)
            nxt = D[32 + lane];
        int done = 0, head = 0, tail = 0;  // done: groups the consumers released; ring in use [tail, head)
        int my_off = 0;                    // lane q: ring offset of the group in queue slot q
        int team = TM - 1;                 // team of the last group queued
#pragma unroll 1
        for (int i = 0; i < n;) {
            while (i >= wbase + 32) {
                cur = nxt;
                wbase += 32;
                if (wbase + 32 + lane < n)
                    nxt = D[wbase + 32 + lane];
            }
            // a tile that would fill most of a group travels alone (every lane holds it)
            ring_desc d = shfl_desc(cur, i - wbase);
            const int est0 = 32 + ((d.info & kFirst) ? XB : 0) + XB + (int)(d.pb_sch & 0xffffffu) + (int)d.nv * VB;
            group_geo gg;
            int yk = 0;
            if (est0 > kSingleBytes || kGroupMax == 1) {
                gg.ntiles = 1;
                gg.io0 = d.io;
                gg.vbase = d.vo - lead<VT>(d);
                gg.pay_bytes = d.pb_sch & 0xffffffu;
                gg.val_bytes = (uint32_t)(((d.vo + d.nv - gg.vbase + G - 1) & ~(int64_t)(G - 1)) * VB);
                gg.y_off = 32;
                gg.x_off = gg.y_off + ((d.info & kFirst) ? XB : 0);
            } else {
                // lane j considers tile i + j (within the two windows: i - wbase < 32)
                const int rel = i - wbase + lane;
                d = shfl_desc(cur, rel & 31);
                if (i - wbase + kGroupMax > 32) {  // only then can the group reach the next window
                    const ring_desc b = shfl_desc(nxt, rel & 31);
                    if (rel >= 32)
                        d = b;
                }
                const bool have = lane < kGroupMax && i + lane < n;
                // contiguous with the previous tile in the format arrays?
                const int64_t pvo = __shfl_up_sync(kFull, d.vo, 1), pio = __shfl_up_sync(kFull, d.io, 1);
                const uint32_t pnv = __shfl_up_sync(kFull, d.nv, 1), ppb = __shfl_up_sync(kFull, d.pb_sch, 1) & 0xffffffu;
                const uint32_t pcol = __shfl_up_sync(kFull, d.col, 1);
            const bool contig =
                lane == 0 || (d.vo == pvo + pnv && d.io == pio + ppb && (!B || mid_of<B>(d.col) == mid_of<B>(pcol)));
                const bool first = (d.info & kFirst) != 0;
                const int est = have ? 32 + (first ? XB : 0) + XB + (int)(d.pb_sch & 0xffffffu) + (int)d.nv * VB : 0;
                const int cum = warp_inclusive_sum(est, lane);
                const unsigned okm = __ballot_sync(kFull, have && contig && (lane == 0 || cum <= kGroupBytes));
                int L = __ffs(~okm) - 1;  // leading tiles that form the group (lane 0 always qualifies)
                // end the group with the last block row it completes, so that
                // the next group starts a block row (and may go to another team)
                const unsigned lasts = __ballot_sync(kFull, lane < L && (d.info & kLast) != 0);
                if (lasts != 0)
                    L = 32 - __clz(lasts);
                const unsigned firsts = __ballot_sync(kFull, lane < L && first);
                yk = __popc(firsts & ((1u << lane) - 1u));
                gg.ntiles = L;
                gg.io0 = __shfl_sync(kFull, d.io, 0);
                gg.vbase = __shfl_sync(kFull, d.vo, 0) - __shfl_sync(kFull, lead<VT>(d), 0);
                const int64_t io_end = __shfl_sync(kFull, d.io + (d.pb_sch & 0xffffffu), L - 1);
                const int64_t vo_end = __shfl_sync(kFull, d.vo + d.nv, L - 1);
                gg.pay_bytes = (uint32_t)(io_end - gg.io0);
                gg.val_bytes = (uint32_t)(((vo_end - gg.vbase + G - 1) & ~(int64_t)(G - 1)) * VB);
                gg.y_off = 32 * L;
                gg.x_off = gg.y_off + __popc(firsts) * XB;
            }
            const int L = gg.ntiles;
            gg.pay_off = gg.x_off + L * XB;
            gg.val_off = gg.pay_off + (int)gg.pay_bytes;
            gg.size = gg.val_off + (int)gg.val_bytes;
            int off = -1;
#pragma unroll 1
            for (;;) {
                if (__any_sync(kFull, *abort != 0))
                    break;
                if (issued - done < kMaxQ) {
                    if (issued == done)
                        off = 0;
                    else if (head > tail)
                        off = head + gg.size <= kRingBytes ? head : (gg.size <= tail ? 0 : -1);
                    else
                        off = head + gg.size <= tail ? head : -1;
                    if (off >= 0)
                        break;
                }
                // wait until the oldest queued group is released
                const bool ok =
                    __all_sync(kFull, mbar_wait(&sm.empty[done % kMaxQ], (uint32_t)(done / kMaxQ) & 1u, P.polls));
                if (!ok)
                    break;
                ++done;
                const int oldest = __shfl_sync(kFull, my_off, done % kMaxQ);
                if (done == issued)
                    head = tail = 0;
                else
                    tail = oldest;
            }
            if (off < 0) {
                if (lane == 0)
                    *abort = 1;
                break;
            }
            const bool drop = P.drop >= eb + i && P.drop < eb + i + L;
            const mat_view mv = view_of<B>(P, mid_of<B>(__shfl_sync(kFull, d.col, 0)));
            // a group that starts a block row goes to the next team; one that
            // continues a block row stays with the team holding its sums
            if (__shfl_sync(kFull, d.info, 0) & kFirst)
                team = team + 1 == TM ? 0 : team + 1;
            issue_group<S, K, VT, B>(P, mv, d, yk, gg, (uint32_t)off, issued % kMaxQ, team, sm, drop, lane);
            if (lane == issued % kMaxQ)
                my_off = off;
            if (issued == done)
                tail = 0;
            head = off + gg.size;
            ++issued;
            i += L;
        }
    } else {
        const int team = warp / NC, wl = warp % NC;  // wl: the warp within its team
        typename val_traits<VT>::T acc[RPL][K];      // the lane's rows of the current block row
#pragma unroll
        for (int i = 0; i < RPL; ++i)
#pragma unroll
            for (int h = 0; h < K; ++h)
                acc[i][h] = 0;
#pragma unroll 1
        for (int g = 0, t = 0; t < n; ++g) {
            const int q = g % kMaxQ;
            const bool ok = __all_sync(kFull, mbar_wait(&sm.full[q], (uint32_t)(g / kMaxQ) & 1u, P.polls));
            if (!ok || __any_sync(kFull, *abort != 0)) {
                if (lane == 0)
                    *abort = 1;
                break;
            }
            const slot_rec& r = sm.rec[q];
            const int L = r.ntiles;
            if (r.team == team) {
                const uint8_t* slot = sm.ring + r.off;
                int yk = 0;
#pragma unroll 1
                for (int j = 0; j < L; ++j)
                    sum_tile<S, K, VT, B, NC>(P, slot, r, j, yk, sm.rng[warp], acc, wl, lane);
            }
            __syncwarp();
            if (lane == 0)
                mbar_arrive(&sm.empty[q]);
            t += L;
        }
    }
    __syncthreads();
    if (sm.abort) {
        // leave no copy in flight into this CTA's shared memory
        if (tid == 0)
            atomicOr(P.status, ABHSF_DEVSTAT_WAIT_TIMEOUT);
        if (warp == NW) {
            for (int i = max(0, issued - kMaxQ); i < issued; ++i)
                mbar_wait(&sm.full[i % kMaxQ], (uint32_t)(i / kMaxQ) & 1u, P.polls);
            cp_wait_all();
        }
        __syncthreads();
    }
}

// Bytes a block row moves through the ring, plus a fixed cost per tile and
// per block row: the weight the build-time deal balances.
__global__ void k_ring_weight(int64_t nr, const uint32_t* __restrict__ rows, tiles_view A, int s, int vsize,
                              uint64_t* __restrict__ weight, uint32_t* __restrict__ ntiles)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nr; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = rows[k], t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        weight[k] = (uint64_t)(vsize * (A.tile_val_off[t1] - A.tile_val_off[t0]) +
                               (A.tile_idx_off[t1] - A.tile_idx_off[t0]) +
                               (t1 - t0) * (8 * (int64_t)s + ABHSF_RING_TILE_COST) + 8 * (int64_t)s + 512);
        ntiles[k] = (uint32_t)(t1 - t0);
    }
}

__global__ void k_ring_fill(int64_t nitems, const uint32_t* __restrict__ rows, const int64_t* __restrict__ base,
                            tiles_view A, int s, uint32_t col_or, ring_desc* __restrict__ out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nitems;
         k += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t I = rows[k];
        const int64_t t0 = A.brow_ptr[I], t1 = A.brow_ptr[I + 1];
        for (int64_t t = t0; t < t1; ++t) {
            ring_desc d;
            d.vo = A.tile_val_off[t];
            d.io = A.tile_idx_off[t];
            d.col = A.tile_col[t] | col_or;
            d.nv = (uint32_t)(A.tile_val_off[t + 1] - d.vo);
            d.pb_sch = (uint32_t)(A.tile_idx_off[t + 1] - d.io) | ((uint32_t)A.tile_scheme[t] << 24);
            if (A.tile_scheme[t] == ABHSF_SCHEME_COO && d.nv > 32 && d.nv <= (uint32_t)s) {
                const uint16_t* key = reinterpret_cast<const uint16_t*>(A.payload + d.io);
                const int lg = s == 32 ? 5 : 6;
                bool distinct = true;
                for (uint32_t e = 1; e < d.nv && distinct; ++e)
                    distinct = (key[e] >> lg) != (key[e - 1] >> lg);
                if (distinct)
                    d.pb_sch |= kDistinctRows;
            }
            d.info = I | (t == t0 ? kFirst : 0u) | (t == t1 - 1 ? kLast : 0u);
            out[base[k] + (t - t0)] = d;
        }
    }
}

// Largest payload + values part of any tile's slot (bytes; vsize-byte values
// copied in 16-byte granules).
__global__ void k_ring_max_pv(int64_t T, tiles_view A, int vsize, unsigned int* __restrict__ out)
{
    const int64_t G = 16 / vsize;
    unsigned int best = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t vo = A.tile_val_off[t], nv = A.tile_val_off[t + 1] - vo;
        const int64_t pv =
            (A.tile_idx_off[t + 1] - A.tile_idx_off[t]) + (((vo & (G - 1)) + nv + G - 1) & ~(G - 1)) * vsize;
        best = max(best, (unsigned int)pv);
    }
    atomicMax(out, best);
}

// The kernel in consumer layout L (single right-hand side; passes of K > 1
// right-hand sides use layout 0).
template <int S, int K, int VT, bool B, int L>
void launch_layout(unsigned grid, const ring_args& P, cudaStream_t st)
{
    k_spmv_f64_ring<S, K, VT, B, L><<<grid, ring_threads<S, L>(), sizeof(ring_smem<S, K, VT>), st>>>(P);
}

template <int S, int K, int VT, bool B>
void launch_any(int layout, unsigned grid, const ring_args& P, cudaStream_t st)
{
    if constexpr (K == 1) {
        switch (layout) {
        case 1: launch_layout<S, K, VT, B, 1>(grid, P, st); break;
        case 2: launch_layout<S, K, VT, B, 2>(grid, P, st); break;
        case 3: launch_layout<S, K, VT, B, 3>(grid, P, st); break;
        default: launch_layout<S, K, VT, B, 0>(grid, P, st); break;
        }
    } else {
        launch_layout<S, K, VT, B, 0>(grid, P, st);
    }
    ABHSF_CUDA(cudaGetLastError());
}

// One pass: K right-hand sides, X and Y starting at their first column.
template <int S, int K, int VT>
void launch_ring(const abhsf_matrix& a, const void* x, int64_t ldx, void* y, int64_t ldy, cudaStream_t st,
                 bool tuning = false, const uint8_t* desc = nullptr, const int64_t* wbeg = nullptr, int ctas = 0)
{
    static_assert(((sizeof(ring_smem<S, K, VT>) + 1023) / 1024 + 1) * 1024 * kCtasPerSm <= 233472,
                  "kCtasPerSm CTAs fit an SM even with shared memory allocated in 1 KiB granules");
    if (!desc) {  // the whole matrix's schedule (else one chunk of block rows, abhsf_spmv_host)
        desc = a.ring_desc.get();
        wbeg = a.ring_wbeg.get();
        ctas = a.ring_warps;
    }
    ring_args P{a.view(), reinterpret_cast<const ring_desc*>(desc), wbeg, x, y, ldx, ldy, nullptr, nullptr, nullptr,
                a.dev_status.get(), a.ring_bulk, tuning ? -1 : g_drop_desc,
                (g_spin_limit && !tuning) ? g_spin_limit : kWaitPolls};
    launch_any<S, K, VT, false>(a.ring_layout, (unsigned)ctas, P, st);
}

template <int S, int K, int VT, bool B = false, int L = 0>
int ring_ctas_per_sm()
{
    int nb = 0;
    ABHSF_CUDA(cudaFuncSetAttribute(k_spmv_f64_ring<S, K, VT, B, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(ring_smem<S, K, VT>)));
    ABHSF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_spmv_f64_ring<S, K, VT, B, L>,
                                                             ring_threads<S, L>(), sizeof(ring_smem<S, K, VT>)));
    return std::max(nb, 1);
}

// Does a pass of K right-hand sides fit every tile of this matrix in the ring?
template <int S, int K, int VT>
bool ring_fits(const abhsf_matrix& a)
{
    return 32 + 2 * S * K * (int64_t)sizeof(typename val_traits<VT>::T) + (int64_t)a.ring_max_pv <=
           ring_bytes<S, K, VT>();
}

// Y += A X over columns [0, k) in passes of the largest K that fits.
template <int S>
void spmm_ring(const abhsf_matrix& a, int k, const double* X, int64_t ldx, double* Y, int64_t ldy, cudaStream_t st)
{
    for (int j = 0; j < k;) {
        const int left = k - j;
        if (left >= 8 && ring_fits<S, 8, ABHSF_VALUE_F64>(a)) {
            launch_ring<S, 8, ABHSF_VALUE_F64>(a, X + j, ldx, Y + j, ldy, st);
            j += 8;
        } else if (left >= 4 && ring_fits<S, 4, ABHSF_VALUE_F64>(a)) {
            launch_ring<S, 4, ABHSF_VALUE_F64>(a, X + j, ldx, Y + j, ldy, st);
            j += 4;
        } else if (left >= 2 && ring_fits<S, 2, ABHSF_VALUE_F64>(a)) {
            launch_ring<S, 2, ABHSF_VALUE_F64>(a, X + j, ldx, Y + j, ldy, st);
            j += 2;
        } else {
            launch_ring<S, 1, ABHSF_VALUE_F64>(a, X + j, ldx, Y + j, ldy, st);
            j += 1;
        }
    }
}

// Resident CTAs per SM of the single-right-hand-side kernels (every layout;
// the grid is sized for the smallest), setting their shared memory.
template <int S, int VT, bool B = false>
int ring_per_sm_of()
{
    return std::min(std::min(ring_ctas_per_sm<S, 1, VT, B, 0>(), ring_ctas_per_sm<S, 1, VT, B, 1>()),
                    std::min(ring_ctas_per_sm<S, 1, VT, B, 2>(), ring_ctas_per_sm<S, 1, VT, B, 3>()));
}

int ring_per_sm(int s, int vt)
{
    if (vt == ABHSF_VALUE_F64)
        return s == 32 ? ring_per_sm_of<32, ABHSF_VALUE_F64>() : ring_per_sm_of<64, ABHSF_VALUE_F64>();
    if (vt == ABHSF_VALUE_F32)
        return s == 32 ? ring_per_sm_of<32, ABHSF_VALUE_F32>() : ring_per_sm_of<64, ABHSF_VALUE_F32>();
    return s == 32 ? ring_per_sm_of<32, ABHSF_VALUE_BF16>() : ring_per_sm_of<64, ABHSF_VALUE_BF16>();
}

struct event_pair {
    cudaEvent_t a = nullptr, b = nullptr;
    event_pair()
    {
        ABHSF_CUDA(cudaEventCreate(&a));
        if (cudaEventCreate(&b) != cudaSuccess) {
            cudaEventDestroy(a);
            fail(ABHSF_ERROR_CUDA, "cudaEventCreate failed");
        }
    }
    ~event_pair()
    {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    event_pair(const event_pair&) = delete;
    event_pair& operator=(const event_pair&) = delete;
};

// ABHSF_RING_VARIANT="<layout>,<bulk>" (e.g. "0,1") fixes the launch variant
// instead of timing the four layouts: for profiles that must show one
// variant, and for runs that must not depend on timing.  Malformed values are
// ignored.
bool forced_variant(int& layout, int& bulk)
{
    const char* v = std::getenv("ABHSF_RING_VARIANT");
    int l = -1, b = -1;
    if (!v || std::sscanf(v, "%d,%d", &l, &b) != 2 || l < 0 || l >= kLayouts || (b != 0 && b != 1))
        return false;
    layout = l;
    bulk = b;
    return true;
}

// The variant (consumer layout, bulk x / y copies or not) whose launches of
// run(layout, bulk) take least time on st: one untimed and five timed each,
// the median compared.  At s = 32 layout 3 is layout 1 and is skipped.
template <typename F>
void time_variants(F&& run, int s, cudaStream_t st, int& layout, int& bulk)
{
    constexpr int kReps = 5;
    event_pair ev[kReps];
    float best = 3.4e38f;
    for (int tm = 0; tm < kLayouts; ++tm)
        for (int bk = 0; bk <= 1; ++bk) {
            if (s == 32 && tm == 3)
                continue;
            run(tm, bk);
            for (int r = 0; r < kReps; ++r) {
                ABHSF_CUDA(cudaEventRecord(ev[r].a, st));
                run(tm, bk);
                ABHSF_CUDA(cudaEventRecord(ev[r].b, st));
            }
            float t[kReps];
            for (int r = 0; r < kReps; ++r) {
                ABHSF_CUDA(cudaEventSynchronize(ev[r].b));
                ABHSF_CUDA(cudaEventElapsedTime(&t[r], ev[r].a, ev[r].b));
            }
            std::sort(t, t + kReps);
            if (t[kReps / 2] < best) {
                best = t[kReps / 2];
                layout = tm;
                bulk = bk;
            }
        }
}

// Times the single-right-hand-side variants on zero x and y and keeps the
// fastest for the matrix (each gives the same y bit for bit).
template <int S, int VT>
void tune_ring(abhsf_matrix& a, cudaStream_t st)
{
    using T = typename val_traits<VT>::T;
    if (forced_variant(a.ring_layout, a.ring_bulk))
        return;
    dbuf<T> x(a.n), y(a.m);
    ABHSF_CUDA(cudaMemsetAsync(x.get(), 0, a.n * sizeof(T), st));
    ABHSF_CUDA(cudaMemsetAsync(y.get(), 0, a.m * sizeof(T), st));
    int layout = 0, bulk = 0;
    time_variants(
        [&](int tm, int bk) {
            a.ring_layout = tm;
            a.ring_bulk = bk;
            launch_ring<S, 1, VT>(a, x.get(), 1, y.get(), 1, st, true);
        },
        S, st, layout, bulk);
    a.ring_layout = layout;
    a.ring_bulk = bulk;
    ABHSF_CUDA(cudaMemsetAsync(a.dev_status.get(), 0, sizeof(int), st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

// Deals the non-empty block rows of one or several matrices (same block size
// and value type) over the ring kernel's grid, longest processing time first,
// and writes every CTA's tile descriptors, matrix i's columns tagged with
// i << col_bits.  Returns false when a CTA would get more tiles than its
// counters hold.
bool build_ring_schedule(const std::vector<const abhsf_matrix*>& mats, int col_bits, dbuf<uint8_t>& desc,
                         dbuf<int64_t>& wbeg_d, int& ctas_out, int& max_pv_out, cudaStream_t st, int64_t brow_lo = 0,
                         int64_t brow_hi = INT64_MAX)
{
    const int s = mats[0]->s, vt = mats[0]->value_type;
    const int vsize = (int)value_size(vt);
    int dev = 0, nsm = 0;
    ABHSF_CUDA(cudaGetDevice(&dev));
    ABHSF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int per_sm = ring_per_sm(s, vt);
    std::vector<uint32_t> mid, rows, ntiles;
    std::vector<uint64_t> wt;
    int64_t total_tiles = 0;
    unsigned int mpv = 0;
    dbuf<unsigned int> max_pv(1);
    for (size_t i = 0; i < mats.size(); ++i) {
        const abhsf_matrix& a = *mats[i];
        const int64_t nr = a.tree_nrows;
        if (nr == 0)
            continue;
        total_tiles += a.T;
        dbuf<uint64_t> w_d(nr);
        dbuf<uint32_t> n_d(nr);
        const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nr + 255) / 256, 4096));
        k_ring_weight<<<g, 256, 0, st>>>(nr, a.tree_rows.get(), a.view(), s, vsize, w_d.get(), n_d.get());
        ABHSF_CUDA(cudaGetLastError());
        ABHSF_CUDA(cudaMemsetAsync(max_pv.get(), 0, sizeof(unsigned int), st));
        const unsigned gt = (unsigned)std::max<int64_t>(1, std::min<int64_t>((a.T + 255) / 256, 4096));
        k_ring_max_pv<<<gt, 256, 0, st>>>(a.T, a.view(), vsize, max_pv.get());
        ABHSF_CUDA(cudaGetLastError());
        const size_t o = rows.size();
        rows.resize(o + nr);
        ntiles.resize(o + nr);
        wt.resize(o + nr);
        mid.resize(o + nr, (uint32_t)i);
        unsigned int m_pv = 0;
        ABHSF_CUDA(cudaMemcpyAsync(rows.data() + o, a.tree_rows.get(), nr * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                   st));
        ABHSF_CUDA(cudaMemcpyAsync(wt.data() + o, w_d.get(), nr * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(ntiles.data() + o, n_d.get(), nr * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(&m_pv, max_pv.get(), sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaStreamSynchronize(st));
        mpv = std::max(mpv, m_pv);
    }
    // the slice kernel's block rows stay out (spmv_stream.cu)
    std::vector<uint8_t> skip(rows.size(), 0);
    bool any_skip = false;
    {
        size_t o = 0;
        for (size_t i = 0; i < mats.size(); ++i) {
            const auto& f = mats[i]->dc_tree_flag;
            const int64_t nr = mats[i]->tree_nrows;
            if (nr == 0)
                continue;
            for (int64_t k = 0; k < nr; ++k, ++o)
                if ((size_t)k < f.size() && f[k]) {
                    skip[o] = 1;
                    any_skip = true;
                }
        }
    }
    if (brow_lo > 0 || brow_hi < INT64_MAX || any_skip) {  // only block rows [brow_lo, brow_hi)
        size_t o = 0;
        total_tiles = 0;
        for (size_t k = 0; k < rows.size(); ++k)
            if (rows[k] >= brow_lo && rows[k] < brow_hi && !skip[k]) {
                rows[o] = rows[k];
                ntiles[o] = ntiles[k];
                wt[o] = wt[k];
                mid[o] = mid[k];
                total_tiles += ntiles[k];
                ++o;
            }
        rows.resize(o);
        ntiles.resize(o);
        wt.resize(o);
        mid.resize(o);
    }
    const int64_t nitems = (int64_t)rows.size();
    if (nitems == 0)
        return false;
    const int64_t ctas = std::min<int64_t>((int64_t)nsm * per_sm, nitems);

    // longest processing time first: heaviest block row to the least loaded CTA
    std::vector<int64_t> order(nitems);
    for (int64_t k = 0; k < nitems; ++k)
        order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int64_t p, int64_t q) { return wt[p] > wt[q]; });
    using load_t = std::pair<uint64_t, int64_t>;
    std::priority_queue<load_t, std::vector<load_t>, std::greater<load_t>> heap;
    for (int64_t c = 0; c < ctas; ++c)
        heap.push({0, c});
    std::vector<std::vector<int64_t>> items(ctas);
    for (int64_t k : order) {
        load_t top = heap.top();
        heap.pop();
        items[top.second].push_back(k);
        heap.push({top.first + wt[k], top.second});
    }
    // every CTA's items in (matrix, block row) order; each item's first descriptor
    std::vector<std::vector<uint32_t>> m_rows(mats.size());
    std::vector<std::vector<int64_t>> m_base(mats.size());
    std::vector<int64_t> wbeg(ctas + 1, 0);
    int64_t tiles = 0;
    for (int64_t c = 0; c < ctas; ++c) {
        std::sort(items[c].begin(), items[c].end(), [&](int64_t p, int64_t q) {
            return mid[p] != mid[q] ? mid[p] < mid[q] : rows[p] < rows[q];
        });
        wbeg[c] = tiles;
        for (int64_t k : items[c]) {
            m_rows[mid[k]].push_back(rows[k]);
            m_base[mid[k]].push_back(tiles);
            tiles += ntiles[k];
        }
        if (tiles - wbeg[c] > INT32_MAX)
            return false;
    }
    wbeg[ctas] = tiles;
    if (tiles != total_tiles)
        fail(ABHSF_ERROR_CUDA, "ring SpMV schedule does not cover every tile");

    desc.alloc(std::max<int64_t>(tiles, 1) * (int64_t)sizeof(ring_desc));
    wbeg_d.alloc(ctas + 1);
    ABHSF_CUDA(cudaMemcpyAsync(wbeg_d.get(), wbeg.data(), (ctas + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    for (size_t i = 0; i < mats.size(); ++i) {
        const int64_t n = (int64_t)m_rows[i].size();
        if (n == 0)
            continue;
        dbuf<uint32_t> rows_d(n);
        dbuf<int64_t> base_d(n);
        ABHSF_CUDA(cudaMemcpyAsync(rows_d.get(), m_rows[i].data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(base_d.get(), m_base[i].data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        const uint32_t col_or = col_bits >= 32 ? 0u : (uint32_t)i << col_bits;
        const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 4096));
        k_ring_fill<<<g, 256, 0, st>>>(n, rows_d.get(), base_d.get(), mats[i]->view(), s, col_or,
                                       reinterpret_cast<ring_desc*>(desc.get()));
        ABHSF_CUDA(cudaGetLastError());
        ABHSF_CUDA(cudaStreamSynchronize(st));  // before the host vectors and staging buffers go
    }
    ctas_out = (int)ctas;
    max_pv_out = (int)mpv;
    return true;
}

template <int S>
void ring_set_up_all()
{
    ring_ctas_per_sm<S, 2, ABHSF_VALUE_F64>();
    ring_ctas_per_sm<S, 4, ABHSF_VALUE_F64>();
    ring_ctas_per_sm<S, 8, ABHSF_VALUE_F64>();
}

void batch_launch(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st, bool tuning)
{
    ring_args P{};
    P.desc = reinterpret_cast<const ring_desc*>(b.desc.get());
    P.wbeg = b.wbeg.get();
    P.ldx = P.ldy = 1;
    P.mats = reinterpret_cast<const ring_mat*>(b.table.get());
    P.xs = reinterpret_cast<const void* const*>(xs);
    P.ys = reinterpret_cast<void* const*>(ys);
    P.status = b.dev_status.get();
    P.bulk = b.bulk;
    P.drop = -1;
    P.polls = (g_spin_limit && !tuning) ? g_spin_limit : kWaitPolls;
    if (b.s == 32)
        launch_any<32, 1, ABHSF_VALUE_F64, true>(b.layout, (unsigned)b.ctas, P, st);
    else
        launch_any<64, 1, ABHSF_VALUE_F64, true>(b.layout, (unsigned)b.ctas, P, st);
}


}  // namespace

// The non-empty block rows outside the slices, heaviest first (seq_rows).
void keep_rows(abhsf_matrix& a, cudaStream_t st)
{
    a.seq_nrows = 0;
    if (a.dc_rows == 0)
        return;
    std::vector<uint32_t> rows(a.tree_nrows), keep;
    ABHSF_CUDA(cudaMemcpyAsync(rows.data(), a.tree_rows.get(), a.tree_nrows * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    for (int64_t k = 0; k < a.tree_nrows; ++k)
        if (!a.dc_tree_flag[k])
            keep.push_back(rows[k]);
    a.seq_nrows = (int64_t)keep.size();
    a.seq_rows.alloc(std::max<size_t>(keep.size(), 1));
    if (!keep.empty())
        ABHSF_CUDA(cudaMemcpyAsync(a.seq_rows.get(), keep.data(), keep.size() * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

void prepare_ring(abhsf_matrix& a, cudaStream_t st)
{
    a.ring_warps = 0;
    a.ring_ready = false;
    if (a.tree_nrows == 0)
        return;
    if (a.s != 32 && a.s != 64) {
        // no ring kernel: the slices take the hypersparse block rows, the
        // streaming kernel (spmv_seq.cu) the rest
        prepare_stream(a, a.dc_avg, st);
        keep_rows(a, st);
        prepare_wide(a, st);
        return;
    }
    if (a.M > (int64_t)kRowMask)
        return;
    if (a.value_type == ABHSF_VALUE_F64) {
        if (a.s == 32)
            ring_set_up_all<32>();
        else
            ring_set_up_all<64>();
    }
    prepare_stream(a, a.dc_avg, st);
    keep_rows(a, st);
    prepare_wide(a, st);
    int ctas = 0, mpv = 0;
    if (!build_ring_schedule({&a}, 32, a.ring_desc, a.ring_wbeg, ctas, mpv, st)) {
        // every block row is a slice row, or the ring's counters would overflow
        a.ring_ready = (a.dc_warps > 0 || a.dc_cwarps > 0) && a.dc_rows == a.tree_nrows;
        return;  // else the streaming kernel serves this matrix
    }
    a.ring_ready = true;
    a.ring_max_pv = mpv;
    a.ring_warps = ctas;
    if (ctas > 0)
        slices_beside_ring(a, st);
    if (a.value_type == ABHSF_VALUE_F64)
        a.s == 32 ? tune_ring<32, ABHSF_VALUE_F64>(a, st) : tune_ring<64, ABHSF_VALUE_F64>(a, st);
    else if (a.value_type == ABHSF_VALUE_F32)
        a.s == 32 ? tune_ring<32, ABHSF_VALUE_F32>(a, st) : tune_ring<64, ABHSF_VALUE_F32>(a, st);
    else
        a.s == 32 ? tune_ring<32, ABHSF_VALUE_BF16>(a, st) : tune_ring<64, ABHSF_VALUE_BF16>(a, st);
}

void prepare_batch(abhsf_batch& b, cudaStream_t st)
{
    if (b.s == 32)
        ring_per_sm_of<32, ABHSF_VALUE_F64, true>();
    else
        ring_per_sm_of<64, ABHSF_VALUE_F64, true>();
    std::vector<ring_mat> table;
    for (const abhsf_matrix* a : b.mats)
        table.push_back(ring_mat{a->payload.get(), a->values.get(), a->m, a->n});
    b.table.alloc((int64_t)(table.size() * sizeof(ring_mat)));
    ABHSF_CUDA(cudaMemcpyAsync(b.table.get(), table.data(), table.size() * sizeof(ring_mat), cudaMemcpyHostToDevice,
                               st));
    b.dev_status.alloc(1);
    ABHSF_CUDA(cudaMemsetAsync(b.dev_status.get(), 0, sizeof(int), st));
    int mpv = 0;
    b.ctas = 0;
    prepare_batch_stream(b, st);
    int64_t ring_rows = 0;  // non-empty block rows left to the ring kernel
    for (const abhsf_matrix* a : b.mats)
        for (uint8_t f : a->dc_tree_flag)
            ring_rows += f ? 0 : 1;
    for (const abhsf_matrix* a : b.mats)
        if (a->dc_tree_flag.size() != (size_t)a->tree_nrows)
            ring_rows += a->tree_nrows;
    if (!build_ring_schedule(b.mats, kBatchColBits, b.desc, b.wbeg, b.ctas, mpv, st) && ring_rows > 0)
        fail(ABHSF_ERROR_UNSUPPORTED, "batch too large for the ring kernel's per-CTA counters");
    if (b.ctas > 0) {
        // time the variants with every matrix reading one zero x and writing one scratch y
        int64_t mx = 1, my = 1;
        for (const abhsf_matrix* a : b.mats) {
            mx = std::max(mx, a->n);
            my = std::max(my, a->m);
        }
        dbuf<double> x(mx), y(my);
        ABHSF_CUDA(cudaMemsetAsync(x.get(), 0, mx * sizeof(double), st));
        ABHSF_CUDA(cudaMemsetAsync(y.get(), 0, my * sizeof(double), st));
        std::vector<const double*> xs(b.mats.size(), x.get());
        std::vector<double*> ys(b.mats.size(), y.get());
        dbuf<const double*> xs_d(xs.size());
        dbuf<double*> ys_d(ys.size());
        ABHSF_CUDA(cudaMemcpyAsync(xs_d.get(), xs.data(), xs.size() * sizeof(double*), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(ys_d.get(), ys.data(), ys.size() * sizeof(double*), cudaMemcpyHostToDevice, st));
        int layout = 0, bulk = 0;
        if (!forced_variant(layout, bulk))
            time_variants(
                [&](int tm, int bk) {
                    b.layout = tm;
                    b.bulk = bk;
                    batch_launch(b, xs_d.get(), ys_d.get(), st, true);
                },
                b.s, st, layout, bulk);
        b.layout = layout;
        b.bulk = bulk;
        ABHSF_CUDA(cudaMemsetAsync(b.dev_status.get(), 0, sizeof(int), st));
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

void batch_spmv(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st)
{
    std::lock_guard<std::mutex> lock(b.dc_mu);
    batch_stream_begin(b, xs, ys, st);  // the chains, beside the rest
    if (b.ctas > 0)
        batch_launch(b, xs, ys, st, false);
    batch_stream_end(b, xs, ys, st);
}



bool spmv_f64_ring(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (!a.ring_ready || a.value_type != ABHSF_VALUE_F64)
        return false;
    std::lock_guard<std::mutex> lock(a.dc_mu);
    const dc_plan p = plan_of(a);
    slices_begin(a, p, x, 1, y, 1, st);  // the chains, beside the rest
    if (a.ring_warps) {
        if (a.s == 32)
            launch_ring<32, 1, ABHSF_VALUE_F64>(a, x, 1, y, 1, st);
        else
            launch_ring<64, 1, ABHSF_VALUE_F64>(a, x, 1, y, 1, st);
    }
    slices_end(a, p, x, 1, y, 1, st);
    return true;
}

void spmv_f32_dispatch(const abhsf_matrix& a, const float* x, float* y, cudaStream_t st)
{
    if (a.value_type == ABHSF_VALUE_F64)
        fail(ABHSF_ERROR_INVALID_VALUE, "the f32 SpMV needs a matrix stored as f32 or bf16");
    if (!a.ring_ready) {
        spmv_f32_seq(a, x, y, st);  // block sizes 16, 128, 256 (slices beside it), or no ring schedule
        return;
    }
    std::lock_guard<std::mutex> lock(a.dc_mu);
    const dc_plan p = plan_of(a);
    slices_begin(a, p, x, 1, y, 1, st);
    if (a.ring_warps) {
        if (a.value_type == ABHSF_VALUE_F32) {
            if (a.s == 32)
                launch_ring<32, 1, ABHSF_VALUE_F32>(a, x, 1, y, 1, st);
            else
                launch_ring<64, 1, ABHSF_VALUE_F32>(a, x, 1, y, 1, st);
        } else {
            if (a.s == 32)
                launch_ring<32, 1, ABHSF_VALUE_BF16>(a, x, 1, y, 1, st);
            else
                launch_ring<64, 1, ABHSF_VALUE_BF16>(a, x, 1, y, 1, st);
        }
    }
    slices_end(a, p, x, 1, y, 1, st);
}

bool spmv_f64_ring_host(abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    constexpr int kChunks = kHostChunks;
    if (!a.ring_ready || a.value_type != ABHSF_VALUE_F64 || a.sum_order != ABHSF_SUM_REFERENCE ||
        a.M < 4 * kChunks || a.m < (int64_t(1) << 20))
        return false;  // small matrices: one copy each way is as fast
    if (!a.host_ready) {
        a.host_chunks.clear();
        a.host_chunks.resize(kChunks);
        for (int c = 0; c < kChunks; ++c) {
            auto& ch = a.host_chunks[c];
            ch.brow0 = a.M * c / kChunks;
            ch.brow1 = a.M * (c + 1) / kChunks;
            int mpv = 0;
            if (a.ring_warps == 0 ||
                !build_ring_schedule({&a}, 32, ch.desc, ch.wbeg, ch.ctas, mpv, st, ch.brow0, ch.brow1))
                ch.ctas = 0;  // no ring tiles in these block rows
            deal_slices({&a}, ch.dc_sched, ch.dc_wbeg, ch.dc_warps, st, ch.brow0, ch.brow1, kDealSliced);
            deal_slices({&a}, ch.dc_csched, ch.dc_cwbeg, ch.dc_cwarps, st, ch.brow0, ch.brow1, kDealChains);
        }
        if (!a.host_in)
            ABHSF_CUDA(cudaStreamCreateWithFlags(&a.host_in, cudaStreamNonBlocking));
        if (!a.host_out)
            ABHSF_CUDA(cudaStreamCreateWithFlags(&a.host_out, cudaStreamNonBlocking));
        while (a.host_events.size() < 2 * kChunks + 2) {  // the matrix destroys what was created
            cudaEvent_t e = nullptr;
            ABHSF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            a.host_events.push_back(e);
        }
        a.host_ready = true;
    }
    cudaEvent_t* ev = a.host_events.data();  // [0] start, [1..C] y chunk in, [C+1..2C] chunk summed, [2C+1] end
    double* xs = a.x_stage.get();
    double* ys = a.y_stage.get();
    ABHSF_CUDA(cudaEventRecord(ev[0], st));  // after the caller's earlier work on st
    ABHSF_CUDA(cudaStreamWaitEvent(a.host_in, ev[0], 0));
    ABHSF_CUDA(cudaMemcpyAsync(xs, x, a.n * sizeof(double), cudaMemcpyHostToDevice, a.host_in));
    for (int c = 0; c < kChunks; ++c) {
        const auto& ch = a.host_chunks[c];
        const int64_t r0 = ch.brow0 * a.s, r1 = std::min(ch.brow1 * a.s, a.m);
        ABHSF_CUDA(cudaMemcpyAsync(ys + r0, y + r0, (r1 - r0) * sizeof(double), cudaMemcpyHostToDevice, a.host_in));
        ABHSF_CUDA(cudaEventRecord(ev[1 + c], a.host_in));
    }
    std::lock_guard<std::mutex> lock(a.dc_mu);
    for (int c = 0; c < kChunks; ++c) {
        const auto& ch = a.host_chunks[c];
        ABHSF_CUDA(cudaStreamWaitEvent(st, ev[1 + c], 0));
        dc_plan p;
        p.sched = ch.dc_sched.get();
        p.wbeg = ch.dc_wbeg.get();
        p.warps = ch.dc_warps;
        p.csched = ch.dc_csched.get();
        p.cwbeg = ch.dc_cwbeg.get();
        p.cwarps = ch.dc_cwarps;
        slices_begin(a, p, xs, 1, ys, 1, st);
        if (ch.ctas > 0) {
            if (a.s == 32)
                launch_ring<32, 1, ABHSF_VALUE_F64>(a, xs, 1, ys, 1, st, false, ch.desc.get(), ch.wbeg.get(), ch.ctas);
            else
                launch_ring<64, 1, ABHSF_VALUE_F64>(a, xs, 1, ys, 1, st, false, ch.desc.get(), ch.wbeg.get(), ch.ctas);
        }
        slices_end(a, p, xs, 1, ys, 1, st);
        ABHSF_CUDA(cudaEventRecord(ev[1 + kChunks + c], st));
    }
    for (int c = 0; c < kChunks; ++c) {
        const auto& ch = a.host_chunks[c];
        const int64_t r0 = ch.brow0 * a.s, r1 = std::min(ch.brow1 * a.s, a.m);
        ABHSF_CUDA(cudaStreamWaitEvent(a.host_out, ev[1 + kChunks + c], 0));
        ABHSF_CUDA(cudaMemcpyAsync(y + r0, ys + r0, (r1 - r0) * sizeof(double), cudaMemcpyDeviceToHost, a.host_out));
    }
    ABHSF_CUDA(cudaEventRecord(ev[2 * kChunks + 1], a.host_out));
    ABHSF_CUDA(cudaStreamWaitEvent(st, ev[2 * kChunks + 1], 0));
    return true;
}

void spmm_staged(const abhsf_matrix& a, int kt, const uint32_t* rows, int64_t nrows, const double* X, int64_t ldx,
                 double* Y, int64_t ldy, cudaStream_t st)
{
    // 16 columns: 4 a warp, so that a CTA keeps as many warps as at 32 (tiled
    // mixture, 16 columns: 0.76 ms with 8 a warp, 0.75 with 4).  Two rows a
    // lane (RPL = 2, each x row read once for the 64 rows) measured 1.31 ms
    // at 32 columns against 1.07 with one: fewer warps for the same stages.
    if (a.s == 32) {
        kt == 32 ? launch_staged<32, 32, 8, 1>(a, rows, nrows, X, ldx, Y, ldy, st)
                 : launch_staged<32, 16, 4, 1>(a, rows, nrows, X, ldx, Y, ldy, st);
    } else {
        kt == 32 ? launch_staged<64, 32, 8, 1>(a, rows, nrows, X, ldx, Y, ldy, st)
                 : launch_staged<64, 16, 4, 1>(a, rows, nrows, X, ldx, Y, ldy, st);
    }
}

bool spmm_f64_ring(const abhsf_matrix& a, int k, const double* X, int64_t ldx, double* Y, int64_t ldy,
                   cudaStream_t st)
{
    if (!a.ring_ready || a.value_type != ABHSF_VALUE_F64)
        return false;
    std::lock_guard<std::mutex> lock(a.dc_mu);
    const dc_plan p = plan_of(a);
    if (a.ring_warps) {
        if (a.s == 32)
            spmm_ring<32>(a, k, X, ldx, Y, ldy, st);
        else
            spmm_ring<64>(a, k, X, ldx, Y, ldy, st);
    }
    for (int j = 0; j < k;) {  // the slice rows, up to 32 columns a pass
        int cols = 32;
        while (cols > k - j)
            cols /= 2;
        slices_begin(a, p, X + j, ldx, Y + j, ldy, st, cols);
        slices_end(a, p, X + j, ldx, Y + j, ldy, st, cols);
        j += cols;
    }
    return true;
}

}  // namespace abhsf

extern "C" abhsf_status abhsf_test_ring_variant(abhsf_matrix* a, int32_t set, int32_t* layout, int32_t* bulk)
{
    return abhsf::guarded([&] {
        if (!a || !layout || !bulk)
            abhsf::fail(ABHSF_ERROR_INVALID_VALUE, "NULL argument");
        if (set) {
            if (*layout < 0 || *layout >= abhsf::kLayouts || (*bulk != 0 && *bulk != 1))
                abhsf::fail(ABHSF_ERROR_INVALID_VALUE, "layout 0 .. 3, bulk 0 or 1");
            a->ring_layout = *layout;
            a->ring_bulk = *bulk;
        }
        *layout = a->ring_warps ? a->ring_layout : -1;
        *bulk = a->ring_bulk;
    });
}

extern "C" void abhsf_test_set_hooks(int64_t drop_desc, uint32_t spin_limit)
{
    abhsf::g_drop_desc = drop_desc < 0 ? -1 : drop_desc;
    abhsf::g_spin_limit = spin_limit;
}

extern "C" int64_t abhsf_test_device_allocations(void) { return abhsf::dbuf_allocations().load(); }
