// spmm_stage.cuh -- staging one tile for the one-pass SpMM kernels (FP64):
// the tile's S x K block of X, its payload and its values, brought into a
// shared-memory stage by cp.async (16 bytes a copy) from all threads of the
// CTA.  A stage is the X block (S rows of K doubles) followed by the payload
// and then the values, starting at the 16-byte granule that holds the first
// value (the value's index in that granule is vo & 1).
#pragma once

#include "common.cuh"

namespace abhsf {
namespace stage {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(uint32_t dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// every group but the last committed one has landed (for this thread's copies)
__device__ __forceinline__ void wait_all_but_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int S, int K>
constexpr int x_block_bytes()
{
    return S * K * 8;
}

// Tile t into a stage by NT threads: X's rows c0 .. min(c0 + S, n) - 1 (the
// others are never read: no element lies past n, and a dense tile's padding
// holds zeros, which the sums skip), the payload (16-byte multiples at
// 16-byte offsets), the values (the value array has 16 bytes of padding past
// its end).  X and ldx: 16-byte aligned rows.
template <int S, int K, int NT>
__device__ __forceinline__ void tile(const tiles_view& A, const double* X, int64_t ldx, int64_t t, uint8_t* dst,
                                     int tid)
{
    constexpr int CPR = K * 8 / 16;  // 16-byte pieces of an X row
    const int64_t c0 = (int64_t)A.tile_col[t] * S;
    const int xr = A.n - c0 < S ? (int)(A.n - c0) : S;
    const uint32_t xb = smem_u32(dst);
    for (int i = tid; i < xr * CPR; i += NT) {
        const int r = i / CPR, q = i - r * CPR;
        cp16(xb + (uint32_t)(r * K * 8 + q * 16), X + (c0 + r) * ldx + 2 * q);
    }
    const int64_t io = A.tile_idx_off[t];
    const int pb = (int)(A.tile_idx_off[t + 1] - io);
    const uint32_t ab = xb + x_block_bytes<S, K>();
    for (int i = tid; i < pb / 16; i += NT)
        cp16(ab + 16 * i, A.payload + io + 16 * i);
    const int64_t vo = A.tile_val_off[t], nv = A.tile_val_off[t + 1] - vo;
    const int64_t v0 = vo & ~int64_t(1);
    const int pieces = (int)((vo - v0 + nv + 1) / 2);
    const double* V = static_cast<const double*>(A.values);
    for (int i = tid; i < pieces; i += NT)
        cp16(ab + pb + 16 * i, V + v0 + 2 * i);
}

// A tile's place in the format arrays, read one step before it is staged.
struct tile_meta {
    int64_t io, vo;  // payload byte offset, first value
    int pb, nv;      // payload bytes, stored values
    uint32_t col;    // block column
    int sch;
};

__device__ __forceinline__ tile_meta meta_of(const tiles_view& A, int64_t t)
{
    tile_meta m;
    m.io = A.tile_idx_off[t];
    m.pb = (int)(A.tile_idx_off[t + 1] - m.io);
    m.vo = A.tile_val_off[t];
    m.nv = (int)(A.tile_val_off[t + 1] - m.vo);
    m.col = A.tile_col[t];
    m.sch = A.tile_scheme[t];
    return m;
}

// tile() with the tile's offsets already at hand.
template <int S, int K, int NT>
__device__ __forceinline__ void tile(const tiles_view& A, const double* X, int64_t ldx, const tile_meta& m,
                                     uint8_t* dst, int tid)
{
    constexpr int CPR = K * 8 / 16;
    const int64_t c0 = (int64_t)m.col * S;
    const int xr = A.n - c0 < S ? (int)(A.n - c0) : S;
    const uint32_t xb = smem_u32(dst);
    for (int i = tid; i < xr * CPR; i += NT) {
        const int r = i / CPR, q = i - r * CPR;
        cp16(xb + (uint32_t)(r * K * 8 + q * 16), X + (c0 + r) * ldx + 2 * q);
    }
    const uint32_t ab = xb + x_block_bytes<S, K>();
    for (int i = tid; i < m.pb / 16; i += NT)
        cp16(ab + 16 * i, A.payload + m.io + 16 * i);
    const int64_t v0 = m.vo & ~int64_t(1);
    const int pieces = (int)((m.vo - v0 + m.nv + 1) / 2);
    const double* V = static_cast<const double*>(A.values);
    for (int i = tid; i < pieces; i += NT)
        cp16(ab + m.pb + 16 * i, V + v0 + 2 * i);
}

}  // namespace stage
}  // namespace abhsf
