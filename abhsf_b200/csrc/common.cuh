// common.cuh -- internal definitions shared by the ABHSF sm_100a sources.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "abhsf/abhsf_cost.h"
#include "abhsf/abhsf_gpu.h"

namespace abhsf {

// Thrown inside the library, caught at every extern "C" boundary.
struct error {
    abhsf_status status;
    std::string msg;
};

[[noreturn]] inline void fail(abhsf_status s, std::string msg) { throw error{s, std::move(msg)}; }

inline void cuda_check(cudaError_t e, const char* what)
{
    if (e == cudaSuccess)
        return;
    cudaGetLastError();  // clear a non-sticky error
    if (e == cudaErrorMemoryAllocation)
        fail(ABHSF_ERROR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    fail(ABHSF_ERROR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define ABHSF_CUDA(call) ::abhsf::cuda_check((call), #call)

void set_last_error(const std::string& msg);
void clear_last_error();

// Runs f and converts exceptions to a status; the message goes to the
// thread's last-error string.
template <typename F>
abhsf_status guarded(F&& f) noexcept
{
    try {
        f();
        clear_last_error();
        return ABHSF_SUCCESS;
    } catch (const error& e) {
        set_last_error(e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return ABHSF_ERROR_OUT_OF_MEMORY;
    } catch (...) {
        set_last_error("unknown internal error");
        return ABHSF_ERROR_CUDA;
    }
}

// Device allocations made by dbuf since the library was loaded (read by the
// test hook abhsf_test_device_allocations).
inline std::atomic<int64_t>& dbuf_allocations()
{
    static std::atomic<int64_t> count{0};
    return count;
}

// Owning device allocation (cudaMalloc / cudaFree).
template <typename T>
class dbuf {
  public:
    dbuf() = default;
    explicit dbuf(size_t count) { alloc(count); }
    ~dbuf() { reset(); }
    dbuf(const dbuf&) = delete;
    dbuf& operator=(const dbuf&) = delete;
    dbuf(dbuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    dbuf& operator=(dbuf&& o) noexcept
    {
        if (this != &o) {
            reset();
            p_ = o.p_; n_ = o.n_;
            o.p_ = nullptr; o.n_ = 0;
        }
        return *this;
    }
    void alloc(size_t count)
    {
        reset();
        if (count == 0)
            count = 1;
        ABHSF_CUDA(cudaMalloc(reinterpret_cast<void**>(&p_), count * sizeof(T)));
        dbuf_allocations().fetch_add(1, std::memory_order_relaxed);
        n_ = count;
    }
    void reset()
    {
        if (p_)
            cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* release() { T* p = p_; p_ = nullptr; n_ = 0; return p; }
    T* get() const { return p_; }
    size_t size() const { return n_; }

  private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

// Plain view of a built matrix passed to kernels by value.
struct tiles_view {
    int64_t m, n, M;
    const int64_t* brow_ptr;
    const uint32_t* tile_col;
    const uint32_t* tile_nnz;
    const uint8_t* tile_scheme;
    const int64_t* tile_val_off;
    const int64_t* tile_idx_off;
    const uint8_t* payload;
    const void* values;
};

// Mean elements per tile up to which a block row goes to the delta-coded
// row slices unless abhsf_build_opts.slice_tile_nnz says otherwise.
constexpr float kSliceTileNnzDefault = 32.f;

inline int log2_exact(int64_t s)
{
    int lg = 0;
    while ((int64_t(1) << lg) < s)
        ++lg;
    return (int64_t(1) << lg) == s ? lg : -1;
}

inline int bit_length(uint64_t v)
{
    int b = 0;
    while (b < 64 && (v >> b) != 0)
        ++b;
    return b;
}

inline int64_t pad16(int64_t b) { return (b + 15) & ~int64_t(15); }

inline size_t value_size(int vt) { return vt == ABHSF_VALUE_F64 ? 8 : vt == ABHSF_VALUE_F32 ? 4 : 2; }

__host__ __device__ inline int64_t tile_payload_bytes(int scheme, int64_t s, int64_t nnz)
{
    switch (scheme) {
    case ABHSF_SCHEME_COO: return (2 * nnz + 15) & ~int64_t(15);
    case ABHSF_SCHEME_CSR: return (2 * s + nnz + 15) & ~int64_t(15);
    case ABHSF_SCHEME_BITMAP: return (s * s / 8 + 15) & ~int64_t(15);
    default: return 0;
    }
}

}  // namespace abhsf

// The handle behind abhsf_matrix*.
struct abhsf_matrix {
    int64_t m = 0, n = 0, nnz = 0;
    int32_t s = 0, lg = 0, value_type = ABHSF_VALUE_F64, matrix_type = ABHSF_MATRIX_REAL;
    int64_t M = 0, N = 0, T = 0, n_values = 0, payload_bytes = 0;
    int device = 0;
    abhsf::dbuf<int64_t> brow_ptr;
    abhsf::dbuf<uint32_t> tile_col;
    abhsf::dbuf<uint32_t> tile_nnz;
    abhsf::dbuf<uint8_t> tile_scheme;
    abhsf::dbuf<int64_t> tile_val_off;
    abhsf::dbuf<int64_t> tile_idx_off;
    abhsf::dbuf<uint8_t> payload;
    abhsf::dbuf<uint8_t> values;  // n_values * value_size(value_type) bytes (+16 padding)
    abhsf_stats stats{};
    int32_t sum_order = ABHSF_SUM_REFERENCE;
    // tree-order SpMV: non-empty block rows and the work counter of its persistent warps
    abhsf::dbuf<uint32_t> tree_rows;
    int64_t tree_nrows = 0;
    abhsf::dbuf<unsigned int> tree_counter;
    int tree_ctas = 0;
    // reference-order SpMV, s = 32 / 64: every CTA's tile descriptors and their ranges
    abhsf::dbuf<uint8_t> ring_desc;
    abhsf::dbuf<int64_t> ring_wbeg;
    int ring_max_pv = 0;  // largest payload + values bytes of one tile (picks the SpMM pass width)
    int ring_warps = 0;  // CTAs of the ring kernel; 0: the streaming kernel serves this matrix
    int ring_layout = 0;  // consumer layout of its single-right-hand-side launches (timed at build)
    int ring_bulk = 0;   // x / y blocks as bulk copies (timed at build)
    bool ring_ready = false;  // the ring kernel and the slice kernel together serve this matrix
    bool dc_beside_ring = false;  // the sliced rows run on dc_side beside the ring kernel (one CTA an SM)
    // delta-coded row slices of the hypersparse block rows (spmv_stream.cu)
    struct dc_slice_host {
        int64_t base = 0;   // first slot of its words and values
        int64_t meta = 0;   // sliced: first of its 32 lane records; chain: the row within the block row
        uint32_t brow = 0, steps = 0, lanes = 0;
        bool chain = false;
    };
    std::vector<dc_slice_host> dc_host;  // block rows ascending; per block row its chains, then its sliced rows
    std::vector<uint8_t> dc_tree_flag;   // per non-empty block row (tree_rows order): served by the slices
    abhsf::dbuf<uint32_t> dc_words;      // one word per slot (delta-coded columns)
    abhsf::dbuf<uint8_t> dc_vals;        // the values in slot order
    abhsf::dbuf<uint32_t> dc_lane;       // lane records: row << 24 | length
    abhsf::dbuf<uint8_t> dc_sched;       // the matrix's own launch: sliced rows in warp order
    abhsf::dbuf<int64_t> dc_wbeg;
    int dc_warps = 0;
    abhsf::dbuf<uint32_t> seq_rows;      // the non-empty block rows outside the slices (where there are slices):
    int64_t seq_nrows = 0;               // the streaming kernel's (s = 16 / 128 / 256) and the wide SpMM's
    int64_t wide_cap = 0;                // wide SpMM (spmm_wide.cu): bytes of a tile's payload and values (0: none)
    abhsf::dbuf<uint8_t> dc_csched;      // ... and its chains, launched on dc_side beside the others
    abhsf::dbuf<int64_t> dc_cwbeg;
    int dc_cwarps = 0;
    cudaStream_t dc_side = nullptr;      // created with the first chain; forked from the caller's stream
    cudaEvent_t dc_fork = nullptr, dc_join = nullptr;
    mutable std::mutex dc_mu;            // one fork / join sequence at a time
    int64_t dc_elements = 0, dc_rows = 0, dc_slots = 0, dc_lane_records = 0;
    float dc_avg = 0.f;                  // largest mean elements per tile of a slice block row (0: none)
    abhsf::dbuf<int> dev_status;  // ABHSF_DEVSTAT_* bits set by kernels
    // staging for abhsf_spmv_host
    abhsf::dbuf<double> x_stage, y_stage;
    // abhsf_spmv_host's pipeline (ring kernel): the block rows in chunks, each
    // with its own schedule, so that copying y in and out overlaps the sums
    struct host_chunk {
        int64_t brow0 = 0, brow1 = 0;  // block rows [brow0, brow1)
        abhsf::dbuf<uint8_t> desc;
        abhsf::dbuf<int64_t> wbeg;
        int ctas = 0;
        abhsf::dbuf<uint8_t> dc_sched;  // the chunk's sliced rows and chains
        abhsf::dbuf<int64_t> dc_wbeg;
        int dc_warps = 0;
        abhsf::dbuf<uint8_t> dc_csched;
        abhsf::dbuf<int64_t> dc_cwbeg;
        int dc_cwarps = 0;
    };
    std::vector<host_chunk> host_chunks;
    bool host_ready = false;
    cudaStream_t host_in = nullptr, host_out = nullptr;
    std::vector<cudaEvent_t> host_events;

    abhsf_matrix() = default;
    abhsf_matrix(const abhsf_matrix&) = delete;
    abhsf_matrix& operator=(const abhsf_matrix&) = delete;
    ~abhsf_matrix()
    {
        if (dc_fork)
            cudaEventDestroy(dc_fork);
        if (dc_join)
            cudaEventDestroy(dc_join);
        if (dc_side)
            cudaStreamDestroy(dc_side);
        for (cudaEvent_t e : host_events)
            cudaEventDestroy(e);
        if (host_in)
            cudaStreamDestroy(host_in);
        if (host_out)
            cudaStreamDestroy(host_out);
    }

    abhsf::tiles_view view() const
    {
        return abhsf::tiles_view{m, n, M, brow_ptr.get(), tile_col.get(), tile_nnz.get(), tile_scheme.get(),
                                 tile_val_off.get(), tile_idx_off.get(), payload.get(), values.get()};
    }
};

// Several f64 matrices of one block size (32 or 64) multiplied by one launch
// of the ring kernel (abhsf_batch_*).  The matrices belong to the caller and
// must outlive the batch.
namespace abhsf {
constexpr int kBatchColBits = 20;  // descriptor column = block column | matrix index << 20
constexpr int kBatchMax = 1 << (32 - kBatchColBits);
}  // namespace abhsf

struct abhsf_batch {
    std::vector<const abhsf_matrix*> mats;
    int32_t s = 0;
    int device = 0;
    int64_t total_tiles = 0;
    abhsf::dbuf<uint8_t> desc;   // every CTA's tile descriptors
    abhsf::dbuf<int64_t> wbeg;   // each CTA's range in desc
    abhsf::dbuf<uint8_t> table;  // per matrix: arrays and shape
    abhsf::dbuf<int> dev_status;
    // block sizes 16 / 128 / 256: the streaming kernel over every matrix's
    // block rows outside the slices, one launch (spmv_seq.cu)
    abhsf::dbuf<uint8_t> seq_mats;  // per matrix: its tiles_view
    abhsf::dbuf<uint2> seq_items;   // (matrix, block row), heaviest ranks first
    int64_t seq_nitems = 0;
    abhsf::dbuf<unsigned int> seq_counter;
    int ctas = 0;
    int layout = 0;  // consumer layout of the ring kernel (timed at creation)
    int bulk = 0;   // x / y blocks as bulk copies (timed at creation)
    // the matrices' delta-coded row slices, one launch (spmv_stream.cu)
    abhsf::dbuf<uint8_t> dc_table;
    abhsf::dbuf<uint8_t> dc_sched;
    abhsf::dbuf<int64_t> dc_wbeg;
    int dc_warps = 0;
    abhsf::dbuf<uint8_t> dc_csched;
    abhsf::dbuf<int64_t> dc_cwbeg;
    int dc_cwarps = 0;
    cudaStream_t dc_side = nullptr;
    cudaEvent_t dc_fork = nullptr, dc_join = nullptr;
    mutable std::mutex dc_mu;

    abhsf_batch() = default;
    abhsf_batch(const abhsf_batch&) = delete;
    abhsf_batch& operator=(const abhsf_batch&) = delete;
    ~abhsf_batch()
    {
        if (dc_fork)
            cudaEventDestroy(dc_fork);
        if (dc_join)
            cudaEventDestroy(dc_join);
        if (dc_side)
            cudaStreamDestroy(dc_side);
    }
};
