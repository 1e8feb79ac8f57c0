// capi.cu -- the extern "C" boundary declared in include/abhsf/abhsf_gpu.h.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {

namespace {
thread_local std::string g_last_error;
}

void spmv_dispatch(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st)
{
    if (a.sum_order == ABHSF_SUM_REFERENCE) {
        if (!spmv_f64_ring(a, x, y, st))
            spmv_f64_seq(a, x, y, st);
    }
    else
        spmv_f64(a, x, y, st);
}

// Y += A X, k columns.  The reference order with k a multiple of 16 (block
// sizes 16, 32, 64; X and Y 16-byte aligned with even leading dimensions)
// runs the wide kernel, 16 or 32 columns a pass over A; for block sizes 32 /
// 64 otherwise the ring kernel with up to 8 columns a pass; otherwise each
// column is gathered into a contiguous vector, multiplied by the SpMV kernels
// and scattered back, so column j is bitwise the SpMV of column j in every
// case.
void spmm_dispatch(const abhsf_matrix& a, int k, const double* X, int64_t ldx, double* Y, int64_t ldy,
                   cudaStream_t st)
{
    if (k == 0 || a.m == 0 || a.T == 0)
        return;
    if (a.sum_order == ABHSF_SUM_REFERENCE && (spmm_f64_wide(a, k, X, ldx, Y, ldy, st) ||
                                               spmm_f64_ring(a, k, X, ldx, Y, ldy, st)))
        return;
    if (k == 1 && ldx == 1 && ldy == 1) {
        spmv_dispatch(a, X, Y, st);
        return;
    }
    dbuf<double> xc(a.n), yc(a.m);
    for (int j = 0; j < k; ++j) {
        ABHSF_CUDA(cudaMemcpy2DAsync(xc.get(), sizeof(double), X + j, ldx * sizeof(double), sizeof(double), a.n,
                                     cudaMemcpyDeviceToDevice, st));
        ABHSF_CUDA(cudaMemcpy2DAsync(yc.get(), sizeof(double), Y + j, ldy * sizeof(double), sizeof(double), a.m,
                                     cudaMemcpyDeviceToDevice, st));
        spmv_dispatch(a, xc.get(), yc.get(), st);
        ABHSF_CUDA(cudaMemcpy2DAsync(Y + j, ldy * sizeof(double), yc.get(), sizeof(double), sizeof(double), a.m,
                                     cudaMemcpyDeviceToDevice, st));
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));  // before the column buffers are freed
}

void set_last_error(const std::string& msg) { g_last_error = msg; }
void clear_last_error() { g_last_error.clear(); }

}  // namespace abhsf

using abhsf::fail;
using abhsf::guarded;

extern "C" {

int32_t abhsf_abi_version(void) { return ABHSF_ABI_VERSION; }

const char* abhsf_last_error_string(void) { return abhsf::g_last_error.c_str(); }

void abhsf_build_opts_default(abhsf_build_opts* o)
{
    if (!o)
        return;
    o->block_size = 64;
    o->value_type = ABHSF_VALUE_F64;
    o->allow_csr = 1;
    o->matrix_type = ABHSF_MATRIX_REAL;
    o->forced_scheme = -1;
    o->inputs_on_device = 0;
    o->sum_order = ABHSF_SUM_REFERENCE;
    o->bits_per_value = 0;
    o->selector = ABHSF_SELECT_MINBSS;
    o->slice_tile_nnz = 0;
    o->selector_model = nullptr;
}

abhsf_status abhsf_build(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m,
                         int64_t n, const abhsf_build_opts* opts, abhsf_stream_t stream, abhsf_matrix** out)
{
    return guarded([&] {
        if (!out)
            fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
        *out = nullptr;
        abhsf_build_opts o;
        abhsf_build_opts_default(&o);
        if (opts)
            o = *opts;
        if (o.block_size == 0) {
            const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
            if (o.selector == ABHSF_SELECT_MINBSS) {
                uint64_t bits[abhsf::kNumBlockSizes];
                abhsf::block_size_storage(rows, cols, nnz, m, n, o, st, bits);
                o.block_size = abhsf::select_block_size(bits);
            } else if (o.selector == ABHSF_SELECT_LEARNED || o.selector == ABHSF_SELECT_LEARNED_TIME) {
                float f[ABHSF_FEATURES];
                abhsf::selector_features(rows, cols, nnz, m, n, o.inputs_on_device != 0, st, f);
                const float* model = o.selector_model ? o.selector_model
                                     : o.selector == ABHSF_SELECT_LEARNED_TIME ? abhsf::builtin_time_model()
                                                                               : nullptr;
                o.block_size = abhsf::mlp_predict(model, f, st);
            } else if (o.selector == ABHSF_SELECT_AUTOTUNE) {
                float ms[abhsf::kNumBlockSizes];
                int best = 0;
                std::unique_ptr<abhsf_matrix> a;
                abhsf::autotune(rows, cols, vals, nnz, m, n, o, 0, 10, st, ms, &best, &a);
                *out = a.release();
                return;
            } else {
                fail(ABHSF_ERROR_INVALID_VALUE, "selector out of range");
            }
        }
        auto a = std::make_unique<abhsf_matrix>();
        abhsf::build_matrix(rows, cols, vals, nnz, m, n, o, reinterpret_cast<cudaStream_t>(stream), *a);
        *out = a.release();
    });
}

abhsf_status abhsf_spmv_kernels(const abhsf_matrix* a, int32_t* kernels)
{
    return guarded([&] {
        if (!a || !kernels)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle and kernels must be non-NULL");
        int k = 0;
        if (a->T > 0) {
            if (a->sum_order != ABHSF_SUM_REFERENCE)
                k = 1;  // the tree-order kernel
            else {
                const bool seq = !a->ring_ready && (a->s == 32 || a->s == 64 ? true : a->seq_nrows > 0 || a->dc_rows == 0);
                k = (a->ring_ready ? (a->ring_warps > 0 ? 1 : 0) : (seq ? 1 : 0)) + (a->dc_warps > 0 ? 1 : 0) +
                    (a->dc_cwarps > 0 ? 1 : 0);
            }
        }
        *kernels = k;
    });
}

abhsf_status abhsf_spmv(const abhsf_matrix* a, const double* x, double* y, abhsf_stream_t stream)
{
    return guarded([&] {
        if (!a)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        if (a->value_type != ABHSF_VALUE_F64)
            fail(ABHSF_ERROR_INVALID_VALUE, "abhsf_spmv needs a matrix stored as f64");
        if ((!x && a->n) || (!y && a->m))
            fail(ABHSF_ERROR_INVALID_VALUE, "x and y must be non-NULL");
        if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 7)
            fail(ABHSF_ERROR_INVALID_VALUE, "x and y must be 8-byte aligned");
        abhsf::spmv_dispatch(*a, x, y, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_spmv_f32(const abhsf_matrix* a, const float* x, float* y, abhsf_stream_t stream)
{
    return guarded([&] {
        if (!a)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        if (a->value_type == ABHSF_VALUE_F64)
            fail(ABHSF_ERROR_INVALID_VALUE, "abhsf_spmv_f32 needs a matrix stored as f32 or bf16");
        if ((!x && a->n) || (!y && a->m))
            fail(ABHSF_ERROR_INVALID_VALUE, "x and y must be non-NULL");
        if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 3)
            fail(ABHSF_ERROR_INVALID_VALUE, "x and y must be 4-byte aligned");
        if (a->m == 0 || a->T == 0)
            return;
        abhsf::spmv_f32_dispatch(*a, x, y, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_cg(const abhsf_matrix* a, const double* b, double* x, double rtol, int32_t max_iters,
                      abhsf_cg_info* info, abhsf_stream_t stream)
{
    return guarded([&] {
        if (!a || !info)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle and info must be non-NULL");
        if (a->value_type != ABHSF_VALUE_F64)
            fail(ABHSF_ERROR_INVALID_VALUE, "abhsf_cg needs a matrix stored as f64");
        if ((!b || !x) && a->n)
            fail(ABHSF_ERROR_INVALID_VALUE, "b and x must be non-NULL");
        if (!(rtol >= 0.0))
            fail(ABHSF_ERROR_INVALID_VALUE, "rtol must be >= 0");
        abhsf::cg_solve(*a, b, x, rtol, max_iters, info, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_cg_mixed(const abhsf_matrix* a64, const abhsf_matrix* a_lo, const double* b, double* x,
                            double rtol, int32_t max_iters, double update_factor, int32_t max_updates,
                            abhsf_cg_info* info, abhsf_stream_t stream)
{
    return guarded([&] {
        if (!a64 || !a_lo || !info)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handles and info must be non-NULL");
        if (a64->value_type != ABHSF_VALUE_F64 || a_lo->value_type == ABHSF_VALUE_F64)
            fail(ABHSF_ERROR_INVALID_VALUE, "abhsf_cg_mixed needs a64 stored as f64 and a_lo as f32 or bf16");
        if ((!b || !x) && a64->n)
            fail(ABHSF_ERROR_INVALID_VALUE, "b and x must be non-NULL");
        if (!(rtol >= 0.0) || !(update_factor > 0.0 && update_factor < 1.0))
            fail(ABHSF_ERROR_INVALID_VALUE, "rtol must be >= 0 and update_factor in (0, 1)");
        abhsf::cg_solve_mixed(*a64, *a_lo, b, x, rtol, max_iters, update_factor, max_updates, info,
                              reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_batch_create(const abhsf_matrix* const* mats, int32_t count, abhsf_stream_t stream,
                                abhsf_batch** out)
{
    return guarded([&] {
        if (!mats || !out || count <= 0)
            fail(ABHSF_ERROR_INVALID_VALUE, "mats and out must be non-NULL and count > 0");
        *out = nullptr;
        if (count > abhsf::kBatchMax)
            fail(ABHSF_ERROR_UNSUPPORTED, "a batch holds at most 4096 matrices");
        auto b = std::make_unique<abhsf_batch>();
        for (int32_t i = 0; i < count; ++i) {
            const abhsf_matrix* a = mats[i];
            if (!a)
                fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
            if (a->value_type != ABHSF_VALUE_F64)
                fail(ABHSF_ERROR_INVALID_VALUE, "batched matrices must be stored as f64");
            if (i > 0 && a->s != mats[0]->s)
                fail(ABHSF_ERROR_INVALID_VALUE, "batched matrices must share one block size");
            if ((a->s == 32 || a->s == 64) &&
                (a->N >= (int64_t(1) << abhsf::kBatchColBits) || a->M >= (int64_t(1) << 30)))
                fail(ABHSF_ERROR_UNSUPPORTED, "a batched matrix has too many block rows or columns");
            b->mats.push_back(a);
            b->total_tiles += a->T;
        }
        b->s = mats[0]->s;
        ABHSF_CUDA(cudaGetDevice(&b->device));
        if (b->s == 32 || b->s == 64)
            abhsf::prepare_batch(*b, reinterpret_cast<cudaStream_t>(stream));
        else
            abhsf::prepare_batch_seq(*b, reinterpret_cast<cudaStream_t>(stream));
        *out = b.release();
    });
}

abhsf_status abhsf_batch_spmv(const abhsf_batch* b, const double* const* xs, double* const* ys,
                              abhsf_stream_t stream)
{
    return guarded([&] {
        if (!b)
            fail(ABHSF_ERROR_INVALID_VALUE, "batch handle is NULL");
        if (!xs || !ys)
            fail(ABHSF_ERROR_INVALID_VALUE, "xs and ys must be non-NULL device arrays");
        if (b->s == 32 || b->s == 64)
            abhsf::batch_spmv(*b, xs, ys, reinterpret_cast<cudaStream_t>(stream));
        else
            abhsf::batch_seq_spmv(*b, xs, ys, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_batch_kernels(const abhsf_batch* b, int32_t* kernels)
{
    return guarded([&] {
        if (!b || !kernels)
            fail(ABHSF_ERROR_INVALID_VALUE, "batch handle and kernels must be non-NULL");
        *kernels = (b->ctas > 0 ? 1 : 0) + (b->seq_nitems > 0 ? 1 : 0) + (b->dc_warps > 0 ? 1 : 0) +
                   (b->dc_cwarps > 0 ? 1 : 0);
    });
}

abhsf_status abhsf_batch_status(abhsf_batch* b, abhsf_stream_t stream, int32_t clear, int32_t* out)
{
    return guarded([&] {
        if (!b || !out)
            fail(ABHSF_ERROR_INVALID_VALUE, "batch handle and out must be non-NULL");
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        int v = 0;
        ABHSF_CUDA(cudaMemcpyAsync(&v, b->dev_status.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        if (clear)
            ABHSF_CUDA(cudaMemsetAsync(b->dev_status.get(), 0, sizeof(int), st));
        ABHSF_CUDA(cudaStreamSynchronize(st));
        *out = v;
    });
}

abhsf_status abhsf_batch_release(abhsf_batch* b)
{
    return guarded([&] { delete b; });
}

abhsf_status abhsf_spmm(const abhsf_matrix* a, int32_t k, const double* X, int64_t ldx, double* Y, int64_t ldy,
                        abhsf_stream_t stream)
{
    return guarded([&] {
        if (!a)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        if (a->value_type != ABHSF_VALUE_F64)
            fail(ABHSF_ERROR_INVALID_VALUE, "abhsf_spmm needs a matrix stored as f64");
        if (k < 0)
            fail(ABHSF_ERROR_INVALID_VALUE, "k must be >= 0");
        if (k == 0)
            return;
        if (ldx < k || ldy < k)
            fail(ABHSF_ERROR_INVALID_VALUE, "ldx and ldy must be >= k");
        if ((!X && a->n) || (!Y && a->m))
            fail(ABHSF_ERROR_INVALID_VALUE, "X and Y must be non-NULL");
        if ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(Y)) & 7)
            fail(ABHSF_ERROR_INVALID_VALUE, "X and Y must be 8-byte aligned");
        abhsf::spmm_dispatch(*a, k, X, ldx, Y, ldy, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_spmv_host(abhsf_matrix* a, const double* x, double* y, abhsf_stream_t stream)
{
    return guarded([&] {
        if (!a)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        if (a->value_type != ABHSF_VALUE_F64)
            fail(ABHSF_ERROR_INVALID_VALUE, "abhsf_spmv_host needs a matrix stored as f64");
        if ((!x && a->n) || (!y && a->m))
            fail(ABHSF_ERROR_INVALID_VALUE, "x and y must be non-NULL");
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        if (!a->x_stage.get() || a->x_stage.size() < (size_t)a->n)
            a->x_stage.alloc(a->n);
        if (!a->y_stage.get() || a->y_stage.size() < (size_t)a->m)
            a->y_stage.alloc(a->m);
        if (!abhsf::spmv_f64_ring_host(*a, x, y, st)) {
            ABHSF_CUDA(cudaMemcpyAsync(a->x_stage.get(), x, a->n * sizeof(double), cudaMemcpyHostToDevice, st));
            ABHSF_CUDA(cudaMemcpyAsync(a->y_stage.get(), y, a->m * sizeof(double), cudaMemcpyHostToDevice, st));
            abhsf::spmv_dispatch(*a, a->x_stage.get(), a->y_stage.get(), st);
            ABHSF_CUDA(cudaMemcpyAsync(y, a->y_stage.get(), a->m * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        ABHSF_CUDA(cudaStreamSynchronize(st));
    });
}

abhsf_status abhsf_device_status(abhsf_matrix* a, abhsf_stream_t stream, int32_t clear, int32_t* out)
{
    return guarded([&] {
        if (!a || !out)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle and out must be non-NULL");
        cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        int v = 0;
        ABHSF_CUDA(cudaMemcpyAsync(&v, a->dev_status.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
        if (clear)
            ABHSF_CUDA(cudaMemsetAsync(a->dev_status.get(), 0, sizeof(int), st));
        ABHSF_CUDA(cudaStreamSynchronize(st));
        *out = v;
    });
}

abhsf_status abhsf_release(abhsf_matrix* a)
{
    return guarded([&] { delete a; });
}

abhsf_status abhsf_stats_get(const abhsf_matrix* a, abhsf_stats* out)
{
    return guarded([&] {
        if (!a || !out)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle and out must be non-NULL");
        *out = a->stats;
    });
}

abhsf_status abhsf_export_host(const abhsf_matrix* a, int64_t* brow_ptr, uint32_t* tile_col, uint32_t* tile_nnz,
                               uint8_t* tile_scheme, int64_t* tile_val_off, int64_t* tile_idx_off, uint8_t* payload,
                               void* values)
{
    return guarded([&] {
        if (!a)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix handle is NULL");
        auto cp = [](void* dst, const void* src, size_t bytes) {
            if (dst && bytes)
                ABHSF_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        };
        cp(brow_ptr, a->brow_ptr.get(), (a->M + 1) * sizeof(int64_t));
        cp(tile_col, a->tile_col.get(), a->T * sizeof(uint32_t));
        cp(tile_nnz, a->tile_nnz.get(), a->T * sizeof(uint32_t));
        cp(tile_scheme, a->tile_scheme.get(), a->T);
        cp(tile_val_off, a->tile_val_off.get(), (a->T + 1) * sizeof(int64_t));
        cp(tile_idx_off, a->tile_idx_off.get(), (a->T + 1) * sizeof(int64_t));
        cp(payload, a->payload.get(), a->payload_bytes);
        cp(values, a->values.get(), a->n_values * abhsf::value_size(a->value_type));
    });
}

abhsf_status abhsf_block_histogram(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n,
                                   int32_t r, int32_t s, int32_t inputs_on_device, abhsf_stream_t stream,
                                   uint64_t* hist, int64_t hist_len, int64_t* blocks)
{
    return guarded([&] {
        abhsf::block_histogram(rows, cols, nnz, m, n, r, s, inputs_on_device != 0,
                               reinterpret_cast<cudaStream_t>(stream), hist, hist_len, blocks);
    });
}

abhsf_status abhsf_block_histogram_all(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n,
                                       int32_t inputs_on_device, abhsf_stream_t stream, uint64_t* hist,
                                       int64_t* blocks)
{
    return guarded([&] {
        abhsf::block_histogram_all(rows, cols, nnz, m, n, inputs_on_device != 0,
                                   reinterpret_cast<cudaStream_t>(stream), hist, blocks);
    });
}

abhsf_status abhsf_block_histogram_noalloc(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m,
                                           int64_t n, int32_t r, int32_t s, abhsf_stream_t stream, uint64_t* hist,
                                           int64_t hist_len, int64_t* blocks)
{
    return guarded([&] {
        abhsf::block_histogram_noalloc(rows, cols, nnz, m, n, r, s, reinterpret_cast<cudaStream_t>(stream), hist,
                                       hist_len, blocks);
    });
}

abhsf_status abhsf_block_size_storage(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n,
                                      const abhsf_build_opts* opts, abhsf_stream_t stream, uint64_t bits[5],
                                      int32_t* best)
{
    static_assert(abhsf::kNumBlockSizes == 5, "bits[5] in the header");
    return guarded([&] {
        if (!bits)
            fail(ABHSF_ERROR_INVALID_VALUE, "bits must be non-NULL");
        if (m <= 0 || n <= 0 || nnz < 0)
            fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
        abhsf_build_opts o;
        abhsf_build_opts_default(&o);
        if (opts)
            o = *opts;
        abhsf::block_size_storage(rows, cols, nnz, m, n, o, reinterpret_cast<cudaStream_t>(stream), bits);
        if (best)
            *best = abhsf::select_block_size(bits);
    });
}

abhsf_status abhsf_autotune(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m,
                            int64_t n, const abhsf_build_opts* opts, int32_t candidates, int32_t reps,
                            abhsf_stream_t stream, float ms[5], int32_t* best, abhsf_matrix** out)
{
    return guarded([&] {
        if (out)
            *out = nullptr;
        if (!ms || !best)
            fail(ABHSF_ERROR_INVALID_VALUE, "ms and best must be non-NULL");
        abhsf_build_opts o;
        abhsf_build_opts_default(&o);
        if (opts)
            o = *opts;
        std::unique_ptr<abhsf_matrix> a;
        int b = 0;
        abhsf::autotune(rows, cols, vals, nnz, m, n, o, candidates, reps, reinterpret_cast<cudaStream_t>(stream), ms,
                        &b, out ? &a : nullptr);
        *best = b;
        if (out)
            *out = a.release();
    });
}

abhsf_status abhsf_selector_features(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n,
                                     int32_t inputs_on_device, abhsf_stream_t stream, float out[12])
{
    static_assert(ABHSF_FEATURES == 12, "out[12] in the header");
    return guarded([&] {
        abhsf::selector_features(rows, cols, nnz, m, n, inputs_on_device != 0,
                                 reinterpret_cast<cudaStream_t>(stream), out);
    });
}

abhsf_status abhsf_selector_predict(const float* model, const float features[12], abhsf_stream_t stream,
                                    int32_t* block_size)
{
    return guarded([&] {
        if (!block_size)
            fail(ABHSF_ERROR_INVALID_VALUE, "block_size must be non-NULL");
        *block_size = abhsf::mlp_predict(model, features, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_selector_builtin_model(float* out)
{
    return guarded([&] {
        if (!out)
            fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
        std::copy(abhsf::builtin_model(), abhsf::builtin_model() + ABHSF_MLP_PARAMS, out);
    });
}

abhsf_status abhsf_selector_builtin_time_model(float* out)
{
    return guarded([&] {
        if (!out)
            fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
        std::copy(abhsf::builtin_time_model(), abhsf::builtin_time_model() + ABHSF_MLP_PARAMS, out);
    });
}

abhsf_status abhsf_mlp_forward(const float* params, const float* x, int32_t batch, float* probs, float* act,
                               abhsf_stream_t stream)
{
    return guarded([&] {
        abhsf::mlp_forward(params, x, batch, probs, act, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_mlp_backward(const float* params, const float* x, const float* targets, int32_t batch,
                                const float* probs, const float* act, float* delta, float* grad, float* loss,
                                abhsf_stream_t stream)
{
    return guarded([&] {
        abhsf::mlp_backward(params, x, targets, batch, probs, act, delta, grad, loss,
                            reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_mlp_adam(float* params, const float* grad, float* m, float* v, int32_t step, float lr,
                            abhsf_stream_t stream)
{
    return guarded([&] {
        abhsf::mlp_adam(params, grad, m, v, step, lr, reinterpret_cast<cudaStream_t>(stream));
    });
}

abhsf_status abhsf_read_mtx(const char* path, int32_t threads, abhsf_coo_host* out)
{
    return guarded([&] {
        if (!out)
            fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
        abhsf::read_mtx(path, threads, *out);
    });
}

abhsf_status abhsf_read_mtx_device(const char* path, abhsf_stream_t stream, abhsf_coo_device* out)
{
    const abhsf_status st = guarded([&] {
        if (!out)
            fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
        abhsf::read_mtx_device(path, reinterpret_cast<cudaStream_t>(stream), *out);
    });
    if (st != ABHSF_SUCCESS && out) {  // nothing half-made stays behind
        cudaFree(out->rows);
        cudaFree(out->cols);
        cudaFree(out->vals);
        *out = abhsf_coo_device{};
    }
    return st;
}

abhsf_status abhsf_coo_device_free(abhsf_coo_device* coo)
{
    return guarded([&] {
        if (!coo)
            fail(ABHSF_ERROR_INVALID_VALUE, "coo must be non-NULL");
        ABHSF_CUDA(cudaFree(coo->rows));
        ABHSF_CUDA(cudaFree(coo->cols));
        ABHSF_CUDA(cudaFree(coo->vals));
        *coo = abhsf_coo_device{};
    });
}

abhsf_status abhsf_coo_device_copy(const abhsf_coo_device* coo, int64_t* rows, int64_t* cols, double* vals,
                                   abhsf_stream_t stream)
{
    return guarded([&] {
        if (!coo)
            fail(ABHSF_ERROR_INVALID_VALUE, "coo must be non-NULL");
        const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
        const size_t k = (size_t)std::max<int64_t>(coo->nnz, 0);
        if (k == 0)
            return;
        if (rows)
            ABHSF_CUDA(cudaMemcpyAsync(rows, coo->rows, k * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
        if (cols)
            ABHSF_CUDA(cudaMemcpyAsync(cols, coo->cols, k * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
        if (vals)
            ABHSF_CUDA(cudaMemcpyAsync(vals, coo->vals, k * sizeof(double), cudaMemcpyDeviceToDevice, st));
    });
}

abhsf_status abhsf_read_mm(const char* path, abhsf_coo_host* out)
{
    return guarded([&] {
        if (!out)
            fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
        abhsf::read_mm(path, *out);
    });
}

abhsf_status abhsf_write_mm(const char* path, const abhsf_coo_host* coo)
{
    return guarded([&] {
        if (!coo)
            fail(ABHSF_ERROR_INVALID_VALUE, "coo must be non-NULL");
        abhsf::write_mm(path, *coo);
    });
}

abhsf_status abhsf_coo_host_free(abhsf_coo_host* coo)
{
    return guarded([&] {
        if (!coo)
            return;
        std::free(coo->rows);
        std::free(coo->cols);
        std::free(coo->vals);
        coo->rows = coo->cols = nullptr;
        coo->vals = nullptr;
        coo->nnz = 0;
    });
}

abhsf_status abhsf_mmf_line(int64_t m, int64_t n, int64_t nnz, int32_t matrix_type, int32_t r, int32_t s,
                            const uint64_t* hist, int64_t hist_len, uint64_t out_single[8], uint64_t out_double[8])
{
    return guarded([&] {
        if (m <= 0 || n <= 0 || nnz < 0 || r <= 0 || s <= 0 || hist_len < 0 || (hist_len && !hist) ||
            !out_single || !out_double)
            fail(ABHSF_ERROR_INVALID_VALUE, "invalid mmf_line arguments");
        if (matrix_type < 0 || matrix_type > 3)
            fail(ABHSF_ERROR_INVALID_VALUE, "matrix_type out of range");
        // block_statistics/mmf.cpp:34-47
        const uint64_t bits1 = (matrix_type == ABHSF_MATRIX_INTEGER || matrix_type == ABHSF_MATRIX_REAL) ? 32
                               : matrix_type == ABHSF_MATRIX_COMPLEX                                    ? 64
                                                                                                        : 0;
        std::map<uint64_t, uint64_t> h;
        for (int64_t z = 0; z < hist_len; ++z)
            if (hist[z])
                h[(uint64_t)z] = hist[z];
        abhsf::mmf_line_from_hist(m, n, nnz, matrix_type, r, s, h, bits1, out_single, out_double);
    });
}

uint64_t abhsf_block_scheme_bits(int32_t scheme, int64_t r, int64_t s, int64_t nnz, int64_t bits_per_value)
{
    switch (scheme) {
    case ABHSF_SCHEME_COO: return abhsf_coo_bits(r, s, nnz);
    case ABHSF_SCHEME_CSR: return abhsf_csr_bits(r, s, nnz);
    case ABHSF_SCHEME_BITMAP: return abhsf_bitmap_bits(r, s);
    case ABHSF_SCHEME_DENSE: return abhsf_dense_bits(r, s, nnz, bits_per_value);
    default: return UINT64_MAX;
    }
}

int32_t abhsf_block_select_scheme(int64_t r, int64_t s, int64_t nnz, int64_t bits_per_value, int32_t is_binary,
                                  int32_t allow_csr)
{
    return abhsf_select_scheme(r, s, nnz, bits_per_value, is_binary, allow_csr, nullptr);
}

}  // extern "C"
