// autotune.cu -- block size by measured SpMV time.
//
// The reference chooses block sizes by storage alone (block_statistics/min-bss.cpp:14-58);
// on the GPU the kernel that serves a size matters as much as its bytes (the
// ring kernel serves 32 and 64, the streaming kernel the others), so the
// autotuner builds the matrix at each candidate size and times that size's
// SpMV on the caller's stream.  The CTA shape of each kernel (warps per tile,
// rows per lane, CTAs per SM) follows from the block size and is fixed per
// size, so the block size is the one free parameter.
#include <cfloat>
#include <memory>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

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

}  // namespace

void autotune(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m, int64_t n,
              const abhsf_build_opts& o_in, int candidates, int reps, cudaStream_t st, float ms[kNumBlockSizes],
              int* best, std::unique_ptr<abhsf_matrix>* keep)
{
    if (candidates == 0)
        candidates = (1 << kNumBlockSizes) - 1;
    if (candidates < 0 || candidates >= (1 << kNumBlockSizes))
        fail(ABHSF_ERROR_INVALID_VALUE, "candidates: bit k selects block size 16 << k, k < 5");
    if (reps < 1 || reps > 10000)
        fail(ABHSF_ERROR_INVALID_VALUE, "reps must be 1 .. 10000");
    if (m <= 0 || n <= 0 || nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
    if (nnz > 0 && (!rows || !cols))
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL");
    abhsf_build_opts o = o_in;
    // host inputs cross to the device once for all candidate builds
    dbuf<int64_t> r_d, c_d;
    dbuf<double> v_d;
    if (!o.inputs_on_device && nnz > 0) {
        r_d.alloc(nnz);
        c_d.alloc(nnz);
        ABHSF_CUDA(cudaMemcpyAsync(r_d.get(), rows, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(c_d.get(), cols, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        rows = r_d.get();
        cols = c_d.get();
        if (vals) {
            v_d.alloc(nnz);
            ABHSF_CUDA(cudaMemcpyAsync(v_d.get(), vals, nnz * sizeof(double), cudaMemcpyHostToDevice, st));
            vals = v_d.get();
        }
    }
    o.inputs_on_device = 1;
    const bool f64 = o.value_type == ABHSF_VALUE_F64;
    // x = 0, y = 0: the kernels' speed does not depend on the values
    dbuf<uint8_t> x((size_t)n * 8 + 16), y((size_t)m * 8 + 16);
    ABHSF_CUDA(cudaMemsetAsync(x.get(), 0, (size_t)n * 8 + 16, st));
    ABHSF_CUDA(cudaMemsetAsync(y.get(), 0, (size_t)m * 8 + 16, st));
    event_pair ev;
    float best_ms = FLT_MAX;
    *best = 0;
    for (int k = 0; k < kNumBlockSizes; ++k) {
        ms[k] = -1.0f;
        if (!((candidates >> k) & 1))
            continue;
        o.block_size = 16 << k;
        auto a = std::make_unique<abhsf_matrix>();
        build_matrix(rows, cols, vals, nnz, m, n, o, st, *a);
        auto run = [&] {
            if (f64)
                spmv_dispatch(*a, reinterpret_cast<const double*>(x.get()), reinterpret_cast<double*>(y.get()), st);
            else
                spmv_f32_dispatch(*a, reinterpret_cast<const float*>(x.get()), reinterpret_cast<float*>(y.get()), st);
        };
        run();
        ABHSF_CUDA(cudaEventRecord(ev.a, st));
        for (int r = 0; r < reps; ++r)
            run();
        ABHSF_CUDA(cudaEventRecord(ev.b, st));
        ABHSF_CUDA(cudaEventSynchronize(ev.b));
        float t = 0.0f;
        ABHSF_CUDA(cudaEventElapsedTime(&t, ev.a, ev.b));
        ms[k] = t / (float)reps;
        if (ms[k] < best_ms) {
            best_ms = ms[k];
            *best = 16 << k;
            if (keep)
                *keep = std::move(a);
        }
    }
    if (*best == 0)
        fail(ABHSF_ERROR_UNSUPPORTED, "no candidate block size has a kernel for this value type");
}

}  // namespace abhsf
