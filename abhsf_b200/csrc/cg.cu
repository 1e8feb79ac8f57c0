// cg.cu -- conjugate gradients on ABHSF matrices: plain FP64, and mixed
// precision (an f32 CG on an f32 or bf16 copy of the matrix whose solution
// accumulates in FP64 and whose residual is replaced by the FP64 residual of
// the f64 matrix each time it has fallen by a set factor: reliable updates).
//
// The reference has no solver; its SpMV is the kernel such a solver calls
// (spmv/bottlenecks/spmv.cpp:58-64).  Both solvers here keep every scalar
// (alpha, beta, r.r) on the device: a CG iteration is one SpMV and five small
// kernels, and chunks of iterations are captured once into a CUDA graph and
// replayed, with one host read of the state per chunk.  Dot products are
// summed in FP64 over a fixed grid (deterministic).  Once the recurrence
// residual meets the tolerance, the state's `done` flag turns the rest of the
// chunk's updates into no-ops.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kChunk = 8;  // CG iterations per captured graph

struct cg_state {
    double rr;     // r . r of the current residual
    double alpha;  // step of this iteration
    double beta;   // p update of this iteration
    double tol2;   // stop when r . r <= tol2
    int done;      // tolerance met, or iteration limit reached
    int iters;     // iterations performed
    int max_iters;
    int active;  // this iteration updates x, r and p (done was not set before it)
};

__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double part[kRedThreads / 32];
    for (int d = 16; d > 0; d >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x >> 5] = v;
    __syncthreads();
    v = threadIdx.x < kRedThreads / 32 ? part[threadIdx.x] : 0.0;
    if (threadIdx.x < 32)
        for (int d = 16; d > 0; d >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;  // valid in thread 0
}

// 16 bytes of T: the unit the vector kernels below load and store when every
// array they touch is 16-byte aligned (VEC), so that an f32 pass moves as
// many bytes per instruction as an f64 one.
template <typename T>
struct __align__(16) pack {
    static constexpr int N = 16 / sizeof(T);
    T v[N];
};

template <typename T>
__device__ __forceinline__ pack<T> ld_pack(const T* p)
{
    return *reinterpret_cast<const pack<T>*>(p);
}

template <typename T>
__device__ __forceinline__ void st_pack(T* p, const pack<T>& v)
{
    *reinterpret_cast<pack<T>*>(p) = v;
}

constexpr int64_t kStride = (int64_t)kRedBlocks * kRedThreads;

// partial[blockIdx.x] = sum over this block's grid-stride share of a[i] b[i]
// (with VEC, packs of 16 bytes, then the tail past the last whole pack)
template <typename T, bool VEC>
__global__ void __launch_bounds__(kRedThreads) k_dot(int64_t n, const T* __restrict__ a, const T* __restrict__ b,
                                                     double* __restrict__ partial)
{
    constexpr int N = pack<T>::N;
    const int64_t tid = blockIdx.x * (int64_t)kRedThreads + threadIdx.x;
    const int64_t nv = VEC ? n / N : 0;
    double s = 0.0;
    for (int64_t i = tid; i < nv; i += kStride) {
        const pack<T> va = ld_pack(a + i * N), vb = ld_pack(b + i * N);
#pragma unroll
        for (int k = 0; k < N; ++k)
            s += (double)va.v[k] * (double)vb.v[k];
    }
    for (int64_t i = nv * N + tid; i < n; i += kStride)
        s += (double)a[i] * (double)b[i];
    s = block_sum(s);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = s;
}

__device__ __forceinline__ double sum_partials(const double* __restrict__ partial)
{
    double s = 0.0;
    for (int i = threadIdx.x; i < kRedBlocks; i += kRedThreads)
        s += partial[i];
    return block_sum(s);
}

// state from r . r (first partials), with tolerance tol2 = rtol^2 * bb
__global__ void __launch_bounds__(kRedThreads) k_cg_init(const double* __restrict__ partial, cg_state* st,
                                                         double tol2, int max_iters)
{
    const double rr = sum_partials(partial);
    if (threadIdx.x == 0) {
        st->rr = rr;
        st->alpha = st->beta = 0.0;
        st->tol2 = tol2;
        st->iters = 0;
        st->max_iters = max_iters;
        st->active = 0;
        st->done = (rr <= tol2 || max_iters <= 0) ? 1 : 0;
    }
}

// restart the recurrence from a replaced residual: r . r from the partials,
// the tolerance factor2 * r . r, the search direction and iteration count kept
__global__ void __launch_bounds__(kRedThreads) k_cg_resume(const double* __restrict__ partial, cg_state* st,
                                                           double factor2)
{
    const double rr = sum_partials(partial);
    if (threadIdx.x == 0) {
        const double tol2 = factor2 * rr;
        st->rr = rr;
        st->tol2 = tol2;
        st->done = (rr <= tol2 || st->iters >= st->max_iters) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_cg_alpha(const double* __restrict__ partial, cg_state* st)
{
    const double pap = sum_partials(partial);
    if (threadIdx.x == 0) {
        if (st->done || !(pap > 0.0)) {  // converged, or breakdown (p = 0 or A not positive definite on p)
            st->alpha = 0.0;
            st->done = 1;
            st->active = 0;
        } else {
            st->alpha = st->rr / pap;
            st->active = 1;
        }
    }
}

// x += alpha p; r -= alpha Ap; Ap = 0 (ready for the next y += A p); partial r . r
template <typename T, bool VEC>
__global__ void __launch_bounds__(kRedThreads) k_cg_update_xr(int64_t n, T* __restrict__ x, T* __restrict__ r,
                                                              T* __restrict__ ap, const T* __restrict__ p,
                                                              const cg_state* st, double* __restrict__ partial)
{
    constexpr int N = pack<T>::N;
    const T alpha = (T)st->alpha;
    const int64_t tid = blockIdx.x * (int64_t)kRedThreads + threadIdx.x;
    const int64_t nv = VEC ? n / N : 0;
    double s = 0.0;
    for (int64_t i = tid; i < nv; i += kStride) {
        pack<T> vr = ld_pack(r + i * N), vx = ld_pack(x + i * N);
        const pack<T> va = ld_pack(ap + i * N), vp = ld_pack(p + i * N);
        pack<T> zero;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            vr.v[k] = vr.v[k] - alpha * va.v[k];
            vx.v[k] += alpha * vp.v[k];
            zero.v[k] = T(0);
            s += (double)vr.v[k] * (double)vr.v[k];
        }
        st_pack(x + i * N, vx);
        st_pack(r + i * N, vr);
        st_pack(ap + i * N, zero);
    }
    for (int64_t i = nv * N + tid; i < n; i += kStride) {
        const T ri = r[i] - alpha * ap[i];
        x[i] += alpha * p[i];
        r[i] = ri;
        ap[i] = T(0);
        s += (double)ri * (double)ri;
    }
    s = block_sum(s);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads) k_cg_beta(const double* __restrict__ partial, cg_state* st)
{
    const double rr_new = sum_partials(partial);
    if (threadIdx.x == 0 && !st->done) {
        st->beta = rr_new / st->rr;
        st->rr = rr_new;
        st->iters += 1;
        if (rr_new <= st->tol2 || st->iters >= st->max_iters)
            st->done = 1;
    }
}

// p = r + beta p, also in the iteration that met the tolerance, so that a
// recurrence resumed from a replaced residual continues from the right p
template <typename T, bool VEC>
__global__ void k_cg_update_p(int64_t n, T* __restrict__ p, const T* __restrict__ r, const cg_state* st)
{
    if (!st->active)
        return;
    constexpr int N = pack<T>::N;
    const T beta = (T)st->beta;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t nv = VEC ? n / N : 0;
    for (int64_t i = tid; i < nv; i += stride) {
        pack<T> vp = ld_pack(p + i * N);
        const pack<T> vr = ld_pack(r + i * N);
#pragma unroll
        for (int k = 0; k < N; ++k)
            vp.v[k] = vr.v[k] + beta * vp.v[k];
        st_pack(p + i * N, vp);
    }
    for (int64_t i = nv * N + tid; i < n; i += stride)
        p[i] = r[i] + beta * p[i];
}

template <typename T>
__global__ void k_neg(int64_t n, const T* __restrict__ a, T* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = -a[i];
}

// out = (float) r
__global__ void k_to_f32(int64_t n, const double* __restrict__ r, float* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)r[i];
}

// x += d; d = 0 (the f32 correction folded into the FP64 solution)
__global__ void k_fold(int64_t n, double* __restrict__ x, float* __restrict__ d)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += (double)d[i];
        d[i] = 0.0f;
    }
}

unsigned elem_grid(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

// y += A x in T (f64 or f32 kernels)
void spmv_t(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st) { spmv_dispatch(a, x, y, st); }
void spmv_t(const abhsf_matrix& a, const float* x, float* y, cudaStream_t st) { spmv_f32_dispatch(a, x, y, st); }

template <typename T>
struct cg_work {
    dbuf<T> r, p, ap;
    explicit cg_work(int64_t n) : r(n), p(n), ap(n) {}
};

// r = b - A x (xn: scratch)
template <typename T>
void residual(const abhsf_matrix& a, const T* b, const T* x, T* r, T* xn, int64_t n, cudaStream_t st)
{
    k_neg<T><<<elem_grid(n), 256, 0, st>>>(n, x, xn);
    ABHSF_CUDA(cudaMemcpyAsync(r, b, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
    spmv_t(a, xn, r, st);
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename T>
void dot(const T* a, const T* b, int64_t n, double* partial, cudaStream_t st)
{
    if (aligned16(a) && aligned16(b))
        k_dot<T, true><<<kRedBlocks, kRedThreads, 0, st>>>(n, a, b, partial);
    else
        k_dot<T, false><<<kRedBlocks, kRedThreads, 0, st>>>(n, a, b, partial);
}

// p = r, Ap = 0 and the state from r . r: the start of a CG recurrence.
template <typename T>
void cg_start(cg_work<T>& w, int64_t n, cg_state* st_d, double* partial, double tol2, int max_iters,
              cudaStream_t cs)
{
    ABHSF_CUDA(cudaMemcpyAsync(w.p.get(), w.r.get(), n * sizeof(T), cudaMemcpyDeviceToDevice, cs));
    ABHSF_CUDA(cudaMemsetAsync(w.ap.get(), 0, n * sizeof(T), cs));
    dot<T>(w.r.get(), w.r.get(), n, partial, cs);
    k_cg_init<<<1, kRedThreads, 0, cs>>>(partial, st_d, tol2, max_iters);
    ABHSF_CUDA(cudaGetLastError());
}

// kChunk CG iterations on A x = b (x, w.r, w.p, w.ap and the state on the
// device), captured once into a graph and replayed until the state is done.
template <typename T>
class cg_graph {
  public:
    cg_graph(const abhsf_matrix& a, T* x, cg_work<T>& w, int64_t n, cg_state* st_d, double* partial, cudaStream_t cs)
    {
        cudaGraph_t graph = nullptr;
        const bool vec = aligned16(x) && aligned16(w.r.get()) && aligned16(w.ap.get()) && aligned16(w.p.get());
        ABHSF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < kChunk; ++it) {
            spmv_t(a, w.p.get(), w.ap.get(), cs);
            dot<T>(w.p.get(), w.ap.get(), n, partial, cs);
            k_cg_alpha<<<1, kRedThreads, 0, cs>>>(partial, st_d);
            if (vec)
                k_cg_update_xr<T, true>
                    <<<kRedBlocks, kRedThreads, 0, cs>>>(n, x, w.r.get(), w.ap.get(), w.p.get(), st_d, partial);
            else
                k_cg_update_xr<T, false>
                    <<<kRedBlocks, kRedThreads, 0, cs>>>(n, x, w.r.get(), w.ap.get(), w.p.get(), st_d, partial);
            k_cg_beta<<<1, kRedThreads, 0, cs>>>(partial, st_d);
            if (vec)
                k_cg_update_p<T, true><<<elem_grid(n), 256, 0, cs>>>(n, w.p.get(), w.r.get(), st_d);
            else
                k_cg_update_p<T, false><<<elem_grid(n), 256, 0, cs>>>(n, w.p.get(), w.r.get(), st_d);
        }
        const cudaError_t cap = cudaStreamEndCapture(cs, &graph);
        if (cap != cudaSuccess || !graph)
            fail(ABHSF_ERROR_CUDA, std::string("CG graph capture: ") + cudaGetErrorString(cap));
        const cudaError_t ins = cudaGraphInstantiate(&exec_, graph, 0);
        cudaGraphDestroy(graph);
        if (ins != cudaSuccess)
            fail(ABHSF_ERROR_CUDA, std::string("CG graph instantiation: ") + cudaGetErrorString(ins));
    }
    ~cg_graph() { cudaGraphExecDestroy(exec_); }
    cg_graph(const cg_graph&) = delete;
    cg_graph& operator=(const cg_graph&) = delete;

    // replays chunks until the state says done; returns the iteration count
    int run(cg_state* st_d, cg_state* st_h, cudaStream_t cs)
    {
        for (;;) {
            ABHSF_CUDA(cudaMemcpyAsync(st_h, st_d, sizeof(cg_state), cudaMemcpyDeviceToHost, cs));
            ABHSF_CUDA(cudaStreamSynchronize(cs));
            if (st_h->done)
                return st_h->iters;
            ABHSF_CUDA(cudaGraphLaunch(exec_, cs));
        }
    }

  private:
    cudaGraphExec_t exec_ = nullptr;
};

struct solve_stream {
    cudaStream_t user, cs = nullptr;
    cudaEvent_t ev = nullptr;
    explicit solve_stream(cudaStream_t u) : user(u)
    {
        ABHSF_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        ABHSF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        ABHSF_CUDA(cudaEventRecord(ev, user));  // the solve starts after the caller's queued work
        ABHSF_CUDA(cudaStreamWaitEvent(cs, ev, 0));
    }
    ~solve_stream()
    {
        cudaStreamSynchronize(cs);
        cudaEventDestroy(ev);
        cudaStreamDestroy(cs);
    }
};

double norm2(const double* a, int64_t n, double* partial, cg_state* st_d, cg_state* st_h, cudaStream_t cs)
{
    dot<double>(a, a, n, partial, cs);
    k_cg_init<<<1, kRedThreads, 0, cs>>>(partial, st_d, 0.0, 0);
    ABHSF_CUDA(cudaMemcpyAsync(st_h, st_d, sizeof(cg_state), cudaMemcpyDeviceToHost, cs));
    ABHSF_CUDA(cudaStreamSynchronize(cs));
    return st_h->rr;
}

void check_square(const abhsf_matrix& a)
{
    if (a.m != a.n)
        fail(ABHSF_ERROR_INVALID_VALUE, "CG needs a square matrix");
}

}  // namespace

void cg_solve(const abhsf_matrix& a, const double* b, double* x, double rtol, int max_iters, abhsf_cg_info* info,
              cudaStream_t user)
{
    check_square(a);
    const int64_t n = a.n;
    solve_stream ss(user);
    cudaStream_t cs = ss.cs;
    cg_work<double> w(n);
    dbuf<double> xn(n), partial(kRedBlocks);
    dbuf<cg_state> st_d(1);
    cg_state st_h{};
    const double bb = norm2(b, n, partial.get(), st_d.get(), &st_h, cs);
    residual<double>(a, b, x, w.r.get(), xn.get(), n, cs);
    cg_start<double>(w, n, st_d.get(), partial.get(), rtol * rtol * bb, max_iters, cs);
    cg_graph<double> g(a, x, w, n, st_d.get(), partial.get(), cs);
    const int iters = g.run(st_d.get(), &st_h, cs);
    residual<double>(a, b, x, w.r.get(), xn.get(), n, cs);
    const double rr = norm2(w.r.get(), n, partial.get(), st_d.get(), &st_h, cs);
    info->iterations = iters;
    info->outer_iterations = 1;
    info->rel_residual = bb > 0.0 ? std::sqrt(rr / bb) : std::sqrt(rr);
    info->converged = info->rel_residual <= rtol ? 1 : 0;
}

void cg_solve_mixed(const abhsf_matrix& a64, const abhsf_matrix& a32, const double* b, double* x, double rtol,
                    int max_iters, double update_factor, int max_updates, abhsf_cg_info* info, cudaStream_t user)
{
    check_square(a64);
    if (a32.m != a64.m || a32.n != a64.n)
        fail(ABHSF_ERROR_INVALID_VALUE, "the two matrices of the mixed solver differ in shape");
    const int64_t n = a64.n;
    const double f2 = update_factor * update_factor;
    solve_stream ss(user);
    cudaStream_t cs = ss.cs;
    dbuf<double> r64(n), xn(n), partial(kRedBlocks);
    cg_work<float> w(n);
    dbuf<float> d(n);  // the f32 solution since the last update
    dbuf<cg_state> st_d(1), st64_d(1);
    cg_state st_h{};
    const double bb = norm2(b, n, partial.get(), st64_d.get(), &st_h, cs);
    const double tol2 = rtol * rtol * bb;
    residual<double>(a64, b, x, r64.get(), xn.get(), n, cs);
    double rr = norm2(r64.get(), n, partial.get(), st64_d.get(), &st_h, cs);
    int iters = 0, updates = 0;
    if (rr > tol2 && max_iters > 0) {
        k_to_f32<<<elem_grid(n), 256, 0, cs>>>(n, r64.get(), w.r.get());
        ABHSF_CUDA(cudaMemsetAsync(d.get(), 0, n * sizeof(float), cs));
        cg_start<float>(w, n, st_d.get(), partial.get(), 0.0, max_iters, cs);
        k_cg_resume<<<1, kRedThreads, 0, cs>>>(partial.get(), st_d.get(), f2);  // partials of r32 . r32
        cg_graph<float> g(a32, d.get(), w, n, st_d.get(), partial.get(), cs);
        for (;;) {
            iters = g.run(st_d.get(), &st_h, cs);
            // reliable update: fold the f32 solution into x, replace r by b - A x in FP64
            k_fold<<<elem_grid(n), 256, 0, cs>>>(n, x, d.get());
            residual<double>(a64, b, x, r64.get(), xn.get(), n, cs);
            rr = norm2(r64.get(), n, partial.get(), st64_d.get(), &st_h, cs);
            ++updates;
            if (rr <= tol2 || iters >= max_iters || updates >= max_updates)
                break;
            k_to_f32<<<elem_grid(n), 256, 0, cs>>>(n, r64.get(), w.r.get());
            dot<float>(w.r.get(), w.r.get(), n, partial.get(), cs);
            k_cg_resume<<<1, kRedThreads, 0, cs>>>(partial.get(), st_d.get(), f2);
            ABHSF_CUDA(cudaGetLastError());
        }
    }
    info->iterations = iters;
    info->outer_iterations = updates;
    info->rel_residual = bb > 0.0 ? std::sqrt(rr / bb) : std::sqrt(rr);
    info->converged = info->rel_residual <= rtol ? 1 : 0;
}

}  // namespace abhsf
