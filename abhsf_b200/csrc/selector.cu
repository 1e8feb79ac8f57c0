// selector.cu -- the learned block-size selector: matrix features on the GPU
// and a small MLP (2 hidden layers of 64 ReLU units, FP32) with its own
// forward, backward and Adam kernels.
//
// The reference picks the block size by exhaustive storage: every candidate
// size's block statistics, then the minimum (block_statistics/min-bss.cpp:14-58),
// and scores restricted choices by their regret, the storage above that
// minimum in percent (block_statistics/consistency.cpp:140-174).  The MLP
// predicts the minimum-storage size from one pass of features instead of five
// histograms; block_size_storage (builder.cu) gives the exhaustive answer it
// is trained on and scored against.
//
// Model layout (ABHSF_MLP_PARAMS floats): W1[F][H] b1[H] W2[H][H] b2[H]
// W3[H][C] b3[C] mean[F] inv_std[F]; the input is (features - mean) * inv_std.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

constexpr int F = ABHSF_FEATURES, H = ABHSF_MLP_HIDDEN, C = ABHSF_MLP_CLASSES;
constexpr int OW1 = 0, OB1 = OW1 + F * H, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H * C,
              OMEAN = OB3 + C, OISTD = OMEAN + F;
static_assert(OISTD + F == ABHSF_MLP_PARAMS, "model layout");
static_assert(F <= H && C <= H, "one thread per hidden unit covers the inputs and outputs");
constexpr int kTrainable = OMEAN;  // the normalisation is fixed, not trained
constexpr int ACT = 2 * H;         // per-sample activations kept for backward: h1, h2
constexpr int DLT = C + 2 * H;     // per-sample deltas: logits, h2, h1

// The trained models shipped with the library (written by abhsf_b200/selector.py):
// one trained on the storage of each size, one on the measured SpMV time.
#include "selector_model.inc"
#include "selector_model_time.inc"
static_assert(sizeof(kBuiltinModel) == ABHSF_MLP_PARAMS * sizeof(float), "built-in model size");
static_assert(sizeof(kBuiltinTimeModel) == ABHSF_MLP_PARAMS * sizeof(float), "built-in model size");

// ---------------------------------------------------------------- features

struct feat_acc {
    unsigned long long max_dist;
    double sum_dist;
    int bad;
};

// Row counts, the largest and the summed |i - j|; an index outside m x n sets
// bad and is skipped.
__global__ void k_row_counts(int64_t nnz, int64_t m, int64_t n, const int64_t* __restrict__ rows,
                             const int64_t* __restrict__ cols, unsigned int* __restrict__ count, feat_acc* acc)
{
    unsigned long long mx = 0;
    double sd = 0.0;
    int bad = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = rows[k], j = cols[k];
        if (i < 0 || i >= m || j < 0 || j >= n) {
            bad = 1;
            continue;
        }
        atomicAdd(&count[i], 1u);
        const int64_t d = i > j ? i - j : j - i;
        mx = max(mx, (unsigned long long)d);
        sd += (double)d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&acc->max_dist, mx);
        atomicAdd(&acc->sum_dist, sd);
        if (bad)
            atomicOr(&acc->bad, 1);
    }
}

// Sum over rows of (count - mean)^2.
__global__ void k_row_var(int64_t m, const unsigned int* __restrict__ count, double mean, double* out)
{
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = (double)count[i] - mean;
        s += d * d;
    }
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(out, s);
}

// ---------------------------------------------------------------- MLP kernels

// One CTA of H threads per sample: normalised input, h1, h2, softmax(logits).
__global__ void __launch_bounds__(H) k_mlp_forward(const float* __restrict__ p, const float* __restrict__ x, int batch,
                                                   float* __restrict__ probs, float* __restrict__ act)
{
    __shared__ float xn[F], h1[H], h2[H], lg[C];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= batch)
        return;
    if (j < F)
        xn[j] = (x[(int64_t)b * F + j] - p[OMEAN + j]) * p[OISTD + j];
    __syncthreads();
    float s = p[OB1 + j];
    for (int f = 0; f < F; ++f)
        s += xn[f] * p[OW1 + f * H + j];
    h1[j] = fmaxf(s, 0.0f);
    __syncthreads();
    s = p[OB2 + j];
    for (int k = 0; k < H; ++k)
        s += h1[k] * p[OW2 + k * H + j];
    h2[j] = fmaxf(s, 0.0f);
    __syncthreads();
    if (j < C) {
        float t = p[OB3 + j];
        for (int k = 0; k < H; ++k)
            t += h2[k] * p[OW3 + k * C + j];
        lg[j] = t;
    }
    __syncthreads();
    if (j < C) {
        float mx = lg[0];
        for (int c = 1; c < C; ++c)
            mx = fmaxf(mx, lg[c]);
        float z = 0.0f;
        for (int c = 0; c < C; ++c)
            z += expf(lg[c] - mx);
        probs[(int64_t)b * C + j] = expf(lg[j] - mx) / z;
    }
    if (act) {
        act[(int64_t)b * ACT + j] = h1[j];
        act[(int64_t)b * ACT + H + j] = h2[j];
    }
}

// Per sample: dlogits = (probs - target) / batch, dh2 = W3 dlogits masked by
// h2 > 0, dh1 = W2 dh2 masked by h1 > 0.
__global__ void __launch_bounds__(H) k_mlp_delta(const float* __restrict__ p, const float* __restrict__ target,
                                                 int batch, const float* __restrict__ probs,
                                                 const float* __restrict__ act, float* __restrict__ delta)
{
    __shared__ float dl[C], d2[H];
    const int b = blockIdx.x, j = threadIdx.x;
    if (b >= batch)
        return;
    if (j < C)
        dl[j] = (probs[(int64_t)b * C + j] - target[(int64_t)b * C + j]) / (float)batch;
    __syncthreads();
    float s = 0.0f;
    for (int c = 0; c < C; ++c)
        s += p[OW3 + j * C + c] * dl[c];
    d2[j] = act[(int64_t)b * ACT + H + j] > 0.0f ? s : 0.0f;
    __syncthreads();
    s = 0.0f;
    for (int k = 0; k < H; ++k)
        s += p[OW2 + j * H + k] * d2[k];
    float* o = delta + (int64_t)b * DLT;
    if (j < C)
        o[j] = dl[j];
    o[C + j] = d2[j];
    o[C + H + j] = act[(int64_t)b * ACT + j] > 0.0f ? s : 0.0f;
}

// One thread per trainable parameter: its gradient summed over the batch in
// sample order (deterministic).  Thread 0 of block 0 also writes the mean
// cross-entropy.
__global__ void k_mlp_grad(const float* __restrict__ p, const float* __restrict__ x,
                           const float* __restrict__ target, int batch, const float* __restrict__ probs,
                           const float* __restrict__ act, const float* __restrict__ delta, float* __restrict__ grad,
                           float* loss)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q == 0 && loss) {
        float l = 0.0f;
        for (int b = 0; b < batch; ++b)
            for (int c = 0; c < C; ++c) {
                const float t = target[(int64_t)b * C + c];
                if (t > 0.0f)
                    l -= t * logf(fmaxf(probs[(int64_t)b * C + c], 1e-30f));
            }
        *loss = l / (float)batch;
    }
    if (q >= kTrainable)
        return;
    float g = 0.0f;
    for (int b = 0; b < batch; ++b) {
        const float* dl = delta + (int64_t)b * DLT;
        const float* d2 = dl + C;
        const float* d1 = dl + C + H;
        const float* h1 = act + (int64_t)b * ACT;
        const float* h2 = h1 + H;
        if (q < OB1) {
            const int f = q / H, j = q % H;
            g += (x[(int64_t)b * F + f] - p[OMEAN + f]) * p[OISTD + f] * d1[j];
        } else if (q < OW2) {
            g += d1[q - OB1];
        } else if (q < OB2) {
            const int k = (q - OW2) / H, j = (q - OW2) % H;
            g += h1[k] * d2[j];
        } else if (q < OW3) {
            g += d2[q - OB2];
        } else if (q < OB3) {
            const int k = (q - OW3) / C, c = (q - OW3) % C;
            g += h2[k] * dl[c];
        } else {
            g += dl[q - OB3];
        }
    }
    grad[q] = g;
}

__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, int step, float lr)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kTrainable)
        return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    m[q] = b1 * m[q] + (1.0f - b1) * g[q];
    v[q] = b2 * v[q] + (1.0f - b2) * g[q] * g[q];
    const float mh = m[q] / (1.0f - powf(b1, (float)step));
    const float vh = v[q] / (1.0f - powf(b2, (float)step));
    p[q] -= lr * mh / (sqrtf(vh) + eps);
}

unsigned grid_of(int64_t work)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 8));
}

}  // namespace

const float* builtin_model() { return kBuiltinModel; }
const float* builtin_time_model() { return kBuiltinTimeModel; }

void selector_features(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, bool on_device,
                       cudaStream_t st, float out[ABHSF_FEATURES])
{
    if (m <= 0 || n <= 0 || nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "m and n must be positive and nnz non-negative");
    if (nnz > 0 && (!rows || !cols))
        fail(ABHSF_ERROR_INVALID_VALUE, "rows and cols must be non-NULL");
    if (!out)
        fail(ABHSF_ERROR_INVALID_VALUE, "out must be non-NULL");
    dbuf<int64_t> r_d, c_d;
    const int64_t* r = rows;
    const int64_t* c = cols;
    if (!on_device && nnz > 0) {
        r_d.alloc(nnz);
        c_d.alloc(nnz);
        ABHSF_CUDA(cudaMemcpyAsync(r_d.get(), rows, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(c_d.get(), cols, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        r = r_d.get();
        c = c_d.get();
    }
    dbuf<unsigned int> count(m);
    dbuf<feat_acc> acc(1);
    dbuf<double> var(1);
    ABHSF_CUDA(cudaMemsetAsync(count.get(), 0, m * sizeof(unsigned int), st));
    ABHSF_CUDA(cudaMemsetAsync(acc.get(), 0, sizeof(feat_acc), st));
    ABHSF_CUDA(cudaMemsetAsync(var.get(), 0, sizeof(double), st));
    if (nnz > 0) {
        k_row_counts<<<grid_of(nnz), 256, 0, st>>>(nnz, m, n, r, c, count.get(), acc.get());
        ABHSF_CUDA(cudaGetLastError());
    }
    feat_acc a{};
    ABHSF_CUDA(cudaMemcpyAsync(&a, acc.get(), sizeof(feat_acc), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    if (a.bad)
        fail(ABHSF_ERROR_INDEX_OUT_OF_RANGE, "an element lies outside the m x n matrix");
    const double mean = (double)nnz / (double)m;
    k_row_var<<<grid_of(m), 256, 0, st>>>(m, count.get(), mean, var.get());
    ABHSF_CUDA(cudaGetLastError());
    double v = 0.0;
    ABHSF_CUDA(cudaMemcpyAsync(&v, var.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    // tile density profile at s = 64: share of the nonzeros in tiles of each fill class
    std::vector<uint64_t> h(64 * 64 + 1);
    int64_t blocks = 0;
    block_histogram(r, c, nnz, m, n, 64, 64, true, st, h.data(), (int64_t)h.size(), &blocks);
    ABHSF_CUDA(cudaStreamSynchronize(st));  // v
    double share[5] = {0, 0, 0, 0, 0};
    for (size_t z = 1; z < h.size(); ++z) {
        const int k = z <= 4 ? 0 : z <= 32 ? 1 : z <= 256 ? 2 : z <= 1024 ? 3 : 4;
        share[k] += (double)z * (double)h[z];
    }
    const double dn = std::max<double>((double)nnz, 1.0);
    const double mn = (double)std::max(m, n);
    const double M64 = (double)((m + 63) / 64);
    out[0] = (float)std::log2((double)m);
    out[1] = (float)std::log2((double)n);
    out[2] = (float)std::log2(mean + 1.0);
    out[3] = (float)std::log2(std::sqrt(v / (double)m) + 1.0);
    out[4] = (float)((double)a.max_dist / mn);
    out[5] = (float)(a.sum_dist / dn / mn);
    for (int k = 0; k < 5; ++k)
        out[6 + k] = (float)(share[k] / dn);
    out[11] = (float)std::log2((double)blocks / M64 + 1.0);
}

void mlp_forward(const float* p, const float* x, int batch, float* probs, float* act, cudaStream_t st)
{
    if (batch < 0 || (batch > 0 && (!p || !x || !probs)))
        fail(ABHSF_ERROR_INVALID_VALUE, "invalid mlp_forward arguments");
    if (batch == 0)
        return;
    k_mlp_forward<<<batch, H, 0, st>>>(p, x, batch, probs, act);
    ABHSF_CUDA(cudaGetLastError());
}

void mlp_backward(const float* p, const float* x, const float* target, int batch, const float* probs, const float* act,
                  float* delta, float* grad, float* loss, cudaStream_t st)
{
    if (batch <= 0 || !p || !x || !target || !probs || !act || !delta || !grad)
        fail(ABHSF_ERROR_INVALID_VALUE, "invalid mlp_backward arguments");
    k_mlp_delta<<<batch, H, 0, st>>>(p, target, batch, probs, act, delta);
    ABHSF_CUDA(cudaGetLastError());
    k_mlp_grad<<<(kTrainable + 255) / 256, 256, 0, st>>>(p, x, target, batch, probs, act, delta, grad, loss);
    ABHSF_CUDA(cudaGetLastError());
}

void mlp_adam(float* p, const float* g, float* m, float* v, int step, float lr, cudaStream_t st)
{
    if (!p || !g || !m || !v || step < 1)
        fail(ABHSF_ERROR_INVALID_VALUE, "invalid mlp_adam arguments");
    k_mlp_adam<<<(kTrainable + 255) / 256, 256, 0, st>>>(p, g, m, v, step, lr);
    ABHSF_CUDA(cudaGetLastError());
}

int mlp_predict(const float* model_host, const float features[ABHSF_FEATURES], cudaStream_t st)
{
    if (!features)
        fail(ABHSF_ERROR_INVALID_VALUE, "features must be non-NULL");
    const float* model = model_host ? model_host : kBuiltinModel;
    dbuf<float> p(ABHSF_MLP_PARAMS), x(F), probs(C);
    ABHSF_CUDA(cudaMemcpyAsync(p.get(), model, ABHSF_MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, st));
    ABHSF_CUDA(cudaMemcpyAsync(x.get(), features, F * sizeof(float), cudaMemcpyHostToDevice, st));
    mlp_forward(p.get(), x.get(), 1, probs.get(), nullptr, st);
    float pr[C];
    ABHSF_CUDA(cudaMemcpyAsync(pr, probs.get(), sizeof(pr), cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    int best = 0;
    for (int k = 1; k < C; ++k)
        if (pr[k] > pr[best])
            best = k;
    return 16 << best;
}

}  // namespace abhsf
