// internal.cuh -- entry points shared between the library's translation units.
#pragma once

#include <map>
#include <string>
#include <memory>

#include "common.cuh"

namespace abhsf {

// Matrix Market ingest on the host (mtx.cu).
void read_mtx(const char* path, int threads, abhsf_coo_host& out);
std::string read_file(const char* path);
struct mtx_header {
    int type = 0, symmetry = 0;
    long long m = 0, n = 0, nnz = 0;
    size_t pos = 0;  // first byte after the size line
};
mtx_header read_mtx_header(const std::string& buf);
// One entry from the text at b (leading white space, line ends included, skipped),
// read as the host reader reads it: 0 read, 1 nothing but white space, 2 not
// an entry.
int parse_entry_host(const char* b, const char* e, bool pattern, unsigned long long& r, unsigned long long& c,
                     double& v);
// ... and on the device: the arrays in device memory (mtx_device.cu).
void read_mtx_device(const char* path, cudaStream_t st, abhsf_coo_device& out);
void read_mm(const char* path, abhsf_coo_host& out);
void write_mm(const char* path, const abhsf_coo_host& a);

void build_matrix(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m, int64_t n,
                  const abhsf_build_opts& o, cudaStream_t st, abhsf_matrix& a);

void block_histogram(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, int r, int s,
                     bool on_device, cudaStream_t st, uint64_t* hist, int64_t hist_len, int64_t* blocks);

// All 64 block sizes 2^k x 2^l (k, l = 1..8) in one call (abhsf_block_histogram_all).
void block_histogram_all(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, bool on_device,
                         cudaStream_t st, uint64_t* hist, int64_t* blocks);

// abhsf_block_histogram with device inputs and all scratch in a static array.
void block_histogram_noalloc(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, int r,
                             int s, cudaStream_t st, uint64_t* hist, int64_t hist_len, int64_t* blocks);

// ABHSF storage of square block sizes 16 .. 256 (index k: size 16 << k) and
// the size of least storage, ties to the smaller (min-bss).
constexpr int kNumBlockSizes = 5;
void block_size_storage(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n,
                        const abhsf_build_opts& o, cudaStream_t st, uint64_t bits[kNumBlockSizes]);
int select_block_size(const uint64_t bits[kNumBlockSizes]);

// Block size by measured SpMV time (autotune.cu): builds each candidate size
// (bit k of candidates: 16 << k), times reps SpMVs of it, ms[k] = -1 where not
// timed; keep (may be NULL) receives the fastest size's matrix.
void autotune(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m, int64_t n,
              const abhsf_build_opts& o, int candidates, int reps, cudaStream_t st, float ms[kNumBlockSizes],
              int* best, std::unique_ptr<abhsf_matrix>* keep);

// Learned block-size selector (selector.cu): per-matrix features and the MLP.
void selector_features(const int64_t* rows, const int64_t* cols, int64_t nnz, int64_t m, int64_t n, bool on_device,
                       cudaStream_t st, float out[ABHSF_FEATURES]);
void mlp_forward(const float* p, const float* x, int batch, float* probs, float* act, cudaStream_t st);
void mlp_backward(const float* p, const float* x, const float* target, int batch, const float* probs, const float* act,
                  float* delta, float* grad, float* loss, cudaStream_t st);
void mlp_adam(float* p, const float* g, float* m, float* v, int step, float lr, cudaStream_t st);
int mlp_predict(const float* model_host, const float features[ABHSF_FEATURES], cudaStream_t st);
const float* builtin_model();       // ABHSF_MLP_PARAMS floats, host memory: trained on storage
const float* builtin_time_model();  // ... trained on measured SpMV time

void mmf_line_from_hist(int64_t m, int64_t n, int64_t nnz, int type, int64_t r, int64_t s,
                        const std::map<uint64_t, uint64_t>& hist, uint64_t bits1, uint64_t o1[8], uint64_t o2[8]);

// y += A x for an f64 matrix, device pointers, ordered on st: warp-tree sums.
void spmv_f64(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st);

// y += A x with the reference CSR's per-row summation order (bitwise equal).

// Per-matrix set-up of the tree-order kernel (non-empty block rows, counter).
void prepare_tree(abhsf_matrix& a, cudaStream_t st);
// Per-matrix set-up of the ring kernel (block rows dealt to warps, tile
// descriptors); leaves ring_warps = 0 where that kernel does not apply.
void prepare_ring(abhsf_matrix& a, cudaStream_t st);

// y += A x with the reference CSR's per-row summation order, streaming through
// registers (shares the tree kernel's work list).
void spmv_f64_seq(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st);
// The same order through per-warp shared-memory rings (s = 32, 64); false
// when the matrix has no ring schedule.
bool spmv_f64_ring(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st);
// y += A x with x and y in host memory through the ring kernel, the block rows
// in chunks so that y's copies overlap the sums (ordered on st, not
// synchronised); false where the one-shot path serves (other kernels, small m).
bool spmv_f64_ring_host(abhsf_matrix& a, const double* x, double* y, cudaStream_t st);
// Batches (spmv_ring.cu): the ring kernel's schedule over every matrix of the
// batch, and y_i += A_i x_i for all of them in one launch (xs, ys: device
// arrays of device pointers).
void prepare_batch(abhsf_batch& b, cudaStream_t st);
void batch_spmv(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st);
// ... block sizes 16, 128, 256 (spmv_seq.cu): the streaming kernel over every
// matrix's block rows outside the slices in one launch, the slices beside it.
void prepare_batch_seq(abhsf_batch& b, cudaStream_t st);
void batch_seq_spmv(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st);

// Delta-coded row slices of the hypersparse block rows (spmv_stream.cu):
// prepare_stream picks the block rows (no dense tile, at most `avg`
// elements per tile on average), encodes them and deals the slices;
// deal_slices deals the slices of one kind (deal_kind) of block rows
// [brow_lo, brow_hi) of several matrices over one launch.  A launch plan
// names the schedules; slices_begin forks the chains onto the side stream
// (call it before the ring kernel, so that they run beside it) and
// slices_end adds the sliced rows on st and joins the chains back (x[i * ldx],
// y[i * ldy]).  The caller holds dc_mu across the pair.
void prepare_stream(abhsf_matrix& a, float avg, cudaStream_t st);
// Parts of a matrix's block rows the host-memory SpMV (abhsf_spmv_host)
// copies in, sums and copies out one after another: [M c / kHostChunks,
// M (c + 1) / kHostChunks).
constexpr int kHostChunks = 4;
enum deal_kind {
    kDealSliced = 0,  // the sliced rows
    kDealChains = 1,  // the chains
};
void deal_slices(const std::vector<const abhsf_matrix*>& mats, dbuf<uint8_t>& sched, dbuf<int64_t>& wbeg,
                 int& warps, cudaStream_t st, int64_t brow_lo, int64_t brow_hi, int kind, bool beside_ring = false);
// After the ring schedule: deal the sliced rows to run beside the ring kernel.
void slices_beside_ring(abhsf_matrix& a, cudaStream_t st);
struct dc_plan {
    const uint8_t* sched = nullptr;
    const int64_t* wbeg = nullptr;
    int warps = 0;
    const uint8_t* csched = nullptr;
    const int64_t* cwbeg = nullptr;
    int cwarps = 0;
};
dc_plan plan_of(const abhsf_matrix& a);
// cols > 1 (FP64 only: 2, 4, 8, 16 or 32): Y += A X over that many columns
// in one pass, each column bitwise its SpMV.
void slices_begin(const abhsf_matrix& a, const dc_plan& p, const void* x, int64_t ldx, void* y, int64_t ldy,
                  cudaStream_t st, int cols = 1);
void slices_end(const abhsf_matrix& a, const dc_plan& p, const void* x, int64_t ldx, void* y, int64_t ldy,
                cudaStream_t st, int cols = 1);
void prepare_batch_stream(abhsf_batch& b, cudaStream_t st);
void batch_stream_begin(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st);
void batch_stream_end(const abhsf_batch& b, const double* const* xs, double* const* ys, cudaStream_t st);

// Conjugate gradients (cg.cu).
void cg_solve(const abhsf_matrix& a, const double* b, double* x, double rtol, int max_iters, abhsf_cg_info* info,
              cudaStream_t st);
void cg_solve_mixed(const abhsf_matrix& a64, const abhsf_matrix& a32, const double* b, double* x, double rtol,
                    int max_iters, double update_factor, int max_updates, abhsf_cg_info* info, cudaStream_t st);

// y += A x in f32 for matrices stored as f32 or bf16 (values widened to f32,
// same per-row order): the ring kernel and slices where the matrix has a ring
// schedule, else the streaming kernel (beside the slices of block sizes 16,
// 128 and 256).
void spmv_f32_dispatch(const abhsf_matrix& a, const float* x, float* y, cudaStream_t st);
void spmv_f32_seq(const abhsf_matrix& a, const float* x, float* y, cudaStream_t st);
// The non-empty block rows outside the slices (seq_rows; none without slices).
void keep_rows(abhsf_matrix& a, cudaStream_t st);
// Wide SpMM (spmm_wide.cu): sets wide_cap where the matrix can take it.
void prepare_wide(abhsf_matrix& a, cudaStream_t st);
// Y += A X with k a multiple of 16 columns, 16 or 32 per pass, each pass
// reading A once (block sizes 32 / 64: spmm_staged below; 16: lanes as
// columns); false where it does not apply (value type, sum order, block
// size, alignment of X and Y).
bool spmm_f64_wide(const abhsf_matrix& a, int k, const double* X, int64_t ldx, double* Y, int64_t ldy,
                   cudaStream_t st);
// ... its block sizes 32 and 64 (spmv_ring.cu): kt = 16 or 32 columns of X and
// Y over the block rows given, with the ring's per-scheme sums (a row a lane).
void spmm_staged(const abhsf_matrix& a, int kt, const uint32_t* rows, int64_t nrows, const double* X, int64_t ldx,
                 double* Y, int64_t ldy, cudaStream_t st);
// Y += A X (k columns, row-major X and Y) through the same kernel, several
// right-hand sides per pass; false when the matrix has no ring schedule.
bool spmm_f64_ring(const abhsf_matrix& a, int k, const double* X, int64_t ldx, double* Y, int64_t ldy,
                   cudaStream_t st);


// abhsf_spmv's choice between the two f64 kernels (abhsf_matrix::sum_order).
void spmv_dispatch(const abhsf_matrix& a, const double* x, double* y, cudaStream_t st);

void inclusive_scan_i64(const int64_t* in, int64_t* out, int64_t count, cudaStream_t st);
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t count, cudaStream_t st);

}  // namespace abhsf
