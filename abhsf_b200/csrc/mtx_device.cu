// mtx_device.cu -- Matrix Market ingest with the parse on the GPU.
//
// Reads what abhsf_read_mtx reads (the reference's read_mtx_real_or_binary,
// include/abhsf/utils/matrix_market_reader.h:146-200: real or pattern,
// 0-based, explicit zeros dropped, a symmetric file's stored triangle kept
// and both triangles rejected, the first nnz entries), with the entry lines
// parsed on the device:
//
// * The host reads the file and its banner and size line (mtx.cu's header
//   parse) and copies the entry lines to the device.
// * Line heads are flagged and compacted (one pass over the bytes); one
//   thread per line reads the entry: two indices and a value in their plain
//   spellings.  A value is rounded to the nearest double as strtod rounds
//   it: its significand (at most 19 significant digits) times 5^q in 128 bits
//   (pow5_table.inc), the rounding decided from the product wherever its
//   truncation cannot change the outcome -- the method of D. Lemire, "Number
//   parsing at a gigabyte per second" (Software: Practice and Experience,
//   2021), restated with a two-unit error bound and no table of exact cases.
// * Anything else -- a '+' sign, hexadecimal, inf / nan, more than 19
//   significant digits, a tie or near-tie the product cannot decide, a
//   subnormal or out-of-range value -- is read on the host by mtx.cu's own
//   line parser, line by line; a line that ends before its entry does
//   (an entry spread over lines) sends the whole file to the host reader.
// * The first nnz entries (the non-blank lines by rank, a scan) are checked
//   for range and triangles, and the kept ones compacted in file order.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "abhsf/abhsf_test.h"
#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

#include "pow5_table.inc"

__device__ const unsigned long long kPow5Dev[] = {ABHSF_POW5_WORDS};
__device__ const short kPow5ExpDev[] = {ABHSF_POW5_EXPS};
const unsigned long long kPow5Host[] = {ABHSF_POW5_WORDS};
const short kPow5ExpHost[] = {ABHSF_POW5_EXPS};
static_assert(sizeof(kPow5Host) == 2 * 8 * (ABHSF_POW5_MAX - ABHSF_POW5_MIN + 1), "one 128-bit word per exponent");
static_assert(sizeof(kPow5ExpHost) == 2 * (ABHSF_POW5_MAX - ABHSF_POW5_MIN + 1), "one exponent per power");

struct pow5_view {
    const unsigned long long* words;
    const short* exps;
};

__host__ __device__ inline int clz64(uint64_t x)
{
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

__host__ __device__ inline uint64_t mulhi64(uint64_t a, uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

__host__ __device__ inline double bits_to_double(uint64_t b)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    std::memcpy(&d, &b, sizeof d);
    return d;
#endif
}

// w 10^q (w > 0) rounded to the nearest double, ties to even.  With W = w
// shifted so that its top bit is set and T = floor(5^q 2^(127 - e5)), the
// 128-bit (hi, lo) = floor(W T / 2^64) is at most 2 units of lo below the
// exact W 5^q 2^(127 - e5) / 2^64 (T is short by less than 1, W < 2^64).  The
// value is (hi, lo) 2^(q + e5 - 63 - lz), its leading bit bit 126 or 127 of
// (hi, lo); the 53 bits from there are the significand and the bits below
// decide the rounding -- unless they lie within 2 units below one half, where
// the exact value could be below, at or above the half.  Returns false there,
// and for results outside the normal range.  For 0 <= q <= 55, T is 5^q
// itself and the product's lowest word settles every case.
__host__ __device__ inline bool round_decimal(uint64_t w, int q, const pow5_view& T, double& out)
{
    if (q < ABHSF_POW5_MIN || q > ABHSF_POW5_MAX)
        return false;
    const int k = q - ABHSF_POW5_MIN;
    const uint64_t t1 = T.words[2 * k], t0 = T.words[2 * k + 1];
    const int e5 = T.exps[k];
    const int lz = clz64(w);
    const uint64_t W = w << lz;
    const uint64_t a1 = mulhi64(W, t1), a0 = W * t1, b1 = mulhi64(W, t0);
    const uint64_t lo = a0 + b1;
    const uint64_t hi = a1 + (lo < a0 ? 1u : 0u);
    const int upper = (int)(hi >> 63);
    const int sh = 10 + upper;  // bits of hi below the 53-bit significand
    const uint64_t rh = hi & ((uint64_t(1) << sh) - 1), half = uint64_t(1) << (sh - 1);
    uint64_t mant = hi >> sh;
    if (q >= 0 && q <= 55) {
        // 5^q fits 128 bits, so T is exact and (hi, lo, W t0 mod 2^64) is the
        // whole product: every case is decided, ties to even
        const uint64_t b0 = W * t0;
        const bool above = rh > half || (rh == half && (lo != 0 || b0 != 0));
        const bool tie = rh == half && lo == 0 && b0 == 0;
        mant += (above || (tie && (mant & 1))) ? 1u : 0u;
    } else {
        if ((rh == half && lo == 0) || (rh == half - 1 && lo == ~uint64_t(0)))
            return false;
        mant += (rh > half || (rh == half && lo != 0)) ? 1u : 0u;
    }
    int e = 126 + upper + q + e5 - 63 - lz;  // exponent of the leading bit
    if (mant == (uint64_t(1) << 53)) {
        mant >>= 1;
        ++e;
    }
    const int biased = e + 1023;
    if (biased <= 0 || biased >= 2047)
        return false;
    out = bits_to_double((uint64_t)biased << 52 | (mant & ((uint64_t(1) << 52) - 1)));
    return true;
}

__host__ __device__ inline bool digit(char c) { return c >= '0' && c <= '9'; }

// [-]digits[.digits][(e|E)[+|-]digits] at p, read as std::from_chars reads it
// (an 'e' without exponent digits ends the number before it).  0: *v and
// *end set; 1: left to the host's parser.
__host__ __device__ inline int parse_decimal(const char* p, const char* e, const pow5_view& T, double& v,
                                             const char*& end)
{
    const char* s = p;
    bool neg = false;
    if (s < e && *s == '-') {
        neg = true;
        ++s;
    }
    uint64_t w = 0;
    int nd = 0, q = 0;
    bool any = false;
    for (; s < e && digit(*s); ++s) {
        any = true;
        if (w == 0 && *s == '0')
            continue;  // a leading zero
        if (++nd > 19)
            return 1;
        w = w * 10 + (uint64_t)(*s - '0');
    }
    if (s < e && *s == '.') {
        for (++s; s < e && digit(*s); ++s) {
            any = true;
            --q;
            if (w == 0 && *s == '0')
                continue;
            if (++nd > 19)
                return 1;
            w = w * 10 + (uint64_t)(*s - '0');
        }
    }
    if (!any)
        return 1;
    if (s < e && (*s == 'e' || *s == 'E')) {
        const char* t = s + 1;
        bool eneg = false;
        if (t < e && (*t == '+' || *t == '-')) {
            eneg = *t == '-';
            ++t;
        }
        if (t < e && digit(*t)) {
            int x = 0, xd = 0;
            for (; t < e && digit(*t); ++t) {
                if (++xd > 5)
                    return 1;
                x = x * 10 + (*t - '0');
            }
            q += eneg ? -x : x;
            s = t;
        }
    }
    if (s < e && (*s == 'x' || *s == 'X'))
        return 1;  // the host reads a hexadecimal spelling
    double r = 0.0;
    if (w != 0 && !round_decimal(w, q, T, r))
        return 1;
    v = neg ? -r : r;
    end = s;
    return 0;
}

enum line_kind : uint8_t {
    kBlank = 0,  // white space only
    kEntry = 1,  // an entry, read here
    kHost = 2,   // an entry in a spelling the host reads
    kShort = 3,  // the line ends before its entry does
};

__device__ inline bool space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// An index in plain digits (at most 18: no overflow); false leaves the line to the host.
__device__ inline bool read_index_dev(const char*& p, const char* e, unsigned long long& v)
{
    if (p >= e || !digit(*p))
        return false;
    v = 0;
    int nd = 0;
    for (; p < e && digit(*p); ++p) {
        if (++nd > 18)
            return false;
        v = v * 10 + (unsigned long long)(*p - '0');
    }
    return true;
}

// Line [p, e) (e is one past its line end, or the end of the data).
__device__ uint8_t read_line(const char* p, const char* e, bool pattern, const pow5_view& T, unsigned long long& r,
                             unsigned long long& c, double& v)
{
    while (p < e && space(*p))
        ++p;
    if (p >= e || *p == '\n')
        return kBlank;
    if (!read_index_dev(p, e, r))
        return kHost;
    if (p >= e || *p == '\n')
        return kShort;
    if (!space(*p))
        return kHost;
    while (p < e && space(*p))
        ++p;
    if (p >= e || *p == '\n')
        return kShort;
    if (!read_index_dev(p, e, c))
        return kHost;
    v = 1.0;
    if (pattern)
        return kEntry;  // the rest of the line is not read
    if (p >= e || *p == '\n')
        return kShort;
    if (!space(*p))
        return kHost;
    while (p < e && space(*p))
        ++p;
    if (p >= e || *p == '\n')
        return kShort;
    const char* end = nullptr;
    return parse_decimal(p, e, T, v, end) == 0 ? kEntry : kHost;
}

// Line index, two passes over the bytes: kLineChunk bytes a block, kLineBytes
// a thread.  A line starts at 0 and after every '\n' that is not the last byte.
constexpr int kLineThreads = 256, kLineBytes = 64, kLineChunk = kLineThreads * kLineBytes;

__device__ inline int line_ends(const char* buf, int64_t a, int64_t b)
{
    int k = 0;
    for (int64_t i = a; i < b; ++i)
        k += buf[i] == '\n';
    return k;
}

__global__ void __launch_bounds__(kLineThreads) k_count_lines(int64_t R, const char* __restrict__ buf,
                                                              int64_t* __restrict__ cnt)
{
    using reduce = cub::BlockReduce<int, kLineThreads>;
    __shared__ typename reduce::TempStorage tmp;
    const int64_t a = blockIdx.x * (int64_t)kLineChunk + threadIdx.x * (int64_t)kLineBytes;
    const int k = a < R - 1 ? line_ends(buf, a, min(a + kLineBytes, R - 1)) : 0;  // not the last byte
    const int total = reduce(tmp).Sum(k);
    if (threadIdx.x == 0)
        cnt[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kLineThreads) k_write_lines(int64_t R, const char* __restrict__ buf,
                                                              const int64_t* __restrict__ off,
                                                              int64_t* __restrict__ start)
{
    using scan = cub::BlockScan<int, kLineThreads>;
    __shared__ typename scan::TempStorage tmp;
    const int64_t a = blockIdx.x * (int64_t)kLineChunk + threadIdx.x * (int64_t)kLineBytes;
    const int64_t b = min(a + kLineBytes, R - 1);
    const int k = a < R - 1 ? line_ends(buf, a, b) : 0;
    int before = 0;
    scan(tmp).ExclusiveSum(k, before);
    int64_t at = 1 + off[blockIdx.x] + before;  // start[0] = 0
    for (int64_t i = a; i < b; ++i)
        if (buf[i] == '\n')
            start[at++] = i + 1;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        start[0] = 0;
}

__global__ void k_read_lines(int64_t L, int64_t R, const char* __restrict__ buf, const int64_t* __restrict__ start,
                             bool pattern, uint8_t* __restrict__ kind, unsigned long long* __restrict__ ri,
                             unsigned long long* __restrict__ ci, double* __restrict__ vi,
                             uint8_t* __restrict__ live)
{
    const pow5_view T{kPow5Dev, kPow5ExpDev};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < L; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = start[t], e = t + 1 < L ? start[t + 1] : R;
        unsigned long long r = 0, c = 0;
        double v = 0.0;
        const uint8_t k = read_line(buf + b, buf + e, pattern, T, r, c, v);
        kind[t] = k;
        live[t] = k != kBlank ? 1 : 0;
        ri[t] = r;
        ci[t] = c;
        vi[t] = v;
    }
}

// Lines among the first nnz entries that the host must read.
__global__ void k_host_lines(int64_t L, int64_t nnz, const uint8_t* __restrict__ kind,
                             const int64_t* __restrict__ rank, uint8_t* __restrict__ flag)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < L; t += (int64_t)gridDim.x * blockDim.x)
        flag[t] = (kind[t] >= kHost && rank[t] < nnz) ? 1 : 0;
}

// Byte span and kind of lines idx[0..k).
__global__ void k_line_spans(int64_t k, const int64_t* __restrict__ idx, int64_t L, int64_t R,
                             const int64_t* __restrict__ start, const uint8_t* __restrict__ kind,
                             int64_t* __restrict__ b, int64_t* __restrict__ e, uint8_t* __restrict__ kk)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < k; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = idx[j];
        b[j] = start[t];
        e[j] = t + 1 < L ? start[t + 1] : R;
        kk[j] = kind[t];
    }
}

// The host's reading of lines idx[0..k).
__global__ void k_put_host(int64_t k, const int64_t* __restrict__ idx, const unsigned long long* __restrict__ hr,
                           const unsigned long long* __restrict__ hc, const double* __restrict__ hv,
                           uint8_t* __restrict__ kind, unsigned long long* __restrict__ ri,
                           unsigned long long* __restrict__ ci, double* __restrict__ vi)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < k; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = idx[j];
        kind[t] = kEntry;
        ri[t] = hr[j];
        ci[t] = hc[j];
        vi[t] = hv[j];
    }
}

struct check_out {
    unsigned long long first_range;  // rank of the first entry outside m x n (~0: none)
    int lower, upper;
};

// The first nnz entries: range, triangles, and which are kept (not an
// explicit zero of a real matrix).
__global__ void k_check(int64_t L, int64_t nnz, int64_t m, int64_t n, bool pattern, const uint8_t* __restrict__ kind,
                        const int64_t* __restrict__ rank, const unsigned long long* __restrict__ ri,
                        const unsigned long long* __restrict__ ci, const double* __restrict__ vi,
                        uint8_t* __restrict__ keep, check_out* out)
{
    bool lo = false, up = false;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < L; t += (int64_t)gridDim.x * blockDim.x) {
        uint8_t k = 0;
        if (kind[t] == kEntry && rank[t] < nnz) {
            const unsigned long long r = ri[t], c = ci[t];
            if (r < 1 || c < 1 || r > (unsigned long long)m || c > (unsigned long long)n) {
                atomicMin(&out->first_range, (unsigned long long)rank[t]);
            } else {
                lo = lo || r > c;
                up = up || c > r;
                k = (pattern || vi[t] != 0.0) ? 1 : 0;
            }
        }
        keep[t] = k;
    }
    if (__any_sync(0xffffffffu, lo) && (threadIdx.x & 31) == 0)
        atomicOr(&out->lower, 1);
    if (__any_sync(0xffffffffu, up) && (threadIdx.x & 31) == 0)
        atomicOr(&out->upper, 1);
}

__global__ void k_gather(int64_t k, const int64_t* __restrict__ idx, const unsigned long long* __restrict__ ri,
                         const unsigned long long* __restrict__ ci, const double* __restrict__ vi,
                         int64_t* __restrict__ rows, int64_t* __restrict__ cols, double* __restrict__ vals)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < k; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = idx[j];
        rows[j] = (int64_t)ri[t] - 1;
        cols[j] = (int64_t)ci[t] - 1;
        vals[j] = vi[t];
    }
}

inline unsigned grid_for(int64_t n)
{
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32));
}

// Device memory from the stream-ordered allocator, freed on the stream: the
// reader's scratch neither waits for the device to go idle nor makes it.
template <typename T>
class sbuf {
  public:
    sbuf(size_t count, cudaStream_t st) : st_(st)
    {
        ABHSF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p_), std::max<size_t>(count, 1) * sizeof(T), st));
        dbuf_allocations().fetch_add(1, std::memory_order_relaxed);
    }
    ~sbuf() { cudaFreeAsync(p_, st_); }
    sbuf(const sbuf&) = delete;
    sbuf& operator=(const sbuf&) = delete;
    T* get() const { return p_; }

  private:
    T* p_ = nullptr;
    cudaStream_t st_;
};

// Indices of the set flags (cub select over a counting iterator) into out (n long).
int64_t select_flagged(const uint8_t* flags, int64_t n, int64_t* out, cudaStream_t st)
{
    sbuf<int64_t> count(1, st);
    cub::CountingInputIterator<int64_t> it(0);
    size_t tb = 0;
    ABHSF_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flags, out, count.get(), n, st));
    sbuf<uint8_t> tmp(tb, st);
    ABHSF_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, it, flags, out, count.get(), n, st));
    int64_t k = 0;
    ABHSF_CUDA(cudaMemcpyAsync(&k, count.get(), sizeof k, cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    return k;
}

// The host reader's result, moved to the device.
void host_fallback(const char* path, cudaStream_t st, abhsf_coo_device& out)
{
    abhsf_coo_host h{};
    read_mtx(path, 0, h);
    struct freer {
        abhsf_coo_host* p;
        ~freer()
        {
            std::free(p->rows);
            std::free(p->cols);
            std::free(p->vals);
        }
    } f{&h};
    out.m = h.m;
    out.n = h.n;
    out.nnz = h.nnz;
    out.matrix_type = h.matrix_type;
    out.symmetry = h.symmetry;
    out.stored_triangle = h.stored_triangle;
    out.host_parsed = h.nnz;
    const size_t k = (size_t)std::max<int64_t>(h.nnz, 1);
    ABHSF_CUDA(cudaMalloc(&out.rows, k * sizeof(int64_t)));
    ABHSF_CUDA(cudaMalloc(&out.cols, k * sizeof(int64_t)));
    ABHSF_CUDA(cudaMalloc(&out.vals, k * sizeof(double)));
    if (h.nnz > 0) {
        ABHSF_CUDA(cudaMemcpyAsync(out.rows, h.rows, h.nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(out.cols, h.cols, h.nnz * sizeof(int64_t), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(out.vals, h.vals, h.nnz * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

// Pinned host staging for the file's way to the device: two chunks, so that
// reading one overlaps the copy of the other.  Allocated once per process.
constexpr size_t kStage = size_t(16) << 20;

struct staging {
    std::mutex mu;
    char* p[2] = {nullptr, nullptr};
};

staging& stage()
{
    static staging s;
    return s;
}

// The file into device memory d (size bytes); its first min(size, kStage)
// bytes also into head.  false: not a regular file of that size (the caller
// reads it the plain way).
bool file_to_device(FILE* f, int64_t size, char* d, std::string& head, cudaStream_t st)
{
    staging& S = stage();
    std::lock_guard<std::mutex> lock(S.mu);
    for (int k = 0; k < 2; ++k)
        if (!S.p[k])
            ABHSF_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&S.p[k]), kStage, cudaHostAllocPortable));
    cudaEvent_t ev[2];
    for (auto& e : ev)
        ABHSF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    bool ok = true;
    int64_t off = 0;
    for (int i = 0; off < size; ++i) {
        const int k = i & 1;
        if (i >= 2)
            cudaEventSynchronize(ev[k]);  // the copy that last used this chunk is done
        const size_t want = (size_t)std::min<int64_t>((int64_t)kStage, size - off);
        const size_t got = std::fread(S.p[k], 1, want, f);
        if (got != want) {
            ok = false;
            break;
        }
        if (i == 0)
            head.assign(S.p[0], got);
        ABHSF_CUDA(cudaMemcpyAsync(d + off, S.p[k], got, cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaEventRecord(ev[k], st));
        off += (int64_t)got;
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));  // before the staging is reused
    for (auto& e : ev)
        cudaEventDestroy(e);
    return ok;
}

// Byte copies of lines [b[j], e[j]) of the device text, packed at at[j].
__global__ void k_pack_lines(int64_t k, const char* __restrict__ text, const int64_t* __restrict__ b,
                             const int64_t* __restrict__ e, const int64_t* __restrict__ at, char* __restrict__ out)
{
    for (int64_t j = blockIdx.x; j < k; j += gridDim.x)
        for (int64_t i = b[j] + threadIdx.x; i < e[j]; i += blockDim.x)
            out[at[j] + (i - b[j])] = text[i];
}

}  // namespace

void read_mtx_device(const char* path, cudaStream_t st, abhsf_coo_device& out)
{
    out = abhsf_coo_device{};
    if (!path)
        fail(ABHSF_ERROR_INVALID_VALUE, "path must be non-NULL");
    FILE* f = std::fopen(path, "rb");
    if (!f)
        fail(ABHSF_ERROR_INVALID_VALUE, std::string("cannot open input file: ") + path);
    struct closer {
        FILE* f;
        ~closer() { std::fclose(f); }
    } fc{f};
    int64_t size = -1;
    if (std::fseek(f, 0, SEEK_END) == 0)
        size = (int64_t)std::ftell(f);
    if (size < 0 || std::fseek(f, 0, SEEK_SET) != 0) {
        host_fallback(path, st, out);  // not a seekable file: the host reader
        return;
    }
    sbuf<char> d_file(size, st);
    std::string head;
    if (!file_to_device(f, size, d_file.get(), head, st)) {
        host_fallback(path, st, out);  // the file changed under us: the host reader reports what it finds
        return;
    }
    // banner and size line: from the first chunk (the whole file when they
    // reach past it)
    mtx_header hd;
    const bool whole = (int64_t)head.size() == size;
    try {
        hd = read_mtx_header(head);
    } catch (...) {
        if (whole)
            throw;
        hd.pos = head.size();  // comments longer than the first chunk: read below
    }
    if (!whole && hd.pos >= head.size())  // the size line may not have ended inside the chunk
        hd = read_mtx_header(read_file(path));
    const bool pattern = hd.type == ABHSF_MATRIX_BINARY;
    const int64_t R = size - (int64_t)hd.pos;
    const char* text = d_file.get() + hd.pos;  // device
    out.m = hd.m;
    out.n = hd.n;
    out.matrix_type = hd.type;
    out.symmetry = hd.symmetry;
    if (hd.nnz == 0 || R <= 0) {
        if (hd.nnz > 0)
            fail(ABHSF_ERROR_INVALID_VALUE, "could not read matrix element (fewer entries than declared)");
        out.stored_triangle = hd.symmetry == ABHSF_SYMMETRY_GENERAL ? 0 : 2;
        ABHSF_CUDA(cudaMalloc(&out.rows, sizeof(int64_t)));
        ABHSF_CUDA(cudaMalloc(&out.cols, sizeof(int64_t)));
        ABHSF_CUDA(cudaMalloc(&out.vals, sizeof(double)));
        return;
    }
    // the lines
    const int64_t nb = (R + kLineChunk - 1) / kLineChunk;
    sbuf<int64_t> bcnt(nb, st), boff(nb, st);
    k_count_lines<<<(unsigned)nb, kLineThreads, 0, st>>>(R, text, bcnt.get());
    ABHSF_CUDA(cudaGetLastError());
    int64_t L = 0;
    {
        size_t tb = 0;
        ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, bcnt.get(), boff.get(), nb, st));
        sbuf<uint8_t> tmp(tb, st);
        ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, bcnt.get(), boff.get(), nb, st));
        int64_t lo = 0, lc = 0;
        ABHSF_CUDA(cudaMemcpyAsync(&lo, boff.get() + nb - 1, sizeof lo, cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(&lc, bcnt.get() + nb - 1, sizeof lc, cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaStreamSynchronize(st));
        L = 1 + lo + lc;
    }
    sbuf<int64_t> start(L, st);
    k_write_lines<<<(unsigned)nb, kLineThreads, 0, st>>>(R, text, boff.get(), start.get());
    ABHSF_CUDA(cudaGetLastError());
    sbuf<uint8_t> kind(L, st), live(L, st), flag(L, st);
    sbuf<unsigned long long> ri(L, st), ci(L, st);
    sbuf<double> vi(L, st);
    sbuf<int64_t> rank(L, st), idx(L, st);
    k_read_lines<<<grid_for(L), 256, 0, st>>>(L, R, text, start.get(), pattern, kind.get(), ri.get(), ci.get(),
                                              vi.get(), live.get());
    ABHSF_CUDA(cudaGetLastError());
    int64_t entries = 0;  // non-blank lines
    {
        // rank = exclusive count of non-blank lines before each line
        size_t tb = 0;
        ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, live.get(), rank.get(), L, st));
        sbuf<uint8_t> tmp(tb, st);
        ABHSF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, live.get(), rank.get(), L, st));
        int64_t last_rank = 0;
        uint8_t last_live = 0;
        ABHSF_CUDA(cudaMemcpyAsync(&last_rank, rank.get() + L - 1, sizeof last_rank, cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(&last_live, live.get() + L - 1, 1, cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaStreamSynchronize(st));
        entries = last_rank + last_live;
    }
    // lines the host reads
    k_host_lines<<<grid_for(L), 256, 0, st>>>(L, hd.nnz, kind.get(), rank.get(), flag.get());
    ABHSF_CUDA(cudaGetLastError());
    const int64_t nh = select_flagged(flag.get(), L, idx.get(), st);
    if (nh > 0) {
        std::vector<int64_t> hb(nh), he(nh), at(nh + 1, 0);
        std::vector<uint8_t> hk(nh);
        sbuf<int64_t> d_b(nh, st), d_e(nh, st), d_at(nh + 1, st);
        sbuf<uint8_t> d_k(nh, st);
        k_line_spans<<<grid_for(nh), 256, 0, st>>>(nh, idx.get(), L, R, start.get(), kind.get(), d_b.get(), d_e.get(),
                                                   d_k.get());
        ABHSF_CUDA(cudaGetLastError());
        ABHSF_CUDA(cudaMemcpyAsync(hb.data(), d_b.get(), nh * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(he.data(), d_e.get(), nh * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaMemcpyAsync(hk.data(), d_k.get(), nh, cudaMemcpyDeviceToHost, st));
        ABHSF_CUDA(cudaStreamSynchronize(st));
        for (int64_t j = 0; j < nh; ++j) {
            if (hk[j] == kShort) {  // an entry spread over lines: the host reader, on the whole file
                host_fallback(path, st, out);
                return;
            }
            at[j + 1] = at[j] + (he[j] - hb[j]);
        }
        // the lines' text, packed on the device and brought over in one copy
        std::string lines((size_t)at[nh], '\0');
        {
            sbuf<char> packed(at[nh], st);
            ABHSF_CUDA(cudaMemcpyAsync(d_at.get(), at.data(), (nh + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
            k_pack_lines<<<(unsigned)std::min<int64_t>(nh, 4096), 128, 0, st>>>(nh, text, d_b.get(), d_e.get(),
                                                                             d_at.get(), packed.get());
            ABHSF_CUDA(cudaGetLastError());
            ABHSF_CUDA(cudaMemcpyAsync(&lines[0], packed.get(), at[nh], cudaMemcpyDeviceToHost, st));
            ABHSF_CUDA(cudaStreamSynchronize(st));
        }
        std::vector<unsigned long long> hr(nh), hc(nh);
        std::vector<double> hv(nh);
        std::string line;
        for (int64_t j = 0; j < nh; ++j) {
            // the line alone (no line end), so that the host's parse cannot run into the next
            line.assign(lines, (size_t)at[j], (size_t)(at[j + 1] - at[j]));
            while (!line.empty() && line.back() == '\n')
                line.pop_back();
            if (parse_entry_host(line.c_str(), line.c_str() + line.size(), pattern, hr[j], hc[j], hv[j]) != 0) {
                host_fallback(path, st, out);  // not an entry of its own line: the host reader decides
                return;
            }
        }
        sbuf<unsigned long long> d_hr(nh, st), d_hc(nh, st);
        sbuf<double> d_hv(nh, st);
        ABHSF_CUDA(cudaMemcpyAsync(d_hr.get(), hr.data(), nh * sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(d_hc.get(), hc.data(), nh * sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
        ABHSF_CUDA(cudaMemcpyAsync(d_hv.get(), hv.data(), nh * sizeof(double), cudaMemcpyHostToDevice, st));
        k_put_host<<<grid_for(nh), 256, 0, st>>>(nh, idx.get(), d_hr.get(), d_hc.get(), d_hv.get(), kind.get(),
                                                 ri.get(), ci.get(), vi.get());
        ABHSF_CUDA(cudaGetLastError());
        ABHSF_CUDA(cudaStreamSynchronize(st));  // before the host vectors go
    }
    out.host_parsed = nh;
    // checks and the kept entries
    sbuf<check_out> chk(1, st);
    const check_out init{~0ull, 0, 0};
    ABHSF_CUDA(cudaMemcpyAsync(chk.get(), &init, sizeof init, cudaMemcpyHostToDevice, st));
    k_check<<<grid_for(L), 256, 0, st>>>(L, hd.nnz, hd.m, hd.n, pattern, kind.get(), rank.get(), ri.get(), ci.get(),
                                         vi.get(), flag.get(), chk.get());
    ABHSF_CUDA(cudaGetLastError());
    check_out res{};
    ABHSF_CUDA(cudaMemcpyAsync(&res, chk.get(), sizeof res, cudaMemcpyDeviceToHost, st));
    ABHSF_CUDA(cudaStreamSynchronize(st));
    if (res.first_range != ~0ull)
        fail(ABHSF_ERROR_INDEX_OUT_OF_RANGE, "an element lies outside the declared m x n");
    if (entries < hd.nnz)
        fail(ABHSF_ERROR_INVALID_VALUE, "could not read matrix element (fewer entries than declared)");
    if (hd.symmetry != ABHSF_SYMMETRY_GENERAL && res.lower && res.upper)
        fail(ABHSF_ERROR_INVALID_VALUE, "elements from both L and U parts stored for not-unsymmetric matrix");
    out.stored_triangle = hd.symmetry == ABHSF_SYMMETRY_GENERAL ? 0 : (res.lower ? 1 : 2);
    const int64_t kept = select_flagged(flag.get(), L, idx.get(), st);
    out.nnz = kept;
    const size_t k = (size_t)std::max<int64_t>(kept, 1);
    ABHSF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&out.rows), k * sizeof(int64_t), st));
    ABHSF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&out.cols), k * sizeof(int64_t), st));
    ABHSF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&out.vals), k * sizeof(double), st));
    if (kept > 0) {
        k_gather<<<grid_for(kept), 256, 0, st>>>(kept, idx.get(), ri.get(), ci.get(), vi.get(), out.rows, out.cols,
                                                 out.vals);
        ABHSF_CUDA(cudaGetLastError());
    }
    ABHSF_CUDA(cudaStreamSynchronize(st));
}

}  // namespace abhsf

extern "C" int32_t abhsf_test_parse_decimal(const char* text, int64_t len, double* value, int64_t* used)
{
    if (!text || len < 0)
        return 1;
    const abhsf::pow5_view T{abhsf::kPow5Host, abhsf::kPow5ExpHost};
    double v = 0.0;
    const char* end = text;
    if (abhsf::parse_decimal(text, text + len, T, v, end) != 0)
        return 1;
    if (value)
        *value = v;
    if (used)
        *used = (int64_t)(end - text);
    return 0;
}
