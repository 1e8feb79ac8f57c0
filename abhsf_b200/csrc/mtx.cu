// mtx.cu -- Matrix Market ingest on the host (the library's data loader).
//
// Reads a coordinate-format Matrix Market file the way the reference's
// read_mtx_real_or_binary does (include/abhsf/utils/matrix_market_reader.h:146-200,
// banner and size line through mmio's mm_read_banner / mm_read_mtx_crd_size):
// real or pattern matrices (pattern values 1.0), 1-based indices made 0-based,
// explicit zeros of a real matrix dropped, a symmetric / skew / hermitian
// file's stored triangle kept as stored (no expansion) and rejected when both
// triangles appear.  Values are converted by strtod, which rounds exactly as
// the reference's fscanf("%lf") does.  Unlike the reference, indices outside
// the declared m x n are an error here, and the entry lines are parsed by
// several host threads at once (the file is read whole, split at line ends).
// Numbers in their plain spellings go through std::from_chars, which rounds
// a decimal exactly as strtod does; every other spelling (a sign on an index,
// '+', hexadecimal, inf / nan words, a value out of the double range) goes
// through strtoull / strtod as before.
#include <algorithm>
#include <cctype>
#include <charconv>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "internal.cuh"

namespace abhsf {
namespace {

std::string lower(std::string s)
{
    for (char& c : s)
        c = (char)std::tolower((unsigned char)c);
    return s;
}

// The next line of buf starting at pos (without the line end); pos moves past it.
bool next_line(const std::string& buf, size_t& pos, std::string& line)
{
    if (pos >= buf.size())
        return false;
    size_t e = buf.find('\n', pos);
    if (e == std::string::npos)
        e = buf.size();
    line.assign(buf, pos, e - pos);
    if (!line.empty() && line.back() == '\r')
        line.pop_back();
    pos = e + 1;
    return true;
}

struct chunk_out {
    std::vector<int64_t> rows, cols;
    std::vector<double> vals;
    int64_t entries = 0, zeros = 0;
    bool lower = false, upper = false, bad = false, range = false, oom = false;
};

inline bool is_space(char c)
{
    return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

// An index at p (leading white space skipped, as strtoull skips it); false if
// none can be read.  p is within a NUL-terminated buffer.
inline bool read_index(const char*& p, const char* e, unsigned long long& v)
{
    const char* s = p;
    while (s < e && is_space(*s))
        ++s;
    if (s < e && *s >= '0' && *s <= '9') {
        const auto r = std::from_chars(s, e, v);
        if (r.ec == std::errc()) {
            p = r.ptr;
            return true;
        }
    }
    char* q = nullptr;
    errno = 0;
    v = std::strtoull(p, &q, 10);
    if (q == p || errno)
        return false;
    p = q;
    return true;
}

// A value at p, rounded as strtod rounds it.
inline bool read_value(const char*& p, const char* e, double& v)
{
    const char* s = p;
    while (s < e && is_space(*s))
        ++s;
    if (s < e && ((*s >= '0' && *s <= '9') || *s == '-' || *s == '.')) {
        const auto r = std::from_chars(s, e, v);
        if (r.ec == std::errc() && (r.ptr == e || (*r.ptr != 'x' && *r.ptr != 'X'))) {
            p = r.ptr;
            return true;
        }
    }
    char* q = nullptr;
    v = std::strtod(p, &q);
    if (q == p)
        return false;
    p = q;
    return true;
}

// Entries of buf[b, e) (whole lines), at most `limit` of them.
void parse_chunk(const char* b, const char* e, bool pattern, int64_t m, int64_t n, int64_t limit, chunk_out& o)
{
    if (e <= b)
        return;
    // about 24 bytes per entry line in the files this reads; growth past it is amortised
    const size_t guess = size_t(e - b) / 24 + 16;
    o.rows.reserve(guess);
    o.cols.reserve(guess);
    if (!pattern)
        o.vals.reserve(guess);
    const char* p = b;
    while (p < e && o.entries < limit) {
        while (p < e && is_space(*p))
            ++p;
        if (p >= e)
            break;
        unsigned long long r, c;
        if (!read_index(p, e, r) || !read_index(p, e, c)) {
            o.bad = true;
            return;
        }
        double v = 1.0;
        if (!pattern && !read_value(p, e, v)) {
            o.bad = true;
            return;
        }
        while (p < e && *p != '\n')  // the rest of the line (a complex part, a comment) is not read
            ++p;
        ++o.entries;
        // unsigned compares: a signed index ("-1") wraps to 2^64 - 1 and fails r <= m
        if (r < 1 || c < 1 || r > (unsigned long long)m || c > (unsigned long long)n) {
            o.range = true;
            return;
        }
        const int64_t i = (int64_t)r - 1, j = (int64_t)c - 1;
        if (i > j)
            o.lower = true;
        if (j > i)
            o.upper = true;
        if (!pattern && v == 0.0) {
            ++o.zeros;
            continue;
        }
        o.rows.push_back(i);
        o.cols.push_back(j);
        o.vals.push_back(v);
    }
}

}  // namespace

std::string read_file(const char* path)
{
    if (!path)
        fail(ABHSF_ERROR_INVALID_VALUE, "path must be non-NULL");
    FILE* f = std::fopen(path, "rb");
    if (!f)
        fail(ABHSF_ERROR_INVALID_VALUE, std::string("cannot open input file: ") + path);
    std::string buf;
    // one read of the whole file when its size is known, else by pieces
    long size = -1;
    if (std::fseek(f, 0, SEEK_END) == 0)
        size = std::ftell(f);
    if (size >= 0 && std::fseek(f, 0, SEEK_SET) == 0) {
        buf.resize(size_t(size));
        buf.resize(std::fread(&buf[0], 1, buf.size(), f));
    }
    char tmp[1 << 16];
    size_t k;
    while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0)
        buf.append(tmp, k);
    std::fclose(f);
    return buf;
}

mtx_header read_mtx_header(const std::string& buf)
{
    mtx_header h;
    size_t pos = 0;
    std::string line;
    // banner: %%MatrixMarket matrix coordinate <field> <symmetry>
    if (!next_line(buf, pos, line))
        fail(ABHSF_ERROR_INVALID_VALUE, "could not process Matrix Market banner");
    char w[5][64] = {};
    if (std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5 ||
        std::string(w[0]) != "%%MatrixMarket")
        fail(ABHSF_ERROR_INVALID_VALUE, "could not process Matrix Market banner");
    if (lower(w[1]) != "matrix" || lower(w[2]) != "coordinate")
        fail(ABHSF_ERROR_UNSUPPORTED, "only sparse matrices in coordinate format are supported");
    const std::string field = lower(w[3]), sym = lower(w[4]);
    if (field == "pattern")
        h.type = ABHSF_MATRIX_BINARY;
    else if (field == "real")
        h.type = ABHSF_MATRIX_REAL;
    else if (field == "integer" || field == "complex")
        fail(ABHSF_ERROR_UNSUPPORTED, "only real and pattern matrices are read (read_mtx_real_or_binary)");
    else
        fail(ABHSF_ERROR_INVALID_VALUE, "unsupported matrix type");
    if (sym == "general")
        h.symmetry = ABHSF_SYMMETRY_GENERAL;
    else if (sym == "symmetric")
        h.symmetry = ABHSF_SYMMETRY_SYMMETRIC;
    else if (sym == "skew-symmetric")
        h.symmetry = ABHSF_SYMMETRY_SKEW;
    else if (sym == "hermitian")
        h.symmetry = ABHSF_SYMMETRY_HERMITIAN;
    else
        fail(ABHSF_ERROR_INVALID_VALUE, "unsupported type of matrix symmetry");
    // comments, then the size line
    for (;;) {
        if (!next_line(buf, pos, line))
            fail(ABHSF_ERROR_INVALID_VALUE, "could not retrieve matrix sizes");
        if (!line.empty() && line[0] == '%')
            continue;
        if (line.find_first_not_of(" \t") == std::string::npos)
            continue;
        if (std::sscanf(line.c_str(), "%lld %lld %lld", &h.m, &h.n, &h.nnz) != 3 || h.m <= 0 || h.n <= 0 ||
            h.nnz < 0)
            fail(ABHSF_ERROR_INVALID_VALUE, "could not retrieve matrix sizes");
        break;
    }
    // a size line without a line end leaves pos one past the buffer
    h.pos = std::min(pos, buf.size());
    return h;
}

int parse_entry_host(const char* b, const char* e, bool pattern, unsigned long long& r, unsigned long long& c,
                     double& v)
{
    const char* p = b;
    while (p < e && is_space(*p))
        ++p;
    if (p >= e)
        return 1;
    v = 1.0;
    if (!read_index(p, e, r) || !read_index(p, e, c) || (!pattern && !read_value(p, e, v)))
        return 2;
    return 0;
}

void read_mtx(const char* path, int threads, abhsf_coo_host& out)
{
    out = abhsf_coo_host{};
    const std::string buf = read_file(path);
    const mtx_header hd = read_mtx_header(buf);
    const int type = hd.type, symmetry = hd.symmetry;
    const long long m = hd.m, n = hd.n, nnz = hd.nnz;
    const size_t pos = hd.pos;
    // entry lines: split the rest at line ends over the threads
    const size_t rest = buf.size() - pos;
    int T = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    T = (int)std::max<size_t>(1, std::min<size_t>((size_t)T, rest / (1 << 20) + 1));
    std::vector<size_t> cut(T + 1, pos);
    cut[T] = buf.size();
    for (int t = 1; t < T; ++t) {
        size_t c = pos + rest * t / T;
        c = std::max(c, cut[t - 1]);
        const size_t e = buf.find('\n', c);
        cut[t] = e == std::string::npos ? buf.size() : e + 1;
    }
    std::vector<chunk_out> parts(T);
    const bool pattern = type == ABHSF_MATRIX_BINARY;
    {
        std::vector<std::thread> pool;
        for (int t = 0; t < T; ++t)
            pool.emplace_back([&, t] {
                try {  // nothing may leave a worker thread
                    parse_chunk(buf.data() + cut[t], buf.data() + cut[t + 1], pattern, m, n, (int64_t)nnz, parts[t]);
                } catch (...) {
                    parts[t].oom = true;
                }
            });
        for (auto& th : pool)
            th.join();
    }
    for (const chunk_out& c : parts)
        if (c.oom)
            fail(ABHSF_ERROR_OUT_OF_MEMORY, "host allocation failed while parsing");
    // the first nnz entries in file order, as the reference reads exactly nnz
    // (lines after them are not looked at)
    int64_t left = nnz, kept = 0;
    bool L = false, U = false;
    std::vector<int64_t> take;
    for (int t = 0; t < T && left > 0; ++t) {
        if (parts[t].entries > left || (parts[t].bad && parts[t].entries >= left)) {
            chunk_out again;  // this chunk holds the nnz-th entry: read only up to it
            parse_chunk(buf.data() + cut[t], buf.data() + cut[t + 1], pattern, m, n, left, again);
            parts[t] = std::move(again);
        }
        const chunk_out& c = parts[t];
        if (c.range)
            fail(ABHSF_ERROR_INDEX_OUT_OF_RANGE, "an element lies outside the declared m x n");
        if (c.bad)
            fail(ABHSF_ERROR_INVALID_VALUE, "could not read matrix element");
        take.push_back((int64_t)c.rows.size());
        L = L || c.lower;
        U = U || c.upper;
        left -= c.entries;
    }
    if (left > 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "could not read matrix element (fewer entries than declared)");
    const int used = (int)take.size();
    if (symmetry != ABHSF_SYMMETRY_GENERAL && L && U)
        fail(ABHSF_ERROR_INVALID_VALUE, "elements from both L and U parts stored for not-unsymmetric matrix");
    for (int64_t k : take)
        kept += k;
    out.m = m;
    out.n = n;
    out.nnz = kept;
    out.matrix_type = type;
    out.symmetry = symmetry;
    out.stored_triangle = symmetry == ABHSF_SYMMETRY_GENERAL ? 0 : (L ? 1 : 2);
    out.rows = static_cast<int64_t*>(std::malloc(std::max<int64_t>(kept, 1) * sizeof(int64_t)));
    out.cols = static_cast<int64_t*>(std::malloc(std::max<int64_t>(kept, 1) * sizeof(int64_t)));
    out.vals = static_cast<double*>(std::malloc(std::max<int64_t>(kept, 1) * sizeof(double)));
    if (!out.rows || !out.cols || !out.vals) {
        std::free(out.rows);
        std::free(out.cols);
        std::free(out.vals);
        out = abhsf_coo_host{};
        fail(ABHSF_ERROR_OUT_OF_MEMORY, "host allocation failed");
    }
    std::vector<int64_t> at(used + 1, 0);
    for (int t = 0; t < used; ++t)
        at[t + 1] = at[t] + take[t];
    auto copy_part = [&](int t) {
        const chunk_out& c = parts[t];
        std::copy(c.rows.begin(), c.rows.begin() + take[t], out.rows + at[t]);
        std::copy(c.cols.begin(), c.cols.begin() + take[t], out.cols + at[t]);
        std::copy(c.vals.begin(), c.vals.begin() + take[t], out.vals + at[t]);
    };
    if (used > 1) {
        std::vector<std::thread> pool;
        for (int t = 0; t < used; ++t)
            pool.emplace_back(copy_part, t);
        for (auto& th : pool)
            th.join();
    } else if (used == 1) {
        copy_part(0);
    }
}

// ---------------------------------------------------------------- .mm binary
// The reference's binary matrix file, written by utils/mtx2mm/mtx2mm.cpp:102-135
// (and read back by the commented-out read_mm of preprocessing/test.cpp:194-235):
// five u64 words m, n, nnz, type (matrix_type_t numbering: 0 pattern, 1 integer,
// 2 real, 3 complex) and a symmetry flag (mtx2mm's bool `hermit`), then u32
// rows[nnz] and u32 cols[nnz] (0-based), then the values by type: f64[nnz] for
// real, none for pattern.  The flag is written here as 0 for a general matrix and
// 1 / 2 / 3 for symmetric / hermitian / skew, so a reader that takes it as a
// bool (the reference) sees "not general" for all three, and a 1 written by
// mtx2mm reads as symmetric.

namespace {

struct file_closer {
    FILE* f;
    ~file_closer()
    {
        if (f)
            std::fclose(f);
    }
};

constexpr uint64_t kMmHeaderWords = 5;

void set_triangle(abhsf_coo_host& o)
{
    bool L = false, U = false;
    for (int64_t k = 0; k < o.nnz; ++k) {
        L = L || o.rows[k] > o.cols[k];
        U = U || o.cols[k] > o.rows[k];
    }
    if (o.symmetry != ABHSF_SYMMETRY_GENERAL && L && U)
        fail(ABHSF_ERROR_INVALID_VALUE, "elements from both L and U parts stored for not-unsymmetric matrix");
    o.stored_triangle = o.symmetry == ABHSF_SYMMETRY_GENERAL ? 0 : (L ? 1 : 2);
}

}  // namespace

void read_mm(const char* path, abhsf_coo_host& out)
{
    out = abhsf_coo_host{};
    if (!path)
        fail(ABHSF_ERROR_INVALID_VALUE, "path must be non-NULL");
    file_closer fc{std::fopen(path, "rb")};
    if (!fc.f)
        fail(ABHSF_ERROR_INVALID_VALUE, std::string("cannot open input file: ") + path);
    uint64_t h[kMmHeaderWords];
    if (std::fread(h, sizeof(uint64_t), kMmHeaderWords, fc.f) != kMmHeaderWords)
        fail(ABHSF_ERROR_INVALID_VALUE, "could not read the .mm header");
    const uint64_t m = h[0], n = h[1], nnz = h[2], type = h[3], flag = h[4];
    if (type == ABHSF_MATRIX_INTEGER || type == ABHSF_MATRIX_COMPLEX)
        fail(ABHSF_ERROR_UNSUPPORTED, "only real and pattern matrices are read (read_mtx_real_or_binary)");
    if (type != ABHSF_MATRIX_REAL && type != ABHSF_MATRIX_BINARY)
        fail(ABHSF_ERROR_INVALID_VALUE, "unsupported matrix type");
    if (flag > 3)
        fail(ABHSF_ERROR_INVALID_VALUE, "unsupported type of matrix symmetry");
    if (m < 1 || n < 1 || m > (uint64_t(1) << 32) || n > (uint64_t(1) << 32))
        fail(ABHSF_ERROR_INVALID_VALUE, "matrix sizes out of the .mm range (1 .. 2^32)");
    // the file holds exactly the arrays the header announces
    const uint64_t per = 8 + (type == ABHSF_MATRIX_REAL ? 8 : 0);
    if (std::fseek(fc.f, 0, SEEK_END) != 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "cannot seek in the .mm file");
    const long size = std::ftell(fc.f);
    if (size < 0 || nnz > (uint64_t(size) / per) || uint64_t(size) != 8 * kMmHeaderWords + nnz * per)
        fail(ABHSF_ERROR_INVALID_VALUE, "the .mm file size does not match its header");
    std::fseek(fc.f, long(8 * kMmHeaderWords), SEEK_SET);
    std::vector<uint32_t> r32(nnz), c32(nnz);
    std::vector<double> v(type == ABHSF_MATRIX_REAL ? nnz : 0);
    if (std::fread(r32.data(), 4, nnz, fc.f) != nnz || std::fread(c32.data(), 4, nnz, fc.f) != nnz ||
        std::fread(v.data(), 8, v.size(), fc.f) != v.size())
        fail(ABHSF_ERROR_INVALID_VALUE, "could not read matrix element");
    // explicit zeros of a real matrix are dropped, as read_mtx_real_or_binary
    // drops them from the text file the .mm was made from
    int64_t kept = 0;
    for (uint64_t k = 0; k < nnz; ++k) {
        if (r32[k] >= m || c32[k] >= n)
            fail(ABHSF_ERROR_INDEX_OUT_OF_RANGE, "an element lies outside the declared m x n");
        kept += type == ABHSF_MATRIX_BINARY || v[k] != 0.0;
    }
    abhsf_coo_host o{};
    o.m = int64_t(m);
    o.n = int64_t(n);
    o.matrix_type = int32_t(type);
    o.symmetry = flag == 0 ? ABHSF_SYMMETRY_GENERAL
                           : (flag == 1 ? ABHSF_SYMMETRY_SYMMETRIC
                                        : (flag == 2 ? ABHSF_SYMMETRY_HERMITIAN : ABHSF_SYMMETRY_SKEW));
    o.rows = static_cast<int64_t*>(std::malloc(std::max<int64_t>(kept, 1) * sizeof(int64_t)));
    o.cols = static_cast<int64_t*>(std::malloc(std::max<int64_t>(kept, 1) * sizeof(int64_t)));
    o.vals = static_cast<double*>(std::malloc(std::max<int64_t>(kept, 1) * sizeof(double)));
    if (!o.rows || !o.cols || !o.vals) {
        std::free(o.rows);
        std::free(o.cols);
        std::free(o.vals);
        fail(ABHSF_ERROR_OUT_OF_MEMORY, "host allocation failed");
    }
    int64_t j = 0;
    for (uint64_t k = 0; k < nnz; ++k) {
        const double val = type == ABHSF_MATRIX_BINARY ? 1.0 : v[k];
        if (val == 0.0)
            continue;
        o.rows[j] = r32[k];
        o.cols[j] = c32[k];
        o.vals[j] = val;
        ++j;
    }
    o.nnz = kept;
    try {
        set_triangle(o);
    } catch (...) {
        std::free(o.rows);
        std::free(o.cols);
        std::free(o.vals);
        throw;
    }
    out = o;
}

void write_mm(const char* path, const abhsf_coo_host& a)
{
    if (!path)
        fail(ABHSF_ERROR_INVALID_VALUE, "path must be non-NULL");
    if (a.matrix_type != ABHSF_MATRIX_REAL && a.matrix_type != ABHSF_MATRIX_BINARY)
        fail(ABHSF_ERROR_UNSUPPORTED, "only real and pattern matrices are written");
    if (a.symmetry < ABHSF_SYMMETRY_SYMMETRIC || a.symmetry > ABHSF_SYMMETRY_GENERAL)
        fail(ABHSF_ERROR_INVALID_VALUE, "symmetry must be an abhsf_symmetry");
    if (a.m < 1 || a.n < 1 || a.m > (int64_t(1) << 32) || a.n > (int64_t(1) << 32) || a.nnz < 0)
        fail(ABHSF_ERROR_INVALID_VALUE, "sizes out of the .mm range (m, n in 1 .. 2^32, nnz >= 0)");
    const bool real = a.matrix_type == ABHSF_MATRIX_REAL;
    if (a.nnz > 0 && (!a.rows || !a.cols || (real && !a.vals)))
        fail(ABHSF_ERROR_INVALID_VALUE, "rows, cols (and vals of a real matrix) must be non-NULL");
    for (int64_t k = 0; k < a.nnz; ++k)
        if (a.rows[k] < 0 || a.rows[k] >= a.m || a.cols[k] < 0 || a.cols[k] >= a.n)
            fail(ABHSF_ERROR_INDEX_OUT_OF_RANGE, "an element lies outside m x n");
    file_closer fc{std::fopen(path, "wb")};
    if (!fc.f)
        fail(ABHSF_ERROR_INVALID_VALUE, std::string("cannot open output file: ") + path);
    const uint64_t flag = a.symmetry == ABHSF_SYMMETRY_GENERAL
                              ? 0
                              : (a.symmetry == ABHSF_SYMMETRY_SYMMETRIC ? 1
                                                                        : (a.symmetry == ABHSF_SYMMETRY_HERMITIAN ? 2 : 3));
    const uint64_t h[kMmHeaderWords] = {uint64_t(a.m), uint64_t(a.n), uint64_t(a.nnz), uint64_t(a.matrix_type), flag};
    bool ok = std::fwrite(h, sizeof(uint64_t), kMmHeaderWords, fc.f) == kMmHeaderWords;
    std::vector<uint32_t> buf;
    for (const int64_t* idx : {a.rows, a.cols}) {
        constexpr int64_t kChunk = 1 << 20;
        for (int64_t k0 = 0; ok && k0 < a.nnz; k0 += kChunk) {
            const int64_t k1 = std::min(a.nnz, k0 + kChunk);
            buf.assign(idx + k0, idx + k1);
            ok = std::fwrite(buf.data(), 4, size_t(k1 - k0), fc.f) == size_t(k1 - k0);
        }
    }
    if (ok && real && a.nnz > 0)
        ok = std::fwrite(a.vals, 8, size_t(a.nnz), fc.f) == size_t(a.nnz);
    ok = (std::fflush(fc.f) == 0) && ok;
    if (!ok)
        fail(ABHSF_ERROR_INVALID_VALUE, std::string("could not write ") + path);
}

}  // namespace abhsf
