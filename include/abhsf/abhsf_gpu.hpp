// abhsf_gpu.hpp -- header-only C++ wrapper over the C ABI in abhsf_gpu.h with
// the call shape the reference's formats share:
//
//   elements_t elements;  matrix_properties props;   // as in the reference
//   abhsf::gpu_matrix A;
//   A.from_elements(elements, props);                 // spmv/bottlenecks/spmv.cpp:43-49
//   A.spmv(x, y);                                     // y += A x, spmv/bottlenecks/spmv.cpp:58-64
//   A.release();                                      // spmv/bottlenecks/spmv.cpp:125-133
//
// Errors throw std::runtime_error, the reference's convention
// (include/abhsf/utils/matrix_market_reader.h:45-55).  Element containers are
// anything iterable whose items support std::get<0..2> (row, col, value), such
// as the reference's std::vector<std::tuple<int, int, double>>
// (spmv/unified/spmv.cpp:68-69).  Unlike the reference's from_elements, the
// caller's elements are not reordered.
//
// The reader has the reference's call shape too:
//
//   abhsf::read_mtx_real_or_binary(filename, elements, props);  // matrix_market_reader.h:146-200
//
// with the library's multi-threaded parser behind it (abhsf_read_mtx), and
// abhsf::read_mm reads the binary .mm layout of utils/mtx2mm the same way.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "abhsf_gpu.h"

namespace abhsf {

inline void throw_if_error(abhsf_status st)
{
    if (st != ABHSF_SUCCESS)
        throw std::runtime_error(std::string("abhsf: ") + abhsf_last_error_string());
}

class gpu_matrix {
  public:
    gpu_matrix() { abhsf_build_opts_default(&opts_); }
    explicit gpu_matrix(const abhsf_build_opts& opts) : opts_(opts) {}
    ~gpu_matrix() { abhsf_release(h_); }
    gpu_matrix(const gpu_matrix&) = delete;
    gpu_matrix& operator=(const gpu_matrix&) = delete;
    gpu_matrix(gpu_matrix&& o) noexcept : h_(o.h_), opts_(o.opts_) { o.h_ = nullptr; }

    abhsf_build_opts& options() { return opts_; }

    // Any props type with members m and n (the reference's matrix_properties,
    // include/abhsf/utils/matrix_properties.h:24-30).
    template <typename Elements, typename Props>
    void from_elements(const Elements& elements, const Props& props)
    {
        std::vector<int64_t> rows, cols;
        std::vector<double> vals;
        rows.reserve(elements.size());
        cols.reserve(elements.size());
        vals.reserve(elements.size());
        for (const auto& e : elements) {
            rows.push_back((int64_t)std::get<0>(e));
            cols.push_back((int64_t)std::get<1>(e));
            vals.push_back((double)std::get<2>(e));
        }
        from_coo(rows.data(), cols.data(), vals.data(), (int64_t)rows.size(), (int64_t)props.m, (int64_t)props.n);
    }

    void from_coo(const int64_t* rows, const int64_t* cols, const double* vals, int64_t nnz, int64_t m, int64_t n,
                  abhsf_stream_t stream = nullptr)
    {
        release();
        throw_if_error(abhsf_build(rows, cols, vals, nnz, m, n, &opts_, stream, &h_));
    }

    // y += A x with x and y in host memory (the reference's spmv(x, y)).
    void spmv(const double* x, double* y) { throw_if_error(abhsf_spmv_host(h_, x, y, nullptr)); }

    // y += A x with x and y in device memory, ordered on stream.
    void spmv_device(const double* x, double* y, abhsf_stream_t stream = nullptr) const
    {
        throw_if_error(abhsf_spmv(h_, x, y, stream));
    }

    abhsf_stats stats() const
    {
        abhsf_stats s;
        throw_if_error(abhsf_stats_get(h_, &s));
        return s;
    }

    void release()
    {
        if (h_) {
            abhsf_matrix* h = h_;
            h_ = nullptr;
            throw_if_error(abhsf_release(h));
        }
    }

    abhsf_matrix* handle() const { return h_; }

  private:
    abhsf_matrix* h_ = nullptr;
    abhsf_build_opts opts_;
};

namespace detail {

struct host_coo {
    abhsf_coo_host c{};
    host_coo() = default;
    host_coo(const host_coo&) = delete;
    host_coo& operator=(const host_coo&) = delete;
    ~host_coo() { abhsf_coo_host_free(&c); }
};

template <typename Elements, typename Props>
void append_elements(const host_coo& f, Elements& elements, Props& props)
{
    elements.reserve(elements.size() + (size_t)f.c.nnz);
    for (int64_t k = 0; k < f.c.nnz; ++k)
        elements.emplace_back(f.c.rows[k], f.c.cols[k], f.c.vals[k]);
    props.m = f.c.m;
    props.n = f.c.n;
    props.nnz = f.c.nnz;  // after the zero-drop, as the reference's props.nnz -= zeros
}

}  // namespace detail

// Appends the elements of a Matrix Market file (0-based row, col, value;
// explicit zeros dropped; pattern values 1.0) and sets props.m, props.n and
// props.nnz, as the reference's read_mtx_real_or_binary does
// (include/abhsf/utils/matrix_market_reader.h:146-200); failures throw
// std::runtime_error.  Props is any type with members m, n and nnz.
template <typename Elements, typename Props>
void read_mtx_real_or_binary(const std::string& filename, Elements& elements, Props& props, int threads = 0)
{
    detail::host_coo f;
    throw_if_error(abhsf_read_mtx(filename.c_str(), threads, &f.c));
    detail::append_elements(f, elements, props);
}

// The same for a binary .mm file (utils/mtx2mm/mtx2mm.cpp:102-135).
template <typename Elements, typename Props>
void read_mm(const std::string& filename, Elements& elements, Props& props)
{
    detail::host_coo f;
    throw_if_error(abhsf_read_mm(filename.c_str(), &f.c));
    detail::append_elements(f, elements, props);
}

}  // namespace abhsf
