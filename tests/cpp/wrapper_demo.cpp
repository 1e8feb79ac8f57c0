// wrapper_demo.cpp -- a reference-style caller of the header-only wrapper:
// elements as std::vector<std::tuple<int,int,double>> (spmv/unified/spmv.cpp:68-69),
// props with m / n, then from_elements / spmv / release.  Built and run by
// tests/test_cpp_wrapper.py; on a machine without a GPU it checks that the
// wrapper compiles, links against libabhsf_b200.so and turns a failing status
// into std::runtime_error.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <tuple>
#include <vector>

#include "abhsf/abhsf_gpu.hpp"

struct props_t {
    long m, n, nnz;
};

int main(int argc, char** argv)
{
    // --read FILE: the reference-shaped reader (host only); prints the sizes
    // and order-sensitive sums of what it appended
    if (argc > 2 && (std::strcmp(argv[1], "--read") == 0 || std::strcmp(argv[1], "--read-mm") == 0)) {
        std::vector<std::tuple<int, int, double>> el{{7, 7, 7.0}};  // appended to, as the reference does
        props_t p{0, 0, 0};
        if (std::strcmp(argv[1], "--read") == 0)
            abhsf::read_mtx_real_or_binary(argv[2], el, p);
        else
            abhsf::read_mm(argv[2], el, p);
        double wr = 0.0, wc = 0.0, sv = 0.0;
        for (size_t k = 1; k < el.size(); ++k) {
            wr += (double)k * std::get<0>(el[k]);
            wc += (double)k * std::get<1>(el[k]);
            sv += std::get<2>(el[k]);
        }
        std::printf("read %ld %ld %ld %zu %.17g %.17g %.17g\n", p.m, p.n, p.nnz, el.size(), wr, wc, sv);
        return 0;
    }
    const bool run_gpu = argc > 1 && std::strcmp(argv[1], "--gpu") == 0;
    // invalid block size: must throw before touching a device
    {
        abhsf::gpu_matrix bad;
        bad.options().block_size = 48;
        std::vector<std::tuple<int, int, double>> el{{0, 0, 1.0}};
        props_t p{1, 1, 1};
        try {
            bad.from_elements(el, p);
            std::printf("FAIL: no exception\n");
            return 1;
        } catch (const std::runtime_error& e) {
            std::printf("caught: %s\n", e.what());
        }
    }
    if (!run_gpu)
        return 0;
    // 3 x 3 example, y += A x against a hand-computed result
    std::vector<std::tuple<int, int, double>> el{{0, 0, 2.0}, {0, 2, -1.0}, {1, 1, 3.0}, {2, 0, 0.5}, {2, 2, 4.0}};
    props_t p{3, 3, 5};
    abhsf::gpu_matrix A;
    A.options().block_size = 16;
    A.from_elements(el, p);
    double x[3] = {1.0, 2.0, 3.0}, y[3] = {1.0, 1.0, 1.0};
    A.spmv(x, y);
    const double want[3] = {1.0 + 2.0 - 3.0, 1.0 + 6.0, 1.0 + 0.5 + 12.0};
    for (int i = 0; i < 3; ++i)
        if (std::fabs(y[i] - want[i]) > 1e-15) {
            std::printf("FAIL: y[%d] = %g, want %g\n", i, y[i], want[i]);
            return 1;
        }
    A.release();
    std::printf("OK\n");
    return 0;
}
