// ref_mtx_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own Matrix Market reader, read_mtx_real_or_binary
// (include/abhsf/utils/matrix_market_reader.h:146-200, with its mmio banner and
// size parsing), unmodified from the reference source tree, behind a small
// extern "C" surface, so that tests/golden/make_mtx_golden.py can record what
// it reads from the fixture files.  Build: oracle/Makefile (target `ref`).
#include <cstdint>
#include <tuple>
#include <vector>

#include "abhsf/utils/matrix_market_reader.h"

extern "C" {

// Reads path; writes m, n and up to cap elements (0-based row, col, value) in
// file order.  Returns the element count, -1 if the reader threw, -2 if more
// than cap elements were read.
long ref_mtx_read(const char* path, long* m, long* n, long cap, long* rows, long* cols, double* vals)
{
    try {
        std::vector<std::tuple<uintmax_t, uintmax_t, double>> el;
        matrix_properties props;
        read_mtx_real_or_binary(std::string(path), el, props);
        *m = (long)props.m;
        *n = (long)props.n;
        if ((long)el.size() > cap)
            return -2;
        for (size_t k = 0; k < el.size(); ++k) {
            rows[k] = (long)std::get<0>(el[k]);
            cols[k] = (long)std::get<1>(el[k]);
            vals[k] = std::get<2>(el[k]);
        }
        return (long)el.size();
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
