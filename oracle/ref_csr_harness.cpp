// ref_csr_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own general CSR SpMV, csr_matrix<double,int,int>::
// spmv_naive (spmv/bottlenecks/spmv.cpp:58-64), unmodified from the reference
// source tree, and exposes it through a small extern "C" surface so tests can
// pin the oracle against it and bench.py can time it as the CPU baseline.
// The reference file is included textually; its main() is renamed so that it
// is never run.  Build: see oracle/Makefile (target `ref`).
#define main abhsf_reference_bottlenecks_main
#include "spmv/bottlenecks/spmv.cpp"
#undef main

#include <omp.h>

extern "C" {

struct ref_csr {
    csr_matrix<double, int, int> a;
    long m;
};

// from_elements (spmv/bottlenecks/spmv.cpp:43-49) sorts a copy of the
// caller's elements with __gnu_parallel::sort and builds CSR (coo2csr.h:10-38).
void* ref_csr_create(const long* rows, const long* cols, const double* vals, long nnz, long m, long n)
{
    elements_t el;
    el.reserve(nnz);
    for (long k = 0; k < nnz; ++k)
        el.emplace_back((int)rows[k], (int)cols[k], vals[k]);
    matrix_properties props;
    props.type = matrix_type_t::REAL;
    props.symmetry = matrix_symmetry_t::UNSYMMETRIC;
    props.m = m;
    props.n = n;
    props.nnz = nnz;
    ref_csr* h = new ref_csr;
    h->m = m;
    h->a.from_elements(el, props);
    return h;
}

// y += A x with the reference's OpenMP static row partition.
void ref_csr_spmv_naive(void* h, const double* x, double* y)
{
    static_cast<ref_csr*>(h)->a.spmv_naive(x, y);
}

void ref_csr_release(void* h)
{
    ref_csr* p = static_cast<ref_csr*>(h);
    p->a.release();
    delete p;
}

int ref_csr_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
