// Device-side building blocks shared by the solver: non-owning views of the
// device-resident matrices and the launch wrappers of every kernel file.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace jxcpr {

// Block CSR view (0-based; diagonal block first in each row; row-major blocks).
template <typename V>
struct BsrView {
    int nb = 0;           // block rows (= block columns)
    int bs = 0;           // block size
    long long nnzb = 0;   // stored blocks
    const int *ia = nullptr;
    const int *ja = nullptr;
    const V *a = nullptr;
};

// Scalar CSR view (0-based; the diagonal entry first in each row where present).
template <typename V>
struct CsrView {
    int nrows = 0;
    int ncols = 0;
    long long nnz = 0;
    const int *ia = nullptr;
    const int *ja = nullptr;
    const V *a = nullptr;
};

// ---- bsr_spmv.cu ---------------------------------------------------------
// y = alpha*A*x + beta*y with the reference's rounding sequence.  `staged`
// selects the TMA-staged persistent kernel (requires `err`, a device int set
// to nonzero if a bounded wait gave up).
template <typename V, typename X>
void bsr_spmv(const BsrView<V> &A, X alpha, const X *x, X beta, X *y, int *err, cudaStream_t stream,
              bool staged = true);

// ---- blas1.cu --------------------------------------------------------------
// Deterministic two-pass reductions: per-CTA partials into `partials`
// (>= reduce_partials() doubles), then one CTA sums them into *out (device).
int reduce_partials();
void dot_dev(long long n, const double *x, const double *y, double *partials, double *out, cudaStream_t s);
void axpy_dev(long long n, double alpha, const double *x, double *y, cudaStream_t s);
void scale_dev(long long n, double alpha, double *x, cudaStream_t s);
void copy_dev(long long n, const double *x, double *y, cudaStream_t s);
void fill_dev(long long n, double v, double *x, cudaStream_t s);

}  // namespace jxcpr
