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

// Owning device CSR / BSR containers.
struct DeviceCsr {
    int nrows = 0, ncols = 0;
    long long nnz = 0;
    DevBuf<int> ia, ja;
    DevBuf<double> a;
    void alloc(int n, int m, long long z) {
        nrows = n;
        ncols = m;
        nnz = z;
        ia.alloc((size_t)n + 1);
        ja.alloc((size_t)(z > 0 ? z : 1));
        a.alloc((size_t)(z > 0 ? z : 1));
    }
    CsrView<double> view() const { return CsrView<double>{nrows, ncols, nnz, ia.get(), ja.get(), a.get()}; }
};

struct DeviceBsr {
    int nb = 0, bs = 0;
    long long nnzb = 0;
    DevBuf<int> ia, ja;
    DevBuf<double> a;
    void alloc(int n, int b, long long z) {
        nb = n;
        bs = b;
        nnzb = z;
        ia.alloc((size_t)n + 1);
        ja.alloc((size_t)(z > 0 ? z : 1));
        a.alloc((size_t)(z > 0 ? z : 1) * b * b);
    }
    BsrView<double> view() const { return BsrView<double>{nb, bs, nnzb, ia.get(), ja.get(), a.get()}; }
};

// ---- scan.cu ---------------------------------------------------------------
// out[0] = 0, out[i] = in[0] + ... + in[i-1]  (n entries; int32 / int64)
void exclusive_scan_int(const int *in, int *out, int n, cudaStream_t s);
void exclusive_scan_ll(const long long *in, long long *out, int n, cudaStream_t s);

// ---- csr_ops.cu ------------------------------------------------------------
void csr_spmv(const CsrView<double> &A, double alpha, const double *x, double beta, double *y, cudaStream_t s);
void csr_transpose(const CsrView<double> &A, DeviceCsr &T, cudaStream_t s);
void pattern_transpose(int n, int m, long long nnz, const int *ia, const int *ja, int *tia, int *tja, int *tperm,
                       cudaStream_t s);
void bsr_pressure_csr(const BsrView<double> &A, int p, DeviceCsr &Ap, cudaStream_t s);
void restrict_pressure(int nb, int bs, int p, const double *r, double *rp, cudaStream_t s);
void prolong_pressure(int nb, int bs, int p, const double *xp, double *x, cudaStream_t s);

// ---- decouple.cu -----------------------------------------------------------
// Matrix part of jxf_BSRMatrixDecouple (type 1 ABF, 5 True-IMPES); `coef`
// (nb * decouple_coef_size) receives what the right-hand side update needs.
int decouple_coef_size(int bs, int type);
// type: 1 ABF, 2 ANL, 3 SEM, 4 QI, 5 True-IMPES, 6 True-IMPES (second form); thermal applies to 2-4
void bsr_decouple_matrix(DeviceBsr &A, int type, double *coef, cudaStream_t s, int thermal = 0);
void bsr_decouple_rhs(int nb, int bs, int type, const double *coef, double *rhs, int consistent_rhs,
                      cudaStream_t s);

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
