// Scalar-CSR kernels of the pressure AMG and the CPR transfer operators.
//
// * csr_spmv: y = alpha*A*x + beta*y in the rounding sequence of
//   jxf_CSRMatrixMatvec (jxfpamg-0220/csrc/operation/mvops/seq_csr_matvec.c:20)
//   -- one thread per row, entries in stored order.
// * csr_transpose: stable transpose (entries of each output row keep the
//   ascending order of their source rows), so that R = P^T applied as a
//   row-oriented product reproduces jxf_CSRMatrixMatvecT's per-column
//   accumulation order (seq_csr_matvec.c:211) bit for bit.
// * bsr_pressure_csr: jxf_BSRMatrixGetSubmatrix (seq_bsr_matrix.c:214-251).
// * restrict / prolong: jxf_RestrictPressureVector / jxf_ProlongatePressureVector
//   type 0 (jxfpamg-0220/csrc/cpr/jxf_cpr.c:74-145).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

__global__ void csr_spmv_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                const double *__restrict__ a, const double *__restrict__ x, double *__restrict__ y,
                                int init_mode, double scale_y, double alpha) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = init_mode == 0 ? 0.0 : (init_mode == 1 ? y[i] : y[i] * scale_y);
    const int kb = ia[i], ke = ia[i + 1];
    for (int k = kb; k < ke; ++k) t = t + __ldg(a + k) * __ldg(x + __ldg(ja + k));
    y[i] = alpha == 1.0 ? t : t * alpha;
}

__global__ void scale_y_kernel(int n, double beta, double *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = y[i] * beta;
}

void csr_spmv(const CsrView<double> &A, double alpha, const double *x, double beta, double *y, cudaStream_t s) {
    if (A.nrows == 0) return;
    if (alpha == 0.0) {
        scale_y_kernel<<<div_up(A.nrows, 256), 256, 0, s>>>(A.nrows, beta, y);
        JX_LAUNCH_CHECK();
        return;
    }
    double t = beta / alpha;
    int mode = (t == 0.0) ? 0 : (t == 1.0 ? 1 : 2);
    csr_spmv_kernel<<<div_up(A.nrows, 256), 256, 0, s>>>(A.nrows, A.ia, A.ja, A.a, x, y, mode, t, alpha);
    JX_LAUNCH_CHECK();
}

// ---- stable transpose ------------------------------------------------------
__global__ void expand_rows_kernel(int n, const int *__restrict__ ia, int *__restrict__ rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = ia[i]; k < ia[i + 1]; ++k) rows[k] = i;
}

__global__ void iota_kernel(long long n, int *__restrict__ v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int)i;
}

__global__ void count_cols_kernel(long long nnz, const int *__restrict__ cols, int *__restrict__ cnt) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) atomicAdd(cnt + cols[k], 1);
}

__global__ void gather_rows_kernel(long long nnz, const int *__restrict__ perm, const int *__restrict__ rows,
                                   int *__restrict__ tja) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) tja[k] = rows[perm[k]];
}

// Stable transpose of a pattern: tia (m+1), tja (source row of each entry) and
// tperm (source entry index), entries of each column in ascending row order.
void pattern_transpose(int n, int m, long long nnz, const int *ia, const int *ja, int *tia, int *tja, int *tperm,
                       cudaStream_t s) {
    if (nnz == 0) {
        JX_CUDA(cudaMemsetAsync(tia, 0, sizeof(int) * (m + 1), s));
        return;
    }
    DevBuf<int> rows(nnz), perm_in(nnz), keys_out(nnz);
    expand_rows_kernel<<<div_up(n, 256), 256, 0, s>>>(n, ia, rows.get());
    JX_LAUNCH_CHECK();
    iota_kernel<<<div_up(nnz, 256), 256, 0, s>>>(nnz, perm_in.get());
    JX_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    int end_bit = 1;
    while (end_bit < 31 && (1LL << end_bit) <= m) ++end_bit;
    JX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, ja, keys_out.get(), perm_in.get(), tperm,
                                            (int)nnz, 0, end_bit, s));
    DevBuf<unsigned char> tmp(tmp_bytes);
    // LSD radix sort is stable: entries of equal column keep ascending source order (= ascending row).
    JX_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, ja, keys_out.get(), perm_in.get(), tperm,
                                            (int)nnz, 0, end_bit, s));
    DevBuf<int> cnt(m + 1);
    cnt.zero(s);
    count_cols_kernel<<<div_up(nnz, 256), 256, 0, s>>>(nnz, ja, cnt.get());
    JX_LAUNCH_CHECK();
    exclusive_scan_int(cnt.get(), tia, m + 1, s);
    gather_rows_kernel<<<div_up(nnz, 256), 256, 0, s>>>(nnz, tperm, rows.get(), tja);
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaStreamSynchronize(s));  // temporaries die with this scope
}

__global__ void gather_vals_kernel(long long nnz, const int *__restrict__ perm, const double *__restrict__ a,
                                   double *__restrict__ ta) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) ta[k] = a[perm[k]];
}

void csr_transpose(const CsrView<double> &A, DeviceCsr &T, cudaStream_t s) {
    T.alloc(A.ncols, A.nrows, A.nnz);
    DevBuf<int> perm(A.nnz > 0 ? A.nnz : 1);
    pattern_transpose(A.nrows, A.ncols, A.nnz, A.ia, A.ja, T.ia.get(), T.ja.get(), perm.get(), s);
    if (A.nnz > 0) {
        gather_vals_kernel<<<div_up(A.nnz, 256), 256, 0, s>>>(A.nnz, perm.get(), A.a, T.a.get());
        JX_LAUNCH_CHECK();
        JX_CUDA(cudaStreamSynchronize(s));
    }
}

// ---- CPR transfer ----------------------------------------------------------
__global__ void pressure_csr_kernel(long long nnzb, int bs, int p, const double *__restrict__ a,
                                    double *__restrict__ ca) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnzb) ca[k] = a[k * bs * bs + p * bs + p];
}

void bsr_pressure_csr(const BsrView<double> &A, int p, DeviceCsr &Ap, cudaStream_t s) {
    Ap.alloc(A.nb, A.nb, A.nnzb);
    JX_CUDA(cudaMemcpyAsync(Ap.ia.get(), A.ia, sizeof(int) * (A.nb + 1), cudaMemcpyDeviceToDevice, s));
    if (A.nnzb) {
        JX_CUDA(cudaMemcpyAsync(Ap.ja.get(), A.ja, sizeof(int) * A.nnzb, cudaMemcpyDeviceToDevice, s));
        pressure_csr_kernel<<<div_up(A.nnzb, 256), 256, 0, s>>>(A.nnzb, A.bs, p, A.a, Ap.a.get());
        JX_LAUNCH_CHECK();
    }
}

__global__ void restrict_kernel(int nb, int bs, int p, const double *__restrict__ r, double *__restrict__ rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) rp[i] = r[(long long)i * bs + p];
}

__global__ void prolong_kernel(int nb, int bs, int p, const double *__restrict__ xp, double *__restrict__ x) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)nb * bs) return;
    const int j = (int)(k % bs);
    x[k] = (j == p) ? xp[k / bs] : 0.0;
}

void restrict_pressure(int nb, int bs, int p, const double *r, double *rp, cudaStream_t s) {
    if (nb == 0) return;
    restrict_kernel<<<div_up(nb, 256), 256, 0, s>>>(nb, bs, p, r, rp);
    JX_LAUNCH_CHECK();
}

void prolong_pressure(int nb, int bs, int p, const double *xp, double *x, cudaStream_t s) {
    if (nb == 0) return;
    prolong_kernel<<<div_up((long long)nb * bs, 256), 256, 0, s>>>(nb, bs, p, xp, x);
    JX_LAUNCH_CHECK();
}

}  // namespace jxcpr
