// Row permutation of CSR / BSR storage (rows in schedule order, so that a
// colour class of a multicolour schedule is a contiguous slab of the copy),
// and the lane count of the vectorised row kernels.
#include "amg.cuh"
#include "common.cuh"

namespace jxcpr {

int lanes_for(double mean_row) {
    int v = 1;
    while (v < 32 && v * 4 < mean_row) v <<= 1;
    return v;
}

// ---- row permutation of CSR / BSR storage (rows in schedule order) ----------
__global__ void perm_row_len_kernel(int n, const int *__restrict__ perm, const int *__restrict__ ia,
                                    int *__restrict__ len) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) len[t] = ia[perm[t] + 1] - ia[perm[t]];
}

template <int W>
__global__ void perm_row_copy_kernel(int n, const int *__restrict__ perm, const int *__restrict__ ia,
                                     const int *__restrict__ ja, const double *__restrict__ a,
                                     const int *__restrict__ pia, int *__restrict__ pja, double *__restrict__ pa) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = perm[t];
    const int k0 = ia[i], k1 = ia[i + 1], q0 = pia[t];
    for (int k = k0; k < k1; ++k) {
        pja[q0 + k - k0] = ja[k];
        for (int w = 0; w < W; ++w) pa[(long long)(q0 + k - k0) * W + w] = a[(long long)k * W + w];
    }
}

void permute_rows_csr(const CsrView<double> &A, const int *perm, DeviceCsr &P, cudaStream_t s) {
    const int n = A.nrows;
    P.alloc(n, A.ncols, A.nnz);
    DevBuf<int> len(n + 1);
    len.zero(s);
    perm_row_len_kernel<<<div_up(n, 256), 256, 0, s>>>(n, perm, A.ia, len.get());
    JX_LAUNCH_CHECK();
    exclusive_scan_int(len.get(), P.ia.get(), n + 1, s);
    perm_row_copy_kernel<1><<<div_up(n, 256), 256, 0, s>>>(n, perm, A.ia, A.ja, A.a, P.ia.get(), P.ja.get(),
                                                          P.a.get());
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaStreamSynchronize(s));
}

void permute_rows_bsr(const BsrView<double> &A, const int *perm, DeviceBsr &P, cudaStream_t s) {
    const int n = A.nb;
    P.alloc(n, A.bs, A.nnzb);
    DevBuf<int> len(n + 1);
    len.zero(s);
    perm_row_len_kernel<<<div_up(n, 256), 256, 0, s>>>(n, perm, A.ia, len.get());
    JX_LAUNCH_CHECK();
    exclusive_scan_int(len.get(), P.ia.get(), n + 1, s);
    if (A.bs == 2)
        perm_row_copy_kernel<4><<<div_up(n, 256), 256, 0, s>>>(n, perm, A.ia, A.ja, A.a, P.ia.get(), P.ja.get(),
                                                              P.a.get());
    else
        perm_row_copy_kernel<9><<<div_up(n, 256), 256, 0, s>>>(n, perm, A.ia, A.ja, A.a, P.ia.get(), P.ja.get(),
                                                              P.a.get());
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaStreamSynchronize(s));
}

}  // namespace jxcpr
