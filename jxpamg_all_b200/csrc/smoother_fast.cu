// Throughput-oriented smoothers and CSR products for the pressure AMG
// ("multicolour" mode).  Unlike the exact-order kernels these do not follow
// the reference's summation order: a row is reduced by V lanes of a warp
// (V = 1..32 chosen from the level's mean row length) with shuffles.
//
// * gs_color:  Gauss-Seidel restricted to one colour class (an independent
//              set): u_i = (f_i - sum_{j != i} a_ij u_j) / a_ii.  Sweeping the
//              classes in order is Gauss-Seidel in colour order; rows of other
//              classes are read in place (earlier classes already updated).
// * jacobi_l1: u_i += (f_i - sum_j a_ij u_j) / d_i with d_i = sum_j |a_ij|
//              (l1-Jacobi), used on coarse levels whose colouring needs many
//              classes.
// * residual / spmv with V lanes per row.
#include "amg.cuh"
#include "common.cuh"

namespace jxcpr {

template <int V>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = V / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, V);
    return v;
}

// sum over the row of a_ij * x_j (skip_first: leave out the first stored entry)
template <int V>
__device__ __forceinline__ double row_dot(const int *__restrict__ ja, const double *__restrict__ a, int kb, int ke,
                                         const double *x, int lane) {
    double s = 0.0;
    for (int k = kb + lane; k < ke; k += V) s += __ldg(a + k) * x[__ldg(ja + k)];
    return group_sum<V>(s);
}

template <int V>
__global__ void gs_color_kernel(int r0, int r1, const int *__restrict__ perm, const int *__restrict__ ia,
                                const int *__restrict__ ja, const double *__restrict__ a,
                                const double *__restrict__ f, double *u) {
    // every lane reaches the shuffles; out-of-range groups reduce an empty row
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = r0 + (int)(gt / V);
    const int lane = (int)(gt % V);
    const bool live = t < r1;
    const int i = live ? perm[t] : 0;
    const int d = live ? ia[i] : 0, e = live ? ia[i + 1] : 0;
    const double diag = d < e ? __ldg(a + d) : 0.0;
    const double s = row_dot<V>(ja, a, d + 1 < e ? d + 1 : e, e, u, lane);
    if (live && lane == 0 && diag != 0.0) u[i] = (f[i] - s) / diag;
}

// Rows stored in schedule order (row t of the copy is row perm[t] of A), so a
// colour class is a contiguous slab of the copy.
template <int V>
__global__ void gs_color_perm_kernel(int r0, int r1, const int *__restrict__ perm, const int *__restrict__ ia,
                                     const int *__restrict__ ja, const double *__restrict__ a,
                                     const double *__restrict__ f, double *u) {
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = r0 + (int)(gt / V);
    const int lane = (int)(gt % V);
    const bool live = t < r1;
    const int d = live ? ia[t] : 0, e = live ? ia[t + 1] : 0;
    const double diag = d < e ? __ldg(a + d) : 0.0;
    const double s = row_dot<V>(ja, a, d + 1 < e ? d + 1 : e, e, u, lane);
    if (live && lane == 0 && diag != 0.0) {
        const int i = perm[t];
        u[i] = (f[i] - s) / diag;
    }
}

template <int V>
__global__ void jacobi_l1_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                 const double *__restrict__ a, const double *__restrict__ dinv,
                                 const double *__restrict__ f, const double *__restrict__ u,
                                 double *__restrict__ unew) {
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(gt / V);
    const int lane = (int)(gt % V);
    const bool live = i < n;
    const double s = row_dot<V>(ja, a, live ? ia[i] : 0, live ? ia[i + 1] : 0, u, lane);
    if (live && lane == 0) unew[i] = u[i] + (f[i] - s) * dinv[i];
}

// r = f - A u
template <int V>
__global__ void residual_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                const double *__restrict__ a, const double *__restrict__ f,
                                const double *__restrict__ u, double *__restrict__ r) {
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(gt / V);
    const int lane = (int)(gt % V);
    const bool live = i < n;
    const double s = row_dot<V>(ja, a, live ? ia[i] : 0, live ? ia[i + 1] : 0, u, lane);
    if (live && lane == 0) r[i] = f[i] - s;
}

// y = alpha * A x + beta * y
template <int V>
__global__ void spmv_vec_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                const double *__restrict__ a, double alpha, const double *__restrict__ x,
                                double beta, double *__restrict__ y) {
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int i = (int)(gt / V);
    const int lane = (int)(gt % V);
    const bool live = i < n;
    const double s = row_dot<V>(ja, a, live ? ia[i] : 0, live ? ia[i + 1] : 0, x, lane);
    if (live && lane == 0) y[i] = beta == 0.0 ? alpha * s : alpha * s + beta * y[i];
}

__global__ void l1_diag_kernel(int n, const int *__restrict__ ia, const double *__restrict__ a,
                               double *__restrict__ dinv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = ia[i]; k < ia[i + 1]; ++k) s += fabs(a[k]);
    dinv[i] = s > 0.0 ? 1.0 / s : 0.0;
}

int lanes_for(double mean_row) {
    int v = 1;
    while (v < 32 && v * 4 < mean_row) v <<= 1;
    return v;
}

#define JX_DISPATCH_V(V, CALL)                    \
    switch (V) {                                  \
        case 1: { constexpr int VV = 1; CALL; } break;   \
        case 2: { constexpr int VV = 2; CALL; } break;   \
        case 4: { constexpr int VV = 4; CALL; } break;   \
        case 8: { constexpr int VV = 8; CALL; } break;   \
        case 16: { constexpr int VV = 16; CALL; } break; \
        default: { constexpr int VV = 32; CALL; } break; \
    }

void l1_diag(const CsrView<double> &A, double *dinv, cudaStream_t s) {
    if (A.nrows == 0) return;
    l1_diag_kernel<<<div_up(A.nrows, 256), 256, 0, s>>>(A.nrows, A.ia, A.a, dinv);
    JX_LAUNCH_CHECK();
}

// Colour classes of `sch` in order; `last_color` carries the class computed
// last (or -1 after u changed by other means): a class is skipped when it
// equals that one, since its rows would be recomputed from unchanged inputs.
// With `Aperm` (rows in fwd-schedule order) each class is a contiguous slab;
// `color_of_group` maps this schedule's groups to fwd class ids.
void gs_sweep_colors_perm(const CsrView<double> &Aperm, const Schedule &fwd, bool backward, int V, const double *f,
                          double *u, int &last_color, cudaStream_t s) {
    const int nc = fwd.ngroups;
    for (int g = 0; g < nc; ++g) {
        const int c = backward ? nc - 1 - g : g;
        if (c == last_color) continue;
        const int r0 = fwd.h_group_ptr[c], r1 = fwd.h_group_ptr[c + 1];
        last_color = c;
        if (r1 <= r0) continue;
        const long long threads = (long long)(r1 - r0) * V;
        JX_DISPATCH_V(V, (gs_color_perm_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(
                             r0, r1, fwd.perm.get(), Aperm.ia, Aperm.ja, Aperm.a, f, u)));
        JX_LAUNCH_CHECK();
    }
}

void gs_sweep_colors(const CsrView<double> &A, const Schedule &sch, int V, const double *f, double *u,
                     cudaStream_t s) {
    for (int g = 0; g < sch.ngroups; ++g) {
        const int r0 = sch.h_group_ptr[g], r1 = sch.h_group_ptr[g + 1];
        if (r1 <= r0) continue;
        const long long threads = (long long)(r1 - r0) * V;
        JX_DISPATCH_V(V, (gs_color_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(r0, r1, sch.perm.get(), A.ia,
                                                                                 A.ja, A.a, f, u)));
        JX_LAUNCH_CHECK();
    }
}

// Two l1-Jacobi sweeps, u -> tmp -> u (no copies).
void jacobi_l1_sweep2(const CsrView<double> &A, int V, const double *dinv, const double *f, double *u, double *tmp,
                      cudaStream_t s) {
    const int n = A.nrows;
    if (n == 0) return;
    const long long threads = (long long)n * V;
    JX_DISPATCH_V(V, (jacobi_l1_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(n, A.ia, A.ja, A.a, dinv, f, u,
                                                                             tmp)));
    JX_LAUNCH_CHECK();
    JX_DISPATCH_V(V, (jacobi_l1_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(n, A.ia, A.ja, A.a, dinv, f, tmp,
                                                                             u)));
    JX_LAUNCH_CHECK();
}

void jacobi_l1_sweep(const CsrView<double> &A, int V, const double *dinv, const double *f, double *u,
                     double *tmp, cudaStream_t s) {
    const int n = A.nrows;
    if (n == 0) return;
    const long long threads = (long long)n * V;
    JX_DISPATCH_V(V, (jacobi_l1_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(n, A.ia, A.ja, A.a, dinv, f, u,
                                                                             tmp)));
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaMemcpyAsync(u, tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
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

void residual_vec(const CsrView<double> &A, int V, const double *f, const double *u, double *r, cudaStream_t s) {
    const int n = A.nrows;
    if (n == 0) return;
    const long long threads = (long long)n * V;
    JX_DISPATCH_V(V, (residual_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(n, A.ia, A.ja, A.a, f, u, r)));
    JX_LAUNCH_CHECK();
}

void spmv_vec(const CsrView<double> &A, int V, double alpha, const double *x, double beta, double *y,
              cudaStream_t s) {
    const int n = A.nrows;
    if (n == 0) return;
    const long long threads = (long long)n * V;
    JX_DISPATCH_V(V, (spmv_vec_kernel<VV><<<div_up(threads, 256), 256, 0, s>>>(n, A.ia, A.ja, A.a, alpha, x, beta,
                                                                            y)));
    JX_LAUNCH_CHECK();
}

}  // namespace jxcpr
