// Block ILU(0) on the device: the reference's fixed-point factorisation and
// Jacobi-iteration triangular solves (bit-identical to a single-threaded run
// of the reference).
//
//   setup  jxf_ILUSetupFGPBILU_v3 (jxfpamg-0220/csrc/ilu/par_bilu_setup.c:4996-5676):
//          A = (I + L)(D + U) on A's block pattern, started from D_r = A_rr,
//          L_rc = A_rc D_c^-1, U_rc = A_rc and improved by `sweeps` sweeps
//          C_rc = A_rc - sum_{k in L-row r} L_rk U_kc; D_r = C_rr;
//          L_rc = C_rc D_c^-1; U_rc = C_rc.  Diagonal blocks with
//          |det| < 1e-14 become the identity; inverses follow
//          jxf_bsr_block_inv (mat_vec_data/jxf_bsr_block_ops.c:75-130).
//          Every row is independent inside a phase, so each phase is one
//          launch over rows: C for all entries, then all D (the reference's
//          row-ordered pass uses the current sweep's D_c^-1 for every c < r,
//          which is what computing all D first gives), then L and U.
//   solve  jxf_BILUSolve with tri_solve 14 (ilu/par_bilu_solve.c:360,
//          2893-3000): ftemp = f - A u, then IR times: y <- ftemp - L y
//          (`lower` sweeps from 0), t <- D^-1 y + D^-1 (-U t) (`upper` sweeps
//          from 0), ftemp <- ftemp - A t, u <- u + t.  The products use the
//          reference's BSR matvec rounding sequence (bsr_spmv).
#include <math.h>

#include "bilu.cuh"

namespace jxcpr {

namespace {
constexpr int kT = 256;
constexpr double kMatTol = 1e-14;   // jx_parilu.h:241
constexpr double kRealMin = 1.0e-300;  // bsr_block_ops.h:21

template <int BS>
__device__ __forceinline__ void blk_matmul(const double *__restrict__ A, const double *__restrict__ B, double *C) {
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
        for (int j = 0; j < BS; ++j) {
            double sum = 0.0;
#pragma unroll
            for (int k = 0; k < BS; ++k) sum += A[i * BS + k] * B[k * BS + j];
            C[i * BS + j] = sum;
        }
}

template <int BS>
__device__ __forceinline__ double blk_det(const double *a) {
    if (BS == 2) return a[0] * a[3] - a[1] * a[2];
    // cofactor expansion along row 0, minors as 2x2 determinants
    double det = 0.0;
#pragma unroll
    for (int col = 0; col < 3; ++col) {
        double sub[4];
        int si = 0;
#pragma unroll
        for (int i = 1; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                if (j != col) sub[si++] = a[i * 3 + j];
        const double sign = (col % 2 == 0) ? 1.0 : -1.0;
        det += sign * a[col] * (sub[0] * sub[3] - sub[1] * sub[2]);
    }
    return det;
}

template <int BS>
__device__ __forceinline__ void blk_inv(double *a) {
    if (BS == 2) {
        const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3];
        const double det = a0 * a3 - a1 * a2;
        if (fabs(det) < kRealMin) {
            a[0] = 1.0; a[1] = 0.0; a[2] = 0.0; a[3] = 1.0;
        } else {
            const double di = 1.0 / det;
            a[0] = a3 * di; a[1] = -a1 * di; a[2] = -a2 * di; a[3] = a0 * di;
        }
        return;
    }
    const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4], a5 = a[5], a6 = a[6], a7 = a[7], a8 = a[8];
    const double M0 = a4 * a8 - a5 * a7, M3 = a2 * a7 - a1 * a8, M6 = a1 * a5 - a2 * a4;
    const double M1 = a5 * a6 - a3 * a8, M4 = a0 * a8 - a2 * a6, M7 = a2 * a3 - a0 * a5;
    const double M2 = a3 * a7 - a4 * a6, M5 = a1 * a6 - a0 * a7, M8 = a0 * a4 - a1 * a3;
    const double det = a0 * M0 + a3 * M3 + a6 * M6;
    if (fabs(det) < kRealMin) {
#pragma unroll
        for (int q = 0; q < 9; ++q) a[q] = (q % 4 == 0) ? 1.0 : 0.0;
    } else {
        const double di = 1.0 / det;
        a[0] = M0 * di; a[1] = M3 * di; a[2] = M6 * di;
        a[3] = M1 * di; a[4] = M4 * di; a[5] = M7 * di;
        a[6] = M2 * di; a[7] = M5 * di; a[8] = M8 * di;
    }
}

// guarded diagonal block -> D (guarded copy) and Dinv
template <int BS>
__device__ __forceinline__ void diag_update(const double *blk, double *D, double *Dinv) {
    constexpr int BN = BS * BS;
    double d[BN];
#pragma unroll
    for (int q = 0; q < BN; ++q) d[q] = blk[q];
    if (fabs(blk_det<BS>(d)) < kMatTol) {
#pragma unroll
        for (int q = 0; q < BN; ++q) d[q] = (q % (BS + 1) == 0) ? 1.0 : 0.0;
    }
#pragma unroll
    for (int q = 0; q < BN; ++q) {
        D[q] = d[q];
        Dinv[q] = d[q];
    }
    blk_inv<BS>(Dinv);
}

__global__ void count_lu_kernel(int nb, const int *__restrict__ ia, const int *__restrict__ ja, int *__restrict__ lc,
                                int *__restrict__ uc) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    int l = 0, u = 0;
    for (int k = ia[r]; k < ia[r + 1]; ++k) {
        l += ja[k] < r;
        u += ja[k] > r;
    }
    lc[r] = l;
    uc[r] = u;
}

__global__ void fill_lu_pattern_kernel(int nb, const int *__restrict__ ia, const int *__restrict__ ja,
                                       const int *__restrict__ lia, const int *__restrict__ uia,
                                       int *__restrict__ lja, int *__restrict__ uja) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    int pl = lia[r], pu = uia[r];
    for (int k = ia[r]; k < ia[r + 1]; ++k) {
        const int c = ja[k];
        if (c < r) lja[pl++] = c;
        else if (c > r) uja[pu++] = c;
    }
}

// D and D^-1 from the diagonal entry of `src` (A at start, C during sweeps)
template <int BS>
__global__ void diag_kernel(int nb, const int *__restrict__ ia, const int *__restrict__ ja,
                            const double *__restrict__ src, double *__restrict__ D, double *__restrict__ Dinv) {
    constexpr int BN = BS * BS;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    for (int k = ia[r]; k < ia[r + 1]; ++k)
        if (ja[k] == r) {
            diag_update<BS>(src + (long long)k * BN, D + (long long)r * BN, Dinv + (long long)r * BN);
            break;
        }
}

// L_rc = src_rc D_c^-1 (c < r), U_rc = src_rc (c > r)
template <int BS>
__global__ void lu_kernel(int nb, const int *__restrict__ ia, const int *__restrict__ ja,
                          const double *__restrict__ src, const double *__restrict__ Dinv,
                          const int *__restrict__ lia, double *__restrict__ la, const int *__restrict__ uia,
                          double *__restrict__ ua) {
    constexpr int BN = BS * BS;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    int pl = lia[r], pu = uia[r];
    for (int k = ia[r]; k < ia[r + 1]; ++k) {
        const int c = ja[k];
        const double *S = src + (long long)k * BN;
        if (c < r) {
            blk_matmul<BS>(S, Dinv + (long long)c * BN, la + (long long)(pl++) * BN);
        } else if (c > r) {
            double *Ub = ua + (long long)(pu++) * BN;
#pragma unroll
            for (int q = 0; q < BN; ++q) Ub[q] = S[q];
        }
    }
}

// C_rc = A_rc - sum_{k in L-row r} L_rk U_kc (U_kc looked up in U-row k)
template <int BS>
__global__ void residual_blocks_kernel(int nb, const int *__restrict__ ia, const int *__restrict__ ja,
                                       const double *__restrict__ a, const int *__restrict__ lia,
                                       const int *__restrict__ lja, const double *__restrict__ la,
                                       const int *__restrict__ uia, const int *__restrict__ uja,
                                       const double *__restrict__ ua, double *__restrict__ C) {
    constexpr int BN = BS * BS;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    for (int jj = ia[r]; jj < ia[r + 1]; ++jj) {
        const int col = ja[jj];
        double c[BN];
#pragma unroll
        for (int q = 0; q < BN; ++q) c[q] = a[(long long)jj * BN + q];
        for (int lj = lia[r]; lj < lia[r + 1]; ++lj) {
            const int k = lja[lj];
            for (int uj = uia[k]; uj < uia[k + 1]; ++uj)
                if (uja[uj] == col) {
                    double t[BN];
                    blk_matmul<BS>(la + (long long)lj * BN, ua + (long long)uj * BN, t);
#pragma unroll
                    for (int q = 0; q < BN; ++q) c[q] -= t[q];
                    break;
                }
        }
#pragma unroll
        for (int q = 0; q < BN; ++q) C[(long long)jj * BN + q] = c[q];
    }
}

// y = t + f
__global__ void add2_kernel(long long n, const double *__restrict__ t, const double *__restrict__ f,
                            double *__restrict__ y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = t[i] + f[i];
}

// per block row: un <- D^-1 un, ut <- D^-1 yt + un
template <int BS>
__global__ void upper_step_kernel(int nb, const double *__restrict__ Dinv, const double *__restrict__ yt,
                                  double *__restrict__ un, double *__restrict__ ut) {
    constexpr int BN = BS * BS;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    const double *D = Dinv + (long long)r * BN;
    double ub[BS], t[BS];
#pragma unroll
    for (int q = 0; q < BS; ++q) ub[q] = un[(long long)r * BS + q];
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < BS; ++j) s += D[q * BS + j] * ub[j];
        t[q] = s;
    }
#pragma unroll
    for (int q = 0; q < BS; ++q) un[(long long)r * BS + q] = t[q];
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < BS; ++j) s += D[q * BS + j] * yt[(long long)r * BS + j];
        ut[(long long)r * BS + q] = s + t[q];
    }
}
}  // namespace

void Bilu::setup(const BsrView<double> &A, cudaStream_t s) {
    nb = A.nb;
    bs = A.bs;
    if (bs != 2 && bs != 3) {
        set_error("BILU: block size %d not supported (2 or 3)", bs);
        throw CudaError{cudaErrorInvalidValue, "bilu block size"};
    }
    const int bn = bs * bs;
    DevBuf<int> lc(nb + 1), uc(nb + 1);
    lc.zero(s);
    uc.zero(s);
    if (nb) {
        count_lu_kernel<<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, lc.get(), uc.get());
        JX_LAUNCH_CHECK();
    }
    L.nb = U.nb = nb;
    L.bs = U.bs = bs;
    L.ia.alloc(nb + 1);
    U.ia.alloc(nb + 1);
    exclusive_scan_int(lc.get(), L.ia.get(), nb + 1, s);
    exclusive_scan_int(uc.get(), U.ia.get(), nb + 1, s);
    int nl = 0, nu = 0;
    JX_CUDA(cudaMemcpyAsync(&nl, L.ia.get() + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaMemcpyAsync(&nu, U.ia.get() + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    L.nnzb = nl;
    U.nnzb = nu;
    L.ja.alloc(nl > 0 ? nl : 1);
    U.ja.alloc(nu > 0 ? nu : 1);
    L.a.alloc((size_t)(nl > 0 ? nl : 1) * bn);
    U.a.alloc((size_t)(nu > 0 ? nu : 1) * bn);
    D.alloc((size_t)(nb > 0 ? nb : 1) * bn);
    Dinv.alloc((size_t)(nb > 0 ? nb : 1) * bn);
    D.zero(s);
    Dinv.zero(s);
    if (nb) {
        fill_lu_pattern_kernel<<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, L.ia.get(), U.ia.get(), L.ja.get(),
                                                            U.ja.get());
        JX_LAUNCH_CHECK();
    }
    auto diag = [&](const double *src) {
        if (!nb) return;
        if (bs == 2) diag_kernel<2><<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, src, D.get(), Dinv.get());
        else diag_kernel<3><<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, src, D.get(), Dinv.get());
        JX_LAUNCH_CHECK();
    };
    auto lu = [&](const double *src) {
        if (!nb) return;
        if (bs == 2)
            lu_kernel<2><<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, src, Dinv.get(), L.ia.get(), L.a.get(),
                                                       U.ia.get(), U.a.get());
        else
            lu_kernel<3><<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, src, Dinv.get(), L.ia.get(), L.a.get(),
                                                       U.ia.get(), U.a.get());
        JX_LAUNCH_CHECK();
    };
    if (exact) {
        setup_exact(A, s);
    } else {
        diag(A.a);
        lu(A.a);
    }
    if (!exact && sweeps > 0 && nb) {
        DevBuf<double> C((size_t)(A.nnzb > 0 ? A.nnzb : 1) * bn);
        for (int sw = 0; sw < sweeps; ++sw) {
            if (bs == 2)
                residual_blocks_kernel<2><<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, A.a, L.ia.get(), L.ja.get(),
                                                                        L.a.get(), U.ia.get(), U.ja.get(), U.a.get(),
                                                                        C.get());
            else
                residual_blocks_kernel<3><<<div_up(nb, kT), kT, 0, s>>>(nb, A.ia, A.ja, A.a, L.ia.get(), L.ja.get(),
                                                                        L.a.get(), U.ia.get(), U.ja.get(), U.a.get(),
                                                                        C.get());
            JX_LAUNCH_CHECK();
            diag(C.get());
            lu(C.get());
        }
        JX_CUDA(cudaStreamSynchronize(s));
    }
    const size_t n = (size_t)(nb > 0 ? nb : 1) * bs;
    ft.alloc(n);
    ut.alloc(n);
    yt.alloc(n);
    un.alloc(n);
    JX_CUDA(cudaStreamSynchronize(s));
}

void Bilu::solve(const BsrView<double> &A, const double *f, double *u, cudaStream_t s) {
    const long long n = (long long)nb * bs;
    if (!n) return;
    const BsrView<double> Lv = L.view(), Uv = U.view();
    copy_dev(n, f, ft.get(), s);
    bsr_spmv<double, double>(A, -1.0, u, 1.0, ft.get(), nullptr, s, false);
    if (exact) {
        for (int it = 0; it < ir_iters; ++it) {
            substitute(ft.get(), yt.get(), ut.get(), s);
            bsr_spmv<double, double>(A, -1.0, ut.get(), 1.0, ft.get(), nullptr, s, false);
            axpy_dev(n, 1.0, ut.get(), u, s);
        }
        return;
    }
    for (int it = 0; it < ir_iters; ++it) {
        JX_CUDA(cudaMemsetAsync(ut.get(), 0, sizeof(double) * n, s));
        JX_CUDA(cudaMemsetAsync(yt.get(), 0, sizeof(double) * n, s));
        JX_CUDA(cudaMemsetAsync(un.get(), 0, sizeof(double) * n, s));
        for (int k = 0; k < lower_iters; ++k) {
            bsr_spmv<double, double>(Lv, -1.0, yt.get(), 0.0, ut.get(), nullptr, s, false);
            add2_kernel<<<div_up(n, kT), kT, 0, s>>>(n, ut.get(), ft.get(), yt.get());
            JX_LAUNCH_CHECK();
        }
        JX_CUDA(cudaMemsetAsync(ut.get(), 0, sizeof(double) * n, s));
        for (int k = 0; k < upper_iters; ++k) {
            bsr_spmv<double, double>(Uv, -1.0, ut.get(), 0.0, un.get(), nullptr, s, false);
            if (bs == 2) upper_step_kernel<2><<<div_up(nb, kT), kT, 0, s>>>(nb, Dinv.get(), yt.get(), un.get(), ut.get());
            else upper_step_kernel<3><<<div_up(nb, kT), kT, 0, s>>>(nb, Dinv.get(), yt.get(), un.get(), ut.get());
            JX_LAUNCH_CHECK();
        }
        bsr_spmv<double, double>(A, -1.0, ut.get(), 1.0, ft.get(), nullptr, s, false);
        axpy_dev(n, 1.0, ut.get(), u, s);
    }
}

}  // namespace jxcpr
