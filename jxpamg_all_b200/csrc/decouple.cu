// Decoupling of the BSR Jacobian and its right-hand side (the pre-solve step
// of CPR), jxf_BSRMatrixDecouple (jxfpamg-0220/csrc/cpr/jxf_bsr_decoup.c:
// 1273-1348): ABF (type 1, :364-510), the analytic, semi-analytic and
// quasi-IMPES row transforms (types 2-4, :529-714, with the thermal variant),
// True-IMPES (type 5, :721-996) and its second form (type 6, :1102-1267), for
// 2x2 and 3x3 blocks.  One thread per block row, the reference's arithmetic
// in its order (the library is compiled without FMA contraction), so the
// results are bit-identical.
//
// The reference updates the right-hand side with an in-place product whose
// input and output alias (:404-408 and :496-498 for ABF; :986-993 for 3x3
// True-IMPES uses a third weight the matrix update does not), which changes
// the solution of the decoupled system.  `consistent_rhs = 0` reproduces that
// arithmetic exactly (the drop-in default); `consistent_rhs = 1` applies the
// same row operation to b as to A, which keeps the solution unchanged.
#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

__device__ __forceinline__ void inv2(double *a) {
    const double a11 = a[0], a12 = a[1], a21 = a[2], a22 = a[3];
    const double det = a11 * a22 - a12 * a21;
    if (fabs(det) < 1e-15) {
        a[0] = 1.0; a[1] = 0.0; a[2] = 0.0; a[3] = 1.0;
    } else {
        const double d = 1.0 / det;
        a[0] = a22 * d;
        a[1] = -a12 * d;
        a[2] = -a21 * d;
        a[3] = a11 * d;
    }
}

__device__ __forceinline__ void inv3(double *a) {
    const double a11 = a[0], a12 = a[1], a13 = a[2];
    const double a21 = a[3], a22 = a[4], a23 = a[5];
    const double a31 = a[6], a32 = a[7], a33 = a[8];
    const double M11 = a22 * a33 - a23 * a32, M12 = a21 * a33 - a23 * a31, M13 = a21 * a32 - a22 * a31;
    const double M21 = a12 * a33 - a13 * a32, M22 = a11 * a33 - a13 * a31, M23 = a11 * a32 - a12 * a31;
    const double M31 = a12 * a23 - a13 * a22, M32 = a11 * a23 - a13 * a21, M33 = a11 * a22 - a12 * a21;
    const double det = a11 * M11 - a12 * M12 + a13 * M13;
    if (fabs(det) < 1e-15) {
        for (int i = 0; i < 9; i++) a[i] = 0.0;
        a[0] = a[4] = a[8] = 1.0;
    } else {
        const double d = 1.0 / det;
        a[0] = M11 * d; a[1] = -M21 * d; a[2] = M31 * d;
        a[3] = -M12 * d; a[4] = M22 * d; a[5] = -M32 * d;
        a[6] = M13 * d; a[7] = -M23 * d; a[8] = M33 * d;
    }
}

template <int BS>
__global__ void abf_kernel(int nb, const int *__restrict__ ia, double *__restrict__ a, double *__restrict__ coef) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    constexpr int B2 = BS * BS;
    double binv[B2];
    const long long kb = ia[i], ke = ia[i + 1];
#pragma unroll
    for (int q = 0; q < B2; ++q) binv[q] = a[kb * B2 + q];
    if (BS == 2) inv2(binv); else inv3(binv);
    for (long long k = kb; k < ke; ++k) {
        double *blk = a + k * B2;
        if (k == kb) {
#pragma unroll
            for (int q = 0; q < B2; ++q) blk[q] = (q % (BS + 1) == 0) ? 1.0 : 0.0;
        } else {
            double in[B2], out[B2];
#pragma unroll
            for (int q = 0; q < B2; ++q) in[q] = blk[q];
            if (BS == 2) {
                out[0] = binv[0] * in[0] + binv[1] * in[2];
                out[1] = binv[0] * in[1] + binv[1] * in[3];
                out[2] = binv[2] * in[0] + binv[3] * in[2];
                out[3] = binv[2] * in[1] + binv[3] * in[3];
            } else {
#pragma unroll
                for (int r = 0; r < BS; ++r)
#pragma unroll
                    for (int c = 0; c < BS; ++c) {
                        double t = 0.0;
#pragma unroll
                        for (int m = 0; m < BS; ++m) t += binv[r * BS + m] * in[m * BS + c];
                        out[r * BS + c] = t;
                    }
            }
#pragma unroll
            for (int q = 0; q < B2; ++q) blk[q] = out[q];
        }
    }
#pragma unroll
    for (int q = 0; q < B2; ++q) coef[(long long)i * B2 + q] = binv[q];
}

// b_i <- D_i b_i with D_i = inv(A_ii) saved by abf_kernel.
template <int BS>
__global__ void abf_rhs_kernel(int nb, const double *__restrict__ coef, double *__restrict__ rhs,
                               int consistent_rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    constexpr int B2 = BS * BS;
    double binv[B2];
#pragma unroll
    for (int q = 0; q < B2; ++q) binv[q] = coef[(long long)i * B2 + q];
    double *r = rhs + (long long)i * BS;
    if (consistent_rhs) {
        double v[BS], o[BS];
#pragma unroll
        for (int p = 0; p < BS; ++p) v[p] = r[p];
#pragma unroll
        for (int p = 0; p < BS; ++p) {
            double t = 0.0;
#pragma unroll
            for (int m = 0; m < BS; ++m) t += binv[p * BS + m] * v[m];
            o[p] = t;
        }
#pragma unroll
        for (int p = 0; p < BS; ++p) r[p] = o[p];
    } else if (BS == 2) {
        double r0 = binv[0] * r[0] + binv[1] * r[1];
        double r1 = binv[2] * r0 + binv[3] * r[1];
        r[0] = r0;
        r[1] = r1;
    } else {
        double v[BS];
#pragma unroll
        for (int p = 0; p < BS; ++p) v[p] = r[p];
#pragma unroll
        for (int p = 0; p < BS; ++p) {
            v[p] = 0.0;
#pragma unroll
            for (int m = 0; m < BS; ++m) v[p] += binv[p * BS + m] * v[m];
        }
#pragma unroll
        for (int p = 0; p < BS; ++p) r[p] = v[p];
    }
}

// Column-sum blocks Ac_c = sum_i A_ic, accumulated in ascending row order
// (the reference's scatter order) via the stable transpose of the pattern.
template <int BS>
__global__ void colsum_kernel(int nb, const int *__restrict__ tia, const int *__restrict__ tperm,
                              const double *__restrict__ a, double *__restrict__ Ac) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nb) return;
    constexpr int B2 = BS * BS;
    double acc[B2];
#pragma unroll
    for (int q = 0; q < B2; ++q) acc[q] = 0.0;
    for (int t = tia[c]; t < tia[c + 1]; ++t) {
        const long long k = tperm[t];
#pragma unroll
        for (int q = 0; q < B2; ++q) acc[q] += a[k * B2 + q];
    }
#pragma unroll
    for (int q = 0; q < B2; ++q) Ac[(long long)c * B2 + q] = acc[q];
}

// Matrix part; coef keeps the weights the right-hand side needs: c (2x2) or
// the first row of inv(Ac_i) (3x3).
template <int BS>
__global__ void timpes_kernel(int nb, const int *__restrict__ ia, const double *__restrict__ Ac,
                              double *__restrict__ a, double *__restrict__ coef) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    constexpr int B2 = BS * BS;
    const long long kb = ia[i], ke = ia[i + 1];
    if (BS == 2) {
        const double *ac = Ac + (long long)i * 4;
        const double det = ac[0] * ac[3] - ac[1] * ac[2];
        double c = 0.0;
        if (!(fabs(det) < 1e-15) && fabs(ac[3]) > 1e-15) c = -ac[1] / ac[3];
        for (long long k = kb; k < ke; ++k) {
            double *blk = a + k * 4;
            blk[0] = blk[0] + c * blk[2];
            blk[1] = blk[1] + c * blk[3];
        }
        coef[(long long)i * 3] = c;
    } else {
        double binv[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) binv[q] = Ac[(long long)i * 9 + q];
        inv3(binv);
        const double c0 = binv[0], c1 = binv[1];
        for (long long k = kb; k < ke; ++k) {
            double *blk = a + k * B2;
            const double n0 = c0 * blk[0] + c1 * blk[3];
            const double n1 = c0 * blk[1] + c1 * blk[4];
            const double n2 = c0 * blk[2] + c1 * blk[5];
            blk[0] = n0;
            blk[1] = n1;
            blk[2] = n2;
        }
        coef[(long long)i * 3] = binv[0];
        coef[(long long)i * 3 + 1] = binv[1];
        coef[(long long)i * 3 + 2] = binv[2];
    }
}

template <int BS>
__global__ void timpes_rhs_kernel(int nb, const double *__restrict__ coef, double *__restrict__ rhs,
                                  int consistent_rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    double *r = rhs + (long long)i * BS;
    const double *c = coef + (long long)i * 3;
    if (BS == 2) {
        r[0] = r[0] + c[0] * r[1];
    } else if (consistent_rhs) {
        r[0] = c[0] * r[0] + c[1] * r[1];
    } else {
        r[0] = c[0] * r[0] + c[1] * r[1] + c[2] * r[2];
    }
}

// Row-transform decouplings ANL (2), SEM (3), QI (4) (:529-714): M_i from the
// row's diagonal block, every block B of the row becomes M_i B (C = 0;
// C += M_ik B_kj) and M_i is kept for the right-hand side.  Thermal mode: the
// last unknown is temperature; the first row changes only in columns
// 1..n-2 and the last row likewise (SEM also zeroes M_0,n-1 and M_n-1,0).
template <int BS>
__device__ __forceinline__ void row_matrix(int type, int thermal, const double *d, double *M) {
    constexpr int B2 = BS * BS;
    if (type == 3) {
#pragma unroll
        for (int q = 0; q < B2; ++q) M[q] = d[q];
        if (BS == 2) inv2(M); else inv3(M);
        if (thermal) {
            M[0] = 1.0;
            M[BS - 1] = 0.0;
            M[(BS - 1) * BS] = 0.0;
            M[B2 - 1] = 1.0;
            for (int l = 0; l < BS - 2; ++l) {
                M[1 + l] = -d[1 + l];
                M[(BS - 1) * BS + 1 + l] = -d[(BS - 1) * BS + 1 + l];
            }
        } else {
            M[0] = 1.0;
            for (int l = 0; l < BS - 1; ++l) M[1 + l] = -d[1 + l];
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < B2; ++q) M[q] = (q % (BS + 1) == 0) ? 1.0 : 0.0;
    const int nl = thermal ? BS - 2 : BS - 1;
    for (int l = 0; l < nl; ++l) {
        if (type == 2) {
            M[1 + l] = -d[1 + l];
            if (thermal) M[(BS - 1) * BS + 1 + l] = -d[(BS - 1) * BS + 1 + l];
        } else {
            M[1 + l] = -d[1 + l] / d[(l + 1) * BS + l + 1];
            if (thermal) M[(BS - 1) * BS + 1 + l] = -d[(BS - 1) * BS + 1 + l] / d[(l + 1) * BS + l + 1];
        }
    }
}

template <int BS>
__global__ void row_transform_kernel(int nb, const int *__restrict__ ia, double *__restrict__ a,
                                     double *__restrict__ coef, int type, int thermal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    constexpr int B2 = BS * BS;
    const long long kb = ia[i], ke = ia[i + 1];
    double d[B2], M[B2];
#pragma unroll
    for (int q = 0; q < B2; ++q) d[q] = a[kb * B2 + q];
    row_matrix<BS>(type, thermal, d, M);
    for (long long k = kb; k < ke; ++k) {
        double *blk = a + k * B2;
        double in[B2], out[B2];
#pragma unroll
        for (int q = 0; q < B2; ++q) in[q] = blk[q];
#pragma unroll
        for (int r = 0; r < BS; ++r)
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                double t = 0.0;
#pragma unroll
                for (int m = 0; m < BS; ++m) t += M[r * BS + m] * in[m * BS + c];
                out[r * BS + c] = t;
            }
#pragma unroll
        for (int q = 0; q < B2; ++q) blk[q] = out[q];
    }
#pragma unroll
    for (int q = 0; q < B2; ++q) coef[(long long)i * B2 + q] = M[q];
}

// b_i <- M_i b_i: the reference's generic helper with input and output aliased
// (c_p = 0, then c_p += M_pk b_k over the partly overwritten vector), or from a
// copy with consistent_rhs.
template <int BS>
__global__ void row_rhs_kernel(int nb, const double *__restrict__ coef, double *__restrict__ rhs,
                               int consistent_rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    constexpr int B2 = BS * BS;
    double M[B2], v[BS];
#pragma unroll
    for (int q = 0; q < B2; ++q) M[q] = coef[(long long)i * B2 + q];
    double *r = rhs + (long long)i * BS;
#pragma unroll
    for (int p = 0; p < BS; ++p) v[p] = r[p];
    if (consistent_rhs) {
        double o[BS];
#pragma unroll
        for (int p = 0; p < BS; ++p) {
            double t = 0.0;
#pragma unroll
            for (int m = 0; m < BS; ++m) t += M[p * BS + m] * v[m];
            o[p] = t;
        }
#pragma unroll
        for (int p = 0; p < BS; ++p) r[p] = o[p];
    } else {
#pragma unroll
        for (int p = 0; p < BS; ++p) {
            v[p] = 0.0;
#pragma unroll
            for (int m = 0; m < BS; ++m) v[p] += M[p * BS + m] * v[m];
        }
#pragma unroll
        for (int p = 0; p < BS; ++p) r[p] = v[p];
    }
}

// True-IMPES, second form (type 6, :1102-1267): pressure row of every block
// of row i += c row1 (2x2: c = -Ac01/Ac11, 0 if |det Ac_i| < 1e-15) or
// c0 row1 + c1 row2 ((c0, c1) = first two entries of inv(Ac_i), 3x3).
template <int BS>
__global__ void timpes2_kernel(int nb, const int *__restrict__ ia, const double *__restrict__ Ac,
                               double *__restrict__ a, double *__restrict__ coef) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const long long kb = ia[i], ke = ia[i + 1];
    if (BS == 2) {
        const double *ac = Ac + (long long)i * 4;
        const double det = ac[0] * ac[3] - ac[1] * ac[2];
        const double c = fabs(det) < 1e-15 ? 0.0 : -ac[1] / ac[3];
        for (long long k = kb; k < ke; ++k) {
            double *blk = a + k * 4;
            blk[0] = blk[0] + c * blk[2];
            blk[1] = blk[1] + c * blk[3];
        }
        coef[(long long)i * 2] = c;
        coef[(long long)i * 2 + 1] = 0.0;
    } else {
        double binv[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) binv[q] = Ac[(long long)i * 9 + q];
        inv3(binv);
        const double c0 = binv[0], c1 = binv[1];
        for (long long k = kb; k < ke; ++k) {
            double *blk = a + k * 9;
            blk[0] = blk[0] + c0 * blk[3] + c1 * blk[6];
            blk[1] = blk[1] + c0 * blk[4] + c1 * blk[7];
            blk[2] = blk[2] + c0 * blk[5] + c1 * blk[8];
        }
        coef[(long long)i * 2] = c0;
        coef[(long long)i * 2 + 1] = c1;
    }
}

template <int BS>
__global__ void timpes2_rhs_kernel(int nb, const double *__restrict__ coef, double *__restrict__ rhs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    double *r = rhs + (long long)i * BS;
    const double c0 = coef[(long long)i * 2], c1 = coef[(long long)i * 2 + 1];
    if (BS == 2) r[0] = r[0] + c0 * r[1];
    else r[0] = r[0] + c0 * r[1] + c1 * r[2];
}

int decouple_coef_size(int bs, int type) {
    switch (type) {
        case 1: case 2: case 3: case 4: return bs * bs;
        case 5: return 3;
        case 6: return 2;
        default: return 0;
    }
}

void bsr_decouple_matrix(DeviceBsr &A, int type, double *coef, cudaStream_t s, int thermal) {
    const int nb = A.nb;
    if (nb == 0 || type == 0) return;
    if (A.bs != 2 && A.bs != 3) {
        set_error("decouple: unsupported block size %d", A.bs);
        throw CudaError{cudaErrorInvalidValue, "block size"};
    }
    if (type == 1) {
        if (A.bs == 2) abf_kernel<2><<<div_up(nb, 128), 128, 0, s>>>(nb, A.ia.get(), A.a.get(), coef);
        else abf_kernel<3><<<div_up(nb, 128), 128, 0, s>>>(nb, A.ia.get(), A.a.get(), coef);
        JX_LAUNCH_CHECK();
    } else if (type >= 2 && type <= 4) {
        if (A.bs == 2)
            row_transform_kernel<2><<<div_up(nb, 128), 128, 0, s>>>(nb, A.ia.get(), A.a.get(), coef, type, thermal);
        else
            row_transform_kernel<3><<<div_up(nb, 128), 128, 0, s>>>(nb, A.ia.get(), A.a.get(), coef, type, thermal);
        JX_LAUNCH_CHECK();
    } else if (type == 5 || type == 6) {
        DevBuf<int> tia(nb + 1), tja(A.nnzb), tperm(A.nnzb);
        pattern_transpose(nb, nb, A.nnzb, A.ia.get(), A.ja.get(), tia.get(), tja.get(), tperm.get(), s);
        DevBuf<double> Ac((size_t)nb * A.bs * A.bs);
        const int g = div_up(nb, 128);
        if (A.bs == 2) {
            colsum_kernel<2><<<g, 128, 0, s>>>(nb, tia.get(), tperm.get(), A.a.get(), Ac.get());
            JX_LAUNCH_CHECK();
            if (type == 5) timpes_kernel<2><<<g, 128, 0, s>>>(nb, A.ia.get(), Ac.get(), A.a.get(), coef);
            else timpes2_kernel<2><<<g, 128, 0, s>>>(nb, A.ia.get(), Ac.get(), A.a.get(), coef);
        } else {
            colsum_kernel<3><<<g, 128, 0, s>>>(nb, tia.get(), tperm.get(), A.a.get(), Ac.get());
            JX_LAUNCH_CHECK();
            if (type == 5) timpes_kernel<3><<<g, 128, 0, s>>>(nb, A.ia.get(), Ac.get(), A.a.get(), coef);
            else timpes2_kernel<3><<<g, 128, 0, s>>>(nb, A.ia.get(), Ac.get(), A.a.get(), coef);
        }
        JX_LAUNCH_CHECK();
        JX_CUDA(cudaStreamSynchronize(s));
    } else {
        set_error("decouple: unsupported type %d (1 ABF, 2 ANL, 3 SEM, 4 QI, 5 True-IMPES, 6 True-IMPES 2)", type);
        throw CudaError{cudaErrorInvalidValue, "decouple type"};
    }
}

void bsr_decouple_rhs(int nb, int bs, int type, const double *coef, double *rhs, int consistent_rhs,
                      cudaStream_t s) {
    if (nb == 0 || type == 0) return;
    if (type == 1) {
        if (bs == 2) abf_rhs_kernel<2><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs, consistent_rhs);
        else abf_rhs_kernel<3><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs, consistent_rhs);
    } else if (type >= 2 && type <= 4) {
        if (bs == 2) row_rhs_kernel<2><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs, consistent_rhs);
        else row_rhs_kernel<3><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs, consistent_rhs);
    } else if (type == 6) {
        if (bs == 2) timpes2_rhs_kernel<2><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs);
        else timpes2_rhs_kernel<3><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs);
    } else {
        if (bs == 2) timpes_rhs_kernel<2><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs, consistent_rhs);
        else timpes_rhs_kernel<3><<<div_up(nb, 256), 256, 0, s>>>(nb, coef, rhs, consistent_rhs);
    }
    JX_LAUNCH_CHECK();
}

}  // namespace jxcpr
