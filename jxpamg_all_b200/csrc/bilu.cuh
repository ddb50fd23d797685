// Block ILU(0) (the reference's jxf_BILUSetup type 3 + jxf_BILUSolve tri-solve 14) on the device.
#pragma once

#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

struct Bilu {
    int nb = 0, bs = 0;
    int sweeps = 3;       // fixed-point factorisation sweeps (the reference driver's setting)
    int ir_iters = 5;     // iterative-refinement loops of the triangular solve
    int lower_iters = 5;  // Jacobi sweeps on (I + L) y = f
    int upper_iters = 5;  // Jacobi sweeps on (D + U) t = y
    // exact = 1: the exact factors and level-scheduled substitutions (bilu_exact.cu) in place of the
    // sweeps and Jacobi iterations; fp32 = 1: the substitutions read FP32 copies of the factors
    int exact = 0, fp32 = 0;
    DeviceBsr L, U;       // strictly lower / upper blocks in A's entry order
    DevBuf<double> D, Dinv;
    DevBuf<double> ft, ut, yt, un;
    // exact mode: per-row levels of the lower / upper DAGs, rows bucketed by level (ptr, rows)
    int nlev_l = 0, nlev_u = 0, widest = 1;  // level counts, rows of the widest level
    DevBuf<int> lev_l, lev_u, lptr, lrows, uptr, urows;
    std::vector<int> h_lptr, h_uptr;
    DevBuf<float> la32, ua32, dinv32;
    DevBuf<int> subst_err;  // [0] a substitution's grid barrier timed out, [2..3] the barrier
    void setup(const BsrView<double> &A, cudaStream_t s);
    // u += BILU^-1 (f - A u) the reference's way (u = 0 gives u = BILU^-1 f)
    void solve(const BsrView<double> &A, const double *f, double *u, cudaStream_t s);
    void setup_exact(const BsrView<double> &A, cudaStream_t s);
    void substitute(const double *f, double *y, double *t, cudaStream_t s);  // y, t of one refinement loop
    int *error_flag() { return exact ? subst_err.get() : nullptr; }
};

}  // namespace jxcpr
