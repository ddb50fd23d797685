// Block ILU(0) (the reference's jxf_BILUSetup type 3 + jxf_BILUSolve tri-solve 14) on the device.
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

struct Bilu {
    int nb = 0, bs = 0;
    int sweeps = 3;       // fixed-point factorisation sweeps (the reference driver's setting)
    int ir_iters = 5;     // iterative-refinement loops of the triangular solve
    int lower_iters = 5;  // Jacobi sweeps on (I + L) y = f
    int upper_iters = 5;  // Jacobi sweeps on (D + U) t = y
    DeviceBsr L, U;       // strictly lower / upper blocks in A's entry order
    DevBuf<double> D, Dinv;
    DevBuf<double> ft, ut, yt, un;
    void setup(const BsrView<double> &A, cudaStream_t s);
    // u += BILU^-1 (f - A u) the reference's way (u = 0 gives u = BILU^-1 f)
    void solve(const BsrView<double> &A, const double *f, double *u, cudaStream_t s);
};

}  // namespace jxcpr
