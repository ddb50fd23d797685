// The small coarse levels of the fast V-cycle in ONE cooperative kernel.
//
// Below a few ten thousand rows a level's passes (smoother steps, residual, restriction,
// prolongation) take 4-8 us each, almost all of it launch and drain latency, and a V-cycle makes
// about ten of them per level.  tail_vcycle_kernel runs every pass of the levels from `first`
// down to the coarsest and back up -- the same passes, in the same order, with the same per-row
// arithmetic as the separate launches (fk::row_kernel's body over a grid-stride loop, dense_gemv's
// warp-per-row product) -- separated by the bounded grid barrier of grid_sync.cuh.  Results are
// bit-identical to the unfused V-cycle.  A barrier that times out raises the hierarchy's error flag
// (the solve then reports a device error) and the kernel returns.
#pragma once

#include "fast.cuh"
#include "fast_kernels.cuh"
#include "grid_sync.cuh"

namespace jxcpr {
namespace tail {

constexpr int kMaxLevels = 12;   // fused levels, the coarsest included
constexpr int kMaxSegs = 10;     // colour classes of a multicolour GS level (max_colors <= 8)
constexpr int kMaxPasses = 40;   // colour passes of one GS smoothing (4 sweeps x classes)

// One operator in its fast-path layout (CSR with `lanes` lanes per row, or sliced ELL with `sell` lanes
// per row).
template <typename TV>
struct Mat {
    int sell, lanes, nstored;
    const int *ia, *ja, *perm;
    const long long *sp;
    const int *rows;
    const TV *a;
    const float *bscale;
};

template <typename TX, typename TV>
struct Level {
    int n, smoother, nseg, npass;
    int seg[kMaxSegs];
    unsigned char pass[kMaxPasses];  // colour class of each GS pass of one smoothing
    Mat<TV> A;                       // the level's operator (TV: its storage type)
    Mat<TX> P, R;                    // P: from level + 1 (n rows); R: to level + 1 (stored as TX)
    TX c0, c1, c2;                   // Chebyshev coefficients
    const TX *dinv, *dinv_l1;
    TX *f, *u, *r, *z, *y1, *y2;
};

template <typename TX, typename TV>
struct Desc {
    int nlev;  // fused levels; lv[nlev - 1] is the coarsest (solved by the dense inverse)
    Level<TX, TV> lv[kMaxLevels];
    int nc;
    const double *Ainv;
};

// fk::row_kernel's body for stored rows [r0, r1) over a grid-stride loop whose trip count is
// uniform across a warp (every lane of a row group reaches the group's shuffles)
template <class Fmt, class Op, typename TX>
__device__ __forceinline__ void rows_pass(const Fmt &fmt, const Op &op, int r0, int r1) {
    const long long total = (long long)(r1 - r0) * Fmt::V;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < total; base += stride) {
        const long long gt = base + threadIdx.x;
        const int t = r0 + (int)(gt / Fmt::V);
        const int lane = (int)(gt % Fmt::V);
        const bool live = t < r1;
        const int i = live ? fmt.row(t) : -1;
        const bool own = i >= 0 && lane == 0;
        typename Op::Pre pre;
        if (own) op.load(i, pre);
        TX s = 0;
        if (op.need_sum()) s = fmt.template sum<TX, TX>(t, i >= 0, lane, op.x(), Op::kstart);
        if (own) op.store(i, s, pre);
    }
}

template <typename TX, typename TV, class Op>
__device__ __noinline__ void mat_pass(const Mat<TV> &M, const Op &op, int r0, int r1) {
    if (r1 <= r0) return;
    if (M.sell == 2) {
        fk::SellFmt<TV, 2> f{M.sp, M.ja, M.a, M.bscale, M.rows};
        rows_pass<fk::SellFmt<TV, 2>, Op, TX>(f, op, r0, r1);
        return;
    }
    if (M.sell) {
        fk::SellFmt<TV> f{M.sp, M.ja, M.a, M.bscale, M.rows};
        rows_pass<fk::SellFmt<TV>, Op, TX>(f, op, r0, r1);
        return;
    }
#define JX_TAIL_CSR(VV)                                          \
    {                                                            \
        fk::CsrFmt<VV, TV> f{M.ia, M.ja, M.a, M.bscale, M.perm}; \
        rows_pass<fk::CsrFmt<VV, TV>, Op, TX>(f, op, r0, r1);    \
    }                                                            \
    break;
    switch (M.lanes) {
        case 1: JX_TAIL_CSR(1)
        case 2: JX_TAIL_CSR(2)
        case 4: JX_TAIL_CSR(4)
        case 8: JX_TAIL_CSR(8)
        case 16: JX_TAIL_CSR(16)
        default: JX_TAIL_CSR(32)
    }
#undef JX_TAIL_CSR
}

// The level's smoother (FastCpr::smooth), a barrier after every pass.  Returns false on a barrier
// time-out.
template <typename TX, typename TV>
__device__ bool smooth(const Level<TX, TV> &L, bool zero, GridBarrier *bar, int *err) {
    if (L.smoother == FS_COLOR_GS) {
        for (int p = 0; p < L.npass; ++p) {
            const int c = L.pass[p];
            fk::OpGs<TX> op{L.f, L.dinv, L.u, zero ? 1 : 0};
            mat_pass<TX, TV>(L.A, op, L.seg[c], L.seg[c + 1]);
            zero = false;
            if (!grid_barrier(bar, gridDim.x, err)) return false;
        }
    } else if (L.smoother == FS_L1_JACOBI) {
        for (int rep = 0; rep < 2; ++rep) {
            fk::OpJacobi<TX> a{L.f, L.dinv_l1, L.u, L.z, zero ? 1 : 0};
            mat_pass<TX, TV>(L.A, a, 0, L.A.nstored);
            if (!grid_barrier(bar, gridDim.x, err)) return false;
            fk::OpJacobi<TX> b{L.f, L.dinv_l1, L.z, L.u, 0};
            mat_pass<TX, TV>(L.A, b, 0, L.A.nstored);
            if (!grid_barrier(bar, gridDim.x, err)) return false;
            zero = false;
        }
    } else {
        fk::OpCheb<TX> c0{0, zero ? 1 : 0, L.c2, L.f, L.dinv, nullptr, L.u, L.z, L.y1};
        mat_pass<TX, TV>(L.A, c0, 0, L.A.nstored);
        if (!grid_barrier(bar, gridDim.x, err)) return false;
        fk::OpCheb<TX> c1{1, 0, L.c1, L.f, L.dinv, L.y1, L.u, L.z, L.y2};
        mat_pass<TX, TV>(L.A, c1, 0, L.A.nstored);
        if (!grid_barrier(bar, gridDim.x, err)) return false;
        fk::OpCheb<TX> c2{2, zero ? 1 : 0, L.c0, L.f, L.dinv, L.y2, L.u, L.z, nullptr};
        mat_pass<TX, TV>(L.A, c2, 0, L.A.nstored);
        if (!grid_barrier(bar, gridDim.x, err)) return false;
    }
    return true;
}

// V-cycle over the fused levels from a zero initial guess: lv[0].f in, lv[0].u out.
template <typename TX, typename TV>
__global__ void __launch_bounds__(256, 4) tail_vcycle_kernel(const Desc<TX, TV> *__restrict__ dp, GridBarrier *bar,
                                                          int *err) {
    const Desc<TX, TV> &d = *dp;
    const int nl = d.nlev;
    const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long gstride = (long long)gridDim.x * blockDim.x;
    for (int l = 0; l + 1 < nl; ++l) {
        const Level<TX, TV> &L = d.lv[l];
        if (L.smoother == FS_COLOR_GS) {
            for (long long e = gtid; e < L.n; e += gstride) L.u[e] = (TX)0;
            if (!grid_barrier(bar, gridDim.x, err)) return;
        }
        if (!smooth<TX, TV>(L, true, bar, err)) return;
        fk::OpResid<TX> res{L.f, L.u, L.r};
        mat_pass<TX, TV>(L.A, res, 0, L.A.nstored);
        if (!grid_barrier(bar, gridDim.x, err)) return;
        fk::OpSpmv<TX> rst{L.r, d.lv[l + 1].f, 0};
        mat_pass<TX, TX>(L.R, rst, 0, L.R.nstored);
        if (!grid_barrier(bar, gridDim.x, err)) return;
    }
    {  // coarsest: u = Ainv f, one warp per row (fk::dense_gemv's order)
        const Level<TX, TV> &C = d.lv[nl - 1];
        const int n = d.nc, lane = threadIdx.x & 31;
        const long long warps = gstride >> 5;
        for (long long row = gtid >> 5; row < n; row += warps) {
            double s = 0.0;
            for (int c = lane; c < n; c += 32) s += d.Ainv[row * n + c] * (double)C.f[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) C.u[row] = (TX)s;
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
    }
    for (int l = nl - 2; l >= 0; --l) {
        const Level<TX, TV> &L = d.lv[l];
        fk::OpSpmv<TX> pro{d.lv[l + 1].u, L.u, 1};
        mat_pass<TX, TX>(L.P, pro, 0, L.P.nstored);
        if (!grid_barrier(bar, gridDim.x, err)) return;
        if (!smooth<TX, TV>(L, false, bar, err)) return;
    }
}

}  // namespace tail
}  // namespace jxcpr
