// Device kernels of the fast (throughput / mixed-precision) CPR path.
//
// Every kernel is templated on the value storage type TV (double, float or
// __nv_bfloat16 with a per-block scale) and the vector type TX (double or float;
// arithmetic is done in TX).  Rows are reduced by V lanes of a warp (V a power
// of two <= 32): lane l takes entries kb+l, kb+l+V, ... and the V partial sums
// are combined with xor-shuffles, so every lane of a group must reach the
// shuffles (out-of-range groups reduce an empty row).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace jxcpr {
namespace fk {

__device__ __forceinline__ double ldv(const double *p, long long k) { return __ldg(p + k); }
__device__ __forceinline__ float ldv(const float *p, long long k) { return __ldg(p + k); }
__device__ __forceinline__ float ldv(const __nv_bfloat16 *p, long long k) { return __bfloat162float(__ldg(p + k)); }
// Value k of an operator's storage: BF16 values carry one power-of-two FP32 scale per 32 consecutive
// stored values (bsc[k / 32]; a block scale, exact to apply), FP64 / FP32 values none.
__device__ __forceinline__ double ldvs(const double *p, const float *, long long k) { return __ldg(p + k); }
__device__ __forceinline__ float ldvs(const float *p, const float *, long long k) { return __ldg(p + k); }
__device__ __forceinline__ float ldvs(const __nv_bfloat16 *p, const float *bsc, long long k) {
    return __bfloat162float(__ldg(p + k)) * __ldg(bsc + (k >> 5));
}

template <int V, typename TA>
__device__ __forceinline__ TA group_sum(TA v) {
#pragma unroll
    for (int o = V / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, V);
    return v;
}

// sum_{k in [kb, ke)} a_k x_{ja_k}, reduced over the V lanes of the group.
// Two entries per lane per trip keep more loads in flight; each product is added with one fused
// multiply-add (the fast path has no bit-exactness contract; the exact path's kernels do not use it).
template <int V, typename TA, typename TV, typename TX>
__device__ __forceinline__ TA row_sum(const int *__restrict__ ja, const TV *__restrict__ a, const float *bsc, int kb,
                                      int ke, const TX *x, int lane) {
    TA s0 = 0, s1 = 0;
    int k = kb + lane;
    for (; k + V < ke; k += 2 * V) {
        const int j0 = __ldg(ja + k), j1 = __ldg(ja + k + V);
        const TA a0 = (TA)ldvs(a, bsc, k), a1 = (TA)ldvs(a, bsc, k + V);
        s0 = fma(a0, (TA)x[j0], s0);
        s1 = fma(a1, (TA)x[j1], s1);
    }
    if (k < ke) s0 = fma((TA)ldvs(a, bsc, k), (TA)x[__ldg(ja + k)], s0);
    return group_sum<V, TA>(s0 + s1);
}

// ---- matrix formats -----------------------------------------------------------
// CSR with V lanes per row.  Stored row t maps to vector row perm[t] (perm ==
// nullptr: identity); bscale (BF16 storage): one scale per 32 consecutive stored values.
template <int V_, typename TV>
struct CsrFmt {
    static constexpr int V = V_;
    const int *ia, *ja;
    const TV *a;
    const float *bscale;
    const int *perm;
    __device__ __forceinline__ int row(int t) const { return perm ? __ldg(perm + t) : t; }
    template <typename TA, typename TX>
    __device__ __forceinline__ TA sum(int t, bool live, int lane, const TX *x, int kstart) const {
        const int e = live ? __ldg(ia + t + 1) : 0;
        int d = live ? __ldg(ia + t) + kstart : 0;
        if (d > e) d = e;
        return row_sum<V, TA>(ja, a, bscale, d, e, x, lane);
    }
};

// Sliced ELL: 32-row slices stored slot-major, entry k of stored row t at
// sp[t/32] + 32 k + t%32 (padding: value 0, column 0).  rows[t] is the vector
// row of stored row t (-1: padding row).  One thread per row: the 32 rows of a
// warp read each slot with one coalesced access.
// P = 2: two lanes per row.  Stored row t is split into the virtual rows 2t and 2t + 1, holding its
// entries of even and odd position; the virtual rows form the 32-row slices (16 stored rows each),
// and the pair's sums are added with one shuffle.
template <typename TV, int P = 1>
struct SellFmt {
    static constexpr int V = P;
    const long long *sp;
    const int *col;
    const TV *a;
    const float *bscale;  // BF16: one scale per 32 stored values (one slot of a slice)
    const int *rows;
    __device__ __forceinline__ int row(int t) const { return __ldg(rows + t); }
    template <typename TA, typename TX>
    __device__ __forceinline__ TA sum(int t, bool live, int lane, const TX *x, int kstart) const {
        if constexpr (P == 1) {
            if (!live) return 0;
            return slots<TA>((long long)t, x, kstart);
        } else {
            // every lane takes part in the shuffle, live or not; lane h holds positions h, h + P, ...
            const TA s = live ? slots<TA>((long long)t * P + lane, x, kstart > lane ? (kstart - lane + P - 1) / P : 0)
                              : (TA)0;
            return group_sum<P, TA>(s);
        }
    }
    // slots [kstart, width) of virtual row vt
    template <typename TA, typename TX>
    __device__ __forceinline__ TA slots(long long vt, const TX *x, int kstart) const {
        const long long b0 = __ldg(sp + (vt >> 5)), b1 = __ldg(sp + (vt >> 5) + 1);
        const int w = (int)((b1 - b0) >> 5);
        const long long o = b0 + (vt & 31);
        TA s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        int k = kstart;
        for (; k + 3 < w; k += 4) {
            const long long p = o + (long long)k * 32;
            const int j0 = __ldg(col + p), j1 = __ldg(col + p + 32), j2 = __ldg(col + p + 64),
                      j3 = __ldg(col + p + 96);
            const TA a0 = (TA)ldvs(a, bscale, p), a1 = (TA)ldvs(a, bscale, p + 32), a2 = (TA)ldvs(a, bscale, p + 64),
                     a3 = (TA)ldvs(a, bscale, p + 96);
            s0 = fma(a0, (TA)x[j0], s0);
            s1 = fma(a1, (TA)x[j1], s1);
            s2 = fma(a2, (TA)x[j2], s2);
            s3 = fma(a3, (TA)x[j3], s3);
        }
        for (; k < w; ++k) {
            const long long p = o + (long long)k * 32;
            s0 = fma((TA)ldvs(a, bscale, p), (TA)x[__ldg(col + p)], s0);
        }
        return (s0 + s1) + (s2 + s3);
    }
};

// ---- row operations (prologue loads issued before the row sum) -----------------
// Gauss-Seidel on one colour class: u_i = (f_i - sum_{j != i} a_ij u_j) dinv_i
// (the diagonal is the first stored entry; dinv_i == 0 leaves the row).
template <typename TX>
struct OpGs {
    static constexpr int kstart = 1;
    const TX *f, *dinv;
    TX *u;
    int zero;  // every neighbour is 0 (first class after u = 0)
    struct Pre { TX f, d; };
    __device__ __forceinline__ const TX *x() const { return u; }
    __device__ __forceinline__ bool need_sum() const { return !zero; }
    __device__ __forceinline__ void load(int i, Pre &p) const { p.f = f[i]; p.d = dinv[i]; }
    __device__ __forceinline__ void store(int i, TX s, const Pre &p) const {
        if (p.d != (TX)0) u[i] = (p.f - s) * p.d;
    }
};
// unew_i = u_i + (f_i - (A u)_i) dinv_i
template <typename TX>
struct OpJacobi {
    static constexpr int kstart = 0;
    const TX *f, *dinv, *u;
    TX *unew;
    int zero;  // u == 0
    struct Pre { TX f, d, u; };
    __device__ __forceinline__ const TX *x() const { return u; }
    __device__ __forceinline__ bool need_sum() const { return !zero; }
    __device__ __forceinline__ void load(int i, Pre &p) const {
        p.f = f[i];
        p.d = dinv[i];
        p.u = zero ? (TX)0 : u[i];
    }
    __device__ __forceinline__ void store(int i, TX s, const Pre &p) const { unew[i] = p.u + (p.f - s) * p.d; }
};
// r_i = f_i - (A u)_i
template <typename TX>
struct OpResid {
    static constexpr int kstart = 0;
    const TX *f, *u;
    TX *r;
    struct Pre { TX f; };
    __device__ __forceinline__ const TX *x() const { return u; }
    __device__ __forceinline__ bool need_sum() const { return true; }
    __device__ __forceinline__ void load(int i, Pre &p) const { p.f = f[i]; }
    __device__ __forceinline__ void store(int i, TX s, const Pre &p) const { r[i] = p.f - s; }
};
// y = A x (+ y)
template <typename TX>
struct OpSpmv {
    static constexpr int kstart = 0;
    const TX *xin;
    TX *y;
    int beta_one;
    struct Pre { TX y; };
    __device__ __forceinline__ const TX *x() const { return xin; }
    __device__ __forceinline__ bool need_sum() const { return true; }
    __device__ __forceinline__ void load(int i, Pre &p) const { p.y = beta_one ? y[i] : (TX)0; }
    __device__ __forceinline__ void store(int i, TX s, const Pre &p) const { y[i] = beta_one ? p.y + s : s; }
};
// Degree-3 polynomial smoother, Horner form of u += p(M) z, M = D^-1 A,
// z = D^-1 (f - A u), p(t) = c0 + c1 t + c2 t^2:
//   mode 0: z = D^-1 (f - A u), yout = c z          (c = c2; zero: u == 0)
//   mode 1: yout = c z + D^-1 A yin                  (c = c1)
//   mode 2: u = (zero ? 0 : u) + c z + D^-1 A yin    (c = c0)
template <typename TX>
struct OpCheb {
    static constexpr int kstart = 0;
    int mode, zero;
    TX c;
    const TX *f, *dinv, *yin;
    TX *u, *z, *yout;
    struct Pre { TX d, a, b; };
    __device__ __forceinline__ const TX *x() const { return mode == 0 ? u : yin; }
    __device__ __forceinline__ bool need_sum() const { return !(mode == 0 && zero); }
    __device__ __forceinline__ void load(int i, Pre &p) const {
        p.d = dinv[i];
        if (mode == 0) {
            p.a = f[i];
        } else {
            p.a = z[i];
            p.b = (mode == 2 && !zero) ? u[i] : (TX)0;
        }
    }
    __device__ __forceinline__ void store(int i, TX s, const Pre &p) const {
        if (mode == 0) {
            const TX zi = (p.a - s) * p.d;
            z[i] = zi;
            yout[i] = c * zi;
        } else if (mode == 1) {
            yout[i] = c * p.a + p.d * s;
        } else {
            u[i] = p.b + c * p.a + p.d * s;
        }
    }
};

// One launch of `op` over stored rows [r0, r1) of a matrix in format Fmt.
template <class Fmt, class Op, typename TX>
__global__ void __launch_bounds__(256) row_kernel(Fmt fmt, Op op, int r0, int r1) {
    grid_dep_wait();
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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

template <typename TX>
__global__ void restrict_p(int nb, int bs, int p, const double *__restrict__ r, TX *__restrict__ rp) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nb) rp[i] = (TX)r[(long long)i * bs + p];
}

template <typename TX, typename TZ>
__global__ void prolong_p(int nb, int bs, int p, const TX *__restrict__ up, TZ *__restrict__ z) {
    grid_dep_wait();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * bs) return;
    const int i = (int)(t / bs), k = (int)(t % bs);
    z[t] = k == p ? (TZ)up[i] : (TZ)0;
}

// rp = r[p-th component] and r32 = r converted (mixed path: stage 2 works in FP32)
template <typename TX>
__global__ void restrict_cvt(int nb, int bs, int p, const double *__restrict__ r, TX *__restrict__ rp,
                             float *__restrict__ r32) {
    grid_dep_wait();
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nb * bs) return;
    const double v = r[t];
    r32[t] = (float)v;
    if ((int)(t % bs) == p) rp[t / bs] = (TX)v;
}

// u = Ainv f (FP64 inverse of the coarsest operator), one warp per row.
template <typename TX>
__global__ void dense_gemv(int n, const double *__restrict__ Ainv, const TX *__restrict__ f, TX *__restrict__ u) {
    grid_dep_wait();
    const int row = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int c = lane; c < n; c += 32) s += Ainv[(long long)row * n + c] * (double)f[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) u[row] = (TX)s;
}

// ---- stage 2: hybrid block Gauss-Seidel, one colour class -------------------
template <int BS, typename TV, typename TA>
__device__ __forceinline__ void load_block(const TV *__restrict__ a, long long k, TA out[BS * BS]) {
#pragma unroll
    for (int q = 0; q < BS * BS; ++q) out[q] = (TA)ldv(a, k * BS * BS + q);
}
template <>
__device__ __forceinline__ void load_block<2, double, double>(const double *__restrict__ a, long long k,
                                                              double out[4]) {
    const double2 *p = reinterpret_cast<const double2 *>(a + k * 4);
    const double2 v0 = __ldg(p), v1 = __ldg(p + 1);
    out[0] = v0.x;
    out[1] = v0.y;
    out[2] = v1.x;
    out[3] = v1.y;
}
template <>
__device__ __forceinline__ void load_block<2, float, float>(const float *__restrict__ a, long long k,
                                                            float out[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(a + k * 4));
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
}

// The same with the cache-streaming hint (ld.global.cs): the chunk-ordered stage-2 sweep streams its
// matrix once per sweep, and marking those lines evict-first keeps the gathered vectors (x, the
// start values) in L1 / L2 (measured 56 -> 47 us per sweep on C1; the CSR level passes, whose lanes
// share sectors across trips, measured slower with it and keep the default loads).
__device__ __forceinline__ double ldv_cs(const double *p, long long k) { return __ldcs(p + k); }
__device__ __forceinline__ float ldv_cs(const float *p, long long k) { return __ldcs(p + k); }
template <int BS, typename TV, typename TA>
__device__ __forceinline__ void load_block_cs(const TV *__restrict__ a, long long k, TA out[BS * BS]) {
#pragma unroll
    for (int q = 0; q < BS * BS; ++q) out[q] = (TA)ldv_cs(a, k * BS * BS + q);
}
template <>
__device__ __forceinline__ void load_block_cs<2, double, double>(const double *__restrict__ a, long long k,
                                                                 double out[4]) {
    const double2 *p = reinterpret_cast<const double2 *>(a + k * 4);
    const double2 v0 = __ldcs(p), v1 = __ldcs(p + 1);
    out[0] = v0.x;
    out[1] = v0.y;
    out[2] = v1.x;
    out[3] = v1.y;
}
template <>
__device__ __forceinline__ void load_block_cs<2, float, float>(const float *__restrict__ a, long long k,
                                                               float out[4]) {
    const float4 v = __ldcs(reinterpret_cast<const float4 *>(a + k * 4));
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
}

template <int BS, typename TA>
__device__ __forceinline__ void block_solve(const TA D[BS * BS], const TA rhs[BS], TA out[BS]) {
    if (BS == 2) {
        const TA det = D[0] * D[3] - D[1] * D[2];
        const TA inv = det != (TA)0 ? (TA)1 / det : (TA)0;
        out[0] = (D[3] * rhs[0] - D[1] * rhs[1]) * inv;
        out[1] = (D[0] * rhs[1] - D[2] * rhs[0]) * inv;
    } else {
        // adjugate / determinant of a 3x3 block
        const TA c00 = D[4] * D[8] - D[5] * D[7], c01 = D[5] * D[6] - D[3] * D[8], c02 = D[3] * D[7] - D[4] * D[6];
        const TA det = D[0] * c00 + D[1] * c01 + D[2] * c02;
        const TA inv = det != (TA)0 ? (TA)1 / det : (TA)0;
        const TA c10 = D[2] * D[7] - D[1] * D[8], c11 = D[0] * D[8] - D[2] * D[6], c12 = D[1] * D[6] - D[0] * D[7];
        const TA c20 = D[1] * D[5] - D[2] * D[4], c21 = D[2] * D[3] - D[0] * D[5], c22 = D[0] * D[4] - D[1] * D[3];
        out[0] = (c00 * rhs[0] + c10 * rhs[1] + c20 * rhs[2]) * inv;
        out[1] = (c01 * rhs[0] + c11 * rhs[1] + c21 * rhs[2]) * inv;
        out[2] = (c02 * rhs[0] + c12 * rhs[1] + c22 * rhs[2]) * inv;
    }
}

// x_i <- (1 - w omega) x_i + w D_i^-1 (omega b_i - sum_{j != i} A_ij (x_j - (1 - omega) vt_j))
// (jxf_ParBSRHGSRelax's update with res = b, res0 = -sum A x, res2 = sum A vt);
// plain (w = omega = 1): x_i <- D_i^-1 (b_i - sum A_ij x_j).  vt_j = x_j at the sweep start.
//
// No start-of-sweep copy: a colour class's launch saves its rows' old values in vt (save = 1)
// before updating them, and a neighbour's vt_j is read only if its class came earlier in this
// sweep -- otherwise x_j still holds the start value.  nmode 0: every neighbour comes later (the
// first class), 1: every neighbour came earlier (the last class), 2: decided per neighbour by its
// class index cls[j] against this launch's cur.  The arithmetic is the copy-based sweep's.
struct SweepOrder {
    int nmode, save, cur;
    const int *cls;
};

template <typename TA, typename TXV>
__device__ __forceinline__ TA start_value(const TXV *x, TXV *vt, long long o, int j, SweepOrder so) {
    const bool earlier = so.nmode == 1 || (so.nmode == 2 && __ldg(so.cls + j) < so.cur);
    return earlier ? (TA)__ldg(vt + o) : (TA)x[o];
}

template <int BS, int V, typename TV, typename TA, typename TXV>
__global__ void hgs_color(int r0, int r1, const int *__restrict__ perm, const int *__restrict__ ia,
                          const int *__restrict__ ja, const TV *__restrict__ a, const TXV *__restrict__ b,
                          TXV *x, TXV *vt, TA w, TA omega, int plain, SweepOrder so) {
    grid_dep_wait();
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int t = r0 + (int)(gt / V);
    const int lane = (int)(gt % V);
    const bool live = t < r1;
    const int d = live ? ia[t] : 0, e = live ? ia[t + 1] : 0;
    const TA omo = (TA)1 - omega;
    TA acc[BS];
#pragma unroll
    for (int q = 0; q < BS; ++q) acc[q] = 0;
    for (int k = d + 1 + lane; k < e; k += V) {
        const int j = __ldg(ja + k);
        TA blk[BS * BS], c[BS];
        load_block<BS, TV, TA>(a, k, blk);
#pragma unroll
        for (int m = 0; m < BS; ++m) {
            const TA xj = (TA)x[(long long)j * BS + m];
            c[m] = plain ? xj : xj - omo * start_value<TA, TXV>(x, vt, (long long)j * BS + m, j, so);
        }
#pragma unroll
        for (int q = 0; q < BS; ++q)
#pragma unroll
            for (int m = 0; m < BS; ++m) acc[q] += blk[q * BS + m] * c[m];
    }
#pragma unroll
    for (int q = 0; q < BS; ++q) acc[q] = group_sum<V, TA>(acc[q]);
    if (!live || lane != 0) return;
    const int i = perm[t];
    TA D[BS * BS], rhs[BS], out[BS];
    load_block<BS, TV, TA>(a, d, D);
#pragma unroll
    for (int q = 0; q < BS; ++q) rhs[q] = (plain ? (TA)1 : omega) * (TA)b[(long long)i * BS + q] - acc[q];
    block_solve<BS, TA>(D, rhs, out);
    const TA prod = (TA)1 - w * omega;
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        const long long o = (long long)i * BS + q;
        const TXV old = x[o];
        if (!plain && so.save) vt[o] = old;
        x[o] = plain ? (TXV)out[q] : (TXV)(prod * (TA)old + w * out[q]);
    }
}

// Stage 2 on a sliced-ELL block copy (one thread per block row, slot 0 = the
// diagonal block, padding blocks are zero): same update as hgs_color.
template <int BS, typename TV, typename TA, typename TXV>
__global__ void __launch_bounds__(256) hgs_sell(int r0, int r1, const long long *__restrict__ sp,
                                                const int *__restrict__ col, const TV *__restrict__ a,
                                                const int *__restrict__ rows, const TXV *__restrict__ b,
                                                TXV *x, TXV *vt, TA w, TA omega, int plain, SweepOrder so) {
    grid_dep_wait();
    const int t = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= r1) return;
    const int i = __ldg(rows + t);
    if (i < 0) return;
    const long long b0 = __ldg(sp + (t >> 5)), b1 = __ldg(sp + (t >> 5) + 1);
    const int wd = (int)((b1 - b0) >> 5);
    const long long o = b0 + (t & 31);
    const TA omo = (TA)1 - omega;
    TA rhs[BS], xv[BS], D[BS * BS], acc[BS];
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        rhs[q] = (TA)__ldg(b + (long long)i * BS + q);
        xv[q] = plain ? (TA)0 : (TA)x[(long long)i * BS + q];
        acc[q] = 0;
    }
    load_block<BS, TV, TA>(a, o, D);
    int k = 1;
    for (; k + 1 < wd; k += 2) {
        const long long p0 = o + (long long)k * 32, p1 = p0 + 32;
        const int j0 = __ldg(col + p0), j1 = __ldg(col + p1);
        TA B0[BS * BS], B1[BS * BS], c0[BS], c1[BS];
        load_block<BS, TV, TA>(a, p0, B0);
        load_block<BS, TV, TA>(a, p1, B1);
#pragma unroll
        for (int m = 0; m < BS; ++m) {
            const TA x0 = (TA)x[(long long)j0 * BS + m], x1 = (TA)x[(long long)j1 * BS + m];
            c0[m] = plain ? x0 : x0 - omo * start_value<TA, TXV>(x, vt, (long long)j0 * BS + m, j0, so);
            c1[m] = plain ? x1 : x1 - omo * start_value<TA, TXV>(x, vt, (long long)j1 * BS + m, j1, so);
        }
#pragma unroll
        for (int q = 0; q < BS; ++q)
#pragma unroll
            for (int m = 0; m < BS; ++m) acc[q] += B0[q * BS + m] * c0[m] + B1[q * BS + m] * c1[m];
    }
    if (k < wd) {
        const long long p0 = o + (long long)k * 32;
        const int j0 = __ldg(col + p0);
        TA B0[BS * BS], c0[BS];
        load_block<BS, TV, TA>(a, p0, B0);
#pragma unroll
        for (int m = 0; m < BS; ++m) {
            const TA x0 = (TA)x[(long long)j0 * BS + m];
            c0[m] = plain ? x0 : x0 - omo * start_value<TA, TXV>(x, vt, (long long)j0 * BS + m, j0, so);
        }
#pragma unroll
        for (int q = 0; q < BS; ++q)
#pragma unroll
            for (int m = 0; m < BS; ++m) acc[q] += B0[q * BS + m] * c0[m];
    }
    TA r2[BS], out[BS];
#pragma unroll
    for (int q = 0; q < BS; ++q) r2[q] = (plain ? (TA)1 : omega) * rhs[q] - acc[q];
    block_solve<BS, TA>(D, r2, out);
    const TA prod = (TA)1 - w * omega;
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        if (!plain && so.save) vt[(long long)i * BS + q] = (TXV)xv[q];
        x[(long long)i * BS + q] = plain ? (TXV)out[q] : (TXV)(prod * xv[q] + w * out[q]);
    }
}

// Stage 2 in chunk order (the throughput path's default): block rows are grouped in chunks of CH
// consecutive rows (natural numbering, chunk = row / CH), the chunks coloured so that no two chunks
// of one colour are coupled; a sweep visits the colours in turn and each chunk's rows in natural
// order, i.e. the block update of hgs_color in that sequential order.  Storage: sliced ELL with each
// colour a run of whole chunks, CH-aligned inside the 32-row slices (lane p of a chunk holds its row
// p; padding rows -1), rows not sorted by length.
//   Phase 1, every row at once: D_i^-1, and the sum over the entries outside the row's chunk
//   (earlier colours: current value and saved start value; later colours: the start value) and over
//   its in-chunk entries of higher index (not updated yet: the start value); of an in-chunk entry of
//   lower index j only the start-value term -(1 - omega) A_ij vt_j.  Then u_i = D_i^-1 (omega b_i -
//   sum) and, for the first in-chunk lower entry, G = D_i^-1 A_ij.
//   Phase 2, CH steps: at step r lane r of every chunk forms out = u - (sum of G x_j(new)), updates
//   and writes x; the new value is shuffled to the chunk's other lanes, whose rows coupled to it add
//   G x_j (the kept entry; any further in-chunk lower entry is re-read and multiplied by D_i^-1).
//   The chain from one row to the next is one shuffle and a BS x BS product.
template <int BS, typename TA>
__device__ __forceinline__ void block_inverse(const TA D[BS * BS], TA Di[BS * BS]) {
    if (BS == 2) {
        const TA det = D[0] * D[3] - D[1] * D[2];
        const TA inv = det != (TA)0 ? (TA)1 / det : (TA)0;
        Di[0] = D[3] * inv;
        Di[1] = -D[1] * inv;
        Di[2] = -D[2] * inv;
        Di[3] = D[0] * inv;
    } else {
        const TA c00 = D[4] * D[8] - D[5] * D[7], c01 = D[5] * D[6] - D[3] * D[8], c02 = D[3] * D[7] - D[4] * D[6];
        const TA det = D[0] * c00 + D[1] * c01 + D[2] * c02;
        const TA inv = det != (TA)0 ? (TA)1 / det : (TA)0;
        const TA c10 = D[2] * D[7] - D[1] * D[8], c11 = D[0] * D[8] - D[2] * D[6], c12 = D[1] * D[6] - D[0] * D[7];
        const TA c20 = D[1] * D[5] - D[2] * D[4], c21 = D[2] * D[3] - D[0] * D[5], c22 = D[0] * D[4] - D[1] * D[3];
        Di[0] = c00 * inv; Di[1] = c10 * inv; Di[2] = c20 * inv;
        Di[3] = c01 * inv; Di[4] = c11 * inv; Di[5] = c21 * inv;
        Di[6] = c02 * inv; Di[7] = c12 * inv; Di[8] = c22 * inv;
    }
}

template <int BS, typename TA>
__device__ __forceinline__ void block_matvec(const TA M[BS * BS], const TA v[BS], TA out[BS]) {
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        TA t = 0;
#pragma unroll
        for (int m = 0; m < BS; ++m) t += M[q * BS + m] * v[m];
        out[q] = t;
    }
}

// The two values of a 2-vector entry j of x (FP32: one 8-byte load; x's base is 8-byte aligned, which
// the stage-2 launcher checks).  NC: through the read-only path, valid where no thread of the launch
// writes the entry before it is read.
template <typename TXV, typename TA, bool NC>
__device__ __forceinline__ void ld_pair(const TXV *p, int j, TA out[2]) {
    if constexpr (sizeof(TXV) == 4) {
        const float2 v = NC ? __ldg(reinterpret_cast<const float2 *>(p) + j) : reinterpret_cast<const float2 *>(p)[j];
        out[0] = (TA)v.x;
        out[1] = (TA)v.y;
    } else {
        out[0] = (TA)(NC ? __ldg(p + 2LL * j) : p[2LL * j]);
        out[1] = (TA)(NC ? __ldg(p + 2LL * j + 1) : p[2LL * j + 1]);
    }
}

// Column words of the chunk-ordered stage-2 matrix: the column in the low 30 bits, bit 30 set when the
// neighbour's colour comes earlier in the sweep (its start value is in vt), bit 31 when it lies in the
// row's own chunk.  The sweep order is fixed at setup, so the relation is stored, not looked up.
constexpr unsigned kChunkColMask = 0x3fffffffu, kChunkEarlier = 1u << 30, kChunkSame = 1u << 31;

// FP32 arithmetic: 5 blocks of 256 threads per SM for 2x2 blocks (<= 51 registers), so that enough rows'
// loads are in flight, 4 for 3x3 (<= 64 registers: the row state of 3x3 blocks spills below that);
// FP64: 3 (<= 85 registers).  To keep the state small, the diagonal block, b and the row's own x are
// loaded after the entry loop, and for 2x2 blocks the kept in-chunk block is re-read by its slot
// rather than held (measured on C1: 46.9 -> 41.1 us per sweep with the paired x gathers; C4: 103 ->
// 79 us).
template <int BS, int CH, typename TV, typename TA, typename TXV>
__global__ void __launch_bounds__(256, sizeof(TA) == 4 ? (BS == 2 ? 5 : 4) : 3) hgs_chunk(int r0, int r1, const long long *__restrict__ sp,
                                                 const unsigned *__restrict__ col, const TV *__restrict__ a,
                                                 const int *__restrict__ rows, const TXV *__restrict__ b,
                                                 TXV *x, TXV *vt, TA w, TA omega, int plain, int save) {
    static_assert(32 % CH == 0, "chunks tile the 32-row slices");
    constexpr bool kKeepSlot = BS == 2;  // hold the kept in-chunk block's slot, not its values
    constexpr int NB = BS == 2 ? 4 : 2;  // entries loaded per batch
    grid_dep_wait();
    const int t = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int p = lane % CH;
    const int i = t < r1 ? __ldg(rows + t) : -1;
    const bool live = i >= 0;
    const int cbase = i - p;  // first row of the chunk (row i sits at lane p of its chunk)
    const TA omo = (TA)1 - omega;
    TA xv[BS], Di[BS * BS], u[BS], G[BS * BS];
    int kq = -1;            // chunk position of the kept in-chunk lower entry
    unsigned lowmask = 0u;  // chunk positions of every in-chunk lower entry
    long long o = 0;
    int wd = 0;
#pragma unroll
    for (int q = 0; q < BS * BS; ++q) G[q] = 0;
#pragma unroll
    for (int q = 0; q < BS; ++q) u[q] = xv[q] = 0;
    if (live) {
        const long long b0 = __ldg(sp + (t >> 5)), b1 = __ldg(sp + (t >> 5) + 1);
        wd = (int)((b1 - b0) >> 5);
        o = b0 + (t & 31);
        TA acc[BS], K[kKeepSlot ? 1 : BS * BS];
        int kslot = 0;  // slot of the kept in-chunk block (kKeepSlot)
#pragma unroll
        for (int q = 0; q < BS; ++q) acc[q] = 0;
#pragma unroll
        for (int q = 0; q < (kKeepSlot ? 1 : BS * BS); ++q) K[q] = 0;
        // one off-diagonal entry in slot kk: its contribution c (A_ij c added to acc) and the in-chunk
        // bookkeeping
        auto entry = [&](unsigned cw, const TA B[BS * BS], int kk) {
            TA c[BS];
            if constexpr (BS == 2) {
                // 2x2 blocks: the three cases (later in the chunk, earlier in the chunk, outside it) as
                // selects, so the lanes of a warp do not diverge (measured 0.55 -> 0.58 of peak on C1;
                // for 3x3 blocks the branches measured faster)
                const int j = (int)(cw & kChunkColMask);
                const int dq = j - cbase;
                const bool same_earlier = (cw & kChunkSame) && dq <= p;  // the row itself never comes here
                const bool earlier_col = (cw & kChunkEarlier) != 0u;
                if (same_earlier) {
                    lowmask |= 1u << dq;
                    if (kq < 0) {
                        kq = dq;
                        kslot = kk;
                    }
                }
                // x is read-only within the launch where it is gathered: the chunks of one colour are
                // not coupled, and the row's own chunk writes only after every lane's phase 1
                TA xp[2], vp[2];
                ld_pair<TXV, TA, true>(x, j, xp);
                vp[0] = xp[0];
                vp[1] = xp[1];
                if (earlier_col) ld_pair<TXV, TA, true>(vt, j, vp);
#pragma unroll
                for (int m = 0; m < BS; ++m) {
                    const TA base = same_earlier ? (TA)0 : xp[m];  // earlier in the chunk: -(1 - omega) A vt_j now
                    const TA sub = same_earlier ? xp[m] : vp[m];
                    c[m] = plain ? base : base - omo * sub;
                }
            } else {
                const int j = (int)(cw & kChunkColMask);
                if (cw & kChunkSame) {
                    const int dq = j - cbase;
                    if (dq > p) {  // later in the chunk: its start value
#pragma unroll
                        for (int m = 0; m < BS; ++m) {
                            const TA xj = (TA)x[(long long)j * BS + m];
                            c[m] = plain ? xj : xj - omo * xj;
                        }
                    } else {  // earlier in the chunk: -(1 - omega) A vt_j now, A x_j(new) in phase 2
                        lowmask |= 1u << dq;
                        if (kq < 0) {
                            kq = dq;
                            if constexpr (!kKeepSlot) {
#pragma unroll
                                for (int q = 0; q < BS * BS; ++q) K[q] = B[q];
                            }
                        }
#pragma unroll
                        for (int m = 0; m < BS; ++m) c[m] = plain ? (TA)0 : -omo * (TA)x[(long long)j * BS + m];
                    }
                } else {
                    const bool earlier = (cw & kChunkEarlier) != 0u;
#pragma unroll
                    for (int m = 0; m < BS; ++m) {
                        const long long oj = (long long)j * BS + m;
                        const TA xj = (TA)x[oj];
                        c[m] = plain ? xj : xj - omo * (earlier ? (TA)__ldg(vt + oj) : xj);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < BS; ++q)
#pragma unroll
                for (int m = 0; m < BS; ++m) acc[q] += B[q * BS + m] * c[m];
        };
        int k = 1;
        for (; k + NB - 1 < wd; k += NB) {
            const long long p0 = o + (long long)k * 32;
            unsigned cw[NB];
            TA B[NB][BS * BS];
#pragma unroll
            for (int e = 0; e < NB; ++e) {
                cw[e] = __ldcs(col + p0 + 32 * e);
                load_block_cs<BS, TV, TA>(a, p0 + 32 * e, B[e]);
            }
#pragma unroll
            for (int e = 0; e < NB; ++e) entry(cw[e], B[e], k + e);
        }
        for (; k < wd; ++k) {
            const long long p0 = o + (long long)k * 32;
            TA B0[BS * BS];
            load_block_cs<BS, TV, TA>(a, p0, B0);
            entry(__ldcs(col + p0), B0, k);
        }
        TA rhs[BS], D[BS * BS];
#pragma unroll
        for (int q = 0; q < BS; ++q) {
            rhs[q] = (TA)__ldg(b + (long long)i * BS + q);
            xv[q] = (TA)x[(long long)i * BS + q];
        }
        load_block_cs<BS, TV, TA>(a, o, D);
        block_inverse<BS, TA>(D, Di);
        TA r2[BS];
#pragma unroll
        for (int q = 0; q < BS; ++q) r2[q] = (plain ? (TA)1 : omega) * rhs[q] - acc[q];
        block_matvec<BS, TA>(Di, r2, u);
        if (kq >= 0) {
            TA Kb[BS * BS];
            if constexpr (kKeepSlot) {
                load_block<BS, TV, TA>(a, o + (long long)kslot * 32, Kb);
            } else {
#pragma unroll
                for (int q = 0; q < BS * BS; ++q) Kb[q] = K[q];
            }
#pragma unroll
            for (int q = 0; q < BS; ++q)
#pragma unroll
                for (int m = 0; m < BS; ++m) {
                    TA g = 0;
#pragma unroll
                    for (int l = 0; l < BS; ++l) g += Di[q * BS + l] * Kb[l * BS + m];
                    G[q * BS + m] = g;
                }
        }
    }
    const TA prod = (TA)1 - w * omega;
    TA gx[BS];    // sum of G x_j(new) over the row's in-chunk lower entries
    TXV mine[BS];  // this row's new value, written after the chunk is done
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        gx[q] = 0;
        mine[q] = 0;
    }
#pragma unroll 1
    for (int r = 0; r < CH; ++r) {
        TA xn[BS];
#pragma unroll
        for (int q = 0; q < BS; ++q) xn[q] = 0;
        if (live && p == r) {
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                const TA out = u[q] - gx[q];
                mine[q] = plain ? (TXV)out : (TXV)(prod * xv[q] + w * out);
                xn[q] = (TA)mine[q];
            }
        }
        TA bx[BS];
#pragma unroll
        for (int q = 0; q < BS; ++q) bx[q] = __shfl_sync(0xffffffffu, xn[q], (lane & ~(CH - 1)) | r);
        if (live && p > r && ((lowmask >> r) & 1u)) {
            if (r == kq) {
#pragma unroll
                for (int q = 0; q < BS; ++q)
#pragma unroll
                    for (int m = 0; m < BS; ++m) gx[q] += G[q * BS + m] * bx[m];
            } else {
                for (int k = 1; k < wd; ++k) {
                    const long long pk = o + (long long)k * 32;
                    if ((int)(__ldg(col + pk) & kChunkColMask) != cbase + r) continue;
                    TA B[BS * BS], v[BS], dv[BS];
                    load_block<BS, TV, TA>(a, pk, B);
                    block_matvec<BS, TA>(B, bx, v);
                    block_matvec<BS, TA>(Di, v, dv);
#pragma unroll
                    for (int q = 0; q < BS; ++q) gx[q] += dv[q];
                }
            }
        }
    }
    // every lane of the warp has read its chunk's start values in phase 1 (before the shuffles above)
    if (live) {
#pragma unroll
        for (int q = 0; q < BS; ++q) {
            if (!plain && save) vt[(long long)i * BS + q] = (TXV)xv[q];
            x[(long long)i * BS + q] = mine[q];
        }
    }
}

// Column words of the chunk-ordered stage-2 matrix (see kChunkSame): stored row t = block row rows[t]
// of colour cls[rows[t]]; the relation of each stored neighbour to the row goes into its top bits.
__global__ void chunk_col_flags(int nstored, const int *__restrict__ rows, const long long *__restrict__ sp,
                                const int *__restrict__ ia, const int *__restrict__ cls, int chunk,
                                unsigned *__restrict__ col) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nstored) return;
    const int i = rows[t];
    if (i < 0) return;
    const long long o = sp[t >> 5] + (t & 31);
    const int len = ia[i + 1] - ia[i], ci = cls[i];
    for (int k = 0; k < len; ++k) {
        const long long p = o + (long long)k * 32;
        const int j = (int)col[p];
        unsigned f = 0u;
        if (j / chunk == i / chunk) f = kChunkSame;
        else if (cls[j] < ci) f = kChunkEarlier;
        col[p] = (unsigned)j | f;
    }
}

// ---- sliced-ELL fill ----------------------------------------------------------
template <typename TV>
__device__ __forceinline__ TV cvt_val(double v, double sc);
template <>
__device__ __forceinline__ double cvt_val<double>(double v, double) { return v; }
template <>
__device__ __forceinline__ float cvt_val<float>(double v, double) { return (float)v; }
template <>
__device__ __forceinline__ __nv_bfloat16 cvt_val<__nv_bfloat16>(double v, double sc) {
    return __float2bfloat16_rn((float)(v / sc));
}

// The power of two 2^e with max/2^e in [0.5, 1) (1 for max = 0): the block scale of BF16 storage.
__device__ __forceinline__ double pow2_scale(double m) {
    if (!(m > 0.0)) return 1.0;
    int e = 0;
    frexp(m, &e);
    return ldexp(1.0, e);
}

// max over the 32 lanes of a warp (every lane takes part)
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Stored row t receives the entries of CSR/BSR row rows[t] (E values per entry, E = 1 or bs*bs) in
// slot-major order.  A warp covers one 32-row slice, so each slot of the slice is one block of 32
// stored values; bscale != nullptr (BF16, E = 1): that block's power-of-two scale goes to
// bscale[p / 32] and the values are stored divided by it.  sorted (E = 1, no bscale): each row's
// entries after the first go to the slots in ascending column order (the first, the diagonal of a
// square operator, stays first), so that the rows of a slice gather nearby columns in each slot.
template <typename TV>
__global__ void sell_fill(int nstored, const int *__restrict__ rows, const long long *__restrict__ sp,
                          const int *__restrict__ ia, const int *__restrict__ ja, const double *__restrict__ a,
                          int E, int *__restrict__ col, TV *__restrict__ val, float *__restrict__ bscale, int sorted) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ((nstored + 31) & ~31)) return;  // whole slices: every lane of a slice's warp stays
    const bool in = t < nstored;
    const int i = in ? rows[t] : -1;
    const long long b0 = sp[t >> 5], b1 = sp[(t >> 5) + 1];
    const int w = (int)((b1 - b0) >> 5);
    const long long o = b0 + (t & 31);
    const int d = i >= 0 ? ia[i] : 0;
    const int len = i >= 0 ? ia[i + 1] - d : 0;
    for (int k = 0; k < w; ++k) {
        const long long p = o + (long long)k * 32;
        double sc = 1.0;
        if (bscale) {  // warp-uniform
            sc = pow2_scale(warp_max(k < len ? fabs(a[(long long)(d + k) * E]) : 0.0));
            if ((t & 31) == 0) bscale[p >> 5] = (float)sc;
        }
        if (!in) continue;
        if (k < len && sorted) {
            // entry k goes to slot 1 + (entries 1.. before it in column order, ties by position)
            const int jk = ja[d + k];
            int pos = 0;
            if (k > 0) {
                pos = 1;
                for (int e = 1; e < len; ++e) pos += ja[d + e] < jk || (ja[d + e] == jk && e < k);
            }
            const long long pp = o + (long long)pos * 32;
            col[pp] = jk;
            val[pp] = cvt_val<TV>(a[d + k], sc);
        } else if (k < len) {
            col[p] = ja[d + k];
            for (int q = 0; q < E; ++q) val[p * E + q] = cvt_val<TV>(a[(long long)(d + k) * E + q], sc);
        } else {
            col[p] = 0;
            for (int q = 0; q < E; ++q) val[p * E + q] = cvt_val<TV>(0.0, 1.0);
        }
    }
}

// The sliced ELL with P lanes per stored row (SellFmt<TV, P>, P > 1; FP32 / FP64 values, no block
// scales): thread u is virtual row u (stored row u / P, lane u % P); the entry at (sorted) position
// q of the row goes to lane q % P, slot q / P.  Unfilled slots are padding (value 0, column 0).
template <typename TV>
__global__ void sell_fill_lanes(int nstored, int P, const int *__restrict__ rows, const long long *__restrict__ sp,
                                const int *__restrict__ ia, const int *__restrict__ ja, const double *__restrict__ a,
                                int *__restrict__ col, TV *__restrict__ val, int sorted) {
    const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (long long)nstored * P) return;
    const int t = (int)(u / P), h = (int)(u % P);
    const int i = rows[t];
    const long long b0 = sp[u >> 5], b1 = sp[(u >> 5) + 1];
    const int w = (int)((b1 - b0) >> 5);
    const long long o = b0 + (u & 31);
    const int d = i >= 0 ? ia[i] : 0, len = i >= 0 ? ia[i + 1] - d : 0;
    for (int k = 0; k < w; ++k)
        if (h + (long long)P * k >= len) {
            col[o + (long long)k * 32] = 0;
            val[o + (long long)k * 32] = cvt_val<TV>(0.0, 1.0);
        }
    for (int e = 0; e < len; ++e) {
        int q = e;
        if (sorted && e > 0) {
            const int je = ja[d + e];
            q = 1;
            for (int f = 1; f < len; ++f) q += ja[d + f] < je || (ja[d + f] == je && f < e);
        }
        if (q % P != h) continue;
        const long long pp = o + (long long)(q / P) * 32;
        col[pp] = ja[d + e];
        val[pp] = cvt_val<TV>(a[d + e], 1.0);
    }
}

// The CSR counterpart of sell_fill's `sorted`: each row's entries after the first in ascending column
// order (the first, the diagonal of a square operator, stays first), by an insertion sort of one
// thread per row.
template <typename TV>
__global__ void sort_row_entries(int n, const int *__restrict__ ia, int *__restrict__ ja, TV *__restrict__ a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = ia[i] + 1, e = ia[i + 1];
    for (int k = b + 1; k < e; ++k) {
        const int jk = ja[k];
        const TV ak = a[k];
        int q = k - 1;
        while (q >= b && ja[q] > jk) {
            ja[q + 1] = ja[q];
            a[q + 1] = a[q];
            --q;
        }
        ja[q + 1] = jk;
        a[q + 1] = ak;
    }
}

// ---- setup helpers ----------------------------------------------------------
__global__ void to_f32(long long n, const double *__restrict__ in, float *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

// BF16 values of a CSR operator, one power-of-two FP32 scale per 32 consecutive stored values (a warp
// per block).
__global__ void to_bf16_blocks(long long nnz, const double *__restrict__ a, float *__restrict__ bscale,
                               __nv_bfloat16 *__restrict__ out) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if ((k & ~31LL) >= nnz) return;  // whole warps
    const double v = k < nnz ? a[k] : 0.0;
    const double sc = pow2_scale(warp_max(fabs(v)));
    if ((k & 31) == 0) bscale[k >> 5] = (float)sc;
    if (k < nnz) out[k] = __float2bfloat16_rn((float)(v / sc));
}

// 1 / a_ii where the diagonal is the first stored entry, else 0 (row skipped).
template <typename TX>
__global__ void dinv_diag(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                          const double *__restrict__ a, TX *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = ia[i];
    const bool has = d < ia[i + 1] && ja[d] == i && a[d] != 0.0;
    out[i] = has ? (TX)(1.0 / a[d]) : (TX)0;
}

template <typename TX>
__global__ void dinv_l1(int n, const int *__restrict__ ia, const double *__restrict__ a, TX *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = ia[i]; k < ia[i + 1]; ++k) s += fabs(a[k]);
    out[i] = s > 0.0 ? (TX)(1.0 / s) : (TX)0;
}

// y = D^-1 A x in FP64 (power iteration); dinv from dinv_diag<double>.
__global__ void dinv_a_x(int n, const int *__restrict__ ia, const int *__restrict__ ja, const double *__restrict__ a,
                         const double *__restrict__ dinv, const double *__restrict__ x, double *__restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = ia[i]; k < ia[i + 1]; ++k) s += a[k] * x[ja[k]];
    y[i] = dinv[i] * s;
}

template <typename TA, typename TB>
__global__ void convert(long long n, const TA *__restrict__ in, TB *__restrict__ out) {
    grid_dep_wait();
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (TB)in[i];
}

}  // namespace fk
}  // namespace jxcpr
