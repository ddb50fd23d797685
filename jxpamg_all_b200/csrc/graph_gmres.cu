// Restarted flexible GMRES(k) with the whole solve on the device, recorded as
// one CUDA graph with conditional WHILE nodes:
//
//   ||b||  ->  WHILE (not done) {                       restart cycle
//                 r = b - A x, ||r||, convergence test, v_0 = r / ||r||
//                 WHILE (cycle continues) {              Arnoldi step i
//                    z_i = M^-1 v_i  (CPR kernels recorded in place)
//                    w = A z_i
//                    h1 = V^T w                          two-pass classical
//                    w -= V h1, h2 = V^T w, s = ||w||^2  Gram-Schmidt (CGS2)
//                    Givens rotation of column i (one thread), test
//                    v_{i+1} = (w - V h2) / sqrt(s - ||h2||^2)
//                 }
//                 x += Z y  (y from the triangular solve at the cycle end)
//              }
//
// The host sees no per-iteration round trip: the Hessenberg matrix, rotations,
// residual estimates and the loop conditions live in device memory.  The
// scalar recurrence (rotations, estimate, convergence and restart rules,
// back substitution) follows the host GMRES (jxfpamg-0220/csrc/krylov/
// pgmres.c:1090-1560) step for step; two things differ by design: each cycle
// restarts from the true residual b - A x instead of the rotated estimate,
// and the orthogonalisation is CGS2 (three passes over the basis -- the first
// products, the first update fused with the second products, the final
// update -- and a fixed number of kernels per step, which a graph needs)
// instead of MGS (i + 1 passes).  The norm of the new vector comes from Pythagoras,
// ||w - V h2||^2 = ||w||^2 - ||h2||^2, as in delayed CGS2 (Swirydowicz et al.,
// 2020).  Flexible: the preconditioned directions z_i are kept and x += Z y.
// Each pass writes per-block partial sums, which one block per row adds up
// (reduce_rows_kernel, reduce_rows2_kernel) before the one-thread Arnoldi
// kernel; the kernels of a step are launched as programmatic dependents.
// Options: the basis and the z_i stored in FP32 (krylov_fp32; every product,
// norm and update still in FP64), and the second pass taken only where the
// first cancelled more than half of ||w||^2 (selective_reorth, the Daniel-
// Gragg-Kaufman-Stewart test): a step without it reads the basis twice.
#include <cmath>
#include <stdexcept>

#include "solver.cuh"

namespace jxcpr {
namespace gg {

constexpr int kThreads = 256;
constexpr int kRedThreads = 1024;
constexpr int kSlice = 2048;  // elements per block of the Gram products
constexpr int kSlice2 = 1024;  // elements per block of the fused update + second Gram products

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// sum over the block; the result is valid in thread 0
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ __forceinline__ double sum_row(const double *row, int G, double *sh) {
    double v = 0.0;
    for (int j = threadIdx.x; j < G; j += blockDim.x) v += row[j];
    return block_sum(v, sh);
}

// partials[blockIdx.x] = sum of x^2 over the block's elements
__global__ void __launch_bounds__(kThreads) sq_partials(long long n, const double *__restrict__ x,
                                                        double *__restrict__ partials) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads)
        acc = fma(x[e], x[e], acc);
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kRedThreads) init_kernel(GgState *st, const double *__restrict__ partials, int G) {
    __shared__ double sh[32];
    const double v = sum_row(partials, G, sh);
    if (threadIdx.x == 0) {
        GgState s{};
        s.b_norm = sqrt(v);
        s.first = 1;
        s.t_start = global_ns();
        *st = s;
    }
}

// Start of a restart cycle: ||r|| of r = b - A x, the convergence and stop
// rules, and the first basis vector's scale.  Sets both loop conditions.
__global__ void __launch_bounds__(kRedThreads) restart_kernel(GgState *st, const double *__restrict__ partials, int G,
                                                              GgParams P, GgWork W, double *__restrict__ norms,
                                                              cudaGraphConditionalHandle h_out,
                                                              cudaGraphConditionalHandle h_in) {
    __shared__ double sh[32];
    const double rn2 = sum_row(partials, G, sh);
    if (threadIdx.x != 0) return;
    GgState &s = *st;
    const double rn = sqrt(rn2);
    bool done = false;
    s.cycles += 1;
    if (s.first) {
        s.first = 0;
        if (s.b_norm != 0.0 && !(s.b_norm / s.b_norm == s.b_norm / s.b_norm)) {
            s.status = 1;  // NaN/Inf in b
            done = true;
        } else if (rn != 0.0 && !(rn / rn == rn / rn)) {
            s.status = 1;  // NaN/Inf in A or x0
            done = true;
        }
        s.r_norm0 = rn;
        s.epsilon = fmax(P.a_tol, P.tol * (s.b_norm > 0.0 ? s.b_norm : rn));
        s.normdown = rn;
        norms[0] = rn;
    }
    // stall rule: a full cycle whose true residual ratio (end / start) stayed above P.stall
    const int ci = s.iter - s.iter0;
    const bool stalled = P.stall > 0.0 && s.cycles > 1 && ci >= P.k && rn > s.r_cycle * P.stall;
    s.r_cycle = rn;
    s.r_norm = rn;
    s.iter0 = s.iter;
    if (!done) {
        if (rn == 0.0 || (rn <= s.epsilon && s.iter >= P.min_iter)) {
            s.converged = 1;
            done = true;
        } else if (s.est_conv && !P.check_restarted) {
            done = true;  // estimate below tolerance, true residual not, no restart allowed
        } else if (s.conv_fail || s.iter >= P.max_iter || s.cycles > P.max_iter + 1) {
            done = true;
        } else if (stalled) {
            s.stalled = 1;
            done = true;
        }
    }
    s.est_conv = 0;
    s.conv_fail = 0;
    s.i = 0;
    s.m = 0;
    if (done) {
        s.done = 1;
        s.cont = 0;
        s.rel = s.b_norm > 0.0 ? rn / s.b_norm : (s.r_norm0 > 0.0 ? rn / s.r_norm0 : 0.0);
        s.t_end = global_ns();
        cudaGraphSetConditional(h_in, 0);
        cudaGraphSetConditional(h_out, 0);
    } else {
        W.rs[0] = rn;
        s.scale = 1.0 / rn;
        s.cont = 1;
        cudaGraphSetConditional(h_in, 1);
    }
}

// v_0 = r * scale (skipped once the solve is done).  TB: the basis' storage type (double, or float
// with every product, norm and update still formed in FP64)
template <typename TB>
__global__ void __launch_bounds__(kThreads) scale0_kernel(long long n, const double *__restrict__ r,
                                                          TB *const *__restrict__ V, const GgState *st) {
    if (st->done) return;
    const double sc = st->scale;
    TB *v0 = V[0];
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads)
        v0[e] = (TB)(r[e] * sc);
}

// dst = V[i] (the preconditioner's input buffer)
template <typename TB>
__global__ void __launch_bounds__(kThreads) gather_kernel(long long n, const TB *const *__restrict__ V,
                                                          const GgState *st, double *__restrict__ dst) {
    grid_dep_wait();
    const TB *src = V[st->i];
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads)
        dst[e] = (double)src[e];
}

// Z[i] = src (the preconditioner's output, kept for the flexible update).  With an FP32 basis and
// round_src set, src is replaced by its FP32 rounding too, so that the product A z_i that follows and
// the update x += Z y use the same direction (a preconditioner with FP32 output needs no rounding).
template <typename TB>
__global__ void __launch_bounds__(kThreads) scatter_kernel(long long n, double *__restrict__ src,
                                                           TB *const *__restrict__ Z, const GgState *st, int round_src) {
    grid_dep_wait();
    TB *dst = Z[st->i];
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < n; e += (long long)gridDim.x * kThreads) {
        const TB v = (TB)src[e];
        dst[e] = v;
        if (round_src) src[e] = (double)v;
    }
}

// Four consecutive entries (a quad) of a basis vector, of w or of x as FP64 values; every vector
// starts on a 32-byte boundary, so a quad at an index divisible by 4 is one float4 or two double2.
__device__ __forceinline__ void ld4(const double *p, double v[4]) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}
__device__ __forceinline__ void ld4(const float *p, double v[4]) {
    const float4 a = *reinterpret_cast<const float4 *>(p);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
}
__device__ __forceinline__ void st4(double *p, const double v[4]) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4(float *p, const double v[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
// Quad q of a vector of n entries; the entries past n of the last, partial quad read as 0.
template <typename T>
__device__ __forceinline__ void ld4n(const T *p, long long q, long long n, double v[4]) {
    if (4 * q + 3 < n) {
        ld4(p + 4 * q, v);
    } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) v[r] = 4 * q + r < n ? (double)p[4 * q + r] : 0.0;
    }
}
template <typename T>
__device__ __forceinline__ void st4n(T *p, long long q, long long n, const double v[4]) {
    if (4 * q + 3 < n) {
        st4(p + 4 * q, v);
    } else {
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (4 * q + r < n) p[4 * q + r] = (T)v[r];
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sum of row[0..G) over one warp (the result in every lane)
__device__ __forceinline__ double warp_row_sum(const double *__restrict__ row, int G, int lane) {
    double v = 0.0;
    for (int j = lane; j < G; j += 32) v += row[j];
    return warp_sum(v);
}

// Block x: partial <V[k], w> over the x-th slice of kSlice elements for every k <= i.  Each thread
// keeps its two quads of w in registers and streams the same quads of every basis vector past them,
// two vectors at a time (eight loads in flight); warps reduce with shuffles and combine through shared
// memory once at the end.
template <typename TB>
__global__ void __launch_bounds__(kThreads) dots_kernel(long long n, const TB *const *__restrict__ V,
                                                        const GgState *st, const double *__restrict__ w,
                                                        double *__restrict__ partials) {
    static_assert(kSlice == kThreads * 8, "two quads per thread");
    __shared__ double part[kGgMaxK + 2][kThreads / 32];
    grid_dep_wait();
    const long long q0 = (long long)blockIdx.x * (kSlice / 4) + threadIdx.x, q1 = q0 + kThreads;
    double w0[4], w1[4];
    ld4n(w, q0, n, w0);
    ld4n(w, q1, n, w1);
    const int m = st->i + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int k = 0;
    for (; k + 1 < m; k += 2) {
        double a0[4], a1[4], b0[4], b1[4];
        ld4n(V[k], q0, n, a0);
        ld4n(V[k], q1, n, a1);
        ld4n(V[k + 1], q0, n, b0);
        ld4n(V[k + 1], q1, n, b1);
        double sa = 0.0, sb = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            sa = fma(a0[r], w0[r], sa);
            sb = fma(b0[r], w0[r], sb);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            sa = fma(a1[r], w1[r], sa);
            sb = fma(b1[r], w1[r], sb);
        }
        sa = warp_sum(sa);
        sb = warp_sum(sb);
        if (lane == 0) {
            part[k][warp] = sa;
            part[k + 1][warp] = sb;
        }
    }
    if (k < m) {
        double a0[4], a1[4];
        ld4n(V[k], q0, n, a0);
        ld4n(V[k], q1, n, a1);
        double sa = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) sa = fma(a0[r], w0[r], sa);
#pragma unroll
        for (int r = 0; r < 4; ++r) sa = fma(a1[r], w1[r], sa);
        sa = warp_sum(sa);
        if (lane == 0) part[k][warp] = sa;
    }
    {  // row m: <w, w> (the selective second pass compares it with the first pass' projection)
        double sw = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) sw = fma(w0[r], w0[r], sw);
#pragma unroll
        for (int r = 0; r < 4; ++r) sw = fma(w1[r], w1[r], sw);
        sw = warp_sum(sw);
        if (lane == 0) part[m][warp] = sw;
    }
    __syncthreads();
    if (threadIdx.x <= m) {
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < kThreads / 32; ++q) v += part[threadIdx.x][q];
        partials[(long long)threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
}

// h1[k] = sum of partials row k, k <= i (one warp per row), and ||w||^2 (row i + 1).  With the
// selective second pass (P.selective) the step skips it when the first pass kept more than half of
// ||w||^2, i.e. ||w - V h1||^2 = ||w||^2 - ||h1||^2 > ||w||^2 / 2 (the Daniel-Gragg-Kaufman-Stewart
// criterion with eta = 1/sqrt(2)): then h2 = h1, h1 = 0 and sig = ||w||^2, so that the Arnoldi and
// final kernels (which use h1 + h2, sig - ||h2||^2 and w - V h2) finish the step from the first pass.
__global__ void __launch_bounds__(kRedThreads) reduce_h_kernel(const double *__restrict__ partials, int G,
                                                               GgState *st, GgParams P, GgWork W) {
    __shared__ double ww;
    grid_dep_wait();
    const int m = st->i + 1, lane = threadIdx.x & 31;
    for (int k = threadIdx.x >> 5; k <= m; k += kRedThreads / 32) {
        const double v = warp_row_sum(partials + (long long)k * G, G, lane);
        if (lane == 0) {
            if (k < m) W.h1[k] = v;
            else ww = v;
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    int skip = 0;
    if (P.selective) {
        double ss = 0.0;
        for (int k = 0; k < m; ++k) ss += W.h1[k] * W.h1[k];
        const double e2 = ww - ss;
        skip = e2 > 0.5 * ww ? 1 : 0;
        if (skip) {
            for (int k = 0; k < m; ++k) {
                W.h2[k] = W.h1[k];
                W.h1[k] = 0.0;
            }
            st->sig = ww;
        }
    }
    st->skip = skip;
}

// h1[k] = sum of partials row k (k <= i), one block per row: the rows are summed side by side
// (without the selective second pass, which reduce_h_kernel decides on from all of them).
__global__ void __launch_bounds__(kThreads) reduce_rows_kernel(const double *__restrict__ partials, int G,
                                                              GgState *st, GgWork W) {
    __shared__ double sh[32];
    grid_dep_wait();
    const int m = st->i + 1, k = blockIdx.x;
    if (k > m) return;
    double v = 0.0;
    for (int j = threadIdx.x; j < G; j += kThreads) v += partials[(long long)k * G + j];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        if (k < m) W.h1[k] = v;
        if (k == 0) st->skip = 0;
    }
}

// The first update and the second Gram products in one pass over the basis:
// w -= sum_{k <= i} h[k] V[k], then partial <V[k], w> (k <= i) and <w, w> of
// the updated w over the block's slice of kSlice2 elements (one quad per thread).
// The update reads the quad of every V[k], two vectors at a time, and the
// products read it again right after, from L1 / L2, so the basis crosses HBM
// once (separate update and product kernels would read it twice); the products
// of two vectors are reduced over the warp together.
template <typename TB>
__global__ void __launch_bounds__(kThreads) update_dots_kernel(long long n, const TB *const *__restrict__ V,
                                                               const GgState *st, const double *__restrict__ h,
                                                               double *__restrict__ w, double *__restrict__ partials) {
    static_assert(kSlice2 == kThreads * 4, "one quad per thread");
    __shared__ const TB *vs[kGgMaxK + 2];
    __shared__ double hs[kGgMaxK + 2];
    __shared__ double part[kGgMaxK + 2][kThreads / 32];
    grid_dep_wait();
    if (st->skip) return;  // the selective rule kept the first pass
    const int m = st->i + 1;
    for (int k = threadIdx.x; k < m; k += kThreads) {
        vs[k] = V[k];
        hs[k] = h[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long q = (long long)blockIdx.x * (kSlice2 / 4) + threadIdx.x;
    const bool live = 4 * q < n;
    double sv[4] = {0.0, 0.0, 0.0, 0.0};
    if (live) {
        ld4n(w, q, n, sv);
        int k = 0;
        for (; k + 1 < m; k += 2) {
            double a[4], b[4];
            ld4n(vs[k], q, n, a);
            ld4n(vs[k + 1], q, n, b);
#pragma unroll
            for (int r = 0; r < 4; ++r) sv[r] = fma(-hs[k], a[r], sv[r]);
#pragma unroll
            for (int r = 0; r < 4; ++r) sv[r] = fma(-hs[k + 1], b[r], sv[r]);
        }
        if (k < m) {
            double a[4];
            ld4n(vs[k], q, n, a);
#pragma unroll
            for (int r = 0; r < 4; ++r) sv[r] = fma(-hs[k], a[r], sv[r]);
        }
        st4n(w, q, n, sv);
    }
    for (int k = 0; k <= m; k += 2) {  // uniform trip count: every lane takes part in the shuffles
        double v0 = 0.0, v1 = 0.0;
        if (live) {
            double a[4], b[4];
            if (k < m)
                ld4n(vs[k], q, n, a);
            else
#pragma unroll
                for (int r = 0; r < 4; ++r) a[r] = sv[r];
            if (k + 1 < m)
                ld4n(vs[k + 1], q, n, b);
            else
#pragma unroll
                for (int r = 0; r < 4; ++r) b[r] = k + 1 == m ? sv[r] : 0.0;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                v0 = fma(a[r], sv[r], v0);
                v1 = fma(b[r], sv[r], v1);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0 += __shfl_xor_sync(0xffffffffu, v0, o);
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        }
        if (lane == 0) {
            part[k][warp] = v0;
            if (k + 1 <= m) part[k + 1][warp] = v1;
        }
    }
    __syncthreads();
    if (threadIdx.x <= m) {
        double v = 0.0;
#pragma unroll
        for (int qq = 0; qq < kThreads / 32; ++qq) v += part[threadIdx.x][qq];
        partials[(long long)threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
}

// The second-pass coefficients h2[k] (k <= i) and ||w||^2 (into st->sig) from the fused update's
// partials, one block per row; nothing when the selective rule kept the first pass (reduce_h_kernel
// set them then).
__global__ void __launch_bounds__(kThreads) reduce_rows2_kernel(const double *__restrict__ partials, int G,
                                                               GgState *st, GgWork W) {
    __shared__ double sh[32];
    grid_dep_wait();
    if (st->skip) return;
    const int m = st->i + 1, k = blockIdx.x;
    if (k > m) return;
    double v = 0.0;
    for (int j = threadIdx.x; j < G; j += kThreads) v += partials[(long long)k * G + j];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) {
        if (k < m) W.h2[k] = v;
        else st->sig = v;
    }
}

// One thread: the Hessenberg column of this step, its Givens rotation, the
// residual estimate, the cycle-end rules and, at a cycle end, y = H^-1 rs.
__global__ void arnoldi_kernel(GgState *st, GgParams P, GgWork W, double *__restrict__ norms,
                               cudaGraphConditionalHandle h_in) {
    grid_dep_wait();
    if (threadIdx.x != 0) return;
    const int i0 = st->i, m = i0 + 1;
    const double sig = st->sig;  // ||w||^2 after the step's last Gram-Schmidt pass
    GgState &s = *st;
    const int K = P.k;
    double *hh = W.hh, *rs = W.rs, *c = W.c, *sn = W.sn;
#define HH(r, q) hh[(long long)(r) * K + (q)]
    double ss = 0.0;
    for (int j = 0; j < m; ++j) {
        HH(j, i0) = W.h1[j] + W.h2[j];
        ss += W.h2[j] * W.h2[j];
    }
    const double t2 = sig - ss;
    double t = t2 > 0.0 ? sqrt(t2) : 0.0;
    HH(m, i0) = t;
    s.scale = t != 0.0 ? 1.0 / t : 0.0;
    const int i = m;  // steps in this cycle, 1-based as in the reference loop
    for (int j = 1; j < i; ++j) {
        t = HH(j - 1, i - 1);
        HH(j - 1, i - 1) = sn[j - 1] * HH(j, i - 1) + c[j - 1] * t;
        HH(j, i - 1) = -sn[j - 1] * t + c[j - 1] * HH(j, i - 1);
    }
    t = HH(i, i - 1) * HH(i, i - 1);
    t += HH(i - 1, i - 1) * HH(i - 1, i - 1);
    double gamma = sqrt(t);
    if (gamma == 0.0) gamma = 1.e-16;
    c[i - 1] = HH(i - 1, i - 1) / gamma;
    sn[i - 1] = HH(i, i - 1) / gamma;
    rs[i] = -HH(i, i - 1) * rs[i - 1];
    rs[i] /= gamma;
    rs[i - 1] = c[i - 1] * rs[i - 1];
    HH(i - 1, i - 1) = sn[i - 1] * HH(i, i - 1) + c[i - 1] * HH(i - 1, i - 1);
    const double r_norm = fabs(rs[i]);
    const double conv = r_norm / s.normdown;
    s.normdown = r_norm;
    s.iter += 1;
    norms[s.iter] = r_norm;
    s.r_norm = r_norm;
    s.i = i;
    s.m = m;
    bool end = i >= K || s.iter >= P.max_iter;
    if (s.iter > 1 && conv > P.convfac) {
        s.conv_fail = 1;
        end = true;
    }
    if (r_norm <= s.epsilon && s.iter >= P.min_iter) {
        s.est_conv = 1;
        end = true;
    }
    if (end) {
        rs[i - 1] = rs[i - 1] / HH(i - 1, i - 1);
        for (int k = i - 2; k >= 0; --k) {
            double a = 0.0;
            for (int j = k + 1; j < i; ++j) a -= HH(k, j) * rs[j];
            a += rs[k];
            rs[k] = a / HH(k, k);
        }
        for (int j = 0; j < i; ++j) W.y[j] = rs[j];
    }
#undef HH
    s.cont = end ? 0 : 1;
    cudaGraphSetConditional(h_in, end ? 0u : 1u);
}

// v_{m} = (w - sum_{k < m} h2[k] V[k]) * scale, skipped at a cycle end; a quad per thread and trip,
// two basis vectors per step of the sum
template <typename TB>
__global__ void __launch_bounds__(kThreads) final_kernel(long long n, TB *const *__restrict__ V,
                                                         const GgState *st, const double *__restrict__ h,
                                                         const double *__restrict__ w) {
    __shared__ const TB *vs[kGgMaxK + 2];
    __shared__ double hs[kGgMaxK + 2];
    grid_dep_wait();
    if (!st->cont) return;
    const int m = st->m;
    const double sc = st->scale;
    TB *dst = V[m];
    for (int k = threadIdx.x; k < m; k += kThreads) {
        vs[k] = V[k];
        hs[k] = h[k];
    }
    __syncthreads();
    const long long nq = (n + 3) / 4;
    for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < nq; q += (long long)gridDim.x * kThreads) {
        double s[4];
        ld4n(w, q, n, s);
        int k = 0;
        for (; k + 1 < m; k += 2) {
            double a[4], b[4];
            ld4n(vs[k], q, n, a);
            ld4n(vs[k + 1], q, n, b);
#pragma unroll
            for (int r = 0; r < 4; ++r) s[r] = fma(-hs[k], a[r], s[r]);
#pragma unroll
            for (int r = 0; r < 4; ++r) s[r] = fma(-hs[k + 1], b[r], s[r]);
        }
        if (k < m) {
            double a[4];
            ld4n(vs[k], q, n, a);
#pragma unroll
            for (int r = 0; r < 4; ++r) s[r] = fma(-hs[k], a[r], s[r]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) s[r] *= sc;
        st4n(dst, q, n, s);
    }
}

// x += sum_{j < i} y[j] Z[j] (latest direction first, as the host update); a quad per thread and trip,
// four directions per step of the sum
template <typename TB>
__global__ void __launch_bounds__(kThreads) update_x_kernel(long long n, TB *const *__restrict__ Z,
                                                            const GgState *st, const double *__restrict__ y,
                                                            double *__restrict__ x) {
    __shared__ const TB *zs[kGgMaxK];
    __shared__ double ys[kGgMaxK];
    const int i = st->i;
    if (i == 0) return;
    for (int k = threadIdx.x; k < i; k += kThreads) {
        zs[k] = Z[k];
        ys[k] = y[k];
    }
    __syncthreads();
    const long long nq = (n + 3) / 4;
    for (long long q = (long long)blockIdx.x * kThreads + threadIdx.x; q < nq; q += (long long)gridDim.x * kThreads) {
        double xe[4];
        ld4n(x, q, n, xe);
        int j = i - 1;
        for (; j >= 3; j -= 4) {
            double a[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u) ld4n(zs[j - u], q, n, a[u]);
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int r = 0; r < 4; ++r) xe[r] = fma(ys[j - u], a[u][r], xe[r]);
        }
        for (; j >= 0; --j) {
            double a[4];
            ld4n(zs[j], q, n, a);
#pragma unroll
            for (int r = 0; r < 4; ++r) xe[r] = fma(ys[j], a[r], xe[r]);
        }
        st4n(x, q, n, xe);
    }
}

__global__ void summary_kernel(const GgState *st, const int *kerr, const int *aerr, const int *berr, double *out) {
    const GgState &s = *st;
    out[0] = s.iter;
    out[1] = s.converged ? 1.0 : (s.stalled ? -1.0 : 0.0);
    out[2] = s.rel;
    out[3] = s.status;
    out[4] = (double)s.t_start;
    out[5] = (double)s.t_end;
    out[6] = s.cycles;
    out[7] = (kerr ? *kerr : 0) + (aerr ? *aerr : 0) + (berr ? *berr : 0);
}

// Adds a WHILE node after the nodes captured so far on s and continues the
// capture after it; returns its body graph.
cudaGraph_t add_while(cudaStream_t s, cudaGraphConditionalHandle h) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    JX_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) {
        set_error("graph gmres: stream is not capturing");
        throw CudaError{cudaErrorStreamCaptureInvalidated, "capture"};
    }
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    JX_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    JX_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return body;
}

cudaGraph_t capture_graph(cudaStream_t s) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    JX_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
    if (cs != cudaStreamCaptureStatusActive) {
        set_error("graph gmres: stream is not capturing");
        throw CudaError{cudaErrorStreamCaptureInvalidated, "capture"};
    }
    return g;
}

void end_capture_quietly(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (!s || cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs == cudaStreamCaptureStatusNone) return;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
}

}  // namespace gg

GraphGmres::~GraphGmres() {
    reset_graph();
    for (auto &a : aux)
        if (a) cudaStreamDestroy(a);
}

void GraphGmres::reset_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
}

void GraphGmres::prepare(Solver &S) {
    const SolverParams &prm = S.prm;
    if (prm.k_dim < 1 || prm.k_dim > kGgMaxK) {
        set_error("graph gmres: k_dim must be in 1..%d", kGgMaxK);
        throw std::invalid_argument("k_dim");
    }
    if (!S.cpr.fast || prm.stage1_solver_type != 1 || S.ext_precond) {
        set_error("graph gmres needs the fast CPR preconditioner (smoother_order 1, stage1_solver_type 1)");
        throw std::invalid_argument("graph gmres");
    }
    n = (long long)S.A.nb * S.A.bs;
    k = prm.k_dim;
    max_iter = prm.max_iter;
    const long long nn = n > 0 ? n : 1;
    G = div_up(nn, gg::kSlice);  // blocks of the Gram products and norms: one slice each
    G2 = div_up(nn, gg::kSlice2);  // blocks of the fused update + second products
    G1 = std::max(1, std::min(8 * sm_count(), div_up(nn, gg::kThreads)));
    Gq = std::max(1, div_up(div_up(nn, 4), gg::kThreads));  // one quad per thread
    state.alloc(1);
    // work: rs (k+1), c (k), sn (k), h1 (k+2), h2 (k+2), y (k), hh ((k+1) k)
    const size_t wsz = (size_t)(k + 1) + 2 * k + 2 * (k + 2) + k + (size_t)(k + 1) * k;
    work.alloc(wsz);
    double *wp = work.get();
    W.rs = wp;
    W.c = W.rs + (k + 1);
    W.sn = W.c + k;
    W.h1 = W.sn + k;
    W.h2 = W.h1 + (k + 2);
    W.y = W.h2 + (k + 2);
    W.hh = W.y + k;
    partials.alloc((size_t)(k + 2) * std::max(G, G2));
    norms.alloc((size_t)max_iter + 2);
    summary.alloc(8);
    cin.alloc(nn);
    cout.alloc(nn);
    // basis: the host GMRES's vectors are reused (same sizes); flexible directions as well if present
    Gmres &g = S.gmres;
    if ((int)g.p.size() < k + 1) {
        set_error("graph gmres: basis not allocated");
        throw CudaError{cudaErrorInvalidValue, "basis"};
    }
    std::vector<double *> vp, zp;
    for (int j = 0; j <= k; ++j) vp.push_back(g.p[j].get());
    own_z.clear();
    fp32 = prm.krylov_fp32 != 0 ? 1 : 0;
    basis32.release();
    if (fp32) {
        // FP32 basis: v_0..v_k then z_0..z_{k-1}, one allocation; each vector starts on a 256-byte
        // boundary (the kernels move four entries per access)
        const size_t stride = ((size_t)nn + 63) / 64 * 64;
        basis32.alloc((size_t)(2 * k + 1) * stride);
        std::vector<float *> v32, z32;
        for (int j = 0; j <= k; ++j) v32.push_back(basis32.get() + (size_t)j * stride);
        for (int j = 0; j < k; ++j) z32.push_back(basis32.get() + (size_t)(k + 1 + j) * stride);
        vptr32.alloc(v32.size());
        vptr32.upload(v32.data(), v32.size(), S.stream);
        zptr32.alloc(z32.size());
        zptr32.upload(z32.data(), z32.size(), S.stream);
    } else if ((int)g.zf.size() >= k) {
        for (int j = 0; j < k; ++j) zp.push_back(g.zf[j].get());
    } else {
        for (int j = 0; j < k; ++j) {
            own_z.emplace_back((size_t)nn);
            zp.push_back(own_z.back().get());
        }
    }
    cudaStream_t s = S.stream;
    vptr.alloc(vp.size());
    vptr.upload(vp.data(), vp.size(), s);
    zptr.alloc(zp.size());
    zptr.upload(zp.data(), zp.size(), s);
    for (auto &a : aux)
        if (!a) JX_CUDA(cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking));
    P.k = k;
    P.max_iter = prm.max_iter;
    P.min_iter = prm.min_iter;
    P.check_restarted = prm.is_check_restarted;
    P.tol = prm.tol;
    P.a_tol = prm.a_tol;
    P.convfac = prm.convfac_threshold;
    P.stall = prm.stall_ratio;
    P.selective = prm.selective_reorth != 0 ? 1 : 0;
    JX_CUDA(cudaStreamSynchronize(s));
    reset_graph();
}

bool GraphGmres::matches(const SolverParams &prm) const {
    return prm.k_dim == P.k && prm.max_iter == P.max_iter && prm.min_iter == P.min_iter &&
           prm.is_check_restarted == P.check_restarted && prm.tol == P.tol && prm.a_tol == P.a_tol &&
           prm.convfac_threshold == P.convfac && prm.stall_ratio == P.stall && (prm.krylov_fp32 != 0) == (fp32 != 0) &&
           (prm.selective_reorth != 0) == (P.selective != 0);
}

void GraphGmres::record(Solver &S, cudaStream_t s, double *out) {
    using namespace gg;
    const long long nn = n;
    const BsrView<double> A = S.A.view();
    const bool staged = S.prm.use_tma_spmv != 0;
    int *kerr = S.kerr.get();
    double *b = S.b.get(), *x = S.x.get(), *r = S.gmres.r.get(), *w = S.gmres.w.get();
    double *const *V = vptr.get();
    double *const *Z = zptr.get();
    float *const *V32 = vptr32.get();
    float *const *Z32 = zptr32.get();
    const bool f32 = fp32 != 0;
    GgState *st = state.get();
    double *pt = partials.get();
    const unsigned long long c0 = launch_count();
    unsigned long long c1 = c0, c2 = c0, c3 = c0, c4 = c0;
    try {
        if (S.prm.decouple)
            bsr_decouple_rhs(S.A.nb, S.A.bs, S.prm.decouple, S.dcoef.get(), b, S.prm.consistent_rhs, s);
        sq_partials<<<G, kThreads, 0, s>>>(nn, b, pt);
        JX_LAUNCH_CHECK();
        init_kernel<<<1, kRedThreads, 0, s>>>(st, pt, G);
        JX_LAUNCH_CHECK();
        cudaGraphConditionalHandle h_out = 0, h_in = 0;
        JX_CUDA(cudaGraphConditionalHandleCreate(&h_out, capture_graph(s), 1, cudaGraphCondAssignDefault));
        cudaGraph_t body_out = add_while(s, h_out);
        c1 = launch_count();
        cudaStream_t s1 = aux[0], s2 = aux[1];
        JX_CUDA(cudaStreamBeginCaptureToGraph(s1, body_out, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        JX_CUDA(cudaGraphConditionalHandleCreate(&h_in, body_out, 0, cudaGraphCondAssignDefault));
        copy_dev(nn, b, r, s1);
        bsr_spmv<double, double>(A, -1.0, x, 1.0, r, kerr, s1, staged);
        sq_partials<<<G, kThreads, 0, s1>>>(nn, r, pt);
        JX_LAUNCH_CHECK();
        restart_kernel<<<1, kRedThreads, 0, s1>>>(st, pt, G, P, W, norms.get(), h_out, h_in);
        JX_LAUNCH_CHECK();
        if (f32)
            scale0_kernel<float><<<G1, kThreads, 0, s1>>>(nn, r, V32, st);
        else
            scale0_kernel<double><<<G1, kThreads, 0, s1>>>(nn, r, V, st);
        JX_LAUNCH_CHECK();
        cudaGraph_t body_in = add_while(s1, h_in);
        c2 = launch_count();
        JX_CUDA(cudaStreamBeginCaptureToGraph(s2, body_in, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        DepLaunchScope dep(S.prm.dep_launch);  // programmatic edges between the step's kernels
        if (f32)
            launch_dep(gather_kernel<float>, dim3(G1), dim3(kThreads), s2, nn, V32, st, cin.get());
        else
            launch_dep(gather_kernel<double>, dim3(G1), dim3(kThreads), s2, nn, V, st, cin.get());
        JX_LAUNCH_CHECK();
        S.cpr.apply_enqueue(cin.get(), cout.get(), s2);
        if (f32)
            launch_dep(scatter_kernel<float>, dim3(G1), dim3(kThreads), s2, nn, cout.get(), Z32, st, 1);
        else
            launch_dep(scatter_kernel<double>, dim3(G1), dim3(kThreads), s2, nn, cout.get(), Z, st, 0);
        JX_LAUNCH_CHECK();
        bsr_spmv<double, double>(A, 1.0, cout.get(), 0.0, w, kerr, s2, staged);
        if (f32)
            launch_dep(dots_kernel<float>, dim3(G), dim3(kThreads), s2, nn, V32, st, w, pt);
        else
            launch_dep(dots_kernel<double>, dim3(G), dim3(kThreads), s2, nn, V, st, w, pt);
        JX_LAUNCH_CHECK();
        if (P.selective)
            launch_dep(reduce_h_kernel, dim3(1), dim3(kRedThreads), s2, pt, G, st, P, W);
        else
            launch_dep(reduce_rows_kernel, dim3(kGgMaxK + 1), dim3(kThreads), s2, pt, G, st, W);
        JX_LAUNCH_CHECK();
        if (f32)
            launch_dep(update_dots_kernel<float>, dim3(G2), dim3(kThreads), s2, nn, V32, st, W.h1, w, pt);
        else
            launch_dep(update_dots_kernel<double>, dim3(G2), dim3(kThreads), s2, nn, V, st, W.h1, w, pt);
        JX_LAUNCH_CHECK();
        launch_dep(reduce_rows2_kernel, dim3(kGgMaxK + 1), dim3(kThreads), s2, pt, G2, st, W);
        JX_LAUNCH_CHECK();
        launch_dep(arnoldi_kernel, dim3(1), dim3(32), s2, st, P, W, norms.get(), h_in);
        JX_LAUNCH_CHECK();
        if (f32)
            launch_dep(final_kernel<float>, dim3(Gq), dim3(kThreads), s2, nn, V32, st, W.h2, w);
        else
            launch_dep(final_kernel<double>, dim3(Gq), dim3(kThreads), s2, nn, V, st, W.h2, w);
        JX_LAUNCH_CHECK();
        cudaGraph_t gchk = nullptr;
        JX_CUDA(cudaStreamEndCapture(s2, &gchk));
        c3 = launch_count();
        if (f32)
            update_x_kernel<float><<<Gq, kThreads, 0, s1>>>(nn, Z32, st, W.y, x);
        else
            update_x_kernel<double><<<Gq, kThreads, 0, s1>>>(nn, Z, st, W.y, x);
        JX_LAUNCH_CHECK();
        JX_CUDA(cudaStreamEndCapture(s1, &gchk));
        c4 = launch_count();
        summary_kernel<<<1, 1, 0, s>>>(st, kerr, S.cpr.amg.err.get(),
                                       S.cpr.bilu ? S.cpr.bilu->error_flag() : nullptr, out);
        JX_LAUNCH_CHECK();
    } catch (...) {
        end_capture_quietly(aux[1]);
        end_capture_quietly(aux[0]);
        uncount_launches(launch_count() - c0);
        throw;
    }
    const unsigned long long c5 = launch_count();
    kernels_step = c3 - c2;
    kernels_cycle = (c2 - c1) + (c4 - c3);
    kernels_fixed = (c1 - c0) + (c5 - c4);
    uncount_launches(c5 - c0);
}

void GraphGmres::build_single(Solver &S) {
    reset_graph();
    cudaStream_t cs = nullptr;
    JX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    try {
        JX_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        try {
            record(S, cs, summary.get());
        } catch (...) {
            gg::end_capture_quietly(cs);
            throw;
        }
        JX_CUDA(cudaStreamEndCapture(cs, &graph));
        JX_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    } catch (...) {
        cudaStreamDestroy(cs);
        reset_graph();
        throw;
    }
    cudaStreamDestroy(cs);
}

void GraphGmres::orth_native(int m, int reps, const double *w, cudaStream_t s) {
    using namespace gg;
    if (!exec || m < 1 || m > k) {
        set_error("krylov_native: needs a device-GMRES solve first and 1 <= m <= k_dim (%d)", k);
        throw std::invalid_argument("krylov_native");
    }
    GgState h{};
    h.i = m - 1;
    h.m = m;
    h.cont = 1;
    h.scale = 1.0;
    state.upload(&h, 1, s);
    const long long nn = n;
    GgState *st = state.get();
    double *pt = partials.get(), *ww = const_cast<double *>(w);
    for (int r = 0; r < reps; ++r) {
        if (fp32)
            dots_kernel<float><<<G, kThreads, 0, s>>>(nn, vptr32.get(), st, ww, pt);
        else
            dots_kernel<double><<<G, kThreads, 0, s>>>(nn, vptr.get(), st, ww, pt);
        JX_LAUNCH_CHECK();
        if (P.selective)
            reduce_h_kernel<<<1, kRedThreads, 0, s>>>(pt, G, st, P, W);
        else
            reduce_rows_kernel<<<kGgMaxK + 1, kThreads, 0, s>>>(pt, G, st, W);
        JX_LAUNCH_CHECK();
        if (fp32)
            update_dots_kernel<float><<<G2, kThreads, 0, s>>>(nn, vptr32.get(), st, W.h1, ww, pt);
        else
            update_dots_kernel<double><<<G2, kThreads, 0, s>>>(nn, vptr.get(), st, W.h1, ww, pt);
        JX_LAUNCH_CHECK();
        if (fp32)
            final_kernel<float><<<Gq, kThreads, 0, s>>>(nn, vptr32.get(), st, W.h2, ww);
        else
            final_kernel<double><<<Gq, kThreads, 0, s>>>(nn, vptr.get(), st, W.h2, ww);
        JX_LAUNCH_CHECK();
    }
}

unsigned long long GraphGmres::kernels_run(int iterations, int cycles) const {
    return kernels_fixed + (unsigned long long)cycles * kernels_cycle + (unsigned long long)iterations * kernels_step;
}

GmresResult GraphGmres::result_from(const double *sm, cudaStream_t s, bool with_norms) {
    GmresResult res;
    res.iterations = (int)sm[0];
    res.converged = sm[1] > 0.5 ? 1 : 0;
    res.stalled = sm[1] < -0.5 ? 1 : 0;
    res.rel_residual = sm[2];
    res.status = sm[3] != 0.0 ? JXCPR_ERROR_GENERIC : 0;
    if (with_norms) {
        res.norms.assign((size_t)res.iterations + 1, 0.0);
        JX_CUDA(cudaMemcpyAsync(res.norms.data(), norms.get(), sizeof(double) * (res.iterations + 1),
                                cudaMemcpyDeviceToHost, s));
        JX_CUDA(cudaStreamSynchronize(s));
    }
    return res;
}

}  // namespace jxcpr
