// Explicit inverse of the coarsest AMG operator (the fast path's coarse solve is a dense GEMV with
// it) by blocked Gauss-Jordan elimination without pivoting, in ONE cooperative kernel whose
// trailing updates run on the FP64 tensor cores (mma.sync m8n8k4 .f64, DMMA).
//
// The reference solves the coarsest level by dense Gaussian elimination without pivoting, assembled
// and eliminated again at every cycle (jxf_gselim, jxfpamg-0220/csrc/operation/matops/par_gs.c:20-74,
// called from par_relax_9.c:20-142).  The exact-order path keeps that elimination's order (amg.cu);
// the fast path inverts once at setup and needs only the same matrix inverse, so this kernel forms it
// with dense blocked updates instead of the 3n single-step launches of a column-by-column inversion.
//
// Algorithm (in place on the n x n matrix padded to N = 32 K with an identity block): for each
// 32-wide block column k,
//   1. P = inverse of the diagonal block X_kk (one CTA, unblocked Gauss-Jordan in shared memory);
//   2. row panel R_j = P X_kj (j != k) and a copy C_i = X_ik (i != k) of the column panel;
//   3. X_ij -= C_i R_j (i, j != k), X_ik = -C_i P, X_kj = R_j, X_kk = P.
// Steps 2 and 3 are 32x32x32 tile products, one warp per tile, each a 4 x 4 grid of 8x8 DMMA
// accumulators over 8 k-steps of 4.  A bounded grid barrier (grid_sync.cuh) separates the phases.
// A zero pivot inside a diagonal block (the elimination would divide by zero, as jxf_gselim's does
// not: it skips the row) raises err[1]; the caller reports the operator as singular.
#include <algorithm>
#include <stdexcept>

#include "amg.cuh"
#include "common.cuh"
#include "grid_sync.cuh"

namespace jxcpr {
namespace {

constexpr int kT = 32;          // block size
constexpr int kThreads = 256;   // 8 warps per CTA
constexpr int kWarps = kThreads / 32;

// d = a * b + d on one 8x8 FP64 tile (A 8x4 row fragment, B 4x8 column fragment, one value per lane each;
// D two values per lane: row lane / 4, columns 2 (lane % 4) and 2 (lane % 4) + 1).
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// acc += sa * A B for 32x32 row-major blocks A (leading dimension lda) and B (ldb); acc holds the 32x32
// result as 16 8x8 tiles (r, c) in the DMMA accumulator layout.
// Every operand of this kernel is rewritten between its phases by other CTAs, so all its loads go to
// L2 (__ldcg): no SM may keep a line of an earlier phase in L1.
__device__ __forceinline__ void tile_mma(const double *A, int lda, const double *B, int ldb, double sa,
                                         double acc[16][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 2
    for (int q = 0; q < kT; q += 4) {
        double a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) a[r] = sa * __ldcg(A + (long long)(r * 8 + g) * lda + q + t);
#pragma unroll
        for (int c = 0; c < 4; ++c) b[c] = __ldcg(B + (long long)(q + t) * ldb + c * 8 + g);
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) dmma(acc[r * 4 + c][0], acc[r * 4 + c][1], a[r], b[c]);
    }
}

__device__ __forceinline__ void tile_zero(double acc[16][2]) {
#pragma unroll
    for (int u = 0; u < 16; ++u) acc[u][0] = acc[u][1] = 0.0;
}

__device__ __forceinline__ void tile_load(const double *X, int ld, double acc[16][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const double2 v = __ldcg(reinterpret_cast<const double2 *>(X + (long long)(r * 8 + g) * ld + c * 8 + 2 * t));
            acc[r * 4 + c][0] = v.x;
            acc[r * 4 + c][1] = v.y;
        }
}

__device__ __forceinline__ void tile_store(double *X, int ld, const double acc[16][2]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
            *reinterpret_cast<double2 *>(X + (long long)(r * 8 + g) * ld + c * 8 + 2 * t) =
                make_double2(acc[r * 4 + c][0], acc[r * 4 + c][1]);
}

// warp copy of a 32x32 block
__device__ __forceinline__ void tile_copy(const double *S, int lds, double *D, int ldd) {
    const int lane = threadIdx.x & 31;
    for (int r = 0; r < kT; ++r) D[(long long)r * ldd + lane] = __ldcg(S + (long long)r * lds + lane);
}

// X: N x N (row-major), P: 32 x 32, R: 32 x N (row panel), C: N x 32 (column panel).
__global__ void __launch_bounds__(kThreads) gj_inverse_kernel(int N, double *X, double *P, double *R, double *C,
                                                              GridBarrier *bar, int *err) {
    __shared__ double sm[kT][kT + 1];
    const int K = N / kT;
    const int warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * kWarps + warp, nw = gridDim.x * kWarps;
    double acc[16][2];
    for (int k = 0; k < K; ++k) {
        // 1. P = inverse of the diagonal block (CTA 0): in-place Gauss-Jordan, 4 entries per thread
        if (blockIdx.x == 0) {
            const double *D = X + (long long)k * kT * N + (long long)k * kT;
            for (int e = threadIdx.x; e < kT * kT; e += kThreads)
                sm[e / kT][e % kT] = __ldcg(D + (long long)(e / kT) * N + e % kT);
            __syncthreads();
            for (int p = 0; p < kT; ++p) {
                const double piv = sm[p][p];
                if (piv == 0.0 && threadIdx.x == 0) atomicExch(err + 1, 1);
                const double d = piv != 0.0 ? 1.0 / piv : 0.0;
                double nv[kT * kT / kThreads];
#pragma unroll
                for (int u = 0; u < kT * kT / kThreads; ++u) {
                    const int e = threadIdx.x + u * kThreads, i = e / kT, j = e % kT;
                    if (i == p && j == p) nv[u] = d;
                    else if (i == p) nv[u] = sm[p][j] * d;
                    else if (j == p) nv[u] = -sm[i][p] * d;
                    else nv[u] = sm[i][j] - sm[i][p] * (sm[p][j] * d);
                }
                __syncthreads();
#pragma unroll
                for (int u = 0; u < kT * kT / kThreads; ++u) {
                    const int e = threadIdx.x + u * kThreads;
                    sm[e / kT][e % kT] = nv[u];
                }
                __syncthreads();
            }
            for (int e = threadIdx.x; e < kT * kT; e += kThreads) P[e] = sm[e / kT][e % kT];
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
        // 2. row panel R_j = P X_kj, column panel copy C_i = X_ik
        for (int task = gw; task < 2 * K; task += nw) {
            if (task < K) {
                const int j = task;
                if (j == k) continue;
                tile_zero(acc);
                tile_mma(P, kT, X + (long long)k * kT * N + (long long)j * kT, N, 1.0, acc);
                tile_store(R + (long long)j * kT, N, acc);
            } else {
                const int i = task - K;
                if (i == k) continue;
                tile_copy(X + (long long)i * kT * N + (long long)k * kT, N, C + (long long)i * kT * kT, kT);
            }
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
        // 3. trailing update and the new block row / column
        for (int task = gw; task < K * K; task += nw) {
            const int i = task / K, j = task % K;
            double *Xij = X + (long long)i * kT * N + (long long)j * kT;
            if (i == k && j == k) {
                tile_copy(P, kT, Xij, N);
            } else if (i == k) {
                tile_copy(R + (long long)j * kT, N, Xij, N);
            } else if (j == k) {
                tile_zero(acc);
                tile_mma(C + (long long)i * kT * kT, kT, P, kT, -1.0, acc);
                tile_store(Xij, N, acc);
            } else {
                tile_load(Xij, N, acc);
                tile_mma(C + (long long)i * kT * kT, kT, R + (long long)j * kT, N, -1.0, acc);
                tile_store(Xij, N, acc);
            }
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
    }
}

// X (N x N) = the n x n CSR operator padded with an identity block
__global__ void pad_assemble_kernel(int n, int N, const int *__restrict__ ia, const int *__restrict__ ja,
                                    const double *__restrict__ a, double *__restrict__ X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (i >= n) {
        X[(long long)i * N + i] = 1.0;
        return;
    }
    for (int k = ia[i]; k < ia[i + 1]; ++k) X[(long long)i * N + ja[k]] = a[k];
}

__global__ void pad_dense_kernel(int n, int N, const double *__restrict__ A, double *__restrict__ X) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * N) return;
    const int i = (int)(t / N), j = (int)(t % N);
    X[t] = (i < n && j < n) ? A[(long long)i * n + j] : (i == j ? 1.0 : 0.0);
}

int coop_blocks(int work_warps) {
    static int per_sm = 0;
    if (!per_sm) {
        JX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gj_inverse_kernel, kThreads, 0));
        if (per_sm < 1) per_sm = 1;
    }
    return std::max(1, std::min(per_sm * sm_count(), div_up(work_warps, kWarps)));
}

// Runs the kernel on the padded matrix X (N x N, device) with the hierarchy-independent scratch;
// err: 4 device ints (err[0] barrier flag, err[1] singular pivot, err[2..3] the barrier).
void gj_inverse_padded(int N, double *X, int *err, cudaStream_t s) {
    DevBuf<double> P((size_t)kT * kT), R((size_t)kT * N), C((size_t)N * kT);
    JX_CUDA(cudaMemsetAsync(err, 0, 4 * sizeof(int), s));
    GridBarrier *bar = reinterpret_cast<GridBarrier *>(err + 2);
    const int K = N / kT;
    int blocks = coop_blocks(K * K);
    int n_ = N;
    double *Xp = X, *Pp = P.get(), *Rp = R.get(), *Cp = C.get();
    void *args[] = {&n_, &Xp, &Pp, &Rp, &Cp, &bar, &err};
    JX_CUDA(cudaLaunchCooperativeKernel((void *)gj_inverse_kernel, blocks, kThreads, args, 0, s));
    count_launch();
    int flags[2] = {0, 0};
    JX_CUDA(cudaMemcpyAsync(flags, err, sizeof(flags), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    if (flags[0]) {
        set_error("coarse inverse: grid barrier timed out");
        throw CudaError{cudaErrorLaunchTimeout, "coarse inverse barrier"};
    }
    if (flags[1]) {
        set_error("coarse inverse: zero pivot (the coarsest operator is singular without pivoting)");
        throw std::invalid_argument("singular coarse operator");
    }
}

}  // namespace

void coarse_inverse_mma(const CsrView<double> &A, double *Ainv, int *err, cudaStream_t s) {
    const int n = A.nrows;
    if (n == 0) return;
    const int N = div_up(n, kT) * kT;
    DevBuf<double> X((size_t)N * N);
    X.zero(s);
    pad_assemble_kernel<<<div_up(N, 128), 128, 0, s>>>(n, N, A.ia, A.ja, A.a, X.get());
    JX_LAUNCH_CHECK();
    gj_inverse_padded(N, X.get(), err, s);
    JX_CUDA(cudaMemcpy2DAsync(Ainv, sizeof(double) * n, X.get(), sizeof(double) * N, sizeof(double) * n, n,
                              cudaMemcpyDeviceToDevice, s));
    JX_CUDA(cudaStreamSynchronize(s));
}

void dense_inverse_mma(int n, const double *A, double *Ainv, cudaStream_t s) {
    if (n == 0) return;
    const int N = div_up(n, kT) * kT;
    DevBuf<double> X((size_t)N * N);
    DevBuf<int> err(4);
    pad_dense_kernel<<<div_up((long long)N * N, 256), 256, 0, s>>>(n, N, A, X.get());
    JX_LAUNCH_CHECK();
    gj_inverse_padded(N, X.get(), err.get(), s);
    JX_CUDA(cudaMemcpy2DAsync(Ainv, sizeof(double) * n, X.get(), sizeof(double) * N, sizeof(double) * n, n,
                              cudaMemcpyDeviceToDevice, s));
    JX_CUDA(cudaStreamSynchronize(s));
}

}  // namespace jxcpr
