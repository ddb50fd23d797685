// Gauss-Seidel smoothers on the device.
//
// A sweep visits the groups of a Schedule in order; the rows of one group are
// updated concurrently.  Row i reads the NEW value of a neighbour j when
// rank[j] < rank[i] and the value at sweep start (a copy, `vt`) otherwise --
// exactly what a sequential sweep in rank order reads.  With the level
// schedule of the natural ordering (rank = i forward, n-1-i backward) this
// reproduces the reference's sequential sweeps bit for bit; with a
// multicolour schedule (rank = colour) it is Gauss-Seidel in colour order.
//
// * gs_sweep:  jxf_PAMGRelax6 with relax_weight = omega = 1 at one rank and
//   one thread (jxfpamg-0220/csrc/operation/relaxations/par_relax_6.c:226-270):
//   u_i = (f_i - sum_{j != i} a_ij u_j) / a_ii, skipped when a_ii == 0.
// * hgs_sweep: jxf_ParBSRHGSRelax (jxfpamg-0220/csrc/amg/par_relax_bsr.c:193-573)
//   with its Kahan-compensated block products (seq_bsr_matrix.c:841-872) and
//   2x2 / 3x3 diagonal-block solves (:945-1100).
//
// Execution: one persistent cooperative kernel per sweep; groups are
// separated by a grid barrier whose wait is bounded (a timeout raises the
// error flag and every CTA leaves).  Small systems run in a single CTA with
// __syncthreads between groups.
#include <cooperative_groups.h>

#include "amg.cuh"
#include "common.cuh"
#include "grid_sync.cuh"

namespace jxcpr {

// ---------------------------------------------------------------------------
// scalar Gauss-Seidel row update
// ---------------------------------------------------------------------------
__device__ __forceinline__ void gs_row(int i, const int *__restrict__ ia, const int *__restrict__ ja,
                                       const double *__restrict__ a, const int *__restrict__ rank,
                                       const double *__restrict__ f, double *u, const double *__restrict__ vt) {
    const int d = ia[i];
    if (d == ia[i + 1]) return;
    const double diag = a[d];
    if (diag == 0.0) return;
    const int ri = rank[i];
    double res = f[i];
    for (int k = d + 1; k < ia[i + 1]; ++k) {
        const int j = ja[k];
        const double uj = (rank[j] < ri) ? ((volatile const double *)u)[j] : vt[j];
        res = res - a[k] * uj;
    }
    u[i] = res / diag;
}

__global__ void gs_sweep_grid_kernel(int ngroups, const int *__restrict__ gptr, const int *__restrict__ perm,
                                     const int *__restrict__ ia, const int *__restrict__ ja,
                                     const double *__restrict__ a, const int *__restrict__ rank,
                                     const double *__restrict__ f, double *u, const double *__restrict__ vt,
                                     GridBarrier *bar, int *err) {
    const int nthreads = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int g = 0; g < ngroups; ++g) {
        const int r0 = gptr[g], r1 = gptr[g + 1];
        for (int t = r0 + tid; t < r1; t += nthreads) gs_row(perm[t], ia, ja, a, rank, f, u, vt);
        if (g + 1 < ngroups) {
            __threadfence();
            if (!grid_barrier(bar, gridDim.x, err)) return;
        }
    }
}

__global__ void gs_sweep_block_kernel(int ngroups, const int *__restrict__ gptr, const int *__restrict__ perm,
                                      const int *__restrict__ ia, const int *__restrict__ ja,
                                      const double *__restrict__ a, const int *__restrict__ rank,
                                      const double *__restrict__ f, double *u, const double *__restrict__ vt) {
    // ngroups == 1: any number of CTAs; otherwise a single CTA (barrier = __syncthreads)
    const int stride = gridDim.x * blockDim.x;
    for (int g = 0; g < ngroups; ++g) {
        const int r0 = gptr[g], r1 = gptr[g + 1];
        for (int t = r0 + blockIdx.x * blockDim.x + threadIdx.x; t < r1; t += stride)
            gs_row(perm[t], ia, ja, a, rank, f, u, vt);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// block hybrid Gauss-Seidel row update
// ---------------------------------------------------------------------------
template <int BS>
__device__ __forceinline__ void blk_matvec_stable(double alpha, const double *__restrict__ mat, const double *v,
                                                  double *ov) {
    double tmp[BS];
#pragma unroll
    for (int j = 0; j < BS; ++j) tmp[j] = ov[j] * 1.0;
#pragma unroll
    for (int i = 0; i < BS; ++i) {
        double sum = 0.0, c = 0.0;
#pragma unroll
        for (int j = 0; j < BS; ++j) {
            const double y = mat[i * BS + j] * v[j] - c;
            const double t = sum + y;
            c = (t - sum) - y;
            sum = t;
        }
        tmp[i] += alpha * sum;
        ov[i] = tmp[i];
    }
}

template <int BS>
__device__ __forceinline__ void blk_inv_matvec(const double *__restrict__ mat, const double *v, double *ov) {
    if (BS == 2) {
        const double a11 = mat[0], a12 = mat[1], a21 = mat[2], a22 = mat[3];
        const double det = a11 * a22 - a12 * a21;
        if (fabs(det) < 1e-12 * (fabs(a11 * a22) + fabs(a12 * a21))) {
            ov[0] = v[0] / (a11 + 1e-12);
            ov[1] = v[1] / (a22 + 1e-12);
            return;
        }
        const double inv_det = 1.0 / det;
        const double b1 = v[0], b2 = v[1];
        ov[0] = (a22 * b1 - a12 * b2) * inv_det;
        ov[1] = (-a21 * b1 + a11 * b2) * inv_det;
        return;
    }
    double m[9], x[3], o[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = mat[q];
#pragma unroll
    for (int q = 0; q < 3; ++q) x[q] = v[q];
    const int n = 3;
    for (int i = 0; i < n; ++i) {
        int mr = i;
        double mv = fabs(m[i * n + i]);
        for (int k = i + 1; k < n; ++k)
            if (fabs(m[k * n + i]) > mv) {
                mv = fabs(m[k * n + i]);
                mr = k;
            }
        if (mv < 1e-15) {
            for (int j = 0; j < n; ++j) {
                const double d = m[j * n + j];
                o[j] = (fabs(d) > 1e-12) ? x[j] / d : 0.0;
            }
            break;
        }
        if (mr != i) {
            for (int j = 0; j < n; ++j) {
                const double t = m[i * n + j];
                m[i * n + j] = m[mr * n + j];
                m[mr * n + j] = t;
            }
            const double t = x[i];
            x[i] = x[mr];
            x[mr] = t;
        }
        const double pivot = m[i * n + i];
        for (int k = i + 1; k < n; ++k) {
            const double fct = m[k * n + i] / pivot;
            m[k * n + i] = fct;
            for (int j = i + 1; j < n; ++j) m[k * n + j] -= fct * m[i * n + j];
        }
    }
    for (int i = 0; i < n; ++i) {
        o[i] = x[i];
        for (int j = 0; j < i; ++j) o[i] -= m[i * n + j] * o[j];
    }
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) o[i] -= m[i * n + j] * o[j];
        const double d = m[i * n + i];
        if (fabs(d) > 1e-15) o[i] /= d; else o[i] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) ov[q] = o[q];
}

// vt: the iterate at the start of the pass (read for neighbours not yet
// updated in it); vt2: the vector of the res2 term (vt for HGS, the CPR's work
// vector for HSGS).
template <int BS>
__device__ __forceinline__ void hgs_row(int i, const int *__restrict__ ia, const int *__restrict__ ja,
                                        const double *__restrict__ a, const int *__restrict__ rank,
                                        const double *__restrict__ b, double *x, const double *__restrict__ vt,
                                        const double *__restrict__ vt2, double w, double omega, bool plain) {
    constexpr int B2 = BS * BS;
    const int ri = rank[i];
    const long long d = ia[i], e = ia[i + 1];
    double res[BS], out[BS];
#pragma unroll
    for (int k = 0; k < BS; ++k) res[k] = b[(long long)i * BS + k];
    if (plain) {
        for (long long jj = d + 1; jj < e; ++jj) {
            const int j = ja[jj];
            double xj[BS];
            const bool fresh = rank[j] < ri;
#pragma unroll
            for (int k = 0; k < BS; ++k)
                xj[k] = fresh ? ((volatile const double *)x)[(long long)j * BS + k] : vt[(long long)j * BS + k];
            blk_matvec_stable<BS>(-1.0, a + jj * B2, xj, res);
        }
        blk_inv_matvec<BS>(a + d * B2, res, out);
#pragma unroll
        for (int k = 0; k < BS; ++k) x[(long long)i * BS + k] = out[k];
        return;
    }
    double res0[BS], res2[BS], tmp[BS];
#pragma unroll
    for (int k = 0; k < BS; ++k) {
        res0[k] = 0.0;
        res2[k] = 0.0;
    }
    for (long long jj = d + 1; jj < e; ++jj) {
        const int j = ja[jj];
        double xj[BS], vj[BS];
        const bool fresh = rank[j] < ri;
#pragma unroll
        for (int k = 0; k < BS; ++k) {
            vj[k] = vt2[(long long)j * BS + k];
            xj[k] = fresh ? ((volatile const double *)x)[(long long)j * BS + k] : vt[(long long)j * BS + k];
        }
        blk_matvec_stable<BS>(-1.0, a + jj * B2, xj, res0);
        blk_matvec_stable<BS>(1.0, a + jj * B2, vj, res2);
    }
    const double prod = 1.0 - w * omega, omo = 1.0 - omega;
#pragma unroll
    for (int k = 0; k < BS; ++k) tmp[k] = omega * res[k] + res0[k] + omo * res2[k];
    blk_inv_matvec<BS>(a + d * B2, tmp, out);
#pragma unroll
    for (int k = 0; k < BS; ++k) {
        double xv = x[(long long)i * BS + k];
        xv *= prod;
        xv += w * out[k];
        x[(long long)i * BS + k] = xv;
    }
}

template <int BS>
__global__ void hgs_sweep_grid_kernel(int ngroups, const int *__restrict__ gptr, const int *__restrict__ perm,
                                      const int *__restrict__ ia, const int *__restrict__ ja,
                                      const double *__restrict__ a, const int *__restrict__ rank,
                                      const double *__restrict__ b, double *x, const double *__restrict__ vt,
                                      const double *__restrict__ vt2, double w, double omega, int plain,
                                      GridBarrier *bar, int *err) {
    const int nthreads = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (int g = 0; g < ngroups; ++g) {
        const int r0 = gptr[g], r1 = gptr[g + 1];
        for (int t = r0 + tid; t < r1; t += nthreads)
            hgs_row<BS>(perm[t], ia, ja, a, rank, b, x, vt, vt2, w, omega, plain);
        if (g + 1 < ngroups) {
            __threadfence();
            if (!grid_barrier(bar, gridDim.x, err)) return;
        }
    }
}

template <int BS>
__global__ void hgs_sweep_block_kernel(int ngroups, const int *__restrict__ gptr, const int *__restrict__ perm,
                                       const int *__restrict__ ia, const int *__restrict__ ja,
                                       const double *__restrict__ a, const int *__restrict__ rank,
                                       const double *__restrict__ b, double *x, const double *__restrict__ vt,
                                       const double *__restrict__ vt2, double w, double omega, int plain) {
    const int stride = gridDim.x * blockDim.x;
    for (int g = 0; g < ngroups; ++g) {
        const int r0 = gptr[g], r1 = gptr[g + 1];
        for (int t = r0 + blockIdx.x * blockDim.x + threadIdx.x; t < r1; t += stride)
            hgs_row<BS>(perm[t], ia, ja, a, rank, b, x, vt, vt2, w, omega, plain);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
namespace {
constexpr int kSweepThreads = 256;
constexpr int kSmallRows = 12288;

// The grid barrier of a cooperative sweep lives beside the hierarchy's error flag (err[0]) in the
// same per-hierarchy allocation (err[2..3]), so exact-order sweeps of different solvers on
// concurrent streams never share a barrier.
GridBarrier *barrier_of(int *err) { return reinterpret_cast<GridBarrier *>(err + 2); }

template <typename K>
int coop_grid(K kernel) {
    int per_sm = 0;
    JX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSweepThreads, 0));
    if (per_sm < 1) per_sm = 1;
    return per_sm * sm_count();
}
}  // namespace

void gs_sweep(const CsrView<double> &A, const Schedule &sch, const double *f, double *u, const int *rank,
              double *vt, int *err, cudaStream_t s) {
    const int n = A.nrows;
    if (n == 0 || sch.ngroups == 0) return;
    JX_CUDA(cudaMemcpyAsync(vt, u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    if (n <= kSmallRows || sch.ngroups == 1) {
        const int threads = sch.ngroups == 1 ? 256 : 1024;
        const int blocks = sch.ngroups == 1 ? div_up(n, 256) : 1;
        gs_sweep_block_kernel<<<blocks, threads, 0, s>>>(sch.ngroups, sch.group_ptr.get(), sch.perm.get(), A.ia,
                                                         A.ja, A.a, rank, f, u, vt);
        JX_LAUNCH_CHECK();
        return;
    }
    static int grid = 0;
    if (!grid) grid = coop_grid(gs_sweep_grid_kernel);
    const int blocks = std::min(grid, div_up(sch.max_group, kSweepThreads));
    GridBarrier *bar = barrier_of(err);
    JX_CUDA(cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s));
    int ng = sch.ngroups;
    const int *gp = sch.group_ptr.get(), *pm = sch.perm.get();
    const int *aia = A.ia, *aja = A.ja;
    const double *aa = A.a;
    void *args[] = {&ng, &gp, &pm, &aia, &aja, &aa, &rank, &f, &u, &vt, &bar, &err};
    JX_CUDA(cudaLaunchCooperativeKernel((void *)gs_sweep_grid_kernel, blocks, kSweepThreads, args, 0, s));
    count_launch();
}

namespace {
// One pass of the block point update along `sch` (vt already holds the iterate at the pass start).
void hgs_pass(const BsrView<double> &A, const Schedule &sch, const double *b, double *x, const int *rank,
              const double *vt, const double *vt2, double w, double omega, int plain, int *err, cudaStream_t s) {
    const int nb = A.nb;
    if (nb <= kSmallRows || sch.ngroups == 1) {
        const int threads = sch.ngroups == 1 ? 256 : 1024;
        const int blocks = sch.ngroups == 1 ? div_up(nb, 256) : 1;
        if (A.bs == 2)
            hgs_sweep_block_kernel<2><<<blocks, threads, 0, s>>>(sch.ngroups, sch.group_ptr.get(), sch.perm.get(),
                                                                 A.ia, A.ja, A.a, rank, b, x, vt, vt2, w, omega,
                                                                 plain);
        else
            hgs_sweep_block_kernel<3><<<blocks, threads, 0, s>>>(sch.ngroups, sch.group_ptr.get(), sch.perm.get(),
                                                                 A.ia, A.ja, A.a, rank, b, x, vt, vt2, w, omega,
                                                                 plain);
        JX_LAUNCH_CHECK();
        return;
    }
    static int grid2 = 0, grid3 = 0;
    if (!grid2) grid2 = coop_grid(hgs_sweep_grid_kernel<2>);
    if (!grid3) grid3 = coop_grid(hgs_sweep_grid_kernel<3>);
    const int grid = A.bs == 2 ? grid2 : grid3;
    const int blocks = std::min(grid, div_up(sch.max_group, kSweepThreads));
    GridBarrier *bar = barrier_of(err);
    JX_CUDA(cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s));
    int ng = sch.ngroups;
    const int *gp = sch.group_ptr.get(), *pm = sch.perm.get();
    const int *aia = A.ia, *aja = A.ja;
    const double *aa = A.a;
    void *args[] = {&ng, &gp, &pm, &aia, &aja, &aa, &rank, &b, &x, &vt, &vt2, &w, &omega, &plain, &bar, &err};
    void *fn = A.bs == 2 ? (void *)hgs_sweep_grid_kernel<2> : (void *)hgs_sweep_grid_kernel<3>;
    JX_CUDA(cudaLaunchCooperativeKernel(fn, blocks, kSweepThreads, args, 0, s));
    count_launch();
}

int plain_weights(double w, double omega) {
    const double eps = 2.220446049250313e-16;
    return (fabs(w - 1) < eps && fabs(omega - 1) < eps) ? 1 : 0;
}
}  // namespace

void hgs_sweep(const BsrView<double> &A, const Schedule &sch, const double *b, double *x, const int *rank,
               double *vt, double w, double omega, int *err, cudaStream_t s) {
    const int nb = A.nb;
    if (nb == 0 || sch.ngroups == 0) return;
    JX_CUDA(cudaMemcpyAsync(vt, x, sizeof(double) * nb * A.bs, cudaMemcpyDeviceToDevice, s));
    hgs_pass(A, sch, b, x, rank, vt, vt, w, omega, plain_weights(w, omega), err, s);
}

void hsgs_sweep(const BsrView<double> &A, const Schedule &fwd, const Schedule &bwd, const double *b, double *x,
                double *vt, double *work, double w, double omega, int *err, cudaStream_t s) {
    const int nb = A.nb;
    if (nb == 0 || fwd.ngroups == 0 || bwd.ngroups == 0) return;
    const int plain = plain_weights(w, omega);
    // the reference refreshes only the first nb (block-row count) entries of its work vector
    if (!plain) JX_CUDA(cudaMemcpyAsync(work, x, sizeof(double) * nb, cudaMemcpyDeviceToDevice, s));
    JX_CUDA(cudaMemcpyAsync(vt, x, sizeof(double) * nb * A.bs, cudaMemcpyDeviceToDevice, s));
    hgs_pass(A, fwd, b, x, fwd.rank.get(), vt, work, w, omega, plain, err, s);
    JX_CUDA(cudaMemcpyAsync(vt, x, sizeof(double) * nb * A.bs, cudaMemcpyDeviceToDevice, s));
    hgs_pass(A, bwd, b, x, bwd.rank.get(), vt, work, w, omega, plain, err, s);
}

}  // namespace jxcpr
