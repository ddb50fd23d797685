// Exact block ILU(0) with level-scheduled block triangular solves (stage2_solver_type 5 with
// bilu_exact 1).  No reference routine computes it in one pass: the reference approximates it by
// fixed-point sweeps and Jacobi triangular iterations (jxf_ILUSetupFGPBILU_v3, jxfpamg-0220/csrc/
// ilu/par_bilu_setup.c:5459-5609; jxf_par_Block_Jacobi_TriangularSolve_B, par_bilu_solve.c:
// 2893-3000), whose fixed point this is.  Every block operation below is the one those routines
// apply to the final values, in their order, so the factors and the solution equal the reference's
// bit for bit once its sweep and Jacobi counts exceed the number of levels.
//
//   levels   lower DAG: row r after every k of its L-row; upper DAG: row r after every c of its
//            U-row.  Longest-path depths by monotone relaxation on the device (one cooperative
//            kernel, one pass over the pattern per round until no level grows), rows then bucketed
//            by level (histogram, scan, scatter).  The row order inside a level does not matter:
//            its rows are independent.
//   factor   one cooperative kernel, a grid barrier per lower level; each row: its L entries by
//            ascending column C_rc = A_rc - sum_{k in L-row r} L_rk U_kc, L_rc = C_rc D_c^-1; then
//            D_r (guarded inverse), then its U entries.
//   solve    one cooperative kernel per refinement loop: forward substitution level by level,
//            y_r = -(sum_k L_rk y_k) + f_r, then backward over the upper levels,
//            t_r = D_r^-1 y_r + D_r^-1 (-(sum_c U_rc t_c)); then f -= A t and u += t (BSR products
//            with the reference's rounding).  Factors in FP64, or FP32 (the mixed path), vectors FP64.
// Values written inside a cooperative kernel by other CTAs are read with L2 loads (__ldcg).
#include <algorithm>
#include <stdexcept>

#include "bilu.cuh"
#include "grid_sync.cuh"

namespace jxcpr {

namespace {
constexpr int kT = 256;
constexpr double kMatTol = 1e-14;      // jx_parilu.h:241
constexpr double kRealMin = 1.0e-300;  // bsr_block_ops.h:21

template <int BS>
__device__ __forceinline__ void bm_mul(const double *A, const double *B, double *C) {
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
__device__ __forceinline__ double bm_det(const double *a) {
    if (BS == 2) return a[0] * a[3] - a[1] * a[2];
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
__device__ __forceinline__ void bm_inv(double *a) {
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

__device__ __forceinline__ int ldcg_i(const int *p) { return __ldcg(p); }

// ---- levels -------------------------------------------------------------------------------
// lev[r] = 1 + max lev[dep] over the row's dependencies (0 without), by rounds of relaxation until
// a round changes nothing (at most nb + 1 rounds); cnt: 3 rotating change counters; maxlev: the
// largest level seen.  Levels only grow and are bounded by the longest path, so the result does not
// depend on the order in which rows see their neighbours' values.
__global__ void __launch_bounds__(kT) levels_kernel(int nb, const int *__restrict__ dp, const int *__restrict__ di,
                                                    int *lev, int *cnt, int *maxlev, GridBarrier *bar, int *err) {
    const int stride = gridDim.x * blockDim.x;
    for (int round = 0; round <= nb + 1; ++round) {
        if (blockIdx.x == 0 && threadIdx.x == 0) cnt[(round + 1) % 3] = 0;
        int changed = 0;
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nb; r += stride) {
            int l = 0;
            for (int k = __ldg(dp + r); k < __ldg(dp + r + 1); ++k) l = max(l, ldcg_i(lev + __ldg(di + k)) + 1);
            if (l > ldcg_i(lev + r)) {
                lev[r] = l;
                changed = 1;
            }
        }
        if (changed) atomicAdd(cnt + round % 3, 1);
        if (!grid_barrier(bar, gridDim.x, err)) return;
        if (ldcg_i(cnt + round % 3) == 0) break;
        if (!grid_barrier(bar, gridDim.x, err)) return;  // every block has read the counter
    }
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nb; r += stride) atomicMax(maxlev, ldcg_i(lev + r));
}

__global__ void level_hist_kernel(int nb, const int *__restrict__ lev, int *__restrict__ cnt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nb) atomicAdd(cnt + lev[r], 1);
}

__global__ void level_scatter_kernel(int nb, const int *__restrict__ lev, const int *__restrict__ ptr,
                                     int *__restrict__ fill, int *__restrict__ rows) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nb) rows[ptr[lev[r]] + atomicAdd(fill + lev[r], 1)] = r;
}

// ---- factorisation ----------------------------------------------------------------------------
// C = A_rc - sum_{lj in L-row r} L_r,lja[lj] U_lja[lj],col (U searched in U-row k): the sweep's sum
template <int BS>
__device__ void c_block(int r, int col, const double *Ablk, const int *__restrict__ lia, const int *__restrict__ lja,
                        const double *la, const int *__restrict__ uia, const int *__restrict__ uja, const double *ua,
                        double *C) {
    constexpr int BN = BS * BS;
#pragma unroll
    for (int q = 0; q < BN; ++q) C[q] = __ldg(Ablk + q);
    for (int lj = __ldg(lia + r); lj < __ldg(lia + r + 1); ++lj) {
        const int k = __ldg(lja + lj);
        for (int uj = __ldg(uia + k); uj < __ldg(uia + k + 1); ++uj)
            if (__ldg(uja + uj) == col) {
                double Lb[BN], Ub[BN], t[BN];
#pragma unroll
                for (int q = 0; q < BN; ++q) {
                    Lb[q] = __ldcg(la + (long long)lj * BN + q);
                    Ub[q] = __ldcg(ua + (long long)uj * BN + q);
                }
                bm_mul<BS>(Lb, Ub, t);
#pragma unroll
                for (int q = 0; q < BN; ++q) C[q] -= t[q];
                break;
            }
    }
}

template <int BS>
__global__ void __launch_bounds__(kT) factor_kernel(int nlev, const int *__restrict__ lptr, const int *__restrict__ lrows,
                                                    const int *__restrict__ ia, const int *__restrict__ ja,
                                                    const double *__restrict__ a, const int *__restrict__ lia,
                                                    const int *__restrict__ lja, double *la, const int *__restrict__ uia,
                                                    const int *__restrict__ uja, double *ua, double *D, double *Dinv,
                                                    GridBarrier *bar, int *err) {
    constexpr int BN = BS * BS;
    const int stride = gridDim.x * blockDim.x;
    for (int lv = 0; lv < nlev; ++lv) {
        for (int t = __ldg(lptr + lv) + blockIdx.x * blockDim.x + threadIdx.x; t < __ldg(lptr + lv + 1); t += stride) {
            const int r = __ldg(lrows + t);
            const int a0 = __ldg(ia + r), a1 = __ldg(ia + r + 1);
            double C[BN];
            // L entries by ascending column; pl = position in L-row r (A's order)
            int last = -1;
            const int nl = __ldg(lia + r + 1) - __ldg(lia + r);
            for (int done = 0; done < nl; ++done) {
                int bc = 0x7fffffff, bpos = -1, bjj = -1, pl = __ldg(lia + r);
                for (int jj = a0; jj < a1; ++jj) {
                    const int c = __ldg(ja + jj);
                    if (c < r) {
                        if (c > last && c < bc) {
                            bc = c;
                            bpos = pl;
                            bjj = jj;
                        }
                        ++pl;
                    }
                }
                c_block<BS>(r, bc, a + (long long)bjj * BN, lia, lja, la, uia, uja, ua, C);
                double Dc[BN], out[BN];
#pragma unroll
                for (int q = 0; q < BN; ++q) Dc[q] = __ldcg(Dinv + (long long)bc * BN + q);
                bm_mul<BS>(C, Dc, out);
#pragma unroll
                for (int q = 0; q < BN; ++q) la[(long long)bpos * BN + q] = out[q];
                last = bc;
            }
            for (int jj = a0; jj < a1; ++jj)
                if (__ldg(ja + jj) == r) {
                    c_block<BS>(r, r, a + (long long)jj * BN, lia, lja, la, uia, uja, ua, C);
                    double d[BN];
#pragma unroll
                    for (int q = 0; q < BN; ++q) d[q] = C[q];
                    if (fabs(bm_det<BS>(d)) < kMatTol) {
#pragma unroll
                        for (int q = 0; q < BN; ++q) d[q] = (q % (BS + 1) == 0) ? 1.0 : 0.0;
                    }
#pragma unroll
                    for (int q = 0; q < BN; ++q) D[(long long)r * BN + q] = d[q];
                    bm_inv<BS>(d);
#pragma unroll
                    for (int q = 0; q < BN; ++q) Dinv[(long long)r * BN + q] = d[q];
                }
            int pu = __ldg(uia + r);
            for (int jj = a0; jj < a1; ++jj) {
                const int c = __ldg(ja + jj);
                if (c > r) {
                    c_block<BS>(r, c, a + (long long)jj * BN, lia, lja, la, uia, uja, ua, C);
#pragma unroll
                    for (int q = 0; q < BN; ++q) ua[(long long)pu * BN + q] = C[q];
                    ++pu;
                }
            }
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
    }
}

template <typename TV>
__global__ void to_value_kernel(long long n, const double *__restrict__ in, TV *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (TV)in[i];
}

// ---- level-scheduled substitution ------------------------------------------------------------
// forward: y_r = -(sum_k L_rk y_k) + f_r; backward: t_r = Dinv_r y_r + Dinv_r (-(sum_c U_rc t_c)),
// each sum in stored order with the BSR product's rounding (per entry, per component, m inner).
template <int BS, typename TV>
__global__ void __launch_bounds__(kT) subst_kernel(int nlev_l, const int *__restrict__ lptr, const int *__restrict__ lrows,
                                                   int nlev_u, const int *__restrict__ uptr, const int *__restrict__ urows,
                                                   const int *__restrict__ lia, const int *__restrict__ lja,
                                                   const TV *__restrict__ la, const int *__restrict__ uia,
                                                   const int *__restrict__ uja, const TV *__restrict__ ua,
                                                   const TV *__restrict__ dinv, const double *__restrict__ f, double *y,
                                                   double *t, GridBarrier *bar, int *err) {
    constexpr int BN = BS * BS;
    const int stride = gridDim.x * blockDim.x;
    for (int lv = 0; lv < nlev_l; ++lv) {
        for (int q0 = __ldg(lptr + lv) + blockIdx.x * blockDim.x + threadIdx.x; q0 < __ldg(lptr + lv + 1); q0 += stride) {
            const int r = __ldg(lrows + q0);
            double s[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) s[q] = 0.0;
            for (int k = __ldg(lia + r); k < __ldg(lia + r + 1); ++k) {
                const int c = __ldg(lja + k);
                double yc[BS];
#pragma unroll
                for (int m = 0; m < BS; ++m) yc[m] = __ldcg(y + (long long)c * BS + m);
#pragma unroll
                for (int q = 0; q < BS; ++q) {
                    double v = s[q];
#pragma unroll
                    for (int m = 0; m < BS; ++m) v += (double)__ldg(la + (long long)k * BN + q * BS + m) * yc[m];
                    s[q] = v;
                }
            }
#pragma unroll
            for (int q = 0; q < BS; ++q) y[(long long)r * BS + q] = s[q] * -1.0 + __ldg(f + (long long)r * BS + q);
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
    }
    for (int lv = 0; lv < nlev_u; ++lv) {
        for (int q0 = __ldg(uptr + lv) + blockIdx.x * blockDim.x + threadIdx.x; q0 < __ldg(uptr + lv + 1); q0 += stride) {
            const int r = __ldg(urows + q0);
            double s[BS], un[BS], tq[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) s[q] = 0.0;
            for (int k = __ldg(uia + r); k < __ldg(uia + r + 1); ++k) {
                const int c = __ldg(uja + k);
                double tc[BS];
#pragma unroll
                for (int m = 0; m < BS; ++m) tc[m] = __ldcg(t + (long long)c * BS + m);
#pragma unroll
                for (int q = 0; q < BS; ++q) {
                    double v = s[q];
#pragma unroll
                    for (int m = 0; m < BS; ++m) v += (double)__ldg(ua + (long long)k * BN + q * BS + m) * tc[m];
                    s[q] = v;
                }
            }
#pragma unroll
            for (int q = 0; q < BS; ++q) un[q] = s[q] * -1.0;
            double Di[BN], yr[BS];
#pragma unroll
            for (int q = 0; q < BN; ++q) Di[q] = (double)__ldg(dinv + (long long)r * BN + q);
#pragma unroll
            for (int m = 0; m < BS; ++m) yr[m] = __ldcg(y + (long long)r * BS + m);
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                double v = 0.0;
#pragma unroll
                for (int m = 0; m < BS; ++m) v += Di[q * BS + m] * un[m];
                tq[q] = v;
            }
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                double v = 0.0;
#pragma unroll
                for (int m = 0; m < BS; ++m) v += Di[q * BS + m] * yr[m];
                t[(long long)r * BS + q] = v + tq[q];
            }
        }
        if (!grid_barrier(bar, gridDim.x, err)) return;
    }
}

template <typename K>
int coop_grid_for(K kernel, int work) {
    int per_sm = 0;
    JX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kT, 0));
    if (per_sm < 1) per_sm = 1;
    return std::max(1, std::min(per_sm * sm_count(), div_up(std::max(work, 1), kT)));
}

void check_flags(int *err, cudaStream_t s, const char *what) {
    int f = 0;
    JX_CUDA(cudaMemcpyAsync(&f, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    if (f) {
        set_error("BILU %s: grid barrier timed out", what);
        throw CudaError{cudaErrorLaunchTimeout, what};
    }
}

// rows bucketed by level; returns the number of levels
int level_schedule(int nb, const int *dp, const int *di, DevBuf<int> &lev, DevBuf<int> &ptr, DevBuf<int> &rows,
                   std::vector<int> &h_ptr, int *err, cudaStream_t s) {
    lev.alloc(nb > 0 ? nb : 1);
    lev.zero(s);
    if (nb == 0) {
        h_ptr.assign(1, 0);
        ptr.alloc(1);
        ptr.zero(s);
        rows.alloc(1);
        return 0;
    }
    DevBuf<int> cnt(4);
    cnt.zero(s);
    JX_CUDA(cudaMemsetAsync(err, 0, 4 * sizeof(int), s));
    GridBarrier *bar = reinterpret_cast<GridBarrier *>(err + 2);
    int *levp = lev.get(), *cntp = cnt.get(), *mx = cnt.get() + 3;
    int n_ = nb;
    void *args[] = {&n_, (void *)&dp, (void *)&di, &levp, &cntp, &mx, &bar, &err};
    JX_CUDA(cudaLaunchCooperativeKernel((void *)levels_kernel, coop_grid_for(levels_kernel, nb), kT, args, 0, s));
    count_launch();
    check_flags(err, s, "levels");
    int maxlev = 0;
    JX_CUDA(cudaMemcpyAsync(&maxlev, mx, sizeof(int), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    const int nlev = maxlev + 1;
    DevBuf<int> hist(nlev + 1), fill(nlev + 1);
    hist.zero(s);
    fill.zero(s);
    level_hist_kernel<<<div_up(nb, kT), kT, 0, s>>>(nb, lev.get(), hist.get());
    JX_LAUNCH_CHECK();
    ptr.alloc(nlev + 1);
    exclusive_scan_int(hist.get(), ptr.get(), nlev + 1, s);
    rows.alloc(nb);
    level_scatter_kernel<<<div_up(nb, kT), kT, 0, s>>>(nb, lev.get(), ptr.get(), fill.get(), rows.get());
    JX_LAUNCH_CHECK();
    h_ptr.resize(nlev + 1);
    ptr.download(h_ptr.data(), nlev + 1, s);
    return nlev;
}
}  // namespace

void Bilu::setup_exact(const BsrView<double> &A, cudaStream_t s) {
    const int bn = bs * bs;
    DevBuf<int> err(4);
    nlev_l = level_schedule(nb, L.ia.get(), L.ja.get(), lev_l, lptr, lrows, h_lptr, err.get(), s);
    nlev_u = level_schedule(nb, U.ia.get(), U.ja.get(), lev_u, uptr, urows, h_uptr, err.get(), s);
    // the widest level bounds the threads a level can use: grids of that size keep the per-level grid
    // barrier (hundreds of levels on a reservoir grid) among as few blocks as possible
    widest = 1;
    for (size_t k = 0; k + 1 < h_lptr.size(); ++k) widest = std::max(widest, h_lptr[k + 1] - h_lptr[k]);
    for (size_t k = 0; k + 1 < h_uptr.size(); ++k) widest = std::max(widest, h_uptr[k + 1] - h_uptr[k]);
    // the upper levels are counted from the last row: level 0 rows have no U entries and come first
    if (nb) {
        JX_CUDA(cudaMemsetAsync(err.get(), 0, 4 * sizeof(int), s));
        GridBarrier *bar = reinterpret_cast<GridBarrier *>(err.get() + 2);
        int nl = nlev_l;
        const int *lp = lptr.get(), *lr = lrows.get(), *aia = A.ia, *aja = A.ja, *llia = L.ia.get(),
                  *llja = L.ja.get(), *luia = U.ia.get(), *luja = U.ja.get();
        const double *aa = A.a;
        double *pla = L.a.get(), *pua = U.a.get(), *pd = D.get(), *pdi = Dinv.get();
        int *pe = err.get();
        void *args[] = {&nl, &lp, &lr, &aia, &aja, &aa, &llia, &llja, &pla, &luia, &luja, &pua, &pd, &pdi, &bar, &pe};
        void *fn = bs == 2 ? (void *)factor_kernel<2> : (void *)factor_kernel<3>;
        const int grid = bs == 2 ? coop_grid_for(factor_kernel<2>, widest) : coop_grid_for(factor_kernel<3>, widest);
        JX_CUDA(cudaLaunchCooperativeKernel(fn, grid, kT, args, 0, s));
        count_launch();
        check_flags(err.get(), s, "factorisation");
    }
    if (fp32) {
        la32.alloc((size_t)(L.nnzb > 0 ? L.nnzb : 1) * bn);
        ua32.alloc((size_t)(U.nnzb > 0 ? U.nnzb : 1) * bn);
        dinv32.alloc((size_t)(nb > 0 ? nb : 1) * bn);
        auto cvt = [&](long long n, const double *in, float *out) {
            if (n) to_value_kernel<float><<<div_up(n, kT), kT, 0, s>>>(n, in, out);
            JX_LAUNCH_CHECK();
        };
        cvt(L.nnzb * bn, L.a.get(), la32.get());
        cvt(U.nnzb * bn, U.a.get(), ua32.get());
        cvt((long long)nb * bn, Dinv.get(), dinv32.get());
    }
    subst_err.alloc(4);
    subst_err.zero(s);
    JX_CUDA(cudaStreamSynchronize(s));
}

void Bilu::substitute(const double *f, double *y, double *t, cudaStream_t s) {
    // reset the barrier only: a time-out flag in subst_err[0] stays until the solver reads it
    JX_CUDA(cudaMemsetAsync(subst_err.get() + 2, 0, 2 * sizeof(int), s));
    GridBarrier *bar = reinterpret_cast<GridBarrier *>(subst_err.get() + 2);
    int nl = nlev_l, nu = nlev_u;
    const int *lp = lptr.get(), *lr = lrows.get(), *up = uptr.get(), *ur = urows.get(), *llia = L.ia.get(),
              *llja = L.ja.get(), *luia = U.ia.get(), *luja = U.ja.get();
    int *pe = subst_err.get();
    void *fn;
    int grid;
    if (fp32) {
        const float *pla = la32.get(), *pua = ua32.get(), *pdi = dinv32.get();
        void *args[] = {&nl, &lp, &lr, &nu, &up, &ur, &llia, &llja, &pla, &luia, &luja, &pua, &pdi,
                        (void *)&f, &y, &t, &bar, &pe};
        fn = bs == 2 ? (void *)subst_kernel<2, float> : (void *)subst_kernel<3, float>;
        grid = bs == 2 ? coop_grid_for(subst_kernel<2, float>, widest) : coop_grid_for(subst_kernel<3, float>, widest);
        JX_CUDA(cudaLaunchCooperativeKernel(fn, grid, kT, args, 0, s));
    } else {
        const double *pla = L.a.get(), *pua = U.a.get(), *pdi = Dinv.get();
        void *args[] = {&nl, &lp, &lr, &nu, &up, &ur, &llia, &llja, &pla, &luia, &luja, &pua, &pdi,
                        (void *)&f, &y, &t, &bar, &pe};
        fn = bs == 2 ? (void *)subst_kernel<2, double> : (void *)subst_kernel<3, double>;
        grid = bs == 2 ? coop_grid_for(subst_kernel<2, double>, widest) : coop_grid_for(subst_kernel<3, double>, widest);
        JX_CUDA(cudaLaunchCooperativeKernel(fn, grid, kT, args, 0, s));
    }
    count_launch();
}



}  // namespace jxcpr
