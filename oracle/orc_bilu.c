/*
 * ORACLE (test infrastructure only): restatement of the reference's block
 * ILU(0) with fixed-point ("fine-grained parallel") factorisation and the
 * Jacobi-iteration triangular solves, single-threaded.
 *
 *   setup  jxf_ILUSetupFGPBILU_v3  jxfpamg-0220/csrc/ilu/par_bilu_setup.c:4996-5676
 *          (initial split :5108-5222, sweeps :5459-5609), block helpers
 *          jxfpamg-0220/csrc/mat_vec_data/jxf_bsr_block_ops.c:26-130,398-460
 *   solve  jxf_BILUSolve (max_iter 1, tol 0, tri_solve 14)
 *          jxfpamg-0220/csrc/ilu/par_bilu_solve.c:17-420, case 14 ->
 *          jxf_par_Block_Jacobi_TriangularSolve_B :2893-3000
 *
 * Factorisation: A = (I + L)(D + U) on the pattern of A (L strictly lower,
 * U strictly upper, D block diagonal).  Start: D_r = A_rr (identity when
 * |det| < 1e-14), L_rc = A_rc D_c^-1, U_rc = A_rc.  Each sweep:
 *   C_rc = A_rc - sum_{k in L-row r} L_rk U_kc   (U_kc found in U-row k)
 *   D_r = C_rr (guarded), L_rc = C_rc D_c^-1, U_rc = C_rc.
 * The reference processes rows in order on one thread, so D_c^-1 of column
 * c < r is already the current sweep's when row r uses it.
 *
 * Solve (u = 0 on entry): ftemp = f - A u; IR times: y = 0, `lower` Jacobi
 * sweeps y <- ftemp - L y; t = 0, `upper` sweeps t <- D^-1 y + D^-1(-U t);
 * ftemp <- ftemp - A t; u <- u + t.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define ORC_MAT_TOL 1e-14    /* jx_parilu.h:241 */
#define ORC_REAL_MIN 1.0e-300 /* bsr_block_ops.h:21 */

static void blk_matmul(const double *A, const double *B, double *C, int n)
{
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            double sum = 0.0;
            for (int k = 0; k < n; k++) sum += A[i * n + k] * B[k * n + j];
            C[i * n + j] = sum;
        }
}

static double blk_det(const double *a, int n)
{
    if (n == 1) return a[0];
    if (n == 2) return a[0] * a[3] - a[1] * a[2];
    /* cofactor expansion along row 0 (n = 3 here) */
    double det = 0.0, sub[4];
    for (int col = 0; col < n; col++) {
        int si = 0;
        for (int i = 1; i < n; i++)
            for (int j = 0; j < n; j++) {
                if (j == col) continue;
                sub[si++] = a[i * n + j];
            }
        const double sign = (col % 2 == 0) ? 1.0 : -1.0;
        det += sign * a[col] * blk_det(sub, n - 1);
    }
    return det;
}

static void blk_inv(double *a, int n)
{
    if (n == 2) {
        const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3];
        const double det = a0 * a3 - a1 * a2;
        if (fabs(det) < ORC_REAL_MIN) {
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
    if (fabs(det) < ORC_REAL_MIN) {
        memset(a, 0, 9 * sizeof(double));
        a[0] = a[4] = a[8] = 1.0;
    } else {
        const double di = 1.0 / det;
        a[0] = M0 * di; a[1] = M3 * di; a[2] = M6 * di;
        a[3] = M1 * di; a[4] = M4 * di; a[5] = M7 * di;
        a[6] = M2 * di; a[7] = M5 * di; a[8] = M8 * di;
    }
}

/* guarded copy of a diagonal block into d, its inverse into dinv */
static void diag_update(const double *blk, double *d, double *dinv, int bs)
{
    const int bn = bs * bs;
    memcpy(d, blk, bn * sizeof(double));
    if (fabs(blk_det(d, bs)) < ORC_MAT_TOL) {
        memset(d, 0, bn * sizeof(double));
        for (int k = 0; k < bs; k++) d[k * bs + k] = 1.0;
    }
    memcpy(dinv, d, bn * sizeof(double));
    blk_inv(dinv, bs);
}

/* L / U patterns: the entries of each row of A with col < r / col > r, in A's order. */
int orc_bilu_pattern(int nb, const int *ia, const int *ja, int *lia, int *lja, int *uia, int *uja)
{
    int nl = 0, nu = 0;
    lia[0] = uia[0] = 0;
    for (int r = 0; r < nb; r++) {
        for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
            if (ja[jj] < r) lja[nl++] = ja[jj];
            else if (ja[jj] > r) uja[nu++] = ja[jj];
        }
        lia[r + 1] = nl;
        uia[r + 1] = nu;
    }
    return 0;
}

int orc_bilu_setup(int nb, int bs, const int *ia, const int *ja, const double *a, int sweeps, const int *lia,
                   const int *lja, double *la, const int *uia, const int *uja, double *ua, double *dinv)
{
    const int bn = bs * bs;
    double *d = malloc(sizeof(double) * (size_t)nb * bn);
    double *C = malloc(sizeof(double) * ((size_t)ia[nb] + 1) * bn);
    double tmp[9];
    /* initial split (rows in order: D_c^-1 of c < r is ready when row r needs it) */
    for (int r = 0; r < nb; r++) {
        int pl = lia[r], pu = uia[r];
        for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
            const int col = ja[jj];
            const double *A = a + (size_t)jj * bn;
            if (col < r) blk_matmul(A, dinv + (size_t)col * bn, la + (size_t)(pl++) * bn, bs);
            else if (col > r) memcpy(ua + (size_t)(pu++) * bn, A, bn * sizeof(double));
            else diag_update(A, d + (size_t)r * bn, dinv + (size_t)r * bn, bs);
        }
    }
    for (int sw = 0; sw < sweeps; sw++) {
        for (int r = 0; r < nb; r++)
            for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
                const int col = ja[jj];
                double *Cb = C + (size_t)jj * bn;
                memcpy(Cb, a + (size_t)jj * bn, bn * sizeof(double));
                for (int lj = lia[r]; lj < lia[r + 1]; lj++) {
                    const int k = lja[lj];
                    for (int uj = uia[k]; uj < uia[k + 1]; uj++)
                        if (uja[uj] == col) {
                            blk_matmul(la + (size_t)lj * bn, ua + (size_t)uj * bn, tmp, bs);
                            for (int q = 0; q < bn; q++) Cb[q] -= tmp[q];
                            break;
                        }
                }
            }
        for (int r = 0; r < nb; r++) {
            for (int jj = ia[r]; jj < ia[r + 1]; jj++)
                if (ja[jj] == r) {
                    diag_update(C + (size_t)jj * bn, d + (size_t)r * bn, dinv + (size_t)r * bn, bs);
                    break;
                }
            int pl = lia[r], pu = uia[r];
            for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
                const int col = ja[jj];
                const double *Cb = C + (size_t)jj * bn;
                if (col < r) blk_matmul(Cb, dinv + (size_t)col * bn, la + (size_t)(pl++) * bn, bs);
                else if (col > r) memcpy(ua + (size_t)(pu++) * bn, Cb, bn * sizeof(double));
            }
        }
    }
    free(C);
    free(d);
    return 0;
}

int orc_bilu_solve(int nb, int bs, const int *ia, const int *ja, const double *a, const int *lia, const int *lja,
                   const double *la, const int *uia, const int *uja, const double *ua, const double *dinv,
                   int ir_iters, int lower_iters, int upper_iters, const double *f, double *u)
{
    const int n = nb * bs, bn = bs * bs;
    double *ft = malloc(sizeof(double) * n), *ut = malloc(sizeof(double) * n), *yt = malloc(sizeof(double) * n),
           *un = malloc(sizeof(double) * n);
    memcpy(ft, f, sizeof(double) * n);
    orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, u, 1.0, ft);
    for (int it = 0; it < ir_iters; it++) {
        memset(ut, 0, sizeof(double) * n);
        memset(yt, 0, sizeof(double) * n);
        memset(un, 0, sizeof(double) * n);
        for (int k = 0; k < lower_iters; k++) {
            orc_bsr_matvec(nb, bs, lia, lja, la, -1.0, yt, 0.0, ut);
            for (int i = 0; i < n; i++) yt[i] = ut[i] + ft[i];
        }
        memset(ut, 0, sizeof(double) * n);
        for (int k = 0; k < upper_iters; k++) {
            orc_bsr_matvec(nb, bs, uia, uja, ua, -1.0, ut, 0.0, un);
            for (int r = 0; r < nb; r++) {
                const double *D = dinv + (size_t)r * bn;
                double *ub = un + (size_t)r * bs, t[3];
                for (int q = 0; q < bs; q++) {
                    double s = 0.0;
                    for (int j = 0; j < bs; j++) s += D[q * bs + j] * ub[j];
                    t[q] = s;
                }
                for (int q = 0; q < bs; q++) ub[q] = t[q];
            }
            for (int r = 0; r < nb; r++) {
                const double *D = dinv + (size_t)r * bn;
                for (int q = 0; q < bs; q++) {
                    double s = 0.0;
                    for (int j = 0; j < bs; j++) s += D[q * bs + j] * yt[r * bs + j];
                    ut[r * bs + q] = s + un[r * bs + q];
                }
            }
        }
        orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, ut, 1.0, ft);
        for (int i = 0; i < n; i++) u[i] = u[i] + 1.0 * ut[i];
    }
    free(ft);
    free(ut);
    free(yt);
    free(un);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Exact block ILU(0) with level-scheduled triangular solves (the device path's bilu_exact mode).
 * No reference routine computes it directly; it is the fixed point the reference's FGPBILU sweeps
 * and Jacobi triangular solves converge to, and every operation below is the one those routines
 * apply to the final values (par_bilu_setup.c:5459-5609, par_bilu_solve.c:2893-3000), so the
 * results equal the reference's bit for bit once its sweep and Jacobi counts exceed the levels.
 * ------------------------------------------------------------------------ */

/* Levels of the lower DAG (row r after every k of its L-row; lev_l) and of the upper DAG (row r
 * after every c of its U-row; lev_u).  Returns the number of lower levels; *nup gets the upper one. */
int orc_bilu_levels(int nb, const int *lia, const int *lja, const int *uia, const int *uja, int *lev_l,
                    int *lev_u, int *nup)
{
    int nl = 0, nu = 0;
    for (int r = 0; r < nb; r++) {
        int l = 0;
        for (int k = lia[r]; k < lia[r + 1]; k++)
            if (lev_l[lja[k]] + 1 > l) l = lev_l[lja[k]] + 1;
        lev_l[r] = l;
        if (l + 1 > nl) nl = l + 1;
    }
    for (int r = nb - 1; r >= 0; r--) {
        int l = 0;
        for (int k = uia[r]; k < uia[r + 1]; k++)
            if (lev_u[uja[k]] + 1 > l) l = lev_u[uja[k]] + 1;
        lev_u[r] = l;
        if (l + 1 > nu) nu = l + 1;
    }
    if (nup) *nup = nu;
    return nl;
}

/* C_rc = A_rc - sum_{lj in L-row r} L_r,lja[lj] U_lja[lj],col (U found in U-row k), the sweep's sum */
static void bilu_c_block(int r, int jj, int bs, const int *ja, const double *a, const int *lia, const int *lja,
                         const double *la, const int *uia, const int *uja, const double *ua, double *Cb)
{
    const int bn = bs * bs, col = ja[jj];
    double tmp[9];
    memcpy(Cb, a + (size_t)jj * bn, bn * sizeof(double));
    for (int lj = lia[r]; lj < lia[r + 1]; lj++) {
        const int k = lja[lj];
        for (int uj = uia[k]; uj < uia[k + 1]; uj++)
            if (uja[uj] == col) {
                blk_matmul(la + (size_t)lj * bn, ua + (size_t)uj * bn, tmp, bs);
                for (int q = 0; q < bn; q++) Cb[q] -= tmp[q];
                break;
            }
    }
}

/* Exact factors, rows in natural order (a topological order of the lower DAG): the row's L entries in
 * ascending column (each needs the L entries of smaller columns), then its diagonal, then its U entries. */
int orc_bilu_setup_exact(int nb, int bs, const int *ia, const int *ja, const double *a, const int *lia,
                         const int *lja, double *la, const int *uia, const int *uja, double *ua, double *dinv)
{
    const int bn = bs * bs;
    double C[9], d[9];
    for (int r = 0; r < nb; r++) {
        /* L entries by ascending column; pl = their position in L-row r (A's order) */
        int done = 0, nlr = lia[r + 1] - lia[r];
        int last = -1;
        while (done < nlr) {
            int best = -1, bestc = nb, pl = lia[r], bj = -1;
            for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
                if (ja[jj] < r) {
                    if (ja[jj] > last && ja[jj] < bestc) {
                        bestc = ja[jj];
                        best = pl;
                        bj = jj;
                    }
                    pl++;
                }
            }
            bilu_c_block(r, bj, bs, ja, a, lia, lja, la, uia, uja, ua, C);
            blk_matmul(C, dinv + (size_t)bestc * bn, la + (size_t)best * bn, bs);
            last = bestc;
            done++;
        }
        int pu = uia[r];
        for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
            if (ja[jj] == r) {
                bilu_c_block(r, jj, bs, ja, a, lia, lja, la, uia, uja, ua, C);
                diag_update(C, d, dinv + (size_t)r * bn, bs);
            }
        }
        for (int jj = ia[r]; jj < ia[r + 1]; jj++) {
            if (ja[jj] > r) {
                bilu_c_block(r, jj, bs, ja, a, lia, lja, la, uia, uja, ua, C);
                memcpy(ua + (size_t)(pu++) * bn, C, bn * sizeof(double));
            }
        }
    }
    return 0;
}

/* u += (I + L)(D + U) solved exactly, `ir_iters` refinement loops as the reference's: ftemp = f - A u;
 * each loop: y by forward substitution, y_r = -(sum_k L_rk y_k) + ftemp_r; t by backward substitution,
 * t_r = D_r^-1 y_r + D_r^-1 (-(sum_c U_rc t_c)); ftemp -= A t; u += t.  Sums in stored row order with
 * the reference BSR product's rounding sequence. */
int orc_bilu_solve_exact(int nb, int bs, const int *ia, const int *ja, const double *a, const int *lia,
                         const int *lja, const double *la, const int *uia, const int *uja, const double *ua,
                         const double *dinv, int ir_iters, const double *f, double *u)
{
    const int n = nb * bs, bn = bs * bs;
    double *ft = malloc(sizeof(double) * n), *yt = malloc(sizeof(double) * n), *ut = malloc(sizeof(double) * n);
    memcpy(ft, f, sizeof(double) * n);
    orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, u, 1.0, ft);
    for (int it = 0; it < ir_iters; it++) {
        for (int r = 0; r < nb; r++) {
            double s[3] = {0.0, 0.0, 0.0};
            for (int k = lia[r]; k < lia[r + 1]; k++)
                for (int q = 0; q < bs; q++) {
                    double t = s[q];
                    for (int m = 0; m < bs; m++) t += la[(size_t)k * bn + q * bs + m] * yt[lja[k] * bs + m];
                    s[q] = t;
                }
            for (int q = 0; q < bs; q++) yt[r * bs + q] = s[q] * -1.0 + ft[r * bs + q];
        }
        for (int r = nb - 1; r >= 0; r--) {
            double s[3] = {0.0, 0.0, 0.0}, un[3], tq[3];
            for (int k = uia[r]; k < uia[r + 1]; k++)
                for (int q = 0; q < bs; q++) {
                    double t = s[q];
                    for (int m = 0; m < bs; m++) t += ua[(size_t)k * bn + q * bs + m] * ut[uja[k] * bs + m];
                    s[q] = t;
                }
            for (int q = 0; q < bs; q++) un[q] = s[q] * -1.0;
            const double *D = dinv + (size_t)r * bn;
            for (int q = 0; q < bs; q++) {
                double v = 0.0;
                for (int m = 0; m < bs; m++) v += D[q * bs + m] * un[m];
                tq[q] = v;
            }
            for (int q = 0; q < bs; q++) {
                double v = 0.0;
                for (int m = 0; m < bs; m++) v += D[q * bs + m] * yt[r * bs + m];
                ut[r * bs + q] = v + tq[q];
            }
        }
        orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, ut, 1.0, ft);
        for (int i = 0; i < n; i++) u[i] = u[i] + 1.0 * ut[i];
    }
    free(ft);
    free(yt);
    free(ut);
    return 0;
}
