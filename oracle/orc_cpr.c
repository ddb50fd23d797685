/*
 * ORACLE (test infrastructure only): plain-C restatement of the CPR stage-2
 * block smoother, the CPR preconditioner and restarted GMRES of the reference
 * (one rank, one thread).  Only tests/ and bench.py's CPU-baseline leg use it.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* jxf_BSRMatrixBlockMatvec_Stable with beta = 1,
 * jxfpamg-0220/csrc/mat_vec_data/seq_bsr_matrix.c:841-872: per output row a
 * Kahan-compensated sum of the block row times v, then ov += alpha*sum. */
static void blk_matvec_stable(double alpha, const double *mat, const double *v, double *ov, int bs)
{
    double tmp[3];
    for (int j = 0; j < bs; j++) tmp[j] = ov[j] * 1.0;
    for (int i = 0; i < bs; i++) {
        double sum = 0.0, c = 0.0;
        for (int j = 0; j < bs; j++) {
            double y = mat[i * bs + j] * v[j] - c;
            double t = sum + y;
            c = (t - sum) - y;
            sum = t;
        }
        tmp[i] += alpha * sum;
        ov[i] = tmp[i];
    }
}

/* jxf_BSRMatrixBlockInvMatvec_Stable, seq_bsr_matrix.c:1054-1100 (2x2 closed
 * form with the conditioning guard) and jxf_BSRMatrixBlockInvMatvec_MixedPrec
 * :945-1051 (partially pivoted LU for 3x3). */
static void blk_inv_matvec(const double *mat, const double *v, double *ov, int bs)
{
    if (bs == 2) {
        double a11 = mat[0], a12 = mat[1], a21 = mat[2], a22 = mat[3];
        double det = a11 * a22 - a12 * a21;
        if (fabs(det) < 1e-12 * (fabs(a11 * a22) + fabs(a12 * a21))) {
            ov[0] = v[0] / (a11 + 1e-12);
            ov[1] = v[1] / (a22 + 1e-12);
            return;
        }
        double inv_det = 1.0 / det;
        double b1 = v[0], b2 = v[1];
        ov[0] = (a22 * b1 - a12 * b2) * inv_det;
        ov[1] = (-a21 * b1 + a11 * b2) * inv_det;
        return;
    }
    double m[9], x[3], o[3] = {0, 0, 0};
    int n = bs;
    memcpy(m, mat, sizeof(double) * 9);
    memcpy(x, v, sizeof(double) * 3);
    for (int i = 0; i < n; i++) {
        int mr = i;
        double mv = fabs(m[i * n + i]);
        for (int k = i + 1; k < n; k++)
            if (fabs(m[k * n + i]) > mv) {
                mv = fabs(m[k * n + i]);
                mr = k;
            }
        if (mv < 1e-15) {
            for (int j = 0; j < n; j++) {
                double d = m[j * n + j];
                o[j] = (fabs(d) > 1e-12) ? x[j] / d : 0.0;
            }
            break;
        }
        if (mr != i) {
            for (int j = 0; j < n; j++) {
                double t = m[i * n + j];
                m[i * n + j] = m[mr * n + j];
                m[mr * n + j] = t;
            }
            double t = x[i];
            x[i] = x[mr];
            x[mr] = t;
        }
        double pivot = m[i * n + i];
        for (int k = i + 1; k < n; k++) {
            double f = m[k * n + i] / pivot;
            m[k * n + i] = f;
            for (int j = i + 1; j < n; j++) m[k * n + j] -= f * m[i * n + j];
        }
    }
    /* forward and backward substitution always run (as in the reference),
       overwriting the diagonal-approximation values computed above */
    for (int i = 0; i < n; i++) {
        o[i] = x[i];
        for (int j = 0; j < i; j++) o[i] -= m[i * n + j] * o[j];
    }
    for (int i = n - 1; i >= 0; i--) {
        for (int j = i + 1; j < n; j++) o[i] -= m[i * n + j] * o[j];
        double d = m[i * n + i];
        if (fabs(d) > 1e-15) o[i] /= d; else o[i] = 0.0;
    }
    memcpy(ov, o, sizeof(double) * bs);
}

/* jxf_ParBSRHGSRelax, jxfpamg-0220/csrc/amg/par_relax_bsr.c:193-573, one rank,
 * one thread; direction 1 forward, -1 backward. */
void orc_hgs_relax(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                   double w, double omega, int direction)
{
    const int b2 = bs * bs;
    double *vt = (double *)malloc(sizeof(double) * (size_t)nb * bs + 8);
    memcpy(vt, x, sizeof(double) * (size_t)nb * bs);
    int begin = 0, end = nb, step = 1;
    if (direction == -1) {
        begin = nb - 1;
        end = -1;
        step = -1;
    }
    const double eps = 2.220446049250313e-16; /* DBL_EPSILON */
    if (fabs(w - 1) < eps && fabs(omega - 1) < eps) {
        for (int i = begin; i != end; i += step) {
            double res[3], out[3];
            for (int k = 0; k < bs; k++) res[k] = b[i * bs + k];
            for (int jj = ia[i] + 1; jj < ia[i + 1]; jj++)
                blk_matvec_stable(-1.0, a + (size_t)jj * b2, x + (size_t)ja[jj] * bs, res, bs);
            blk_inv_matvec(a + (size_t)ia[i] * b2, res, out, bs);
            for (int k = 0; k < bs; k++) x[i * bs + k] = out[k];
        }
    } else {
        double prod = 1.0 - w * omega, omo = 1.0 - omega;
        for (int i = begin; i != end; i += step) {
            double res[3], res0[3], res2[3], tmp[3], out[3];
            for (int k = 0; k < bs; k++) {
                res[k] = b[i * bs + k];
                res0[k] = 0.0;
                res2[k] = 0.0;
            }
            for (int jj = ia[i] + 1; jj < ia[i + 1]; jj++) {
                blk_matvec_stable(-1.0, a + (size_t)jj * b2, x + (size_t)ja[jj] * bs, res0, bs);
                blk_matvec_stable(1.0, a + (size_t)jj * b2, vt + (size_t)ja[jj] * bs, res2, bs);
            }
            for (int k = 0; k < bs; k++) tmp[k] = omega * res[k] + res0[k] + omo * res2[k];
            blk_inv_matvec(a + (size_t)ia[i] * b2, tmp, out, bs);
            for (int k = 0; k < bs; k++) {
                x[i * bs + k] *= prod;
                x[i * bs + k] += w * out[k];
            }
        }
    }
    free(vt);
}

/* Stage-2 chunk order of the throughput path (no reference counterpart; it reorders the natural
 * sweep of par_relax_bsr.c:193-573 for parallel slack): block rows in chunks of `chunk` consecutive
 * rows (chunk c = rows [c*chunk, (c+1)*chunk)), chunks coloured greedily in natural order with the
 * smallest colour that no chunk coupled to it (symmetrised pattern) has; colour[i] gets the colour of
 * row i's chunk.  Returns the number of colours.  The sweep visits colour 0's chunks, then colour
 * 1's, ..., chunks ascending, rows ascending inside a chunk. */
int orc_chunk_colour(int nb, const int *ia, const int *ja, int chunk, int *colour)
{
    int nc = (nb + chunk - 1) / chunk, ncol = 0;
    int *cc = (int *)malloc(sizeof(int) * (nc + 1)), *mark = NULL, nmark = 0;
    for (int c = 0; c < nc; c++) cc[c] = -1;
    /* coupling of chunk c: columns of its rows, and rows whose columns fall in it */
    int *ti = (int *)calloc(nb + 1, sizeof(int)), *tj = (int *)malloc(sizeof(int) * (ia[nb] + 1));
    for (int k = 0; k < ia[nb]; k++) ti[ja[k] + 1]++;
    for (int i = 0; i < nb; i++) ti[i + 1] += ti[i];
    int *pos = (int *)malloc(sizeof(int) * (nb + 1));
    memcpy(pos, ti, sizeof(int) * nb);
    for (int i = 0; i < nb; i++)
        for (int k = ia[i]; k < ia[i + 1]; k++) tj[pos[ja[k]]++] = i;
    for (int c = 0; c < nc; c++) {
        /* colours taken by coupled, already coloured chunks */
        int lo = c * chunk, hi = (c + 1) * chunk < nb ? (c + 1) * chunk : nb;
        for (int pass = 0; pass < 2; pass++)
            for (int i = lo; i < hi; i++) {
                const int *p0 = pass ? tj + ti[i] : ja + ia[i];
                const int *p1 = pass ? tj + ti[i + 1] : ja + ia[i + 1];
                for (const int *q = p0; q < p1; q++) {
                    int d = *q / chunk;
                    if (d != c && cc[d] >= 0) {
                        if (cc[d] >= nmark) {
                            int nm = 2 * cc[d] + 2;
                            mark = (int *)realloc(mark, sizeof(int) * nm);
                            for (int t = nmark; t < nm; t++) mark[t] = -1;
                            nmark = nm;
                        }
                        mark[cc[d]] = c;
                    }
                }
            }
        int col = 0;
        while (col < nmark && mark[col] == c) col++;
        cc[c] = col;
        if (col + 1 > ncol) ncol = col + 1;
    }
    for (int i = 0; i < nb; i++) colour[i] = cc[i / chunk];
    free(cc);
    free(mark);
    free(ti);
    free(tj);
    free(pos);
    return ncol;
}

/* One stage-2 sweep (the jxf_ParBSRHGSRelax update, par_relax_bsr.c:193-573) visiting the block
 * rows in the chunk order given by colour[] (orc_chunk_colour): x_i <- (1 - w omega) x_i +
 * w A_ii^-1 (omega b_i + res0 + (1 - omega) res2), res0 = -sum_j A_ij x_j (current values),
 * res2 = sum_j A_ij vt_j (values at the sweep start). */
void orc_hgs_relax_chunked(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                           double w, double omega, int chunk, const int *colour, int ncolour)
{
    const int b2 = bs * bs;
    double *vt = (double *)malloc(sizeof(double) * (size_t)nb * bs + 8);
    memcpy(vt, x, sizeof(double) * (size_t)nb * bs);
    const double prod = 1.0 - w * omega, omo = 1.0 - omega;
    int nc = (nb + chunk - 1) / chunk;
    for (int col = 0; col < ncolour; col++)
        for (int c = 0; c < nc; c++) {
            if (colour[c * chunk] != col) continue;
            int hi = (c + 1) * chunk < nb ? (c + 1) * chunk : nb;
            for (int i = c * chunk; i < hi; i++) {
                double res0[3] = {0, 0, 0}, res2[3] = {0, 0, 0}, tmp[3], out[3];
                for (int jj = ia[i] + 1; jj < ia[i + 1]; jj++) {
                    blk_matvec_stable(-1.0, a + (size_t)jj * b2, x + (size_t)ja[jj] * bs, res0, bs);
                    blk_matvec_stable(1.0, a + (size_t)jj * b2, vt + (size_t)ja[jj] * bs, res2, bs);
                }
                for (int k = 0; k < bs; k++) tmp[k] = omega * b[i * bs + k] + res0[k] + omo * res2[k];
                blk_inv_matvec(a + (size_t)ia[i] * b2, tmp, out, bs);
                for (int k = 0; k < bs; k++) x[i * bs + k] = prod * x[i * bs + k] + w * out[k];
            }
        }
    free(vt);
}

/* jxf_ParBSRHSGSRelax, jxfpamg-0220/csrc/amg/par_relax_bsr.c:579-1062, one
 * rank, one thread: a forward block Gauss-Seidel pass over the rows, then a
 * backward one, both reading the current iterate.  With w = omega = 1 each
 * point is x_i = A_ii^-1 (b_i - sum_j A_ij x_j); otherwise
 * x_i = (1 - w omega) x_i + w A_ii^-1 (omega b_i + res0 + (1 - omega) res2),
 * res0 = -sum_j A_ij x_j, res2 = sum_j A_ij Vtemp_j, where Vtemp is the
 * caller's work vector of which only the first nb entries (nb = block rows,
 * not nb*bs unknowns) are refreshed from x at the start (:865); the others
 * keep what the work vector held before. */
void orc_hsgs_relax(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                    double *work, double w, double omega)
{
    const int b2 = bs * bs;
    const double eps = 2.220446049250313e-16; /* DBL_EPSILON */
    const int plain = fabs(w - 1) < eps && fabs(omega - 1) < eps;
    const double prod = 1.0 - w * omega, omo = 1.0 - omega;
    if (!plain)
        for (int i = 0; i < nb; i++) work[i] = x[i];
    for (int pass = 0; pass < 2; pass++) {
        const int begin = pass == 0 ? 0 : nb - 1, end = pass == 0 ? nb : -1, step = pass == 0 ? 1 : -1;
        for (int i = begin; i != end; i += step) {
            double res[3], res0[3], res2[3], tmp[3], out[3];
            for (int k = 0; k < bs; k++) {
                res[k] = b[i * bs + k];
                res0[k] = 0.0;
                res2[k] = 0.0;
            }
            if (plain) {
                for (int jj = ia[i] + 1; jj < ia[i + 1]; jj++)
                    blk_matvec_stable(-1.0, a + (size_t)jj * b2, x + (size_t)ja[jj] * bs, res, bs);
                blk_inv_matvec(a + (size_t)ia[i] * b2, res, out, bs);
                for (int k = 0; k < bs; k++) x[i * bs + k] = out[k];
                continue;
            }
            for (int jj = ia[i] + 1; jj < ia[i + 1]; jj++) {
                blk_matvec_stable(-1.0, a + (size_t)jj * b2, x + (size_t)ja[jj] * bs, res0, bs);
                blk_matvec_stable(1.0, a + (size_t)jj * b2, work + (size_t)ja[jj] * bs, res2, bs);
            }
            for (int k = 0; k < bs; k++) tmp[k] = omega * res[k] + res0[k] + omo * res2[k];
            blk_inv_matvec(a + (size_t)ia[i] * b2, tmp, out, bs);
            for (int k = 0; k < bs; k++) {
                x[i * bs + k] *= prod;
                x[i * bs + k] += w * out[k];
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * CPR: setup (jxfpamg-0220/csrc/cpr/jxf_cpr.c:268-422) and apply (:424-610):
 * restrict -> one AMG V-cycle from zero -> prolong (overwrite) -> stage2_maxit
 * stage-2 sweeps (w = 0.7, omega = 0.9): forward HGS (stage2_type 2) or HSGS
 * (3, with the CPR's work vector, zero when created, :396).
 * ------------------------------------------------------------------------ */
void orc_cpr_setup(orc_cpr *C, int nb, int bs, const int *ia, const int *ja, const double *a, int stage2_maxit)
{
    memset(C, 0, sizeof(*C));
    C->nb = nb;
    C->bs = bs;
    C->ia = ia;
    C->ja = ja;
    C->a = a;
    C->stage2_maxit = stage2_maxit;
    C->stage2_type = 2;
    C->work = (double *)calloc((size_t)nb * bs + 1, sizeof(double));
    orc_csr *Ap = &C->Ap;
    Ap->n = nb;
    Ap->m = nb;
    Ap->ia = (int *)malloc(sizeof(int) * (nb + 1));
    Ap->ja = (int *)malloc(sizeof(int) * (ia[nb] + 1));
    Ap->a = (double *)malloc(sizeof(double) * (ia[nb] + 1));
    orc_bsr_submatrix(nb, bs, ia, ja, a, 0, Ap->ia, Ap->ja, Ap->a);
    orc_amg_setup(Ap, 25, 1000, &C->amg);
}

void orc_cpr_apply(const orc_cpr *C, const double *r, double *z)
{
    int nb = C->nb, bs = C->bs;
    double *rp = (double *)malloc(sizeof(double) * nb + 8), *xp = (double *)calloc(nb + 1, sizeof(double));
    orc_restrict(nb, bs, 0, r, rp);
    orc_amg_vcycle(&C->amg, rp, xp);
    orc_prolong(nb, bs, 0, xp, z);
    for (int s = 0; s < C->stage2_maxit; s++) {
        if (C->stage2_type == 3) orc_hsgs_relax(nb, bs, C->ia, C->ja, C->a, z, r, C->work, 0.7, 0.9);
        else if (C->stage2_chunk > 0)
            orc_hgs_relax_chunked(nb, bs, C->ia, C->ja, C->a, z, r, 0.7, 0.9, C->stage2_chunk, C->colour,
                                  C->ncolour);
        else orc_hgs_relax(nb, bs, C->ia, C->ja, C->a, z, r, 0.7, 0.9, 1);
    }
    free(rp);
    free(xp);
}

void orc_cpr_set_stage2_chunk(orc_cpr *C, int chunk)
{
    free(C->colour);
    C->colour = NULL;
    C->stage2_chunk = chunk;
    C->ncolour = 0;
    if (chunk > 0) {
        C->colour = (int *)malloc(sizeof(int) * (C->nb + 1));
        C->ncolour = orc_chunk_colour(C->nb, C->ia, C->ja, chunk, C->colour);
    }
}

void orc_cpr_free(orc_cpr *C)
{
    free(C->colour);
    C->colour = NULL;
    free(C->work);
    C->work = NULL;
    orc_amg_free(&C->amg);
    orc_csr_free(&C->Ap);
}

/* ---------------------------------------------------------------------------
 * Restarted right-preconditioned GMRES(k) with modified Gram-Schmidt and
 * Givens rotations, jxfpamg-0220/csrc/krylov/pgmres.c:950-1713 (rel_change 0,
 * cf_tol 0, min_iter 0, convfac_threshold 1e4, is_check_restarted 1).
 * precond == NULL means the identity.  Returns iterations; *rel = final
 * relative residual as the reference reports it; norms (optional) gets the
 * residual history.
 * ------------------------------------------------------------------------ */
static double dot(int n, const double *x, const double *y)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += y[i] * x[i];
    return s;
}
static void axpy(int n, double a, const double *x, double *y)
{
    for (int i = 0; i < n; i++) y[i] += a * x[i];
}
static void scal(int n, double a, double *x)
{
    for (int i = 0; i < n; i++) x[i] *= a;
}

int orc_gmres(int nb, int bs, const int *ia, const int *ja, const double *a, const double *b, double *x, int k_dim,
              double tol, int max_iter, const orc_cpr *precond, double *rel, int *converged, double *norms)
{
    int n = nb * bs;
    double **p = (double **)malloc(sizeof(double *) * (k_dim + 1));
    for (int i = 0; i <= k_dim; i++) p[i] = (double *)calloc(n + 1, sizeof(double));
    double *r = (double *)calloc(n + 1, sizeof(double)), *w = (double *)calloc(n + 1, sizeof(double));
    double *rs = (double *)calloc(k_dim + 1, sizeof(double)), *c = (double *)calloc(k_dim, sizeof(double));
    double *s = (double *)calloc(k_dim, sizeof(double));
    double **hh = (double **)malloc(sizeof(double *) * (k_dim + 1));
    for (int i = 0; i <= k_dim; i++) hh[i] = (double *)calloc(k_dim, sizeof(double));
    const double epsmac = 1.e-16, convfac_threshold = 1.0e4;
    *converged = 0;
    memcpy(p[0], b, sizeof(double) * n);
    orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, x, 1.0, p[0]);
    double b_norm = sqrt(dot(n, b, b));
    double r_norm = sqrt(dot(n, p[0], p[0]));
    double r_norm_0 = r_norm, normdown = r_norm, conv_factor = 0.0;
    if (norms) norms[0] = r_norm;
    double den = b_norm > 0.0 ? b_norm : r_norm;
    double epsilon = tol * den;
    if (epsilon < 0.0) epsilon = 0.0;
    int iter = 0, i = 0;
    while (iter < max_iter) {
        rs[0] = r_norm;
        if (r_norm == 0.0) break;
        if (r_norm <= epsilon) {
            memcpy(r, b, sizeof(double) * n);
            orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, x, 1.0, r);
            r_norm = sqrt(dot(n, r, r));
            if (r_norm <= epsilon) {
                *converged = 1;
                break;
            }
        }
        scal(n, 1.0 / r_norm, p[0]);
        i = 0;
        while (i < k_dim && iter < max_iter) {
            i++;
            iter++;
            memset(r, 0, sizeof(double) * n);
            if (precond) orc_cpr_apply(precond, p[i - 1], r); else memcpy(r, p[i - 1], sizeof(double) * n);
            orc_bsr_matvec(nb, bs, ia, ja, a, 1.0, r, 0.0, p[i]);
            for (int j = 0; j < i; j++) {
                hh[j][i - 1] = dot(n, p[j], p[i]);
                axpy(n, -hh[j][i - 1], p[j], p[i]);
            }
            double t = sqrt(dot(n, p[i], p[i]));
            hh[i][i - 1] = t;
            if (t != 0.0) scal(n, 1.0 / t, p[i]);
            for (int j = 1; j < i; j++) {
                t = hh[j - 1][i - 1];
                hh[j - 1][i - 1] = s[j - 1] * hh[j][i - 1] + c[j - 1] * t;
                hh[j][i - 1] = -s[j - 1] * t + c[j - 1] * hh[j][i - 1];
            }
            t = hh[i][i - 1] * hh[i][i - 1];
            t += hh[i - 1][i - 1] * hh[i - 1][i - 1];
            double gamma = sqrt(t);
            if (gamma == 0.0) gamma = epsmac;
            c[i - 1] = hh[i - 1][i - 1] / gamma;
            s[i - 1] = hh[i][i - 1] / gamma;
            rs[i] = -hh[i][i - 1] * rs[i - 1];
            rs[i] /= gamma;
            rs[i - 1] = c[i - 1] * rs[i - 1];
            hh[i - 1][i - 1] = s[i - 1] * hh[i][i - 1] + c[i - 1] * hh[i - 1][i - 1];
            r_norm = fabs(rs[i]);
            conv_factor = r_norm / normdown;
            normdown = r_norm;
            if (norms) norms[iter] = r_norm;
            if (iter > 1 && conv_factor > convfac_threshold) break;
            if (r_norm <= epsilon) break;
        }
        rs[i - 1] = rs[i - 1] / hh[i - 1][i - 1];
        for (int k = i - 2; k >= 0; k--) {
            double t = 0.0;
            for (int j = k + 1; j < i; j++) t -= hh[k][j] * rs[j];
            t += rs[k];
            rs[k] = t / hh[k][k];
        }
        memcpy(w, p[i - 1], sizeof(double) * n);
        scal(n, rs[i - 1], w);
        for (int j = i - 2; j >= 0; j--) axpy(n, rs[j], p[j], w);
        memset(r, 0, sizeof(double) * n);
        if (precond) orc_cpr_apply(precond, w, r); else memcpy(r, w, sizeof(double) * n);
        axpy(n, 1.0, r, x);
        if (r_norm <= epsilon) {
            memcpy(r, b, sizeof(double) * n);
            orc_bsr_matvec(nb, bs, ia, ja, a, -1.0, x, 1.0, r);
            r_norm = sqrt(dot(n, r, r));
            if (r_norm <= epsilon) {
                *converged = 1;
                break;
            }
            memcpy(p[0], r, sizeof(double) * n);
            i = 0;
        }
        if (iter > 1 && conv_factor > convfac_threshold) break;
        for (int j = i; j > 0; j--) {
            rs[j - 1] = -s[j - 1] * rs[j];
            rs[j] = c[j - 1] * rs[j];
        }
        if (i) axpy(n, rs[i] - 1.0, p[i], p[i]);
        for (int j = i - 1; j > 0; j--) axpy(n, rs[j], p[j], p[i]);
        if (i) {
            axpy(n, rs[0] - 1.0, p[0], p[0]);
            axpy(n, 1.0, p[i], p[0]);
        }
    }
    *rel = b_norm > 0.0 ? r_norm / b_norm : r_norm / r_norm_0;
    for (int q = 0; q <= k_dim; q++) {
        free(p[q]);
        free(hh[q]);
    }
    free(p); free(hh); free(r); free(w); free(rs); free(c); free(s);
    return iter;
}
