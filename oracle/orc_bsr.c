/*
 * ORACLE (test infrastructure only): plain-C restatement of the reference's
 * BSR kernels on the CPR-GMRES path.  Only tests/, the package's smoke check
 * and bench.py's CPU-baseline leg call this code, and only as a test oracle or
 * baseline; the product library never links it.
 *
 * Each function cites the reference lines it restates (paths relative to the
 * reference project root).  Arithmetic is written in the reference's order
 * and compiled with -ffp-contract=off so that results are bit-identical to
 * the reference library built from source (pinned by tests/test_oracle_pin.py).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* jxf_BSRMatrixMatvec, jxfpamg-0220/csrc/operation/mvops/seq_bsr_matvec.c:22-140 */
int orc_bsr_matvec(int nb, int bs, const int *ia, const int *ja, const double *a, double alpha, const double *x,
                   double beta, double *y)
{
    const int n = nb * bs, bnnz = bs * bs;
    if (alpha == 0.0) {
        for (int i = 0; i < n; i++) y[i] *= beta;
        return 0;
    }
    double temp = beta / alpha;
    if (temp != 1.0) {
        if (temp == 0.0) {
            for (int i = 0; i < n; i++) y[i] = 0.0;
        } else {
            for (int i = 0; i < n; i++) y[i] *= temp;
        }
    }
    for (int i = 0; i < nb; i++) {
        for (int jj = ia[i]; jj < ia[i + 1]; jj++) {
            for (int b1 = 0; b1 < bs; b1++) {
                double t = y[i * bs + b1];
                for (int b2 = 0; b2 < bs; b2++) t += a[(size_t)jj * bnnz + b1 * bs + b2] * x[ja[jj] * bs + b2];
                y[i * bs + b1] = t;
            }
        }
    }
    if (alpha != 1.0)
        for (int i = 0; i < n; i++) y[i] *= alpha;
    return 0;
}

/* ---- small dense helpers (jxfpamg-0220/csrc/cpr/jxf_bsr_decoup.c:47-345) ---- */

/* jxf_smat_inv_2x2, jxf_bsr_decoup.c:47-63: identity when |det| < 1e-15 */
static void inv2(double *a)
{
    const double a11 = a[0], a12 = a[1], a21 = a[2], a22 = a[3];
    const double det = a11 * a22 - a12 * a21;
    if (fabs(det) < 1e-15) {
        a[0] = 1.0; a[1] = 0.0; a[2] = 0.0; a[3] = 1.0;
    } else {
        double d = 1.0 / det;
        a[0] = a22 * d;
        a[1] = -a12 * d;
        a[2] = -a21 * d;
        a[3] = a11 * d;
    }
}

/* jxf_smat_inv_3x3, jxf_bsr_decoup.c:65-101 (cofactors) */
static void inv3(double *a)
{
    const double a11 = a[0], a12 = a[1], a13 = a[2];
    const double a21 = a[3], a22 = a[4], a23 = a[5];
    const double a31 = a[6], a32 = a[7], a33 = a[8];
    const double M11 = a22 * a33 - a23 * a32, M12 = a21 * a33 - a23 * a31, M13 = a21 * a32 - a22 * a31;
    const double M21 = a12 * a33 - a13 * a32, M22 = a11 * a33 - a13 * a31, M23 = a11 * a32 - a12 * a31;
    const double M31 = a12 * a23 - a13 * a22, M32 = a11 * a23 - a13 * a21, M33 = a11 * a22 - a12 * a21;
    const double det = a11 * M11 - a12 * M12 + a13 * M13;
    if (fabs(det) < 1e-15) {
        for (int i = 0; i < 9; i++) a[i] = 0.0;
        a[0] = a[4] = a[8] = 1.0;
    } else {
        double d = 1.0 / det;
        a[0] = M11 * d; a[1] = -M21 * d; a[2] = M31 * d;
        a[3] = -M12 * d; a[4] = M22 * d; a[5] = -M32 * d;
        a[6] = M13 * d; a[7] = -M23 * d; a[8] = M33 * d;
    }
}

/*
 * ABF: D_i = inv(A_ii); every block of row i becomes D_i A_ij (the diagonal
 * block becomes I) and b_i becomes D_i b_i computed IN PLACE, i.e. the
 * reference's matrix-vector helper is called with its input and output
 * aliased (jxf_bsr_decoup.c:404-408 for 2x2 via jxf_smat_vec_mul_2 :335-338;
 * :496-498 for 3x3 via jxf_smat_vec_mul :316-323).  Later rows of the
 * product therefore read already-updated entries; this is reproduced here
 * so that the decoupled right-hand side matches the reference bit for bit.
 * (With `consistent_rhs` the product is formed from a copy instead.)
 */
static void abf(int nb, int bs, const int *ia, double *a, double *rhs, int consistent_rhs)
{
    const int b2 = bs * bs;
    for (int i = 0; i < nb; i++) {
        double binv[9], sm[9];
        double *dblk = a + (size_t)ia[i] * b2;
        memcpy(binv, dblk, sizeof(double) * b2);
        if (bs == 2) inv2(binv); else inv3(binv);
        for (int j = ia[i]; j < ia[i + 1]; j++) {
            double *blk = a + (size_t)j * b2;
            if (j == ia[i]) {
                for (int k = 0; k < b2; k++) blk[k] = 0.0;
                for (int k = 0; k < bs; k++) blk[k * bs + k] = 1.0;
            } else if (bs == 2) {
                /* jxf_smat_mul_2x2, :300-305 */
                sm[0] = binv[0] * blk[0] + binv[1] * blk[2];
                sm[1] = binv[0] * blk[1] + binv[1] * blk[3];
                sm[2] = binv[2] * blk[0] + binv[3] * blk[2];
                sm[3] = binv[2] * blk[1] + binv[3] * blk[3];
                memcpy(blk, sm, sizeof(double) * 4);
            } else {
                /* jxf_smat_mul, :288-298: C = 0; C += A_ik B_kj */
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) {
                        double t = 0.0;
                        for (int k = 0; k < 3; k++) t += binv[r * 3 + k] * blk[k * 3 + c];
                        sm[r * 3 + c] = t;
                    }
                memcpy(blk, sm, sizeof(double) * 9);
            }
        }
        double *r = rhs + (size_t)i * bs;
        if (consistent_rhs) {
            double o[3] = {0, 0, 0}, v[3];
            memcpy(v, r, sizeof(double) * bs);
            for (int p = 0; p < bs; p++) {
                double t = 0.0;
                for (int k = 0; k < bs; k++) t += binv[p * bs + k] * v[k];
                o[p] = t;
            }
            memcpy(r, o, sizeof(double) * bs);
        } else if (bs == 2) {
            r[0] = binv[0] * r[0] + binv[1] * r[1];
            r[1] = binv[2] * r[0] + binv[3] * r[1];
        } else {
            for (int p = 0; p < 3; p++) {
                r[p] = 0.0;
                for (int k = 0; k < 3; k++) r[p] += binv[p * 3 + k] * r[k];
            }
        }
    }
}

/*
 * True-IMPES: column-sum blocks Ac_c = sum over rows of A_ic (accumulated in
 * row order), per-row weights from Ac_i, then the pressure row of every block
 * in row i is replaced by a weighted sum of the equation rows.
 * 2x2: jxf_bsr_decoup.c:721-802, c_i = -Ac12/Ac22 (0 if det or Ac22 < 1e-15).
 * 3x3: :911-996, weights (c0, c1) = first row of inv(Ac_i); the rhs uses all
 * three entries of that row (:986-993) while the matrix uses two.
 */
static void timpes(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs)
{
    const int b2 = bs * bs;
    double *Ac = (double *)calloc((size_t)nb * b2 + 1, sizeof(double));
    for (int i = 0; i < nb; i++)
        for (int j = ia[i]; j < ia[i + 1]; j++)
            for (int k = 0; k < b2; k++) Ac[(size_t)ja[j] * b2 + k] += a[(size_t)j * b2 + k];
    if (bs == 2) {
        for (int i = 0; i < nb; i++) {
            const double *ac = Ac + (size_t)i * 4;
            double det = ac[0] * ac[3] - ac[1] * ac[2];
            double c = 0.0;
            if (!(fabs(det) < 1e-15) && fabs(ac[3]) > 1e-15) c = -ac[1] / ac[3];
            for (int j = ia[i]; j < ia[i + 1]; j++) {
                double *blk = a + (size_t)j * 4;
                blk[0] = blk[0] + c * blk[2];
                blk[1] = blk[1] + c * blk[3];
            }
            rhs[i * 2] = rhs[i * 2] + c * rhs[i * 2 + 1];
        }
    } else {
        for (int i = 0; i < nb; i++) {
            double binv[9];
            memcpy(binv, Ac + (size_t)i * 9, sizeof(binv));
            inv3(binv);
            double c0 = binv[0], c1 = binv[1];
            for (int j = ia[i]; j < ia[i + 1]; j++) {
                double *blk = a + (size_t)j * 9;
                double n0 = c0 * blk[0] + c1 * blk[3];
                double n1 = c0 * blk[1] + c1 * blk[4];
                double n2 = c0 * blk[2] + c1 * blk[5];
                blk[0] = n0; blk[1] = n1; blk[2] = n2;
            }
            double *r = rhs + (size_t)i * 3;
            rhs[i * 3] = binv[0] * r[0] + binv[1] * r[1] + binv[2] * r[2];
        }
    }
    free(Ac);
}

/*
 * Row-transform decouplings: one bs x bs matrix M_i per block row, built from
 * the row's diagonal block (the first block), applied to every block of the
 * row (C = M_i B with C = 0; C += M_ik B_kj, jxf_smat_mul :288-298) and to b_i
 * by the reference's generic matrix-vector helper called with input and
 * output aliased (jxf_smat_vec_mul :306-314: c_p = 0, then c_p += M_pk b_k
 * reading already-overwritten entries; with `consistent_rhs` the product is
 * formed from a copy).
 *   ANL (type 2, :529-588): M = I, first row [1, -d_01, ..., -d_0,n-1].
 *   SEM (type 3, :591-654): M = inv(D_i) (jxf_smat_inv_nc: the 2x2 / 3x3
 *       cofactor inverses) with its first row replaced as in ANL.
 *   QI  (type 4, :657-714): M = I, first row [1, -d_01/d_11, ..., -d_0l/d_ll].
 * Thermal mode (the last unknown is temperature) changes the first row only in
 * columns 1..n-2 and the last row likewise (SEM also sets M_0,n-1 = M_n-1,0 = 0
 * and M_n-1,n-1 = 1).
 */
static void row_matrix(int type, int bs, int thermal, const double *d, double *M)
{
    const int b2 = bs * bs;
    if (type == 3) {
        memcpy(M, d, sizeof(double) * b2);
        if (bs == 2) inv2(M); else inv3(M);
        if (thermal) {
            M[0] = 1.0;
            M[bs - 1] = 0.0;
            M[(bs - 1) * bs] = 0.0;
            M[b2 - 1] = 1.0;
            for (int l = 0; l < bs - 2; l++) {
                M[1 + l] = -d[1 + l];
                M[(bs - 1) * bs + 1 + l] = -d[(bs - 1) * bs + 1 + l];
            }
        } else {
            M[0] = 1.0;
            for (int l = 0; l < bs - 1; l++) M[1 + l] = -d[1 + l];
        }
        return;
    }
    for (int r = 0; r < bs; r++)
        for (int c = 0; c < bs; c++) M[r * bs + c] = (r == c) ? 1.0 : 0.0;
    const int nl = thermal ? bs - 2 : bs - 1;
    for (int l = 0; l < nl; l++) {
        if (type == 2) {
            M[1 + l] = -d[1 + l];
            if (thermal) M[(bs - 1) * bs + 1 + l] = -d[(bs - 1) * bs + 1 + l];
        } else {
            M[1 + l] = -d[1 + l] / d[(l + 1) * bs + l + 1];
            if (thermal) M[(bs - 1) * bs + 1 + l] = -d[(bs - 1) * bs + 1 + l] / d[(l + 1) * bs + l + 1];
        }
    }
}

static void row_transform(int nb, int bs, int type, int thermal, const int *ia, double *a, double *rhs,
                          int consistent_rhs)
{
    const int b2 = bs * bs;
    for (int i = 0; i < nb; i++) {
        double M[9], sm[9];
        row_matrix(type, bs, thermal, a + (size_t)ia[i] * b2, M);
        for (int j = ia[i]; j < ia[i + 1]; j++) {
            double *blk = a + (size_t)j * b2;
            for (int r = 0; r < bs; r++)
                for (int c = 0; c < bs; c++) {
                    double t = 0.0;
                    for (int k = 0; k < bs; k++) t += M[r * bs + k] * blk[k * bs + c];
                    sm[r * bs + c] = t;
                }
            memcpy(blk, sm, sizeof(double) * b2);
        }
        double *r = rhs + (size_t)i * bs;
        if (consistent_rhs) {
            double v[3], o[3];
            memcpy(v, r, sizeof(double) * bs);
            for (int p = 0; p < bs; p++) {
                double t = 0.0;
                for (int k = 0; k < bs; k++) t += M[p * bs + k] * v[k];
                o[p] = t;
            }
            memcpy(r, o, sizeof(double) * bs);
        } else {
            for (int p = 0; p < bs; p++) {
                r[p] = 0.0;
                for (int k = 0; k < bs; k++) r[p] += M[p * bs + k] * r[k];
            }
        }
    }
}

/*
 * True-IMPES, second form (type 6, jxf_bsr_decoup.c:1102-1267): column-sum
 * blocks Ac as for type 5, then the pressure row of every block in row i
 * becomes row0 + c row1 (2x2, c = -Ac01/Ac11, 0 when |det Ac_i| < 1e-15) or
 * row0 + c0 row1 + c1 row2 with (c0, c1) = the first two entries of
 * inv(Ac_i) (3x3); b_i gets the same row operation.
 */
static void timpes2(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs)
{
    const int b2 = bs * bs;
    double *Ac = (double *)calloc((size_t)nb * b2 + 1, sizeof(double));
    for (int i = 0; i < nb; i++)
        for (int j = ia[i]; j < ia[i + 1]; j++)
            for (int k = 0; k < b2; k++) Ac[(size_t)ja[j] * b2 + k] += a[(size_t)j * b2 + k];
    for (int i = 0; i < nb; i++) {
        const double *ac = Ac + (size_t)i * b2;
        if (bs == 2) {
            const double det = ac[0] * ac[3] - ac[1] * ac[2];
            const double c = fabs(det) < 1e-15 ? 0.0 : -ac[1] / ac[3];
            for (int j = ia[i]; j < ia[i + 1]; j++) {
                double *blk = a + (size_t)j * 4;
                blk[0] = blk[0] + c * blk[2];
                blk[1] = blk[1] + c * blk[3];
            }
            rhs[i * 2] = rhs[i * 2] + c * rhs[i * 2 + 1];
        } else {
            double binv[9];
            memcpy(binv, ac, sizeof(binv));
            inv3(binv);
            const double c0 = binv[0], c1 = binv[1];
            for (int j = ia[i]; j < ia[i + 1]; j++) {
                double *blk = a + (size_t)j * 9;
                blk[0] = blk[0] + c0 * blk[3] + c1 * blk[6];
                blk[1] = blk[1] + c0 * blk[4] + c1 * blk[7];
                blk[2] = blk[2] + c0 * blk[5] + c1 * blk[8];
            }
            rhs[i * 3] = rhs[i * 3] + c0 * rhs[i * 3 + 1] + c1 * rhs[i * 3 + 2];
        }
    }
    free(Ac);
}

/* jxf_BSRMatrixDecouple, jxf_bsr_decoup.c:1273-1348 (types: 0 none, 1 ABF, 2 ANL, 3 SEM, 4 QI,
 * 5 TIMPES, 6 TIMPES2; thermal applies to 2-4) */
int orc_bsr_decouple2(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type,
                      int thermal, int consistent_rhs)
{
    if (bs != 2 && bs != 3) return 4;
    switch (type) {
        case 0: return 0;
        case 1: abf(nb, bs, ia, a, rhs, consistent_rhs); return 0;
        case 2:
        case 3:
        case 4: row_transform(nb, bs, type, thermal, ia, a, rhs, consistent_rhs); return 0;
        case 5: timpes(nb, bs, ia, ja, a, rhs); return 0;
        case 6: timpes2(nb, bs, ia, ja, a, rhs); return 0;
        default: return 4;
    }
}

int orc_bsr_decouple(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type,
                     int consistent_rhs)
{
    return orc_bsr_decouple2(nb, bs, ia, ja, a, rhs, type, 0, consistent_rhs);
}

/* jxf_RestrictPressureVector, jxfpamg-0220/csrc/cpr/jxf_cpr.c:74-100 */
void orc_restrict(int nb, int bs, int p, const double *r, double *rp)
{
    for (int i = 0; i < nb; i++) rp[i] = r[i * bs + p];
}

/* jxf_ProlongatePressureVector type 0, jxf_cpr.c:127-133 */
void orc_prolong(int nb, int bs, int p, const double *xp, double *x)
{
    for (int i = 0; i < nb; i++)
        for (int j = 0; j < bs; j++) x[i * bs + j] = (j == p) ? xp[i] : 0.0;
}

/* jxf_BSRMatrixGetSubmatrix, jxfpamg-0220/csrc/mat_vec_data/seq_bsr_matrix.c:214-251:
 * CSR with the block pattern, value = block[p][p] (stored zeros kept). */
void orc_bsr_submatrix(int nb, int bs, const int *ia, const int *ja, const double *a, int p, int *cia, int *cja,
                       double *ca)
{
    for (int i = 0; i <= nb; i++) cia[i] = ia[i];
    for (int k = 0; k < ia[nb]; k++) {
        cja[k] = ja[k];
        ca[k] = a[(size_t)k * bs * bs + p * bs + p];
    }
}
