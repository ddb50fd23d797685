/*
 * ORACLE (test infrastructure only): plain-C restatement of the reference's
 * pressure AMG as CPR configures it (jxfpamg-0220/csrc/cpr/jxf_cpr.c:319-377):
 * classical strength (theta 0.25, max_row_sum 0.9), HMIS coarsening (Ruge
 * first pass + PMIS), extended+i interpolation without truncation,
 * A_c = P^T A P, levels until n_c <= 1000 or 25 levels; the V(1,1) cycle with
 * hybrid symmetric Gauss-Seidel (two full SGS sweeps per pre/post step at
 * one rank and one thread) and Gaussian elimination on the coarsest level.
 *
 * Used only by tests/ and bench.py's CPU-baseline leg as the test oracle; the
 * product library never links it.  Sequential C, -ffp-contract=off.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define C_PT 1
#define F_PT -1
#define Z_PT -2
#define SF_PT -3

static void *xcalloc(size_t n, size_t s)
{
    void *p = calloc(n ? n : 1, s ? s : 1);
    if (!p) {
        fprintf(stderr, "oracle: out of memory\n");
        abort();
    }
    return p;
}

void orc_csr_free(orc_csr *A)
{
    if (!A) return;
    free(A->ia);
    free(A->ja);
    free(A->a);
    memset(A, 0, sizeof(*A));
}

static void csr_alloc(orc_csr *A, int n, int m, int nnz)
{
    A->n = n;
    A->m = m;
    A->ia = (int *)xcalloc(n + 1, sizeof(int));
    A->ja = (int *)xcalloc(nnz, sizeof(int));
    A->a = (double *)xcalloc(nnz, sizeof(double));
}

/* ---------------------------------------------------------------------------
 * Strength: jxf_PAMGCreateS, jxfpamg-0220/csrc/amg/par_strength.c:20-415
 * (num_functions = 1, one rank).  S keeps A's column order minus the
 * diagonal; values unused.
 * ------------------------------------------------------------------------ */
void orc_strength(const orc_csr *A, double theta, double max_row_sum, orc_csr *S)
{
    int n = A->n;
    int nnzA = A->ia[n];
    int *mark = (int *)xcalloc(nnzA, sizeof(int));
    for (int i = 0; i < n; i++) {
        int d = A->ia[i];
        double diag = A->a[d];
        double row_scale = 0.0, row_sum = diag;
        if (diag < 0) {
            for (int k = d + 1; k < A->ia[i + 1]; k++) {
                row_scale = row_scale < A->a[k] ? A->a[k] : row_scale; /* jxf_max */
                row_sum += A->a[k];
            }
        } else {
            for (int k = d + 1; k < A->ia[i + 1]; k++) {
                row_scale = row_scale < A->a[k] ? row_scale : A->a[k]; /* jxf_min(a,b) = a<b?a:b */
                row_sum += A->a[k];
            }
        }
        row_sum = fabs(row_sum / diag);
        mark[d] = 0;
        if ((row_sum > max_row_sum) && (max_row_sum < 1.0)) {
            for (int k = d + 1; k < A->ia[i + 1]; k++) mark[k] = 0;
        } else if (diag < 0) {
            for (int k = d + 1; k < A->ia[i + 1]; k++) mark[k] = !(A->a[k] <= theta * row_scale);
        } else {
            for (int k = d + 1; k < A->ia[i + 1]; k++) mark[k] = !(A->a[k] >= theta * row_scale);
        }
    }
    int cnt = 0;
    for (int k = 0; k < nnzA; k++) cnt += mark[k];
    csr_alloc(S, n, A->m, cnt);
    int p = 0;
    for (int i = 0; i < n; i++) {
        S->ia[i] = p;
        for (int k = A->ia[i]; k < A->ia[i + 1]; k++)
            if (mark[k]) S->ja[p++] = A->ja[k];
    }
    S->ia[n] = p;
    free(mark);
}

/* ---------------------------------------------------------------------------
 * Ruge-Stueben first pass (coarsen_type 10 -> 11 with f_pnt = Z_PT),
 * jxfpamg-0220/csrc/amg/par_coarsen_ruge.c:26-420 with the bucket lists of
 * amg_linklist.c: buckets by measure, highest first; a point enters at the
 * tail of its bucket and the head of the highest bucket is taken next.
 * ------------------------------------------------------------------------ */
typedef struct {
    int *next, *prev;     /* per point, -1 terminated */
    int *bhead, *btail;   /* per measure bucket */
    int maxm, cap;
} buckets;

static void bk_enter(buckets *B, int m, int i)
{
    B->next[i] = -1;
    B->prev[i] = B->btail[m];
    if (B->btail[m] >= 0) B->next[B->btail[m]] = i; else B->bhead[m] = i;
    B->btail[m] = i;
    if (m > B->maxm) B->maxm = m;
}

static void bk_remove(buckets *B, int m, int i)
{
    if (B->prev[i] >= 0) B->next[B->prev[i]] = B->next[i]; else B->bhead[m] = B->next[i];
    if (B->next[i] >= 0) B->prev[B->next[i]] = B->prev[i]; else B->btail[m] = B->prev[i];
    while (B->maxm > 0 && B->bhead[B->maxm] < 0) B->maxm--;
}

/* gia (optional): row offsets of the whole strength pattern when S is the
 * diagonal block of a row range; SF_PT only when that row is empty
 * (par_coarsen_ruge.c:261 tests the diagonal and the off-diagonal block). */
static void rs_first_pass_core(const orc_csr *S, const int *gia, int *CF)
{
    int n = S->n;
    int nnz = S->ia[n];
    int *STi = (int *)xcalloc(n + 1, sizeof(int)), *STj = (int *)xcalloc(nnz, sizeof(int));
    for (int k = 0; k < nnz; k++) STi[S->ja[k] + 1]++;
    for (int i = 0; i < n; i++) STi[i + 1] += STi[i];
    {
        int *pos = (int *)xcalloc(n, sizeof(int));
        for (int i = 0; i < n; i++) pos[i] = STi[i];
        for (int i = 0; i < n; i++)
            for (int k = S->ia[i]; k < S->ia[i + 1]; k++) STj[pos[S->ja[k]]++] = i;
        free(pos);
    }
    int *measure = (int *)xcalloc(n, sizeof(int));
    int maxmeasure = 0;
    for (int i = 0; i < n; i++) {
        measure[i] = STi[i + 1] - STi[i];
        if (measure[i] > maxmeasure) maxmeasure = measure[i];
    }
    buckets B;
    B.cap = maxmeasure + n + 2;
    B.next = (int *)xcalloc(n, sizeof(int));
    B.prev = (int *)xcalloc(n, sizeof(int));
    B.bhead = (int *)malloc(sizeof(int) * B.cap);
    B.btail = (int *)malloc(sizeof(int) * B.cap);
    for (int m = 0; m < B.cap; m++) B.bhead[m] = B.btail[m] = -1;
    B.maxm = 0;
    const int UNDEC = 0;
    int num_left = 0;
    const int *rows = gia ? gia : S->ia;
    for (int j = 0; j < n; j++) {
        if (rows[j + 1] - rows[j] == 0) {
            CF[j] = SF_PT;
            measure[j] = 0;
        } else {
            CF[j] = UNDEC;
            num_left++;
        }
    }
    for (int j = 0; j < n; j++) {
        int m = measure[j];
        if (CF[j] != SF_PT) {
            if (m > 0) {
                bk_enter(&B, m, j);
            } else {
                CF[j] = Z_PT;
                for (int k = S->ia[j]; k < S->ia[j + 1]; k++) {
                    int nb = S->ja[k];
                    if (CF[nb] != SF_PT) {
                        if (nb < j) {
                            int nm = measure[nb];
                            if (nm > 0) bk_remove(&B, nm, nb);
                            nm = ++measure[nb];
                            bk_enter(&B, nm, nb);
                        } else {
                            ++measure[nb];
                        }
                    }
                }
                --num_left;
            }
        }
    }
    while (num_left > 0) {
        int index = B.bhead[B.maxm];
        CF[index] = C_PT;
        int m = measure[index];
        measure[index] = 0;
        --num_left;
        bk_remove(&B, m, index);
        for (int k = STi[index]; k < STi[index + 1]; k++) {
            int nb = STj[k];
            if (CF[nb] == UNDEC) {
                CF[nb] = F_PT;
                bk_remove(&B, measure[nb], nb);
                --num_left;
                for (int q = S->ia[nb]; q < S->ia[nb + 1]; q++) {
                    int n2 = S->ja[q];
                    if (CF[n2] == UNDEC) {
                        bk_remove(&B, measure[n2], n2);
                        int nm = ++measure[n2];
                        bk_enter(&B, nm, n2);
                    }
                }
            }
        }
        for (int k = S->ia[index]; k < S->ia[index + 1]; k++) {
            int nb = S->ja[k];
            if (CF[nb] == UNDEC) {
                int mm = measure[nb];
                bk_remove(&B, mm, nb);
                measure[nb] = --mm;
                if (mm > 0) {
                    bk_enter(&B, mm, nb);
                } else {
                    CF[nb] = F_PT;
                    --num_left;
                    for (int q = S->ia[nb]; q < S->ia[nb + 1]; q++) {
                        int n2 = S->ja[q];
                        if (CF[n2] == UNDEC) {
                            bk_remove(&B, measure[n2], n2);
                            int nm = ++measure[n2];
                            bk_enter(&B, nm, n2);
                        }
                    }
                }
            }
        }
    }
    free(B.next); free(B.prev); free(B.bhead); free(B.btail);
    free(measure); free(STi); free(STj);
}

void orc_rs_first_pass(const orc_csr *S, int *CF)
{
    rs_first_pass_core(S, NULL, CF);
}

/* The first pass on n / range_rows row ranges (range r: rows n*r/nr to
 * n*(r+1)/nr), each on the diagonal block of S for its rows -- what every
 * process of a distributed run does (par_coarsen_ruge.c:37-44 take S_diag,
 * :197 sets the measures from its transpose, :212 adds no off-process
 * measures for the HMIS first pass, coarsen_type 11, and the pass,
 * :250-425, walks S_diag only).  range_rows <= 0 or fewer than two ranges:
 * the whole pattern. */
void orc_rs_first_pass_ranges(const orc_csr *S, int range_rows, int *CF)
{
    int n = S->n;
    int nr = range_rows > 0 ? n / range_rows : 1;
    if (nr < 1) nr = 1;
    for (int r = 0; r < nr; r++) {
        int r0 = (int)((long long)n * r / nr), r1 = (int)((long long)n * (r + 1) / nr), m = r1 - r0;
        orc_csr L;
        L.n = L.m = m;
        L.a = NULL;
        L.ia = (int *)xcalloc(m + 1, sizeof(int));
        L.ja = (int *)xcalloc(S->ia[r1] - S->ia[r0] + 1, sizeof(int));
        int cnt = 0;
        for (int i = r0; i < r1; i++) {
            for (int k = S->ia[i]; k < S->ia[i + 1]; k++)
                if (S->ja[k] >= r0 && S->ja[k] < r1) L.ja[cnt++] = S->ja[k] - r0;
            L.ia[i - r0 + 1] = cnt;
        }
        rs_first_pass_core(&L, S->ia + r0, CF + r0);
        free(L.ia);
        free(L.ja);
    }
}

/* Park-Miller minimal standard generator (Park & Miller, CACM 1988), in the
 * Schrage form of jxfpamg-0220/csrc/utilities/random.c:10-56. */
double orc_park_miller(int *seed)
{
    const int a = 16807, m = 2147483647, q = 127773, r = 2836;
    int high = *seed / q, low = *seed % q;
    int test = a * low - r * high;
    *seed = test > 0 ? test : test + m;
    return (double)(*seed) / m;
}

/* ---------------------------------------------------------------------------
 * PMIS second phase with CF_init = 1, jxfpamg-0220/csrc/amg/par_coarsen_pmis.c
 * :27-719, measures = column counts of S plus a Park-Miller draw (seed 2747,
 * par_indepset.c:19-55), independent sets by par_indepset.c:62-170.
 * ------------------------------------------------------------------------ */
void orc_pmis(const orc_csr *S0, int *CF)
{
    int n = S0->n;
    int nnz = S0->ia[n];
    int *Sj = (int *)xcalloc(nnz, sizeof(int));
    memcpy(Sj, S0->ja, sizeof(int) * nnz);
    const int *Si = S0->ia;
    double *measure = (double *)xcalloc(n, sizeof(double));
    for (int k = 0; k < nnz; k++) measure[Sj[k]] += 1.0;
    int seed = 2747;
    for (int i = 0; i < n; i++) measure[i] += orc_park_miller(&seed);
    int *graph = (int *)xcalloc(n, sizeof(int));
    int gsize = 0;
    for (int i = 0; i < n; i++) {
        if (CF[i] == -1) CF[i] = 0;
        if (CF[i] == Z_PT) {
            if (measure[i] >= 1.0 || (Si[i + 1] - Si[i]) > 0) {
                CF[i] = 0;
                graph[gsize++] = i;
            } else {
                CF[i] = F_PT;
            }
        } else if (CF[i] == SF_PT) {
            measure[i] = 0;
        } else {
            graph[gsize++] = i;
        }
    }
    int iter = 0;
    while (1) {
        if (gsize == 0) break;
        if (iter) {
            /* independent set: par_indepset.c:62-170 */
            for (int ig = 0; ig < gsize; ig++) {
                int i = graph[ig];
                if (measure[i] > 1) CF[i] = 1;
            }
            for (int ig = 0; ig < gsize; ig++) {
                int i = graph[ig];
                if (measure[i] > 1) {
                    for (int k = Si[i]; k < Si[i + 1]; k++) {
                        int j = Sj[k];
                        if (j < 0) j = -j - 1;
                        if (measure[j] > 1) {
                            if (measure[i] > measure[j]) CF[j] = 0;
                            else if (measure[j] > measure[i]) CF[i] = 0;
                        }
                    }
                }
            }
        }
        iter++;
        for (int ig = 0; ig < gsize; ig++) {
            int i = graph[ig];
            if (measure[i] < 1.0) {
                CF[i] = F_PT;
                for (int k = Si[i]; k < Si[i + 1]; k++)
                    if (Sj[k] > -1) Sj[k] = -Sj[k] - 1;
            }
            if (CF[i] > 0) {
                CF[i] = C_PT;
                for (int k = Si[i]; k < Si[i + 1]; k++)
                    if (Sj[k] > -1) Sj[k] = -Sj[k] - 1;
            } else {
                for (int k = Si[i]; k < Si[i + 1]; k++) {
                    int j = Sj[k];
                    if (j < 0) j = -j - 1;
                    if (CF[j] > 0) CF[i] = F_PT;
                }
                if (CF[i] == F_PT)
                    for (int k = Si[i]; k < Si[i + 1]; k++)
                        if (Sj[k] > -1) Sj[k] = -Sj[k] - 1;
            }
        }
        for (int ig = 0; ig < gsize; ig++) {
            int i = graph[ig];
            if (CF[i] == 0) {
                for (int k = Si[i]; k < Si[i + 1]; k++) {
                    int j = Sj[k];
                    if (j < 0) j = -j - 1;
                    if (CF[j] != 0 && Sj[k] > -1) Sj[k] = -Sj[k] - 1;
                }
            }
        }
        for (int ig = 0; ig < gsize; ig++) {
            int i = graph[ig];
            if (CF[i] != 0) {
                measure[i] = 0;
                gsize--;
                graph[ig] = graph[gsize];
                graph[gsize] = i;
                ig--;
            }
        }
    }
    free(Sj);
    free(measure);
    free(graph);
}

void orc_hmis(const orc_csr *S, int *CF)
{
    orc_rs_first_pass(S, CF);
    orc_pmis(S, CF);
}

/* Strength pattern of a CSR operator into the caller's arrays (sia[n+1];
 * with sja == NULL only the entry count is returned). */
int orc_strength_csr(int n, const int *ia, const int *ja, const double *a, double theta, double max_row_sum,
                     int *sia, int *sja)
{
    orc_csr A, S;
    A.n = A.m = n;
    A.ia = (int *)ia;
    A.ja = (int *)ja;
    A.a = (double *)a;
    orc_strength(&A, theta, max_row_sum, &S);
    int nnz = S.ia[n];
    if (sia) memcpy(sia, S.ia, sizeof(int) * (n + 1));
    if (sja) memcpy(sja, S.ja, sizeof(int) * nnz);
    orc_csr_free(&S);
    return nnz;
}

/* The first pass (on row ranges when range_rows > 0) on a strength pattern. */
void orc_rs_first_pass_csr(int n, const int *sia, const int *sja, int range_rows, int *cf)
{
    orc_csr S;
    S.n = S.m = n;
    S.ia = (int *)sia;
    S.ja = (int *)sja;
    S.a = NULL;
    orc_rs_first_pass_ranges(&S, range_rows, cf);
}

/* HMIS with the first pass on row ranges, on a CSR operator: strength
 * (theta, max_row_sum) then orc_rs_first_pass_ranges and the PMIS pass. */
void orc_hmis_ranges(int n, const int *ia, const int *ja, const double *a, double theta, double max_row_sum,
                     int range_rows, int *CF)
{
    orc_csr A, S;
    A.n = A.m = n;
    A.ia = (int *)ia;
    A.ja = (int *)ja;
    A.a = (double *)a;
    orc_strength(&A, theta, max_row_sum, &S);
    orc_rs_first_pass_ranges(&S, range_rows, CF);
    orc_pmis(&S, CF);
    orc_csr_free(&S);
}

/* ---------------------------------------------------------------------------
 * Extended+i interpolation, jxfpamg-0220/csrc/amg/par_interp_6.c:19-790 (one
 * rank, no truncation).  Column order within a row is discovery order.
 * ------------------------------------------------------------------------ */
void orc_extpi_interp(const orc_csr *A, const orc_csr *S, const int *CF, orc_csr *P)
{
    int n = A->n;
    int *f2c = (int *)xcalloc(n, sizeof(int));
    int *Pm = (int *)xcalloc(n, sizeof(int));
    int nc = 0;
    for (int i = 0; i < n; i++) {
        Pm[i] = -1;
        f2c[i] = CF[i] >= 0 ? nc++ : -1;
    }
    int *Pi = (int *)xcalloc(n + 1, sizeof(int));
    int cnt = 0;
    for (int i = 0; i < n; i++) {
        Pi[i] = cnt;
        if (CF[i] >= 0) {
            cnt++;
        } else if (CF[i] != SF_PT) {
            for (int k = S->ia[i]; k < S->ia[i + 1]; k++) {
                int i1 = S->ja[k];
                if (CF[i1] >= 0) {
                    if (Pm[i1] < Pi[i]) Pm[i1] = cnt++;
                } else if (CF[i1] != SF_PT) {
                    for (int q = S->ia[i1]; q < S->ia[i1 + 1]; q++) {
                        int k1 = S->ja[q];
                        if (CF[k1] >= 0 && Pm[k1] < Pi[i]) Pm[k1] = cnt++;
                    }
                }
            }
        }
    }
    Pi[n] = cnt;
    csr_alloc(P, n, nc, cnt);
    memcpy(P->ia, Pi, sizeof(int) * (n + 1));
    free(Pi);
    for (int i = 0; i < n; i++) Pm[i] = -1;
    int jj = 0;
    int strong_f = -2;
    for (int i = 0; i < n; i++) {
        int jb = jj;
        if (CF[i] >= 0) {
            P->ja[jj] = f2c[i];
            P->a[jj] = 1.0;
            jj++;
        } else if (CF[i] != SF_PT) {
            strong_f--;
            for (int k = S->ia[i]; k < S->ia[i + 1]; k++) {
                int i1 = S->ja[k];
                if (CF[i1] >= 0) {
                    if (Pm[i1] < jb) {
                        Pm[i1] = jj;
                        P->ja[jj] = f2c[i1];
                        P->a[jj] = 0.0;
                        jj++;
                    }
                } else if (CF[i1] != SF_PT) {
                    Pm[i1] = strong_f;
                    for (int q = S->ia[i1]; q < S->ia[i1 + 1]; q++) {
                        int k1 = S->ja[q];
                        if (CF[k1] >= 0 && Pm[k1] < jb) {
                            Pm[k1] = jj;
                            P->ja[jj] = f2c[k1];
                            P->a[jj] = 0.0;
                            jj++;
                        }
                    }
                }
            }
            int je = jj;
            double diagonal = A->a[A->ia[i]];
            for (int k = A->ia[i] + 1; k < A->ia[i + 1]; k++) {
                int i1 = A->ja[k];
                if (Pm[i1] >= jb) {
                    P->a[Pm[i1]] += A->a[k];
                } else if (Pm[i1] == strong_f) {
                    double sum = 0.0;
                    int sgn = 1;
                    if (A->a[A->ia[i1]] < 0) sgn = -1;
                    for (int q = A->ia[i1] + 1; q < A->ia[i1 + 1]; q++) {
                        int i2 = A->ja[q];
                        if ((Pm[i2] >= jb || i2 == i) && (sgn * A->a[q]) < 0) sum += A->a[q];
                    }
                    if (sum != 0) {
                        double distribute = A->a[k] / sum;
                        for (int q = A->ia[i1] + 1; q < A->ia[i1 + 1]; q++) {
                            int i2 = A->ja[q];
                            if (Pm[i2] >= jb && (sgn * A->a[q]) < 0) P->a[Pm[i2]] += distribute * A->a[q];
                            if (i2 == i && (sgn * A->a[q]) < 0) diagonal += distribute * A->a[q];
                        }
                    } else {
                        diagonal += A->a[k];
                    }
                } else if (CF[i1] != SF_PT) {
                    diagonal += A->a[k];
                }
            }
            for (int q = jb; q < je; q++) P->a[q] /= -diagonal;
        }
        strong_f--;
    }
    free(f2c);
    free(Pm);
}

/* ---------------------------------------------------------------------------
 * Galerkin product A_c = P^T A P in the order of the reference's
 * jxf_PAMGBuildCoarseOperatorKT (jxfpamg-0220/csrc/operation/matops/
 * par_rap.c:185, one rank): R = P^T by a counting transpose (rows of R list
 * fine points ascending); for coarse row I the diagonal entry is placed first
 * (always present, starting from zero), then columns are appended in the
 * order they are first reached along R row I -> A row i -> P row j, and each
 * product (r*a)*p is added in that traversal order.
 * ------------------------------------------------------------------------ */
void orc_rap(const orc_csr *A, const orc_csr *P, orc_csr *Ac)
{
    int n = A->n, nc = P->m;
    int nnzP = P->ia[n];
    int *Ri = (int *)xcalloc(nc + 1, sizeof(int)), *Rj = (int *)xcalloc(nnzP, sizeof(int));
    double *Ra = (double *)xcalloc(nnzP, sizeof(double));
    for (int k = 0; k < nnzP; k++) Ri[P->ja[k] + 1]++;
    for (int c = 0; c < nc; c++) Ri[c + 1] += Ri[c];
    int *pos = (int *)xcalloc(nc + 1, sizeof(int));
    memcpy(pos, Ri, sizeof(int) * (nc + 1));
    for (int i = 0; i < n; i++)
        for (int k = P->ia[i]; k < P->ia[i + 1]; k++) {
            int c = P->ja[k];
            Rj[pos[c]] = i;
            Ra[pos[c]] = P->a[k];
            pos[c]++;
        }
    free(pos);
    int *slot = (int *)xcalloc(nc, sizeof(int)); /* column -> position in the current row */
    for (int c = 0; c < nc; c++) slot[c] = -1;
    int cap = 16 * nc + 16, cnt = 0;
    int *Ci = (int *)xcalloc(nc + 1, sizeof(int));
    int *Cj = (int *)malloc(sizeof(int) * cap);
    double *Ca = (double *)malloc(sizeof(double) * cap);
    for (int I = 0; I < nc; I++) {
        int row_begin = cnt;
        Ci[I] = cnt;
        if (cnt + 1 > cap) {
            cap *= 2;
            Cj = (int *)realloc(Cj, sizeof(int) * cap);
            Ca = (double *)realloc(Ca, sizeof(double) * cap);
        }
        slot[I] = cnt;
        Cj[cnt] = I;
        Ca[cnt] = 0.0;
        cnt++;
        for (int r = Ri[I]; r < Ri[I + 1]; r++) {
            int i = Rj[r];
            double pr = Ra[r];
            for (int k = A->ia[i]; k < A->ia[i + 1]; k++) {
                int j = A->ja[k];
                double pa = pr * A->a[k];
                for (int q = P->ia[j]; q < P->ia[j + 1]; q++) {
                    int J = P->ja[q];
                    if (slot[J] < row_begin) {
                        if (cnt + 1 > cap) {
                            cap *= 2;
                            Cj = (int *)realloc(Cj, sizeof(int) * cap);
                            Ca = (double *)realloc(Ca, sizeof(double) * cap);
                        }
                        slot[J] = cnt;
                        Cj[cnt] = J;
                        Ca[cnt] = pa * P->a[q];
                        cnt++;
                    } else {
                        Ca[slot[J]] += pa * P->a[q];
                    }
                }
            }
        }
    }
    Ci[nc] = cnt;
    Ac->n = nc;
    Ac->m = nc;
    Ac->ia = Ci;
    Ac->ja = Cj;
    Ac->a = Ca;
    free(slot); free(Ri); free(Rj); free(Ra);
}

/* ---------------------------------------------------------------------------
 * Hierarchy: jxf_PAMGSetup loop, jxfpamg-0220/csrc/amg/par_amg_setup.c:525-1240
 * ------------------------------------------------------------------------ */
void orc_amg_setup(const orc_csr *A0, int max_levels, int coarse_threshold, orc_amg *H)
{
    memset(H, 0, sizeof(*H));
    H->A[0] = *A0; /* borrowed */
    H->owns_A0 = 0;
    int level = 0;
    while (1) {
        orc_csr *A = &H->A[level];
        orc_csr S;
        orc_strength(A, 0.25, 0.9, &S);
        int *CF = (int *)xcalloc(A->n, sizeof(int));
        orc_hmis(&S, CF);
        H->CF[level] = CF;
        int nc = 0;
        for (int i = 0; i < A->n; i++) nc += CF[i] >= 0;
        orc_extpi_interp(A, &S, CF, &H->P[level]);
        orc_csr_free(&S);
        orc_rap(A, &H->P[level], &H->A[level + 1]);
        level++;
        if (level == max_levels - 1 || nc <= coarse_threshold) break;
    }
    H->num_levels = level + 1;
}

void orc_amg_free(orc_amg *H)
{
    for (int l = 0; l < H->num_levels; l++) {
        if (l > 0 || H->owns_A0) orc_csr_free(&H->A[l]);
        if (l < H->num_levels - 1) orc_csr_free(&H->P[l]);
        free(H->CF[l]);
    }
    memset(H, 0, sizeof(*H));
}

/* ---------------------------------------------------------------------------
 * V-cycle pieces
 * ------------------------------------------------------------------------ */

/* y = alpha*A*x + beta*y, jxfpamg-0220/csrc/operation/mvops/seq_csr_matvec.c:20 */
void orc_csr_matvec(const orc_csr *A, double alpha, const double *x, double beta, double *y)
{
    int n = A->n;
    if (alpha == 0.0) {
        for (int i = 0; i < n; i++) y[i] *= beta;
        return;
    }
    double t = beta / alpha;
    if (t != 1.0) {
        if (t == 0.0) for (int i = 0; i < n; i++) y[i] = 0.0;
        else for (int i = 0; i < n; i++) y[i] *= t;
    }
    for (int i = 0; i < n; i++) {
        double s = y[i];
        for (int k = A->ia[i]; k < A->ia[i + 1]; k++) s += A->a[k] * x[A->ja[k]];
        y[i] = s;
    }
    if (alpha != 1.0) for (int i = 0; i < n; i++) y[i] *= alpha;
}

/* y = alpha*A^T*x + beta*y, seq_csr_matvec.c:211 (one thread) */
void orc_csr_matvec_t(const orc_csr *A, double alpha, const double *x, double beta, double *y)
{
    int m = A->m;
    if (alpha == 0.0) {
        for (int i = 0; i < m; i++) y[i] *= beta;
        return;
    }
    double t = beta / alpha;
    if (t != 1.0) {
        if (t == 0.0) for (int i = 0; i < m; i++) y[i] = 0.0;
        else for (int i = 0; i < m; i++) y[i] *= t;
    }
    for (int i = 0; i < A->n; i++)
        for (int k = A->ia[i]; k < A->ia[i + 1]; k++) y[A->ja[k]] += A->a[k] * x[i];
    if (alpha != 1.0) for (int i = 0; i < m; i++) y[i] *= alpha;
}

/* One hybrid symmetric Gauss-Seidel application (relax_weight = omega = 1,
 * one rank, one thread): forward then backward sweep, points with a zero
 * diagonal skipped; jxfpamg-0220/csrc/operation/relaxations/par_relax_6.c:226-270 */
void orc_relax6(const orc_csr *A, const double *f, double *u)
{
    int n = A->n;
    for (int i = 0; i < n; i++) {
        int d = A->ia[i];
        if (A->a[d] != 0.0) {
            double res = f[i];
            for (int k = d + 1; k < A->ia[i + 1]; k++) res -= A->a[k] * u[A->ja[k]];
            u[i] = res / A->a[d];
        }
    }
    for (int i = n - 1; i > -1; i--) {
        int d = A->ia[i];
        if (A->a[d] != 0.0) {
            double res = f[i];
            for (int k = d + 1; k < A->ia[i + 1]; k++) res -= A->a[k] * u[A->ja[k]];
            u[i] = res / A->a[d];
        }
    }
}

/* Dense Gaussian elimination without pivoting on the coarsest level,
 * jxfpamg-0220/csrc/operation/matops/par_gs.c:20-74, matrix assembled by
 * par_relax_9.c:86-114. */
int orc_gselim(const orc_csr *A, const double *f, double *u)
{
    int n = A->n;
    double *M = (double *)xcalloc((size_t)n * n, sizeof(double));
    double *x = (double *)xcalloc(n, sizeof(double));
    for (int i = 0; i < n; i++) {
        for (int k = A->ia[i]; k < A->ia[i + 1]; k++) M[(size_t)i * n + A->ja[k]] = A->a[k];
        x[i] = f[i];
    }
    int err = 0;
    if (n == 1) {
        if (M[0] != 0.0) x[0] = x[0] / M[0]; else err = 1;
    } else {
        for (int k = 0; k < n - 1; k++) {
            if (M[(size_t)k * n + k] != 0.0) {
                for (int j = k + 1; j < n; j++) {
                    if (M[(size_t)j * n + k] != 0.0) {
                        double factor = M[(size_t)j * n + k] / M[(size_t)k * n + k];
                        for (int m = k + 1; m < n; m++) M[(size_t)j * n + m] -= factor * M[(size_t)k * n + m];
                        x[j] -= factor * x[k];
                    }
                }
            }
        }
        for (int k = n - 1; k > 0; --k) {
            x[k] /= M[(size_t)k * n + k];
            for (int j = 0; j < k; j++)
                if (M[(size_t)j * n + k] != 0.0) x[j] -= x[k] * M[(size_t)j * n + k];
        }
        x[0] /= M[0];
    }
    if (!err) memcpy(u, x, sizeof(double) * n);
    free(M);
    free(x);
    return err;
}

/* One V(1,1) cycle, jxfpamg-0220/csrc/amg/par_cycle.c:20-969 with
 * par_relax_if.c:22-76 (two SGS applications per pre/post sweep). */
void orc_amg_vcycle(const orc_amg *H, const double *f0, double *u0)
{
    int L = H->num_levels;
    double *F[ORC_MAX_LEVELS], *U[ORC_MAX_LEVELS];
    int nmax = H->A[0].n;
    double *vt = (double *)xcalloc(nmax, sizeof(double));
    F[0] = (double *)f0;
    U[0] = u0;
    for (int l = 1; l < L; l++) {
        F[l] = (double *)xcalloc(H->A[l].n, sizeof(double));
        U[l] = (double *)xcalloc(H->A[l].n, sizeof(double));
    }
    if (L == 1) {
        orc_relax6(&H->A[0], F[0], U[0]);
    } else {
        for (int l = 0; l < L - 1; l++) {
            orc_relax6(&H->A[l], F[l], U[l]);
            orc_relax6(&H->A[l], F[l], U[l]);
            for (int i = 0; i < H->A[l + 1].n; i++) U[l + 1][i] = 0.0;
            memcpy(vt, F[l], sizeof(double) * H->A[l].n);
            orc_csr_matvec(&H->A[l], -1.0, U[l], 1.0, vt);
            orc_csr_matvec_t(&H->P[l], 1.0, vt, 0.0, F[l + 1]);
        }
        orc_gselim(&H->A[L - 1], F[L - 1], U[L - 1]);
        for (int l = L - 2; l >= 0; l--) {
            orc_csr_matvec(&H->P[l], 1.0, U[l + 1], 1.0, U[l]);
            orc_relax6(&H->A[l], F[l], U[l]);
            orc_relax6(&H->A[l], F[l], U[l]);
        }
    }
    for (int l = 1; l < L; l++) {
        free(F[l]);
        free(U[l]);
    }
    free(vt);
}
