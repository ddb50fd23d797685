/*
 * ORACLE (test infrastructure only): handle-based plain-array entry points of
 * the restatement for the Python tests (ctypes).  Handles own deep copies of
 * the caller's arrays.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct {
    int nb, bs;
    int *ia, *ja;
    double *a;
    orc_cpr cpr;
} orc_cpr_handle;

void *orc_cpr_create(int nb, int bs, const int *ia, const int *ja, const double *a, int stage2_maxit)
{
    orc_cpr_handle *h = (orc_cpr_handle *)calloc(1, sizeof(orc_cpr_handle));
    int nnzb = ia[nb];
    h->nb = nb;
    h->bs = bs;
    h->ia = (int *)malloc(sizeof(int) * (nb + 1));
    h->ja = (int *)malloc(sizeof(int) * (nnzb + 1));
    h->a = (double *)malloc(sizeof(double) * ((size_t)nnzb * bs * bs + 1));
    memcpy(h->ia, ia, sizeof(int) * (nb + 1));
    memcpy(h->ja, ja, sizeof(int) * nnzb);
    memcpy(h->a, a, sizeof(double) * (size_t)nnzb * bs * bs);
    orc_cpr_setup(&h->cpr, nb, bs, h->ia, h->ja, h->a, stage2_maxit);
    return h;
}

void orc_cpr_destroy(void *hv)
{
    orc_cpr_handle *h = (orc_cpr_handle *)hv;
    if (!h) return;
    orc_cpr_free(&h->cpr);
    free(h->ia);
    free(h->ja);
    free(h->a);
    free(h);
}

/* stage2_type 2: forward HGS sweeps, 3: HSGS (jxf_cpr.c:572-585) */
void orc_cpr_set_stage2_type(void *hv, int type) { ((orc_cpr_handle *)hv)->cpr.stage2_type = type; }
void orc_cpr_set_stage2_chunk_h(void *hv, int chunk) { orc_cpr_set_stage2_chunk(&((orc_cpr_handle *)hv)->cpr, chunk); }

void orc_cpr_apply_h(void *hv, const double *r, double *z)
{
    orc_cpr_handle *h = (orc_cpr_handle *)hv;
    orc_cpr_apply(&h->cpr, r, z);
}

int orc_cpr_num_levels(void *hv) { return ((orc_cpr_handle *)hv)->cpr.amg.num_levels; }

/* what: 0 = A_l, 1 = P_l; sizes = {rows, cols, nnz} */
int orc_cpr_level_sizes(void *hv, int lev, int what, int *sizes)
{
    orc_amg *H = &((orc_cpr_handle *)hv)->cpr.amg;
    if (lev < 0 || lev >= H->num_levels || (what == 1 && lev >= H->num_levels - 1)) return -1;
    orc_csr *M = what == 0 ? &H->A[lev] : &H->P[lev];
    sizes[0] = M->n;
    sizes[1] = M->m;
    sizes[2] = M->ia[M->n];
    return 0;
}

int orc_cpr_level_matrix(void *hv, int lev, int what, int *ia, int *ja, double *a)
{
    orc_amg *H = &((orc_cpr_handle *)hv)->cpr.amg;
    if (lev < 0 || lev >= H->num_levels || (what == 1 && lev >= H->num_levels - 1)) return -1;
    orc_csr *M = what == 0 ? &H->A[lev] : &H->P[lev];
    memcpy(ia, M->ia, sizeof(int) * (M->n + 1));
    memcpy(ja, M->ja, sizeof(int) * M->ia[M->n]);
    memcpy(a, M->a, sizeof(double) * M->ia[M->n]);
    return 0;
}

int orc_cpr_level_cf(void *hv, int lev, int *cf)
{
    orc_amg *H = &((orc_cpr_handle *)hv)->cpr.amg;
    if (lev < 0 || lev >= H->num_levels - 1) return -1;
    memcpy(cf, H->CF[lev], sizeof(int) * H->A[lev].n);
    return 0;
}

void orc_cpr_amg_vcycle(void *hv, const double *rp, double *xp)
{
    orc_amg_vcycle(&((orc_cpr_handle *)hv)->cpr.amg, rp, xp);
}

int orc_gmres_solve(int nb, int bs, const int *ia, const int *ja, const double *a, const double *b, double *x,
                    int k_dim, double tol, int max_iter, void *cpr_handle, double *rel, int *converged,
                    double *norms)
{
    const orc_cpr *P = cpr_handle ? &((orc_cpr_handle *)cpr_handle)->cpr : NULL;
    return orc_gmres(nb, bs, ia, ja, a, b, x, k_dim, tol, max_iter, P, rel, converged, norms);
}
