/*
 * ORACLE (test infrastructure only): declarations of the plain-C restatement
 * of the reference CPR-GMRES path.  Used by tests/, the smoke check and the
 * CPU-baseline leg of bench.py as the test oracle; never linked by the product.
 */
#ifndef JXCPR_ORACLE_H
#define JXCPR_ORACLE_H

int orc_bsr_matvec(int nb, int bs, const int *ia, const int *ja, const double *a, double alpha, const double *x,
                   double beta, double *y);
int orc_bsr_decouple(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type,
                     int consistent_rhs);
int orc_bsr_decouple2(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type,
                      int thermal, int consistent_rhs);
void orc_restrict(int nb, int bs, int p, const double *r, double *rp);
void orc_prolong(int nb, int bs, int p, const double *xp, double *x);
void orc_bsr_submatrix(int nb, int bs, const int *ia, const int *ja, const double *a, int p, int *cia, int *cja,
                       double *ca);


/* ---- AMG / CPR / GMRES restatement (orc_amg.c, orc_cpr.c) ---- */
#define ORC_MAX_LEVELS 26

typedef struct {
    int n, m;     /* rows, cols */
    int *ia, *ja; /* 0-based CSR, diagonal first where present */
    double *a;
} orc_csr;

typedef struct {
    int num_levels;
    int owns_A0;
    orc_csr A[ORC_MAX_LEVELS];
    orc_csr P[ORC_MAX_LEVELS];
    int *CF[ORC_MAX_LEVELS];
} orc_amg;

typedef struct {
    int nb, bs, stage2_maxit, stage2_type;
    int stage2_chunk, ncolour; /* > 0: stage 2 in chunk order (orc_chunk_colour), colour per row */
    int *colour;
    const int *ia, *ja;
    const double *a;
    double *work; /* stage-2 work vector (nb * bs), zero at setup */
    orc_csr Ap;
    orc_amg amg;
} orc_cpr;

void orc_csr_free(orc_csr *A);
void orc_strength(const orc_csr *A, double theta, double max_row_sum, orc_csr *S);
void orc_rs_first_pass(const orc_csr *S, int *CF);
double orc_park_miller(int *seed);
void orc_pmis(const orc_csr *S, int *CF);
void orc_hmis(const orc_csr *S, int *CF);
void orc_rs_first_pass_ranges(const orc_csr *S, int range_rows, int *CF);
void orc_hmis_ranges(int n, const int *ia, const int *ja, const double *a, double theta, double max_row_sum,
                     int range_rows, int *CF);
int orc_strength_csr(int n, const int *ia, const int *ja, const double *a, double theta, double max_row_sum,
                     int *sia, int *sja);
void orc_rs_first_pass_csr(int n, const int *sia, const int *sja, int range_rows, int *cf);
void orc_extpi_interp(const orc_csr *A, const orc_csr *S, const int *CF, orc_csr *P);
void orc_rap(const orc_csr *A, const orc_csr *P, orc_csr *Ac);
void orc_amg_setup(const orc_csr *A0, int max_levels, int coarse_threshold, orc_amg *H);
void orc_amg_free(orc_amg *H);
void orc_csr_matvec(const orc_csr *A, double alpha, const double *x, double beta, double *y);
void orc_csr_matvec_t(const orc_csr *A, double alpha, const double *x, double beta, double *y);
void orc_relax6(const orc_csr *A, const double *f, double *u);
int orc_gselim(const orc_csr *A, const double *f, double *u);
void orc_amg_vcycle(const orc_amg *H, const double *f0, double *u0);
void orc_hgs_relax(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                   double w, double omega, int direction);
void orc_hsgs_relax(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                    double *work, double w, double omega);
void orc_cpr_setup(orc_cpr *C, int nb, int bs, const int *ia, const int *ja, const double *a, int stage2_maxit);
int orc_chunk_colour(int nb, const int *ia, const int *ja, int chunk, int *colour);
void orc_hgs_relax_chunked(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                           double w, double omega, int chunk, const int *colour, int ncolour);
void orc_cpr_set_stage2_chunk(orc_cpr *C, int chunk);
void orc_cpr_apply(const orc_cpr *C, const double *r, double *z);
void orc_cpr_free(orc_cpr *C);
int orc_gmres(int nb, int bs, const int *ia, const int *ja, const double *a, const double *b, double *x, int k_dim,
              double tol, int max_iter, const orc_cpr *precond, double *rel, int *converged, double *norms);

/* ---- block ILU(0) restatement (orc_bilu.c) ---- */
int orc_bilu_levels(int nb, const int *lia, const int *lja, const int *uia, const int *uja, int *lev_l,
                    int *lev_u, int *nup);
int orc_bilu_setup_exact(int nb, int bs, const int *ia, const int *ja, const double *a, const int *lia,
                         const int *lja, double *la, const int *uia, const int *uja, double *ua, double *dinv);
int orc_bilu_solve_exact(int nb, int bs, const int *ia, const int *ja, const double *a, const int *lia,
                         const int *lja, const double *la, const int *uia, const int *uja, const double *ua,
                         const double *dinv, int ir_iters, const double *f, double *u);
int orc_bilu_pattern(int nb, const int *ia, const int *ja, int *lia, int *lja, int *uia, int *uja);
int orc_bilu_setup(int nb, int bs, const int *ia, const int *ja, const double *a, int sweeps, const int *lia,
                   const int *lja, double *la, const int *uia, const int *uja, double *ua, double *dinv);
int orc_bilu_solve(int nb, int bs, const int *ia, const int *ja, const double *a, const int *lia, const int *lja,
                   const double *la, const int *uia, const int *uja, const double *ua, const double *dinv,
                   int ir_iters, int lower_iters, int upper_iters, const double *f, double *u);

#endif
