/*
 * ORACLE (test infrastructure only): declarations of the plain-C restatement
 * of the reference CPR-GMRES path.  Used by tests/, the smoke check and the
 * CPU-baseline leg of bench.py as the checker; never linked by the product.
 */
#ifndef JXCPR_ORACLE_H
#define JXCPR_ORACLE_H

int orc_bsr_matvec(int nb, int bs, const int *ia, const int *ja, const double *a, double alpha, const double *x,
                   double beta, double *y);
int orc_bsr_decouple(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type,
                     int consistent_rhs);
void orc_restrict(int nb, int bs, int p, const double *r, double *rp);
void orc_prolong(int nb, int bs, int p, const double *xp, double *x);
void orc_bsr_submatrix(int nb, int bs, const int *ia, const int *ja, const double *a, int p, int *cia, int *cja,
                       double *ca);

#endif
