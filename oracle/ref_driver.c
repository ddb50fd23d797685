/*
 * Plain-array driver around the reference JXFPAMG library (built from its own
 * sources into oracle/_ref/).  Test infrastructure only: it lets the Python
 * tests run the reference's BSR SpMV, decoupling, HGS smoother, CPR setup /
 * apply (with its AMG hierarchy exposed level by level) and the full
 * CPR-GMRES solve of src/test_bsr_cprgmres.c:123-429 on arrays, so that the
 * oracle restatement and the golden fixtures can be pinned to the reference.
 *
 * Every entry takes 0-based BSR arrays (ia[nb+1], ja[nnzb], a[nnzb*b*b],
 * row-major blocks) and copies them into reference containers; the caller's
 * arrays are never retained.  The reference prints unconditionally from its
 * CPR and GMRES code; `quiet` redirects stdout to /dev/null for the call.
 */
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "jxf_bsr_decoup.h"
#include "jxf_bsr_mv.h"
#include "jxf_cpr.h"
#include "jxf_krylov.h"
#include "jxf_mv.h"
#include "jxf_pamg.h"
#include "jxf_parbsr_mv.h"
#include "jxf_parbilu.h"

int ref_driver_version(void) { return 3; }

/* ---- stdout silencing ------------------------------------------------- */
static int g_saved_stdout = -1;
static void quiet_begin(int quiet)
{
    if (!quiet) return;
    fflush(stdout);
    g_saved_stdout = dup(1);
    int fd = open("/dev/null", O_WRONLY);
    dup2(fd, 1);
    close(fd);
}
static void quiet_end(int quiet)
{
    if (!quiet || g_saved_stdout < 0) return;
    fflush(stdout);
    dup2(g_saved_stdout, 1);
    close(g_saved_stdout);
    g_saved_stdout = -1;
}

/* ---- container helpers ------------------------------------------------- */
static jxf_BSRMatrix *make_bsr(int nb, int bs, const int *ia, const int *ja, const double *a)
{
    int nnzb = ia[nb];
    jxf_BSRMatrix *A = jxf_BSRMatrixCreate(bs, nb, nb, nnzb); /* (block_size, rows, cols, nnz) as implemented */
    jxf_BSRMatrixI(A) = (JXF_Int *)malloc(sizeof(JXF_Int) * (nb + 1));
    jxf_BSRMatrixJ(A) = (JXF_Int *)malloc(sizeof(JXF_Int) * (nnzb > 0 ? nnzb : 1));
    jxf_BSRMatrixData(A) = (JXF_Real *)malloc(sizeof(JXF_Real) * ((size_t)nnzb * bs * bs + 1));
    memcpy(jxf_BSRMatrixI(A), ia, sizeof(int) * (nb + 1));
    memcpy(jxf_BSRMatrixJ(A), ja, sizeof(int) * nnzb);
    memcpy(jxf_BSRMatrixData(A), a, sizeof(double) * (size_t)nnzb * bs * bs);
    jxf_BSRMatrixOwnsData(A) = 1;
    return A;
}

static jxf_Vector *make_vec(int n, const double *v)
{
    jxf_Vector *x = jxf_SeqVectorCreate(n);
    jxf_SeqVectorInitialize(x);
    if (v) memcpy(jxf_VectorData(x), v, sizeof(double) * n);
    else memset(jxf_VectorData(x), 0, sizeof(double) * n);
    return x;
}

static jxf_ParBSRMatrix *to_par(jxf_BSRMatrix *A)
{
    JXF_Int *rs = NULL, *cs = NULL;
    jxf_GeneratePartitioning(jxf_BSRMatrixNumRows(A), 1, &rs);
    jxf_GeneratePartitioning(jxf_BSRMatrixNumCols(A), 1, &cs);
    return jxf_BSRMatrixToParBSRMatrix(MPI_COMM_WORLD, A, rs, cs);
}

static jxf_ParVector *to_par_vec(jxf_ParBSRMatrix *Ap, jxf_Vector *v)
{
    JXF_Int *part = NULL;
    jxf_ParBSRMatrixGetRowPartitioning(Ap, &part);
    return jxf_VectorToParVector(jxf_ParBSRMatrixComm(Ap), v, part);
}

static double *pvec_data(jxf_ParVector *v) { return jxf_VectorData(jxf_ParVectorLocalVector(v)); }

/* ---- kernels ------------------------------------------------------------ */

/* y = alpha*A*x + beta*y through jxf_BSRMatrixMatvec (seq_bsr_matvec.c:22-140). */
int ref_bsr_matvec(int nb, int bs, const int *ia, const int *ja, const double *a, double alpha, const double *x,
                   double beta, double *y)
{
    jxf_BSRMatrix *A = make_bsr(nb, bs, ia, ja, a);
    jxf_Vector *vx = make_vec(nb * bs, x);
    jxf_Vector *vy = make_vec(nb * bs, y);
    int ierr = jxf_BSRMatrixMatvec(alpha, A, vx, beta, vy);
    memcpy(y, jxf_VectorData(vy), sizeof(double) * nb * bs);
    jxf_SeqVectorDestroy(vx);
    jxf_SeqVectorDestroy(vy);
    jxf_BSRMatrixDestroy(A);
    return ierr;
}

/* In-place decoupling of a (values only) and rhs (jxf_bsr_decoup.c:1273-1348). */
int ref_bsr_decouple2(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type,
                      int thermal, int quiet)
{
    jxf_BSRMatrix *A = make_bsr(nb, bs, ia, ja, a);
    jxf_Vector *vb = make_vec(nb * bs, rhs);
    quiet_begin(quiet);
    int ierr = jxf_BSRMatrixDecouple(A, vb, (JXF_DecoupType)type, thermal);
    quiet_end(quiet);
    memcpy(a, jxf_BSRMatrixData(A), sizeof(double) * (size_t)ia[nb] * bs * bs);
    memcpy(rhs, jxf_VectorData(vb), sizeof(double) * nb * bs);
    jxf_SeqVectorDestroy(vb);
    jxf_BSRMatrixDestroy(A);
    return ierr;
}

int ref_bsr_decouple(int nb, int bs, const int *ia, const int *ja, double *a, double *rhs, int type, int quiet)
{
    return ref_bsr_decouple2(nb, bs, ia, ja, a, rhs, type, 0, quiet);
}

/* `sweeps` jxf_ParBSRHSGSRelax calls (par_relax_bsr.c:579-1062) updating x in place; work is the
 * caller's Vtemp vector (nb * bs, in/out: the reference refreshes only its first nb entries). */
int ref_hsgs_relax(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                   double *work, double relax_weight, double omega, int sweeps)
{
    jxf_BSRMatrix *A = make_bsr(nb, bs, ia, ja, a);
    jxf_ParBSRMatrix *Ap = to_par(A);
    jxf_Vector *vx = make_vec(nb * bs, x), *vb = make_vec(nb * bs, b), *vw = make_vec(nb * bs, work);
    jxf_ParVector *px = to_par_vec(Ap, vx), *pb = to_par_vec(Ap, vb), *pw = to_par_vec(Ap, vw);
    for (int s = 0; s < sweeps; s++) jxf_ParBSRHSGSRelax(Ap, px, pb, pw, relax_weight, omega, 1);
    memcpy(x, pvec_data(px), sizeof(double) * nb * bs);
    memcpy(work, pvec_data(pw), sizeof(double) * nb * bs);
    return 0;
}

/* One jxf_ParBSRHGSRelax sweep (par_relax_bsr.c:193-573) updating x in place. */
int ref_hgs_relax(int nb, int bs, const int *ia, const int *ja, const double *a, double *x, const double *b,
                  double relax_weight, double omega, int direction, int sweeps)
{
    jxf_BSRMatrix *A = make_bsr(nb, bs, ia, ja, a);
    jxf_ParBSRMatrix *Ap = to_par(A);
    jxf_Vector *vx = make_vec(nb * bs, x), *vb = make_vec(nb * bs, b), *vw = make_vec(nb * bs, NULL);
    jxf_ParVector *px = to_par_vec(Ap, vx), *pb = to_par_vec(Ap, vb), *pw = to_par_vec(Ap, vw);
    for (int s = 0; s < sweeps; s++) jxf_ParBSRHGSRelax(Ap, px, pb, pw, relax_weight, omega, direction);
    memcpy(x, pvec_data(px), sizeof(double) * nb * bs);
    return 0;
}

/* ---- CPR handle: setup (jxf_cpr.c:268-422) + apply (:424-610) ---------- */
typedef struct {
    jxf_BSRMatrix *A;
    jxf_ParBSRMatrix *Ap;
    jxf_CPRPrecond *cpr;
    jxf_ParVector *r, *z;
    int nb, bs;
} ref_cpr_t;

void *ref_cpr_create(int nb, int bs, const int *ia, const int *ja, const double *a, int stage1_maxit,
                     int stage2_maxit, int stage2_type, int quiet)
{
    ref_cpr_t *h = (ref_cpr_t *)calloc(1, sizeof(ref_cpr_t));
    h->nb = nb;
    h->bs = bs;
    h->A = make_bsr(nb, bs, ia, ja, a);
    h->Ap = to_par(h->A);
    quiet_begin(quiet);
    h->cpr = JXF_CPRCreate(MPI_COMM_WORLD);
    JXF_CPRSetParameter(h->cpr, "pressure_index", 0);
    JXF_CPRSetParameter(h->cpr, "block_size", bs);
    JXF_CPRSetParameter(h->cpr, "stage1_maxit", stage1_maxit);
    JXF_CPRSetParameter(h->cpr, "stage2_maxit", stage2_maxit);
    JXF_CPRSetParameter(h->cpr, "stage1_solver_type", 1);
    JXF_CPRSetParameter(h->cpr, "stage2_solver_type", stage2_type);
    JXF_CPRSetParameter(h->cpr, "print_level", 0);
    JXF_CPRSetRealParameter(h->cpr, "threshold", 1e-15);
    int ierr = JXF_CPRSetup(h->cpr, h->Ap);
    quiet_end(quiet);
    if (ierr) return NULL;
    jxf_Vector *vr = make_vec(nb * bs, NULL), *vz = make_vec(nb * bs, NULL);
    h->r = to_par_vec(h->Ap, vr);
    h->z = to_par_vec(h->Ap, vz);
    return h;
}

int ref_cpr_apply(void *hv, const double *r, double *z, int quiet)
{
    ref_cpr_t *h = (ref_cpr_t *)hv;
    int n = h->nb * h->bs;
    memcpy(pvec_data(h->r), r, sizeof(double) * n);
    memset(pvec_data(h->z), 0, sizeof(double) * n);
    quiet_begin(quiet);
    int ierr = JXF_CPRPrecond(h->cpr, h->Ap, h->r, h->z);
    quiet_end(quiet);
    memcpy(z, pvec_data(h->z), sizeof(double) * n);
    return ierr;
}

/* AMG hierarchy inspection (par_amg_setup.c output: A_l, P_l, CF markers). */
static jxf_ParAMGData *cpr_amg(ref_cpr_t *h) { return (jxf_ParAMGData *)h->cpr->stage1_solver; }

int ref_cpr_num_levels(void *hv) { return jxf_ParAMGDataNumLevels(cpr_amg((ref_cpr_t *)hv)); }

/* what: 0 = A_l, 1 = P_l. sizes = {rows, cols, nnz}. Returns -1 if absent. */
int ref_cpr_level_sizes(void *hv, int lev, int what, int *sizes)
{
    jxf_ParAMGData *amg = cpr_amg((ref_cpr_t *)hv);
    jxf_ParCSRMatrix *M = what == 0 ? jxf_ParAMGDataAArray(amg)[lev] : jxf_ParAMGDataPArray(amg)[lev];
    if (!M) return -1;
    jxf_CSRMatrix *d = jxf_ParCSRMatrixDiag(M);
    sizes[0] = jxf_CSRMatrixNumRows(d);
    sizes[1] = jxf_CSRMatrixNumCols(d);
    sizes[2] = jxf_CSRMatrixNumNonzeros(d);
    return jxf_CSRMatrixNumNonzeros(jxf_ParCSRMatrixOffd(M));
}

int ref_cpr_level_matrix(void *hv, int lev, int what, int *ia, int *ja, double *a)
{
    jxf_ParAMGData *amg = cpr_amg((ref_cpr_t *)hv);
    jxf_ParCSRMatrix *M = what == 0 ? jxf_ParAMGDataAArray(amg)[lev] : jxf_ParAMGDataPArray(amg)[lev];
    if (!M) return -1;
    jxf_CSRMatrix *d = jxf_ParCSRMatrixDiag(M);
    int n = jxf_CSRMatrixNumRows(d);
    int nnz = jxf_CSRMatrixNumNonzeros(d);
    memcpy(ia, jxf_CSRMatrixI(d), sizeof(int) * (n + 1));
    memcpy(ja, jxf_CSRMatrixJ(d), sizeof(int) * nnz);
    memcpy(a, jxf_CSRMatrixData(d), sizeof(double) * nnz);
    return 0;
}

int ref_cpr_level_cf(void *hv, int lev, int *cf)
{
    jxf_ParAMGData *amg = cpr_amg((ref_cpr_t *)hv);
    int *m = jxf_ParAMGDataCFMarkerArray(amg)[lev];
    if (!m) return -1;
    int n = jxf_CSRMatrixNumRows(jxf_ParCSRMatrixDiag(jxf_ParAMGDataAArray(amg)[lev]));
    memcpy(cf, m, sizeof(int) * n);
    return 0;
}

/* One stage-1 AMG solve (JXF_PAMGSolve with the CPR settings) on the pressure system. */
int ref_cpr_amg_solve(void *hv, const double *rp, double *xp, int quiet)
{
    ref_cpr_t *h = (ref_cpr_t *)hv;
    jxf_CPRPrecond *cpr = h->cpr;
    memcpy(pvec_data(cpr->rp), rp, sizeof(double) * h->nb);
    memcpy(pvec_data(cpr->xp), xp, sizeof(double) * h->nb);
    quiet_begin(quiet);
    int ierr = JXF_PAMGSolve(cpr->stage1_solver, (JXF_ParCSRMatrix)cpr->A_pressure, (JXF_Vector)cpr->rp,
                             (JXF_ParVector)cpr->xp);
    quiet_end(quiet);
    memcpy(xp, pvec_data(cpr->xp), sizeof(double) * h->nb);
    return ierr;
}

/* The Ruge-Stueben first pass of the reference's HMIS (jxf_PAMGCoarsenRuge
 * with coarsen_type 10, as par_coarsen_hmis.c:32 calls it) on a strength
 * pattern given as CSR, one process.  cf receives its markers (1 C, -1 F,
 * -2 Z, -3 SF). */
int ref_rs_first_pass(int n, const int *ia, const int *ja, int *cf)
{
    int nnz = ia[n];
    JXF_Int *rs = NULL;
    jxf_GeneratePartitioning(n, 1, &rs);
    jxf_ParCSRMatrix *S = jxf_ParCSRMatrixCreate(MPI_COMM_WORLD, n, n, rs, rs, 0, nnz, 0);
    jxf_ParCSRMatrixInitialize(S);
    jxf_CSRMatrix *d = jxf_ParCSRMatrixDiag(S);
    memcpy(jxf_CSRMatrixI(d), ia, sizeof(int) * (n + 1));
    if (nnz) memcpy(jxf_CSRMatrixJ(d), ja, sizeof(int) * nnz);
    for (int k = 0; k < nnz; k++) jxf_CSRMatrixData(d)[k] = 1.0;
    JXF_Int *CF = NULL;
    int ierr = jxf_PAMGCoarsenRuge(S, S, 0, 10, 0, &CF);
    if (CF) {
        memcpy(cf, CF, sizeof(int) * n);
        jxf_TFree(CF);
    }
    jxf_ParCSRMatrixDestroy(S);
    return ierr;
}

void ref_cpr_free(void *hv)
{
    ref_cpr_t *h = (ref_cpr_t *)hv;
    if (!h) return;
    JXF_CPRDestroy(&h->cpr);
    free(h);
}

/* ---- full CPR-GMRES solve (test_bsr_cprgmres.c:123-429) ----------------- */
/*
 * decouple: JXF_DecoupType (0 none, 1 ABF, 5 TIMPES, ...); precond: 0 none
 * (identity), 1 CPR.  On return x holds the solution, info[0] iterations,
 * info[1] converged flag; rel[0] final relative residual from GMRES,
 * rel[1] true ||b - A x|| / ||b|| recomputed on the decoupled system;
 * norms (if not NULL, length max_iter+1) the GMRES residual history.
 * times[0..3] = decouple, CPR setup, solve wall seconds, CPR stage times.
 */
int ref_cpr_gmres_solve(int nb, int bs, const int *ia, const int *ja, const double *a, const double *b, double *x,
                        int decouple, int precond, int kdim, double tol, int max_iter, int stage2_maxit,
                        int stage2_type, int *info, double *rel, double *norms, double *times, int quiet)
{
    int n = nb * bs;
    quiet_begin(quiet);
    jxf_BSRMatrix *A = make_bsr(nb, bs, ia, ja, a);
    jxf_Vector *vb = make_vec(n, b), *vx = make_vec(n, x);
    double t0 = MPI_Wtime();
    if (decouple) jxf_BSRMatrixDecouple(A, vb, (JXF_DecoupType)decouple, 0);
    double t1 = MPI_Wtime();
    jxf_ParBSRMatrix *Ap = to_par(A);
    jxf_ParVector *pb = to_par_vec(Ap, vb), *px = to_par_vec(Ap, vx);

    jxf_CPRPrecond *cpr = NULL;
    double t2 = MPI_Wtime();
    if (precond == 1) {
        cpr = JXF_CPRCreate(MPI_COMM_WORLD);
        JXF_CPRSetParameter(cpr, "pressure_index", 0);
        JXF_CPRSetParameter(cpr, "block_size", bs);
        JXF_CPRSetParameter(cpr, "stage1_maxit", 1);
        JXF_CPRSetParameter(cpr, "stage2_maxit", stage2_maxit);
        JXF_CPRSetParameter(cpr, "stage1_solver_type", 1);
        JXF_CPRSetParameter(cpr, "stage2_solver_type", stage2_type);
        JXF_CPRSetParameter(cpr, "print_level", 0);
        JXF_CPRSetRealParameter(cpr, "threshold", 1e-15);
        JXF_CPRSetup(cpr, Ap);
    }
    double t3 = MPI_Wtime();

    JXF_Solver gm;
    JXF_ParBSRGMRESCreate(MPI_COMM_WORLD, &gm);
    JXF_GMRESSetKDim(gm, kdim);
    JXF_GMRESSetIsCheckRestarted(gm, 1);
    JXF_GMRESSetMaxIter(gm, max_iter);
    JXF_GMRESSetTol(gm, tol);
    JXF_GMRESSetLogging(gm, 1);
    JXF_GMRESSetPrintLevel(gm, 1); /* norms[] are recorded only when printing */
    if (cpr)
        JXF_GMRESSetPrecond(gm, (JXF_PtrToSolverFcn)JXF_CPRPrecond, (JXF_PtrToSolverFcn)JXF_CPRSetup, (JXF_Solver)cpr);
    JXF_GMRESSetup(gm, (JXF_Matrix)Ap, (JXF_Vector)pb, (JXF_Vector)px);
    double t4 = MPI_Wtime();
    JXF_GMRESSolve(gm, (JXF_Matrix)Ap, (JXF_Matrix)Ap, (JXF_Vector)pb, (JXF_Vector)px);
    double t5 = MPI_Wtime();

    JXF_Int iters = 0, conv = 0;
    JXF_Real frel = 0.0;
    JXF_GMRESGetNumIterations(gm, &iters);
    JXF_GMRESGetFinalRelativeResidualNorm(gm, &frel);
    JXF_GMRESGetConverged(gm, &conv);
    info[0] = iters;
    info[1] = conv;
    rel[0] = frel;

    jxf_Vector *vr = make_vec(n, NULL);
    jxf_ParVector *pr = to_par_vec(Ap, vr);
    jxf_ParVectorCopy(pb, pr);
    jxf_ParBSRMatrixMatvec(-1.0, Ap, px, 1.0, pr);
    double rn = jxf_ParVectorNorm2(pr), bn = jxf_ParVectorNorm2(pb);
    rel[1] = bn > 0 ? rn / bn : rn;
    memcpy(x, pvec_data(px), sizeof(double) * n);
    if (norms) {
        jxf_GMRESData *gd = (jxf_GMRESData *)gm;
        for (int k = 0; k <= iters && k <= max_iter; k++) norms[k] = gd->norms[k];
    }
    if (times) {
        times[0] = t1 - t0;
        times[1] = t3 - t2;
        times[2] = t5 - t4;
        if (cpr) {
            JXF_Real st[4];
            JXF_CPRGetStatistics(cpr, st);
            times[3] = st[1];
            times[4] = st[3];
        }
    }
    quiet_end(quiet);
    return 0;
}

/* ---- block ILU(0): jxf_BILUSetup / jxf_BILUSolve ------------------------------
 * Type 3 (jxf_ILUSetupFGPBILU_v3, par_bilu_setup.c:4996) with `sweeps` sweeps,
 * solve with tri_solve 14 (par_bilu_solve.c:360, 2893), max_iter 1, tol 0,
 * the given IR / lower / upper Jacobi iteration counts; u = 0 on entry.  The
 * lower-case entry points are called directly: the upper-case JXF_BILUSetup /
 * JXF_BILUSolve wrappers forward to the CSR ILU (parbsr_bilu.c:36-66).
 * Outputs the factors (L, U strictly lower / upper blocks in A's order, D^-1
 * blocks) and u. */
int ref_bilu(int nb, int bs, const int *ia, const int *ja, const double *a, int sweeps, int ir, int lower, int upper,
             const double *f, double *u, double *la, double *ua, double *dinv, int quiet)
{
    jxf_BSRMatrix *A = make_bsr(nb, bs, ia, ja, a);
    jxf_ParBSRMatrix *Ap = to_par(A);
    jxf_Vector *vf = make_vec(nb * bs, f), *vu = make_vec(nb * bs, NULL), *vt = make_vec(nb * bs, NULL);
    jxf_ParVector *pf = to_par_vec(Ap, vf), *pu = to_par_vec(Ap, vu), *pt = to_par_vec(Ap, vt);
    void *solver = jxf_BILUCreate();
    jxf_ParBILUData *d = (jxf_ParBILUData *)solver;
    jxf_ParILUDataIluType(d) = 3;
    jxf_ParILUDataLfil(d) = 0;
    jxf_ParILUDataMaxIter(d) = 1;
    jxf_ParILUDataTol(d) = 0.0;
    jxf_ParILUDataTriSolve(d) = 14;
    jxf_ParILUDataLogging(d) = 0;
    jxf_ParILUDataPrintLevel(d) = 0;
    jxf_ParILUDatasweep(d) = sweeps;
    jxf_ParILUDataIRIters(d) = ir;
    jxf_ParILUDataLowerJacobiIters(d) = lower;
    jxf_ParILUDataUpperJacobiIters(d) = upper;
    quiet_begin(quiet);
    int ierr = jxf_BILUSetup(solver, Ap, pt, pt);
    if (!ierr) ierr = jxf_BILUSolve(solver, Ap, pf, pu);
    quiet_end(quiet);
    const int bn = bs * bs;
    jxf_BSRMatrix *L = jxf_ParBSRMatrixDiag(jxf_ParILUDataMatL(d));
    jxf_BSRMatrix *U = jxf_ParBSRMatrixDiag(jxf_ParILUDataMatU(d));
    if (la) memcpy(la, jxf_BSRMatrixData(L), sizeof(double) * (size_t)jxf_BSRMatrixI(L)[nb] * bn);
    if (ua) memcpy(ua, jxf_BSRMatrixData(U), sizeof(double) * (size_t)jxf_BSRMatrixI(U)[nb] * bn);
    if (dinv) memcpy(dinv, pvec_data(jxf_ParILUDataD(d)), sizeof(double) * (size_t)nb * bn);
    memcpy(u, pvec_data(pu), sizeof(double) * nb * bs);
    jxf_BILUDestroy(solver);
    return ierr;
}
