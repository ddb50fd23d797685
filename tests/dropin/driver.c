/*
 * A caller of the reference's C interface, compiled against include/jxcpr_dropin.h and linked
 * with libjxcpr_b200.so.  Its call sequence follows the reference's CPR-GMRES driver
 * (src/test_bsr_cprgmres.c:123-429): read BSR -> decouple -> distribute -> CPR create / parameters /
 * setup -> GMRES create / parameters / precond / setup / solve -> statistics.
 *
 *   driver bsr  A.txt b.bin x.bin [decouple]        CPR-GMRES through JXF_*
 *   driver csr  ia.bin ja.bin a.bin b.bin x.bin n bs JXFPAMG_Solver_Interface (solver 220)
 *   driver bin  A.bin b.bin x.bin                   binary reader, then as "bsr"
 * Prints "iterations <it> rel <rel>".
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "jxcpr_dropin.h"

static double *read_doubles(const char *path, long *n) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return NULL;
    fseek(fp, 0, SEEK_END);
    long bytes = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    double *v = malloc(bytes);
    *n = bytes / (long)sizeof(double);
    if (fread(v, sizeof(double), *n, fp) != (size_t)*n) {
        fclose(fp);
        free(v);
        return NULL;
    }
    fclose(fp);
    return v;
}

static int *read_ints(const char *path, long *n) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return NULL;
    fseek(fp, 0, SEEK_END);
    long bytes = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    int *v = malloc(bytes);
    *n = bytes / (long)sizeof(int);
    if (fread(v, sizeof(int), *n, fp) != (size_t)*n) {
        fclose(fp);
        free(v);
        return NULL;
    }
    fclose(fp);
    return v;
}

static int write_doubles(const char *path, const double *v, long n) {
    FILE *fp = fopen(path, "wb");
    if (!fp) return 1;
    fwrite(v, sizeof(double), n, fp);
    fclose(fp);
    return 0;
}

static int run_bsr(jxf_BSRMatrix *A, const char *bpath, const char *xpath, int decouple) {
    long nb_vals = 0;
    double *bv = read_doubles(bpath, &nb_vals);
    const int n = A->num_rows * A->block_size;
    if (!bv || nb_vals != n) return 2;
    jxf_Vector *b = jxf_SeqVectorCreate(n), *x = jxf_SeqVectorCreate(n);
    jxf_SeqVectorInitialize(b);
    jxf_SeqVectorInitialize(x);
    memcpy(jxf_VectorData(b), bv, sizeof(double) * n);
    if (decouple && jxf_BSRMatrixDecouple(A, b, (JXF_DecoupType)decouple, 0)) return 3;

    JXF_Int *rs = NULL, *cs = NULL, *part = NULL;
    jxf_GeneratePartitioning(A->num_rows, 1, &rs);
    jxf_GeneratePartitioning(A->num_cols, 1, &cs);
    jxf_ParBSRMatrix *Ap = jxf_BSRMatrixToParBSRMatrix(MPI_COMM_WORLD, A, rs, cs);
    jxf_ParBSRMatrixGetRowPartitioning(Ap, &part);
    jxf_ParVector *pb = jxf_VectorToParVector(MPI_COMM_WORLD, b, part);
    jxf_ParVector *px = jxf_VectorToParVector(MPI_COMM_WORLD, x, part);

    jxf_CPRPrecond *cpr = JXF_CPRCreate(MPI_COMM_WORLD);
    if (JXF_CPRSetParameter(cpr, "pressure_index", 0) || JXF_CPRSetParameter(cpr, "stage1_maxit", 1) ||
        JXF_CPRSetParameter(cpr, "stage2_maxit", 3) || JXF_CPRSetParameter(cpr, "stage1_solver_type", 1) ||
        JXF_CPRSetParameter(cpr, "stage2_solver_type", 2) || JXF_CPRSetRealParameter(cpr, "threshold", 1e-15))
        return 4;
    if (JXF_CPRSetParameter(cpr, "no_such_parameter", 1) == 0) return 5;  /* unknown keys are errors */
    if (JXF_CPRSetup(cpr, Ap)) return 6;

    JXF_Solver solver;
    JXF_ParBSRGMRESCreate(MPI_COMM_WORLD, &solver);
    JXF_GMRESSetKDim(solver, 30);
    JXF_GMRESSetIsCheckRestarted(solver, 1);
    JXF_GMRESSetMaxIter(solver, 300);
    JXF_GMRESSetTol(solver, 1e-6);
    JXF_GMRESSetLogging(solver, 1);
    JXF_GMRESSetPrintLevel(solver, 0);
    JXF_GMRESSetPrecond(solver, (JXF_PtrToSolverFcn)JXF_CPRPrecond, (JXF_PtrToSolverFcn)JXF_CPRSetup,
                        (JXF_Solver)cpr);
    if (JXF_GMRESSetup(solver, (JXF_Matrix)Ap, (JXF_Vector)pb, (JXF_Vector)px)) return 7;
    if (JXF_GMRESSolve(solver, (JXF_Matrix)Ap, (JXF_Matrix)Ap, (JXF_Vector)pb, (JXF_Vector)px)) return 8;
    JXF_Int it = 0, conv = 0;
    JXF_Real rel = 0.0, stats[4];
    JXF_GMRESGetNumIterations(solver, &it);
    JXF_GMRESGetFinalRelativeResidualNorm(solver, &rel);
    JXF_GMRESGetConverged(solver, &conv);
    JXF_CPRGetStatistics(cpr, stats);
    printf("iterations %d rel %.17e converged %d setup_s %.6f\n", it, rel, conv, stats[0]);
    if (write_doubles(xpath, jxf_VectorData(jxf_ParVectorLocalVector(px)), n)) return 9;

    JXF_ParBSRGMRESDestroy(solver);
    JXF_CPRDestroy(&cpr);
    if (cpr != NULL) return 10;
    jxf_ParVectorDestroy(pb);
    jxf_ParVectorDestroy(px);
    jxf_ParBSRMatrixDestroy(Ap);
    jxf_SeqVectorDestroy(b);
    jxf_SeqVectorDestroy(x);
    free(rs);
    free(cs);
    free(part);
    free(bv);
    return conv ? 0 : 11;
}

int main(int argc, char **argv) {
    if (argc < 2) return 1;
    if (!strcmp(argv[1], "bsr") || !strcmp(argv[1], "bin")) {
        if (argc < 5) return 1;
        jxf_BSRMatrix *A = !strcmp(argv[1], "bsr") ? jxf_BSRMatrixRead(argv[2]) : jxf_BSRMatrixRead_Binary(argv[2]);
        if (!A) {
            fprintf(stderr, "read failed: %s\n", jxcpr_last_error());
            return 12;
        }
        int st = run_bsr(A, argv[3], argv[4], argc > 5 ? atoi(argv[5]) : 1);
        jxf_BSRMatrixDestroy(A);
        if (st) fprintf(stderr, "driver status %d: %s\n", st, jxcpr_last_error());
        return st;
    }
    if (!strcmp(argv[1], "csr")) {
        if (argc < 9) return 1;
        long nia, nja, na, nb;
        int *ia = read_ints(argv[2], &nia), *ja = read_ints(argv[3], &nja);
        double *a = read_doubles(argv[4], &na), *b = read_doubles(argv[5], &nb);
        const int n = atoi(argv[7]), bs = atoi(argv[8]);
        if (!ia || !ja || !a || !b || nia != n + 1 || nb != n) return 13;
        double *x = calloc(n, sizeof(double));
        JXF_Int it = 0;
        int st = JXFPAMG_Solver_Interface(0, NULL, MPI_COMM_WORLD, n, ia, ja, a, x, b, 1e-6, 220, bs, &it);
        printf("iterations %d rel 0 converged %d setup_s 0\n", it, st == 0);
        if (st) fprintf(stderr, "interface status %d: %s\n", st, jxcpr_last_error());
        write_doubles(argv[6], x, n);
        return st;
    }
    return 1;
}
