/*
 * jxcpr_dropin.h -- the reference's C interface for the CPR-GMRES path,
 * served by libjxcpr_b200.so.
 *
 * A program written against the reference (jxfpamg-0220) for this path links
 * against libjxcpr_b200.so instead and keeps its calls:
 *
 *   jxf_BSRMatrixRead / _Binary        seq_bsr_matrix.c:1735,1935
 *   jxf_BSRMatrixDecouple              cpr/jxf_bsr_decoup.c:1273 (jxf_bsr_decoup.h:210-213)
 *   jxf_GeneratePartitioning, jxf_BSRMatrixToParBSRMatrix,
 *   jxf_ParBSRMatrixGetRowPartitioning, jxf_VectorToParVector   (jxf_parbsr_mv.h:156-158)
 *   JXF_CPRCreate / SetParameter / SetRealParameter / Setup / Precond /
 *   GetStatistics / Print / Destroy    cpr/jxf_cpr.c (jxf_cpr.h:75-174)
 *   JXF_ParBSRGMRESCreate              krylov/pbgmres.c:14
 *   JXF_GMRESSet* / Setup / Solve / Get*, jxf_GMRESDestroy   krylov/pgmres.c:101-334
 *   JXFPAMG_Solver_Interface           src/jxpamg_interface.c:118 (solver_id 220)
 *
 * The containers keep the reference's field order (jxf_bsr_mv.h:38-50,
 * jxf_parbsr_mv.h:37-77, jxf_mv.h:30-39 and :390-405) so that objects built
 * with the reference's macros can be passed in; MPI_Comm is laid out as an
 * int (the MPICH ABI, e.g. Intel MPI) and never used: this build runs one
 * process per GPU (np = 1).  JXF_Int, JXF_BigInt = int; JXF_Real = double.
 *
 * When JXF_GMRESSetPrecond receives JXF_CPRPrecond / JXF_CPRSetup, GMRES and
 * CPR run entirely on the GPU; any other preconditioner is called back on
 * the host once per application (device -> host -> device copies).
 *
 * Options for every solver this layer creates can be given in the
 * environment: JXCPR_OPTIONS="smoother_order=1,precision=1,flexible=1" (the
 * keys of jxcpr_solver_set_int / _set_real).  Defaults reproduce the
 * reference's arithmetic (exact-order preconditioner).
 *
 * Return codes are the reference's (0 success, 1 generic, 2 memory, 4
 * argument, 256 not converged) plus 512 for a CUDA failure; nothing aborts.
 */
#ifndef JXCPR_DROPIN_H
#define JXCPR_DROPIN_H

#include "jxcpr_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int JXF_Int;
typedef int JXF_BigInt;
typedef double JXF_Real;

#ifndef MPI_VERSION
typedef int MPI_Comm;
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#endif

typedef struct {
    JXF_Real *data;
    JXF_Int *i;
    JXF_Int *j;
    JXF_BigInt *big_j;
    JXF_Int block_size;
    JXF_Int num_rows;
    JXF_Int num_cols;
    JXF_Int num_nonzeros;
    JXF_Int owns_data;
} jxf_BSRMatrix;

typedef struct {
    JXF_Real *data;
    JXF_Int size;
    JXF_Int owns_data;
    JXF_Int num_vectors;
    JXF_Int multivec_storage_method;
    JXF_Int vecstride, idxstride;
} jxf_Vector;

typedef struct {
    MPI_Comm comm;
    JXF_Int global_size;
    JXF_Int first_index;
    JXF_Int last_index;
    JXF_Int *partitioning;
    jxf_Vector *local_vector;
    JXF_Int owns_data;
    JXF_Int owns_partitioning;
    void *assumed_partition;
} jxf_ParVector;

typedef struct {
    MPI_Comm comm;
    JXF_BigInt global_num_rows;
    JXF_BigInt global_num_cols;
    JXF_BigInt first_row_index;
    JXF_BigInt first_col_diag;
    JXF_BigInt last_row_index;
    JXF_BigInt last_col_diag;
    jxf_BSRMatrix *diag;
    jxf_BSRMatrix *offd;
    JXF_BigInt *col_map_offd;
    JXF_Int *row_starts;
    JXF_Int *col_starts;
    void *comm_pkg;
    void *comm_pkgT;
    JXF_Int owns_data;
    JXF_Int owns_row_starts;
    JXF_Int owns_col_starts;
    JXF_BigInt num_nonzeros;
    JXF_Real d_num_nonzeros;
    JXF_Int *rowindices;
    JXF_Real *rowvalues;
    JXF_Int getrowactive;
    void *assumed_partition;
} jxf_ParBSRMatrix;

#define jxf_BSRMatrixData(m) ((m)->data)
#define jxf_BSRMatrixI(m) ((m)->i)
#define jxf_BSRMatrixJ(m) ((m)->j)
#define jxf_BSRMatrixBlockSize(m) ((m)->block_size)
#define jxf_BSRMatrixNumRows(m) ((m)->num_rows)
#define jxf_BSRMatrixNumCols(m) ((m)->num_cols)
#define jxf_BSRMatrixNumNonzeros(m) ((m)->num_nonzeros)
#define jxf_BSRMatrixOwnsData(m) ((m)->owns_data)
#define jxf_VectorData(v) ((v)->data)
#define jxf_VectorSize(v) ((v)->size)
#define jxf_ParVectorLocalVector(v) ((v)->local_vector)
#define jxf_ParVectorGlobalSize(v) ((v)->global_size)
#define jxf_ParBSRMatrixDiag(m) ((m)->diag)
#define jxf_ParBSRMatrixOffd(m) ((m)->offd)

/* opaque handles (pointers only cross the boundary) */
typedef struct jxf_CPRPrecond_dropin jxf_CPRPrecond;
typedef struct jxf_Solver_struct *JXF_Solver;
typedef struct jxf_Matrix_struct *JXF_Matrix;
typedef struct jxf_Vector_struct *JXF_Vector;
typedef JXF_Int (*JXF_PtrToSolverFcn)(JXF_Solver, JXF_Matrix, JXF_Vector, JXF_Vector);

typedef enum {
    JXF_DECOUP_NONE = 0,
    JXF_DECOUP_ABF,
    JXF_DECOUP_ANL,
    JXF_DECOUP_SEM,
    JXF_DECOUP_QI,
    JXF_DECOUP_TIMPES,
    JXF_DECOUP_TIMPES2
} JXF_DecoupType;

/* ---- containers (host memory) ------------------------------------------------ */
JXCPR_API jxf_BSRMatrix *jxf_BSRMatrixCreate(JXF_Int block_size, JXF_Int num_rows, JXF_Int num_cols,
                                             JXF_Int num_nonzeros);
JXCPR_API JXF_Int jxf_BSRMatrixInitialize(jxf_BSRMatrix *A);
JXCPR_API JXF_Int jxf_BSRMatrixDestroy(jxf_BSRMatrix *A);
/* Text / binary BSR files: "rows cols nnz / block_size / storage (0 row-major, 1 column-major) /
 * n+1 IA / nnz JA / nnz*b*b values"; 1-based IA is detected.  NULL on a malformed file (the
 * reference exits instead).  The binary reader also reads column-major values (the reference's
 * column-major branch leaves them zero, seq_bsr_matrix.c:1995-2008). */
JXCPR_API jxf_BSRMatrix *jxf_BSRMatrixRead(const char *file_name);
JXCPR_API jxf_BSRMatrix *jxf_BSRMatrixRead_Binary(const char *file_name);
/* Writers of the same formats (1-based, row-major blocks). */
JXCPR_API JXF_Int jxf_BSRMatrixPrint(const jxf_BSRMatrix *A, const char *file_name);
JXCPR_API JXF_Int jxf_BSRMatrixPrint_Binary(const jxf_BSRMatrix *A, const char *file_name);

JXCPR_API jxf_Vector *jxf_SeqVectorCreate(JXF_Int size);
JXCPR_API JXF_Int jxf_SeqVectorInitialize(jxf_Vector *v);
JXCPR_API JXF_Int jxf_SeqVectorDestroy(jxf_Vector *v);

JXCPR_API JXF_Int jxf_GeneratePartitioning(JXF_Int length, JXF_Int num_procs, JXF_Int **part_ptr);
JXCPR_API jxf_ParBSRMatrix *jxf_BSRMatrixToParBSRMatrix(MPI_Comm comm, jxf_BSRMatrix *A, JXF_BigInt *row_starts,
                                                        JXF_BigInt *col_starts);
/* scalar-row partitioning {0, num_rows * block_size} (np = 1) */
JXCPR_API JXF_Int jxf_ParBSRMatrixGetRowPartitioning(jxf_ParBSRMatrix *A, JXF_Int **part_ptr);
JXCPR_API JXF_Int jxf_ParBSRMatrixDestroy(jxf_ParBSRMatrix *A);
JXCPR_API jxf_ParVector *jxf_VectorToParVector(MPI_Comm comm, jxf_Vector *v, JXF_Int *partitioning);
JXCPR_API jxf_ParVector *jxf_ParVectorCreate(MPI_Comm comm, JXF_Int global_size, JXF_Int *partitioning);
JXCPR_API JXF_Int jxf_ParVectorInitialize(jxf_ParVector *v);
JXCPR_API JXF_Int jxf_ParVectorSetConstantValues(jxf_ParVector *v, JXF_Real value);
JXCPR_API JXF_Int jxf_ParVectorDestroy(jxf_ParVector *v);

/* ---- decoupling on the GPU: ABF 1, ANL 2, SEM 3, QI 4, True-IMPES 5, True-IMPES (2nd) 6; thermal for 2-4 -- */
JXCPR_API JXF_Int jxf_BSRMatrixDecouple(jxf_BSRMatrix *A, jxf_Vector *rhs, JXF_DecoupType decoup_type,
                                        JXF_Int is_thermal);
JXCPR_API const char *jxf_DecoupTypeToString(JXF_DecoupType decoup_type);

/* ---- CPR ------------------------------------------------------------------------ */
JXCPR_API jxf_CPRPrecond *JXF_CPRCreate(MPI_Comm comm);
JXCPR_API JXF_Int JXF_CPRDestroy(jxf_CPRPrecond **cpr);
JXCPR_API JXF_Int JXF_CPRSetParameter(jxf_CPRPrecond *cpr, const char *param_name, JXF_Int value);
JXCPR_API JXF_Int JXF_CPRSetRealParameter(jxf_CPRPrecond *cpr, const char *param_name, JXF_Real value);
JXCPR_API JXF_Int JXF_CPRSetup(jxf_CPRPrecond *cpr, jxf_ParBSRMatrix *par_matrix);
JXCPR_API JXF_Int JXF_CPRPrecond(jxf_CPRPrecond *cpr, jxf_ParBSRMatrix *par_matrix, jxf_ParVector *par_rhs,
                                 jxf_ParVector *par_sol);
/* stats[4]: stage-1 setup s, stage-1 solve s, stage-2 setup s, stage-2 solve s */
JXCPR_API JXF_Int JXF_CPRGetStatistics(jxf_CPRPrecond *cpr, JXF_Real *stats);
JXCPR_API JXF_Int JXF_CPRPrint(jxf_CPRPrecond *cpr, JXF_Int level);

/* ---- GMRES ---------------------------------------------------------------------- */
JXCPR_API JXF_Int JXF_ParBSRGMRESCreate(MPI_Comm comm, JXF_Solver *solver);
JXCPR_API JXF_Int JXF_ParBSRGMRESDestroy(JXF_Solver solver);
JXCPR_API JXF_Int jxf_GMRESDestroy(void *gmres_vdata);
JXCPR_API JXF_Int JXF_GMRESSetKDim(JXF_Solver solver, JXF_Int k_dim);
JXCPR_API JXF_Int JXF_GMRESSetTol(JXF_Solver solver, JXF_Real tol);
JXCPR_API JXF_Int JXF_GMRESSetAbsoluteTol(JXF_Solver solver, JXF_Real a_tol);
JXCPR_API JXF_Int JXF_GMRESSetMaxIter(JXF_Solver solver, JXF_Int max_iter);
JXCPR_API JXF_Int JXF_GMRESSetMinIter(JXF_Solver solver, JXF_Int min_iter);
JXCPR_API JXF_Int JXF_GMRESSetIsCheckRestarted(JXF_Solver solver, JXF_Int is_check_restarted);
JXCPR_API JXF_Int JXF_GMRESSetConvFacThreshold(JXF_Solver solver, JXF_Real convfac_threshold);
JXCPR_API JXF_Int JXF_GMRESSetLogging(JXF_Solver solver, JXF_Int level);
JXCPR_API JXF_Int JXF_GMRESSetPrintLevel(JXF_Solver solver, JXF_Int level);
JXCPR_API JXF_Int JXF_GMRESSetPrecond(JXF_Solver solver, JXF_PtrToSolverFcn precond,
                                      JXF_PtrToSolverFcn precond_setup, JXF_Solver precond_data);
JXCPR_API JXF_Int JXF_GMRESSetup(JXF_Solver solver, JXF_Matrix matA, JXF_Vector vecB, JXF_Vector vecX);
JXCPR_API JXF_Int JXF_GMRESSolve(JXF_Solver solver, JXF_Matrix preOperator, JXF_Matrix matA, JXF_Vector vecB,
                                 JXF_Vector vecX);
JXCPR_API JXF_Int JXF_GMRESGetNumIterations(JXF_Solver solver, JXF_Int *num_iterations);
JXCPR_API JXF_Int JXF_GMRESGetFinalRelativeResidualNorm(JXF_Solver solver, JXF_Real *norm);
JXCPR_API JXF_Int JXF_GMRESGetConverged(JXF_Solver solver, JXF_Int *converged);

/* ---- one-call interface (src/jxpamg_interface.c:118-257) --------------------------------
 * CSR matrix of `row` scalar rows (0- or 1-based, detected from ia[0] and converted in place as
 * the reference does; each row's diagonal entry is moved to the front in place), solved for
 * ser_b into ser_x (overwritten).  solver_id 220: CPR-GMRES with the unknowns of each node
 * (num_functions >= 2 consecutive rows) gathered into num_functions x num_functions blocks,
 * CPR stage 2 with one block-GS sweep as the reference's case 220 sets, k_dim 30,
 * max_iter 1000.  *iter receives the GMRES iterations.  Other solver ids return 4. */
JXCPR_API JXF_Int JXFPAMG_Solver_Interface(JXF_Int argc, char *argv[], MPI_Comm comm, JXF_Int row, JXF_Int *ia,
                                           JXF_Int *ja, JXF_Real *a, JXF_Real *ser_x, JXF_Real *ser_b,
                                           JXF_Real tol, JXF_Int solver_id, JXF_Int num_functions,
                                           JXF_Int *iter);

#ifdef __cplusplus
}
#endif

#endif
