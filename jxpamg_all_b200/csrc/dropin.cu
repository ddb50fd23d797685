// The reference's C interface for the CPR-GMRES path (include/jxcpr_dropin.h)
// on top of the solver object.  Host code only: containers, readers/writers,
// the CPR / GMRES handles and JXFPAMG_Solver_Interface.  Matrices cross to
// the GPU in JXF_CPRSetup (a device copy is cached in the handle and rebuilt
// by the next setup); vectors are copied per call.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "jxcpr_dropin.h"
#include "handle.cuh"

using namespace jxcpr;


struct jxf_CPRPrecond_dropin {
    jxcpr_solver *h = nullptr;
    std::vector<std::pair<std::string, int>> ints;
    std::vector<std::pair<std::string, double>> reals;
    const jxf_ParBSRMatrix *A = nullptr;
    int ready = 0;
    int print_level = 0;
};

struct jxf_Solver_struct {  // GMRES handle
    int k_dim = 5, max_iter = 1000, min_iter = 0, is_check_restarted = 0, logging = 0, print_level = 0;
    double tol = 1e-6, a_tol = 0.0, convfac_threshold = 1e4;
    JXF_PtrToSolverFcn precond = nullptr, precond_setup = nullptr;
    JXF_Solver precond_data = nullptr;
    const jxf_ParBSRMatrix *A = nullptr;
    jxcpr_solver *own = nullptr;  // solver for a foreign / identity preconditioner
    int iterations = 0, converged = 0;
    double rel = 0.0;
};

namespace {

template <typename F>
int guard(F &&f) {
    try {
        return f();
    } catch (const CudaError &) {
        return JXCPR_ERROR_DEVICE;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return JXCPR_ERROR_MEMORY;
    } catch (...) {
        set_error("unexpected exception");
        return JXCPR_ERROR_GENERIC;
    }
}

// JXCPR_OPTIONS="key=value,key=value": applied to every solver this layer creates
void apply_env_options(jxcpr_solver *h) {
    const char *env = getenv("JXCPR_OPTIONS");
    if (!env) return;
    std::string all(env);
    size_t pos = 0;
    while (pos < all.size()) {
        size_t end = all.find(',', pos);
        if (end == std::string::npos) end = all.size();
        const std::string kv = all.substr(pos, end - pos);
        const size_t eq = kv.find('=');
        if (eq != std::string::npos) {
            const std::string k = kv.substr(0, eq), v = kv.substr(eq + 1);
            if (v.find_first_of(".eE") != std::string::npos) jxcpr_solver_set_real(h, k.c_str(), atof(v.c_str()));
            else jxcpr_solver_set_int(h, k.c_str(), atoi(v.c_str()));
        }
        pos = end + 1;
    }
}

jxcpr_solver *new_solver() {
    jxcpr_solver *h = nullptr;
    if (jxcpr_solver_create(&h) != JXCPR_SUCCESS) return nullptr;
    return h;
}

const jxf_BSRMatrix *local(const jxf_ParBSRMatrix *A) { return A ? A->diag : nullptr; }

bool read_ints(FILE *fp, int *v, long long n) {
    for (long long k = 0; k < n; ++k)
        if (fscanf(fp, "%d", v + k) != 1) return false;
    return true;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// containers
// ---------------------------------------------------------------------------
jxf_BSRMatrix *jxf_BSRMatrixCreate(JXF_Int block_size, JXF_Int num_rows, JXF_Int num_cols, JXF_Int num_nonzeros) {
    jxf_BSRMatrix *A = (jxf_BSRMatrix *)calloc(1, sizeof(jxf_BSRMatrix));
    if (!A) return nullptr;
    A->block_size = block_size;
    A->num_rows = num_rows;
    A->num_cols = num_cols;
    A->num_nonzeros = num_nonzeros;
    A->owns_data = 1;
    return A;
}

JXF_Int jxf_BSRMatrixInitialize(jxf_BSRMatrix *A) {
    if (!A) return JXCPR_ERROR_ARG;
    const long long bn = (long long)A->block_size * A->block_size;
    if (!A->i) A->i = (JXF_Int *)calloc((size_t)A->num_rows + 1, sizeof(JXF_Int));
    if (!A->j) A->j = (JXF_Int *)calloc((size_t)std::max(A->num_nonzeros, 1), sizeof(JXF_Int));
    if (!A->data) A->data = (JXF_Real *)calloc((size_t)std::max<long long>(A->num_nonzeros * bn, 1), sizeof(JXF_Real));
    return (A->i && A->j && A->data) ? JXCPR_SUCCESS : JXCPR_ERROR_MEMORY;
}

JXF_Int jxf_BSRMatrixDestroy(jxf_BSRMatrix *A) {
    if (!A) return JXCPR_SUCCESS;
    if (A->owns_data) {
        free(A->i);
        free(A->j);
        free(A->data);
        free(A->big_j);
    }
    free(A);
    return JXCPR_SUCCESS;
}

// Column-major blocks of a file are transposed into the container's row-major layout.
static void blocks_to_row_major(double *data, long long nnz, int bs) {
    const int bn = bs * bs;
    std::vector<double> t(bn);
    for (long long k = 0; k < nnz; ++k) {
        double *b = data + k * bn;
        for (int q = 0; q < bn; ++q) t[q] = b[q];
        for (int bi = 0; bi < bs; ++bi)
            for (int bj = 0; bj < bs; ++bj) b[bi * bs + bj] = t[bj * bs + bi];
    }
}

static jxf_BSRMatrix *finish_read(int rows, int cols, int nnz, int bs, int *ia, int *ja, double *a) {
    jxf_BSRMatrix *A = jxf_BSRMatrixCreate(bs, rows, cols, nnz);
    if (!A) {
        free(ia);
        free(ja);
        free(a);
        return nullptr;
    }
    A->i = ia;
    A->j = ja;
    A->data = a;
    return A;
}

jxf_BSRMatrix *jxf_BSRMatrixRead(const char *file_name) {
    FILE *fp = file_name ? fopen(file_name, "r") : nullptr;
    if (!fp) {
        set_error("jxf_BSRMatrixRead: cannot open %s", file_name ? file_name : "(null)");
        return nullptr;
    }
    int rows = 0, cols = 0, nnz = 0, bs = 0, storage = 0, n = 0;
    int *ia = nullptr, *ja = nullptr;
    double *a = nullptr;
    bool ok = fscanf(fp, "%d %d %d", &rows, &cols, &nnz) == 3 && fscanf(fp, "%d", &bs) == 1 &&
              fscanf(fp, "%d", &storage) == 1 && rows >= 0 && nnz >= 0 && bs >= 1;
    const long long bn = (long long)bs * bs;
    if (ok) {
        ia = (int *)calloc((size_t)rows + 1, sizeof(int));
        ja = (int *)calloc((size_t)std::max(nnz, 1), sizeof(int));
        a = (double *)calloc((size_t)std::max<long long>(nnz * bn, 1), sizeof(double));
        ok = ia && ja && a;
    }
    ok = ok && fscanf(fp, "%d", &n) == 1 && n == rows + 1 && read_ints(fp, ia, n);
    ok = ok && fscanf(fp, "%d", &n) == 1 && n == nnz && read_ints(fp, ja, n);
    ok = ok && fscanf(fp, "%d", &n) == 1 && (long long)n == nnz * bn;
    for (long long k = 0; ok && k < (long long)nnz * bn; ++k) ok = fscanf(fp, "%le", a + k) == 1;
    fclose(fp);
    if (!ok) {
        free(ia);
        free(ja);
        free(a);
        set_error("jxf_BSRMatrixRead: malformed file %s", file_name);
        return nullptr;
    }
    const int base = ia[0] == 1 ? 1 : 0;
    int max_col = 0;
    for (int k = 0; k <= rows; ++k) ia[k] -= base;
    for (int k = 0; k < nnz; ++k) {
        ja[k] -= base;
        max_col = std::max(max_col, ja[k]);
    }
    if (nnz > 0 && max_col + 1 != cols) {
        free(ia);
        free(ja);
        free(a);
        set_error("jxf_BSRMatrixRead: max column %d + 1 != num_cols %d", max_col, cols);
        return nullptr;
    }
    if (storage == 1) blocks_to_row_major(a, nnz, bs);
    return finish_read(rows, cols, nnz, bs, ia, ja, a);
}

jxf_BSRMatrix *jxf_BSRMatrixRead_Binary(const char *file_name) {
    FILE *fp = file_name ? fopen(file_name, "rb") : nullptr;
    if (!fp) {
        set_error("jxf_BSRMatrixRead_Binary: cannot open %s", file_name ? file_name : "(null)");
        return nullptr;
    }
    int hdr[5] = {0, 0, 0, 0, 0}, n = 0;
    bool ok = fread(hdr, sizeof(int), 5, fp) == 5 && hdr[0] >= 0 && hdr[2] >= 0 && hdr[3] >= 1;
    const int rows = hdr[0], cols = hdr[1], nnz = hdr[2], bs = hdr[3], storage = hdr[4];
    const long long bn = (long long)bs * bs;
    int *ia = nullptr, *ja = nullptr;
    double *a = nullptr;
    if (ok) {
        ia = (int *)calloc((size_t)rows + 1, sizeof(int));
        ja = (int *)calloc((size_t)std::max(nnz, 1), sizeof(int));
        a = (double *)calloc((size_t)std::max<long long>(nnz * bn, 1), sizeof(double));
        ok = ia && ja && a;
    }
    ok = ok && fread(&n, sizeof(int), 1, fp) == 1 && n == rows + 1 && fread(ia, sizeof(int), n, fp) == (size_t)n;
    ok = ok && fread(&n, sizeof(int), 1, fp) == 1 && n == nnz && fread(ja, sizeof(int), n, fp) == (size_t)n;
    ok = ok && fread(&n, sizeof(int), 1, fp) == 1 && (long long)n == nnz * bn &&
         fread(a, sizeof(double), n, fp) == (size_t)n;
    fclose(fp);
    if (!ok) {
        free(ia);
        free(ja);
        free(a);
        set_error("jxf_BSRMatrixRead_Binary: malformed file %s", file_name);
        return nullptr;
    }
    if (ia[0] == 1) {
        for (int k = 0; k <= rows; ++k) ia[k] -= 1;
        for (int k = 0; k < nnz; ++k) ja[k] -= 1;
    }
    if (storage == 1) blocks_to_row_major(a, nnz, bs);
    return finish_read(rows, cols, nnz, bs, ia, ja, a);
}

JXF_Int jxf_BSRMatrixPrint(const jxf_BSRMatrix *A, const char *file_name) {
    if (!A || !file_name) return JXCPR_ERROR_ARG;
    FILE *fp = fopen(file_name, "w");
    if (!fp) return JXCPR_ERROR_GENERIC;
    const int n = A->num_rows, nnz = A->num_nonzeros, bs = A->block_size;
    fprintf(fp, "%d %d %d\n%d\n0\n%d\n", n, A->num_cols, nnz, bs, n + 1);
    for (int k = 0; k <= n; ++k) fprintf(fp, "%d\n", A->i[k] + 1);
    fprintf(fp, "%d\n", nnz);
    for (int k = 0; k < nnz; ++k) fprintf(fp, "%d\n", A->j[k] + 1);
    fprintf(fp, "%lld\n", (long long)nnz * bs * bs);
    for (long long k = 0; k < (long long)nnz * bs * bs; ++k) fprintf(fp, "%.17e\n", A->data[k]);
    fclose(fp);
    return JXCPR_SUCCESS;
}

JXF_Int jxf_BSRMatrixPrint_Binary(const jxf_BSRMatrix *A, const char *file_name) {
    if (!A || !file_name) return JXCPR_ERROR_ARG;
    FILE *fp = fopen(file_name, "wb");
    if (!fp) return JXCPR_ERROR_GENERIC;
    const int n = A->num_rows, nnz = A->num_nonzeros, bs = A->block_size;
    const int hdr[5] = {n, A->num_cols, nnz, bs, 0};
    fwrite(hdr, sizeof(int), 5, fp);
    int m = n + 1;
    fwrite(&m, sizeof(int), 1, fp);
    for (int k = 0; k <= n; ++k) {
        const int v = A->i[k] + 1;
        fwrite(&v, sizeof(int), 1, fp);
    }
    fwrite(&nnz, sizeof(int), 1, fp);
    for (int k = 0; k < nnz; ++k) {
        const int v = A->j[k] + 1;
        fwrite(&v, sizeof(int), 1, fp);
    }
    m = nnz * bs * bs;
    fwrite(&m, sizeof(int), 1, fp);
    fwrite(A->data, sizeof(double), (size_t)m, fp);
    fclose(fp);
    return JXCPR_SUCCESS;
}

jxf_Vector *jxf_SeqVectorCreate(JXF_Int size) {
    jxf_Vector *v = (jxf_Vector *)calloc(1, sizeof(jxf_Vector));
    if (!v) return nullptr;
    v->size = size;
    v->owns_data = 1;
    v->num_vectors = 1;
    return v;
}

JXF_Int jxf_SeqVectorInitialize(jxf_Vector *v) {
    if (!v) return JXCPR_ERROR_ARG;
    if (!v->data) v->data = (JXF_Real *)calloc((size_t)std::max(v->size, 1), sizeof(JXF_Real));
    return v->data ? JXCPR_SUCCESS : JXCPR_ERROR_MEMORY;
}

JXF_Int jxf_SeqVectorDestroy(jxf_Vector *v) {
    if (!v) return JXCPR_SUCCESS;
    if (v->owns_data) free(v->data);
    free(v);
    return JXCPR_SUCCESS;
}

JXF_Int jxf_GeneratePartitioning(JXF_Int length, JXF_Int num_procs, JXF_Int **part_ptr) {
    if (!part_ptr || num_procs < 1) return JXCPR_ERROR_ARG;
    JXF_Int *p = (JXF_Int *)calloc((size_t)num_procs + 1, sizeof(JXF_Int));
    if (!p) return JXCPR_ERROR_MEMORY;
    const int size = length / num_procs, rest = length - size * num_procs;
    for (int k = 0; k < num_procs; ++k) p[k + 1] = p[k] + size + (k < rest ? 1 : 0);
    *part_ptr = p;
    return JXCPR_SUCCESS;
}

jxf_ParBSRMatrix *jxf_BSRMatrixToParBSRMatrix(MPI_Comm comm, jxf_BSRMatrix *A, JXF_BigInt *row_starts,
                                              JXF_BigInt *col_starts) {
    if (!A) return nullptr;
    jxf_ParBSRMatrix *P = (jxf_ParBSRMatrix *)calloc(1, sizeof(jxf_ParBSRMatrix));
    if (!P) return nullptr;
    const int bs = A->block_size, nb = A->num_rows, nnz = A->num_nonzeros;
    const long long bn = (long long)bs * bs;
    jxf_BSRMatrix *D = jxf_BSRMatrixCreate(bs, nb, A->num_cols, nnz);
    if (!D || jxf_BSRMatrixInitialize(D) != JXCPR_SUCCESS) return nullptr;
    memcpy(D->i, A->i, sizeof(int) * ((size_t)nb + 1));
    memcpy(D->j, A->j, sizeof(int) * (size_t)nnz);
    memcpy(D->data, A->data, sizeof(double) * (size_t)(nnz * bn));
    P->comm = comm;
    P->global_num_rows = nb;
    P->global_num_cols = A->num_cols;
    P->first_row_index = 0;
    P->first_col_diag = 0;
    P->last_row_index = nb - 1;
    P->last_col_diag = A->num_cols - 1;
    P->diag = D;
    P->offd = jxf_BSRMatrixCreate(bs, nb, 0, 0);
    jxf_BSRMatrixInitialize(P->offd);
    P->row_starts = row_starts;
    P->col_starts = col_starts;
    P->owns_data = 1;
    P->num_nonzeros = nnz;
    P->d_num_nonzeros = (double)nnz;
    return P;
}

JXF_Int jxf_ParBSRMatrixGetRowPartitioning(jxf_ParBSRMatrix *A, JXF_Int **part_ptr) {
    if (!A || !A->diag || !part_ptr) return JXCPR_ERROR_ARG;
    JXF_Int *p = (JXF_Int *)calloc(2, sizeof(JXF_Int));
    if (!p) return JXCPR_ERROR_MEMORY;
    p[1] = A->diag->num_rows * A->diag->block_size;
    *part_ptr = p;
    return JXCPR_SUCCESS;
}

JXF_Int jxf_ParBSRMatrixDestroy(jxf_ParBSRMatrix *A) {
    if (!A) return JXCPR_SUCCESS;
    if (A->owns_data) {
        jxf_BSRMatrixDestroy(A->diag);
        jxf_BSRMatrixDestroy(A->offd);
    }
    free(A);
    return JXCPR_SUCCESS;
}

jxf_ParVector *jxf_ParVectorCreate(MPI_Comm comm, JXF_Int global_size, JXF_Int *partitioning) {
    jxf_ParVector *v = (jxf_ParVector *)calloc(1, sizeof(jxf_ParVector));
    if (!v) return nullptr;
    v->comm = comm;
    v->global_size = global_size;
    v->first_index = 0;
    v->last_index = global_size - 1;
    v->partitioning = partitioning;
    v->local_vector = jxf_SeqVectorCreate(global_size);
    v->owns_data = 1;
    return v;
}

JXF_Int jxf_ParVectorInitialize(jxf_ParVector *v) {
    if (!v) return JXCPR_ERROR_ARG;
    return jxf_SeqVectorInitialize(v->local_vector);
}

JXF_Int jxf_ParVectorSetConstantValues(jxf_ParVector *v, JXF_Real value) {
    if (!v || !v->local_vector || !v->local_vector->data) return JXCPR_ERROR_ARG;
    for (int k = 0; k < v->local_vector->size; ++k) v->local_vector->data[k] = value;
    return JXCPR_SUCCESS;
}

jxf_ParVector *jxf_VectorToParVector(MPI_Comm comm, jxf_Vector *v, JXF_Int *partitioning) {
    if (!v) return nullptr;
    jxf_ParVector *p = jxf_ParVectorCreate(comm, v->size, partitioning);
    if (!p || jxf_ParVectorInitialize(p) != JXCPR_SUCCESS) return nullptr;
    if (v->size) memcpy(p->local_vector->data, v->data, sizeof(double) * (size_t)v->size);
    return p;
}

JXF_Int jxf_ParVectorDestroy(jxf_ParVector *v) {
    if (!v) return JXCPR_SUCCESS;
    if (v->owns_data) jxf_SeqVectorDestroy(v->local_vector);
    if (v->owns_partitioning) free(v->partitioning);
    free(v);
    return JXCPR_SUCCESS;
}

// ---------------------------------------------------------------------------
// decoupling: on the GPU through a solver object (matrix and rhs overwritten)
// ---------------------------------------------------------------------------
const char *jxf_DecoupTypeToString(JXF_DecoupType t) {
    static const char *names[] = {"NONE", "ABF", "ANL", "SEM", "QI", "TIMPES", "TIMPES2"};
    return (t >= 0 && t <= 6) ? names[t] : "UNKNOWN";
}

JXF_Int jxf_BSRMatrixDecouple(jxf_BSRMatrix *A, jxf_Vector *rhs, JXF_DecoupType type, JXF_Int is_thermal) {
    if (!A) return JXCPR_ERROR_ARG;
    if (type == JXF_DECOUP_NONE) return JXCPR_SUCCESS;
    if ((int)type < 1 || (int)type > 6) {
        set_error("jxf_BSRMatrixDecouple: unknown decoupling type %d", (int)type);
        return JXCPR_ERROR_ARG;
    }
    return guard([&] {
        const int nb = A->num_rows, bs = A->block_size;
        const long long nnzb = A->num_nonzeros;
        cudaStream_t s = nullptr;
        DeviceBsr D;
        D.alloc(nb, bs, nnzb);
        D.ia.upload(A->i, (size_t)nb + 1, s);
        D.ja.upload(A->j, (size_t)nnzb, s);
        D.a.upload(A->data, (size_t)nnzb * bs * bs, s);
        DevBuf<double> coef((size_t)std::max(nb, 1) * std::max(decouple_coef_size(bs, (int)type), 1));
        bsr_decouple_matrix(D, (int)type, coef.get(), s, is_thermal ? 1 : 0);
        D.a.download(A->data, (size_t)nnzb * bs * bs, s);
        if (rhs && rhs->data) {
            DevBuf<double> b((size_t)std::max(nb * bs, 1));
            b.upload(rhs->data, (size_t)nb * bs, s);
            bsr_decouple_rhs(nb, bs, (int)type, coef.get(), b.get(), 0, s);
            b.download(rhs->data, (size_t)nb * bs, s);
        }
        JX_CUDA(cudaStreamSynchronize(s));
        return JXCPR_SUCCESS;
    });
}

// ---------------------------------------------------------------------------
// CPR
// ---------------------------------------------------------------------------
jxf_CPRPrecond *JXF_CPRCreate(MPI_Comm) {
    jxf_CPRPrecond *c = new (std::nothrow) jxf_CPRPrecond_dropin();
    return c;
}

JXF_Int JXF_CPRDestroy(jxf_CPRPrecond **cpr) {
    if (!cpr || !*cpr) return JXCPR_ERROR_ARG;
    if ((*cpr)->h) jxcpr_solver_destroy((*cpr)->h);
    delete *cpr;
    *cpr = nullptr;
    return JXCPR_SUCCESS;
}

JXF_Int JXF_CPRSetParameter(jxf_CPRPrecond *cpr, const char *name, JXF_Int value) {
    if (!cpr || !name) return JXCPR_ERROR_ARG;
    // validate against the solver's option table (unknown keys fail as in the reference)
    jxcpr_solver *probe = new_solver();
    if (!probe) return JXCPR_ERROR_MEMORY;
    int st = strcmp(name, "print_level") == 0 ? JXCPR_SUCCESS : jxcpr_solver_set_int(probe, name, value);
    jxcpr_solver_destroy(probe);
    if (st) return st;
    if (!strcmp(name, "print_level")) cpr->print_level = value;
    cpr->ints.emplace_back(name, value);
    return JXCPR_SUCCESS;
}

JXF_Int JXF_CPRSetRealParameter(jxf_CPRPrecond *cpr, const char *name, JXF_Real value) {
    if (!cpr || !name) return JXCPR_ERROR_ARG;
    jxcpr_solver *probe = new_solver();
    if (!probe) return JXCPR_ERROR_MEMORY;
    int st = jxcpr_solver_set_real(probe, name, value);
    jxcpr_solver_destroy(probe);
    if (st) return st;
    cpr->reals.emplace_back(name, value);
    return JXCPR_SUCCESS;
}

JXF_Int JXF_CPRSetup(jxf_CPRPrecond *cpr, jxf_ParBSRMatrix *par_matrix) {
    const jxf_BSRMatrix *A = local(par_matrix);
    if (!cpr || !A) return JXCPR_ERROR_ARG;
    if (cpr->h) jxcpr_solver_destroy(cpr->h);
    cpr->h = new_solver();
    if (!cpr->h) return JXCPR_ERROR_MEMORY;
    jxcpr_solver_set_int(cpr->h, "decouple", 0);  // the caller decouples (jxf_BSRMatrixDecouple)
    for (auto &kv : cpr->ints)
        if (kv.first != "print_level") jxcpr_solver_set_int(cpr->h, kv.first.c_str(), kv.second);
    for (auto &kv : cpr->reals) jxcpr_solver_set_real(cpr->h, kv.first.c_str(), kv.second);
    apply_env_options(cpr->h);
    const int st = jxcpr_solver_setup(cpr->h, A->num_rows, A->block_size, A->num_nonzeros, A->i, A->j, A->data, 0);
    cpr->A = par_matrix;
    cpr->ready = st == JXCPR_SUCCESS;
    return st;
}

JXF_Int JXF_CPRPrecond(jxf_CPRPrecond *cpr, jxf_ParBSRMatrix *, jxf_ParVector *par_rhs, jxf_ParVector *par_sol) {
    if (!cpr || !cpr->ready || !par_rhs || !par_sol || !par_rhs->local_vector || !par_sol->local_vector)
        return JXCPR_ERROR_ARG;
    return jxcpr_solver_cpr_apply(cpr->h, par_rhs->local_vector->data, par_sol->local_vector->data, 0);
}

JXF_Int JXF_CPRGetStatistics(jxf_CPRPrecond *cpr, JXF_Real *stats) {
    if (!cpr || !stats || !cpr->h) return JXCPR_ERROR_ARG;
    const CprPrecond &C = cpr->h->s.cpr;
    for (int k = 0; k < 4; ++k) stats[k] = C.stats[k];
    return JXCPR_SUCCESS;
}

JXF_Int JXF_CPRPrint(jxf_CPRPrecond *cpr, JXF_Int level) {
    if (!cpr) return JXCPR_ERROR_ARG;
    if (level <= 0 || !cpr->h) return JXCPR_SUCCESS;
    const Solver &S = cpr->h->s;
    printf("CPR (GPU): %d AMG levels, setup %.3f ms, last solve %.3f ms\n", S.cpr.amg.num_levels(), S.setup_ms,
           S.solve_ms);
    if (level > 1) {
        char buf[8192];
        jxcpr_solver_setup_report(cpr->h, buf, sizeof buf);
        printf("%s", buf);
    }
    return JXCPR_SUCCESS;
}

// ---------------------------------------------------------------------------
// GMRES
// ---------------------------------------------------------------------------
JXF_Int JXF_ParBSRGMRESCreate(MPI_Comm, JXF_Solver *solver) {
    if (!solver) return JXCPR_ERROR_ARG;
    *solver = new (std::nothrow) jxf_Solver_struct();
    return *solver ? JXCPR_SUCCESS : JXCPR_ERROR_MEMORY;
}

JXF_Int JXF_ParBSRGMRESDestroy(JXF_Solver solver) {
    if (!solver) return JXCPR_ERROR_ARG;
    if (solver->own) jxcpr_solver_destroy(solver->own);
    delete solver;
    return JXCPR_SUCCESS;
}

JXF_Int jxf_GMRESDestroy(void *gmres_vdata) { return JXF_ParBSRGMRESDestroy((JXF_Solver)gmres_vdata); }

#define JXF_GMRES_SETTER(NAME, TYPE, FIELD)           \
    JXF_Int NAME(JXF_Solver solver, TYPE v) {          \
        if (!solver) return JXCPR_ERROR_ARG;           \
        solver->FIELD = v;                             \
        return JXCPR_SUCCESS;                          \
    }
JXF_GMRES_SETTER(JXF_GMRESSetKDim, JXF_Int, k_dim)
JXF_GMRES_SETTER(JXF_GMRESSetTol, JXF_Real, tol)
JXF_GMRES_SETTER(JXF_GMRESSetAbsoluteTol, JXF_Real, a_tol)
JXF_GMRES_SETTER(JXF_GMRESSetMaxIter, JXF_Int, max_iter)
JXF_GMRES_SETTER(JXF_GMRESSetMinIter, JXF_Int, min_iter)
JXF_GMRES_SETTER(JXF_GMRESSetIsCheckRestarted, JXF_Int, is_check_restarted)
JXF_GMRES_SETTER(JXF_GMRESSetConvFacThreshold, JXF_Real, convfac_threshold)
JXF_GMRES_SETTER(JXF_GMRESSetLogging, JXF_Int, logging)
JXF_GMRES_SETTER(JXF_GMRESSetPrintLevel, JXF_Int, print_level)
#undef JXF_GMRES_SETTER

JXF_Int JXF_GMRESSetPrecond(JXF_Solver solver, JXF_PtrToSolverFcn precond, JXF_PtrToSolverFcn precond_setup,
                            JXF_Solver precond_data) {
    if (!solver) return JXCPR_ERROR_ARG;
    solver->precond = precond;
    solver->precond_setup = precond_setup;
    solver->precond_data = precond_data;
    return JXCPR_SUCCESS;
}

static bool uses_device_cpr(JXF_Solver solver) {
    return solver->precond == (JXF_PtrToSolverFcn)JXF_CPRPrecond;
}

JXF_Int JXF_GMRESSetup(JXF_Solver solver, JXF_Matrix matA, JXF_Vector vecB, JXF_Vector vecX) {
    if (!solver || !matA) return JXCPR_ERROR_ARG;
    solver->A = (const jxf_ParBSRMatrix *)matA;
    if (uses_device_cpr(solver)) {
        jxf_CPRPrecond *cpr = (jxf_CPRPrecond *)solver->precond_data;
        // the reference's setup calls the preconditioner setup again; skip it when CPR already holds this matrix
        if (!cpr) return JXCPR_ERROR_ARG;
        if (cpr->ready && cpr->A == solver->A) return JXCPR_SUCCESS;
        return JXF_CPRSetup(cpr, (jxf_ParBSRMatrix *)matA);
    }
    if (solver->precond_setup) {
        const int st = solver->precond_setup(solver->precond_data, matA, vecB, vecX);
        if (st) return st;
    }
    return JXCPR_SUCCESS;
}

static void copy_gmres_params(JXF_Solver solver, jxcpr_solver *h) {
    jxcpr_solver_set_int(h, "k_dim", solver->k_dim);
    jxcpr_solver_set_int(h, "max_iter", solver->max_iter);
    jxcpr_solver_set_int(h, "min_iter", solver->min_iter);
    jxcpr_solver_set_int(h, "is_check_restarted", solver->is_check_restarted);
    jxcpr_solver_set_real(h, "tol", solver->tol);
    jxcpr_solver_set_real(h, "a_tol", solver->a_tol);
    jxcpr_solver_set_real(h, "convfac_threshold", solver->convfac_threshold);
}

JXF_Int JXF_GMRESSolve(JXF_Solver solver, JXF_Matrix, JXF_Matrix matA, JXF_Vector vecB, JXF_Vector vecX) {
    if (!solver || !matA || !vecB || !vecX) return JXCPR_ERROR_ARG;
    jxf_ParVector *b = (jxf_ParVector *)vecB, *x = (jxf_ParVector *)vecX;
    if (!b->local_vector || !x->local_vector) return JXCPR_ERROR_ARG;
    int it = 0, st = 0;
    double rel = 0.0;
    if (uses_device_cpr(solver)) {
        jxf_CPRPrecond *cpr = (jxf_CPRPrecond *)solver->precond_data;
        if (!cpr || !cpr->ready) return JXCPR_ERROR_ARG;
        // k_dim must be known at setup for the Krylov basis: re-set up when it changed
        if (cpr->h->s.gmres.prm.k_dim != solver->k_dim) {
            jxcpr_solver_set_int(cpr->h, "k_dim", solver->k_dim);
            cpr->h->s.gmres.prm.k_dim = solver->k_dim;
            st = guard([&] {
                cpr->h->s.gmres.setup(cpr->h->s.A.nb * cpr->h->s.A.bs, cpr->h->s.stream);
                return JXCPR_SUCCESS;
            });
            if (st) return st;
        }
        copy_gmres_params(solver, cpr->h);
        st = jxcpr_solver_solve(cpr->h, b->local_vector->data, x->local_vector->data, 0, &it, &rel);
    } else {
        // identity or a host preconditioner called back once per application
        const jxf_BSRMatrix *A = local((const jxf_ParBSRMatrix *)matA);
        if (!A) return JXCPR_ERROR_ARG;
        if (!solver->own) {
            solver->own = new_solver();
            if (!solver->own) return JXCPR_ERROR_MEMORY;
        }
        jxcpr_solver_set_int(solver->own, "stage1_solver_type", 0);
        jxcpr_solver_set_int(solver->own, "decouple", 0);
        copy_gmres_params(solver, solver->own);
        st = jxcpr_solver_setup(solver->own, A->num_rows, A->block_size, A->num_nonzeros, A->i, A->j, A->data, 0);
        if (st) return st;
        Solver &S = solver->own->s;
        S.ext_precond = nullptr;
        if (solver->precond) {
            const int n = A->num_rows * A->block_size;
            std::vector<double> hr(n), hz(n);
            jxf_ParVector *pr = jxf_ParVectorCreate(0, n, nullptr), *pz = jxf_ParVectorCreate(0, n, nullptr);
            pr->local_vector->data = hr.data();
            pr->local_vector->owns_data = 0;
            pz->local_vector->data = hz.data();
            pz->local_vector->owns_data = 0;
            S.ext_precond = [&, pr, pz](const double *in, double *out) {
                JX_CUDA(cudaMemcpyAsync(hr.data(), in, sizeof(double) * n, cudaMemcpyDeviceToHost, S.stream));
                JX_CUDA(cudaStreamSynchronize(S.stream));
                std::fill(hz.begin(), hz.end(), 0.0);
                solver->precond(solver->precond_data, matA, (JXF_Vector)pr, (JXF_Vector)pz);
                JX_CUDA(cudaMemcpyAsync(out, hz.data(), sizeof(double) * n, cudaMemcpyHostToDevice, S.stream));
            };
            st = jxcpr_solver_solve(solver->own, b->local_vector->data, x->local_vector->data, 0, &it, &rel);
            S.ext_precond = nullptr;
            jxf_ParVectorDestroy(pr);
            jxf_ParVectorDestroy(pz);
        } else {
            st = jxcpr_solver_solve(solver->own, b->local_vector->data, x->local_vector->data, 0, &it, &rel);
        }
    }
    solver->iterations = it;
    solver->rel = rel;
    solver->converged = st == JXCPR_SUCCESS;
    if (solver->print_level > 0)
        printf("GMRES (GPU): %d iterations, final relative residual %.6e\n", it, rel);
    return st == JXCPR_ERROR_CONV ? JXCPR_SUCCESS : st;  // the reference reports non-convergence through GetConverged
}

JXF_Int JXF_GMRESGetNumIterations(JXF_Solver solver, JXF_Int *num_iterations) {
    if (!solver || !num_iterations) return JXCPR_ERROR_ARG;
    *num_iterations = solver->iterations;
    return JXCPR_SUCCESS;
}

JXF_Int JXF_GMRESGetFinalRelativeResidualNorm(JXF_Solver solver, JXF_Real *norm) {
    if (!solver || !norm) return JXCPR_ERROR_ARG;
    *norm = solver->rel;
    return JXCPR_SUCCESS;
}

JXF_Int JXF_GMRESGetConverged(JXF_Solver solver, JXF_Int *converged) {
    if (!solver || !converged) return JXCPR_ERROR_ARG;
    *converged = solver->converged;
    return JXCPR_SUCCESS;
}

// ---------------------------------------------------------------------------
// JXFPAMG_Solver_Interface: CSR of `row` scalar rows -> b x b BSR -> CPR-GMRES
// ---------------------------------------------------------------------------
JXF_Int JXFPAMG_Solver_Interface(JXF_Int, char *[], MPI_Comm, JXF_Int row, JXF_Int *ia, JXF_Int *ja, JXF_Real *a,
                                 JXF_Real *ser_x, JXF_Real *ser_b, JXF_Real tol, JXF_Int solver_id,
                                 JXF_Int num_functions, JXF_Int *iter) {
    if (row < 0 || !ia || !ja || !a || !ser_x || !ser_b) return JXCPR_ERROR_ARG;
    if (solver_id != 220) {
        set_error("JXFPAMG_Solver_Interface: solver_id %d not provided by this build (220 = CPR-GMRES is)",
                  solver_id);
        return JXCPR_ERROR_ARG;
    }
    const int bs = num_functions;
    if (bs < 2 || bs > 3 || row % bs) {
        set_error("JXFPAMG_Solver_Interface: num_functions %d must be 2 or 3 and divide row = %d", bs, row);
        return JXCPR_ERROR_ARG;
    }
    // 1-based input converted in place, as the reference does (jxpamg_interface.c:143-150)
    if (ia[0] == 1) {
        const int nnz = ia[row] - 1;
        for (int k = 0; k <= row; ++k) ia[k]--;
        for (int k = 0; k < nnz; ++k) ja[k]--;
    }
    // diagonal entry of each row moved to the front in place (jxf_CSRMatrixReorder)
    for (int r = 0; r < row; ++r)
        for (int k = ia[r]; k < ia[r + 1]; ++k)
            if (ja[k] == r) {
                std::swap(ja[k], ja[ia[r]]);
                std::swap(a[k], a[ia[r]]);
                break;
            }
    // block rows: node I holds scalar rows I*bs .. I*bs+bs-1; blocks: diagonal first, then ascending columns
    const int nb = row / bs, bn = bs * bs;
    std::vector<int> bia(nb + 1, 0), bja;
    std::vector<double> ba;
    std::vector<int> cols;
    for (int I = 0; I < nb; ++I) {
        cols.clear();
        for (int q = 0; q < bs; ++q)
            for (int k = ia[I * bs + q]; k < ia[I * bs + q + 1]; ++k) cols.push_back(ja[k] / bs);
        cols.push_back(I);
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        std::vector<int> order;
        order.push_back(I);
        for (int J : cols)
            if (J != I) order.push_back(J);
        const int base = (int)bja.size();
        for (int J : order) bja.push_back(J);
        ba.resize(bja.size() * bn, 0.0);
        for (int q = 0; q < bs; ++q)
            for (int k = ia[I * bs + q]; k < ia[I * bs + q + 1]; ++k) {
                const int J = ja[k] / bs, m = ja[k] % bs;
                const int slot = (int)(std::find(order.begin(), order.end(), J) - order.begin());
                ba[(size_t)(base + slot) * bn + q * bs + m] += a[k];
            }
        bia[I + 1] = (int)bja.size();
    }
    jxcpr_solver *h = new_solver();
    if (!h) return JXCPR_ERROR_MEMORY;
    // the reference's case 220 (jxpamg_interface.c:1967-2043) with JXFPAMG_Solver's defaults
    jxcpr_solver_set_int(h, "pressure_index", 0);
    jxcpr_solver_set_int(h, "stage1_maxit", 1);
    jxcpr_solver_set_int(h, "stage2_maxit", 1);
    jxcpr_solver_set_int(h, "stage1_solver_type", 1);
    jxcpr_solver_set_int(h, "stage2_solver_type", 2);
    jxcpr_solver_set_int(h, "k_dim", 30);
    jxcpr_solver_set_int(h, "max_iter", 1000);
    jxcpr_solver_set_int(h, "is_check_restarted", 1);
    jxcpr_solver_set_real(h, "tol", tol);
    apply_env_options(h);
    int st = jxcpr_solver_setup(h, nb, bs, (long long)bja.size(), bia.data(), bja.data(), ba.data(), 0);
    int it = 0;
    double rel = 0.0;
    if (st == JXCPR_SUCCESS) {
        std::vector<double> x(row, 0.0);
        st = jxcpr_solver_solve(h, ser_b, x.data(), 0, &it, &rel);
        if (st == JXCPR_SUCCESS || st == JXCPR_ERROR_CONV) memcpy(ser_x, x.data(), sizeof(double) * row);
    }
    jxcpr_solver_destroy(h);
    if (iter) *iter = it;
    return st == JXCPR_ERROR_CONV ? JXCPR_SUCCESS : st;
}

}  // extern "C"
