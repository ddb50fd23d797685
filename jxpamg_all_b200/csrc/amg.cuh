// AMG hierarchy, smoother schedules and the setup / cycle entry points.
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

// Sparsity pattern only (strength matrix).
struct DevPattern {
    int n = 0;
    long long nnz = 0;
    DevBuf<int> ia, ja;
};

// Rows grouped so that rows of one group can be relaxed concurrently and the
// groups, taken in order, reproduce a Gauss-Seidel sweep.
struct Schedule {
    int ngroups = 0;
    int max_group = 0;
    DevBuf<int> perm;       // rows, group by group
    DevBuf<int> group_ptr;  // ngroups + 1 offsets into perm
    DevBuf<int> rank;       // per row: neighbours of lower rank are read updated
    std::vector<int> h_group_ptr;
};

enum SmootherOrder {
    // Level schedule of the natural ordering: identical results to the
    // reference's sequential sweeps.
    ORDER_EXACT = 0,
    // Greedy multicolour ordering: Gauss-Seidel in colour order, far fewer
    // groups (a different but equally valid smoother).
    ORDER_MULTICOLOR = 1,
};

enum LevelSmoother {
    SMOOTH_EXACT_GS = 0,  // sequential-order Gauss-Seidel (level schedule, bit-exact)
    SMOOTH_COLOR_GS = 1,  // multicolour Gauss-Seidel, one launch per colour
    SMOOTH_L1_JACOBI = 2, // l1-Jacobi (dense coarse levels in multicolour mode)
};

struct AmgLevel {
    int smoother = SMOOTH_EXACT_GS;
    double theta = 0.25;  // strength threshold this level was coarsened with
    DeviceCsr A;          // level operator (diagonal first in every row)
    DeviceCsr P;          // interpolation to this level from level+1 (n x nc)
    DeviceCsr R;          // P^T, rows listing fine points ascending
    std::vector<int> cf;  // host copy of the C/F splitting (tests)
    Schedule fwd, bwd;    // Gauss-Seidel schedules
    std::vector<int> chunk_order, chunk_seg;  // level 0 of the fast path: stage-2 chunk order (host)
    DevBuf<double> f, u;  // right-hand side and iterate of this level
};

struct AmgParams {
    int max_levels = 25;
    int coarse_threshold = 1000;
    double strong_threshold = 0.25;
    double max_row_sum = 0.9;
    int order = ORDER_EXACT;
    int coarse_exact = 1;  // 1: substitution in the reference's order; 0: explicit inverse (GEMV)
    int max_colors = 8;    // multicolour mode: levels needing more colours use l1-Jacobi
    double jacobi_mean_row = 12.0;  // multicolour mode: levels with longer mean rows go straight to l1-Jacobi
    int rs_range_rows = 0;  // > 0: the coarsening's first pass runs on row ranges of this size (host threads)
    int rs_range_rows_coarse = 0;  // the same on the levels below the finest
    int stage2_chunk = 0;   // > 0 (fast path): level 0 also gets the stage-2 chunk order (build_chunk_order_host)
    // Optional per-level strength thresholds: called before level l is
    // coarsened with its operator; returns the threshold to use (learned model).
    std::function<double(int level, const CsrView<double> &A)> theta_for_level;
};

// Wall-clock phase log of a setup (host time between marks, stream drained at each mark).
struct PhaseLog {
    std::vector<std::pair<std::string, double>> items;
    double t_last = 0.0;
    void start();
    void mark(const char *name, cudaStream_t s);
};

struct Amg {
    AmgParams prm;
    PhaseLog log;
    std::vector<std::unique_ptr<AmgLevel>> levels;
    // coarsest level dense factors (row-major n x n), L stored transposed
    int nc = 0;
    DevBuf<double> Ufac, Lt, Ainv;
    DevBuf<double> work;  // residual of the finest level
    DevBuf<int> err;      // [0] device error flag of the smoothers, [2..3] their grid barrier
    int num_levels() const { return (int)levels.size(); }
};

// amg_setup.cu
void amg_strength(const CsrView<double> &A, double theta, double max_row_sum, DevPattern &S, cudaStream_t s);
void amg_pmis(const DevPattern &S, int *cf_dev, cudaStream_t s);
int amg_extpi_interp(const CsrView<double> &A, const DevPattern &S, const int *cf_dev, DeviceCsr &P,
                     cudaStream_t s);
void amg_rap(const CsrView<double> &A, const DeviceCsr &P, const DeviceCsr &R, DeviceCsr &Ac, cudaStream_t s,
             long long table_budget_entries = (1LL << 27));

// setup_host.cu (sequential graph passes)
void rs_first_pass_host(int n, const int *sia, const int *sja, int *cf, const int *gia = nullptr);
void rs_first_pass_host(int n, const int *sia, const int *sja, const int *stia, const int *stja, int *cf,
                        const int *gia = nullptr);
// The first pass on row ranges of range_rows rows (n / range_rows ranges; one range: the whole pattern).
void rs_first_pass_ranges(int n, const int *sia, const int *sja, int range_rows, int *cf);
void build_schedule_host(int n, const int *ia, const int *ja, int order, bool forward, std::vector<int> &perm,
                         std::vector<int> &group_ptr, std::vector<int> &rank);
void upload_schedule(const std::vector<int> &perm, const std::vector<int> &gptr, const std::vector<int> &rank,
                     Schedule &S, cudaStream_t s);
// Stage-2 order of the throughput path: chunks of `chunk` (a divisor of 32) consecutive rows, coloured;
// order = stored rows (colour by colour, chunk by chunk, -1 padding), seg = colour segment offsets.
void build_chunk_order_host(int n, const int *ia, const int *ja, int chunk, std::vector<int> &order,
                            std::vector<int> &seg);

// coarse_mma.cu: explicit inverse by blocked Gauss-Jordan (no pivoting) in one cooperative kernel with
// FP64 tensor-core (DMMA) trailing updates.  err: 4 device ints (flags, grid barrier); a zero pivot
// throws std::invalid_argument, a barrier time-out CudaError.
void coarse_inverse_mma(const CsrView<double> &A, double *Ainv, int *err, cudaStream_t s);
void dense_inverse_mma(int n, const double *A, double *Ainv, cudaStream_t s);

// amg.cu
void amg_setup(Amg &H, DeviceCsr &&A0, cudaStream_t s);
void amg_vcycle(Amg &H, const double *f0, double *u0, cudaStream_t s);  // one V(1,1), u0 in/out
void coarse_setup(Amg &H, cudaStream_t s);
void coarse_solve(Amg &H, const double *f, double *u, cudaStream_t s);

// smoother_fast.cu
int lanes_for(double mean_row);
void permute_rows_csr(const CsrView<double> &A, const int *perm, DeviceCsr &P, cudaStream_t s);
void permute_rows_bsr(const BsrView<double> &A, const int *perm, DeviceBsr &P, cudaStream_t s);

// smoother.cu
// err: the hierarchy's 4-int device buffer (err[0] the error flag; err[2..3] the grid barrier of the
// cooperative sweeps, reset by each launch on `s`), so solvers on concurrent streams do not share it.
// One Gauss-Seidel sweep of A u = f along `sch` (relax_weight = omega = 1,
// rows with a zero diagonal skipped): jxf_PAMGRelax6's forward or backward
// pass.
void gs_sweep(const CsrView<double> &A, const Schedule &sch, const double *f, double *u, const int *rank,
              double *vt, int *err, cudaStream_t s);
// Stage-2 block hybrid Gauss-Seidel (jxf_ParBSRHGSRelax) along `sch`; vt is
// scratch (nb*bs) that receives the iterate at sweep start.
void hgs_sweep(const BsrView<double> &A, const Schedule &sch, const double *b, double *x, const int *rank,
               double *vt, double w, double omega, int *err, cudaStream_t s);
// Stage-2 block hybrid symmetric Gauss-Seidel (jxf_ParBSRHSGSRelax, par_relax_bsr.c:579-1062): a
// forward pass along `fwd`, then a backward pass along `bwd`.  vt: scratch (nb*bs); work: the CPR's
// work vector (nb*bs, zero when created), of which only the first nb entries are refreshed from x,
// as the reference does, and which feeds the res2 term of the weighted update.
void hsgs_sweep(const BsrView<double> &A, const Schedule &fwd, const Schedule &bwd, const double *b, double *x,
                double *vt, double *work, double w, double omega, int *err, cudaStream_t s);

}  // namespace jxcpr
