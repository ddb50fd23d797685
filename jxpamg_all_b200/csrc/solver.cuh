// CPR preconditioner and restarted GMRES on one GPU.
#pragma once

#include <string>
#include <vector>

#include <functional>
#include <memory>

#include "amg.cuh"
#include "bilu.cuh"
#include "common.cuh"
#include "fast.cuh"
#include "kernels.cuh"
#include "learned.cuh"

namespace jxcpr {

struct SolverParams {
    // GMRES (jxfpamg-0220/csrc/krylov/pgmres.c:431-470 defaults; the CPR
    // driver sets k_dim 30, is_check_restarted 1, src/test_bsr_cprgmres.c:351-367)
    int k_dim = 30;
    int max_iter = 100;
    int min_iter = 0;
    double tol = 1e-6;
    double a_tol = 0.0;
    int is_check_restarted = 1;
    double convfac_threshold = 1e4;
    // Internal (not an option): > 0 ends the solve with `stalled` set when a full restart cycle leaves
    // a residual ratio (end / start) above stall_ratio (the learned settings' guard, Solver::solve).
    double stall_ratio = 0.0;
    int print_level = 0;
    int logging = 1;
    // CPR (jxfpamg-0220/csrc/cpr/jxf_cpr.c:151-182, 226-262)
    int pressure_index = 0;
    int stage1_maxit = 1;
    int stage2_maxit = 3;
    int stage1_solver_type = 1;  // 1: AMG
    int stage2_solver_type = 2;  // 2: block hybrid Gauss-Seidel (HGS); 3: symmetric HGS (HSGS, exact-order
                                 // mode); 5: block ILU(0) correction (BILU)
    // BILU stage 2 (jxf_BILUSetup type 3 / jxf_BILUSolve tri-solve 14 parameters)
    int bilu_sweeps = 3;
    int bilu_ir_iters = 5;
    int bilu_lower_iters = 5;
    int bilu_upper_iters = 5;
    int bilu_exact = 0;  // 1: exact BILU(0) factors and level-scheduled triangular solves (bilu_exact.cu)
    double threshold = 1e-15;    // accepted and ignored, as in the reference
    double stage2_relax_weight = 0.7;
    double stage2_omega = 0.9;
    // decoupling applied by the solver object (JXF_DecoupType: 0 none, 1 ABF, 2 ANL, 3 SEM, 4 QI,
    // 5 True-IMPES, 6 True-IMPES second form); thermal: the last unknown is temperature (types 2-4)
    int decouple = 0;
    int thermal = 0;
    int consistent_rhs = 0;
    // AMG strength threshold (jxf_cpr.c:331 sets 0.25)
    double strong_threshold = 0.25;
    double strong_threshold_coarse = -1.0;  // levels >= 1 (fast path); < 0: strong_threshold
    // device execution choices
    int smoother_order = ORDER_EXACT;  // 0 exact order (bit-identical), 1 throughput / mixed path
    int coarse_exact = 1;
    int max_colors = 8;
    double jacobi_mean_row = 12.0;  // multicolour mode: levels with longer mean rows use l1-Jacobi
    // fast path: the coarsening's first pass on row ranges of this many rows, one host thread per
    // range (levels with fewer than twice as many rows, and the exact order always, take one pass)
    int rs_range_rows = 131072;
    int rs_range_rows_coarse = 0;  // the levels below the finest (0: rs_range_rows)
    int dep_launch = 1;  // fast path: programmatic dependent launches inside each CPR application
    int use_tma_spmv = 0;
    // fast path (smoother_order 1)
    int precision = 0;       // 0 FP64, 1 FP32 preconditioner, 2 FP32 + BF16 coarse levels, 3 the reference's
                             // hybrid form: FP32 restriction / AMG / prolongation, FP64 stage 2 on the FP64 matrix
    int bf16_level = 1;      // precision 2: first BF16 level
    int fast_smoother = 0;   // 0 colour GS / l1-Jacobi; 1 Chebyshev-3 on the levels without a GS colouring;
                             // 2 as 1 with learned thresholds and intervals; 3 Chebyshev-3 on every level
    int autotune = 1;        // fast path: time the operator layouts at setup and keep the fastest (2: share per shape class)
    int graphs = 1;          // fast path: each CPR application replays one captured CUDA graph
    int orthog = 0;          // 0 modified Gram-Schmidt (the reference's), 1 classical Gram-Schmidt (one pass)
    int flexible = 0;        // 1: flexible GMRES (stores M^-1 v_j; for inexact / low-precision preconditioners)
    int graph_gmres = 0;     // 1: the whole GMRES solve on the device as one CUDA graph (fast path; flexible, CGS2)
    int krylov_fp32 = 0;     // graph GMRES: basis and flexible directions stored in FP32 (products, norms,
                             // Hessenberg, rotations, residuals and x in FP64)
    int selective_reorth = 0;  // graph GMRES: the second Gram-Schmidt pass only when the first removed
                               // more than half of ||w||^2 (0: always, classical Gram-Schmidt twice)
    double cheb_lower = 0.3; // Chebyshev interval [lower, upper] * lambda_max(D^-1 A)
    double cheb_upper = 1.1;
    int stage2_lanes = 4;
    int stage2_chunk = 4;      // fast path: stage 2 in chunk order (4, 8 or 16 consecutive block rows; 0 colour order)
    int tail_rows = 0;         // fast path: the V-cycle's levels from the first with at most this many rows
                               // (the coarsest included) run as one cooperative kernel (0: one launch per pass)
    int tail_ctas = 0;         // its grid (0: sized by the largest fused pass, at most the co-resident blocks)
    int sell_lanes = 1;        // fast path without autotuning: lanes per row of the sliced-ELL operators (1 or 2)
    int learned_fallback = 1;  // learned mode: keep the plain smoothers when their V-cycle factor is lower
    int record_features = 0;   // fast path: record the per-level features (training data)
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { cudaEventRecord(a, s); }
    float stop_ms(cudaStream_t s) {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

// CPR two-stage preconditioner: restrict -> AMG V-cycle -> prolong -> stage 2.
struct CprPrecond {
    SolverParams prm;
    BsrView<double> A;  // decoupled system matrix (owned by the solver)
    Amg amg;
    std::unique_ptr<FastCprBase> fast;  // smoother_order 1: throughput / mixed-precision preconditioner
    bool probe_pending = false;  // learned mode: the plain-vs-learned probe runs after GMRES setup
    std::unique_ptr<Bilu> bilu;         // stage2_solver_type 5
    DevBuf<double> bres, bdelta;        // BILU stage: r - A z and its correction
    double factor_fast = 0.0, factor_plain = 0.0;  // learned mode: GMRES residual reduction per iteration
    double probe_bytes[2] = {0, 0};                 // modelled bytes per GMRES iteration (learned, plain)
    int learned_used = 0;
    LearnedPlan plan;  // per-level features and learned settings of the last setup
    DevBuf<double> rp, xp, vt;
    DevBuf<double> hsgs_work;  // stage2_solver_type 3: the reference's persistent Vtemp vector
    double stats[4] = {0, 0, 0, 0};  // stage1 setup, stage1 solve, stage2 setup, stage2 solve (seconds)
    bool ready = false;
    void setup(const BsrView<double> &A_, cudaStream_t s);
    void apply(const double *r, double *z, cudaStream_t s);
    // one stage-2 block hybrid Gauss-Seidel sweep on A z = r (z in/out)
    void stage2_sweep(const double *r, double *z, cudaStream_t s);
    void bilu_stage(const double *r, double *z, cudaStream_t s);
    // apply() with every kernel queued on s (fast path only; no private graph), for capture
    void apply_enqueue(const double *r, double *z, cudaStream_t s);
    // one pressure V-cycle on A_p u = f, u in/out (FP64)
    void vcycle(const double *f, double *u, cudaStream_t s);
    int *err() { return amg.err.get(); }
};

struct GmresResult {
    int iterations = 0;
    int converged = 0;
    int stalled = 0;  // ended by the stall rule (stall_ratio)
    double rel_residual = 0.0;
    std::vector<double> norms;
    int status = 0;
};

// Restarted right-preconditioned GMRES(k) with modified Gram-Schmidt and
// Givens rotations (jxfpamg-0220/csrc/krylov/pgmres.c:950-1713).
struct Gmres {
    SolverParams prm;
    int n = 0;
    // Krylov basis p_0..p_k and (flexible GMRES) z_j = M^-1 p_j: slices of one allocation
    struct VecRef {
        double *ptr;
        double *get() const { return ptr; }
    };
    DevBuf<double> basis;
    std::vector<VecRef> p;
    std::vector<VecRef> zf;
    DevBuf<double> r, w, partials, scal;  // scal: device scalars (dots)
    DevBuf<const double *> vptrs;         // device array of the basis pointers (classical Gram-Schmidt)
    int cgs_blocks = 1;
    int *kerr = nullptr;
    void setup(int n_, cudaStream_t s);
    // ext (optional): any other right preconditioner z = M^-1 r on device vectors
    GmresResult solve(const BsrView<double> &A, CprPrecond *M, const double *b, double *x, cudaStream_t s,
                      const std::function<void(const double *, double *)> *ext = nullptr);
};

struct Solver;

// Device-side state of the graph GMRES (one per solve).
constexpr int kGgMaxK = 64;
struct GgState {
    int i, m, iter, cycles;
    int converged, done, status, first;
    int est_conv, conv_fail, cont, stalled;
    int iter0;       // iterations at the current cycle's start
    int skip;        // this step keeps the first Gram-Schmidt pass (selective second pass)
    double b_norm, r_norm, r_norm0, epsilon, normdown, scale, rel;
    double r_cycle;  // true residual norm at the current cycle's start (stall rule)
    double sig;      // ||w||^2 of a step that skips the second pass
    unsigned long long t_start, t_end;  // device global timer (ns) at the solve's start and end
};
struct GgParams {
    int k, max_iter, min_iter, check_restarted;
    double tol, a_tol, convfac;
    double stall;  // SolverParams::stall_ratio
    int selective;  // SolverParams::selective_reorth
};
struct GgWork {  // device arrays: rotations, Hessenberg matrix, coefficients
    double *rs, *c, *sn, *h1, *h2, *y, *hh;
};

// Restarted flexible GMRES(k) run on the device without host round trips:
// the whole solve is recorded into a CUDA graph (nested conditional WHILE
// nodes for the restart cycles and the Arnoldi steps).  Single-system solves
// replay a graph of their own; batches record many solvers into one graph.
struct GraphGmres {
    long long n = 0;
    int k = 0, max_iter = 0, G = 1, G1 = 1, G2 = 1, Gq = 1;
    GgParams P{};
    GgWork W{};
    DevBuf<GgState> state;
    DevBuf<double> work, partials, norms, summary, cin, cout;
    std::vector<DevBuf<double>> own_z;  // flexible directions when the host GMRES keeps none
    DevBuf<double *> vptr, zptr;
    int fp32 = 0;              // krylov_fp32: v_0..v_k and z_0..z_{k-1} stored in FP32 (basis32)
    DevBuf<float> basis32;
    DevBuf<float *> vptr32, zptr32;
    cudaStream_t aux[2] = {nullptr, nullptr};  // capture streams of the loop bodies
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels_fixed = 0, kernels_cycle = 0, kernels_step = 0;
    ~GraphGmres();
    void reset_graph();
    // buffers and parameters for the solver's current setup (throws if it has no fast CPR)
    void prepare(Solver &S);
    bool matches(const SolverParams &prm) const;
    // Records decoupling of S.b, the solve of A x = b into S.x and an 8-value
    // summary written to `out` into the capture running on s.
    void record(Solver &S, cudaStream_t s, double *out);
    void build_single(Solver &S);
    unsigned long long kernels_run(int iterations, int cycles) const;
    // `reps` times the orthogonalisation kernels of one Arnoldi step with m basis vectors (first
    // products, fused update + second products, final update into v_m), outside the graph, on the
    // basis the last solve left and the work vector w (profiling and roofline timing)
    void orth_native(int m, int reps, const double *w, cudaStream_t s);
    // summary: iterations, converged, rel. residual, status, t_start, t_end, cycles, device error flags
    GmresResult result_from(const double *summary_host, cudaStream_t s, bool with_norms);
};

// Full solver object: owns the device matrix, decoupling coefficients, CPR, GMRES.
struct Solver {
    SolverParams prm;
    DeviceBsr A;
    DevBuf<double> dcoef;  // decoupling weights per block row
    CprPrecond cpr;
    Gmres gmres;
    DevBuf<double> b, x;
    DevBuf<int> kerr;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    bool stream_set = false;  // the caller chose the stream (possibly the legacy default stream)
    double setup_ms = 0.0, solve_ms = 0.0, upload_ms = 0.0, decouple_ms = 0.0;
    double alloc_stats[4] = {0, 0, 0, 0};  // during the last setup (process-wide): cudaMalloc calls / ms, device syncs / ms
    GmresResult last;
    // a preconditioner supplied by the caller instead of CPR (stage1_solver_type 0 then applies it)
    std::function<void(const double *, double *)> ext_precond;
    std::unique_ptr<GraphGmres> ggmres;  // graph_gmres 1
    // A on the host or the device (device = 1), copied into the solver.
    void setup(int nb, int bs, long long nnzb, const int *ia, const int *ja, const double *a, int device);
    // b, x host or device; x holds the initial guess on entry.
    GmresResult solve(const double *b_in, double *x_io, int device);
    GmresResult solve_once(const double *b_in, double *x_io, int device);
    int learned_fallbacks = 0;  // solves in which the learned settings stalled and the plain ones took over
    int learned_rebuilt = 0;    // the plain preconditioner replaced the learned one (probe or stall)
    void rebuild_plain(cudaStream_t s);
    void learned_probe(cudaStream_t s);
};

}  // namespace jxcpr
