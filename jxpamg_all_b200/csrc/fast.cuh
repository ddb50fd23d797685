// Throughput and mixed-precision CPR preconditioner ("fast path").
//
// The exact-order path (smoother_order 0) reproduces the reference's
// preconditioner bit for bit and lives in amg.cu / smoother.cu.  The fast path
// keeps the reference's algorithm -- restrict -> AMG V(1,1) on the pressure
// hierarchy -> prolong -> block Gauss-Seidel stage 2 (jxfpamg-0220/csrc/cpr/
// jxf_cpr.c:424-610) -- on the SAME hierarchy (strength, HMIS, ext+i, RAP from
// amg_setup.cu), but relaxes it with parallel orderings and stores it in a
// precision chosen per level:
//
//   precision 0: values, vectors and arithmetic in FP64 (plain FP64 path);
//   precision 1: FP32 values / vectors / accumulation throughout the
//                preconditioner (GMRES, its SpMV, the true residual and the
//                coarsest dense solve stay FP64);
//   precision 2: as 1, plus BF16 values with a per-block FP32 scale on levels
//                >= bf16_level;
//   precision 3: the reference's hybrid form (src/test_bsr_cprgmres_hybrid.c:
//                217-439): restriction, AMG and prolongation in FP32, the
//                stage-2 sweeps in FP64 on the FP64 block matrix (that driver
//                polishes with weights 1.0 / 0.8, stage2_relax_weight /
//                stage2_omega).
//
// Level smoothers: multicolour Gauss-Seidel (sparse levels, one launch per
// colour class over a colour-contiguous row copy), l1-Jacobi (dense levels),
// or a degree-3 polynomial (Chebyshev) smoother u += p(D^-1 A) D^-1 (f - A u)
// with per-level coefficients (given intervals, or predicted by the learned
// model).  Stage 2 is the reference's hybrid block GS (w, omega) in chunk order
// (chunks of consecutive block rows visited in natural order, the chunks
// coloured; fk::hgs_chunk), or in the level-0 colour order (stage2_chunk 0).
#pragma once

#include <cuda_bf16.h>

#include <string>
#include <vector>

#include "amg.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

enum ValKind { VAL_F64 = 0, VAL_F32 = 1, VAL_BF16 = 2 };
enum FastSmoother { FS_COLOR_GS = 1, FS_L1_JACOBI = 2, FS_CHEB = 3 };

// Operator of the fast path in one value precision and one of two layouts:
//   CSR with `lanes` lanes per row (short or few rows), or
//   sliced ELL (sell = 1): 32-row slices stored slot-major, rows sorted by
//   length inside windows of each segment so that a slice wastes little padding.
// Stored row t maps to vector row perm[t] (CSR; nullptr = identity) or rows[t]
// (sliced ELL; -1 = padding).  Segments (colour classes) are contiguous stored
// rows [seg[c], seg[c+1]).  E values per entry (1 scalar, bs*bs blocks).
// BF16 values carry one power-of-two FP32 scale per block of 32 consecutive stored values
// (a = bscale[k / 32] * val[k]; in sliced ELL a block is one slot of a 32-row slice).
struct LevelMat {
    int n = 0, m = 0;
    long long nnz = 0;
    int E = 1;
    int kind = VAL_F64;
    int sell = 0;
    int chunk = 0;  // sliced ELL in chunk order (stage 2, fk::hgs_chunk): rows per chunk
    int lanes = 1;
    int nstored = 0;
    const int *perm = nullptr;  // CSR: not owned
    DevBuf<int> ia, ja;         // CSR pattern; sliced ELL: columns in ja
    DevBuf<long long> sp;       // sliced ELL: slice offsets (entries)
    DevBuf<int> rows;           // sliced ELL: vector row of each stored row
    std::vector<int> seg;
    DevBuf<double> a64;
    DevBuf<float> a32;
    DevBuf<__nv_bfloat16> a16;
    DevBuf<float> bscale;
};

// One level of the fast hierarchy (vectors in TX = double or float).
template <typename TX>
struct FastLevel {
    int n = 0;
    int smoother = FS_L1_JACOBI;  // in use
    int smoother_cfg = FS_L1_JACOBI, smoother_plain = FS_L1_JACOBI;  // configured / plain settings
    LevelMat A;          // colour classes as segments (FS_COLOR_GS) or one segment
    const int *src_ia = nullptr, *src_ja = nullptr;  // the hierarchy's CSR operator's pattern (not owned)
    int last_color = -1;
    LevelMat P, R;       // interpolation from level+1 / restriction to it
    DevBuf<TX> dinv;     // 1/a_ii (GS, Chebyshev); 0 skips the row
    DevBuf<TX> dinv_l1;  // 1/sum_j |a_ij| (l1-Jacobi)
    double cheb[3] = {0, 0, 0};  // p(t) = c0 + c1 t + c2 t^2
    double cheb_lo = 0, cheb_hi = 0, lambda_max = 0;
    DevBuf<TX> f, u, r, z, y1, y2;
    DevBuf<TX> c;        // level 0: correction of repeated stage-1 cycles
};

struct FastOptions {
    int precision = 0;      // 0 FP64, 1 FP32, 2 FP32 + BF16 coarse levels, 3 FP32 stage 1 + FP64 stage 2
    int bf16_level = 1;     // precision 2: first level stored in BF16
    int smoother = 0;       // 0 colour GS / l1-Jacobi, 1 Chebyshev-3 on the l1-Jacobi levels, 2 on every level
    double cheb_lower = 0.3, cheb_upper = 1.1;  // interval [lower, upper] * lambda_max(D^-1 A)
    int stage2_lanes = 4;      // CSR stage 2 (small systems): lanes per block row
    int stage2_chunk = 4;      // stage 2 in chunk order (chunks of this many consecutive block rows; 0: the
                               // level-0 colour order)
    int sell_min_rows = 16384; // without autotuning: sliced ELL for operators with at least this many rows ...
    double sell_max_mean = 40; // ... and at most this mean row length
    int sell_lanes = 1;        // ... with this many lanes per row (1 or 2; FP32 / FP64 values)
    int graphs = 1;            // replay each preconditioner application as one captured CUDA graph
    int dep_launch = 1;        // kernels of an application launched as programmatic dependents (launch_dep)
    int tail_rows = 0;         // levels from the first with at most this many rows run as one cooperative kernel (0: off)
    int tail_ctas = 0;         // its grid (0: enough for the largest fused pass, at most the co-resident blocks)
    int autotune = 1;          // time the layouts (CSR with 1..32 lanes, sliced ELL) of every operator, keep the fastest;
                               // 2: share the choice among operators of one shape class (batches)
    // per-level Chebyshev interval overrides (learned); empty = use cheb_lower/upper
    std::vector<double> level_lower, level_upper;
    // per-level lambda_max(D^-1 A) after 12 power steps, from the learned-features pass (0: compute)
    std::vector<double> level_lambda;
};

// Precision-independent interface.
struct FastCprBase {
    virtual ~FastCprBase() = default;
    virtual void apply(const double *r, double *z, cudaStream_t s) = 0;
    // The application's kernels queued on s, never through the private graph:
    // for callers that capture the application into a graph of their own.
    virtual void apply_enqueue(const double *r, double *z, cudaStream_t s) = 0;
    virtual void vcycle(const double *fp, double *up, cudaStream_t s) = 0;  // FP64 pressure in/out
    virtual void stage2_sweep(const double *r, double *z, cudaStream_t s) = 0;
    virtual int num_levels() const = 0;
    virtual void level_info(int l, int *smoother, int *kind, double *cheb) const = 0;
    // Asymptotic convergence factor of the V-cycle on A_0 e = 0 (power method, `cycles` cycles)
    virtual double vcycle_factor(int cycles, cudaStream_t s) = 0;
    // plain = true: the plain smoothers (colour GS / l1-Jacobi) on every level, on
    // the same storage; false: the configured ones (Chebyshev / learned)
    virtual void set_plain_mode(bool plain) = 0;
    // Modelled bytes one application moves (operator and vector traffic of
    // every smoother pass, residual, transfer and stage-2 sweep).
    virtual double apply_bytes() const = 0;
    // `sweeps` stage-2 sweeps in the preconditioner's own precision on internal
    // vectors (no conversions), queued on s: the kernel the roofline times.
    virtual void stage2_native(int sweeps, cudaStream_t s) = 0;
    // `reps` passes over level l's operator in its storage precision on the level's own work vectors,
    // queued on s (what a roofline measurement times): op 0 y = A x, 1 one Chebyshev step
    // (y = c z + D^-1 A x), 2 the residual r = f - A u.  Returns false if the level has no operator.
    virtual bool level_native(int level, int op, int reps, cudaStream_t s) = 0;
    // Level l's operator values as stored (FP64, FP32, or BF16 times its block scale), widened to FP64 in
    // the entry order of the hierarchy's CSR operator (out: device, nnz values).  False if no operator.
    virtual bool stored_values(int level, double *out, cudaStream_t s) = 0;
    // One line per tuned operator: "name rows mean_row layout time_us".
    std::vector<std::string> tune_log;
};

struct CprConfig {
    int pressure_index = 0;
    int stage1_maxit = 1;
    int stage2_maxit = 3;
    int stage2_solver_type = 2;
    double stage2_w = 0.7, stage2_omega = 0.9;
};

// Builds the fast preconditioner on an existing hierarchy (H.levels[l]->A, P, R,
// fwd schedules of the colour levels, coarse inverse Ainv) and the decoupled
// block matrix A.
FastCprBase *make_fast_cpr(Amg &H, const BsrView<double> &A, const CprConfig &cfg, const FastOptions &opt,
                           cudaStream_t s);

// Largest eigenvalue estimate of D^-1 A (D = diag), FP64 power iteration.
double estimate_lambda_max(const CsrView<double> &A, int iters, cudaStream_t s, int iters2 = 0,
                           double *lam2 = nullptr);
// Coefficients of the degree-2 polynomial p with 1 - t p(t) = the degree-3
// Chebyshev polynomial of [lo, hi] normalised to 1 at t = 0.
void chebyshev3_coefficients(double lo, double hi, double c[3]);

}  // namespace jxcpr
