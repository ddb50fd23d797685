// CPR preconditioner (jxfpamg-0220/csrc/cpr/jxf_cpr.c:268-610) and restarted
// GMRES (jxfpamg-0220/csrc/krylov/pgmres.c:950-1713) driving the device kernels.
//
// GMRES runs its vector work on the device; the Hessenberg / Givens scalars
// (k <= 30 of them) are updated on the host in the reference's exact scalar
// order, so the only difference from the reference's iteration is the
// summation order inside the device dot products.  Modified Gram-Schmidt is
// fused: the update w -= h_{j-1} p_{j-1} and the next product <p_j, w> share
// one pass over w.
#include <math.h>

#include <algorithm>
#include <chrono>

#include <stdexcept>

#include "solver.cuh"

namespace jxcpr {

// ---------------------------------------------------------------------------
// CPR
// ---------------------------------------------------------------------------
void CprPrecond::setup(const BsrView<double> &A_, cudaStream_t s) {
    A = A_;
    Timer t;
    t.start(s);
    const bool fast_path = prm.smoother_order != ORDER_EXACT;
    if (fast_path && prm.stage2_solver_type == 3) {
        set_error("stage2_solver_type 3 (HSGS) is provided in the exact-order mode (smoother_order 0) only");
        throw std::invalid_argument("hsgs");
    }
    amg.prm.order = prm.smoother_order;
    amg.prm.coarse_exact = fast_path ? 0 : prm.coarse_exact;
    amg.prm.max_colors = prm.max_colors;
    amg.prm.jacobi_mean_row = prm.jacobi_mean_row;
    amg.prm.stage2_chunk = fast_path ? prm.stage2_chunk : 0;
    amg.prm.rs_range_rows = fast_path ? prm.rs_range_rows : 0;
    amg.prm.rs_range_rows_coarse = fast_path ? (prm.rs_range_rows_coarse > 0 ? prm.rs_range_rows_coarse
                                                                              : prm.rs_range_rows) : 0;
    amg.prm.strong_threshold = prm.strong_threshold;
    amg.prm.theta_for_level = nullptr;
    fast.reset();
    probe_pending = false;
    learned_used = 0;
    factor_fast = factor_plain = 0.0;
    plan = LearnedPlan();
    const double th0 = prm.strong_threshold;
    const double thc = (fast_path && prm.strong_threshold_coarse >= 0.0) ? prm.strong_threshold_coarse : th0;
    if (fast_path && (prm.fast_smoother == 2 || prm.record_features)) {
        plan.active = prm.fast_smoother == 2;
        plan.record = true;
        amg.prm.theta_for_level = [this, th0, thc, s](int level, const CsrView<double> &Al) {
            return learned_predict_level(plan, level, Al, level == 0 ? th0 : thc, s);
        };
    } else if (thc != th0) {
        amg.prm.theta_for_level = [th0, thc](int level, const CsrView<double> &) { return level == 0 ? th0 : thc; };
    }
    DeviceCsr Ap;
    bsr_pressure_csr(A, prm.pressure_index, Ap, s);
    amg_setup(amg, std::move(Ap), s);
    amg.prm.theta_for_level = nullptr;
    if (fast_path) {
        CprConfig cfg;
        cfg.pressure_index = prm.pressure_index;
        cfg.stage1_maxit = prm.stage1_maxit;
        cfg.stage2_maxit = prm.stage2_maxit;
        cfg.stage2_solver_type = prm.stage2_solver_type;
        cfg.stage2_w = prm.stage2_relax_weight;
        cfg.stage2_omega = prm.stage2_omega;
        FastOptions opt;
        opt.precision = prm.precision;
        opt.bf16_level = prm.bf16_level;
        opt.smoother = prm.fast_smoother == 0 ? 0 : (prm.fast_smoother == 3 ? 2 : 1);
        opt.cheb_lower = prm.cheb_lower;
        opt.cheb_upper = prm.cheb_upper;
        opt.stage2_lanes = prm.stage2_lanes;
        opt.stage2_chunk = prm.stage2_chunk;
        opt.tail_rows = prm.tail_rows;
        opt.tail_ctas = prm.tail_ctas;
        opt.sell_lanes = prm.sell_lanes;
        opt.autotune = prm.autotune;
        opt.graphs = prm.graphs;
        opt.dep_launch = prm.dep_launch;
        if (plan.active) {
            opt.level_lower = plan.lower;
            opt.level_upper = plan.upper;
            opt.level_lambda = plan.lambda12;
        }
        fast.reset(make_fast_cpr(amg, A, cfg, opt, s));
        amg.log.mark("fast_build", s);
        if (plan.active) {
            learned_used = 1;
            // plain smoother settings on the same hierarchy and storage; Solver::setup keeps
            // whichever reduces the GMRES residual faster per byte
            probe_pending = prm.learned_fallback != 0;
        }
    }
    rp.alloc(A.nb > 0 ? A.nb : 1);
    xp.alloc(A.nb > 0 ? A.nb : 1);
    vt.alloc((size_t)(A.nb > 0 ? A.nb : 1) * A.bs);
    hsgs_work.release();
    if (prm.stage2_solver_type == 3) {
        // the CPR's work vector, zero when created (jxf_cpr.c:396); HSGS keeps state in it
        hsgs_work.alloc((size_t)(A.nb > 0 ? A.nb : 1) * A.bs);
        hsgs_work.zero(s);
    }
    stats[0] = t.stop_ms(s) * 1e-3;
    stats[2] = 0.0;  // stage 2 (HGS) needs no setup beyond the level-0 schedule
    bilu.reset();
    if (prm.stage2_solver_type == 5) {
        Timer t2;
        t2.start(s);
        bilu.reset(new Bilu());
        bilu->sweeps = prm.bilu_sweeps;
        bilu->ir_iters = prm.bilu_ir_iters;
        bilu->lower_iters = prm.bilu_lower_iters;
        bilu->upper_iters = prm.bilu_upper_iters;
        bilu->exact = prm.bilu_exact;
        // the mixed path keeps the exact factors in FP32 for the substitutions
        bilu->fp32 = prm.bilu_exact && prm.smoother_order != ORDER_EXACT && (prm.precision == 1 || prm.precision == 2);
        bilu->setup(A, s);
        amg.log.mark("bilu_setup", s);
        bres.alloc((size_t)(A.nb > 0 ? A.nb : 1) * A.bs);
        bdelta.alloc((size_t)(A.nb > 0 ? A.nb : 1) * A.bs);
        stats[2] = t2.stop_ms(s) * 1e-3;
    }
    ready = true;
}

void CprPrecond::apply(const double *r, double *z, cudaStream_t s) {
    if (fast) {
        fast->apply(r, z, s);
        bilu_stage(r, z, s);
        return;
    }
    const int nb = A.nb, bs = A.bs;
    restrict_pressure(nb, bs, prm.pressure_index, r, rp.get(), s);
    JX_CUDA(cudaMemsetAsync(xp.get(), 0, sizeof(double) * nb, s));
    for (int it = 0; it < prm.stage1_maxit; ++it) amg_vcycle(amg, rp.get(), xp.get(), s);
    prolong_pressure(nb, bs, prm.pressure_index, xp.get(), z, s);
    if (prm.stage2_solver_type == 2 || prm.stage2_solver_type == 3)
        for (int it = 0; it < prm.stage2_maxit; ++it) stage2_sweep(r, z, s);
    bilu_stage(r, z, s);
}

void CprPrecond::apply_enqueue(const double *r, double *z, cudaStream_t s) {
    if (!fast) {
        set_error("apply_enqueue: needs the fast CPR preconditioner");
        throw CudaError{cudaErrorInvalidValue, "apply_enqueue"};
    }
    fast->apply_enqueue(r, z, s);
    bilu_stage(r, z, s);
}

// Stage 2 as a block-ILU(0) correction: r' = r - A z, z += BILU^-1 r'
// (the composition of JXF_CPRPrecond without stage-2 sweeps, jxf_ParBSRMatrixMatvec
// and jxf_BILUSolve that the reference's drivers use).
void CprPrecond::bilu_stage(const double *r, double *z, cudaStream_t s) {
    if (!bilu) return;
    const long long n = (long long)A.nb * A.bs;
    copy_dev(n, r, bres.get(), s);
    bsr_spmv<double, double>(A, -1.0, z, 1.0, bres.get(), nullptr, s, false);
    JX_CUDA(cudaMemsetAsync(bdelta.get(), 0, sizeof(double) * n, s));
    bilu->solve(A, bres.get(), bdelta.get(), s);
    axpy_dev(n, 1.0, bdelta.get(), z, s);
}

void CprPrecond::stage2_sweep(const double *r, double *z, cudaStream_t s) {
    if (fast) {
        fast->stage2_sweep(r, z, s);
        return;
    }
    const AmgLevel &L0 = *amg.levels[0];
    if (prm.stage2_solver_type == 3) {
        hsgs_sweep(A, L0.fwd, L0.bwd, r, z, vt.get(), hsgs_work.get(), prm.stage2_relax_weight, prm.stage2_omega,
                   amg.err.get(), s);
        return;
    }
    hgs_sweep(A, L0.fwd, r, z, L0.fwd.rank.get(), vt.get(), prm.stage2_relax_weight, prm.stage2_omega,
              amg.err.get(), s);
}

void CprPrecond::vcycle(const double *f, double *u, cudaStream_t s) {
    if (!fast) {
        amg_vcycle(amg, f, u, s);
        return;
    }
    // fast path cycles start from zero: u += V(f - A_p u)
    const CsrView<double> Ap = amg.levels[0]->A.view();
    double *res = vt.get(), *cor = vt.get() + Ap.nrows;
    copy_dev(Ap.nrows, f, res, s);
    csr_spmv(Ap, -1.0, u, 1.0, res, s);
    fast->vcycle(res, cor, s);
    axpy_dev(Ap.nrows, 1.0, cor, u, s);
}

// ---------------------------------------------------------------------------
// fused MGS pass: w += (-h_prev) * p_prev (if p_prev), then partial <p_j, w>
// ---------------------------------------------------------------------------
static constexpr int kMgsThreads = 512;

// pj == nullptr with self_dot: <w, w> after the update (the normalisation pass).
__global__ void __launch_bounds__(kMgsThreads) mgs_pass_kernel(long long n, double *__restrict__ w,
                                                               const double *__restrict__ p_prev,
                                                               const double *__restrict__ h_prev,
                                                               const double *__restrict__ pj, int self_dot,
                                                               double *__restrict__ partials) {
    __shared__ double ws[kMgsThreads / 32];
    const double a = p_prev ? -(*h_prev) : 0.0;
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * kMgsThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kMgsThreads) {
        double wv = w[i];
        if (p_prev) {
            wv = wv + a * p_prev[i];
            w[i] = wv;
        }
        if (self_dot) acc += wv * wv;
        else if (pj) acc += wv * pj[i];
    }
    if (!pj && !self_dot) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < kMgsThreads / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = r;
    }
}

__global__ void sum_partials_kernel(int np, const double *__restrict__ partials, double *__restrict__ out) {
    __shared__ double ws[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partials[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < (int)(blockDim.x / 32) ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) *out = r;
    }
}

// ---------------------------------------------------------------------------
// classical Gram-Schmidt (one pass): h = V^T w in one sweep over the basis,
// then w -= V h with ||w||^2 in a second sweep.  V is an array of m device
// pointers (m <= kCgsMax).
// ---------------------------------------------------------------------------
static constexpr int kCgsMax = 32;
static constexpr int kCgsThreads = 256;

__global__ void __launch_bounds__(kCgsThreads) cgs_dots_kernel(long long n, int m, const double *const *__restrict__ V,
                                                               const double *__restrict__ w,
                                                               double *__restrict__ partials) {
    double acc[kCgsMax];
#pragma unroll
    for (int k = 0; k < kCgsMax; ++k) acc[k] = 0.0;
    for (long long i = (long long)blockIdx.x * kCgsThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kCgsThreads) {
        const double wi = w[i];
#pragma unroll
        for (int k = 0; k < kCgsMax; ++k)
            if (k < m) acc[k] += V[k][i] * wi;
    }
    __shared__ double sh[kCgsThreads / 32][kCgsMax];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kCgsMax; ++k) {
        if (k >= m) break;
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) sh[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < m) {
        double v = 0.0;
        for (int q = 0; q < kCgsThreads / 32; ++q) v += sh[q][threadIdx.x];
        partials[(long long)blockIdx.x * kCgsMax + threadIdx.x] = v;
    }
}

// out[k] = sum over blocks of partials[b][k], k < m (one warp per k)
__global__ void cgs_sum_kernel(int nblocks, int m, const double *__restrict__ partials, double *__restrict__ out) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= m) return;
    double v = 0.0;
    for (int b = lane; b < nblocks; b += 32) v += partials[(long long)b * kCgsMax + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[k] = v;
}

// w -= sum_k h_k V_k, partial ||w||^2 per block
__global__ void __launch_bounds__(kCgsThreads) cgs_update_kernel(long long n, int m,
                                                                 const double *const *__restrict__ V,
                                                                 const double *__restrict__ h, double *__restrict__ w,
                                                                 double *__restrict__ partials) {
    __shared__ double hs[kCgsMax];
    if (threadIdx.x < kCgsMax) hs[threadIdx.x] = threadIdx.x < m ? h[threadIdx.x] : 0.0;
    __syncthreads();
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * kCgsThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kCgsThreads) {
        double s = w[i];
#pragma unroll
        for (int k = 0; k < kCgsMax; ++k)
            if (k < m) s -= hs[k] * V[k][i];
        w[i] = s;
        acc += s * s;
    }
    __shared__ double ws[kCgsThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < kCgsThreads / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = r;
    }
}

void Gmres::setup(int n_, cudaStream_t s) {
    n = n_;
    const size_t stride = ((size_t)(n > 0 ? n : 1) + 31) / 32 * 32;  // 256-byte aligned slices
    const int nvec = prm.k_dim + 1 + (prm.flexible ? prm.k_dim : 0);
    basis.alloc(stride * nvec);
    p.clear();
    zf.clear();
    for (int i = 0; i < nvec; ++i) {
        VecRef v{basis.get() + stride * i};
        if (i <= prm.k_dim) p.push_back(v);
        else zf.push_back(v);
    }
    r.alloc(n > 0 ? n : 1);
    w.alloc(n > 0 ? n : 1);
    cgs_blocks = std::max(1, std::min(4 * sm_count(), div_up(n > 0 ? n : 1, kCgsThreads)));
    partials.alloc(std::max<size_t>(reduce_partials() + 8, (size_t)cgs_blocks * kCgsMax));
    scal.alloc(prm.k_dim + 8);
    std::vector<const double *> ptrs;
    for (auto &v : p) ptrs.push_back(v.get());
    vptrs.alloc(ptrs.size());
    vptrs.upload(reinterpret_cast<const double **>(ptrs.data()), ptrs.size(), s);
    JX_CUDA(cudaStreamSynchronize(s));
}

namespace {
struct DevOps {
    cudaStream_t s;
    long long n;
    double *partials, *scal;
    int np;
    // <x, y> into scal[slot] (device) -- reference order y*x irrelevant (commutative products)
    void dot_to(const double *x, const double *y, int slot) {
        dot_dev(n, x, y, partials, scal + slot, s);
    }
    double fetch(int slot) {
        double v = 0.0;
        JX_CUDA(cudaMemcpyAsync(&v, scal + slot, sizeof(double), cudaMemcpyDeviceToHost, s));
        JX_CUDA(cudaStreamSynchronize(s));
        return v;
    }
};
}  // namespace

GmresResult Gmres::solve(const BsrView<double> &A, CprPrecond *M, const double *b, double *x, cudaStream_t s,
                         const std::function<void(const double *, double *)> *ext) {
    GmresResult res;
    const int k_dim = prm.k_dim;
    const long long nl = n;
    DevOps ops{s, nl, partials.get(), scal.get(), reduce_partials()};
    std::vector<double> rs(k_dim + 1, 0.0), c(k_dim, 0.0), sn(k_dim, 0.0);
    std::vector<std::vector<double>> hh(k_dim + 1, std::vector<double>(k_dim, 0.0));
    const double epsmac = 1.e-16;
    auto spmv = [&](double alpha, const double *xx, double beta, double *yy) {
        bsr_spmv<double, double>(A, alpha, xx, beta, yy, kerr, s, prm.use_tma_spmv != 0 && kerr != nullptr);
    };
    auto precond = [&](const double *in, double *out) {
        if (ext && *ext) (*ext)(in, out);
        else if (M) M->apply(in, out, s);
        else copy_dev(nl, in, out, s);
    };
    const int np = ops.np;
    const bool flexible = prm.flexible && (int)zf.size() >= k_dim;

    copy_dev(nl, b, p[0].get(), s);
    spmv(-1.0, x, 1.0, p[0].get());
    ops.dot_to(b, b, 0);
    const double b_norm = sqrt(ops.fetch(0));
    if (b_norm != 0.0 && !(b_norm / b_norm == b_norm / b_norm)) {
        set_error("gmres: NaN/Inf in b");
        res.status = JXCPR_ERROR_GENERIC;
        return res;
    }
    ops.dot_to(p[0].get(), p[0].get(), 0);
    double r_norm = sqrt(ops.fetch(0));
    if (r_norm != 0.0 && !(r_norm / r_norm == r_norm / r_norm)) {
        set_error("gmres: NaN/Inf in A or x0");
        res.status = JXCPR_ERROR_GENERIC;
        return res;
    }
    const double r_norm_0 = r_norm;
    double normdown = r_norm, conv_factor = 0.0;
    res.norms.assign(prm.max_iter + 1, 0.0);
    res.norms[0] = r_norm;
    const double den_norm = b_norm > 0.0 ? b_norm : r_norm;
    const double epsilon = std::max(prm.a_tol, prm.tol * den_norm);
    int iter = 0, i = 0;
    int converged = 0;
    while (iter < prm.max_iter) {
        rs[0] = r_norm;
        const double cycle_r0 = r_norm;
        if (r_norm == 0.0) {
            res.iterations = iter;
            res.converged = 1;
            res.rel_residual = 0.0;
            res.norms.resize(iter + 1);
            return res;
        }
        if (r_norm <= epsilon && iter >= prm.min_iter) {
            copy_dev(nl, b, r.get(), s);
            spmv(-1.0, x, 1.0, r.get());
            ops.dot_to(r.get(), r.get(), 0);
            r_norm = sqrt(ops.fetch(0));
            if (r_norm <= epsilon) {
                converged = 1;
                break;
            }
            if (prm.is_check_restarted == 0) break;
        }
        scale_dev(nl, 1.0 / r_norm, p[0].get(), s);
        i = 0;
        while (i < k_dim && iter < prm.max_iter) {
            ++i;
            ++iter;
            double *zi = flexible ? zf[i - 1].get() : r.get();
            JX_CUDA(cudaMemsetAsync(zi, 0, sizeof(double) * nl, s));
            precond(p[i - 1].get(), zi);
            spmv(1.0, zi, 0.0, p[i].get());
            if (prm.orthog == 1 && i <= kCgsMax) {
                // classical Gram-Schmidt: h = V_i^T w, w -= V_i h, ||w||^2 -> scal[i]
                const double *const *V = vptrs.get();
                cgs_dots_kernel<<<cgs_blocks, kCgsThreads, 0, s>>>(nl, i, V, p[i].get(), ops.partials);
                JX_LAUNCH_CHECK();
                cgs_sum_kernel<<<1, 32 * kCgsMax, 0, s>>>(cgs_blocks, i, ops.partials, ops.scal);
                JX_LAUNCH_CHECK();
                cgs_update_kernel<<<cgs_blocks, kCgsThreads, 0, s>>>(nl, i, V, ops.scal, p[i].get(), ops.partials);
                JX_LAUNCH_CHECK();
                sum_partials_kernel<<<1, 512, 0, s>>>(cgs_blocks, ops.partials, ops.scal + i);
                JX_LAUNCH_CHECK();
            } else
            // modified Gram-Schmidt, fused passes
            for (int j = 0; j <= i; ++j) {
                const double *pprev = j > 0 ? p[j - 1].get() : nullptr;
                const double *hprev = j > 0 ? ops.scal + (j - 1) : nullptr;
                const double *pj = j < i ? p[j].get() : nullptr;  // j == i: norm pass
                mgs_pass_kernel<<<np, kMgsThreads, 0, s>>>(nl, p[i].get(), pprev, hprev, pj, j == i ? 1 : 0,
                                                           ops.partials);
                JX_LAUNCH_CHECK();
                sum_partials_kernel<<<1, 512, 0, s>>>(np, ops.partials, ops.scal + j);
                JX_LAUNCH_CHECK();
            }
            std::vector<double> hv(i + 1);
            JX_CUDA(cudaMemcpyAsync(hv.data(), ops.scal, sizeof(double) * (i + 1), cudaMemcpyDeviceToHost, s));
            JX_CUDA(cudaStreamSynchronize(s));
            for (int j = 0; j < i; ++j) hh[j][i - 1] = hv[j];
            double t = sqrt(hv[i]);
            hh[i][i - 1] = t;
            if (t != 0.0) {
                t = 1.0 / t;
                scale_dev(nl, t, p[i].get(), s);
            }
            for (int j = 1; j < i; ++j) {
                t = hh[j - 1][i - 1];
                hh[j - 1][i - 1] = sn[j - 1] * hh[j][i - 1] + c[j - 1] * t;
                hh[j][i - 1] = -sn[j - 1] * t + c[j - 1] * hh[j][i - 1];
            }
            t = hh[i][i - 1] * hh[i][i - 1];
            t += hh[i - 1][i - 1] * hh[i - 1][i - 1];
            double gamma = sqrt(t);
            if (gamma == 0.0) gamma = epsmac;
            c[i - 1] = hh[i - 1][i - 1] / gamma;
            sn[i - 1] = hh[i][i - 1] / gamma;
            rs[i] = -hh[i][i - 1] * rs[i - 1];
            rs[i] /= gamma;
            rs[i - 1] = c[i - 1] * rs[i - 1];
            hh[i - 1][i - 1] = sn[i - 1] * hh[i][i - 1] + c[i - 1] * hh[i - 1][i - 1];
            r_norm = fabs(rs[i]);
            conv_factor = r_norm / normdown;
            normdown = r_norm;
            res.norms[iter] = r_norm;
            if (iter > 1 && conv_factor > prm.convfac_threshold) break;
            if (r_norm <= epsilon && iter >= prm.min_iter) break;
        }
        // solution update: back-solve H y = rs, w = sum y_j p_j, x += M^{-1} w
        rs[i - 1] = rs[i - 1] / hh[i - 1][i - 1];
        for (int k = i - 2; k >= 0; --k) {
            double t = 0.0;
            for (int j = k + 1; j < i; ++j) t -= hh[k][j] * rs[j];
            t += rs[k];
            rs[k] = t / hh[k][k];
        }
        if (flexible) {
            // x += Z y (the preconditioned directions were kept)
            for (int j = i - 1; j >= 0; --j) axpy_dev(nl, rs[j], zf[j].get(), x, s);
        } else {
            copy_dev(nl, p[i - 1].get(), w.get(), s);
            scale_dev(nl, rs[i - 1], w.get(), s);
            for (int j = i - 2; j >= 0; --j) axpy_dev(nl, rs[j], p[j].get(), w.get(), s);
            JX_CUDA(cudaMemsetAsync(r.get(), 0, sizeof(double) * nl, s));
            precond(w.get(), r.get());
            axpy_dev(nl, 1.0, r.get(), x, s);
        }
        if (r_norm <= epsilon && iter >= prm.min_iter) {
            copy_dev(nl, b, r.get(), s);
            spmv(-1.0, x, 1.0, r.get());
            ops.dot_to(r.get(), r.get(), 0);
            r_norm = sqrt(ops.fetch(0));
            if (r_norm <= epsilon) {
                converged = 1;
                break;
            }
            if (prm.is_check_restarted == 1) {
                copy_dev(nl, r.get(), p[0].get(), s);
                i = 0;
            } else {
                break;
            }
        }
        if (iter > 1 && conv_factor > prm.convfac_threshold) break;
        // stall rule: a full cycle whose residual ratio (end / start) stayed above stall_ratio
        if (prm.stall_ratio > 0.0 && i == k_dim && iter < prm.max_iter && r_norm > cycle_r0 * prm.stall_ratio) {
            res.stalled = 1;
            break;
        }
        for (int j = i; j > 0; --j) {
            rs[j - 1] = -sn[j - 1] * rs[j];
            rs[j] = c[j - 1] * rs[j];
        }
        if (i) axpy_dev(nl, rs[i] - 1.0, p[i].get(), p[i].get(), s);
        for (int j = i - 1; j > 0; --j) axpy_dev(nl, rs[j], p[j].get(), p[i].get(), s);
        if (i) {
            axpy_dev(nl, rs[0] - 1.0, p[0].get(), p[0].get(), s);
            axpy_dev(nl, 1.0, p[i].get(), p[0].get(), s);
        }
    }
    res.iterations = iter;
    res.converged = converged;
    res.rel_residual = b_norm > 0.0 ? r_norm / b_norm : r_norm / r_norm_0;
    res.norms.resize(iter + 1);
    JX_CUDA(cudaStreamSynchronize(s));
    return res;
}

// ---------------------------------------------------------------------------
// Solver
// ---------------------------------------------------------------------------
void Solver::setup(int nb, int bs, long long nnzb, const int *ia, const int *ja, const double *a, int device) {
    if (!stream && !stream_set) {
        JX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        owns_stream = true;
    }
    cudaStream_t s = stream;
    PoolStream scope(s);  // this setup's buffers are made for the solver's stream
    double al0[4];
    pool_stats(al0);
    auto t0 = std::chrono::steady_clock::now();
    ggmres.reset();  // its graph holds the previous setup's buffers
    learned_fallbacks = 0;
    learned_rebuilt = 0;
    A.alloc(nb, bs, nnzb);
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    JX_CUDA(cudaMemcpyAsync(A.ia.get(), ia, sizeof(int) * (nb + 1), kind, s));
    JX_CUDA(cudaMemcpyAsync(A.ja.get(), ja, sizeof(int) * nnzb, kind, s));
    JX_CUDA(cudaMemcpyAsync(A.a.get(), a, sizeof(double) * nnzb * bs * bs, kind, s));
    JX_CUDA(cudaStreamSynchronize(s));
    upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const int csz = decouple_coef_size(bs, prm.decouple);
    dcoef.alloc((size_t)(nb > 0 ? nb : 1) * (csz > 0 ? csz : 1));
    if (prm.decouple) bsr_decouple_matrix(A, prm.decouple, dcoef.get(), s, prm.thermal);
    JX_CUDA(cudaStreamSynchronize(s));
    decouple_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() - upload_ms;
    kerr.alloc(1);
    kerr.zero(s);
    cpr.prm = prm;
    cpr.ready = false;
    if (prm.stage1_solver_type) cpr.setup(A.view(), s);  // 0: GMRES without CPR (identity or caller's preconditioner)
    gmres.prm = prm;
    gmres.kerr = kerr.get();
    gmres.setup(nb * bs, s);
    b.alloc((size_t)(nb > 0 ? nb : 1) * bs);
    x.alloc((size_t)(nb > 0 ? nb : 1) * bs);
    cpr.amg.log.mark("gmres_vectors", s);
    if (cpr.probe_pending) {
        learned_probe(s);
        cpr.probe_pending = false;
        cpr.amg.log.mark("learned_probe", s);
    }
    JX_CUDA(cudaStreamSynchronize(s));
    setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    pool_stats(alloc_stats);
    for (int i = 0; i < 4; ++i) alloc_stats[i] -= al0[i];
}

// Learned settings against the plain smoothers: a few GMRES iterations (tol 0)
// on A x = A 1 with each preconditioner.  GMRES's own residual reduction per
// iteration, weighted by the bytes one iteration moves (the preconditioner's
// modelled traffic plus the SpMV and orthogonalisation common to both), is
// compared: the learned settings stay unless their residual reduction per
// byte is worse.
void Solver::learned_probe(cudaStream_t s) {
    const int m = 8;
    const long long n = (long long)A.nb * A.bs;
    SolverParams saved = gmres.prm;
    gmres.prm.max_iter = m;
    gmres.prm.min_iter = 0;
    gmres.prm.tol = 0.0;
    gmres.prm.a_tol = 0.0;
    gmres.prm.is_check_restarted = 0;
    fill_dev(n, 1.0, x.get(), s);
    bsr_spmv<double, double>(A.view(), 1.0, x.get(), 0.0, b.get(), kerr.get(), s, false);
    auto probe = [&]() {
        JX_CUDA(cudaMemsetAsync(x.get(), 0, sizeof(double) * n, s));
        GmresResult r = gmres.solve(A.view(), &cpr, b.get(), x.get(), s);
        return r.rel_residual;
    };
    const double bl = cpr.fast->apply_bytes();
    const double rl = probe();
    cpr.fast->set_plain_mode(true);
    const double bp = cpr.fast->apply_bytes();
    const double rp = probe();
    cpr.factor_fast = pow(rl, 1.0 / m);
    cpr.factor_plain = pow(rp, 1.0 / m);
    // common per-iteration traffic: BSR SpMV (FP64) and about k/2 orthogonalisation passes
    const double common = (double)A.nnzb * (A.bs * A.bs * 8.0 + 4.0) + 2.0 * n * 8.0 + 15.0 * 4.0 * n * 8.0;
    const double el = rl > 0.0 ? -log(rl) / (bl + common) : 1e300;
    const double ep = rp > 0.0 ? -log(rp) / (bp + common) : 1e300;
    cpr.probe_bytes[0] = bl + common;
    cpr.probe_bytes[1] = bp + common;
    gmres.prm = saved;
    if (el >= ep) {
        cpr.fast->set_plain_mode(false);  // learned settings stay
    } else {
        // The learned settings lose: the plain method replaces them entirely -- the learned
        // strength thresholds shaped the hierarchy too, so the plain smoothers on it are no
        // fallback (they can stall where the default hierarchy converges quickly).
        rebuild_plain(s);
    }
}

// The plain fast-path preconditioner (default strength thresholds, plain smoothers) in place of
// the learned one, on the already decoupled matrix.
void Solver::rebuild_plain(cudaStream_t s) {
    const int fs = cpr.prm.fast_smoother;
    const double ff = cpr.factor_fast, fp = cpr.factor_plain, pb0 = cpr.probe_bytes[0], pb1 = cpr.probe_bytes[1];
    cpr.prm.fast_smoother = 0;
    cpr.ready = false;
    cpr.setup(A.view(), s);
    // the probe's figures stay reported (learned_status): they are why the plain method runs now
    cpr.factor_fast = ff;
    cpr.factor_plain = fp;
    cpr.probe_bytes[0] = pb0;
    cpr.probe_bytes[1] = pb1;
    cpr.prm.fast_smoother = fs;
    cpr.learned_used = 0;
    cpr.probe_pending = false;
    learned_rebuilt = 1;
    if (ggmres) ggmres->reset_graph();
}

// Learned settings are kept by a short probe at setup.  The full solve then runs with a stall
// rule: a full restart cycle of k iterations that reduces the residual by less than a factor
// 1 / kStallCycleRatio ends it early (the probe's 8 iterations measure the fast early reduction and
// cannot predict a stall; a learned hierarchy that stalls does so within its first cycle).  The plain
// preconditioner (default thresholds, plain smoothers) is then built in place of the learned one and
// GMRES continues from the current iterate with the remaining iterations.
static constexpr double kStallCycleRatio = 0.1;
GmresResult Solver::solve(const double *b_in, double *x_io, int device) {
    const bool guard = cpr.fast && cpr.learned_used && prm.learned_fallback && cpr.factor_fast > 0.0 &&
                       cpr.factor_fast < 1.0 && prm.tol > 0.0 && prm.tol < 1.0;
    if (!guard) return solve_once(b_in, x_io, device);
    const SolverParams saved = prm;
    prm.stall_ratio = kStallCycleRatio;
    GmresResult first;
    try {
        first = solve_once(b_in, x_io, device);
    } catch (...) {
        prm = saved;
        throw;
    }
    prm = saved;
    if (!first.stalled || first.status) return first;
    const double ms0 = solve_ms;
    {
        PoolStream scope(stream);
        rebuild_plain(stream);
    }
    learned_fallbacks += 1;
    prm.max_iter = saved.max_iter - first.iterations;
    try {
        last = solve_once(b_in, x_io, device);
    } catch (...) {
        prm = saved;
        throw;
    }
    prm = saved;
    last.iterations += first.iterations;
    std::vector<double> h = first.norms;
    if (last.norms.size() > 1) h.insert(h.end(), last.norms.begin() + 1, last.norms.end());
    last.norms = h;
    solve_ms += ms0;
    return last;
}

GmresResult Solver::solve_once(const double *b_in, double *x_io, int device) {
    cudaStream_t s = stream;
    PoolStream scope(s);
    const long long n = (long long)A.nb * A.bs;
    auto t0 = std::chrono::steady_clock::now();
    const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    JX_CUDA(cudaMemcpyAsync(b.get(), b_in, sizeof(double) * n, in, s));
    JX_CUDA(cudaMemcpyAsync(x.get(), x_io, sizeof(double) * n, in, s));
    if (prm.graph_gmres) {
        if (!ggmres) ggmres.reset(new GraphGmres());
        if (!ggmres->exec || !ggmres->matches(prm)) {
            ggmres->prepare(*this);
            ggmres->build_single(*this);
        }
        double sm[8];
        JX_CUDA(cudaGraphLaunch(ggmres->exec, s));
        JX_CUDA(cudaMemcpyAsync(sm, ggmres->summary.get(), sizeof(sm), cudaMemcpyDeviceToHost, s));
        const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        JX_CUDA(cudaMemcpyAsync(x_io, x.get(), sizeof(double) * n, out, s));
        JX_CUDA(cudaStreamSynchronize(s));
        last = ggmres->result_from(sm, s, true);
        count_launches(ggmres->kernels_run(last.iterations, (int)sm[6]));
        if (sm[7] != 0.0) {
            set_error("device wait timed out (spmv / smoother / BILU substitution flags set)");
            last.status = JXCPR_ERROR_DEVICE;
            kerr.zero(s);
            cpr.amg.err.zero(s);
            if (cpr.bilu && cpr.bilu->error_flag()) JX_CUDA(cudaMemsetAsync(cpr.bilu->error_flag(), 0, sizeof(int), s));
            JX_CUDA(cudaStreamSynchronize(s));
        }
        solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return last;
    }
    if (prm.decouple) bsr_decouple_rhs(A.nb, A.bs, prm.decouple, dcoef.get(), b.get(), prm.consistent_rhs, s);
    gmres.prm = prm;
    cpr.prm.stage2_maxit = prm.stage2_maxit;
    cpr.prm.stage1_maxit = prm.stage1_maxit;
    last = gmres.solve(A.view(), prm.stage1_solver_type ? &cpr : nullptr, b.get(), x.get(), s, &ext_precond);
    const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    JX_CUDA(cudaMemcpyAsync(x_io, x.get(), sizeof(double) * n, out, s));
    JX_CUDA(cudaStreamSynchronize(s));
    int kflag = 0, aflag = 0, bflag = 0;
    JX_CUDA(cudaMemcpy(&kflag, kerr.get(), sizeof(int), cudaMemcpyDeviceToHost));
    JX_CUDA(cudaMemcpy(&aflag, cpr.amg.err.get(), sizeof(int), cudaMemcpyDeviceToHost));
    int *bf = cpr.bilu ? cpr.bilu->error_flag() : nullptr;
    if (bf) JX_CUDA(cudaMemcpy(&bflag, bf, sizeof(int), cudaMemcpyDeviceToHost));
    if (kflag || aflag || bflag) {
        set_error("device wait timed out (spmv flag %d, smoother flag %d, BILU substitution flag %d)", kflag, aflag,
                  bflag);
        last.status = JXCPR_ERROR_DEVICE;
        kerr.zero(s);
        cpr.amg.err.zero(s);
        if (bf) JX_CUDA(cudaMemsetAsync(bf, 0, sizeof(int), s));
    }
    solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return last;
}

}  // namespace jxcpr
