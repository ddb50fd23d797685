// Pressure AMG: hierarchy construction and the V(1,1) cycle of CPR stage 1.
//
// Setup follows jxf_PAMGSetup (jxfpamg-0220/csrc/amg/par_amg_setup.c:525-1240):
// per level strength -> HMIS -> ext+i -> Galerkin product, stopping after the
// level whose coarse size is <= coarse_threshold (1000) or at max_levels-1.
//
// The cycle follows jxf_PAMGCycle (amg/par_cycle.c:20-969) with
// jxf_PAMGRelaxIF (par_relax_if.c:22-76) as CPR configures it: on every level
// but the coarsest, two symmetric Gauss-Seidel applications before and two
// after the coarse correction (relax_order 1 visits "C then F" and "F then C",
// and jxf_PAMGRelax resets the point selection to "all points", par_relax.c:48);
// residual r = f - A u, restriction f_c = P^T r, prolongation u += P u_c; on the
// coarsest level the dense Gaussian elimination of jxf_gselim
// (operation/matops/par_gs.c:20-74), here factored once at setup.
#include <algorithm>
#include <chrono>
#include <future>
#include <memory>
#include <vector>

#include "amg.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace jxcpr {

// ---------------------------------------------------------------------------
// coarsest level: dense LU without pivoting in jxf_gselim's order
// ---------------------------------------------------------------------------
__global__ void dense_assemble_kernel(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                                      const double *__restrict__ a, double *__restrict__ M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = ia[i]; k < ia[i + 1]; ++k) M[(long long)i * n + ja[k]] = a[k];
}

// One elimination step k on the trailing block; also records the multipliers.
__global__ void lu_step_kernel(int n, int k, double *__restrict__ M, double *__restrict__ Lt) {
    const int j = k + 1 + blockIdx.y;            // row
    const int m = k + 1 + blockIdx.x * blockDim.x + threadIdx.x;  // column
    if (j >= n) return;
    const double akk = M[(long long)k * n + k];
    const double ajk = M[(long long)j * n + k];
    const bool active = (akk != 0.0) && (ajk != 0.0);
    if (blockIdx.x == 0 && threadIdx.x == 0) Lt[(long long)k * n + j] = active ? ajk / akk : 0.0;
    if (!active || m >= n) return;
    const double factor = ajk / akk;
    M[(long long)j * n + m] -= factor * M[(long long)k * n + m];
}

__global__ void transpose_upper_kernel(int n, const double *__restrict__ M, double *__restrict__ Ut) {
    const int j = blockIdx.y;  // row of U
    const int k = blockIdx.x * blockDim.x + threadIdx.x;  // column of U
    if (j >= n || k >= n) return;
    Ut[(long long)k * n + j] = (j <= k) ? M[(long long)j * n + k] : 0.0;
}

// Forward and back substitution with the stored factors, column oriented, in
// jxf_gselim's order (bit-identical to re-running the elimination).
__global__ void __launch_bounds__(1024) lu_solve_kernel(int n, const double *__restrict__ Lt,
                                                        const double *__restrict__ Ut, const double *__restrict__ f,
                                                        double *__restrict__ u) {
    extern __shared__ double xs[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = f[i];
    __syncthreads();
    if (n == 1) {
        if (threadIdx.x == 0 && Ut[0] != 0.0) u[0] = xs[0] / Ut[0];
        else if (threadIdx.x == 0) u[0] = xs[0];
        return;
    }
    for (int k = 0; k < n - 1; ++k) {
        const double xk = xs[k];
        const double *col = Lt + (long long)k * n;
        for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
            const double l = col[j];
            if (l != 0.0) xs[j] -= l * xk;
        }
        __syncthreads();
    }
    for (int k = n - 1; k > 0; --k) {
        if (threadIdx.x == 0) xs[k] /= Ut[(long long)k * n + k];
        __syncthreads();
        const double xk = xs[k];
        const double *col = Ut + (long long)k * n;
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            const double v = col[j];
            if (v != 0.0) xs[j] -= xk * v;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) xs[0] /= Ut[0];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) u[i] = xs[i];
}

// u = Ainv f, one warp per row.
__global__ void dense_gemv_kernel(int n, const double *__restrict__ Ainv, const double *__restrict__ f,
                                  double *__restrict__ u) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int c = lane; c < n; c += 32) s += Ainv[(long long)row * n + c] * f[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) u[row] = s;
}

void coarse_setup(Amg &H, cudaStream_t s) {
    AmgLevel &L = *H.levels.back();
    const int n = L.A.nrows;
    H.nc = n;
    if (n == 0) return;
    if (n > 8192) {
        set_error("coarsest level has %d rows (dense solve limited to 8192); coarsening stalled", n);
        throw CudaError{cudaErrorInvalidValue, "coarse size"};
    }
    if (!H.prm.coarse_exact) {
        // fast coarse solve: only the inverse is needed (one cooperative DMMA kernel, coarse_mma.cu)
        H.Ainv.alloc((size_t)n * n);
        coarse_inverse_mma(L.A.view(), H.Ainv.get(), H.err.get(), s);
        return;
    }
    DevBuf<double> M((size_t)n * n);
    M.zero(s);
    dense_assemble_kernel<<<div_up(n, 128), 128, 0, s>>>(n, L.A.ia.get(), L.A.ja.get(), L.A.a.get(), M.get());
    JX_LAUNCH_CHECK();
    H.Lt.alloc((size_t)n * n);
    H.Lt.zero(s);
    for (int k = 0; k < n - 1; ++k) {
        dim3 grid(div_up(std::max(1, n - k - 1), 256), n - k - 1);
        lu_step_kernel<<<grid, 256, 0, s>>>(n, k, M.get(), H.Lt.get());
        JX_LAUNCH_CHECK();
    }
    H.Ufac.alloc((size_t)n * n);
    transpose_upper_kernel<<<dim3(div_up(n, 256), n), 256, 0, s>>>(n, M.get(), H.Ufac.get());
    JX_LAUNCH_CHECK();
    JX_CUDA(cudaStreamSynchronize(s));
}

void coarse_solve(Amg &H, const double *f, double *u, cudaStream_t s) {
    const int n = H.nc;
    if (n == 0) return;
    if (H.prm.coarse_exact) {
        const size_t smem = sizeof(double) * (size_t)n;
        if (smem > 48 * 1024) {
            JX_CUDA(cudaFuncSetAttribute(lu_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        }
        lu_solve_kernel<<<1, 1024, smem, s>>>(n, H.Lt.get(), H.Ufac.get(), f, u);
    } else {
        dense_gemv_kernel<<<div_up((long long)n * 32, 256), 256, 0, s>>>(n, H.Ainv.get(), f, u);
    }
    JX_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// hierarchy
// ---------------------------------------------------------------------------
// Gauss-Seidel schedules of a level, built on the host from its pattern.  The
// pattern's copy to the host and the host work run on a worker thread while the
// setup carries on with the strength, coarsening and the next levels: the copy
// waits for the pattern on a stream of its own (an event recorded on the
// setup's stream), so the setup's stream is not stalled by it.
struct ScheduleJob {
    std::vector<int> perm[2], gptr[2], rank[2];
    bool both = false;
    std::vector<int> chunk_order, chunk_seg;
};

namespace {
// A stream and an event owned by the worker thread's copy, released on every exit path.
struct CopyStream {
    cudaStream_t stream = nullptr;
    cudaEvent_t ready = nullptr;
    ~CopyStream() {
        if (stream) cudaStreamDestroy(stream);
        if (ready) cudaEventDestroy(ready);
    }
};
}  // namespace

// chunk > 0: also the stage-2 chunk order of the pattern (level 0 of the fast path), on a host thread
// of its own beside the Gauss-Seidel schedule
static std::future<ScheduleJob> start_level_schedules(AmgLevel &L, int order, int chunk, cudaStream_t s) {
    const int n = L.A.nrows;
    const long long nnz = L.A.nnz;
    const int *dia = L.A.ia.get(), *dja = L.A.ja.get();
    int dev = 0;
    JX_CUDA(cudaGetDevice(&dev));
    auto cs = std::make_shared<CopyStream>();
    JX_CUDA(cudaEventCreateWithFlags(&cs->ready, cudaEventDisableTiming));
    JX_CUDA(cudaEventRecord(cs->ready, s));
    using Chunks = std::pair<std::vector<int>, std::vector<int>>;
    return std::async(std::launch::async, [n, nnz, dia, dja, dev, cs, order, chunk]() {
        JX_CUDA(cudaSetDevice(dev));
        JX_CUDA(cudaStreamCreateWithFlags(&cs->stream, cudaStreamNonBlocking));
        JX_CUDA(cudaStreamWaitEvent(cs->stream, cs->ready, 0));
        auto ia = std::make_shared<std::vector<int>>(n + 1), ja = std::make_shared<std::vector<int>>(nnz > 0 ? nnz : 1);
        JX_CUDA(cudaMemcpyAsync(ia->data(), dia, sizeof(int) * (size_t)(n + 1), cudaMemcpyDeviceToHost, cs->stream));
        if (nnz > 0)
            JX_CUDA(cudaMemcpyAsync(ja->data(), dja, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, cs->stream));
        JX_CUDA(cudaStreamSynchronize(cs->stream));
        std::future<Chunks> chunks;
        if (chunk > 0)
            chunks = std::async(std::launch::async, [n, chunk, ia, ja]() {
                Chunks c;
                build_chunk_order_host(n, ia->data(), ja->data(), chunk, c.first, c.second);
                return c;
            });
        ScheduleJob J;
        build_schedule_host(n, ia->data(), ja->data(), order, true, J.perm[0], J.gptr[0], J.rank[0]);
        if (order == ORDER_EXACT) {
            J.both = true;
            build_schedule_host(n, ia->data(), ja->data(), order, false, J.perm[1], J.gptr[1], J.rank[1]);
        }
        // multicolour: the backward sweep visits the same classes in reverse order (fwd schedule, reversed)
        if (chunks.valid()) {
            Chunks c = chunks.get();
            J.chunk_order = std::move(c.first);
            J.chunk_seg = std::move(c.second);
        }
        return J;
    });
}

static void finish_level_schedules(AmgLevel &L, ScheduleJob J, cudaStream_t s) {
    upload_schedule(J.perm[0], J.gptr[0], J.rank[0], L.fwd, s);
    if (J.both) upload_schedule(J.perm[1], J.gptr[1], J.rank[1], L.bwd, s);
    L.chunk_order = std::move(J.chunk_order);
    L.chunk_seg = std::move(J.chunk_seg);
}

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
void PhaseLog::start() {
    items.clear();
    t_last = now_ms();
}
void PhaseLog::mark(const char *name, cudaStream_t s) {
    cudaStreamSynchronize(s);
    const double t = now_ms();
    for (auto &kv : items)
        if (kv.first == name) {
            kv.second += t - t_last;
            t_last = t;
            return;
        }
    items.emplace_back(name, t - t_last);
    t_last = t;
}

void amg_setup(Amg &H, DeviceCsr &&A0, cudaStream_t s) {
    H.log.start();
    H.levels.clear();
    H.levels.emplace_back(new AmgLevel());
    H.levels[0]->A = std::move(A0);
    // which levels get Gauss-Seidel schedules: all in the exact order; in the fast path level 0
    // (stage 2 sweeps the block matrix, which has its pattern) and the levels sparse enough for GS
    auto wants_schedule = [&](const AmgLevel &L, bool first) {
        const double mean_row = L.A.nrows > 0 ? (double)L.A.nnz / L.A.nrows : 0.0;
        const bool dense = H.prm.order != ORDER_EXACT && mean_row > H.prm.jacobi_mean_row;
        return !dense || first;
    };
    std::vector<std::future<ScheduleJob>> jobs;
    int level = 0;
    while (true) {
        AmgLevel &L = *H.levels[level];
        const int n = L.A.nrows;
        jobs.emplace_back();
        if (wants_schedule(L, level == 0))
            jobs.back() = start_level_schedules(
                L, H.prm.order, (level == 0 && H.prm.order != ORDER_EXACT) ? H.prm.stage2_chunk : 0, s);
        DevPattern S;
        if (H.prm.theta_for_level) {
            L.theta = H.prm.theta_for_level(level, L.A.view());
            H.log.mark("level_features", s);
        } else {
            L.theta = H.prm.strong_threshold;
        }
        amg_strength(L.A.view(), L.theta, H.prm.max_row_sum, S, s);
        H.log.mark("strength", s);
        L.cf.assign(n, 0);
        const int range_rows = level == 0 ? H.prm.rs_range_rows : H.prm.rs_range_rows_coarse;
        if (range_rows > 0 && n >= 2 * range_rows) {
            std::vector<int> sia(n + 1), sja(S.nnz > 0 ? S.nnz : 1);
            S.ia.download(sia.data(), n + 1, s);
            S.ja.download(sja.data(), S.nnz, s);
            JX_CUDA(cudaStreamSynchronize(s));
            rs_first_pass_ranges(n, sia.data(), sja.data(), range_rows, L.cf.data());
        } else {
            // the pattern and its transpose (stable: rows ascending in each column) go to the host
            std::vector<int> sia(n + 1), sja(S.nnz > 0 ? S.nnz : 1), stia(n + 1), stja(S.nnz > 0 ? S.nnz : 1);
            {
                DevBuf<int> tia(n + 1), tja(S.nnz > 0 ? S.nnz : 1), tperm(S.nnz > 0 ? S.nnz : 1);
                pattern_transpose(n, n, S.nnz, S.ia.get(), S.ja.get(), tia.get(), tja.get(), tperm.get(), s);
                S.ia.download(sia.data(), n + 1, s);
                S.ja.download(sja.data(), S.nnz, s);
                tia.download(stia.data(), n + 1, s);
                tja.download(stja.data(), S.nnz, s);
                JX_CUDA(cudaStreamSynchronize(s));
            }
            rs_first_pass_host(n, sia.data(), sja.data(), stia.data(), stja.data(), L.cf.data());
        }
        H.log.mark("rs_first_pass(host)", s);
        DevBuf<int> cf(n > 0 ? n : 1);
        cf.upload(L.cf.data(), n, s);
        amg_pmis(S, cf.get(), s);
        cf.download(L.cf.data(), n, s);
        H.log.mark("pmis", s);
        const int nc = amg_extpi_interp(L.A.view(), S, cf.get(), L.P, s);
        H.log.mark("interp_extpi", s);
        csr_transpose(L.P.view(), L.R, s);
        H.log.mark("transpose_P", s);
        std::unique_ptr<AmgLevel> next(new AmgLevel());
        amg_rap(L.A.view(), L.P, L.R, next->A, s);
        H.log.mark("rap", s);
        H.levels.push_back(std::move(next));
        ++level;
        if (level == H.prm.max_levels - 1 || nc <= H.prm.coarse_threshold) break;
    }
    for (size_t l = 0; l < H.levels.size(); ++l) {
        AmgLevel &L = *H.levels[l];
        const int n = L.A.nrows;
        if (H.prm.order == ORDER_EXACT) {
            L.f.alloc(n > 0 ? n : 1);
            L.u.alloc(n > 0 ? n : 1);
        }
        if (l + 1 == H.levels.size()) continue;  // the coarsest level is solved directly
        const double mean_row = n > 0 ? (double)L.A.nnz / n : 0.0;
        const bool dense = H.prm.order != ORDER_EXACT && mean_row > H.prm.jacobi_mean_row;
        if (l < jobs.size() && jobs[l].valid()) finish_level_schedules(L, jobs[l].get(), s);
        H.log.mark("schedules(host)", s);
        if (H.prm.order == ORDER_EXACT)
            L.smoother = SMOOTH_EXACT_GS;
        else if (!dense && L.fwd.ngroups <= H.prm.max_colors)
            L.smoother = SMOOTH_COLOR_GS;  // storage built by the fast path
        else
            L.smoother = SMOOTH_L1_JACOBI;
    }
    const int n0 = H.levels[0]->A.nrows;
    H.work.alloc((size_t)(n0 > 0 ? n0 : 1) * 2);
    H.err.alloc(4);  // [0] error flag, [2..3] grid barrier of the cooperative sweeps
    H.err.zero(s);
    H.log.mark("vectors", s);
    coarse_setup(H, s);
    H.log.mark("coarse_lu", s);
    JX_CUDA(cudaStreamSynchronize(s));
}

// One symmetric Gauss-Seidel application (forward then backward sweep).
static void sgs(Amg &H, AmgLevel &L, const double *f, double *u, double *vt, cudaStream_t s) {
    gs_sweep(L.A.view(), L.fwd, f, u, L.fwd.rank.get(), vt, H.err.get(), s);
    gs_sweep(L.A.view(), L.bwd, f, u, L.bwd.rank.get(), vt, H.err.get(), s);
}

void amg_vcycle(Amg &H, const double *f0, double *u0, cudaStream_t s) {
    // exact-order cycle; the throughput / mixed cycles are in fast_cpr.cu
    const int L = H.num_levels();
    double *vt = H.work.get();
    double *res = H.work.get() + H.levels[0]->A.nrows;
    auto F = [&](int l) -> const double * { return l == 0 ? f0 : H.levels[l]->f.get(); };
    auto U = [&](int l) -> double * { return l == 0 ? u0 : H.levels[l]->u.get(); };
    if (L == 1) {
        // a single level cannot happen with coarse_threshold >= 1 unless n <= threshold; solve directly
        coarse_solve(H, f0, u0, s);
        return;
    }
    for (int l = 0; l < L - 1; ++l) {
        AmgLevel &Lv = *H.levels[l];
        sgs(H, Lv, F(l), U(l), vt, s);
        sgs(H, Lv, F(l), U(l), vt, s);
        const int n = Lv.A.nrows;
        JX_CUDA(cudaMemsetAsync(U(l + 1), 0, sizeof(double) * H.levels[l + 1]->A.nrows, s));
        JX_CUDA(cudaMemcpyAsync(res, F(l), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        csr_spmv(Lv.A.view(), -1.0, U(l), 1.0, res, s);
        csr_spmv(Lv.R.view(), 1.0, res, 0.0, H.levels[l + 1]->f.get(), s);
    }
    coarse_solve(H, F(L - 1), U(L - 1), s);
    for (int l = L - 2; l >= 0; --l) {
        AmgLevel &Lv = *H.levels[l];
        csr_spmv(Lv.P.view(), 1.0, U(l + 1), 1.0, U(l), s);
        sgs(H, Lv, F(l), U(l), vt, s);
        sgs(H, Lv, F(l), U(l), vt, s);
    }
}

}  // namespace jxcpr
