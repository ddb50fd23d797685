// Batched solves: many independent systems (uneven sizes) solved by ONE graph
// launch.  Every system's whole GMRES solve (right-hand-side decoupling,
// restart cycles, Arnoldi steps with the CPR kernels recorded in place; see
// graph_gmres.cu) is recorded as its own branch of a single CUDA graph; the
// branches share no dependency, so the GPU runs them side by side and the
// host launches once and reads back once.  Each solver keeps its own device
// matrix, hierarchy, autotuned layouts and Krylov basis.  Per-system solve
// times come from the device global timer at each branch's start and end.
// No counterpart in the reference.
#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <stdexcept>
#include <memory>
#include <vector>

#include "jxcpr_b200.h"
#include "handle.cuh"

using namespace jxcpr;

struct jxcpr_batch {
    std::vector<Solver *> sys;
    cudaStream_t s0 = nullptr;
    std::vector<cudaStream_t> br;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DevBuf<double> summary;      // 8 values per system
    std::vector<double> sm_host;
    float last_ms = 0.f;
    ~jxcpr_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto e : join)
            if (e) cudaEventDestroy(e);
        for (auto s : br)
            if (s) cudaStreamDestroy(s);
        if (fork) cudaEventDestroy(fork);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (s0) cudaStreamDestroy(s0);
    }
};

namespace {
template <typename F>
int guarded(F &&f) {
    try {
        return f();
    } catch (const CudaError &) {
        return JXCPR_ERROR_DEVICE;
    } catch (const std::invalid_argument &) {
        return JXCPR_ERROR_ARG;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return JXCPR_ERROR_MEMORY;
    } catch (...) {
        set_error("unexpected exception");
        return JXCPR_ERROR_GENERIC;
    }
}

void end_capture_quietly(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (!s || cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs == cudaStreamCaptureStatusNone) return;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
}
}  // namespace

extern "C" {

int jxcpr_batch_setup(int nsys, jxcpr_solver *const *solvers, const int *nb, const int *bs, const long long *nnzb,
                      const int *const *ia, const int *const *ja, const double *const *a, int device, int threads,
                      int *status) {
    if (nsys < 0 || (nsys > 0 && (!solvers || !nb || !bs || !nnzb || !ia || !ja || !a))) return JXCPR_ERROR_ARG;
    if (nsys == 0) return JXCPR_SUCCESS;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        set_error("batch_setup: no current CUDA device");
        return JXCPR_ERROR_DEVICE;
    }
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    // The exact-order smoothers share one grid barrier per device and the BILU
    // stage was not written for concurrent setups: such batches set up in turn.
    for (int k = 0; k < nsys; ++k)
        if (solvers[k] && (solvers[k]->s.prm.smoother_order == ORDER_EXACT || solvers[k]->s.prm.stage2_solver_type == 5))
            threads = 1;
    threads = std::min(threads, nsys);
    std::vector<int> st(nsys, JXCPR_SUCCESS);
    std::vector<std::string> msg(nsys);
    std::atomic<int> next{0};
    auto worker = [&]() {
        cudaSetDevice(dev);
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= nsys) break;
            st[k] = solvers[k] ? jxcpr_solver_setup(solvers[k], nb[k], bs[k], nnzb[k], ia[k], ja[k], a[k], device)
                               : JXCPR_ERROR_ARG;
            if (st[k] != JXCPR_SUCCESS) msg[k] = last_error();
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
    int worst = JXCPR_SUCCESS;
    for (int k = 0; k < nsys; ++k) {
        if (status) status[k] = st[k];
        if (st[k] != JXCPR_SUCCESS && worst == JXCPR_SUCCESS) {
            worst = st[k];
            set_error("batch_setup: system %d: %s", k, msg[k].c_str());
        }
    }
    return worst;
}

int jxcpr_batch_create(jxcpr_batch **out, int nsys, jxcpr_solver *const *solvers) {
    if (!out || nsys < 1 || !solvers) return JXCPR_ERROR_ARG;
    *out = nullptr;
    for (int k = 0; k < nsys; ++k)
        if (!solvers[k] || !solvers[k]->s.cpr.ready) {
            set_error("batch_create: system %d has no setup", k);
            return JXCPR_ERROR_ARG;
        }
    std::unique_ptr<jxcpr_batch> B(new (std::nothrow) jxcpr_batch());
    if (!B) return JXCPR_ERROR_MEMORY;
    const int st = guarded([&] {
        B->sys.resize(nsys);
        for (int k = 0; k < nsys; ++k) B->sys[k] = &solvers[k]->s;
        for (Solver *S : B->sys) {
            PoolStream scope(S->stream);
            S->prm.graph_gmres = 1;
            if (!S->ggmres) S->ggmres.reset(new GraphGmres());
            S->ggmres->prepare(*S);
        }
        JX_CUDA(cudaStreamCreateWithFlags(&B->s0, cudaStreamNonBlocking));
        JX_CUDA(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
        JX_CUDA(cudaEventCreate(&B->t0));
        JX_CUDA(cudaEventCreate(&B->t1));
        B->br.assign(nsys, nullptr);
        B->join.assign(nsys, nullptr);
        for (int k = 0; k < nsys; ++k) {
            JX_CUDA(cudaStreamCreateWithFlags(&B->br[k], cudaStreamNonBlocking));
            JX_CUDA(cudaEventCreateWithFlags(&B->join[k], cudaEventDisableTiming));
        }
        B->summary.alloc((size_t)8 * nsys);
        B->sm_host.assign((size_t)8 * nsys, 0.0);
        JX_CUDA(cudaStreamBeginCapture(B->s0, cudaStreamCaptureModeThreadLocal));
        try {
            JX_CUDA(cudaEventRecord(B->fork, B->s0));
            for (int k = 0; k < nsys; ++k) {
                JX_CUDA(cudaStreamWaitEvent(B->br[k], B->fork, 0));
                B->sys[k]->ggmres->record(*B->sys[k], B->br[k], B->summary.get() + 8 * (size_t)k);
                JX_CUDA(cudaEventRecord(B->join[k], B->br[k]));
                JX_CUDA(cudaStreamWaitEvent(B->s0, B->join[k], 0));
            }
        } catch (...) {
            for (auto s : B->br) end_capture_quietly(s);
            end_capture_quietly(B->s0);
            throw;
        }
        JX_CUDA(cudaStreamEndCapture(B->s0, &B->graph));
        JX_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
        return JXCPR_SUCCESS;
    });
    if (st != JXCPR_SUCCESS) return st;
    *out = B.release();
    return JXCPR_SUCCESS;
}

int jxcpr_batch_destroy(jxcpr_batch *h) {
    if (!h) return JXCPR_ERROR_ARG;
    return guarded([&] {
        delete h;
        return JXCPR_SUCCESS;
    });
}

int jxcpr_batch_solve(jxcpr_batch *h, const double *const *b, double *const *x, int device, int *iterations,
                      double *rel_residual, double *latency_ms, double *finish_ms, int *status) {
    if (!h || !b || !x) return JXCPR_ERROR_ARG;
    const int nsys = (int)h->sys.size();
    for (int k = 0; k < nsys; ++k)
        if (!b[k] || !x[k]) return JXCPR_ERROR_ARG;
    return guarded([&] {
        cudaStream_t s = h->s0;
        const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        const cudaMemcpyKind outk = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        JX_CUDA(cudaEventRecord(h->t0, s));
        for (int k = 0; k < nsys; ++k) {
            Solver &S = *h->sys[k];
            const size_t bytes = sizeof(double) * (size_t)S.A.nb * S.A.bs;
            JX_CUDA(cudaMemcpyAsync(S.b.get(), b[k], bytes, in, s));
            JX_CUDA(cudaMemcpyAsync(S.x.get(), x[k], bytes, in, s));
        }
        JX_CUDA(cudaGraphLaunch(h->exec, s));
        for (int k = 0; k < nsys; ++k) {
            Solver &S = *h->sys[k];
            const size_t bytes = sizeof(double) * (size_t)S.A.nb * S.A.bs;
            JX_CUDA(cudaMemcpyAsync(x[k], S.x.get(), bytes, outk, s));
        }
        JX_CUDA(cudaEventRecord(h->t1, s));
        JX_CUDA(cudaMemcpyAsync(h->sm_host.data(), h->summary.get(), sizeof(double) * 8 * nsys,
                                cudaMemcpyDeviceToHost, s));
        JX_CUDA(cudaStreamSynchronize(s));
        JX_CUDA(cudaEventElapsedTime(&h->last_ms, h->t0, h->t1));
        double tmin = 0.0;
        for (int k = 0; k < nsys; ++k) {
            const double ts = h->sm_host[8 * (size_t)k + 4];
            if (k == 0 || ts < tmin) tmin = ts;
        }
        int worst = JXCPR_SUCCESS;
        for (int k = 0; k < nsys; ++k) {
            const double *sm = &h->sm_host[8 * (size_t)k];
            Solver &S = *h->sys[k];
            S.last = S.ggmres->result_from(sm, s, false);
            count_launches(S.ggmres->kernels_run(S.last.iterations, (int)sm[6]));
            int stk = S.last.status ? S.last.status : (S.last.converged ? JXCPR_SUCCESS : JXCPR_ERROR_CONV);
            if (sm[7] != 0.0) {
                set_error("batch: device wait timed out in system %d", k);
                stk = JXCPR_ERROR_DEVICE;
                S.kerr.zero(s);
                S.cpr.amg.err.zero(s);
            }
            if (iterations) iterations[k] = S.last.iterations;
            if (rel_residual) rel_residual[k] = S.last.rel_residual;
            if (latency_ms) latency_ms[k] = (sm[5] - sm[4]) * 1e-6;
            if (finish_ms) finish_ms[k] = (sm[5] - tmin) * 1e-6;
            if (status) status[k] = stk;
            if (stk != JXCPR_SUCCESS && stk != JXCPR_ERROR_CONV) worst = stk;
        }
        JX_CUDA(cudaStreamSynchronize(s));
        return worst;
    });
}

int jxcpr_batch_last_ms(jxcpr_batch *h, double *ms) {
    if (!h || !ms) return JXCPR_ERROR_ARG;
    *ms = h->last_ms;
    return JXCPR_SUCCESS;
}

int jxcpr_batch_launch(jxcpr_batch *h, void *stream) {
    if (!h) return JXCPR_ERROR_ARG;
    return guarded([&] {
        JX_CUDA(cudaGraphLaunch(h->exec, stream ? (cudaStream_t)stream : h->s0));
        return JXCPR_SUCCESS;
    });
}

}  // extern "C"
