// C ABI of the solver object: setup / solve with host or device arrays,
// string-keyed options (the reference's JXF_CPRSetParameter style), and
// inspection of the AMG hierarchy for parity tests.
#include <string.h>

#include <algorithm>
#include <stdexcept>
#include <new>
#include <string>

#include "jxcpr_b200.h"
#include "handle.cuh"

using namespace jxcpr;


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

int set_int_param(SolverParams &p, const char *key, int v) {
    struct {
        const char *k;
        int *f;
    } tab[] = {{"k_dim", &p.k_dim},
               {"max_iter", &p.max_iter},
               {"min_iter", &p.min_iter},
               {"is_check_restarted", &p.is_check_restarted},
               {"print_level", &p.print_level},
               {"logging", &p.logging},
               {"pressure_index", &p.pressure_index},
               {"stage1_maxit", &p.stage1_maxit},
               {"stage2_maxit", &p.stage2_maxit},
               {"stage1_solver_type", &p.stage1_solver_type},
               {"stage2_solver_type", &p.stage2_solver_type},
               {"decouple", &p.decouple},
               {"thermal", &p.thermal},
               {"consistent_rhs", &p.consistent_rhs},
               {"smoother_order", &p.smoother_order},
               {"coarse_exact", &p.coarse_exact},
               {"max_colors", &p.max_colors},
               {"rs_range_rows", &p.rs_range_rows},
               {"rs_range_rows_coarse", &p.rs_range_rows_coarse},
               {"dep_launch", &p.dep_launch},
               {"use_tma_spmv", &p.use_tma_spmv},
               {"precision", &p.precision},
               {"bf16_level", &p.bf16_level},
               {"fast_smoother", &p.fast_smoother},
               {"stage2_lanes", &p.stage2_lanes},
               {"stage2_chunk", &p.stage2_chunk},
               {"tail_rows", &p.tail_rows},
               {"sell_lanes", &p.sell_lanes},
               {"tail_ctas", &p.tail_ctas},
               {"learned_fallback", &p.learned_fallback},
               {"record_features", &p.record_features},
               {"flexible", &p.flexible},
               {"autotune", &p.autotune},
               {"graphs", &p.graphs},
               {"orthog", &p.orthog},
               {"graph_gmres", &p.graph_gmres},
               {"krylov_fp32", &p.krylov_fp32},
               {"selective_reorth", &p.selective_reorth},
               {"bilu_sweeps", &p.bilu_sweeps},
               {"bilu_ir_iters", &p.bilu_ir_iters},
               {"bilu_lower_iters", &p.bilu_lower_iters},
               {"bilu_upper_iters", &p.bilu_upper_iters},
               {"bilu_exact", &p.bilu_exact}};
    if (!key) return JXCPR_ERROR_ARG;
    if (!strcmp(key, "block_size")) return JXCPR_SUCCESS;  // taken from the matrix, as the reference's setup does
    if (!strcmp(key, "stage2_chunk") && v != 0 && v != 4 && v != 8 && v != 16) {
        set_error("stage2_chunk must be 0, 4, 8 or 16 (got %d)", v);
        return JXCPR_ERROR_ARG;
    }
    for (auto &e : tab)
        if (!strcmp(key, e.k)) {
            *e.f = v;
            return JXCPR_SUCCESS;
        }
    set_error("unknown integer parameter '%s'", key);
    return JXCPR_ERROR_ARG;
}

int set_real_param(SolverParams &p, const char *key, double v) {
    struct {
        const char *k;
        double *f;
    } tab[] = {{"tol", &p.tol},
               {"a_tol", &p.a_tol},
               {"threshold", &p.threshold},
               {"convfac_threshold", &p.convfac_threshold},
               {"stage2_relax_weight", &p.stage2_relax_weight},
               {"stage2_omega", &p.stage2_omega},
               {"strong_threshold", &p.strong_threshold},
               {"strong_threshold_coarse", &p.strong_threshold_coarse},
               {"cheb_lower", &p.cheb_lower},
               {"cheb_upper", &p.cheb_upper},
               {"jacobi_mean_row", &p.jacobi_mean_row}};
    if (!key) return JXCPR_ERROR_ARG;
    for (auto &e : tab)
        if (!strcmp(key, e.k)) {
            *e.f = v;
            return JXCPR_SUCCESS;
        }
    set_error("unknown real parameter '%s'", key);
    return JXCPR_ERROR_ARG;
}
}  // namespace

extern "C" {

int jxcpr_solver_create(jxcpr_solver **h) {
    if (!h) return JXCPR_ERROR_ARG;
    *h = new (std::nothrow) jxcpr_solver();
    return *h ? JXCPR_SUCCESS : JXCPR_ERROR_MEMORY;
}

int jxcpr_solver_destroy(jxcpr_solver *h) {
    if (!h) return JXCPR_ERROR_ARG;
    return guarded([&] {
        const bool owns = h->s.owns_stream;
        cudaStream_t st = h->s.stream;
        if (owns) cudaStreamSynchronize(st);
        delete h;
        if (owns) {
            pool_forget_stream(st, true);  // synchronised above: its blocks are free for any stream
            cudaStreamDestroy(st);
        }
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_set_stream(jxcpr_solver *h, void *stream) {
    if (!h) return JXCPR_ERROR_ARG;
    // Blocks made for the previous stream must not be reused on it once the solver's work goes to
    // another stream (that work is not ordered after the old stream's).
    cudaStream_t old = h->s.stream;
    if (h->s.owns_stream && old) {
        cudaStreamSynchronize(old);
        pool_forget_stream(old, true);
        cudaStreamDestroy(old);
    } else if (h->s.stream_set && old != (cudaStream_t)stream) {
        pool_forget_stream(old, false);
    }
    h->s.stream = (cudaStream_t)stream;
    h->s.owns_stream = false;
    h->s.stream_set = true;
    return JXCPR_SUCCESS;
}

int jxcpr_solver_set_int(jxcpr_solver *h, const char *key, int value) {
    if (!h) return JXCPR_ERROR_ARG;
    return set_int_param(h->s.prm, key, value);
}

int jxcpr_solver_set_real(jxcpr_solver *h, const char *key, double value) {
    if (!h) return JXCPR_ERROR_ARG;
    return set_real_param(h->s.prm, key, value);
}

int jxcpr_solver_setup(jxcpr_solver *h, int nb, int bs, long long nnzb, const int *ia, const int *ja,
                       const double *a, int device) {
    if (!h || nb < 0 || nnzb < 0 || (bs != 2 && bs != 3) || !ia || (nnzb && (!ja || !a))) {
        set_error("solver_setup: bad arguments");
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] {
        h->s.setup(nb, bs, nnzb, ia, ja, a, device);
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_solve(jxcpr_solver *h, const double *b, double *x, int device, int *iterations,
                       double *rel_residual) {
    if (!h || !b || !x || !h->s.cpr.ready) {
        set_error("solver_solve: bad arguments or no setup");
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] {
        GmresResult r = h->s.solve(b, x, device);
        if (iterations) *iterations = r.iterations;
        if (rel_residual) *rel_residual = r.rel_residual;
        if (r.status) return r.status;
        return r.converged ? JXCPR_SUCCESS : JXCPR_ERROR_CONV;
    });
}

int jxcpr_solver_get_norms(jxcpr_solver *h, double *norms, int capacity) {
    if (!h || !norms) return -1;
    const int n = (int)h->s.last.norms.size();
    for (int i = 0; i < n && i < capacity; ++i) norms[i] = h->s.last.norms[i];
    return n;
}

int jxcpr_solver_stats(jxcpr_solver *h, double *stats) {
    if (!h || !stats) return JXCPR_ERROR_ARG;
    stats[0] = h->s.setup_ms;
    stats[1] = h->s.solve_ms;
    stats[2] = h->s.cpr.stats[0];
    stats[3] = (double)h->s.cpr.amg.num_levels();
    return JXCPR_SUCCESS;
}

int jxcpr_solver_setup_report(jxcpr_solver *h, char *buf, int capacity) {
    if (!h || !buf || capacity <= 0) return -1;
    std::string out;
    char line[160];
    snprintf(line, sizeof line, "upload %.2f ms\ndecouple %.2f ms\n", h->s.upload_ms, h->s.decouple_ms);
    out += line;
    for (auto &kv : h->s.cpr.amg.log.items) {
        snprintf(line, sizeof line, "%s %.2f ms\n", kv.first.c_str(), kv.second);
        out += line;
    }
    snprintf(line, sizeof line, "total %.2f ms\n", h->s.setup_ms);
    out += line;
    const double *al = h->s.alloc_stats;
    snprintf(line, sizeof line, "device memory: %.0f cudaMalloc (%.2f ms), %.0f device syncs (%.2f ms)\n", al[0],
             al[1], al[2], al[3]);
    out += line;
    if (h->s.cpr.fast)
        for (const std::string &t : h->s.cpr.fast->tune_log) out += "tuned " + t + "\n";
    const int n = (int)std::min<size_t>(out.size(), (size_t)capacity - 1);
    memcpy(buf, out.data(), n);
    buf[n] = 0;
    return n;
}

int jxcpr_solver_num_levels(jxcpr_solver *h) { return h ? h->s.cpr.amg.num_levels() : -1; }

int jxcpr_solver_level_sizes(jxcpr_solver *h, int lev, int what, int *sizes) {
    if (!h || !sizes || lev < 0 || lev >= h->s.cpr.amg.num_levels()) return -1;
    const AmgLevel &L = *h->s.cpr.amg.levels[lev];
    const DeviceCsr &M = what == 0 ? L.A : (what == 1 ? L.P : L.R);
    if (what != 0 && lev == h->s.cpr.amg.num_levels() - 1) return -1;
    sizes[0] = M.nrows;
    sizes[1] = M.ncols;
    sizes[2] = (int)M.nnz;
    return 0;
}

int jxcpr_solver_level_matrix(jxcpr_solver *h, int lev, int what, int *ia, int *ja, double *a) {
    int sz[3];
    if (jxcpr_solver_level_sizes(h, lev, what, sz) < 0) return -1;
    return guarded([&] {
        const AmgLevel &L = *h->s.cpr.amg.levels[lev];
        const DeviceCsr &M = what == 0 ? L.A : (what == 1 ? L.P : L.R);
        JX_CUDA(cudaMemcpy(ia, M.ia.get(), sizeof(int) * (sz[0] + 1), cudaMemcpyDeviceToHost));
        JX_CUDA(cudaMemcpy(ja, M.ja.get(), sizeof(int) * sz[2], cudaMemcpyDeviceToHost));
        JX_CUDA(cudaMemcpy(a, M.a.get(), sizeof(double) * sz[2], cudaMemcpyDeviceToHost));
        return 0;
    });
}

int jxcpr_solver_level_info(jxcpr_solver *h, int lev, int *smoother, int *storage, double *theta,
                            double *cheb) {
    if (!h || lev < 0 || lev >= h->s.cpr.amg.num_levels()) return -1;
    const CprPrecond &C = h->s.cpr;
    if (theta) *theta = C.amg.levels[lev]->theta;
    if (C.fast) {
        C.fast->level_info(lev, smoother, storage, cheb);
    } else {
        if (smoother) *smoother = 0;
        if (storage) *storage = 0;
        if (cheb)
            for (int k = 0; k < 6; ++k) cheb[k] = 0.0;
    }
    return 0;
}

int jxcpr_solver_level_features(jxcpr_solver *h, int lev, float *out) {
    if (!h || !out || lev < 0 || lev >= (int)h->s.cpr.plan.features.size()) return -1;
    const std::vector<float> &f = h->s.cpr.plan.features[lev];
    memcpy(out, f.data(), sizeof(float) * f.size());
    return (int)f.size();
}

int jxcpr_solver_learned_status(jxcpr_solver *h, double *out) {
    if (!h || !out) return JXCPR_ERROR_ARG;
    out[0] = h->s.cpr.learned_used;
    out[1] = h->s.cpr.factor_fast;
    out[2] = h->s.cpr.factor_plain;
    out[3] = h->s.cpr.probe_bytes[0];
    out[4] = h->s.cpr.probe_bytes[1];
    return JXCPR_SUCCESS;
}

int jxcpr_solver_learned_fallbacks(jxcpr_solver *h) { return h ? h->s.learned_fallbacks : -1; }

int jxcpr_solver_level_cf(jxcpr_solver *h, int lev, int *cf) {
    if (!h || !cf || lev < 0 || lev >= h->s.cpr.amg.num_levels() - 1) return -1;
    const std::vector<int> &v = h->s.cpr.amg.levels[lev]->cf;
    memcpy(cf, v.data(), sizeof(int) * v.size());
    return 0;
}

int jxcpr_solver_decoupled_values(jxcpr_solver *h, double *a_host) {
    if (!h || !a_host) return JXCPR_ERROR_ARG;
    return guarded([&] {
        const DeviceBsr &A = h->s.A;
        JX_CUDA(cudaMemcpy(a_host, A.a.get(), sizeof(double) * A.nnzb * A.bs * A.bs, cudaMemcpyDeviceToHost));
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_cpr_apply(jxcpr_solver *h, const double *r, double *z, int device) {
    if (!h || !r || !z || !h->s.cpr.ready) return JXCPR_ERROR_ARG;
    return guarded([&] {
        Solver &S = h->s;
        const long long n = (long long)S.A.nb * S.A.bs;
        cudaStream_t st = S.stream;
        const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        JX_CUDA(cudaMemcpyAsync(S.b.get(), r, sizeof(double) * n, in, st));
        JX_CUDA(cudaMemsetAsync(S.x.get(), 0, sizeof(double) * n, st));
        S.cpr.apply(S.b.get(), S.x.get(), st);
        const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        JX_CUDA(cudaMemcpyAsync(z, S.x.get(), sizeof(double) * n, out, st));
        JX_CUDA(cudaStreamSynchronize(st));
        int f = 0;
        JX_CUDA(cudaMemcpy(&f, S.cpr.amg.err.get(), sizeof(int), cudaMemcpyDeviceToHost));
        if (f) {
            set_error("smoother wait timed out");
            return JXCPR_ERROR_DEVICE;
        }
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_stage2_sweep(jxcpr_solver *h, const double *b, double *x, int device) {
    if (!h || !b || !x || !h->s.cpr.ready) return JXCPR_ERROR_ARG;
    return guarded([&] {
        Solver &S = h->s;
        const long long n = (long long)S.A.nb * S.A.bs;
        cudaStream_t st = S.stream;
        const double *bd = b;
        double *xd = x;
        if (!device) {
            JX_CUDA(cudaMemcpyAsync(S.b.get(), b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
            JX_CUDA(cudaMemcpyAsync(S.x.get(), x, sizeof(double) * n, cudaMemcpyHostToDevice, st));
            bd = S.b.get();
            xd = S.x.get();
        }
        S.cpr.stage2_sweep(bd, xd, st);
        if (!device) {
            JX_CUDA(cudaMemcpyAsync(x, S.x.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, st));
            JX_CUDA(cudaStreamSynchronize(st));
        }
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_bilu_sizes(jxcpr_solver *h, long long *sizes) {
    if (!h || !sizes || !h->s.cpr.bilu) return JXCPR_ERROR_ARG;
    sizes[0] = h->s.cpr.bilu->L.nnzb;
    sizes[1] = h->s.cpr.bilu->U.nnzb;
    return JXCPR_SUCCESS;
}

int jxcpr_solver_bilu_factors(jxcpr_solver *h, double *la, double *ua, double *dinv) {
    if (!h || !h->s.cpr.bilu) return JXCPR_ERROR_ARG;
    return guarded([&] {
        const Bilu &B = *h->s.cpr.bilu;
        const size_t bn = (size_t)B.bs * B.bs;
        if (la && B.L.nnzb) JX_CUDA(cudaMemcpy(la, B.L.a.get(), sizeof(double) * B.L.nnzb * bn, cudaMemcpyDeviceToHost));
        if (ua && B.U.nnzb) JX_CUDA(cudaMemcpy(ua, B.U.a.get(), sizeof(double) * B.U.nnzb * bn, cudaMemcpyDeviceToHost));
        if (dinv && B.nb) JX_CUDA(cudaMemcpy(dinv, B.Dinv.get(), sizeof(double) * B.nb * bn, cudaMemcpyDeviceToHost));
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_bilu_apply(jxcpr_solver *h, const double *f, double *u, int device) {
    if (!h || !f || !u || !h->s.cpr.bilu) return JXCPR_ERROR_ARG;
    return guarded([&] {
        Solver &S = h->s;
        const long long n = (long long)S.A.nb * S.A.bs;
        cudaStream_t st = S.stream;
        const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        JX_CUDA(cudaMemcpyAsync(S.b.get(), f, sizeof(double) * n, in, st));
        JX_CUDA(cudaMemsetAsync(S.x.get(), 0, sizeof(double) * n, st));
        S.cpr.bilu->solve(S.A.view(), S.b.get(), S.x.get(), st);
        const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        JX_CUDA(cudaMemcpyAsync(u, S.x.get(), sizeof(double) * n, out, st));
        JX_CUDA(cudaStreamSynchronize(st));
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_stage2_native(jxcpr_solver *h, int sweeps) {
    if (!h || sweeps < 0 || !h->s.cpr.ready) return JXCPR_ERROR_ARG;
    if (!h->s.cpr.fast) {
        set_error("stage2_native needs the fast path (smoother_order 1)");
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] {
        h->s.cpr.fast->stage2_native(sweeps, h->s.stream);
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_vcycle(jxcpr_solver *h, const double *rp, double *xp, int device) {
    if (!h || !rp || !xp || !h->s.cpr.ready) return JXCPR_ERROR_ARG;
    return guarded([&] {
        Solver &S = h->s;
        const int nb = S.A.nb;
        cudaStream_t st = S.stream;
        const cudaMemcpyKind in = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        JX_CUDA(cudaMemcpyAsync(S.cpr.rp.get(), rp, sizeof(double) * nb, in, st));
        JX_CUDA(cudaMemcpyAsync(S.cpr.xp.get(), xp, sizeof(double) * nb, in, st));
        S.cpr.vcycle(S.cpr.rp.get(), S.cpr.xp.get(), st);
        const cudaMemcpyKind out = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        JX_CUDA(cudaMemcpyAsync(xp, S.cpr.xp.get(), sizeof(double) * nb, out, st));
        JX_CUDA(cudaStreamSynchronize(st));
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_bilu_levels(jxcpr_solver *h, int *lev_l, int *lev_u, int *counts) {
    if (!h || !h->s.cpr.bilu) return JXCPR_ERROR_ARG;
    const Bilu &B = *h->s.cpr.bilu;
    if (!B.exact) {
        set_error("bilu_levels: the level schedule exists with bilu_exact 1 only");
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] {
        if (counts) {
            counts[0] = B.nlev_l;
            counts[1] = B.nlev_u;
        }
        if (lev_l && B.nb) JX_CUDA(cudaMemcpy(lev_l, B.lev_l.get(), sizeof(int) * B.nb, cudaMemcpyDeviceToHost));
        if (lev_u && B.nb) JX_CUDA(cudaMemcpy(lev_u, B.lev_u.get(), sizeof(int) * B.nb, cudaMemcpyDeviceToHost));
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_level_stored_values(jxcpr_solver *h, int level, double *values) {
    if (!h || !values || !h->s.cpr.ready || !h->s.cpr.fast) return JXCPR_ERROR_ARG;
    return guarded([&] {
        Solver &S = h->s;
        if (level < 0 || level >= (int)S.cpr.amg.levels.size()) {
            set_error("level_stored_values: no level %d", level);
            return JXCPR_ERROR_ARG;
        }
        const long long nnz = S.cpr.amg.levels[level]->A.nnz;
        DevBuf<double> out(nnz > 0 ? nnz : 1);
        JX_CUDA(cudaMemsetAsync(out.get(), 0, sizeof(double) * (nnz > 0 ? nnz : 1), S.stream));
        if (!S.cpr.fast->stored_values(level, out.get(), S.stream)) {
            set_error("level_stored_values: level %d has no smoothed operator", level);
            return JXCPR_ERROR_ARG;
        }
        if (nnz) JX_CUDA(cudaMemcpyAsync(values, out.get(), sizeof(double) * nnz, cudaMemcpyDeviceToHost, S.stream));
        JX_CUDA(cudaStreamSynchronize(S.stream));
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_level_native(jxcpr_solver *h, int level, int op, int reps) {
    if (!h || reps < 0 || op < 0 || op > 2 || !h->s.cpr.ready) return JXCPR_ERROR_ARG;
    if (!h->s.cpr.fast) {
        set_error("level_native needs the fast path (smoother_order 1)");
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] {
        if (!h->s.cpr.fast->level_native(level, op, reps, h->s.stream)) {
            set_error("level_native: level %d has no smoothed operator", level);
            return JXCPR_ERROR_ARG;
        }
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_krylov_native(jxcpr_solver *h, int m, int reps) {
    if (!h || reps < 0) return JXCPR_ERROR_ARG;
    if (!h->s.ggmres || !h->s.ggmres->exec) {
        set_error("krylov_native needs a solve with graph_gmres 1 first");
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] {
        h->s.ggmres->orth_native(m, reps, h->s.gmres.w.get(), h->s.stream);
        return JXCPR_SUCCESS;
    });
}

int jxcpr_solver_apply_bytes(jxcpr_solver *h, double *bytes) {
    if (!h || !bytes || !h->s.cpr.ready) return JXCPR_ERROR_ARG;
    if (!h->s.cpr.fast) {
        set_error("apply_bytes needs the fast path (smoother_order 1)");
        return JXCPR_ERROR_ARG;
    }
    *bytes = h->s.cpr.fast->apply_bytes();
    return JXCPR_SUCCESS;
}

int jxcpr_stage2_chunk_order(int nb, const int *ia, const int *ja, int chunk, int *order, int capacity,
                             int *segments, int seg_capacity) {
    if (nb < 0 || (nb > 0 && (!ia || !ja)) || (chunk != 4 && chunk != 8 && chunk != 16) || capacity < 0) {
        set_error("stage2_chunk_order: bad arguments");
        return -JXCPR_ERROR_ARG;
    }
    try {
        std::vector<int> ord, seg;
        build_chunk_order_host(nb, ia, ja, chunk, ord, seg);
        if (order && (size_t)capacity >= ord.size()) std::copy(ord.begin(), ord.end(), order);
        if (segments && (size_t)seg_capacity >= seg.size()) std::copy(seg.begin(), seg.end(), segments);
        return (int)ord.size();
    } catch (...) {
        set_error("stage2_chunk_order: host allocation failed");
        return -JXCPR_ERROR_MEMORY;
    }
}

}  // extern "C"
