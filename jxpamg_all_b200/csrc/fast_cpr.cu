// Fast CPR preconditioner: storage conversion (CSR / sliced ELL, FP64 / FP32 /
// BF16), V-cycle and stage 2 (see fast.cuh for the modes).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <memory>
#include <numeric>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>

#include "fast.cuh"
#include "fast_kernels.cuh"
#include "fast_tail.cuh"

namespace jxcpr {

namespace {
constexpr int kThreads = 256;
constexpr int kSellWindow = 512;  // rows sorted by length inside windows of this many rows

// Calls f(values pointer) with the storage type of M: FP64 for the FP64 path,
// FP32 / BF16 for the mixed path.
template <typename TX, typename F>
void with_values(const LevelMat &M, F &&f) {
    if constexpr (std::is_same<TX, double>::value) {
        f(M.a64.get());
    } else {
        if (M.kind == VAL_BF16) f(M.a16.get());
        else f(M.a32.get());
    }
}

template <typename T>
void alloc_vec(DevBuf<T> &b, long long n) {
    b.alloc(n > 0 ? n : 1);
}

// ---- launch of a row operation over stored rows [r0, r1) -------------------------
template <typename TX, int V, typename TV, class Op>
void launch_csr(const LevelMat &M, const TV *a, const Op &op, int r0, int r1, cudaStream_t s) {
    fk::CsrFmt<V, TV> f{M.ia.get(), M.ja.get(), a, M.bscale.get(), M.perm};
    const long long threads = (long long)(r1 - r0) * V;
    launch_dep(fk::row_kernel<fk::CsrFmt<V, TV>, Op, TX>, dim3(div_up(threads, kThreads)), dim3(kThreads), s,
               f, op, r0, r1);
}

template <typename TX, class Op>
void launch_rows(const LevelMat &M, const Op &op, int r0, int r1, cudaStream_t s) {
    if (r1 <= r0) return;
    with_values<TX>(M, [&](auto a) {
        using TV = typename std::remove_cv<typename std::remove_pointer<decltype(a)>::type>::type;
        if (M.sell == 2) {
            fk::SellFmt<TV, 2> f{M.sp.get(), M.ja.get(), a, M.bscale.get(), M.rows.get()};
            launch_dep(fk::row_kernel<fk::SellFmt<TV, 2>, Op, TX>, dim3(div_up((long long)(r1 - r0) * 2, kThreads)),
                       dim3(kThreads), s, f, op, r0, r1);
            return;
        }
        if (M.sell) {
            fk::SellFmt<TV> f{M.sp.get(), M.ja.get(), a, M.bscale.get(), M.rows.get()};
            launch_dep(fk::row_kernel<fk::SellFmt<TV>, Op, TX>, dim3(div_up(r1 - r0, kThreads)), dim3(kThreads), s,
                       f, op, r0, r1);
            return;
        }
        switch (M.lanes) {
            case 1: launch_csr<TX, 1>(M, a, op, r0, r1, s); break;
            case 2: launch_csr<TX, 2>(M, a, op, r0, r1, s); break;
            case 4: launch_csr<TX, 4>(M, a, op, r0, r1, s); break;
            case 8: launch_csr<TX, 8>(M, a, op, r0, r1, s); break;
            case 16: launch_csr<TX, 16>(M, a, op, r0, r1, s); break;
            default: launch_csr<TX, 32>(M, a, op, r0, r1, s); break;
        }
    });
    JX_LAUNCH_CHECK();
}

// ---- construction -----------------------------------------------------------------
// Sliced-ELL layout on the host: segments of `order` (offsets seg_in), rows
// sorted by decreasing length inside windows (a stable counting sort: equal
// lengths keep their order), a segment's windows heaviest first, each segment
// padded to whole slices.  Windows
// are independent (each starts on a slice boundary), so large layouts sort
// them on host threads.  P lanes per row (SellFmt<TV, P>): a slice holds 32 / P
// stored rows, and its width is the slots of its longest row's lane 0.
void sell_layout(const std::vector<int> &ia, const std::vector<int> &order, const std::vector<int> &seg_in,
                 std::vector<int> &rows, std::vector<long long> &sp, std::vector<int> &seg_out, int P = 1) {
    const int SR = 32 / P;  // stored rows per slice
    struct Win {
        int w0, w1;
        size_t pos;
    };
    std::vector<Win> wins;
    seg_out.assign(1, 0);
    size_t pos = 0;
    for (size_t c = 0; c + 1 < seg_in.size(); ++c) {
        // a segment's full windows heaviest first (most entries; stable), its short last window last:
        // the blocks launched last, which run with the grid's tail, then hold the lightest rows
        std::vector<std::pair<long long, int>> full;
        int tail0 = seg_in[c + 1];
        for (int w0 = seg_in[c]; w0 < seg_in[c + 1]; w0 += kSellWindow) {
            if (w0 + kSellWindow > seg_in[c + 1]) {
                tail0 = w0;
                break;
            }
            long long work = 0;
            for (int t = w0; t < w0 + kSellWindow; ++t) work += ia[order[t] + 1] - ia[order[t]];
            full.push_back({work, w0});
        }
        std::stable_sort(full.begin(), full.end(),
                         [](const std::pair<long long, int> &x, const std::pair<long long, int> &y) {
                             return x.first > y.first;
                         });
        for (const auto &f : full) {
            wins.push_back({f.second, f.second + kSellWindow, pos});
            pos += kSellWindow;
        }
        if (tail0 < seg_in[c + 1]) {
            wins.push_back({tail0, seg_in[c + 1], pos});
            pos += seg_in[c + 1] - tail0;
        }
        pos = (pos + SR - 1) / SR * SR;
        seg_out.push_back((int)pos);
    }
    const size_t total = pos, ns = total / SR;
    rows.assign(total, -1);
    std::vector<int> width(ns, 0);
    auto sort_windows = [&](size_t b, size_t e) {
        std::vector<int> len, cnt, slen;
        for (size_t k = b; k < e; ++k) {
            const Win &W = wins[k];
            const int nw = W.w1 - W.w0;
            len.resize(nw);
            slen.resize(nw);
            int maxlen = 0;
            for (int t = 0; t < nw; ++t) {
                const int i = order[W.w0 + t];
                len[t] = ia[i + 1] - ia[i];
                maxlen = std::max(maxlen, len[t]);
            }
            cnt.assign((size_t)maxlen + 2, 0);  // key maxlen - len: longest rows first
            for (int t = 0; t < nw; ++t) cnt[maxlen - len[t] + 1]++;
            for (int q = 0; q <= maxlen; ++q) cnt[q + 1] += cnt[q];
            for (int t = 0; t < nw; ++t) {
                const int q = cnt[maxlen - len[t]]++;
                rows[W.pos + q] = order[W.w0 + t];
                slen[q] = len[t];
            }
            // a window starts on a slice boundary and its slices hold its rows alone (the
            // padding of a segment's last slice follows its last window), longest first
            for (int q = 0; q < nw; q += SR) width[W.pos / SR + q / SR] = (slen[q] + P - 1) / P;
        }
    };
    const size_t nwin = wins.size();
    const int threads = total >= (size_t)(1 << 16)
                            ? (int)std::min<size_t>(std::min<size_t>(nwin, 16),
                                                    std::max(1u, std::thread::hardware_concurrency()))
                            : 1;
    if (threads <= 1) {
        sort_windows(0, nwin);
    } else {
        std::vector<std::thread> pool;
        for (int t = 1; t < threads; ++t) pool.emplace_back(sort_windows, nwin * t / threads, nwin * (t + 1) / threads);
        sort_windows(0, nwin / threads);
        for (auto &th : pool) th.join();
    }
    sp.assign(ns + 1, 0);
    for (size_t sl = 0; sl < ns; ++sl) sp[sl + 1] = sp[sl] + 32LL * width[sl];
}

template <typename TV>
void sell_fill_launch(LevelMat &M, const int *ia, const int *ja, const double *a, TV *val, float *bscale,
                      cudaStream_t s, int sorted = 0) {
    if (!M.nstored) return;
    fk::sell_fill<TV><<<div_up(M.nstored, kThreads), kThreads, 0, s>>>(M.nstored, M.rows.get(), M.sp.get(), ia, ja,
                                                                      a, M.E, M.ja.get(), val, bscale, sorted);
    JX_LAUNCH_CHECK();
}

// Builds M from a CSR (E = 1) or BSR (E = bs*bs) operator on the device.
//  order / seg: host storage order of the rows and its segments (empty order:
//  natural order, one segment); order_dev: the same order on the device (CSR layout).
//  FP32 CSR operators (E = 1) keep each row's entries after the first in ascending column order: the
//  lanes and slots of a warp then gather nearby columns (measured on C1: level-1 step 27.9 -> 27.0 us,
//  level 2 12.6 -> 11.9 us; C4 level 1 20.2 -> 19.0 us).  The row sums' order changes with it; the
//  fast path's contract is the FP64 true residual, not a fixed summation order.
void build_level_mat(int n, int m, long long nnz, int E, const int *ia, const int *ja, const double *a, int kind,
                     int sell, const std::vector<int> &order, const std::vector<int> &seg, const int *order_dev,
                     LevelMat &M, cudaStream_t s) {
    // sell: 0 CSR, 1 sliced ELL, 2 sliced ELL with two lanes per row (E = 1, FP32 / FP64 values)
    if (sell == 2 && (E != 1 || kind == VAL_BF16)) sell = 1;
    M.n = n;
    M.m = m;
    M.nnz = nnz;
    M.E = E;
    M.kind = kind;
    M.sell = sell;
    const bool natural = order.empty();
    if (sell) {
        std::vector<int> ia_h(n + 1);
        JX_CUDA(cudaMemcpyAsync(ia_h.data(), ia, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
        JX_CUDA(cudaStreamSynchronize(s));
        std::vector<int> ord, sg;
        if (natural) {
            ord.resize(n);
            std::iota(ord.begin(), ord.end(), 0);
            sg = {0, n};
        }
        std::vector<int> rows;
        std::vector<long long> sp;
        sell_layout(ia_h, natural ? ord : order, natural ? sg : seg, rows, sp, M.seg, sell);
        M.nstored = (int)rows.size();
        const long long slots = sp.back();
        M.rows.alloc(rows.size() + 1);
        M.rows.upload(rows.data(), rows.size(), s);
        M.sp.alloc(sp.size());
        M.sp.upload(sp.data(), sp.size(), s);
        M.ja.alloc(slots > 0 ? slots : 1);
        const long long nv = (slots > 0 ? slots : 1) * E;
        if (sell == 2) {
            const long long lanes = (long long)M.nstored * 2;
            if (kind == VAL_F64) {
                M.a64.alloc(nv);
                if (lanes)
                    fk::sell_fill_lanes<double><<<div_up(lanes, kThreads), kThreads, 0, s>>>(
                        M.nstored, 2, M.rows.get(), M.sp.get(), ia, ja, a, M.ja.get(), M.a64.get(), 0);
            } else {
                M.a32.alloc(nv);
                if (lanes)
                    fk::sell_fill_lanes<float><<<div_up(lanes, kThreads), kThreads, 0, s>>>(
                        M.nstored, 2, M.rows.get(), M.sp.get(), ia, ja, a, M.ja.get(), M.a32.get(), 1);
            }
            JX_LAUNCH_CHECK();
        } else if (kind == VAL_F64) {
            M.a64.alloc(nv);
            sell_fill_launch<double>(M, ia, ja, a, M.a64.get(), nullptr, s);
        } else if (kind == VAL_F32) {
            M.a32.alloc(nv);
            sell_fill_launch<float>(M, ia, ja, a, M.a32.get(), nullptr, s, E == 1);
        } else {
            M.a16.alloc(nv);
            M.bscale.alloc((size_t)(slots > 0 ? slots : 1) / 32 + 1);
            sell_fill_launch<__nv_bfloat16>(M, ia, ja, a, M.a16.get(), M.bscale.get(), s);
        }
        JX_CUDA(cudaStreamSynchronize(s));
        return;
    }
    // CSR layout (rows permuted into `order` when given)
    M.nstored = n;
    M.seg = natural ? std::vector<int>{0, n} : seg;
    M.perm = natural ? nullptr : order_dev;
    M.lanes = lanes_for(n > 0 ? (double)nnz / n : 1.0);
    const int *src_ia = ia, *src_ja = ja;
    const double *src_a = a;
    DeviceCsr pc;
    DeviceBsr pb;
    if (!natural) {
        if (E == 1) {
            permute_rows_csr(CsrView<double>{n, m, nnz, ia, ja, a}, order_dev, pc, s);
            src_ia = pc.ia.get();
            src_ja = pc.ja.get();
            src_a = pc.a.get();
        } else {
            const int bs = E == 4 ? 2 : 3;
            permute_rows_bsr(BsrView<double>{n, bs, nnz, ia, ja, a}, order_dev, pb, s);
            src_ia = pb.ia.get();
            src_ja = pb.ja.get();
            src_a = pb.a.get();
        }
    }
    M.ia.alloc((size_t)n + 1);
    JX_CUDA(cudaMemcpyAsync(M.ia.get(), src_ia, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
    M.ja.alloc(nnz > 0 ? nnz : 1);
    if (nnz) JX_CUDA(cudaMemcpyAsync(M.ja.get(), src_ja, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
    const long long nv = (nnz > 0 ? nnz : 1) * E;
    if (kind == VAL_F64) {
        M.a64.alloc(nv);
        if (nnz) JX_CUDA(cudaMemcpyAsync(M.a64.get(), src_a, sizeof(double) * nnz * E, cudaMemcpyDeviceToDevice, s));
    } else if (kind == VAL_F32) {
        M.a32.alloc(nv);
        if (nnz) {
            fk::to_f32<<<div_up(nnz * E, kThreads), kThreads, 0, s>>>(nnz * E, src_a, M.a32.get());
            JX_LAUNCH_CHECK();
            if (E == 1 && n > 0) {
                fk::sort_row_entries<float><<<div_up(n, kThreads), kThreads, 0, s>>>(n, M.ia.get(), M.ja.get(), M.a32.get());
                JX_LAUNCH_CHECK();
            }
        }
    } else {
        M.a16.alloc(nv);
        M.bscale.alloc((size_t)(nnz > 0 ? nnz : 1) / 32 + 1);
        if (nnz) {
            fk::to_bf16_blocks<<<div_up(nnz, kThreads), kThreads, 0, s>>>(nnz, src_a, M.bscale.get(), M.a16.get());
            JX_LAUNCH_CHECK();
        }
    }
    JX_CUDA(cudaStreamSynchronize(s));
}

// Stage-2 block matrix in chunk order (fk::hgs_chunk): stored rows = `order` (chunks of `chunk`
// consecutive rows, -1 padding, colour segments `seg` on slice boundaries), sliced ELL without the
// length sort, so that every chunk keeps its rows in order at lanes 0..chunk-1 of its slice part.
void build_chunk_mat(int n, long long nnz, int E, const int *ia, const int *ja, const double *a, int kind,
                     const std::vector<int> &order, const std::vector<int> &seg, int chunk, const int *cls_dev,
                     LevelMat &M, cudaStream_t s) {
    if (n >= (1 << 30)) {
        set_error("stage 2 in chunk order: %d block rows exceed the 30-bit column words", n);
        throw std::invalid_argument("chunk order size");
    }
    M.n = n;
    M.m = n;
    M.nnz = nnz;
    M.E = E;
    M.kind = kind;
    M.sell = 1;
    M.chunk = chunk;
    M.seg = seg;
    M.nstored = (int)order.size();
    std::vector<int> ia_h(n + 1);
    JX_CUDA(cudaMemcpyAsync(ia_h.data(), ia, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    const size_t ns = order.size() / 32;
    std::vector<long long> sp(ns + 1, 0);
    for (size_t sl = 0; sl < ns; ++sl) {
        int wd = 0;
        for (int q = 0; q < 32; ++q) {
            const int i = order[sl * 32 + q];
            if (i >= 0) wd = std::max(wd, ia_h[i + 1] - ia_h[i]);
        }
        sp[sl + 1] = sp[sl] + 32LL * wd;
    }
    M.rows.alloc(order.size() + 1);
    M.rows.upload(order.data(), order.size(), s);
    M.sp.alloc(sp.size());
    M.sp.upload(sp.data(), sp.size(), s);
    const long long slots = sp.back();
    M.ja.alloc(slots > 0 ? slots : 1);
    const long long nv = (slots > 0 ? slots : 1) * E;
    if (kind == VAL_F64) {
        M.a64.alloc(nv);
        sell_fill_launch<double>(M, ia, ja, a, M.a64.get(), nullptr, s);
    } else {
        M.a32.alloc(nv);
        sell_fill_launch<float>(M, ia, ja, a, M.a32.get(), nullptr, s);
    }
    if (M.nstored) {
        fk::chunk_col_flags<<<div_up(M.nstored, kThreads), kThreads, 0, s>>>(
            M.nstored, M.rows.get(), M.sp.get(), ia, cls_dev, chunk, reinterpret_cast<unsigned *>(M.ja.get()));
        JX_LAUNCH_CHECK();
    }
    JX_CUDA(cudaStreamSynchronize(s));
}

bool use_sell(const FastOptions &o, int n, long long nnz) {
    return n >= o.sell_min_rows && n > 0 && (double)nnz / n <= o.sell_max_mean;
}

// Device time (us) of `body`: the best of `trials` means over `reps` runs, after a warm-up run
// (the minimum keeps one slow trial -- a clock ramp, another stream's burst -- from deciding).
template <typename F>
double time_best(F &&body, cudaStream_t s, int reps = 3, int trials = 3) {
    body();
    cudaEvent_t e0, e1;
    JX_CUDA(cudaEventCreate(&e0));
    JX_CUDA(cudaEventCreate(&e1));
    double best = 1e30;
    for (int t = 0; t < trials; ++t) {
        JX_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < reps; ++k) body();
        JX_CUDA(cudaEventRecord(e1, s));
        JX_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        JX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, 1e3 * ms / reps);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// Device time (us) of one y = A x pass over M.
template <typename TX>
double time_pass(const LevelMat &M, const TX *x, TX *y, cudaStream_t s) {
    fk::OpSpmv<TX> op{x, y, 0};
    return time_best([&] { launch_rows<TX>(M, op, 0, M.nstored, s); }, s);
}

std::string layout_name(const LevelMat &M) {
    return M.sell == 2 ? std::string("sell/2") : M.sell ? std::string("sell") : ("csr/" + std::to_string(M.lanes));
}

// Layout choices of earlier setups, keyed by operator role, shape and storage:
// a repeated setup of the same system skips the timing runs.
struct TuneChoice {
    int sell = 0, lanes = 1;
    double us = 0.0;
};
// With JXCPR_TUNE_CACHE=<file> the choices also persist across processes: the
// file is read at the first lookup and rewritten after every new timing, so a
// later run (a profiler run, whose own timings would be distorted) uses the
// layouts an undisturbed run chose.  Lines: key sell lanes us.
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> &tune_cache() {  // the caller holds g_tune_mu
    static std::map<std::string, TuneChoice> *c = nullptr;
    if (!c) {
        c = new std::map<std::string, TuneChoice>();
        if (const char *path = getenv("JXCPR_TUNE_CACHE")) {
            if (FILE *f = fopen(path, "r")) {
                char key[200];
                TuneChoice t;
                while (fscanf(f, "%199s %d %d %lf", key, &t.sell, &t.lanes, &t.us) == 4) (*c)[key] = t;
                fclose(f);
            }
        }
    }
    return *c;
}
// The caller holds g_tune_mu.
void tune_store(const std::string &key, const TuneChoice &t) {
    tune_cache()[key] = t;
    if (const char *path = getenv("JXCPR_TUNE_CACHE")) {
        if (FILE *f = fopen(path, "w")) {
            for (auto &kv : tune_cache())
                fprintf(f, "%s %d %d %.6f\n", kv.first.c_str(), kv.second.sell, kv.second.lanes, kv.second.us);
            fclose(f);
        }
    }
}
// mode 1: the exact shape; mode 2 (shared): the shape class -- rows within a
// half octave, mean row length within 0.5 -- so similar operators of other
// systems (a batch) reuse one timing.
std::string tune_key(const char *name, int n, long long nnz, int kind, int E, int mode) {
    char k[160];
    if (mode == 2 && n > 0)
        snprintf(k, sizeof k, "%s/class/%d/%lld/%d/%d", name, (int)floor(2.0 * log2((double)n)),
                 (long long)llround(2.0 * (double)nnz / n), kind, E);
    else
        snprintf(k, sizeof k, "%s/%d/%lld/%d/%d", name, n, nnz, kind, E);
    return k;
}

// Builds a scalar operator in the layout that runs fastest here: CSR with
// 1..32 lanes per row (the candidates around the mean row length), or sliced
// ELL (operators with >= 2048 rows).
template <typename TX>
void build_tuned(const char *name, int n, int m, long long nnz, const int *ia, const int *ja, const double *a,
                 int kind, const std::vector<int> &order, const std::vector<int> &seg, const int *order_dev,
                 const FastOptions &opt, LevelMat &M, std::vector<std::string> &log, cudaStream_t s) {
    if (!opt.autotune || n == 0) {
        build_level_mat(n, m, nnz, 1, ia, ja, a, kind, use_sell(opt, n, nnz) ? (opt.sell_lanes == 2 ? 2 : 1) : 0,
                        order, seg, order_dev, M, s);
        if (n) {
            char line[200];
            snprintf(line, sizeof line, "%s rows %d mean %.1f layout %s (heuristic)", name, n, (double)nnz / n,
                     layout_name(M).c_str());
            log.emplace_back(line);
        }
        return;
    }
    const std::string key = tune_key(name, n, nnz, kind, 1, opt.autotune);
    TuneChoice best;
    bool cached = false;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            best = it->second;
            cached = true;
        }
    }
    if (cached) {
        build_level_mat(n, m, nnz, 1, ia, ja, a, kind, best.sell, order, seg, order_dev, M, s);
        if (!best.sell) M.lanes = best.lanes;
    } else {
        build_level_mat(n, m, nnz, 1, ia, ja, a, kind, false, order, seg, order_dev, M, s);
        DevBuf<TX> x(m > 0 ? m : 1), y(n > 0 ? n : 1);
        x.zero(s);
        y.zero(s);
        best.us = 1e30;
        const int v0 = lanes_for(n ? (double)nnz / n : 1.0);
        for (int V = 1; V <= 32; V *= 2) {
            if (V * 4 < v0 || V > v0 * 4) continue;  // candidates within a factor 4 of the mean-based choice
            M.lanes = V;
            const double t = time_pass<TX>(M, x.get(), y.get(), s);
            if (t < best.us) {
                best.us = t;
                best.lanes = V;
            }
        }
        M.lanes = best.lanes;
        if (n >= 2048) {
            // sliced ELL with one lane per row, and (FP32 / FP64 values) with two
            for (int P = 1; P <= (kind == VAL_BF16 ? 1 : 2); ++P) {
                LevelMat S;
                build_level_mat(n, m, nnz, 1, ia, ja, a, kind, P, order, seg, order_dev, S, s);
                const double t = time_pass<TX>(S, x.get(), y.get(), s);
                if (t < best.us) {
                    best.us = t;
                    best.sell = P;
                    M = std::move(S);
                }
            }
        }
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_store(key, best);
    }
    char line[200];
    snprintf(line, sizeof line, "%s rows %d mean %.1f layout %s %.2f us%s", name, n, n ? (double)nnz / n : 0.0,
             layout_name(M).c_str(), best.us, cached ? " (cached)" : "");
    log.emplace_back(line);
}

std::vector<int> download_ints(const int *d, int n, cudaStream_t s) {
    std::vector<int> h(n > 0 ? n : 0);
    if (n) {
        JX_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        JX_CUDA(cudaStreamSynchronize(s));
    }
    return h;
}

// Stored values back to the source CSR's entry order (inspection).  The stored order of a row can
// differ from the source's (FP32 operators keep the entries after the first in column order), so each
// stored entry goes to the source entry of the same column -- the r-th such stored entry to the r-th
// such source entry, should a row repeat a column.
__device__ __forceinline__ int source_slot(const int *__restrict__ src_ja, int d, int len, int cj, int r) {
    for (int q = 0; q < len; ++q)
        if (src_ja[d + q] == cj && r-- == 0) return q;
    return -1;
}

// sliced ELL with P lanes per row: stored row t = row rows[t]; its entry at stored position q sits in
// virtual row v = P t + q % P, slot q / P: at sp[v / 32] + 32 (q / P) + v % 32
__device__ __forceinline__ long long sell_slot(const long long *__restrict__ sp, int P, int t, int q) {
    const long long v = (long long)t * P + q % P;
    return sp[v >> 5] + (v & 31) + 32LL * (q / P);
}
template <typename TV>
__global__ void unpack_sell_kernel(int nstored, int P, const int *__restrict__ rows, const long long *__restrict__ sp,
                                   const int *__restrict__ col, const int *__restrict__ src_ia,
                                   const int *__restrict__ src_ja, const TV *__restrict__ val,
                                   const float *__restrict__ bsc, double *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nstored) return;
    const int i = rows[t];
    if (i < 0) return;
    const int d = src_ia[i], len = src_ia[i + 1] - d;
    for (int k = 0; k < len; ++k) {
        const long long pk = sell_slot(sp, P, t, k);
        const int cj = col[pk];
        int r = 0;
        for (int q = 0; q < k; ++q) r += col[sell_slot(sp, P, t, q)] == cj;
        const int pos = source_slot(src_ja, d, len, cj, r);
        if (pos >= 0) out[d + pos] = (double)fk::ldvs(val, bsc, pk);
    }
}

// CSR copy: stored row t = row perm[t] (identity without perm)
template <typename TV>
__global__ void unpack_csr_kernel(int n, const int *__restrict__ perm, const int *__restrict__ ia,
                                  const int *__restrict__ col, const int *__restrict__ src_ia,
                                  const int *__restrict__ src_ja, const TV *__restrict__ val,
                                  const float *__restrict__ bsc, double *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = perm ? perm[t] : t;
    const int d = src_ia[i], len = src_ia[i + 1] - d;
    for (int k = ia[t]; k < ia[t + 1]; ++k) {
        const int cj = col[k];
        int r = 0;
        for (int q = ia[t]; q < k; ++q) r += col[q] == cj;
        const int pos = source_slot(src_ja, d, len, cj, r);
        if (pos >= 0) out[d + pos] = (double)fk::ldvs(val, bsc, k);
    }
}

template <typename TX>
__global__ void add_kernel(int n, TX *__restrict__ u, const TX *__restrict__ c) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) u[i] += c[i];
}

// deterministic pseudo-random probe in [-1, 1) (splitmix-style integer hash)
__global__ void probe_kernel(int n, double *__restrict__ e) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long z = (unsigned long long)i * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    e[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
}  // namespace

void chebyshev3_coefficients(double lo, double hi, double c[3]) {
    // q(t) = T3(sigma - tau t) / T3(sigma), T3(s) = 4 s^3 - 3 s, sigma = (hi+lo)/(hi-lo), tau = 2/(hi-lo);
    // p(t) = (1 - q(t)) / t = -(q1 + q2 t + q3 t^2).
    if (!(hi > lo) || lo <= 0.0) {
        c[0] = hi > 0.0 ? 1.0 / hi : 0.0;  // degenerate interval: damped Jacobi
        c[1] = c[2] = 0.0;
        return;
    }
    const double sg = (hi + lo) / (hi - lo), tau = 2.0 / (hi - lo);
    const double n0 = 4.0 * sg * sg * sg - 3.0 * sg;
    const double n1 = -12.0 * sg * sg * tau + 3.0 * tau;
    const double n2 = 12.0 * sg * tau * tau;
    const double n3 = -4.0 * tau * tau * tau;
    c[0] = -n1 / n0;
    c[1] = -n2 / n0;
    c[2] = -n3 / n0;
}

// One power step's scalars on the device: lam = sqrt(<y,y> / <x,x>) and the scale 1 / ||y|| of the
// next iterate (the correctly rounded FP64 operations the host would do), or the stop flag once a
// norm is not positive (lam keeps its last value).  st = {lam, scale, stop}.
__global__ void power_scalars_kernel(const double *__restrict__ nrm, double *st) {
    if (st[2] != 0.0) return;
    const double yy = nrm[0], xx = nrm[1];
    if (!(yy > 0.0) || !(xx > 0.0)) {
        st[2] = 1.0;
        return;
    }
    st[0] = sqrt(yy / xx);
    st[1] = 1.0 / sqrt(yy);
}
__global__ void power_scale_kernel(int n, const double *__restrict__ st, double *__restrict__ y) {
    if (st[2] != 0.0) return;
    const double a = st[1];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a * y[i];
}

// lambda_max(D^-1 A) by `iters` power steps from x = 1, with the host reading the result once.
// iters2 > iters: the power steps go on to iters2 and *lam2 receives that estimate too (the same
// sequence of iterates, so each value equals a separate run of that many steps).
double estimate_lambda_max(const CsrView<double> &A, int iters, cudaStream_t s, int iters2, double *lam2) {
    const int n = A.nrows;
    if (n == 0) {
        if (lam2) *lam2 = 1.0;
        return 1.0;
    }
    DevBuf<double> dinv(n), x(n), y(n), partials(reduce_partials() + 8), nrm(2), st(3);
    fk::dinv_diag<double><<<div_up(n, kThreads), kThreads, 0, s>>>(n, A.ia, A.ja, A.a, dinv.get());
    JX_LAUNCH_CHECK();
    fill_dev(n, 1.0, x.get(), s);
    const double init[3] = {1.0, 1.0, 0.0};
    JX_CUDA(cudaMemcpyAsync(st.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
    DevBuf<double> at_iters(1);
    const int total = (lam2 && iters2 > iters) ? iters2 : iters;
    for (int it = 0; it < total; ++it) {
        if (it == iters)
            JX_CUDA(cudaMemcpyAsync(at_iters.get(), st.get(), sizeof(double), cudaMemcpyDeviceToDevice, s));
        fk::dinv_a_x<<<div_up(n, kThreads), kThreads, 0, s>>>(n, A.ia, A.ja, A.a, dinv.get(), x.get(), y.get());
        JX_LAUNCH_CHECK();
        dot_dev(n, y.get(), y.get(), partials.get(), nrm.get(), s);
        dot_dev(n, x.get(), x.get(), partials.get(), nrm.get() + 1, s);
        power_scalars_kernel<<<1, 1, 0, s>>>(nrm.get(), st.get());
        JX_LAUNCH_CHECK();
        power_scale_kernel<<<div_up(n, kThreads), kThreads, 0, s>>>(n, st.get(), y.get());
        JX_LAUNCH_CHECK();
        std::swap(x.p, y.p);
    }
    double h[3], first = 0.0;
    JX_CUDA(cudaMemcpyAsync(h, st.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    if (total > iters) JX_CUDA(cudaMemcpyAsync(&first, at_iters.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    JX_CUDA(cudaStreamSynchronize(s));
    if (total > iters) {
        *lam2 = h[0];
        return first;
    }
    if (lam2) *lam2 = h[0];
    return h[0];
}

template <typename TX>
struct FastCpr final : FastCprBase {
    using TA = TX;
    CprConfig cfg;
    FastOptions opt;
    int nb = 0, bs = 0;
    std::vector<std::unique_ptr<FastLevel<TX>>> lv;
    const double *Ainv = nullptr;
    int nc = 0;
    LevelMat st2;  // decoupled block matrix, level-0 colour classes as segments
    DevBuf<double> vt;
    DevBuf<int> st2_cls;  // stage 2: colour class of each block row (the sweeps' order)
    DevBuf<float> r32, z32, vt32;  // mixed path: stage-2 vectors in FP32
    CsrView<double> A0;  // FP64 level-0 operator (convergence-factor probe)
    DevBuf<double> pe, pr, pc, partials, nrm;
    // levels tail_first.. (the coarsest included) run as one cooperative kernel (fast_tail.cuh);
    // -1: every level launches its own passes
    int tail_first = -1, tail_kind = VAL_F64, tail_grid = 0;
    DevBuf<char> tail_desc;
    DevBuf<GridBarrier> tail_bar;
    int *amg_err = nullptr;  // the hierarchy's device error flag (a fused-kernel barrier time-out)

    int num_levels() const override { return (int)lv.size(); }
    void level_info(int l, int *smoother, int *kind, double *cheb) const override {
        const FastLevel<TX> &L = *lv[l];
        const bool coarsest = l + 1 == (int)lv.size();
        if (smoother) *smoother = coarsest ? 0 : L.smoother;
        if (kind) *kind = coarsest ? VAL_F64 : L.A.kind;
        if (cheb) {
            cheb[0] = L.cheb[0];
            cheb[1] = L.cheb[1];
            cheb[2] = L.cheb[2];
            cheb[3] = L.cheb_lo;
            cheb[4] = L.cheb_hi;
            cheb[5] = L.lambda_max;
        }
    }

    // ---- level operations ----------------------------------------------------
    void smooth(FastLevel<TX> &L, const TX *f, TX *u, bool zero, cudaStream_t s) {
        if (L.n == 0) return;
        const LevelMat &M = L.A;
        if (L.smoother == FS_COLOR_GS) {
            const int ncol = (int)M.seg.size() - 1;
            L.last_color = -1;
            for (int rep = 0; rep < 4; ++rep) {  // two symmetric GS applications: fwd, bwd, fwd, bwd
                const bool backward = rep & 1;
                for (int g = 0; g < ncol; ++g) {
                    const int c = backward ? ncol - 1 - g : g;
                    if (c == L.last_color) continue;  // recomputing the last class changes nothing
                    L.last_color = c;
                    fk::OpGs<TX> op{f, L.dinv.get(), u, zero ? 1 : 0};
                    launch_rows<TX>(M, op, M.seg[c], M.seg[c + 1], s);
                    zero = false;
                }
            }
        } else if (L.smoother == FS_L1_JACOBI) {
            for (int rep = 0; rep < 2; ++rep) {  // 2 x (u -> tmp -> u)
                fk::OpJacobi<TX> a{f, L.dinv_l1.get(), u, L.z.get(), zero ? 1 : 0};
                launch_rows<TX>(M, a, 0, M.nstored, s);
                fk::OpJacobi<TX> b{f, L.dinv_l1.get(), L.z.get(), u, 0};
                launch_rows<TX>(M, b, 0, M.nstored, s);
                zero = false;
            }
        } else {
            fk::OpCheb<TX> c0{0, zero ? 1 : 0, (TX)L.cheb[2], f, L.dinv.get(), nullptr, u, L.z.get(), L.y1.get()};
            launch_rows<TX>(M, c0, 0, M.nstored, s);
            fk::OpCheb<TX> c1{1, 0, (TX)L.cheb[1], f, L.dinv.get(), L.y1.get(), u, L.z.get(), L.y2.get()};
            launch_rows<TX>(M, c1, 0, M.nstored, s);
            fk::OpCheb<TX> c2{2, zero ? 1 : 0, (TX)L.cheb[0], f, L.dinv.get(), L.y2.get(), u, L.z.get(), nullptr};
            launch_rows<TX>(M, c2, 0, M.nstored, s);
        }
    }
    void residual(FastLevel<TX> &L, const TX *f, const TX *u, TX *r, cudaStream_t s) {
        fk::OpResid<TX> op{f, u, r};
        launch_rows<TX>(L.A, op, 0, L.A.nstored, s);
    }
    void spmv(const LevelMat &M, const TX *x, bool beta_one, TX *y, cudaStream_t s) {
        fk::OpSpmv<TX> op{x, y, beta_one ? 1 : 0};
        launch_rows<TX>(M, op, 0, M.nstored, s);
    }
    void coarse(const TX *f, TX *u, cudaStream_t s) {
        if (nc == 0) return;
        launch_dep(fk::dense_gemv<TX>, dim3(div_up((long long)nc * 32, kThreads)), dim3(kThreads), s, nc, Ainv, f,
                   u);
        JX_LAUNCH_CHECK();
    }

    // ---- the fused coarse levels (fast_tail.cuh) ---------------------------------------
    template <typename TV>
    static tail::Mat<TV> tail_mat(const LevelMat &M, const TV *a) {
        tail::Mat<TV> m{};
        m.sell = M.sell;
        m.lanes = M.lanes;
        m.nstored = M.nstored;
        m.ia = M.ia.get();
        m.ja = M.ja.get();
        m.perm = M.perm;
        m.sp = M.sp.get();
        m.rows = M.rows.get();
        m.a = a;
        m.bscale = M.bscale.get();
        return m;
    }
    template <typename TV>
    void upload_tail(cudaStream_t s) {
        std::unique_ptr<tail::Desc<TX, TV>> d(new tail::Desc<TX, TV>());
        const int L = (int)lv.size();
        d->nlev = L - tail_first;
        d->nc = nc;
        d->Ainv = Ainv;
        for (int l = tail_first; l < L; ++l) {
            const FastLevel<TX> &Lv = *lv[l];
            tail::Level<TX, TV> &T = d->lv[l - tail_first];
            T.n = Lv.n;
            T.smoother = Lv.smoother;
            T.f = Lv.f.get();
            T.u = Lv.u.get();
            if (l == L - 1) continue;  // the coarsest: f, u and the inverse only
            const TV *av;
            if constexpr (std::is_same<TV, double>::value) av = Lv.A.a64.get();
            else if constexpr (std::is_same<TV, float>::value) av = Lv.A.a32.get();
            else av = Lv.A.a16.get();
            T.A = tail_mat<TV>(Lv.A, av);
            // transfer operators are stored as TX (FP64 path: FP64, mixed path: FP32)
            if constexpr (std::is_same<TX, double>::value) {
                T.P = tail_mat<TX>(Lv.P, Lv.P.a64.get());
                T.R = tail_mat<TX>(Lv.R, Lv.R.a64.get());
            } else {
                T.P = tail_mat<TX>(Lv.P, Lv.P.a32.get());
                T.R = tail_mat<TX>(Lv.R, Lv.R.a32.get());
            }
            T.nseg = std::min((int)Lv.A.seg.size(), tail::kMaxSegs);
            for (int c = 0; c < T.nseg; ++c) T.seg[c] = Lv.A.seg[c];
            T.npass = 0;
            if (Lv.smoother == FS_COLOR_GS) {  // FastCpr::smooth's sequence of colour passes
                const int ncol = (int)Lv.A.seg.size() - 1;
                int last = -1;
                for (int rep = 0; rep < 4; ++rep)
                    for (int g = 0; g < ncol; ++g) {
                        const int c = (rep & 1) ? ncol - 1 - g : g;
                        if (c == last) continue;
                        last = c;
                        T.pass[T.npass++] = (unsigned char)c;
                    }
            }
            T.c0 = (TX)Lv.cheb[0];
            T.c1 = (TX)Lv.cheb[1];
            T.c2 = (TX)Lv.cheb[2];
            T.dinv = Lv.dinv.get();
            T.dinv_l1 = Lv.dinv_l1.get();
            T.r = Lv.r.get();
            T.z = Lv.z.get();
            T.y1 = Lv.y1.get();
            T.y2 = Lv.y2.get();
        }
        tail_desc.alloc(sizeof(tail::Desc<TX, TV>));
        JX_CUDA(cudaMemcpyAsync(tail_desc.get(), d.get(), sizeof(tail::Desc<TX, TV>), cudaMemcpyHostToDevice, s));
        JX_CUDA(cudaStreamSynchronize(s));
    }
    // (Re)writes the fused kernel's description after the smoothers are chosen or switched.
    void refresh_tail(cudaStream_t s) {
        if (tail_first <= 0) return;
        if (tail_kind == VAL_F64) {
            if constexpr (std::is_same<TX, double>::value) upload_tail<double>(s);
        } else if (tail_kind == VAL_BF16) {
            if constexpr (std::is_same<TX, float>::value) upload_tail<__nv_bfloat16>(s);
        } else {
            if constexpr (std::is_same<TX, float>::value) upload_tail<float>(s);
        }
    }
    // Chooses the fused levels: every level from the first with at most `rows` rows (the coarsest
    // included), all stored in one precision, at least one of them smoothed; sizes the grid.
    void setup_tail(int rows, int ctas, cudaStream_t s) {
        tail_first = -1;
        const int L = (int)lv.size();
        if (rows <= 0 || L < 3) return;
        int first = -1;
        for (int l = 1; l < L; ++l)
            if (lv[l]->n <= rows) {
                first = l;
                break;
            }
        if (first < 0 || first > L - 2) return;
        for (int l = first; l < L - 1; ++l) {
            const LevelMat &A = lv[l]->A;
            if ((int)A.seg.size() - 1 > tail::kMaxSegs - 1 || lv[l]->n == 0) return;
        }
        if (L - first > tail::kMaxLevels) first = L - tail::kMaxLevels;
        // one storage type over the fused levels (precision 2 changes it at bf16_level)
        while (first < L - 1 && lv[first]->A.kind != lv[L - 2]->A.kind) ++first;
        if (first > L - 2) return;
        tail_first = first;
        tail_kind = lv[L - 2]->A.kind;
        void *fn = nullptr;
        if constexpr (std::is_same<TX, double>::value)
            fn = (void *)tail::tail_vcycle_kernel<double, double>;
        else
            fn = tail_kind == VAL_BF16 ? (void *)tail::tail_vcycle_kernel<float, __nv_bfloat16>
                                       : (void *)tail::tail_vcycle_kernel<float, float>;
        int per_sm = 0;
        JX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0));
        long long want = 1;
        for (int l = first; l < L - 1; ++l) {
            const LevelMat &A = lv[l]->A;
            want = std::max(want, (long long)A.nstored * (A.sell ? A.sell : A.lanes));
        }
        want = std::max(want, (long long)nc * 32);
        int grid = std::max(1, std::min(std::max(per_sm, 1) * sm_count(), div_up(want, kThreads)));
        if (ctas > 0) grid = std::min(grid, ctas);
        tail_grid = grid;
        tail_bar.alloc(1);
        refresh_tail(s);
    }
    void launch_tail(cudaStream_t s) {
        JX_CUDA(cudaMemsetAsync(tail_bar.get(), 0, sizeof(GridBarrier), s));
        cudaLaunchConfig_t lc{};
        lc.gridDim = dim3(tail_grid);
        lc.blockDim = dim3(kThreads);
        lc.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        GridBarrier *bar = tail_bar.get();
        int *err = amg_err;
        if constexpr (std::is_same<TX, double>::value) {
            const auto *d = reinterpret_cast<const tail::Desc<double, double> *>(tail_desc.get());
            JX_CUDA(cudaLaunchKernelEx(&lc, tail::tail_vcycle_kernel<double, double>, d, bar, err));
        } else if (tail_kind == VAL_BF16) {
            const auto *d = reinterpret_cast<const tail::Desc<float, __nv_bfloat16> *>(tail_desc.get());
            JX_CUDA(cudaLaunchKernelEx(&lc, tail::tail_vcycle_kernel<float, __nv_bfloat16>, d, bar, err));
        } else {
            const auto *d = reinterpret_cast<const tail::Desc<float, float> *>(tail_desc.get());
            JX_CUDA(cudaLaunchKernelEx(&lc, tail::tail_vcycle_kernel<float, float>, d, bar, err));
        }
        JX_LAUNCH_CHECK();
    }

    // u0 = V-cycle(f0) from a zero initial guess
    void vcycle_tx(const TX *f0, TX *u0, cudaStream_t s) {
        const int L = (int)lv.size();
        auto F = [&](int l) -> const TX * { return l == 0 ? f0 : lv[l]->f.get(); };
        auto U = [&](int l) -> TX * { return l == 0 ? u0 : lv[l]->u.get(); };
        if (L == 1) {
            coarse(f0, u0, s);
            return;
        }
        const int top = tail_first > 0 ? tail_first : L - 1;  // levels above the fused ones
        for (int l = 0; l < top; ++l) {
            FastLevel<TX> &Lv = *lv[l];
            if (Lv.smoother == FS_COLOR_GS && Lv.n) JX_CUDA(cudaMemsetAsync(U(l), 0, sizeof(TX) * Lv.n, s));
            smooth(Lv, F(l), U(l), true, s);
            residual(Lv, F(l), U(l), Lv.r.get(), s);
            spmv(Lv.R, Lv.r.get(), false, lv[l + 1]->f.get(), s);
        }
        if (tail_first > 0)
            launch_tail(s);
        else
            coarse(F(L - 1), U(L - 1), s);
        for (int l = top - 1; l >= 0; --l) {
            FastLevel<TX> &Lv = *lv[l];
            spmv(Lv.P, U(l + 1), true, U(l), s);
            smooth(Lv, F(l), U(l), false, s);
        }
    }

    template <typename TV, typename TXV, typename TAC>
    void launch_hgs_csr(int V, const LevelMat &M, const TV *a, int r0, int r1, const TXV *r, TXV *z, TXV *vtp,
                        TAC w, TAC om, int plain, fk::SweepOrder so, cudaStream_t s) {
        const int grid = div_up((long long)(r1 - r0) * V, 128);
#define JX_HGS_CSR(VV)                                                                                        \
    do {                                                                                                      \
        if (bs == 2)                                                                                          \
            launch_dep(fk::hgs_color<2, VV, TV, TAC, TXV>, dim3(grid), dim3(128), s, r0, r1, M.perm, M.ia.get(), \
                       M.ja.get(), a, r, z, vtp, w, om, plain, so);                                          \
        else                                                                                                  \
            launch_dep(fk::hgs_color<3, VV, TV, TAC, TXV>, dim3(grid), dim3(128), s, r0, r1, M.perm, M.ia.get(), \
                       M.ja.get(), a, r, z, vtp, w, om, plain, so);                                          \
    } while (0)
        switch (V) {
            case 1: JX_HGS_CSR(1); break;
            case 2: JX_HGS_CSR(2); break;
            case 4: JX_HGS_CSR(4); break;
            case 8: JX_HGS_CSR(8); break;
            case 16: JX_HGS_CSR(16); break;
            default: JX_HGS_CSR(32); break;
        }
#undef JX_HGS_CSR
    }

    // One stage-2 sweep on vectors of type TXV (FP64 path: the caller's r, z;
    // mixed path: FP32 copies); vtp receives each colour class's start values as
    // the class is updated (no start-of-sweep copy, see fk::hgs_color).
    template <typename TXV>
    void sweep_typed(const TXV *r, TXV *z, TXV *vtp, cudaStream_t s) {
        const LevelMat &M = st2;
        if (M.n == 0) return;
        const double eps = 2.220446049250313e-16;
        const int plain = (fabs(cfg.stage2_w - 1) < eps && fabs(cfg.stage2_omega - 1) < eps) ? 1 : 0;
        const TA w = (TA)cfg.stage2_w, om = (TA)cfg.stage2_omega;
        int first = -1, last = -1;
        for (size_t c = 0; c + 1 < M.seg.size(); ++c)
            if (M.seg[c + 1] > M.seg[c]) {
                if (first < 0) first = (int)c;
                last = (int)c;
            }
        for (size_t c = 0; c + 1 < M.seg.size(); ++c) {
            const int r0 = M.seg[c], r1 = M.seg[c + 1];
            if (r1 <= r0) continue;
            fk::SweepOrder so;
            so.nmode = (int)c == first ? 0 : ((int)c == last ? 1 : 2);
            so.save = (int)c != last ? 1 : 0;
            so.cur = (int)c;
            so.cls = st2_cls.get();
            if (M.kind == VAL_F64)  // FP64 path, and the hybrid form's FP64 stage 2: FP64 values and arithmetic
                launch_stage2<double, TXV, double>(M, M.a64.get(), r0, r1, r, z, vtp, cfg.stage2_w, cfg.stage2_omega,
                                                   plain, so, s);
            else
                launch_stage2<float, TXV, TA>(M, M.a32.get(), r0, r1, r, z, vtp, w, om, plain, so, s);
            JX_LAUNCH_CHECK();
        }
    }
    // FP64 interface (C ABI / tests): the mixed path converts in and out.
    void stage2_sweep(const double *r, double *z, cudaStream_t s) override {
        DepLaunchScope dep(opt.dep_launch);
        if (std::is_same<TX, double>::value || st2.kind == VAL_F64) {
            sweep_typed<double>(r, z, vt.get(), s);
        } else {
            const long long n = (long long)nb * bs;
            if (!n) return;
            launch_dep(fk::convert<double, float>, dim3(div_up(n, kThreads)), dim3(kThreads), s, n, r, r32.get());
            JX_LAUNCH_CHECK();
            launch_dep(fk::convert<double, float>, dim3(div_up(n, kThreads)), dim3(kThreads), s, n, z, z32.get());
            JX_LAUNCH_CHECK();
            sweep_typed<float>(r32.get(), z32.get(), vt32.get(), s);
            launch_dep(fk::convert<float, double>, dim3(div_up(n, kThreads)), dim3(kThreads), s, n, z32.get(), z);
            JX_LAUNCH_CHECK();
        }
    }
    template <typename TV, typename TXV, typename TAC>
    void launch_stage2(const LevelMat &M, const TV *a, int r0, int r1, const TXV *r, TXV *z, TXV *vtp, TAC w,
                       TAC om, int plain, fk::SweepOrder so, cudaStream_t s) {
        if (M.chunk) {
            // the 2x2 sweep gathers x and the start values as pairs (one 8-byte load in FP32)
            if (bs == 2 && ((reinterpret_cast<uintptr_t>(z) | reinterpret_cast<uintptr_t>(vtp)) % 8) != 0) {
                set_error("stage 2: the iterate and start-value vectors must be 8-byte aligned");
                throw CudaError{cudaErrorInvalidValue, "stage 2 alignment"};
            }
            const int grid = div_up(r1 - r0, kThreads);
#define JX_HGS_CHUNK(BSV, CHV)                                                                              \
    launch_dep(fk::hgs_chunk<BSV, CHV, TV, TAC, TXV>, dim3(grid), dim3(kThreads), s, r0, r1, M.sp.get(),     \
               reinterpret_cast<const unsigned *>(M.ja.get()), a, M.rows.get(), r, z, vtp, w, om, plain, so.save)
            if (bs == 2) {
                if (M.chunk == 4) JX_HGS_CHUNK(2, 4);
                else if (M.chunk == 16) JX_HGS_CHUNK(2, 16);
                else JX_HGS_CHUNK(2, 8);
            } else {
                if (M.chunk == 4) JX_HGS_CHUNK(3, 4);
                else if (M.chunk == 16) JX_HGS_CHUNK(3, 16);
                else JX_HGS_CHUNK(3, 8);
            }
#undef JX_HGS_CHUNK
            return;
        }
        if (M.sell) {
            const int grid = div_up(r1 - r0, kThreads);
            if (bs == 2)
                launch_dep(fk::hgs_sell<2, TV, TAC, TXV>, dim3(grid), dim3(kThreads), s,
                           r0, r1, M.sp.get(), M.ja.get(), a,
                                                                       M.rows.get(), r, z, vtp, w, om, plain, so);
            else
                launch_dep(fk::hgs_sell<3, TV, TAC, TXV>, dim3(grid), dim3(kThreads), s,
                           r0, r1, M.sp.get(), M.ja.get(), a,
                                                                       M.rows.get(), r, z, vtp, w, om, plain, so);
        } else {
            launch_hgs_csr<TV, TXV, TAC>(opt.stage2_lanes, M, a, r0, r1, r, z, vtp, w, om, plain, so, s);
        }
    }

    // CUDA graph of apply_direct(in_buf -> out_buf), captured on a private
    // stream at the first application and replayed on the caller's stream.
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    unsigned long long graph_kernels = 0;
    DevBuf<double> in_buf, out_buf;

    ~FastCpr() override {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap_stream) cudaStreamDestroy(cap_stream);
    }

    void capture() {
        const size_t n = (size_t)nb * bs;
        in_buf.alloc(n > 0 ? n : 1);
        out_buf.alloc(n > 0 ? n : 1);
        if (!cap_stream) JX_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
        const unsigned long long k0 = launch_count();
        JX_CUDA(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal));
        try {
            apply_direct(in_buf.get(), out_buf.get(), cap_stream);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(cap_stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        JX_CUDA(cudaStreamEndCapture(cap_stream, &graph));
        graph_kernels = launch_count() - k0;
        uncount_launches(graph_kernels);
        JX_CUDA(cudaGraphInstantiate(&graph_exec, graph, 0));
    }

    void apply(const double *r, double *z, cudaStream_t s) override {
        if (!opt.graphs) {
            apply_direct(r, z, s);
            return;
        }
        if (!graph_exec) capture();
        const size_t bytes = sizeof(double) * (size_t)nb * bs;
        JX_CUDA(cudaMemcpyAsync(in_buf.get(), r, bytes, cudaMemcpyDeviceToDevice, s));
        JX_CUDA(cudaGraphLaunch(graph_exec, s));
        count_launches(graph_kernels);
        JX_CUDA(cudaMemcpyAsync(z, out_buf.get(), bytes, cudaMemcpyDeviceToDevice, s));
    }

    void apply_enqueue(const double *r, double *z, cudaStream_t s) override { apply_direct(r, z, s); }

    void apply_direct(const double *r, double *z, cudaStream_t s) {
        DepLaunchScope dep(opt.dep_launch);
        FastLevel<TX> &L0 = *lv[0];
        constexpr bool fp64 = std::is_same<TX, double>::value;
        const long long n = (long long)nb * bs;
        if (fp64) {
            launch_dep(fk::restrict_p<TX>, dim3(div_up(nb, kThreads)), dim3(kThreads), s,
                       nb, bs, cfg.pressure_index, r, L0.f.get());
        } else {
            launch_dep(fk::restrict_cvt<TX>, dim3(div_up(n, kThreads)), dim3(kThreads), s,
                       nb, bs, cfg.pressure_index, r, L0.f.get(),
                                                                        r32.get());
        }
        JX_LAUNCH_CHECK();
        vcycle_tx(L0.f.get(), L0.u.get(), s);
        for (int it = 1; it < cfg.stage1_maxit; ++it) {
            // further AMG iterations as residual corrections: u += V(f - A u)
            residual(L0, L0.f.get(), L0.u.get(), L0.r.get(), s);
            vcycle_tx(L0.r.get(), L0.c.get(), s);
            launch_dep(add_kernel<TX>, dim3(div_up(L0.n, kThreads)), dim3(kThreads), s, L0.n, L0.u.get(),
                       L0.c.get());
            JX_LAUNCH_CHECK();
        }
        const bool st2_on = cfg.stage2_solver_type == 2 && cfg.stage2_maxit > 0;
        if (fp64 || !st2_on || st2.kind == VAL_F64) {
            // FP64 stage 2 on the caller's vectors (FP64 path; hybrid form: FP32 stage 1, FP64 polish)
            launch_dep(fk::prolong_p<TX, double>, dim3(div_up(n, kThreads)), dim3(kThreads), s,
                       nb, bs, cfg.pressure_index,
                                                                              L0.u.get(), z);
            JX_LAUNCH_CHECK();
            if (st2_on)
                for (int it = 0; it < cfg.stage2_maxit; ++it) sweep_typed<double>(r, z, vt.get(), s);
            return;
        }
        // mixed path: stage 2 on FP32 copies of r and z, result converted to FP64
        launch_dep(fk::prolong_p<TX, float>, dim3(div_up(n, kThreads)), dim3(kThreads), s,
                   nb, bs, cfg.pressure_index, L0.u.get(),
                                                                         z32.get());
        JX_LAUNCH_CHECK();
        for (int it = 0; it < cfg.stage2_maxit; ++it) sweep_typed<float>(r32.get(), z32.get(), vt32.get(), s);
        launch_dep(fk::convert<float, double>, dim3(div_up(n, kThreads)), dim3(kThreads), s, n, z32.get(), z);
        JX_LAUNCH_CHECK();
    }

    void vcycle(const double *fp, double *up, cudaStream_t s) override {
        DepLaunchScope dep(opt.dep_launch);
        FastLevel<TX> &L0 = *lv[0];
        const int n = L0.n;
        launch_dep(fk::convert<double, TX>, dim3(div_up(n, kThreads)), dim3(kThreads), s, n, fp, L0.f.get());
        JX_LAUNCH_CHECK();
        vcycle_tx(L0.f.get(), L0.u.get(), s);
        launch_dep(fk::convert<TX, double>, dim3(div_up(n, kThreads)), dim3(kThreads), s, n, L0.u.get(), up);
        JX_LAUNCH_CHECK();
    }

    void set_plain_mode(bool plain) override {
        for (auto &lp : lv) lp->smoother = plain ? lp->smoother_plain : lp->smoother_cfg;
        refresh_tail(nullptr);
        if (graph_exec) {  // the captured sequence depends on the smoothers
            cudaGraphExecDestroy(graph_exec);
            graph_exec = nullptr;
        }
        if (graph) {
            cudaGraphDestroy(graph);
            graph = nullptr;
        }
    }

    DevBuf<TX> nat_r, nat_z;
    DevBuf<double> nat_r64, nat_z64;  // hybrid form: the FP64 stage 2 timed on FP64 vectors
    void stage2_native(int sweeps, cudaStream_t s) override {
        DepLaunchScope dep(opt.dep_launch);
        const long long n = (long long)nb * bs;
        if (!n) return;
        if (!nat_r.get()) {
            nat_r.alloc(n);
            nat_z.alloc(n);
            nat_r.zero(s);
            nat_z.zero(s);
        }
        for (int k = 0; k < sweeps; ++k) {
            if constexpr (std::is_same<TX, double>::value) {
                sweep_typed<double>(nat_r.get(), nat_z.get(), vt.get(), s);
            } else if (st2.kind == VAL_F64) {
                if (!nat_r64.get()) {
                    nat_r64.alloc(n);
                    nat_z64.alloc(n);
                    nat_r64.zero(s);
                    nat_z64.zero(s);
                }
                sweep_typed<double>(nat_r64.get(), nat_z64.get(), vt.get(), s);
            } else {
                sweep_typed<float>(nat_r.get(), nat_z.get(), vt32.get(), s);
            }
        }
    }

    bool level_native(int level, int op, int reps, cudaStream_t s) override {
        if (level < 0 || level + 1 >= (int)lv.size()) return false;
        FastLevel<TX> &L = *lv[level];
        if (L.n == 0) return false;
        DepLaunchScope dep(opt.dep_launch);
        if (!L.y1.get()) alloc_vec(L.y1, L.n);
        if (!L.y2.get()) alloc_vec(L.y2, L.n);
        for (int k = 0; k < reps; ++k) {
            if (op == 0) {
                spmv(L.A, L.u.get(), false, L.y1.get(), s);
            } else if (op == 1) {
                fk::OpCheb<TX> c1{1, 0, (TX)0.5, L.f.get(), L.dinv.get(), L.u.get(), L.u.get(), L.z.get(), L.y1.get()};
                launch_rows<TX>(L.A, c1, 0, L.A.nstored, s);
            } else {
                residual(L, L.f.get(), L.u.get(), L.r.get(), s);
            }
        }
        return true;
    }

    bool stored_values(int level, double *out, cudaStream_t s) override {
        if (level < 0 || level + 1 >= (int)lv.size()) return false;
        const FastLevel<TX> &L = *lv[level];
        const LevelMat &M = L.A;
        if (L.n == 0 || !L.src_ia || !L.src_ja) return false;
        with_values<TX>(M, [&](auto a) {
            if (M.sell)
                unpack_sell_kernel<<<div_up(M.nstored, kThreads), kThreads, 0, s>>>(
                    M.nstored, M.sell, M.rows.get(), M.sp.get(), M.ja.get(), L.src_ia, L.src_ja, a, M.bscale.get(), out);
            else
                unpack_csr_kernel<<<div_up(M.n, kThreads), kThreads, 0, s>>>(
                    M.n, M.perm, M.ia.get(), M.ja.get(), L.src_ia, L.src_ja, a, M.bscale.get(), out);
        });
        JX_LAUNCH_CHECK();
        return true;
    }

    double apply_bytes() const override {
        auto vb = [](int kind) { return kind == VAL_F64 ? 8.0 : (kind == VAL_F32 ? 4.0 : 2.0); };
        const double xb = sizeof(TX);
        double total = 0.0;
        for (size_t l = 0; l + 1 < lv.size(); ++l) {
            const FastLevel<TX> &L = *lv[l];
            // matrix passes per V-cycle incl. the residual: GS 2 x 1.5 + 2 x 2.5 sweeps -> 6, l1-Jacobi 7 + 1,
            // Chebyshev 2 + 3 + 1
            const double passes = L.smoother == FS_L1_JACOBI ? 8.0 : 6.0;
            total += passes * ((double)L.A.nnz * (vb(L.A.kind) + 4.0) + 3.0 * L.n * xb);
            total += (double)L.P.nnz * (vb(L.P.kind) + 4.0) + (double)L.R.nnz * (vb(L.R.kind) + 4.0) +
                     2.0 * (L.P.n + L.P.m) * xb;
        }
        total += (double)nc * nc * 8.0;
        const double bsz = bs * bs;
        const double xb2 = st2.kind == VAL_F64 ? 8.0 : xb;
        total += cfg.stage2_maxit * ((double)st2.nnz * (bsz * vb(st2.kind) + 4.0) + 4.0 * nb * bs * xb2);
        return total;
    }

    double vcycle_factor(int cycles, cudaStream_t s) override {
        const int n = A0.nrows;
        if (n == 0 || cycles <= 0) return 0.0;
        pe.alloc(n);
        pr.alloc(n);
        pc.alloc(n);
        partials.alloc(reduce_partials() + 8);
        nrm.alloc(2);
        probe_kernel<<<div_up(n, kThreads), kThreads, 0, s>>>(n, pe.get());
        JX_LAUNCH_CHECK();
        auto norm = [&](const double *v) {
            double h = 0.0;
            dot_dev(n, v, v, partials.get(), nrm.get(), s);
            JX_CUDA(cudaMemcpyAsync(&h, nrm.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
            JX_CUDA(cudaStreamSynchronize(s));
            return sqrt(h);
        };
        double prev = norm(pe.get()), rho = 0.0;
        for (int k = 0; k < cycles; ++k) {
            csr_spmv(A0, -1.0, pe.get(), 0.0, pr.get(), s);  // r = -A e (f = 0)
            vcycle(pr.get(), pc.get(), s);
            axpy_dev(n, 1.0, pc.get(), pe.get(), s);         // e <- e + B r
            const double cur = norm(pe.get());
            rho = prev > 0.0 ? cur / prev : 0.0;
            if (!(cur > 0.0) || !(cur == cur)) break;
            prev = cur;
        }
        return rho;
    }
};

template <typename TX>
static FastCprBase *build_fast(Amg &H, const BsrView<double> &A, const CprConfig &cfg, const FastOptions &opt,
                               cudaStream_t s) {
    std::unique_ptr<FastCpr<TX>> F(new FastCpr<TX>());
    F->cfg = cfg;
    F->opt = opt;
    F->nb = A.nb;
    F->bs = A.bs;
    F->A0 = H.levels[0]->A.view();
    const int L = H.num_levels();
    const bool fp64 = std::is_same<TX, double>::value;
    for (int l = 0; l < L; ++l) {
        AmgLevel &HL = *H.levels[l];
        std::unique_ptr<FastLevel<TX>> lev(new FastLevel<TX>());
        FastLevel<TX> &Lv = *lev;
        const int n = HL.A.nrows;
        Lv.n = n;
        alloc_vec(Lv.f, n);
        alloc_vec(Lv.u, n);
        if (l < L - 1) {
            const int kind = fp64 ? VAL_F64 : ((opt.precision == 2 && l >= opt.bf16_level) ? VAL_BF16 : VAL_F32);
            const int plain_sm = HL.smoother == SMOOTH_COLOR_GS ? FS_COLOR_GS : FS_L1_JACOBI;
            int sm = plain_sm;
            if (opt.smoother == 2 || (opt.smoother == 1 && sm == FS_L1_JACOBI)) sm = FS_CHEB;
            Lv.smoother = Lv.smoother_cfg = sm;
            Lv.smoother_plain = (opt.smoother == 2) ? FS_CHEB : plain_sm;
            const CsrView<double> Av = HL.A.view();
            Lv.src_ia = Av.ia;
            Lv.src_ja = Av.ja;
            const std::string nm = "A" + std::to_string(l);
            if (sm == FS_COLOR_GS) {
                std::vector<int> order = download_ints(HL.fwd.perm.get(), n, s);
                build_tuned<TX>(nm.c_str(), n, n, Av.nnz, Av.ia, Av.ja, Av.a, kind, order, HL.fwd.h_group_ptr,
                                HL.fwd.perm.get(), opt, Lv.A, F->tune_log, s);
            } else {
                build_tuned<TX>(nm.c_str(), n, n, Av.nnz, Av.ia, Av.ja, Av.a, kind, {}, {}, nullptr, opt, Lv.A,
                                F->tune_log, s);
            }
            H.log.mark("fast_operators", s);
            alloc_vec(Lv.dinv, n);
            if (n) {
                fk::dinv_diag<TX><<<div_up(n, kThreads), kThreads, 0, s>>>(n, Av.ia, Av.ja, Av.a, Lv.dinv.get());
                JX_LAUNCH_CHECK();
            }
            if (Lv.smoother_plain == FS_L1_JACOBI || sm == FS_L1_JACOBI) {
                alloc_vec(Lv.dinv_l1, n);
                if (n) {
                    fk::dinv_l1<TX><<<div_up(n, kThreads), kThreads, 0, s>>>(n, Av.ia, Av.a, Lv.dinv_l1.get());
                    JX_LAUNCH_CHECK();
                }
            }
            if (sm == FS_CHEB) {
                // the learned-features pass ran the same power steps on this operator already
                const bool known = (size_t)l < opt.level_lambda.size() && opt.level_lambda[l] > 0.0;
                Lv.lambda_max = known ? opt.level_lambda[l] : estimate_lambda_max(Av, 12, s);
                const double lo = (size_t)l < opt.level_lower.size() ? opt.level_lower[l] : opt.cheb_lower;
                const double hi = (size_t)l < opt.level_upper.size() ? opt.level_upper[l] : opt.cheb_upper;
                Lv.cheb_lo = lo * Lv.lambda_max;
                Lv.cheb_hi = hi * Lv.lambda_max;
                chebyshev3_coefficients(Lv.cheb_lo, Lv.cheb_hi, Lv.cheb);
                alloc_vec(Lv.y1, n);
                alloc_vec(Lv.y2, n);
                H.log.mark("fast_lambda_max", s);
            }
            alloc_vec(Lv.r, n);
            alloc_vec(Lv.z, n);
            if (l == 0) alloc_vec(Lv.c, n);
            const int pk = fp64 ? VAL_F64 : VAL_F32;  // transfer operators: FP32 in the mixed path
            const CsrView<double> Pv = HL.P.view(), Rv = HL.R.view();
            build_tuned<TX>(("P" + std::to_string(l)).c_str(), Pv.nrows, Pv.ncols, Pv.nnz, Pv.ia, Pv.ja, Pv.a, pk, {},
                            {}, nullptr, opt, Lv.P, F->tune_log, s);
            build_tuned<TX>(("R" + std::to_string(l)).c_str(), Rv.nrows, Rv.ncols, Rv.nnz, Rv.ia, Rv.ja, Rv.a, pk, {},
                            {}, nullptr, opt, Lv.R, F->tune_log, s);
            H.log.mark("fast_transfers", s);
        }
        F->lv.push_back(std::move(lev));
    }
    F->nc = H.nc;
    F->Ainv = H.Ainv.get();
    if (F->nc > 0 && !F->Ainv) {
        set_error("fast CPR path needs the explicit coarse inverse");
        throw CudaError{cudaErrorInvalidValue, "coarse inverse"};
    }
    // stage 2: block rows in the level-0 colour order
    AmgLevel &H0 = *H.levels[0];
    F->vt.alloc((size_t)(A.nb > 0 ? A.nb : 1) * A.bs);
    F->vt.zero(s);  // padding slots of the sliced-ELL copy read entry 0 (times a zero block): keep it finite
    if (!fp64) {
        const size_t nv = (size_t)(A.nb > 0 ? A.nb : 1) * A.bs;
        F->r32.alloc(nv);
        F->z32.alloc(nv);
        F->vt32.alloc(nv);
        F->vt32.zero(s);
    }
    if (opt.stage2_chunk > 0 && !H0.chunk_order.empty() && A.nb > 0) {
        // chunk order: no layout timing (one layout)
        const std::vector<int> &ord = H0.chunk_order;
        const std::vector<int> &sg = H0.chunk_seg;
        std::vector<int> cls(A.nb, 0);
        for (size_t c = 0; c + 1 < sg.size(); ++c)
            for (int t = sg[c]; t < sg[c + 1]; ++t)
                if (ord[t] >= 0) cls[ord[t]] = (int)c;
        F->st2_cls.alloc(A.nb);
        F->st2_cls.upload(cls.data(), A.nb, s);
        const int kind = (fp64 || opt.precision == 3) ? VAL_F64 : VAL_F32;
        build_chunk_mat(A.nb, A.nnzb, A.bs * A.bs, A.ia, A.ja, A.a, kind, ord, sg, opt.stage2_chunk,
                        F->st2_cls.get(), F->st2, s);
        char line[200];
        snprintf(line, sizeof line, "stage2 rows %d blocks/row %.1f layout chunk%d colours %d", A.nb,
                 (double)A.nnzb / A.nb, opt.stage2_chunk, (int)sg.size() - 1);
        F->tune_log.emplace_back(line);
    } else if (H0.fwd.ngroups > 0 && A.nb > 0) {
        std::vector<int> order = download_ints(H0.fwd.perm.get(), A.nb, s);
        {
            const std::vector<int> &g = H0.fwd.h_group_ptr;
            std::vector<int> cls(A.nb, 0);
            for (size_t c = 0; c + 1 < g.size(); ++c)
                for (int t = g[c]; t < g[c + 1]; ++t) cls[order[t]] = (int)c;
            F->st2_cls.alloc(A.nb);
            F->st2_cls.upload(cls.data(), A.nb, s);
        }
        // the hybrid form (precision 3) keeps the stage-2 block matrix in FP64
        const int kind = (fp64 || opt.precision == 3) ? VAL_F64 : VAL_F32;
        const std::string key = tune_key("stage2", A.nb, A.nnzb, kind, A.bs * A.bs, opt.autotune);
        TuneChoice cached_choice;
        bool cached = false;
        if (opt.autotune) {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = tune_cache().find(key);
            if (it != tune_cache().end()) {
                cached_choice = it->second;
                cached = true;
            }
        }
        if (!opt.autotune || cached) {
            const bool sell = cached ? cached_choice.sell != 0 : A.nb >= opt.sell_min_rows;
            build_level_mat(A.nb, A.nb, A.nnzb, A.bs * A.bs, A.ia, A.ja, A.a, kind, sell, order, H0.fwd.h_group_ptr,
                            H0.fwd.perm.get(), F->st2, s);
            if (cached) {
                F->opt.stage2_lanes = cached_choice.lanes;
                char line[200];
                snprintf(line, sizeof line, "stage2 rows %d blocks/row %.1f layout %s %.2f us (cached)", A.nb,
                         (double)A.nnzb / A.nb,
                         F->st2.sell ? "sell" : ("csr/" + std::to_string(F->opt.stage2_lanes)).c_str(),
                         cached_choice.us);
                F->tune_log.emplace_back(line);
            }
        } else {
            // time one stage-2 sweep per layout (CSR with 1..8 lanes per block row, sliced ELL)
            build_level_mat(A.nb, A.nb, A.nnzb, A.bs * A.bs, A.ia, A.ja, A.a, kind, false, order, H0.fwd.h_group_ptr,
                            H0.fwd.perm.get(), F->st2, s);
            DevBuf<double> rb((size_t)A.nb * A.bs), zb((size_t)A.nb * A.bs);
            rb.zero(s);
            zb.zero(s);
            if (!fp64) {
                F->r32.zero(s);
                F->z32.zero(s);
            }
            // one sweep in the precision the preconditioner runs it in (no conversions timed)
            auto time_sweep = [&]() {
                return time_best([&] {
                    if (fp64 || F->st2.kind == VAL_F64) F->template sweep_typed<double>(rb.get(), zb.get(), F->vt.get(), s);
                    else F->template sweep_typed<float>(F->r32.get(), F->z32.get(), F->vt32.get(), s);
                }, s);
            };
            double best = 1e30;
            int best_lanes = 4;
            for (int V = 1; V <= 8; V *= 2) {
                F->opt.stage2_lanes = V;
                const double t = time_sweep();
                if (t < best) {
                    best = t;
                    best_lanes = V;
                }
            }
            F->opt.stage2_lanes = best_lanes;
            if (A.nb >= 2048) {
                LevelMat S;
                build_level_mat(A.nb, A.nb, A.nnzb, A.bs * A.bs, A.ia, A.ja, A.a, kind, true, order,
                                H0.fwd.h_group_ptr, H0.fwd.perm.get(), S, s);
                std::swap(F->st2, S);
                const double t = time_sweep();
                if (t < best) best = t;
                else std::swap(F->st2, S);
            }
            char line[200];
            snprintf(line, sizeof line, "stage2 rows %d blocks/row %.1f layout %s %.2f us", A.nb,
                     (double)A.nnzb / A.nb,
                     F->st2.sell ? "sell" : ("csr/" + std::to_string(F->opt.stage2_lanes)).c_str(), best);
            F->tune_log.emplace_back(line);
            TuneChoice c;
            c.sell = F->st2.sell;
            c.lanes = F->opt.stage2_lanes;
            c.us = best;
            std::lock_guard<std::mutex> lk(g_tune_mu);
            tune_store(key, c);
        }
    }
    H.log.mark("fast_stage2", s);
    F->amg_err = H.err.get();
    F->setup_tail(opt.tail_rows, opt.tail_ctas, s);
    JX_CUDA(cudaStreamSynchronize(s));
    return F.release();
}

FastCprBase *make_fast_cpr(Amg &H, const BsrView<double> &A, const CprConfig &cfg, const FastOptions &opt,
                           cudaStream_t s) {
    if (opt.precision == 0) return build_fast<double>(H, A, cfg, opt, s);
    return build_fast<float>(H, A, cfg, opt, s);
}

}  // namespace jxcpr
