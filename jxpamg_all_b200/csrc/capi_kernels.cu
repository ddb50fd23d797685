// C ABI of the individual device kernels (device pointers, caller's stream).
// These are the building blocks the solver chains; they are exported so that
// tests and benchmarks can drive each kernel alone.  Every entry returns a
// status code (0 = success) and never aborts; jxcpr_last_error() explains a
// failure.
#include <mutex>
#include <stdexcept>

#include "amg.cuh"
#include "common.cuh"
#include "jxcpr_b200.h"
#include "kernels.cuh"

using namespace jxcpr;

namespace {
// Per-device error flag used by the staged kernels when the caller gives none.
int *device_err_flag() {
    static std::mutex mu;
    static int *flags[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!flags[dev]) {
        if (cudaMalloc(&flags[dev], sizeof(int)) != cudaSuccess) return nullptr;
        cudaMemset(flags[dev], 0, sizeof(int));
    }
    return flags[dev];
}

template <typename F>
int guarded(F &&f) {
    try {
        f();
        return JXCPR_SUCCESS;
    } catch (const CudaError &) {
        return JXCPR_ERROR_DEVICE;
    } catch (const std::invalid_argument &) {
        return JXCPR_ERROR_ARG;  // the message was set where it was thrown
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return JXCPR_ERROR_MEMORY;
    } catch (...) {
        set_error("unexpected exception");
        return JXCPR_ERROR_GENERIC;
    }
}

template <typename V>
int bsr_check(int nb, int bs, long long nnzb, const int *ia, const int *ja, const V *a) {
    if (nb < 0 || nnzb < 0 || (bs != 2 && bs != 3)) {
        set_error("bsr: bad sizes nb=%d bs=%d nnzb=%lld", nb, bs, nnzb);
        return JXCPR_ERROR_ARG;
    }
    if (nb > 0 && (!ia || (nnzb > 0 && (!ja || !a)))) {
        set_error("bsr: null array");
        return JXCPR_ERROR_ARG;
    }
    return JXCPR_SUCCESS;
}
}  // namespace

extern "C" {

int jxcpr_version(void) { return 10000; }

unsigned long long jxcpr_launch_count(void) { return launch_count(); }

const char *jxcpr_last_error(void) { return last_error(); }

int jxcpr_bsr_matvec_dev(int nb, int bs, long long nnzb, const int *ia, const int *ja, const double *a,
                         double alpha, const double *x, double beta, double *y, int staged, void *stream) {
    int st = bsr_check(nb, bs, nnzb, ia, ja, a);
    if (st) return st;
    return guarded([&] {
        BsrView<double> A{nb, bs, nnzb, ia, ja, a};
        bsr_spmv<double, double>(A, alpha, x, beta, y, staged ? device_err_flag() : nullptr,
                                 (cudaStream_t)stream, staged != 0);
    });
}

int jxcpr_bsr_matvec_dev_f32(int nb, int bs, long long nnzb, const int *ia, const int *ja, const float *a,
                             double alpha, const double *x, double beta, double *y, int staged, void *stream) {
    int st = bsr_check(nb, bs, nnzb, ia, ja, a);
    if (st) return st;
    return guarded([&] {
        BsrView<float> A{nb, bs, nnzb, ia, ja, a};
        bsr_spmv<float, double>(A, alpha, x, beta, y, staged ? device_err_flag() : nullptr,
                                (cudaStream_t)stream, staged != 0);
    });
}

// Reads and clears the per-device kernel error flag (nonzero: a bounded wait gave up).
int jxcpr_kernel_error_flag(void) {
    int *f = device_err_flag();
    if (!f) return -1;
    int v = 0;
    if (cudaMemcpy(&v, f, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    cudaMemset(f, 0, sizeof(int));
    return v;
}

int jxcpr_dot_dev(long long n, const double *x, const double *y, double *out_host, void *stream) {
    return guarded([&] {
        cudaStream_t s = (cudaStream_t)stream;
        DevBuf<double> part(reduce_partials() + 1);
        dot_dev(n, x, y, part.get(), part.get() + reduce_partials(), s);
        JX_CUDA(cudaMemcpyAsync(out_host, part.get() + reduce_partials(), sizeof(double), cudaMemcpyDeviceToHost,
                                s));
        JX_CUDA(cudaStreamSynchronize(s));
    });
}

int jxcpr_dense_inverse_dev(int n, const double *a, double *ainv, void *stream) {
    if (n < 0 || n > 8192 || (n > 0 && (!a || !ainv))) {
        set_error("dense_inverse: n must be in [0, 8192] and the pointers set (n = %d)", n);
        return JXCPR_ERROR_ARG;
    }
    return guarded([&] { dense_inverse_mma(n, a, ainv, (cudaStream_t)stream); });
}

}  // extern "C"

extern "C" int jxcpr_pool_stats(double *out) {
    if (!out) return JXCPR_ERROR_ARG;
    jxcpr::pool_stats(out);
    return JXCPR_SUCCESS;
}

extern "C" int jxcpr_release_cached_memory(void) {
    try {
        jxcpr::pool_trim();
    } catch (...) {
        return JXCPR_ERROR_DEVICE;
    }
    return JXCPR_SUCCESS;
}
