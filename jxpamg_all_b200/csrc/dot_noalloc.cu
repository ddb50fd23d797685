// Inner product that allocates nothing: jxcpr_dot_dev_noalloc.
//
// Some callers cannot allocate device memory at the moment they need an inner
// product -- a host application whose memory pool has reserved the whole
// device, or a time-critical loop that forbids allocator calls on its critical
// path (cudaMalloc can synchronise the device and stall every stream).  jxcpr_dot_dev allocates its per-CTA partial sums on
// every call, which these callers cannot accept.  This variant keeps the
// partial sums and the result in a fixed file-scope device array:
// JXCPR_NOALLOC_DOT_MAX_PARTIALS doubles of partial sums (one per
// JXCPR_NOALLOC_DOT_CHUNK elements) plus one result slot, 512 KB per GPU,
// held until the process exits.
//
// When the array comes into being: the library is built one module per source
// file and CUDA loads modules lazily, so this file's module -- and with it the
// array -- is loaded on a device by the first call on that device (the
// cudaGetSymbolAddress below).  That load takes device memory like any other
// module load.  A caller whose pool will later reserve the whole device makes
// one warm-up call (n = 0 is enough) on each device before the pool does;
// every later call allocates nothing.
//
// The array is shared by every call on a device and keeps the last call's
// contents.  Each call writes every partial it reads and overwrites the
// result, so nothing has to start at zero; but two calls that overlap on the
// GPU (concurrent streams) race on the array and must be serialised by the
// caller.  Host code cannot use the array's name as a device address: on the
// first call on each device (that device current) the library resolves the
// address with cudaGetSymbolAddress and caches it.  Every call copies the
// result to the host and synchronises its stream, so it must not be called
// while that stream is being captured into a CUDA graph.
#include <mutex>

#include "common.cuh"
#include "jxcpr_b200.h"

namespace {

constexpr long long kChunk = JXCPR_NOALLOC_DOT_CHUNK;
constexpr int kMaxPartials = JXCPR_NOALLOC_DOT_MAX_PARTIALS;
constexpr int kThreads = 256;

// partial sums [0, kMaxPartials), result at [kMaxPartials]
static __device__ __align__(256) double g_dot_scratch[kMaxPartials + 32];

std::mutex g_mu;
// Cached per device; a cudaDeviceReset by the application would unload the module and leave the
// cached address stale (the library assumes the context lives as long as the process).
double *g_addr[64] = {nullptr};

// Device address of g_dot_scratch for the current device (resolved once).
int scratch_address(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        jxcpr::set_error("dot_noalloc: no current CUDA device (%s)", cudaGetErrorString(e));
        return JXCPR_ERROR_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess || !p) {
            jxcpr::set_error("dot_noalloc: cudaGetSymbolAddress failed on device %d (%s)", dev,
                             cudaGetErrorString(e));
            return JXCPR_ERROR_DEVICE;
        }
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return JXCPR_SUCCESS;
}

// One CTA per chunk of kChunk elements: partials[blockIdx.x] = sum x*y.
__global__ void __launch_bounds__(kThreads) chunk_dot_kernel(long long n, const double *__restrict__ x,
                                                             const double *__restrict__ y,
                                                             double *__restrict__ partials) {
    __shared__ double ws[kThreads / 32];
    const long long base = (long long)blockIdx.x * kChunk;
    const long long end = base + kChunk < n ? base + kChunk : n;
    double acc = 0.0;
    for (long long i = base + threadIdx.x; i < end; i += kThreads) acc += x[i] * y[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < kThreads / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = r;
    }
}

// One CTA adds the partials in a fixed order into *out.
__global__ void __launch_bounds__(kThreads) sum_chunks_kernel(int np, const double *__restrict__ partials,
                                                              double *__restrict__ out) {
    __shared__ double ws[kThreads / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += kThreads) acc += partials[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < kThreads / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) *out = r;
    }
}

}  // namespace

extern "C" int jxcpr_dot_dev_noalloc(long long n, const double *x, const double *y, double *out_host,
                                     void *stream) {
    if (n < 0 || !out_host || (n > 0 && (!x || !y))) {
        jxcpr::set_error("dot_noalloc: bad arguments");
        return JXCPR_ERROR_ARG;
    }
    const long long max_n = kChunk * (long long)kMaxPartials;
    if (n > max_n) {
        jxcpr::set_error("dot_noalloc: n = %lld exceeds the static scratch limit of %lld elements "
                         "(%d partial sums of %lld elements); use jxcpr_dot_dev",
                         n, max_n, kMaxPartials, kChunk);
        return JXCPR_ERROR_ARG;
    }
    double *scratch = nullptr;
    int st = scratch_address(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    double *partials = scratch, *result = scratch + kMaxPartials;
    const int np = (int)((n + kChunk - 1) / kChunk);
    if (np > 0) chunk_dot_kernel<<<np, kThreads, 0, s>>>(n, x, y, partials);
    sum_chunks_kernel<<<1, kThreads, 0, s>>>(np, partials, result);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_host, result, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        jxcpr::set_error("dot_noalloc: %s", cudaGetErrorString(e));
        return JXCPR_ERROR_DEVICE;
    }
    return JXCPR_SUCCESS;
}
