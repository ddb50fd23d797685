// Shared definitions for the B200 CPR-GMRES library: status codes, CUDA
// error plumbing, device buffers and small launch helpers.
//
// Status codes follow the reference (jxfpamg-0220/include/jxf_util.h:152-159):
// 0 success, 1 generic, 2 memory, 4 argument, 256 convergence; this library
// adds JXCPR_ERROR_DEVICE for a failed CUDA call and JXCPR_ERROR_NUMERIC for a
// NaN/Inf seen on the device.  No entry point aborts the process.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <cstddef>
#include <string>
#include <utility>

#define JXCPR_SUCCESS 0
#define JXCPR_ERROR_GENERIC 1
#define JXCPR_ERROR_MEMORY 2
#define JXCPR_ERROR_ARG 4
#define JXCPR_ERROR_CONV 256
#define JXCPR_ERROR_DEVICE 512
#define JXCPR_ERROR_NUMERIC 1024

namespace jxcpr {

// Last error message (thread-local) for diagnostics through the C ABI.
void set_error(const char *fmt, ...);
const char *last_error();
unsigned long long launch_count();
// kernels recorded into a graph are counted when the graph runs, not when captured
void uncount_launches(unsigned long long n);

// Number of SMs of the current device (cached per device).
int sm_count();

struct CudaError {
    cudaError_t code;
    const char *what;
};

#define JX_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e__ = (call);                                                      \
        if (e__ != cudaSuccess) {                                                      \
            ::jxcpr::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,              \
                               cudaGetErrorString(e__));                               \
            throw ::jxcpr::CudaError{e__, #call};                                      \
        }                                                                              \
    } while (0)

// Every kernel launch site is followed by JX_LAUNCH_CHECK(), which also counts
// the launch (reported through jxcpr_launch_count()).
void count_launch();
void count_launches(unsigned long long n);  // kernels replayed by a CUDA graph launch
#define JX_LAUNCH_CHECK()                     \
    do {                                      \
        ::jxcpr::count_launch();              \
        JX_CUDA(cudaGetLastError());          \
    } while (0)

// Programmatic dependent launch.  A kernel launched by launch_dep while
// tl_dep_launch is set carries the programmatic-stream-serialization
// attribute (in a captured graph: a programmatic edge), so the GPU may start
// scheduling its blocks while the kernel before it drains.  Every kernel
// launched that way calls grid_dep_wait() before it reads or writes global
// memory: the wait returns once the previous kernel has completed and its
// writes are visible (at once for a kernel launched without the attribute).
__device__ __forceinline__ void grid_dep_wait() {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}
extern thread_local int tl_dep_launch;
struct DepLaunchScope {
    int saved;
    explicit DepLaunchScope(int on) : saved(tl_dep_launch) { tl_dep_launch = on; }
    ~DepLaunchScope() { tl_dep_launch = saved; }
};
template <typename... KArgs, typename... Args>
void launch_dep(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = tl_dep_launch ? 1 : 0;
    JX_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
}

// Device memory cache behind DevBuf.  Blocks are bucketed (powers of two up
// to 1 GiB, 256 MiB multiples above); buckets up to 1 MiB are carved from
// 32 MiB slabs, so a setup makes few cudaMalloc calls.
//  * Inside a PoolStream scope the thread's work goes to one stream: blocks
//    are tagged with it, and a freed tagged block is reused at once by the
//    next allocation under the same stream (stream order puts the new work
//    after every earlier use), with no device synchronisation.
//  * Other blocks are parked when freed and become reusable after a device
//    synchronisation (the one cudaFree would have done).
// pool_forget_stream(s, drained) is called before a tagged stream is
// destroyed or replaced: its idle blocks become reusable by any stream if
// nothing is left queued on s (drained), else they are parked; its live
// blocks park when freed.
void *pool_alloc(size_t bytes);
void pool_free(void *p);
void pool_trim();
void pool_forget_stream(cudaStream_t s, bool drained);
// process-wide: cudaMalloc calls, their total ms, device synchronisations, their total ms
void pool_stats(double out[4]);

struct PoolStream {
    explicit PoolStream(cudaStream_t s);
    ~PoolStream();
    PoolStream(const PoolStream &) = delete;
    PoolStream &operator=(const PoolStream &) = delete;
    cudaStream_t prev;
    bool prev_set;
};

// Owning device buffer (256-byte aligned, padded by 64 bytes so that
// 16-byte-rounded bulk copies of the tail stay inside the allocation).
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        const size_t bytes = count * sizeof(T) + 64;
        p = static_cast<T *>(pool_alloc(bytes));
        n = count;
    }
    void release() {
        if (p) pool_free(p);
        p = nullptr;
        n = 0;
    }
    void zero(cudaStream_t s) { if (n) JX_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void upload(const T *h, size_t count, cudaStream_t s) {
        if (count) JX_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T *h, size_t count, cudaStream_t s) const {
        if (count) JX_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    T *get() const { return p; }
};

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace jxcpr
