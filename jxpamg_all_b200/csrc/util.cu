// Error-message storage and device queries shared by the library.
#include <stdarg.h>

#include <atomic>
#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.cuh"

namespace jxcpr {

static thread_local char g_err[512] = {0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char *last_error() { return g_err; }

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void uncount_launches(unsigned long long n) { g_launches.fetch_sub(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ---- device memory cache --------------------------------------------------
namespace {
struct MemPool {
    std::mutex mu;
    std::map<int, std::multimap<size_t, void *>> idle;                  // per device: reusable blocks
    std::map<int, std::vector<std::pair<size_t, void *>>> parked;       // freed since the last sync
    std::unordered_map<void *, std::pair<int, size_t>> owner;          // block -> (device, bucket)
    size_t cached = 0;                                                  // idle + parked bytes
    size_t limit = 24ull << 30;
};
MemPool &mem_pool() {
    static MemPool *p = new MemPool();  // never destroyed: DevBufs may be released at exit
    return *p;
}
size_t bucket_of(size_t bytes) {
    if (bytes <= 256) return 256;
    if (bytes < (1ull << 30)) {
        size_t b = 256;
        while (b < bytes) b <<= 1;
        return b;
    }
    const size_t q = 256ull << 20;
    return (bytes + q - 1) / q * q;
}
// caller holds the lock
void release_all(MemPool &P, int dev) {
    for (auto &kv : P.idle[dev]) {
        cudaFree(kv.second);
        P.owner.erase(kv.second);
        P.cached -= kv.first;
    }
    P.idle[dev].clear();
    for (auto &kv : P.parked[dev]) {
        cudaFree(kv.second);
        P.owner.erase(kv.second);
        P.cached -= kv.first;
    }
    P.parked[dev].clear();
}
}  // namespace

void *pool_alloc(size_t bytes) {
    MemPool &P = mem_pool();
    int dev = 0;
    JX_CUDA(cudaGetDevice(&dev));
    const size_t b = bucket_of(bytes);
    std::lock_guard<std::mutex> lk(P.mu);
    for (int attempt = 0; attempt < 2; ++attempt) {
        auto &fl = P.idle[dev];
        auto it = fl.find(b);
        if (it != fl.end()) {
            void *p = it->second;
            fl.erase(it);
            P.cached -= b;
            return p;
        }
        auto &pk = P.parked[dev];
        if (attempt == 0 && !pk.empty()) {
            // parked blocks become reusable once everything queued before their release is done
            JX_CUDA(cudaDeviceSynchronize());
            for (auto &kv : pk) fl.emplace(kv.first, kv.second);
            pk.clear();
            continue;
        }
        break;
    }
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaDeviceSynchronize();
        release_all(P, dev);
        e = cudaMalloc(&p, b);
    }
    if (e != cudaSuccess) {
        set_error("cudaMalloc(%zu bytes): %s", b, cudaGetErrorString(e));
        throw CudaError{e, "cudaMalloc"};
    }
    P.owner[p] = {dev, b};
    return p;
}

void pool_free(void *p) {
    if (!p) return;
    MemPool &P = mem_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.owner.find(p);
    if (it == P.owner.end()) {
        cudaFree(p);
        return;
    }
    const int dev = it->second.first;
    const size_t b = it->second.second;
    P.parked[dev].emplace_back(b, p);
    P.cached += b;
    if (P.cached > P.limit) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(dev);
        cudaDeviceSynchronize();
        release_all(P, dev);
        cudaSetDevice(cur);
    }
}

void pool_trim() {
    MemPool &P = mem_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    int cur = 0;
    cudaGetDevice(&cur);
    std::vector<int> devs;
    for (auto &kv : P.idle) devs.push_back(kv.first);
    for (auto &kv : P.parked) devs.push_back(kv.first);
    for (int d : devs) {
        cudaSetDevice(d);
        cudaDeviceSynchronize();
        release_all(P, d);
    }
    cudaSetDevice(cur);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

}  // namespace jxcpr
