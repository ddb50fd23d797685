// Error-message storage and device queries shared by the library.
#include <stdarg.h>

#include <algorithm>
#include <atomic>
#include <chrono>
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

thread_local int tl_dep_launch = 0;

// ---- device memory cache --------------------------------------------------
namespace {
thread_local cudaStream_t t_stream = nullptr;
thread_local bool t_stream_set = false;

constexpr size_t kSlabBucketMax = 1ull << 20;  // buckets carved from slabs
constexpr size_t kSlabBytes = 32ull << 20;

struct Block {
    int dev;
    size_t bucket;
    bool tagged;
    bool carved;
    cudaStream_t stream;
    unsigned long long epoch;
};
using TagKey = std::pair<int, std::pair<cudaStream_t, unsigned long long>>;

struct MemPool {
    std::mutex mu;
    std::map<int, std::multimap<size_t, void *>> idle;              // per device: reusable on any stream
    std::map<TagKey, std::multimap<size_t, void *>> idle_tagged;     // reusable on their own stream
    std::map<int, std::vector<std::pair<size_t, void *>>> parked;    // freed since the last device sync
    std::unordered_map<void *, Block> owner;
    std::map<cudaStream_t, unsigned long long> epoch;                // bumped by pool_forget_stream
    std::map<int, std::vector<void *>> slabs;
    std::map<int, std::pair<char *, size_t>> slab_cur;               // bump pointer, bytes left
    size_t cached = 0;                                               // idle + parked bytes, not carved
    size_t limit = 24ull << 30;
    double n_malloc = 0, ms_malloc = 0, n_sync = 0, ms_sync = 0;
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
double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}
// The caller holds the lock.
void device_sync(MemPool &P) {
    const auto t = std::chrono::steady_clock::now();
    JX_CUDA(cudaDeviceSynchronize());
    P.n_sync += 1;
    P.ms_sync += ms_since(t);
}
// The caller holds the lock and has synchronised the device: every cached block is idle.
void unpark_all(MemPool &P, int dev) {
    for (auto &kv : P.parked[dev]) P.idle[dev].emplace(kv.first, kv.second);
    P.parked[dev].clear();
    for (auto it = P.idle_tagged.begin(); it != P.idle_tagged.end();) {
        if (it->first.first != dev) {
            ++it;
            continue;
        }
        for (auto &kv : it->second) {
            P.owner[kv.second].tagged = false;
            P.idle[dev].emplace(kv.first, kv.second);
        }
        it = P.idle_tagged.erase(it);
    }
}
// The caller holds the lock and has synchronised the device: the idle blocks
// that are not carved from a slab go back to the driver.
void release_idle(MemPool &P, int dev) {
    unpark_all(P, dev);
    auto &fl = P.idle[dev];
    for (auto it = fl.begin(); it != fl.end();) {
        auto o = P.owner.find(it->second);
        if (o != P.owner.end() && o->second.carved) {
            ++it;
            continue;
        }
        cudaFree(it->second);
        if (o != P.owner.end()) P.owner.erase(o);
        P.cached -= it->first;
        it = fl.erase(it);
    }
}
void *carve(MemPool &P, int dev, size_t b) {
    auto &cur = P.slab_cur[dev];
    if (cur.second < b) {
        void *slab = nullptr;
        const auto t = std::chrono::steady_clock::now();
        const cudaError_t e = cudaMalloc(&slab, kSlabBytes);
        P.n_malloc += 1;
        P.ms_malloc += ms_since(t);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        P.slabs[dev].push_back(slab);
        cur = {static_cast<char *>(slab), kSlabBytes};
    }
    void *p = cur.first;
    cur.first += b;
    cur.second -= b;
    return p;
}
}  // namespace

PoolStream::PoolStream(cudaStream_t s) : prev(t_stream), prev_set(t_stream_set) {
    t_stream = s;
    t_stream_set = true;
}
PoolStream::~PoolStream() {
    t_stream = prev;
    t_stream_set = prev_set;
}

void *pool_alloc(size_t bytes) {
    MemPool &P = mem_pool();
    int dev = 0;
    JX_CUDA(cudaGetDevice(&dev));
    const size_t b = bucket_of(bytes);
    std::lock_guard<std::mutex> lk(P.mu);
    const bool tag = t_stream_set;
    const cudaStream_t ts = t_stream;
    const unsigned long long ep = tag ? P.epoch[ts] : 0;
    auto take = [&](std::multimap<size_t, void *> &fl) -> void * {
        auto it = fl.find(b);
        if (it == fl.end()) return nullptr;
        void *p = it->second;
        fl.erase(it);
        Block &B = P.owner[p];
        if (!B.carved) P.cached -= b;
        B.tagged = tag;
        B.stream = ts;
        B.epoch = ep;
        return p;
    };
    if (tag) {
        auto it = P.idle_tagged.find(TagKey{dev, {ts, ep}});
        if (it != P.idle_tagged.end())
            if (void *p = take(it->second)) return p;
    }
    if (void *p = take(P.idle[dev])) return p;
    if (!tag && !P.parked[dev].empty()) {
        // parked blocks become reusable once everything queued before their release is done
        device_sync(P);
        unpark_all(P, dev);
        if (void *p = take(P.idle[dev])) return p;
    }
    void *p = nullptr;
    bool carved = false;
    if (b <= kSlabBucketMax) {
        p = carve(P, dev, b);
        carved = p != nullptr;
    }
    if (!p) {
        const auto t = std::chrono::steady_clock::now();
        cudaError_t e = cudaMalloc(&p, b);
        P.n_malloc += 1;
        P.ms_malloc += ms_since(t);
        if (e != cudaSuccess) {
            cudaGetLastError();
            device_sync(P);
            release_idle(P, dev);
            e = cudaMalloc(&p, b);
        }
        if (e != cudaSuccess) {
            set_error("cudaMalloc(%zu bytes): %s", b, cudaGetErrorString(e));
            throw CudaError{e, "cudaMalloc"};
        }
    }
    P.owner[p] = Block{dev, b, tag, carved, ts, ep};
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
    const Block B = it->second;
    auto ep = P.epoch.find(B.stream);
    const unsigned long long cur = ep == P.epoch.end() ? 0 : ep->second;
    if (B.tagged && cur == B.epoch)
        P.idle_tagged[TagKey{B.dev, {B.stream, B.epoch}}].emplace(B.bucket, p);
    else
        P.parked[B.dev].emplace_back(B.bucket, p);
    if (!B.carved) P.cached += B.bucket;
    if (P.cached > P.limit) {
        int dv = 0;
        cudaGetDevice(&dv);
        cudaSetDevice(B.dev);
        cudaDeviceSynchronize();
        release_idle(P, B.dev);
        cudaSetDevice(dv);
    }
}

void pool_forget_stream(cudaStream_t s, bool drained) {
    MemPool &P = mem_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    const unsigned long long old = P.epoch[s];
    P.epoch[s] = old + 1;
    for (auto it = P.idle_tagged.begin(); it != P.idle_tagged.end();) {
        if (it->first.second.first != s || it->first.second.second != old) {
            ++it;
            continue;
        }
        for (auto &kv : it->second) {
            P.owner[kv.second].tagged = false;
            if (drained) P.idle[it->first.first].emplace(kv.first, kv.second);  // nothing left queued on s
            else P.parked[it->first.first].emplace_back(kv.first, kv.second);
        }
        it = P.idle_tagged.erase(it);
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
    for (auto &kv : P.idle_tagged) devs.push_back(kv.first.first);
    for (auto &kv : P.slabs) devs.push_back(kv.first);
    std::sort(devs.begin(), devs.end());
    devs.erase(std::unique(devs.begin(), devs.end()), devs.end());
    for (int d : devs) {
        cudaSetDevice(d);
        cudaDeviceSynchronize();
        release_idle(P, d);
        // the slabs go back only when none of their blocks is in use (every carved block idle)
        size_t carved_total = 0;
        for (auto &kv : P.owner)
            if (kv.second.dev == d && kv.second.carved) ++carved_total;
        if (carved_total == P.idle[d].size()) {
            for (auto &kv : P.idle[d]) P.owner.erase(kv.second);
            P.idle[d].clear();
            for (void *sl : P.slabs[d]) cudaFree(sl);
            P.slabs[d].clear();
            P.slab_cur[d] = {nullptr, 0};
        }
    }
    cudaSetDevice(cur);
}

void pool_stats(double out[4]) {
    MemPool &P = mem_pool();
    std::lock_guard<std::mutex> lk(P.mu);
    out[0] = P.n_malloc;
    out[1] = P.ms_malloc;
    out[2] = P.n_sync;
    out[3] = P.ms_sync;
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
