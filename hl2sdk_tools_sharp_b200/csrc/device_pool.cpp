// device_pool.cpp -- the caching allocator of device_pool.h.

#include "device_pool.h"

#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

namespace vrad {

namespace {

struct Pool {
    std::mutex mu;
    std::unordered_map<void *, std::pair<int, size_t>> live;  // handed out: device, block size
    std::map<int, std::multimap<size_t, void *>> cached;      // per device: block size -> block
    PoolCounters counters;
};

// Never destroyed: blocks may be released from static destructors after
// main returns.
Pool &pool() {
    static Pool *p = new Pool;
    return *p;
}

// Size classes: 512 B steps below 1 MiB, 2 MiB steps above.
size_t size_class(size_t bytes) {
    if (bytes == 0) bytes = 1;
    const size_t step = bytes < ((size_t)1 << 20) ? 512 : ((size_t)2 << 20);
    return (bytes + step - 1) / step * step;
}

void trim_locked(Pool &p, int device) {
    std::vector<void *> drop;
    for (auto it = p.cached.begin(); it != p.cached.end(); ++it) {
        if (device >= 0 && it->first != device) continue;
        for (auto &kv : it->second) drop.push_back(kv.second);
        it->second.clear();
    }
    for (void *q : drop) cudaFree(q);
}

// How much larger than the request a cached block may be and still be
// taken: a quarter below 1 MiB; up to twice the request above, so that a
// stream of maps of different sizes (a batch) reuses the blocks of the
// larger maps instead of mapping new memory for every map (a cudaMalloc
// costs about 25 ms per GB).
size_t slack(size_t want) { return want < ((size_t)1 << 20) ? want / 4 : want; }

}  // namespace

cudaError_t dev_alloc(void **out, size_t bytes) {
    *out = nullptr;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    const size_t want = size_class(bytes);
    Pool &p = pool();
    {
        std::lock_guard<std::mutex> g(p.mu);
        auto &c = p.cached[device];
        auto it = c.lower_bound(want);
        if (it != c.end() && it->first - want <= slack(want)) {
            *out = it->second;
            p.live[*out] = {device, it->first};
            c.erase(it);
            return cudaSuccess;
        }
    }
    e = cudaMalloc(out, want);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the recorded error before the retry
        {
            std::lock_guard<std::mutex> g(p.mu);
            trim_locked(p, device);
            p.counters.trims++;
        }
        e = cudaMalloc(out, want);
    }
    if (e != cudaSuccess) {
        *out = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> g(p.mu);
    p.live[*out] = {device, want};
    p.counters.mallocs++;
    p.counters.malloc_bytes += (int64_t)want;
    return cudaSuccess;
}

void dev_free(void *q) {
    if (!q) return;
    Pool &p = pool();
    {
        std::lock_guard<std::mutex> g(p.mu);
        auto it = p.live.find(q);
        if (it != p.live.end()) {
            p.cached[it->second.first].emplace(it->second.second, q);
            p.live.erase(it);
            return;
        }
    }
    cudaFree(q);  // not this pool's block
}

void dev_trim(int device) {
    Pool &p = pool();
    std::lock_guard<std::mutex> g(p.mu);
    trim_locked(p, device);
}

PoolCounters dev_counters() {
    Pool &p = pool();
    std::lock_guard<std::mutex> g(p.mu);
    return p.counters;
}

size_t dev_cached_bytes(int device) {
    Pool &p = pool();
    std::lock_guard<std::mutex> g(p.mu);
    size_t n = 0;
    auto it = p.cached.find(device);
    if (it != p.cached.end())
        for (auto &kv : it->second) n += kv.first;
    return n;
}

}  // namespace vrad
