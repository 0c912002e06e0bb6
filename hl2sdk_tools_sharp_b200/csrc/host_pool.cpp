// host_pool.cpp -- the cache of large host blocks behind uvector
// (host_parallel.h).
//
// A table of a few hundred MB that is freed and allocated again on every
// upload would otherwise be unmapped and mapped afresh each time, and its
// first writes would fault once per 4 KiB page (the kernel zeroes every
// page): about a tenth of the set-up's CPU time on the 8x8 map.  Blocks of
// 1 MiB and more are therefore kept when freed, up to a cap, and handed out
// again to a request of at most their size and at least half of it; new
// blocks are 2 MiB aligned and offered to the kernel for huge pages.

#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <cstdlib>
#include <iterator>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>

#include "host_parallel.h"

namespace vrad {

namespace {

constexpr size_t kAlign = (size_t)2 << 20;

struct HostCache {
    std::mutex mu;
    std::multimap<size_t, void *> cached;       // block size -> block
    std::unordered_map<void *, size_t> size_of;  // every live or cached block
    size_t cached_bytes = 0;
    size_t cap = 0;
};

HostCache &cache() {
    static HostCache *c = [] {
        HostCache *h = new HostCache;  // never destroyed: blocks may be freed after main returns
        const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
        const size_t phys = pages > 0 && page > 0 ? (size_t)pages * (size_t)page : ((size_t)16 << 30);
        h->cap = std::min(phys / 8, (size_t)32 << 30);
        return h;
    }();
    return *c;
}

}  // namespace

void *host_block_alloc(size_t bytes) {
    const size_t want = (bytes + kAlign - 1) / kAlign * kAlign;
    HostCache &c = cache();
    {
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.cached.lower_bound(want);
        if (it != c.cached.end() && it->first <= 2 * want) {
            void *p = it->second;
            c.cached_bytes -= it->first;
            c.cached.erase(it);
            return p;
        }
    }
    void *p = std::aligned_alloc(kAlign, want);
    if (!p) throw std::bad_alloc();
#ifdef MADV_HUGEPAGE
    madvise(p, want, MADV_HUGEPAGE);
#endif
    std::lock_guard<std::mutex> g(c.mu);
    c.size_of[p] = want;
    return p;
}

void host_block_free(void *p) {
    if (!p) return;
    HostCache &c = cache();
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.size_of.find(p);
    if (it == c.size_of.end()) return;  // not a block of this cache: never handed out by it
    const size_t size = it->second;
    // Over the cap, the largest cached blocks go first.
    while (c.cached_bytes + size > c.cap && !c.cached.empty()) {
        auto big = std::prev(c.cached.end());
        c.cached_bytes -= big->first;
        c.size_of.erase(big->second);
        std::free(big->second);
        c.cached.erase(big);
    }
    if (size > c.cap) {
        c.size_of.erase(it);
        std::free(p);
        return;
    }
    c.cached.emplace(size, p);
    c.cached_bytes += size;
}

}  // namespace vrad
