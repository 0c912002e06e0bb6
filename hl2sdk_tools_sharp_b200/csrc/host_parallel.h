// host_parallel.h -- the host set-up's two tools for large tables:
// parallel_for over an index range on the host's cores, and vectors whose
// elements start uninitialised (a resize writes nothing, so the pages are
// first touched by the parallel writers, not by one thread's zero fill).
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <memory>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace vrad {

// Threads the set-up uses: the host's cores, at most 32.
inline unsigned host_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    return std::max(1u, std::min(32u, hw));
}

// body(i) for every i in [0, n), chunks of `grain` indices handed out from a
// shared counter; the calling thread works too.  Bodies must not throw.
template <class F>
void parallel_for(int64_t n, int64_t grain, F &&body) {
    if (n <= 0) return;
    grain = std::max<int64_t>(1, grain);
    const int64_t chunks = (n + grain - 1) / grain;
    const unsigned nt = (unsigned)std::min<int64_t>(chunks, (int64_t)host_threads());
    std::atomic<int64_t> next{0};
    auto work = [&]() {
        for (int64_t i; (i = next.fetch_add(grain)) < n;) {
            const int64_t end = std::min(n, i + grain);
            for (int64_t k = i; k < end; k++) body(k);
        }
    };
    if (nt <= 1) {
        work();
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (unsigned t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
}

// An allocator whose value-initialising construct() default-initialises
// instead, so resize() of a trivial type leaves the memory untouched.
template <class T, class A = std::allocator<T>>
struct DefaultInitAllocator : A {
    using traits = std::allocator_traits<A>;
    template <class U>
    struct rebind {
        using other = DefaultInitAllocator<U, typename traits::template rebind_alloc<U>>;
    };
    using A::A;
    template <class U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... Args>
    void construct(U *p, Args &&...args) {
        traits::construct(static_cast<A &>(*this), p, std::forward<Args>(args)...);
    }
};

template <class T>
using uvector = std::vector<T, DefaultInitAllocator<T>>;

// Ordered concatenation of per-item lists: off[i]..off[i+1] is item i's
// run in `flat`; the copies run in parallel.
template <class T>
void concat_lists(const std::vector<std::vector<T>> &lists, std::vector<int32_t> &off, uvector<T> &flat) {
    const size_t n = lists.size();
    off.assign(n + 1, 0);
    int64_t total = 0;
    for (size_t i = 0; i < n; i++) {
        total += (int64_t)lists[i].size();
        off[i + 1] = (int32_t)total;
    }
    flat.resize((size_t)total);
    parallel_for((int64_t)n, 16, [&](int64_t i) {
        std::copy(lists[(size_t)i].begin(), lists[(size_t)i].end(), flat.begin() + off[(size_t)i]);
    });
}

}  // namespace vrad
