// host_parallel.h -- the host set-up's tools for large tables:
// parallel_for over an index range on a persistent pool of worker threads
// (started on first use, one per host core, at most 32), and vectors whose
// elements start uninitialised (a resize writes nothing, so the pages are
// first touched by the parallel writers, not by one thread's zero fill).
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
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

// The workers behind parallel_for.  Several callers (a batch's workers,
// each setting up its own map) may run jobs at once: the jobs wait in
// arrival order, and a free pool thread joins the oldest job that still
// wants threads, so a job's tail (its last chunks, worked on by a few
// threads) leaves the other threads free for the next job.  The calling
// thread works on its own job too.
class HostPool {
public:
    static HostPool &get() {
        static HostPool *p = new HostPool(host_threads() - 1);  // never destroyed: workers may outlive statics
        return *p;
    }

    // fn() on up to `workers` pool threads and on the caller.  fn must
    // return at once when the job has no work left (a late joiner finds
    // none).
    void run(unsigned workers, const std::function<void()> &fn) {
        Job job;
        job.fn = &fn;
        job.want = std::min<unsigned>(workers, (unsigned)threads_.size());
        if (job.want > 0) {
            {
                std::lock_guard<std::mutex> g(mu_);
                queue_.push_back(&job);
            }
            cv_.notify_all();
        }
        fn();
        std::unique_lock<std::mutex> g(mu_);
        // No thread joins the job after this point.
        for (size_t k = 0; k < queue_.size(); k++)
            if (queue_[k] == &job) {
                queue_.erase(queue_.begin() + (std::ptrdiff_t)k);
                break;
            }
        done_cv_.wait(g, [&] { return job.done == job.taken; });
    }

private:
    struct Job {
        const std::function<void()> *fn = nullptr;
        unsigned want = 0, taken = 0, done = 0;
    };

    explicit HostPool(unsigned n) {
        for (unsigned i = 0; i < n; i++) threads_.emplace_back([this] { loop(); });
        for (auto &t : threads_) t.detach();
    }

    void loop() {
        std::unique_lock<std::mutex> g(mu_);
        while (true) {
            cv_.wait(g, [&] { return !queue_.empty(); });
            Job *job = queue_.front();
            if (++job->taken == job->want) queue_.erase(queue_.begin());
            g.unlock();
            (*job->fn)();
            g.lock();
            if (++job->done == job->taken) done_cv_.notify_all();
        }
    }

    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::vector<Job *> queue_;   // jobs that still want threads, oldest first
};

// Whether this thread is running a parallel_for body.
inline bool &in_parallel_body() {
    thread_local bool inside = false;
    return inside;
}

// body(i) for every i in [0, n), chunks of `grain` indices handed out from a
// shared counter to the pool's workers and the calling thread.  Bodies must
// not throw.  A call from inside a body runs serially.
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
    if (nt <= 1 || in_parallel_body()) {
        work();
        return;
    }
    const std::function<void()> job = [&]() {
        bool &inside = in_parallel_body();
        const bool was = inside;
        inside = true;
        work();
        inside = was;
    };
    HostPool::get().run(nt - 1, job);
}

// Large host blocks (host_pool.cpp): at least `bytes`, 2 MiB aligned, kept
// when freed and handed out again, so that their pages stay mapped.
void *host_block_alloc(size_t bytes);
void host_block_free(void *p);
constexpr size_t kHostBlockMin = (size_t)1 << 20;

// An allocator whose value-initialising construct() default-initialises
// instead, so resize() of a trivial type leaves the memory untouched, and
// whose blocks of 1 MiB and more come from the cache of host blocks.
template <class T, class A = std::allocator<T>>
struct DefaultInitAllocator : A {
    using traits = std::allocator_traits<A>;
    template <class U>
    struct rebind {
        using other = DefaultInitAllocator<U, typename traits::template rebind_alloc<U>>;
    };
    using A::A;
    T *allocate(size_t n) {
        if (n * sizeof(T) >= kHostBlockMin) return static_cast<T *>(host_block_alloc(n * sizeof(T)));
        return A::allocate(n);
    }
    void deallocate(T *p, size_t n) {
        if (n * sizeof(T) >= kHostBlockMin) host_block_free(p);
        else A::deallocate(p, n);
    }
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
