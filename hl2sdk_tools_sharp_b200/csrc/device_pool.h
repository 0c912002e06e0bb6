// device_pool.h -- a caching allocator for the device tables that the world
// and bounce uploads build and the light pass's per-call buffers.
//
// A released block goes back to a per-device cache instead of to cudaFree,
// and a later request takes the smallest cached block that holds it (at
// most a quarter larger below 1 MiB, at most twice the request above)
// before calling cudaMalloc: re-uploading a map of the same or a smaller
// size maps no new memory and unmaps none.  A cudaMalloc that runs out of
// memory empties that device's cache and tries once more.  dev_free does not
// wait for the device: callers synchronize before releasing blocks that
// kernels may still read (an upload first waits for its context's stream).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace vrad {

// A block of at least `bytes` on the current device (1 byte for 0).
cudaError_t dev_alloc(void **p, size_t bytes);

template <class T>
cudaError_t dev_alloc(T **p, size_t bytes) {
    void *q = nullptr;
    const cudaError_t e = dev_alloc(&q, bytes);
    *p = static_cast<T *>(q);
    return e;
}

// Back to the cache; null is ignored, a block the pool did not hand out
// goes to cudaFree.
void dev_free(void *p);

// cudaFree of every cached block of `device` (-1: of every device).
void dev_trim(int device);

// Bytes cached (not handed out) on `device`.
size_t dev_cached_bytes(int device);

// What the pool has asked of CUDA since the library loaded: cudaMalloc
// calls and their bytes, and the times an out-of-memory emptied a cache.
struct PoolCounters {
    int64_t mallocs = 0;
    int64_t malloc_bytes = 0;
    int64_t trims = 0;
};
PoolCounters dev_counters();

}  // namespace vrad
