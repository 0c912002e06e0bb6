// staging.h -- host-to-device copies of the set-up's tables through pinned
// memory (staging.cu).  Each copy is packed into kSlots pinned slots of
// kSlotBytes: the host copies a piece into the current slot (in parallel
// for large pieces) and the DMA runs asynchronously on the upload's stream,
// overlapping the host's next piece and its next table; a slot is refilled
// only after the copies from its last use completed.  The source may be
// freed as soon as put() returns; the destination is written once finish()
// (a stream synchronisation) returns.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "device_pool.h"

namespace vrad {

class Stager {
public:
    static constexpr int kSlots = 8;
    static constexpr size_t kSlotBytes = (size_t)16 << 20;

    Stager() = default;
    Stager(const Stager &) = delete;
    Stager &operator=(const Stager &) = delete;
    ~Stager();

    cudaError_t put(void *dst, const void *src, size_t bytes, cudaStream_t stream);
    cudaError_t finish(cudaStream_t stream);
    void release();

private:
    cudaError_t advance(cudaStream_t stream);

    char *slot_[kSlots] = {};
    cudaEvent_t done_[kSlots] = {};
    bool pending_[kSlots] = {};
    int cur_ = 0;
    size_t off_ = 0;
};

// Pinned host tables a context keeps between uploads.  A table the set-up
// writes straight into a slot here reaches the device by one DMA, with no
// copy through the stager.  A slot that is too small gets a new block; the
// outgrown one is kept until release(), because freeing pinned memory can
// stall the device.  A slot's table may be rewritten only after the DMA
// that read it has completed (the uploads end with a stream wait).
class PinnedShelf {
public:
    static constexpr int kSlots = 16;

    PinnedShelf() = default;
    PinnedShelf(const PinnedShelf &) = delete;
    PinnedShelf &operator=(const PinnedShelf &) = delete;
    ~PinnedShelf();

    cudaError_t get(int slot, size_t bytes, void **out);
    template <class T>
    cudaError_t get(int slot, size_t n, T **out) {
        void *p = nullptr;
        const cudaError_t e = get(slot, sizeof(T) * (n ? n : 1), &p);
        *out = static_cast<T *>(p);
        return e;
    }
    void release();

private:
    void *ptr_[kSlots] = {};
    size_t cap_[kSlots] = {};
    std::vector<void *> retired_;
};

// A device block from the pool for n elements at src (one at least),
// filled by one asynchronous copy on `stream` (src is pinned).
template <class T>
cudaError_t dma_table(T **dst, const T *src, size_t n, cudaStream_t stream) {
    cudaError_t e = dev_alloc(dst, sizeof(T) * (n ? n : 1));
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, stream);
    return e;
}

// A device block from the pool for the table v (one element at least),
// filled through the stager on `stream`.
template <class T, class V>
cudaError_t stage_table(Stager &st, cudaStream_t stream, T **dst, const V &v) {
    static_assert(sizeof(typename V::value_type) == sizeof(T), "element size");
    cudaError_t e = dev_alloc(dst, sizeof(T) * (v.empty() ? 1 : v.size()));
    if (e == cudaSuccess && !v.empty()) e = st.put(*dst, v.data(), sizeof(T) * v.size(), stream);
    return e;
}

}  // namespace vrad
