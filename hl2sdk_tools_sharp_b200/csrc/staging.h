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
