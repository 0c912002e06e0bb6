// staging.cu -- the pinned staging of staging.h.

#include "staging.h"

#include <algorithm>
#include <cstring>

#include "host_parallel.h"
#include "sync_wait.h"

namespace vrad {

PinnedShelf::~PinnedShelf() { release(); }

cudaError_t PinnedShelf::get(int slot, size_t bytes, void **out) {
    *out = nullptr;
    if (slot < 0 || slot >= kSlots) return cudaErrorInvalidValue;
    if (cap_[slot] < bytes) {
        if (ptr_[slot]) retired_.push_back(ptr_[slot]);
        ptr_[slot] = nullptr;
        cap_[slot] = 0;
        const size_t want = bytes + bytes / 4;
        const cudaError_t e = cudaHostAlloc(&ptr_[slot], want, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            ptr_[slot] = nullptr;
            return e;
        }
        cap_[slot] = want;
    }
    *out = ptr_[slot];
    return cudaSuccess;
}

void PinnedShelf::release() {
    for (int k = 0; k < kSlots; k++) {
        if (ptr_[k]) cudaFreeHost(ptr_[k]);
        ptr_[k] = nullptr;
        cap_[k] = 0;
    }
    for (void *p : retired_) cudaFreeHost(p);
    retired_.clear();
}

Stager::~Stager() { release(); }

void Stager::release() {
    for (int k = 0; k < kSlots; k++) {
        if (done_[k]) cudaEventSynchronize(done_[k]);
        if (slot_[k]) cudaFreeHost(slot_[k]);
        if (done_[k]) cudaEventDestroy(done_[k]);
        slot_[k] = nullptr;
        done_[k] = nullptr;
        pending_[k] = false;
    }
    cur_ = 0;
    off_ = 0;
}

// Leaves the current slot (its copies marked by an event) for the next,
// once that one's last copies are done.
cudaError_t Stager::advance(cudaStream_t stream) {
    cudaError_t e = cudaEventRecord(done_[cur_], stream);
    if (e != cudaSuccess) return e;
    pending_[cur_] = true;
    cur_ = (cur_ + 1) % kSlots;
    off_ = 0;
    if (pending_[cur_]) {
        e = cudaEventSynchronize(done_[cur_]);
        pending_[cur_] = false;
    }
    return e;
}

cudaError_t Stager::put(void *dst, const void *src, size_t bytes, cudaStream_t stream) {
    char *d = static_cast<char *>(dst);
    const char *s = static_cast<const char *>(src);
    while (bytes > 0) {
        if (!slot_[cur_]) {
            cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&slot_[cur_]), kSlotBytes, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done_[cur_], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        // A piece that fits the slot's rest goes there; a larger one starts
        // a fresh slot unless this one is nearly empty.
        if (off_ > 0 && kSlotBytes - off_ < std::min(bytes, kSlotBytes / 4)) {
            const cudaError_t e = advance(stream);
            if (e != cudaSuccess) return e;
            continue;
        }
        const size_t n = std::min(bytes, kSlotBytes - off_);
        char *stage = slot_[cur_] + off_;
        constexpr size_t kChunk = (size_t)1 << 20;
        if (n >= 2 * kChunk) {
            parallel_for((int64_t)((n + kChunk - 1) / kChunk), 1, [&](int64_t c) {
                const size_t a = (size_t)c * kChunk;
                std::memcpy(stage + a, s + a, std::min(kChunk, n - a));
            });
        } else {
            std::memcpy(stage, s, n);
        }
        const cudaError_t e = cudaMemcpyAsync(d, stage, n, cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return e;
        off_ += (n + 255) & ~(size_t)255;
        d += n;
        s += n;
        bytes -= n;
        if (off_ >= kSlotBytes) {
            const cudaError_t e2 = advance(stream);
            if (e2 != cudaSuccess) return e2;
        }
    }
    return cudaSuccess;
}

cudaError_t Stager::finish(cudaStream_t stream) {
    const cudaError_t e = vrad::wait_stream(stream);
    for (int k = 0; k < kSlots; k++) pending_[k] = false;
    cur_ = 0;
    off_ = 0;
    return e;
}

}  // namespace vrad
