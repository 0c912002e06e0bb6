// sync_wait.h -- how the library's host threads wait for a stream.
//
// By default a wait is cudaStreamSynchronize, which spins on a core and
// answers a few microseconds sooner.  A thread that turns on sleeping waits
// (a batch's workers do) waits on an event made with cudaEventBlockingSync
// instead: its core goes to the other maps' host set-up meanwhile.
#pragma once

#include <cuda_runtime.h>

namespace vrad {

struct ThreadWait {
    bool sleep = false;
    int device = -1;
    cudaEvent_t event = nullptr;
};

inline ThreadWait &thread_wait() {
    thread_local ThreadWait w;
    return w;
}

// Sleeping waits on (or off) for the calling thread; off releases the event.
inline void set_sleeping_waits(bool on) {
    ThreadWait &w = thread_wait();
    w.sleep = on;
    if (!on && w.event) {
        cudaEventDestroy(w.event);
        w.event = nullptr;
        w.device = -1;
    }
}

// Waits until the work queued on s so far has finished.
inline cudaError_t wait_stream(cudaStream_t s) {
    ThreadWait &w = thread_wait();
    if (!w.sleep) return cudaStreamSynchronize(s);
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (!w.event || w.device != device) {
        if (w.event) cudaEventDestroy(w.event);
        w.event = nullptr;
        e = cudaEventCreateWithFlags(&w.event, cudaEventBlockingSync | cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
        w.device = device;
    }
    e = cudaEventRecord(w.event, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(w.event);
    return e;
}

}  // namespace vrad
