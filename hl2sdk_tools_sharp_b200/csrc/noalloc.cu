// noalloc.cu -- a visibility trace over HOST buffers that allocates nothing.
//
// vrad_trace_visibility stages the caller's rays and hit bits through device
// buffers it grows with cudaMalloc.  Some callers cannot have that happen in
// the middle of a run: a process that reserves all of its device memory up
// front and lets nothing else allocate, or a host that must not stall on
// the device-wide synchronisation that freeing device memory can bring.  This entry point stages through one fixed
// array instead, declared below with a stated maximum, so its calls make no
// cudaMalloc, cudaFree or other allocating call.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds it (sizeof(vrad_ray) x VRAD_STATIC_MAX_RAYS for the rays,
// 8 KiB for the bits and 256 B for a status word: 1,843,456 bytes) until
// the process exits.  Host code cannot use its name as a device address;
// its address on each device is looked up by cudaGetSymbolAddress, with
// that device current, and that pointer is what the kernel is given.
//
// With lazy module loading (the CUDA 12 default) the array and the trace
// kernels' code are placed on a device only when first used, and placing
// them takes device memory.  vrad_create therefore calls
// prepare_static_trace for its device, so the look-up and the loads happen
// at set-up and no later call of the entry point makes them.  The cached
// address belongs to the device's primary context: the library does not
// survive a cudaDeviceReset (no call of it may follow one).

#include <cuda_runtime.h>

#include <mutex>

#include "scene.cuh"

namespace {

constexpr int64_t kMaxRays = VRAD_STATIC_MAX_RAYS;
constexpr size_t kRayBytes = sizeof(vrad_ray) * (size_t)kMaxRays;
constexpr size_t kBitBytes = 8 * (size_t)((kMaxRays + 63) / 64);
// Layout: [rays | hit bits | status word (traversal stack overflow)].
constexpr size_t kStatusOffset = kRayBytes + kBitBytes;
constexpr size_t kScratchBytes = kStatusOffset + 256;

static_assert(kRayBytes % 256 == 0, "bits must start 256-byte aligned");
static_assert(kScratchBytes == 1843456, "the size the header and the comment above state");

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// The device address of g_scratch on `device`, which must be current.
// Looked up on the first call for that device and kept.
cudaError_t scratch_on(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

}  // namespace

namespace vrad {

cudaError_t prepare_static_trace(int device) {
    unsigned char *base = nullptr;
    cudaError_t e = scratch_on(device, &base);
    if (e == cudaSuccess) e = load_visibility_kernels();
    return e;
}

// Called by vrad_trace_visibility_static in abi.cu with the context's lock
// held and its device current.
cudaError_t trace_visibility_static(const DeviceScene &scene, int device, cudaStream_t stream,
                                    const vrad_ray *h_rays, int64_t n, const TraceParams &p,
                                    uint64_t *h_bits) {
    unsigned char *base = nullptr;
    cudaError_t e = scratch_on(device, &base);
    if (e != cudaSuccess) return e;
    vrad_ray *d_rays = reinterpret_cast<vrad_ray *>(base);
    uint32_t *d_bits = reinterpret_cast<uint32_t *>(base + kRayBytes);
    uint32_t *d_status = reinterpret_cast<uint32_t *>(base + kStatusOffset);
    const size_t words64 = (size_t)((n + 63) / 64);
    // The array keeps the previous call's contents: clear the status word
    // and the bit words (the last one may belong to no warp).
    e = cudaMemsetAsync(d_status, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bits, 0, 8 * words64, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_rays, h_rays, sizeof(vrad_ray) * (size_t)n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = launch_trace(scene, d_rays, n, p, d_bits, nullptr, d_status, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_bits, d_bits, 8 * words64, cudaMemcpyDeviceToHost, stream);
    uint32_t status = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&status, d_status, sizeof status, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && status != 0) return cudaErrorLaunchOutOfResources;  // stack overflow
    return e;
}

}  // namespace vrad
