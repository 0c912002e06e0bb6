// trace.cu -- ray traversal kernels: any-hit visibility, closest hit, and
// sky-passing visibility, over the BVH built in scene.cu.
//
// Per-triangle arithmetic is the reference's KdRayTracer.IntersectTriangle
// (MapTools/Tracing/KdRayTracer.cs:1194-1267) operation for operation, each
// an explicitly rounded intrinsic, so an accepted/rejected decision and a
// hit distance are the CPU's bits.  What the traversal adds is only WHICH
// triangles get tested: every triangle whose padded box the segment meets,
// which includes every triangle the predicate can accept (the pad is far
// above the rounding of the box test and of the predicate's hit point).
//
// Work distribution: one ray per thread, 128-thread CTAs scheduled by the
// hardware (no shared work counter, so launches on different streams never
// interfere); a warp's 32 visibility bits are one 32-bit word written with
// a single store after a ballot.  The traversal stack lives in shared
// memory, one column per thread.

#include <cfloat>

#include "scene.cuh"
#include "traverse.cuh"

namespace vrad {

namespace {

template <int MODE>
__global__ void __launch_bounds__(kBlock) k_trace(DeviceScene s, const vrad_ray *__restrict__ rays,
                                                  int64_t n, TraceParams p, uint32_t *__restrict__ bits,
                                                  vrad_hit *__restrict__ hits,
                                                  uint32_t *__restrict__ overflow) {
    extern __shared__ int stack_mem[];  // sc.stack_depth() entries per thread
    int *stack = stack_mem + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i - lane >= n) return;  // whole warp past the end
    bool hit = false;
    float best_t = 0.0f, reach = 1.0f;
    int32_t best_orig = -1;
    uint32_t best_meta = 0;
    if (i < n) {
        const float *f = reinterpret_cast<const float *>(rays + i);
        RayState r;
        r.ox = __ldg(f + 0);
        r.oy = __ldg(f + 1);
        r.oz = __ldg(f + 2);
        r.dx = __ldg(f + 3);
        r.dy = __ldg(f + 4);
        r.dz = __ldg(f + 5);
        reach = __ldg(f + 6);
        r.ix = recip_saturate(r.dx);
        r.iy = recip_saturate(r.dy);
        r.iz = recip_saturate(r.dz);
        r.nox = -r.ox * r.ix;
        r.noy = -r.oy * r.iy;
        r.noz = -r.oz * r.iz;
        trace_ray<MODE>(s, r, p.tmin, reach, p.skip_id, stack, overflow, hit, best_t, best_orig,
                        best_meta);
    }
    if (MODE == kModeClosest) {
        if (i < n) {
            vrad_hit h;
            if (hit) {
                h.surface = __ldg(&s.tri_id[best_orig]);
                h.fraction = reach == 1.0f ? best_t : __fdiv_rn(best_t, reach);
            } else {
                h.surface = -1;
                h.fraction = 1.0f;
            }
            hits[i] = h;
        }
    } else {
        const uint32_t word = __ballot_sync(kFull, hit);
        if (lane == 0) bits[i >> 5] = word;
    }
}

}  // namespace

cudaError_t launch_trace(const DeviceScene &scene, const vrad_ray *d_rays, int64_t n,
                         const TraceParams &p, uint32_t *d_bits, vrad_hit *d_hits,
                         uint32_t *d_overflow, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int64_t grid = (n + kBlock - 1) / kBlock;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
    const size_t smem = sizeof(int) * (size_t)scene.stack_depth() * kBlock;
    switch (p.mode) {
        case kModeAny:
            k_trace<kModeAny><<<(unsigned)grid, kBlock, smem, stream>>>(scene, d_rays, n, p, d_bits, d_hits, d_overflow);
            break;
        case kModeClosest:
            k_trace<kModeClosest><<<(unsigned)grid, kBlock, smem, stream>>>(scene, d_rays, n, p, d_bits, d_hits, d_overflow);
            break;
        default:
            k_trace<kModeSkyPass><<<(unsigned)grid, kBlock, smem, stream>>>(scene, d_rays, n, p, d_bits, d_hits, d_overflow);
            break;
    }
    return cudaGetLastError();
}

cudaError_t load_visibility_kernels() {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, k_trace<kModeAny>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_trace<kModeSkyPass>);
    return e;
}

}  // namespace vrad
