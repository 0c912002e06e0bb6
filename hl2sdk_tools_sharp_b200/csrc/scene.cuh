// scene.cuh -- device-resident scene of one context, and its GPU build.
#pragma once

#include <cuda_runtime.h>

#include "vrad_internal.cuh"

namespace vrad {

// One BVH over a subset of the scene's triangles.
struct BvhBuffers {
    float4 *tri0 = nullptr;
    float4 *tri1 = nullptr;
    float4 *tri2 = nullptr;
    float4 *nodes = nullptr;
    int32_t ntris = 0;
    int32_t depth = 0;  // inner nodes on the longest root-to-leaf path

    void release();
    DeviceBvh view() const { return DeviceBvh{tri0, tri1, tri2, nodes, ntris, depth}; }
};

struct SceneBuffers {
    BvhBuffers opaque;
    BvhBuffers sky;
    int32_t *tri_id = nullptr;  // caller ids by original index
    int32_t ntris = 0;

    void release();
    DeviceScene view() const { return DeviceScene{opaque.view(), sky.view(), tri_id}; }
};

struct SceneBuildReport {
    int32_t nodes = 0;
    int32_t leaves = 0;
    int32_t max_leaf = 0;
    int32_t max_depth = 0;
    float bounds[6] = {0, 0, 0, 0, 0, 0};
    float pad = 0;
    float build_ms = 0;
    double sah_cost = 0;       // the SAH trees' expected cost per ray (node visits + triangle tests)
    int64_t device_bytes = 0;
};

// Builds one BVH from n host triangles (and, optionally, their
// intersection form); h_orig gives each triangle's original index in the
// whole scene.  Synchronises `stream` before returning.  report is
// accumulated into (counts added, bounds merged).
cudaError_t build_bvh(BvhBuffers &bb, const vrad_triangle *h_tris,
                      const vrad_kd_triangle *h_prepared, const int32_t *h_orig, int n,
                      cudaStream_t stream, SceneBuildReport *report);

// Traversal launches (trace.cu).  d_bits is written as 32-bit words.
cudaError_t launch_trace(const DeviceScene &scene, const vrad_ray *d_rays, int64_t n,
                         const TraceParams &p, uint32_t *d_bits, vrad_hit *d_hits,
                         uint32_t *d_overflow, cudaStream_t stream);

// Loads the visibility trace kernels' code on the current device (with lazy
// module loading a kernel's code is otherwise placed on the device, which
// takes device memory, at its first launch).
cudaError_t load_visibility_kernels();

// Host-buffer visibility through the library's fixed staging array
// (noalloc.cu); allocates nothing.  n <= VRAD_STATIC_MAX_RAYS.
cudaError_t trace_visibility_static(const DeviceScene &scene, int device, cudaStream_t stream,
                                    const vrad_ray *h_rays, int64_t n, const TraceParams &p,
                                    uint64_t *h_bits);

// Places the fixed staging array and the kernels trace_visibility_static
// launches on `device` (current) and looks up the array's address, so that
// no later call does either.  vrad_create calls it.
cudaError_t prepare_static_trace(int device);

}  // namespace vrad
