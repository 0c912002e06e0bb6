// scene.cuh -- device-resident scene of one context, and its GPU build.
#pragma once

#include <cuda_runtime.h>

#include "vrad_internal.cuh"

namespace vrad {

struct SceneBuffers {
    float4 *tri0 = nullptr;
    float4 *tri1 = nullptr;
    float4 *tri2 = nullptr;
    int32_t *tri_id = nullptr;
    float4 *nodes = nullptr;
    int32_t ntris = 0;
    int32_t root_ref = 0;

    void release();
    DeviceScene view() const { return DeviceScene{tri0, tri1, tri2, tri_id, nodes, root_ref, ntris}; }
};

struct SceneBuildReport {
    int32_t nodes = 0;
    int32_t leaves = 0;
    int32_t max_leaf = 0;
    float bounds[6] = {0, 0, 0, 0, 0, 0};
    float pad = 0;
    float build_ms = 0;
    int64_t device_bytes = 0;
};

// Builds `sb` from n host triangles (and, optionally, their intersection
// form).  Synchronises `stream` before returning.
cudaError_t build_scene(SceneBuffers &sb, const vrad_triangle *h_tris,
                        const vrad_kd_triangle *h_prepared, int n, cudaStream_t stream,
                        SceneBuildReport *report);

// Traversal launches (trace.cu).  d_bits is written as 32-bit words.
cudaError_t launch_trace(const DeviceScene &scene, const vrad_ray *d_rays, int64_t n,
                         const TraceParams &p, uint32_t *d_bits, vrad_hit *d_hits,
                         uint32_t *d_overflow, cudaStream_t stream);

}  // namespace vrad
