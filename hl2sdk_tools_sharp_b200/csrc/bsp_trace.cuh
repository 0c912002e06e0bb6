// bsp_trace.cuh -- a map's own BSP tree resident on the device, for the
// BSP surface walk (bsp_trace.cu).
//
// Layout in HBM (the arrays BspTraceGeometry.Build makes, one to one):
//   nodes[n]       2 x float4: (plane normal, dist), (child0, child1, first
//                  node face, packed) -- the last four as int bits; packed =
//                  lit face count | sky face count << 15 | axis << 30
//   surfaces[f]    4 x float4: (plane normal, dist), (lightmap s, offset),
//                  (lightmap t, offset), (mins s, t, sizes s, t)
//   node_faces     each node's candidate faces, lit then sky
//   leaf_faces     each leaf's candidate faces; leaf_run[l] = (start, count)
//   sky_points     the sky faces' windings (float4); sky_run[f] = (start, count)
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vrad {

struct DeviceBsp {
    const float4 *nodes;
    const float4 *surfaces;
    const int32_t *node_faces;
    const int32_t *leaf_faces;
    const int2 *leaf_run;
    int32_t nleaves;
    const float4 *sky_points;
    const int2 *sky_run;
};

struct BspBuffers {
    float4 *nodes = nullptr;
    float4 *surfaces = nullptr;
    int32_t *node_faces = nullptr;
    int32_t *leaf_faces = nullptr;
    int2 *leaf_run = nullptr;
    float4 *sky_points = nullptr;
    int2 *sky_run = nullptr;
    int32_t nnodes = 0, nsurfaces = 0, nleaves = 0;
    bool ready = false;
    DeviceBsp view{};

    void release();
};

}  // namespace vrad
