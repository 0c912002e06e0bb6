// vrad_internal.cuh -- device-side layout shared by the scene build and the
// traversal kernels of libvrad_cuda.
//
// Scene layout in HBM.  The triangles are split by the sky bit of their id
// into two BVHs, opaque and sky, each laid out as below (structure of
// arrays, every record 16-byte aligned so each is one or more 128-bit
// loads); tri_id is shared and indexed by the original triangle index.
//
//   tri0[i]  float4 (nx, ny, nz, d)          plane of the i-th triangle in
//   tri1[i]  float4 (e0, e1, e2, e3)         BVH leaf order: the reference's
//   tri2[i]  float4 (e4, e5, idx, meta)      KdTriangle, 48 B
//            idx  = original triangle index (int bits), the tie-break key
//            meta = drop axis (bits 0-1) | sky (bit 2) | FCACHETRI flags << 8
//   tri_id[orig]  int  the caller's id, read only for skip_id and outputs
//
//   node[k]  4 x float4 = 64 B, two child boxes and two child references:
//            n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//            n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//            n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//            n3 = (ref0, ref1, -, -)
//            ref >= 0 is an inner node; ref < 0 is a leaf, ~ref packing
//            (first triangle << 3) | (count - 1), so a leaf holds 1..8.
#pragma once

#include <cstdint>

#include "../../include/vrad_cuda.h"

namespace vrad {

constexpr int kMaxLeaf = 8;
constexpr int kStackDepth = 64;
constexpr uint32_t kTraceIdSky = 0x01000000u;   // TraceId.Sky (MapTools/Rad/TraceId.cs)
constexpr float kKdEps = 1.0e-10f;              // KdRayTracer.cs:1209-1230
constexpr float kKdHuge = 1.0e23f;              // KdRayTracer.cs:985

struct DeviceBvh {
    const float4 *tri0;
    const float4 *tri1;
    const float4 *tri2;
    const float4 *nodes;
    int32_t ntris;  // 0: empty, never traversed
    int32_t depth;  // stack entries a walk can need: the tree's depth in inner nodes
};

struct DeviceScene {
    DeviceBvh opaque;
    DeviceBvh sky;
    const int32_t *tri_id;
    // The traversal stack's entries per thread (kernels size their shared
    // memory by it): the deeper tree's depth, at least 1, at most kStackDepth.
    __host__ __device__ int32_t stack_depth() const {
        const int32_t d = opaque.depth > sky.depth ? opaque.depth : sky.depth;
        return d < 1 ? 1 : (d > kStackDepth ? kStackDepth : d);
    }
};

enum TraceMode : int { kModeAny = 0, kModeClosest = 1, kModeSkyPass = 2 };

struct TraceParams {
    float tmin;
    int32_t skip_id;
    int32_t mode;
};

__host__ __device__ inline int32_t leaf_ref(int32_t first, int32_t count) {
    return ~((first << 3) | (count - 1));
}

}  // namespace vrad
