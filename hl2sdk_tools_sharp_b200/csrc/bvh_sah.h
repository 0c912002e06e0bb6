// bvh_sah.h -- the scene BVH's topology, built on the host by the surface
// area heuristic over the triangles' padded boxes (bvh_sah.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace vrad {

struct SahTree {
    std::vector<float4> nodes;   // 4 per inner node, the walk's two-child layout; the root at 0
    std::vector<int32_t> order;  // leaf slot k holds triangle order[k]
    int32_t inner = 0;           // inner nodes
    int32_t leaves = 0;
    int32_t max_leaf = 0;        // triangles in the largest leaf
    int32_t depth = 0;           // inner nodes on the longest root-to-leaf path
    double sah_cost = 0.0;       // expected cost per ray: (node visits + triangle tests) weighted by area
};

// n >= 2 triangles, box[6 i .. 6 i + 5] = triangle i's padded box (lo xyz,
// hi xyz).  The root is always an inner node; leaves hold at most kMaxLeaf
// triangles; the depth stays within kStackDepth (ranges that would go
// deeper are split at their median).
// parallel: the subtrees below the top few splits are built on the host's
// threads; the tree is the same either way.
void build_sah(const float *box, int32_t n, SahTree &out, bool parallel = true);

}  // namespace vrad
