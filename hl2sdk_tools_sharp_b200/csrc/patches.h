// patches.h -- the bounce's patch tree, built on the host (patches.cpp)
// and read by the device set-up (bounce.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vrad_cuda.h"
#include "host_parallel.h"

namespace vrad {

struct PatchTree {
    uvector<vrad_patch> patches;       // the reference's patch indices
    uvector<float> points;             // windings, xyz each (vrad_patch.first_point)
    std::vector<int32_t> face_root;    // per face: its root patch, -1 for none
    std::vector<int32_t> face_first;   // per face: its descendants are [face_first, face_end)
    std::vector<int32_t> face_end;
    int32_t roots = 0;
};

bool build_patch_tree(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                      const float *reflectivity, float max_chop, float min_chop, PatchTree &out, std::string &why);

}  // namespace vrad
