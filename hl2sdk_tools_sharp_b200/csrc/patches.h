// patches.h -- the bounce's patch tree, built on the host (patches.cpp)
// and read by the device set-up (bounce.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vrad_cuda.h"
#include "host_parallel.h"

namespace vrad {

// The tree's shape by face.  Patches are numbered as the reference numbers
// them: the roots 0 .. roots - 1 in face order, then each root's
// descendants in creation order.
struct PatchTree {
    std::vector<int32_t> face_root;    // per face: its root patch, -1 for none
    std::vector<int32_t> face_first;   // per face: its descendants are [face_first, face_end)
    std::vector<int32_t> face_end;
    int32_t roots = 0;
    int32_t npatches = 0;
    int64_t npoints = 0;
};

// Receives the patches in their final numbering: prepare() once with the
// counts, then put() for every patch from several threads at once (each
// index once; p.first_point and p.num_points give its winding's place in
// the flat point array, xyz its points, three floats each).
struct PatchSink {
    virtual ~PatchSink() = default;
    virtual bool prepare(int32_t npatches, int64_t npoints) = 0;
    virtual void put(int32_t index, const vrad_patch &p, const float *xyz) = 0;
};

// The patches as one array and the windings as one point array.
struct PatchArrays : PatchSink {
    uvector<vrad_patch> patches;
    uvector<float> points;  // xyz each
    bool prepare(int32_t npatches, int64_t npoints) override {
        patches.resize((size_t)npatches);
        points.resize(3 * (size_t)npoints);
        return true;
    }
    void put(int32_t index, const vrad_patch &p, const float *xyz) override {
        patches[(size_t)index] = p;
        for (int32_t k = 0; k < 3 * p.num_points; k++) points[3 * (size_t)p.first_point + (size_t)k] = xyz[k];
    }
};

bool build_patch_tree(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                      const float *reflectivity, float max_chop, float min_chop, PatchTree &out, PatchSink &sink,
                      std::string &why);

}  // namespace vrad
