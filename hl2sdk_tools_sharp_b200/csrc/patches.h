// patches.h -- the bounce's patch tree, built on the host (patches.cpp)
// and read by the device set-up (bounce.cu).
#pragma once

#include <cstdint>
#include <memory>
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

// The first half of the patch tree: every face's root and its subdivided
// subtree (PatchBuilder.Build, PatchSubdivider.Subdivide), before the
// patches are numbered and given their reflectivity.  It reads only the
// faces, their windings and the chop sizes, which the world upload already
// has, so a context can grow it ahead of the bounce upload.  The faces and
// vertices must outlive the forest.
class PatchForest {
public:
    PatchForest();
    ~PatchForest();
    PatchForest(PatchForest &&) noexcept;
    PatchForest &operator=(PatchForest &&) noexcept;

    bool grow(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices, float max_chop,
              float min_chop, std::string &why);
    // The patches numbered as the reference numbers them, each with its
    // face's reflectivity (nfaces x 3, clamped to 0.99), handed to the sink.
    bool merge(const float *reflectivity, PatchTree &out, PatchSink &sink, std::string &why);

    bool grown() const;
    float max_chop() const;
    float min_chop() const;

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// grow, then merge.
bool build_patch_tree(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                      const float *reflectivity, float max_chop, float min_chop, PatchTree &out, PatchSink &sink,
                      std::string &why);

}  // namespace vrad
