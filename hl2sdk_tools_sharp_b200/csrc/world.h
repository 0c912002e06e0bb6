// world.h -- host-side set-up helpers shared between world.cpp and the
// CUDA files (face luxel frames, neighbour candidate boxes).
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/vrad_cuda.h"
#include "host_parallel.h"

namespace vrad {

// FaceLightInfo's luxel frame (FaceLightInfo.cs:79-160).
struct FaceFrameOut {
    float origin[3];
    float w2l_s[3], w2l_t[3];
    float l2w_s[3], l2w_t[3];
    int32_t min_s, min_t, width, height;
};

void face_frame_of(const vrad_face &f, FaceFrameOut &out);

// LuxelToWorld / WorldToLuxel in the reference's float order.
void frame_luxel_to_world(const FaceFrameOut &fr, float s, float t, float out[3]);
void frame_world_to_luxel(const FaceFrameOut &fr, const float p[3], float &s, float &t);

// The cell windings (world space) of the partial samples, as
// FaceSampleBuilder keeps them for supersampling: wind holds (first point,
// count) per sample, count 0 for a sample whose cell the face covers
// whole; pts the points (xyz each).  False unless the samples the builder
// makes from these faces are exactly `given`.
bool sample_windings(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                     const vrad_sample *given, int64_t ngiven, uvector<int32_t> &wind, uvector<float> &pts);

// The welded vertex numbers of each face's winding (vertices identified by
// position) and, per vertex, the faces touching it in face order.  False
// when a face's winding lies outside the vertex array.
bool weld_faces(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                std::vector<std::vector<int32_t>> &face_verts, std::vector<std::vector<int32_t>> &vertex_face);

// FaceNeighbours.Build's corner normals (FaceNeighbours.cs:230-340, rule 2):
// per face, per winding vertex (xyz each), the normalised sum of the
// smoothing neighbours' normals and the face's own.
bool corner_normals(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                    float smoothing_threshold, std::vector<std::vector<float>> &out);

}  // namespace vrad
