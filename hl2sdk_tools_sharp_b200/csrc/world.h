// world.h -- host-side set-up helpers shared between world.cpp and the
// CUDA files (face luxel frames, neighbour candidate boxes).
#pragma once

#include <cstdint>
#include <string>
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

// BuildFacesamples' row strips of every face, for the cell clipping on the
// device (windings.cu): row k is face[k]'s strip t[k], the luxel-space
// winding's part between t and t + 1 as the builder cuts it, its points
// (luxel x, y; z is 0) at xy[2 first[k] ..] (first[nrows] = the point
// count); apl = each face's world area per luxel.  Rows the builder leaves
// empty are left out.  False, with `why`, when a face's winding lies
// outside the vertex array or has more than kStripMax points.
constexpr int kStripMax = 56;
struct RowStrips {
    std::vector<int32_t> face, t;
    std::vector<int64_t> first;
    uvector<float> xy;
    std::vector<float> apl;
};
bool face_row_strips(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices, RowStrips &out,
                     std::string &why);

// FaceNeighbours.Build's smoothing neighbours: face f's are
// list[off[f] .. off[f + 1]), in the reference's order.  VRAD_ERR_ARG for
// a winding outside the vertex array or more than 64 neighbours.
int32_t face_neighbours(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                        float smoothing_threshold, std::vector<int32_t> &off, std::vector<int32_t> &list);

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
