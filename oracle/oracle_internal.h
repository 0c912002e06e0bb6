// oracle_internal.h -- C++ helpers shared between the oracle's files.
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).
#pragma once

#include "vrad_oracle.h"

struct OrcKd {
    const orc_kdnode *nodes;
    const int32_t *indices;
    const orc_tri *tris;
    float bounds[6];
};

bool orc_kd_segment_blocked(const OrcKd &kd, const orc_ray &r, bool sky_pass);

#include <vector>

// A leaf patch as the final pass's bounced radial reads it
// (FinalLightFace.AddFacePatches): winding (xyz each), origin, TotalLight.
struct OrcBouncedPatch {
    std::vector<float> winding;
    float origin[3];
    float light[3];
};

// Per face, its leaf patches in FacePatches order.
struct OrcBounced {
    std::vector<std::vector<OrcBouncedPatch>> face_leaves;
};

// FinalLightFace over every face; bounced = nullptr for -bounce 0.
int orc_final_impl(const orc_face *faces, int32_t nfaces, const float *verts, const orc_sample *samples,
                   const int64_t *face_first, const float *sample_light, uint8_t *lighting, int64_t capacity,
                   int32_t *lightofs, int64_t *total, const OrcBounced *bounced,
                   const float *slots_light = nullptr, const uint8_t *face_styles = nullptr);
