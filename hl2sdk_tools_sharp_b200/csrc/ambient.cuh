// ambient.cuh -- what the leaf ambient sample reads besides the BSP tree:
// the map's lighting lump and each face's lookup record, resident on the
// device (vrad_ambient_upload).
//
// Layout in HBM:
//   light[b]        the lighting lump's bytes, unchanged (RGBE luxels,
//                   each face's style averages just before its lightmap)
//   faces[f]        vrad_ambient_face, one per BSP face (the BSP tree's
//                   surface order): lightmap offset, size, style slots,
//                   sky flag, reflectivity, decoded tinted averages
//   directions[i]   the 162 sample directions, float x 3
//   power2n[k]      (float)(2^(k - 128) / 255), the RGBE decode table
//   rad             scratch: each sample's 162 ray colours (float x 3),
//                   for the samples of one chunk
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "vrad_cuda.h"

namespace vrad {

constexpr int kAmbientDirs = 162;
constexpr int kAmbientSides = 6;

struct AmbientView {
    const uint8_t *light;
    int64_t light_bytes;
    const vrad_ambient_face *faces;
    int32_t nfaces;
    const float *directions;
    const float *power2n;
    float tan_theta;
    int32_t has_sky;
    float sky[3];
};

struct AmbientBuffers {
    uint8_t *light = nullptr;
    vrad_ambient_face *faces = nullptr;
    float *directions = nullptr;
    float *power2n = nullptr;
    float *rad = nullptr;          // chunk x 162 x 3
    int64_t rad_samples = 0;       // samples the scratch holds
    uint32_t *flags = nullptr;     // sticky error bits of the last cubes call
    bool ready = false;
    AmbientView view{};

    void release();
};

}  // namespace vrad
