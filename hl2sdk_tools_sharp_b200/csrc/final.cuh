// final.cuh -- device tables of the final pass (final.cu).
//
//   frames[5f..5f+4]  float4: (luxel origin, width) (world->luxel s, height)
//                     (world->luxel t, min s) (luxel->world s, min t)
//                     (luxel->world t, lightofs); ints as bits
//   face_cells[f]     first radial cell / luxel of face f (cells = luxels,
//                     row-major, width = lightmap size + 1)
//   cell_face, cell_sample   per cell: its face; the sample whose lightmap
//                     cell it is, or -1
//   sample_box[k]     (MinS, MinT, MaxS, MaxT) in its own face's luxel space
//   cand_*            per face, the neighbours' samples that can reach it,
//                     in neighbour order then sample order, their boxes
//                     moved into this face's luxel space
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vrad_cuda.h"

namespace vrad {

struct FinalView {
    const float4 *frames;
    const int32_t *face_cells;
    const int32_t *face_nsamples;
    const int32_t *cell_face;
    const int32_t *cell_sample;
    const float4 *sample_pos;
    const float4 *sample_box;
    const int32_t *cand_off;
    const int32_t *cand_sample;
    const float4 *cand_box;
    int64_t ncells;
};

struct FinalBuffers {
    float4 *frames = nullptr;
    int32_t *face_cells = nullptr;
    int32_t *face_nsamples = nullptr;
    int32_t *cell_face = nullptr;
    int32_t *cell_sample = nullptr;
    float4 *sample_box = nullptr;
    int32_t *cand_off = nullptr;
    int32_t *cand_sample = nullptr;
    float4 *cand_box = nullptr;
    float4 *rad_light = nullptr;
    float *rad_weight = nullptr;
    float4 *flat = nullptr;
    int64_t lighting_bytes = 0;
    int32_t nfaces = 0;
    std::vector<int32_t> lightofs;
    FinalView view{};
    bool ready = false;

    void release();
};

cudaError_t build_final(FinalBuffers &fb, const vrad_face *faces, int32_t nfaces, const vrad_sample *samples,
                        int64_t nsamples, const float *vertices, int64_t nvertices, std::string &why);

cudaError_t launch_final(const FinalView &v, const float4 *sample_light, float4 *rad_light, float *rad_weight,
                         float4 *flat, uint8_t *lighting, int nfaces, cudaStream_t stream);

}  // namespace vrad
