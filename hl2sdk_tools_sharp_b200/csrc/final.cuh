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
#include "staging.h"

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
    // The pass's light style: each face's slot for it (-1: not the face's
    // style, the face is skipped and its samples reach no neighbour); null:
    // style 0, slot 0 on every face.
    const int8_t *style_slot;
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
    std::vector<float4> h_frames;   // host copy of frames (its lightofs words change with the styles)
    FinalView view{};
    bool ready = false;

    void release();
};

// run_first / run_end (nullable, per face): each face's sample run as the
// caller already found it (-1 for a face without samples); otherwise the
// runs are found here.
cudaError_t build_final(FinalBuffers &fb, const vrad_face *faces, int32_t nfaces, const vrad_sample *samples,
                        int64_t nsamples, const float *vertices, int64_t nvertices, std::vector<int32_t> &noff,
                        std::vector<int32_t> &nlist, Stager &stager, cudaStream_t stream, std::string &why,
                        const int64_t *run_first = nullptr, const int64_t *run_end = nullptr);

// The bounced light's radial grid (FinalLightFace.BuildPatchRadial): per
// face, the leaf patches of the face and of its smoothing neighbours whose
// radial box reaches it, in the reference's order, with the box and the
// patch's luxel-space centre and extent; the patches' bounced light; and
// the per-cell accumulators.
struct PatchRadialView {
    const int32_t *off;      // F + 1
    const int32_t *patch;
    const int4 *box;         // sMin, tMin, sMax, tMax (clamped to the face)
    const float4 *coord;     // coordS, coordT, distS, distT
    const float4 *light;     // TotalLight.Flat per patch
    float4 *rad_light;       // per cell
    float *rad_weight;
};

// prad = nullptr: no bounce (-bounce 0).
cudaError_t launch_final(const FinalView &v, const float4 *sample_light, float4 *rad_light, float *rad_weight,
                         float4 *flat, uint8_t *lighting, int nfaces, const PatchRadialView *prad,
                         cudaStream_t stream);

}  // namespace vrad
