// supersample.cuh -- the direct gather's supersampling passes, resident on
// one device (supersample.cu).
//
// Layout in HBM (S samples, K selected in a pass, G four-lane row groups):
//   origin_st[S]   float2  the sample's position in its face's luxel space
//   cell[S]        int32   the sample's radial cell (final-pass numbering)
//   wind[S]        int2    (first point, count) of a partial sample's cell
//                          winding in points[] (world space); count 0 for a
//                          whole cell
//   intensity[S]   float   the perceptual intensity the gradient compares
//   processed[S]   u8      supersampled already (never again)
//   selected[K]    int32   this pass's samples
//   rows[G]        int32   per row group: selected index * 5 + row (row 0
//                          the ambient 2x2, rows 1-4 the direct 4x4), or -1
//                          for a padding group; groups run cluster by
//                          cluster, ambient rows then direct rows, each run
//                          padded to whole warps so a warp has one light list
//   row_out[K*20]  float4  each lane's LightingValue
//   row_bits[K*5]  int32   each row's invalid-lane bits, -1 for a row whose
//                          four points all lie outside the cell winding
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "direct.cuh"
#include "final.cuh"
#include "host_parallel.h"
#include "scene.cuh"
#include "world.h"

namespace vrad {

struct SupersampleBuffers {
    float2 *origin_st = nullptr;
    int32_t *cell = nullptr;
    int2 *wind = nullptr;
    float4 *points = nullptr;
    float *intensity = nullptr;
    uint8_t *processed = nullptr;
    int32_t *selected = nullptr;
    int32_t *counts = nullptr;      // [0] selected, [1 + c] selected in cluster c, then placement cursors
    int32_t *base = nullptr;        // 2C + 1: group offsets of each cluster's ambient then direct runs
    int32_t *rows = nullptr;        // group capacity: 5 * S + 16 * C
    float4 *row_out = nullptr;
    int32_t *row_bits = nullptr;
    int32_t *h_counts = nullptr;    // pinned, kept across uploads (h_counts_cap entries)
    size_t h_counts_cap = 0;
    int64_t nsamples = 0;
    int32_t nclusters = 0;
    int32_t extra_passes = 4;       // DirectLightingSettings.ExtraPasses; 0 = -noextra
    bool ready = false;             // the partial samples' windings are known
    // Statistics of the last run.
    int64_t supersampled = 0;
    int32_t passes_run = 0;
    float ms = 0.0f;

    void release();      // the device tables; the pinned counts stay
    void free_pinned();  // the pinned counts
};

// Builds the tables from the uploaded world (host copies of its faces,
// vertices and samples) and the final pass's cell numbering.  `why` is set
// and false returned when the samples are not the builder's own (their
// windings cannot be known).
// area_coord: each sample's area and coord (x, y, z), which the rebuilt
// samples must match (pinned host memory, nsamples entries).
cudaError_t build_supersample(SupersampleBuffers &ss, const std::vector<vrad_face> &faces,
                              const std::vector<float> &vertices, const float4 *area_coord, int64_t nsamples,
                              const FinalBuffers &fb, int32_t nclusters, Stager &stager, cudaStream_t stream,
                              bool &have, std::string &why);

// The partial cells' windings, the samples' luxel origins and cells,
// rebuilt on the device from the faces' row strips (windings.cu) into
// ss.wind, ss.points, ss.cell and ss.origin_st; match = the world's
// samples are the builder's own (else `why`).  Synchronises `stream`.
cudaError_t device_windings(SupersampleBuffers &ss, const RowStrips &rs, const FinalView &fv,
                            const float4 *check, int64_t nsamples, Stager &stager, cudaStream_t stream, bool &match,
                            std::string &why);

// The supersampling passes over `light` (the direct gather's output, one
// float4 per sample), on `stream`.  Blocks once per pass.
cudaError_t run_supersample(SupersampleBuffers &ss, const DeviceScene &scene, const DeviceWorld &world,
                            const FinalView &fv, float4 *light, unsigned long long *counters, uint32_t *overflow,
                            cudaStream_t stream);

}  // namespace vrad
