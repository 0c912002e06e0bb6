// bounce_host.h -- the bounce's host entry points the light pass calls
// (bounce_abi.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "final.cuh"
#include "vrad_cuda.h"

struct vrad_ctx;

namespace vrad {

// Whether the uploaded world bounces (vrad_bounce_upload with bounces > 0).
bool bounce_active(const vrad_ctx *ctx);

// The bounce of a light pass on stream s, after the direct gather wrote
// sample_light (the range's).  build_transfers false reuses the transfers
// the previous range of the same pass built (they are geometry).
cudaError_t run_bounce(vrad_ctx *ctx, cudaStream_t s, const float4 *sample_light, bool build_transfers,
                       std::string &why);

// The statistics of the bounce that ran last.
void fill_bounce_stats(const vrad_ctx *ctx, vrad_bounce_stats *st);

// The final pass's view of the bounced light.
PatchRadialView patch_radial_view(vrad_ctx *ctx);

}  // namespace vrad
