// bounce_host.h -- the bounce's host entry points the light pass calls
// (bounce_abi.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "final.cuh"

struct vrad_ctx;

namespace vrad {

// Whether the uploaded world bounces (vrad_bounce_upload with bounces > 0).
bool bounce_active(const vrad_ctx *ctx);

// The bounce of a light pass on stream s, after the direct gather.
cudaError_t run_bounce(vrad_ctx *ctx, cudaStream_t s, std::string &why);

// The final pass's view of the bounced light.
PatchRadialView patch_radial_view(vrad_ctx *ctx);

}  // namespace vrad
