// context.cuh -- the opaque vrad_ctx behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "bounce.cuh"
#include "direct.cuh"
#include "final.cuh"
#include "host_parallel.h"
#include "scene.cuh"
#include "staging.h"
#include "supersample.cuh"

struct vrad_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    vrad::SceneBuffers scene;
    vrad::SceneBuildReport report;
    bool has_scene = false;
    uint32_t *status = nullptr;   // [0] traversal stack overflow flag (sticky)
    // Staging for the host-buffer entry points, grown on demand.
    void *d_rays = nullptr;
    size_t d_rays_cap = 0;
    void *d_out = nullptr;
    size_t d_out_cap = 0;
    vrad::WorldBuffers world;
    vrad::FinalBuffers final_pass;
    float4 *sample_light = nullptr;  // the direct gather's output, one per sample
    // Host copies of the uploaded world the bounce set-up reads.
    std::vector<vrad_face> h_faces;
    std::vector<float> h_vertices;
    vrad::uvector<vrad_sample> h_samples;
    // The smoothing neighbours (FaceNeighbours, threshold 0.7071067) of
    // h_faces: face f's are h_nlist[h_noff[f] .. h_noff[f + 1]).
    std::vector<int32_t> h_noff, h_nlist;
    int32_t nclusters = 0;
    vrad::BounceBuffers bounce;
    const vrad_mlp *bounce_model = nullptr;  // the warm start's network, or none
    vrad::SupersampleBuffers supersample;
    std::string supersample_why;     // why the world's samples cannot be supersampled
    vrad::Stager stager;             // pinned staging of the uploads' tables
    std::string last_error;
    std::string identity;
};


// The direct gather with its supersampling passes into d_out (direct.cu).
namespace vrad {
int32_t direct_pass(vrad_ctx *ctx, float4 *d_out, cudaStream_t s);
}

// Shared error reporting (abi.cu).
int32_t vrad_fail(vrad_ctx *ctx, int32_t code, const char *fmt, ...);
int32_t vrad_cuda_fail(vrad_ctx *ctx, cudaError_t e, const char *what);
