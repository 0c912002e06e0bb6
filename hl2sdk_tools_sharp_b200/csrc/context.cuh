// context.cuh -- the opaque vrad_ctx behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ambient.cuh"
#include "bounce.cuh"
#include "bsp_trace.cuh"
#include "direct.cuh"
#include "final.cuh"
#include "host_parallel.h"
#include "patches.h"
#include "scene.cuh"
#include "staging.h"
#include "supersample.cuh"
#include "sync_wait.h"

namespace vrad {
// One range's supersampling passes in the last direct gather.
struct RangeSupersample {
    int32_t passes_run = 0;
    int64_t supersampled = 0;
    float ms = 0.0f;
};
}  // namespace vrad

struct vrad_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t join = nullptr;   // orders `stream` after work queued on callers' streams
    // When set, vrad_light_pass runs on this stream instead of `stream`
    // (a batch gives its contexts' uploads the higher priority).
    cudaStream_t pass_stream = nullptr;
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
    float4 *sample_light = nullptr;      // the direct gather's output, one per sample (LDR)
    float4 *sample_light_hdr = nullptr;  // the HDR range's, when the world has an HDR list
    vrad::RangeSupersample range_ss[2];  // the last gather's supersampling, LDR and HDR
    vrad::StyleState styles;             // light styles above 0, when the world has any
    vrad_bounce_stats range_bounce[2] = {};  // the last pass's bounce per range (zero: not lit)
    // Host copies of the uploaded world the bounce set-up reads.
    std::vector<vrad_face> h_faces;
    std::vector<float> h_vertices;
    vrad::uvector<float> h_sample_area;     // per sample
    std::vector<int2> h_face_samples;       // per face: first sample, count
    // The smoothing neighbours (FaceNeighbours, threshold 0.7071067) of
    // h_faces: face f's are h_nlist[h_noff[f] .. h_noff[f + 1]).
    std::vector<int32_t> h_noff, h_nlist;
    int32_t nclusters = 0;
    vrad::BounceBuffers bounce;
    vrad::BspBuffers bsp;            // a map's BSP tree for the surface walk (vrad_bsp_upload)
    vrad::AmbientBuffers ambient;    // its lighting for the leaf ambient sample (vrad_ambient_upload)
    // The uploaded world's patch forest, grown ahead on a host thread while
    // the rest of the world upload runs, with the chop sizes of this
    // context's last bounce upload; the next bounce upload takes it when
    // its chop sizes match.  Only a context that has bounced grows one.
    std::thread ahead_thread;
    vrad::PatchForest ahead;
    bool ahead_ok = false;
    std::string ahead_why;
    bool bounced = false;
    float last_max_chop = 0.0f, last_min_chop = 0.0f;
    // The light pass's first step queued ahead: at the end of a world
    // upload a host thread runs the direct gather with its supersampling
    // passes into sample_light on ahead_stream (the pass stream when there
    // is one), so that it overlaps the bounce upload's host work.  The next
    // vrad_light_pass takes it; every other call that reads or changes what
    // it depends on first waits for it and drops it.
    std::thread direct_thread;
    cudaStream_t ahead_stream = nullptr;
    cudaEvent_t ahead_start = nullptr;  // recorded before and after the gather queued ahead
    cudaEvent_t ahead_done = nullptr;
    bool direct_ahead = false;
    int32_t direct_ahead_rc = 0;
    int32_t ahead_ranges = 0;           // the ranges the gather queued ahead lights
    const vrad_mlp *bounce_model = nullptr;  // the warm start's network, or none
    vrad::SupersampleBuffers supersample;
    std::string supersample_why;     // why the world's samples cannot be supersampled
    vrad::Stager stager;             // pinned staging of the uploads' tables
    vrad::PinnedShelf shelf;         // pinned tables the bounce upload writes in place
    std::string last_error;
    std::string identity;
};


// The direct gather with its supersampling passes into d_out (direct.cu).
namespace vrad {
int32_t direct_pass(vrad_ctx *ctx, float4 *ldr_out, float4 *hdr_out, cudaStream_t s);

// After an entry point queued this context's kernels on a caller's stream
// s: the context's own stream waits for them, so that waiting for the
// context's stream waits for every kernel of the context.  Work captured
// into a caller's graph is not tracked (the caller waits for its graph).
inline cudaError_t join_stream(vrad_ctx *ctx, cudaStream_t s) {
    if (s == ctx->stream) return cudaSuccess;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess || cap != cudaStreamCaptureStatusNone) return e;
    e = cudaEventRecord(ctx->join, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->join, 0);
    return e;
}

// Recreates the context's stream at the device's greatest priority and
// gives its light passes their own stream at the least: on a device shared
// by several contexts, an upload's short kernels then take SMs ahead of the
// long kernels of other contexts' passes (abi.cu).
cudaError_t prioritise_uploads(vrad_ctx *ctx);

// Hands every device table of the context back to the device pool (scene,
// world, final pass, bounce, supersampling), once its kernels are done; the
// pinned host buffers stay.  A batch worker calls it after each map, so an
// idle worker holds no device memory that another worker's map could use.
cudaError_t release_tables(vrad_ctx *ctx);

// Queues the direct gather ahead (direct.cu); nothing when the world is
// not ready for a light pass.
void start_direct_ahead(vrad_ctx *ctx);

// Waits for the direct gather queued ahead, if one was, and drops it.
// Returns whether it completed without error: the caller may then take its
// sample_light (after ahead_done) instead of gathering again.
inline bool settle_direct(vrad_ctx *ctx) {
    if (ctx->direct_thread.joinable()) ctx->direct_thread.join();
    const bool ok = ctx->direct_ahead && ctx->direct_ahead_rc == 0;
    ctx->direct_ahead = false;
    return ok;
}

// Waits for the patch forest growing ahead, if one is.
inline void join_ahead(vrad_ctx *ctx) {
    if (ctx->ahead_thread.joinable()) ctx->ahead_thread.join();
}

// Waits for every kernel of this context (its streams, the first joined by
// the callers' streams it ran on) and for no other context's: an upload
// that hands the old tables back to the device pool waits here, so
// contexts on one device run their passes side by side.  A direct gather
// queued ahead must be settled first (settle_direct), so that its thread
// queues nothing more.
inline cudaError_t quiesce(vrad_ctx *ctx) {
    cudaError_t e = vrad::wait_stream(ctx->stream);
    if (e == cudaSuccess && ctx->ahead_stream) e = vrad::wait_stream(ctx->ahead_stream);
    if (e == cudaSuccess && ctx->pass_stream) e = vrad::wait_stream(ctx->pass_stream);
    return e;
}
}

// Shared error reporting (abi.cu).
int32_t vrad_fail(vrad_ctx *ctx, int32_t code, const char *fmt, ...);
int32_t vrad_cuda_fail(vrad_ctx *ctx, cudaError_t e, const char *what);
