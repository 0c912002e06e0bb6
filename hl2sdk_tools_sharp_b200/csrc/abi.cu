// abi.cu -- the C ABI of libvrad_cuda.so (include/vrad_cuda.h): contexts,
// scene upload, and the host- and device-buffer trace entry points.
//
// Reference behaviour kept at this boundary (muflub/hl2sdk_tools_sharp):
//  * a short output buffer is an argument error, as KdRayTracer's
//    ArgumentException (MapTools/Tracing/KdRayTracer.cs:671-678);
//  * options the tracer cannot honour are refused, never silently ignored
//    (IRayTracer.Supports, IRayTracer.cs:183-206; VulkanRayTracer
//    RequireSupported, MapTools.Gpu/VulkanRayTracer.cs:971-990);
//  * sky pass-through applies to visibility only; a closest-hit call asking
//    for it is an argument error (KdRayTracer.TraceClosest,
//    KdRayTracer.cs:456-462);
//  * there is no CPU fallback: a device failure is a status code.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "context.cuh"
#include "device_pool.h"
#include "sync_wait.h"

namespace {

std::mutex g_err_mu;
std::string g_last_error;

int32_t fail(vrad_ctx *ctx, int32_t code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) {
        ctx->last_error = buf;
    } else {
        std::lock_guard<std::mutex> g(g_err_mu);
        g_last_error = buf;
    }
    return code;
}

int32_t cuda_fail(vrad_ctx *ctx, cudaError_t e, const char *what) {
    int32_t code = (e == cudaErrorMemoryAllocation) ? VRAD_ERR_OOM : VRAD_ERR_CUDA;
    return fail(ctx, code, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

bool options_ok(const vrad_trace_options *o) {
    return o == nullptr || (o->min_distance >= 0.0f);  // false for NaN too
}

vrad::TraceParams params_of(const vrad_trace_options *o, int mode) {
    vrad::TraceParams p;
    p.tmin = o ? o->min_distance : 0.0f;
    p.skip_id = o ? o->skip_id : -1;
    p.mode = mode;
    if (p.skip_id < -1) p.skip_id = -1;  // any negative id means none, as stock's -1
    return p;
}

cudaError_t ensure(void **buf, size_t *cap, size_t need) {
    if (*cap >= need) return cudaSuccess;
    cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
    size_t grow = need + need / 4;
    cudaError_t e = cudaMalloc(buf, grow);
    if (e == cudaSuccess) *cap = grow;
    return e;
}

int32_t check_overflow(vrad_ctx *ctx) {
    uint32_t flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, ctx->status, sizeof flag, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "reading the traversal status");
    if (flag) {
        cudaMemsetAsync(ctx->status, 0, sizeof(uint32_t), ctx->stream);
        return fail(ctx, VRAD_ERR_CUDA, "traversal stack overflow (BVH deeper than %d)",
                    vrad::kStackDepth);
    }
    return VRAD_OK;
}

int32_t upload(vrad_ctx *ctx, const vrad_triangle *tris, const vrad_kd_triangle *prep, int32_t n) {
    if (!ctx) return fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n <= 0 || !tris)
        return fail(ctx, VRAD_ERR_ARG,
                    "a scene needs at least one triangle (the reference refuses an empty KD build)");
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    ctx->has_scene = false;
    vrad::settle_direct(ctx);
    // The old scene's blocks go back to the device pool once no kernel of
    // this context reads them.
    e = vrad::quiesce(ctx);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "waiting for the context's kernels");
    ctx->scene.release();
    ctx->report = vrad::SceneBuildReport();
    // Split by the id's sky bit (TraceId.Sky): two BVHs, so a sky test can
    // find the nearest sky hit in the small one and then ask the large one
    // only whether anything opaque lies before it.
    std::vector<vrad_triangle> part[2];
    std::vector<vrad_kd_triangle> ppart[2];
    std::vector<int32_t> orig[2];
    std::vector<int32_t> ids((size_t)n);
    for (int32_t i = 0; i < n; i++) {
        const int32_t id = prep ? prep[i].id : tris[i].id;
        const int k = ((uint32_t)id & vrad::kTraceIdSky) ? 1 : 0;
        ids[(size_t)i] = id;
        part[k].push_back(tris[i]);
        if (prep) ppart[k].push_back(prep[i]);
        orig[k].push_back(i);
    }
    e = vrad::dev_alloc(&ctx->scene.tri_id, sizeof(int32_t) * (size_t)n);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->scene.tri_id, ids.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e != cudaSuccess) {
        ctx->scene.release();
        return cuda_fail(ctx, e, "scene ids");
    }
    ctx->scene.ntris = n;
    vrad::BvhBuffers *dst[2] = {&ctx->scene.opaque, &ctx->scene.sky};
    for (int k = 0; k < 2; k++) {
        e = vrad::build_bvh(*dst[k], part[k].data(), prep ? ppart[k].data() : nullptr, orig[k].data(),
                            (int)part[k].size(), ctx->stream, &ctx->report);
        if (e != cudaSuccess) {
            ctx->scene.release();
            if (e == cudaErrorInvalidValue && prep)
                return fail(ctx, VRAD_ERR_ARG,
                            "a supplied triangle's projection axes are not the successors of its drop axis");
            return cuda_fail(ctx, e, "scene build");
        }
    }
    ctx->report.device_bytes += (int64_t)n * 4;
    ctx->has_scene = true;
    return VRAD_OK;
}

int32_t trace_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n,
                     const vrad_trace_options *opts, uint32_t *d_bits, vrad_hit *d_hits, int mode,
                     cudaStream_t stream) {
    cudaError_t e = vrad::launch_trace(ctx->scene.view(), d_rays, n, params_of(opts, mode), d_bits,
                                       d_hits, ctx->status, stream);
    if (e == cudaSuccess) e = vrad::join_stream(ctx, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "trace launch");
    return VRAD_OK;
}

int32_t validate(vrad_ctx *ctx, const void *rays, int64_t n, const vrad_trace_options *opts,
                 const void *out) {
    if (!ctx) return fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n < 0) return fail(ctx, VRAD_ERR_ARG, "negative ray count %lld", (long long)n);
    if (n > 0 && (!rays || !out)) return fail(ctx, VRAD_ERR_ARG, "null ray or output buffer");
    if (!options_ok(opts))
        return fail(ctx, VRAD_ERR_UNSUPPORTED,
                    "minimum distance must be a non-negative number, got %g", (double)opts->min_distance);
    if (!ctx->has_scene) return fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    return VRAD_OK;
}

}  // namespace

int32_t vrad_fail(vrad_ctx *ctx, int32_t code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return fail(ctx, code, "%s", buf);
}

int32_t vrad_cuda_fail(vrad_ctx *ctx, cudaError_t e, const char *what) { return cuda_fail(ctx, e, what); }

namespace vrad {
cudaError_t prioritise_uploads(vrad_ctx *ctx) {
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    settle_direct(ctx);
    if (e == cudaSuccess) e = quiesce(ctx);
    if (e != cudaSuccess) return e;
    cudaStream_t up = nullptr, pass = nullptr;
    e = cudaStreamCreateWithPriority(&up, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&pass, cudaStreamNonBlocking, least);
    if (e != cudaSuccess) {
        if (up) cudaStreamDestroy(up);
        return e;
    }
    cudaStreamDestroy(ctx->stream);
    if (ctx->pass_stream) cudaStreamDestroy(ctx->pass_stream);
    ctx->stream = up;
    ctx->pass_stream = pass;
    return cudaSuccess;
}

cudaError_t release_tables(vrad_ctx *ctx) {
    std::lock_guard<std::mutex> g(ctx->mu);
    join_ahead(ctx);
    settle_direct(ctx);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = quiesce(ctx);
    if (e != cudaSuccess) return e;
    ctx->ahead = PatchForest();
    ctx->ahead_ok = false;
    ctx->has_scene = false;
    ctx->scene.release();
    ctx->world.release();
    ctx->styles.release();
    ctx->final_pass.release();
    ctx->bounce.release();
    ctx->supersample.release();
    ctx->bsp.release();
    ctx->ambient.release();
    vrad::dev_free(ctx->sample_light);
    ctx->sample_light = nullptr;
    vrad::dev_free(ctx->sample_light_hdr);
    ctx->sample_light_hdr = nullptr;
    return cudaSuccess;
}
}  // namespace vrad

extern "C" {

int32_t vrad_abi_version(void) { return VRAD_ABI_VERSION; }

int32_t vrad_create(int32_t device, vrad_ctx **out) {
    if (!out) return fail(nullptr, VRAD_ERR_ARG, "null output pointer");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(nullptr, VRAD_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= count)
        return fail(nullptr, VRAD_ERR_NO_DEVICE, "device %d out of range (%d present)", device, count);
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return fail(nullptr, VRAD_ERR_NO_DEVICE, "%s", cudaGetErrorString(e));
    if (prop.major != 10 || prop.minor != 0)
        return fail(nullptr, VRAD_ERR_NO_DEVICE,
                    "device %d is sm_%d%d; this library holds sm_100a code only", device, prop.major,
                    prop.minor);
    vrad_ctx *ctx = new vrad_ctx();
    ctx->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->ahead_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ahead_start);
    if (e == cudaSuccess) e = cudaEventCreate(&ctx->ahead_done);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->status, 4 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->status, 0, 4 * sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e == cudaSuccess) {
        // Places vrad_trace_visibility_static's fixed array and kernels on
        // the device now, at set-up.  A failure here is not the context's:
        // that entry point repeats the look-up and reports it.
        if (vrad::prepare_static_trace(device) != cudaSuccess) (void)cudaGetLastError();
    }
    if (e != cudaSuccess) {
        int32_t rc = cuda_fail(nullptr, e, "context setup");
        vrad_destroy(ctx);
        return rc;
    }
    char id[320];
    snprintf(id, sizeof id, "cuda-bvh-kdexact-1-%s-sm%d%d", prop.name, prop.major, prop.minor);
    for (char *c = id; *c; c++)
        if (*c == ' ') *c = '-';
    ctx->identity = id;
    *out = ctx;
    return VRAD_OK;
}

int32_t vrad_destroy(vrad_ctx *ctx) {
    if (!ctx) return VRAD_OK;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        vrad::join_ahead(ctx);
        vrad::settle_direct(ctx);
        cudaSetDevice(ctx->device);
        // Kernels of this context may run on callers' streams too.
        cudaDeviceSynchronize();
        ctx->scene.release();
        ctx->world.release();
        ctx->styles.release();
        ctx->final_pass.release();
        ctx->bounce.release();
        ctx->bounce.free_pinned();
        ctx->supersample.release();
        ctx->supersample.free_pinned();
        ctx->shelf.release();
        ctx->bsp.release();
        ctx->ambient.release();
        vrad::dev_free(ctx->sample_light);
        vrad::dev_free(ctx->sample_light_hdr);
        cudaFree(ctx->status);
        cudaFree(ctx->d_rays);
        cudaFree(ctx->d_out);
        if (ctx->join) cudaEventDestroy(ctx->join);
        if (ctx->ahead_start) cudaEventDestroy(ctx->ahead_start);
        if (ctx->ahead_done) cudaEventDestroy(ctx->ahead_done);
        if (ctx->ahead_stream) cudaStreamDestroy(ctx->ahead_stream);
        if (ctx->pass_stream) cudaStreamDestroy(ctx->pass_stream);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        vrad::dev_trim(ctx->device);
    }
    delete ctx;
    return VRAD_OK;
}

int32_t vrad_scene_upload(vrad_ctx *ctx, const vrad_triangle *tris, int32_t n) {
    return upload(ctx, tris, nullptr, n);
}

int32_t vrad_scene_upload_prepared(vrad_ctx *ctx, const vrad_triangle *tris,
                                   const vrad_kd_triangle *prepared, int32_t n) {
    if (!prepared) return fail(ctx, VRAD_ERR_ARG, "null prepared triangles");
    return upload(ctx, tris, prepared, n);
}

int32_t vrad_scene_get_info(vrad_ctx *ctx, vrad_scene_info *out) {
    if (!ctx || !out) return fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->has_scene) return fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    out->triangles = ctx->scene.ntris;
    out->bvh_nodes = ctx->report.nodes;
    out->bvh_leaves = ctx->report.leaves;
    out->max_leaf = ctx->report.max_leaf;
    out->bvh_depth = ctx->report.max_depth;
    for (int a = 0; a < 3; a++) {
        out->bounds_min[a] = ctx->report.bounds[a];
        out->bounds_max[a] = ctx->report.bounds[3 + a];
    }
    out->box_pad = ctx->report.pad;
    out->build_ms = ctx->report.build_ms;
    out->device_bytes = ctx->report.device_bytes;
    return VRAD_OK;
}

int32_t vrad_supports(const vrad_trace_options *opts) { return options_ok(opts) ? 1 : 0; }

int32_t vrad_trace_visibility(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                              const vrad_trace_options *opts, uint64_t *hit_bits) {
    int32_t rc = validate(ctx, rays, n, opts, hit_bits);
    if (rc != VRAD_OK) return rc;
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    const size_t words32 = (size_t)((n + 31) / 32);
    const size_t words64 = (size_t)((n + 63) / 64);
    if (e == cudaSuccess) e = ensure(&ctx->d_rays, &ctx->d_rays_cap, sizeof(vrad_ray) * (size_t)n);
    if (e == cudaSuccess) e = ensure(&ctx->d_out, &ctx->d_out_cap, 8 * words64);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->d_rays, rays, sizeof(vrad_ray) * (size_t)n, cudaMemcpyHostToDevice,
                            ctx->stream);
    // The last 32-bit word of an odd count belongs to no warp; clear it.
    if (e == cudaSuccess && (words32 & 1))
        e = cudaMemsetAsync((uint32_t *)ctx->d_out + words32, 0, 4, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "staging rays");
    const int mode = (opts && opts->sky_does_not_block) ? vrad::kModeSkyPass : vrad::kModeAny;
    rc = trace_device(ctx, (const vrad_ray *)ctx->d_rays, n, opts, (uint32_t *)ctx->d_out, nullptr,
                      mode, ctx->stream);
    if (rc != VRAD_OK) return rc;
    e = cudaMemcpyAsync(hit_bits, ctx->d_out, 8 * words64, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "visibility trace");
    return check_overflow(ctx);
}

int32_t vrad_trace_closest(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                           const vrad_trace_options *opts, vrad_hit *hits) {
    int32_t rc = validate(ctx, rays, n, opts, hits);
    if (rc != VRAD_OK) return rc;
    if (opts && opts->sky_does_not_block)
        return fail(ctx, VRAD_ERR_ARG,
                    "sky pass-through is a visibility option; a closest-hit trace reports the sky hit itself");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = ensure(&ctx->d_rays, &ctx->d_rays_cap, sizeof(vrad_ray) * (size_t)n);
    if (e == cudaSuccess) e = ensure(&ctx->d_out, &ctx->d_out_cap, sizeof(vrad_hit) * (size_t)n);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->d_rays, rays, sizeof(vrad_ray) * (size_t)n, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "staging rays");
    rc = trace_device(ctx, (const vrad_ray *)ctx->d_rays, n, opts, nullptr, (vrad_hit *)ctx->d_out,
                      vrad::kModeClosest, ctx->stream);
    if (rc != VRAD_OK) return rc;
    e = cudaMemcpyAsync(hits, ctx->d_out, sizeof(vrad_hit) * (size_t)n, cudaMemcpyDeviceToHost,
                        ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "closest trace");
    return check_overflow(ctx);
}

int32_t vrad_trace_visibility_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n,
                                     const vrad_trace_options *opts, uint64_t *d_hit_bits,
                                     void *stream) {
    int32_t rc = validate(ctx, d_rays, n, opts, d_hit_bits);
    if (rc != VRAD_OK) return rc;
    if (((uintptr_t)d_hit_bits & 3) != 0) return fail(ctx, VRAD_ERR_ARG, "hit bits not 4-byte aligned");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;  // NULL is the CUDA default stream
    const size_t words32 = (size_t)((n + 31) / 32);
    if (words32 & 1) {
        cudaError_t e = cudaMemsetAsync((uint32_t *)d_hit_bits + words32, 0, 4, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "clearing the last word");
    }
    const int mode = (opts && opts->sky_does_not_block) ? vrad::kModeSkyPass : vrad::kModeAny;
    return trace_device(ctx, d_rays, n, opts, (uint32_t *)d_hit_bits, nullptr, mode, s);
}

int32_t vrad_trace_closest_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n,
                                  const vrad_trace_options *opts, vrad_hit *d_hits, void *stream) {
    int32_t rc = validate(ctx, d_rays, n, opts, d_hits);
    if (rc != VRAD_OK) return rc;
    if (opts && opts->sky_does_not_block)
        return fail(ctx, VRAD_ERR_ARG,
                    "sky pass-through is a visibility option; a closest-hit trace reports the sky hit itself");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaStream_t s = (cudaStream_t)stream;  // NULL is the CUDA default stream
    return trace_device(ctx, d_rays, n, opts, nullptr, d_hits, vrad::kModeClosest, s);
}

int32_t vrad_trace_visibility_static(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                                     const vrad_trace_options *opts, uint64_t *hit_bits) {
    int32_t rc = validate(ctx, rays, n, opts, hit_bits);
    if (rc != VRAD_OK) return rc;
    if (n > VRAD_STATIC_MAX_RAYS)
        return fail(ctx, VRAD_ERR_ARG,
                    "%lld rays exceed the %d this allocation-free entry point stages; split the batch",
                    (long long)n, VRAD_STATIC_MAX_RAYS);
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    const int mode = (opts && opts->sky_does_not_block) ? vrad::kModeSkyPass : vrad::kModeAny;
    e = vrad::trace_visibility_static(ctx->scene.view(), ctx->device, ctx->stream, rays, n,
                                      params_of(opts, mode), hit_bits);
    if (e == cudaErrorLaunchOutOfResources)
        return fail(ctx, VRAD_ERR_CUDA, "traversal stack overflow (BVH deeper than %d)", vrad::kStackDepth);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "allocation-free visibility trace");
    return VRAD_OK;
}

int32_t vrad_tracer_identity(vrad_ctx *ctx, char *buf, int32_t cap) {
    if (!ctx) return fail(nullptr, VRAD_ERR_ARG, "null context");
    if (buf && cap > 0) snprintf(buf, (size_t)cap, "%s", ctx->identity.c_str());
    return (int32_t)ctx->identity.size();
}

int32_t vrad_last_error(vrad_ctx *ctx, char *buf, int32_t cap) {
    std::string msg;
    if (ctx) {
        msg = ctx->last_error;
    } else {
        std::lock_guard<std::mutex> g(g_err_mu);
        msg = g_last_error;
    }
    if (buf && cap > 0) snprintf(buf, (size_t)cap, "%s", msg.c_str());
    return (int32_t)msg.size();
}

}  // extern "C"
