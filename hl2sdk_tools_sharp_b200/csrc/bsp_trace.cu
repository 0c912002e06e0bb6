// bsp_trace.cu -- the BSP surface walk: stock vrad's CLightSurface over
// EnumerateNodesAlongRay, the tracer leaf ambient uses, on the device.
//
// The walk itself (MapTools/Tracing/BspSurfaceTracer.cs:233-512, restated
// in bsp_walk.cuh) is shared with the leaf ambient sample (ambient.cu).
//
// Work distribution: one ray per thread.  The walk needs no sorting and no
// box tests: a node is one plane test, and the walk stops at the first hit
// in front-to-back order.  The pending-split stack lives in local memory
// (64 records of 16 B; L1-resident at this occupancy); a walk that needs
// more sets the context's overflow flag and the call fails, as the
// reference throws.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "bsp_walk.cuh"
#include "context.cuh"
#include "device_pool.h"

namespace vrad {

void BspBuffers::release() {
    for (void *p : {(void *)nodes, (void *)surfaces, (void *)node_faces, (void *)leaf_faces, (void *)leaf_run,
                    (void *)sky_points, (void *)sky_run})
        dev_free(p);
    nodes = surfaces = sky_points = nullptr;
    node_faces = leaf_faces = nullptr;
    leaf_run = sky_run = nullptr;
    nnodes = nsurfaces = nleaves = 0;
    ready = false;
    view = DeviceBsp{};
}

namespace {

constexpr int kBspBlock = 128;

__global__ void __launch_bounds__(kBspBlock) k_bsp_trace(DeviceBsp g, const vrad_ray *__restrict__ rays, int64_t n,
                                                         float min_frac, vrad_hit *__restrict__ hits,
                                                         uint32_t *overflow) {
    const int64_t i = (int64_t)blockIdx.x * kBspBlock + threadIdx.x;
    if (i >= n) return;
    const float *r = reinterpret_cast<const float *>(rays + i);
    bspwalk::Walk c;
    c.ox = __ldg(r + 0);
    c.oy = __ldg(r + 1);
    c.oz = __ldg(r + 2);
    const float reach = __ldg(r + 6);
    c.dx = __fmul_rn(__ldg(r + 3), reach);
    c.dy = __fmul_rn(__ldg(r + 4), reach);
    c.dz = __fmul_rn(__ldg(r + 5), reach);
    c.hit_frac = 1.0f;
    c.min_frac = min_frac;
    c.surface = -1;
    c.has_luxel = false;
    const bool ok = bspwalk::walk(g, c);
    if (!ok) atomicOr(overflow, 1u);
    vrad_hit h;
    h.surface = ok ? c.surface : -1;
    h.fraction = (ok && c.surface != -1) ? c.hit_frac : 1.0f;
    hits[i] = h;
}

}  // namespace

cudaError_t launch_bsp_trace(const DeviceBsp &g, const vrad_ray *d_rays, int64_t n, float min_frac, vrad_hit *d_hits,
                             uint32_t *overflow, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int64_t grid = (n + kBspBlock - 1) / kBspBlock;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_bsp_trace<<<(unsigned)grid, kBspBlock, 0, s>>>(g, d_rays, n, min_frac, d_hits, overflow);
    return cudaGetLastError();
}

}  // namespace vrad

extern "C" int32_t vrad_bsp_upload(vrad_ctx *ctx, const vrad_bsp_geometry *b) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (!b || b->nnodes < 1 || b->nsurfaces < 0 || b->nleaves < 0 || b->nnode_faces < 0 || b->nleaf_faces < 0 ||
        b->nsky_points < 0 || !b->nodes || (b->nsurfaces && !b->surfaces) || (b->nnode_faces && !b->node_faces) ||
        (b->nleaf_faces && !b->leaf_faces) || (b->nleaves && (!b->leaf_start || !b->leaf_count)) ||
        (b->nsurfaces && (!b->sky_start || !b->sky_count)) || (b->nsky_points && !b->sky_points))
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid BSP description");
    // Every index the walk follows is checked once, here.
    const int32_t *nw = reinterpret_cast<const int32_t *>(b->nodes);
    for (int32_t n = 0; n < b->nnodes; n++) {
        const int32_t c0 = nw[8 * n + 4], c1 = nw[8 * n + 5], first = nw[8 * n + 6], packed = nw[8 * n + 7];
        const int64_t cnt = (int64_t)(packed & 0x7FFF) + ((packed >> 15) & 0x7FFF);
        if (c0 >= b->nnodes || c1 >= b->nnodes || first < 0 || first + cnt > b->nnode_faces)
            return vrad_fail(ctx, VRAD_ERR_ARG, "BSP node %d names a child or faces the map does not have", n);
    }
    for (int32_t k = 0; k < b->nnode_faces; k++)
        if (b->node_faces[k] < 0 || b->node_faces[k] >= b->nsurfaces)
            return vrad_fail(ctx, VRAD_ERR_ARG, "node face %d names face %d", k, b->node_faces[k]);
    for (int32_t k = 0; k < b->nleaf_faces; k++)
        if (b->leaf_faces[k] < 0 || b->leaf_faces[k] >= b->nsurfaces)
            return vrad_fail(ctx, VRAD_ERR_ARG, "leaf face %d names face %d", k, b->leaf_faces[k]);
    std::vector<int2> leaf_run((size_t)(b->nleaves ? b->nleaves : 1)), sky_run((size_t)(b->nsurfaces ? b->nsurfaces : 1));
    for (int32_t l = 0; l < b->nleaves; l++) {
        if (b->leaf_start[l] < 0 || b->leaf_count[l] < 0 || (int64_t)b->leaf_start[l] + b->leaf_count[l] > b->nleaf_faces)
            return vrad_fail(ctx, VRAD_ERR_ARG, "BSP leaf %d's faces lie outside the list", l);
        leaf_run[(size_t)l] = make_int2(b->leaf_start[l], b->leaf_count[l]);
    }
    for (int32_t f = 0; f < b->nsurfaces; f++) {
        if (b->sky_start[f] < 0 || b->sky_count[f] < 0 || (int64_t)b->sky_start[f] + b->sky_count[f] > b->nsky_points)
            return vrad_fail(ctx, VRAD_ERR_ARG, "face %d's sky winding lies outside the point list", f);
        sky_run[(size_t)f] = make_int2(b->sky_start[f], b->sky_count[f]);
    }
    std::vector<float4> sky((size_t)(b->nsky_points ? b->nsky_points : 1));
    for (int32_t k = 0; k < b->nsky_points; k++)
        sky[(size_t)k] = make_float4(b->sky_points[3 * k], b->sky_points[3 * k + 1], b->sky_points[3 * k + 2], 0.0f);
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = vrad::quiesce(ctx);
    vrad::BspBuffers &bb = ctx->bsp;
    bb.release();
    auto up = [&](auto **dst, const void *src, size_t bytes) {
        cudaError_t r = vrad::dev_alloc(dst, bytes ? bytes : 16);
        if (r == cudaSuccess && bytes) r = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
        return r;
    };
    if (e == cudaSuccess) e = up(&bb.nodes, b->nodes, sizeof(float) * 8 * (size_t)b->nnodes);
    if (e == cudaSuccess) e = up(&bb.surfaces, b->surfaces, sizeof(float) * 16 * (size_t)b->nsurfaces);
    if (e == cudaSuccess) e = up(&bb.node_faces, b->node_faces, sizeof(int32_t) * (size_t)b->nnode_faces);
    if (e == cudaSuccess) e = up(&bb.leaf_faces, b->leaf_faces, sizeof(int32_t) * (size_t)b->nleaf_faces);
    if (e == cudaSuccess) e = up(&bb.leaf_run, leaf_run.data(), sizeof(int2) * (size_t)b->nleaves);
    if (e == cudaSuccess) e = up(&bb.sky_run, sky_run.data(), sizeof(int2) * (size_t)b->nsurfaces);
    if (e == cudaSuccess) e = up(&bb.sky_points, sky.data(), sizeof(float4) * (size_t)b->nsky_points);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);  // the host vectors die at return
    if (e != cudaSuccess) {
        bb.release();
        return vrad_cuda_fail(ctx, e, "BSP upload");
    }
    bb.nnodes = b->nnodes;
    bb.nsurfaces = b->nsurfaces;
    bb.nleaves = b->nleaves;
    bb.view = vrad::DeviceBsp{bb.nodes, bb.surfaces, bb.node_faces, bb.leaf_faces, bb.leaf_run, b->nleaves,
                              bb.sky_points, bb.sky_run};
    bb.ready = true;
    return VRAD_OK;
}

namespace {

int32_t bsp_trace_on(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n, float min_frac, vrad_hit *d_hits,
                     cudaStream_t s) {
    if (!ctx->bsp.ready) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no BSP uploaded");
    const cudaError_t e = vrad::launch_bsp_trace(ctx->bsp.view, d_rays, n, min_frac, d_hits, ctx->status + 2, s);
    return e == cudaSuccess ? VRAD_OK : vrad_cuda_fail(ctx, e, "BSP walk launch");
}

}  // namespace

extern "C" int32_t vrad_bsp_trace_closest_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n, float min_distance,
                                                 vrad_hit *d_hits, void *stream) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n < 0 || (n && (!d_rays || !d_hits))) return vrad_fail(ctx, VRAD_ERR_ARG, "invalid rays or hits");
    if (std::isnan(min_distance) || min_distance < 0.0f)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "min_distance must be a non-negative number");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    const int32_t rc = bsp_trace_on(ctx, d_rays, n, min_distance, d_hits, (cudaStream_t)stream);
    e = vrad::join_stream(ctx, (cudaStream_t)stream);
    return rc != VRAD_OK || e == cudaSuccess ? rc : vrad_cuda_fail(ctx, e, "joining the caller's stream");
}

extern "C" int32_t vrad_bsp_trace_closest(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                                          const vrad_trace_options *opts, vrad_hit *hits) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n < 0 || (n && (!rays || !hits))) return vrad_fail(ctx, VRAD_ERR_ARG, "invalid rays or hits");
    const float min_frac = opts ? opts->min_distance : 0.0f;
    if (std::isnan(min_frac) || min_frac < 0.0f)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "min_distance must be a non-negative number");
    if (opts && opts->skip_id != -1)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "the BSP walk has no skip id");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    vrad_ray *d_rays = nullptr;
    vrad_hit *d_hits = nullptr;
    uint32_t overflow = 0;
    if (e == cudaSuccess) e = vrad::dev_alloc(&d_rays, sizeof(vrad_ray) * (size_t)n);
    if (e == cudaSuccess) e = vrad::dev_alloc(&d_hits, sizeof(vrad_hit) * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rays, rays, sizeof(vrad_ray) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    int32_t rc = e == cudaSuccess ? bsp_trace_on(ctx, d_rays, n, min_frac, d_hits, ctx->stream)
                                  : vrad_cuda_fail(ctx, e, "BSP walk set-up");
    if (rc == VRAD_OK) {
        e = cudaMemcpyAsync(hits, d_hits, sizeof(vrad_hit) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&overflow, ctx->status + 2, sizeof overflow, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
        if (e != cudaSuccess) rc = vrad_cuda_fail(ctx, e, "BSP walk");
    }
    if (rc == VRAD_OK && overflow) {
        cudaMemsetAsync(ctx->status + 2, 0, sizeof(uint32_t), ctx->stream);
        vrad::wait_stream(ctx->stream);
        rc = vrad_fail(ctx, VRAD_ERR_CUDA, "the BSP walk went deeper than %d pending splits", vrad::bspwalk::kStack);
    }
    vrad::dev_free(d_rays);
    vrad::dev_free(d_hits);
    return rc;
}
