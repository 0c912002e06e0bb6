// recheck.cu -- the FP64 recheck of visibility rays near a decision
// boundary (vrad_trace_visibility_recheck).
//
// The FP32 answer stays the reference's: every triangle decision is
// KdRayTracer.IntersectTriangle's arithmetic (traverse.cuh:kd_hit).  What
// this adds is the check the reference's own GPU tracer is held to
// (Tests/MapTools/Tracing/VulkanRayTracerFacts.cs:1215-1300): a ray is
// flagged when some triangle's FP32 edge values or t lie within a margin
// of a boundary (an edge, the sum's 1, either end of the segment), and
// each flagged ray is re-tested in FP64 against every triangle
// (Moller-Trumbore over the original vertices) into miss, hit, or
// ambiguous (within the FP64 margin of a boundary).  A flagged ray whose
// FP64 class is a clear hit or miss that differs from its FP32 bit is a
// disagreement; ambiguous rays are those on which two correct tracers may
// differ.
//
// Kernels:
//   k_trace_flag   one ray per thread: the any-hit walk of k_trace with
//                  the near-boundary flag (boxes widened by the margin),
//                  the visibility bits and a list of flagged rays
//   k_fp64_class   one warp per flagged ray: the lanes stride over the
//                  triangles in FP64, the warp's votes give the class.
// The FP64 operations are explicitly rounded in the oracle's order
// (oracle/tracer_oracle.cpp:orc_fp64_classify), so the classes are its.

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "context.cuh"
#include "device_pool.h"
#include "traverse.cuh"

namespace vrad {
namespace {

__global__ void __launch_bounds__(kBlock) k_trace_flag(DeviceScene s, const vrad_ray *__restrict__ rays, int64_t n,
                                                       float tmin, int32_t skip_id, float margin,
                                                       uint32_t *__restrict__ bits, int32_t *__restrict__ flagged,
                                                       int32_t *count, uint32_t *overflow) {
    extern __shared__ int stack_mem[];
    int *stack = stack_mem + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    if (i - lane >= n) return;
    bool hit = false;
    NearCheck nc{margin, tmin, 1.0f, false};
    if (i < n) {
        const float *f = reinterpret_cast<const float *>(rays + i);
        RayState r;
        r.ox = __ldg(f + 0);
        r.oy = __ldg(f + 1);
        r.oz = __ldg(f + 2);
        r.dx = __ldg(f + 3);
        r.dy = __ldg(f + 4);
        r.dz = __ldg(f + 5);
        const float reach = __ldg(f + 6);
        r.ix = recip_saturate(r.dx);
        r.iy = recip_saturate(r.dy);
        r.iz = recip_saturate(r.dz);
        r.nox = -r.ox * r.ix;
        r.noy = -r.oy * r.iy;
        r.noz = -r.oz * r.iz;
        nc.thi = reach;
        trace_ray_flagged(s, r, tmin, reach, skip_id, stack, overflow, hit, nc);
        if (nc.near) flagged[atomicAdd(count, 1)] = (int32_t)i;
    }
    const uint32_t word = __ballot_sync(kFull, hit);
    if (lane == 0) bits[i >> 5] = word;
}

constexpr int kClassWarps = 8;

__device__ __forceinline__ double dot3d(double ax, double ay, double az, double bx, double by, double bz) {
    return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

// The FP64 class of each flagged ray: 0 miss, 1 hit, 2 ambiguous.
__global__ void __launch_bounds__(32 * kClassWarps) k_fp64_class(const vrad_ray *__restrict__ rays,
                                                                 const int32_t *__restrict__ flagged, int32_t nflagged,
                                                                 const float *__restrict__ v9,
                                                                 const int32_t *__restrict__ ids, int32_t ntris,
                                                                 double tmin, int32_t skip_id, double m,
                                                                 int8_t *__restrict__ cls_out) {
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (w >= nflagged) return;
    const float *f = reinterpret_cast<const float *>(rays + __ldg(&flagged[w]));
    const double ox = __ldg(f), oy = __ldg(f + 1), oz = __ldg(f + 2);
    const double dx = __ldg(f + 3), dy = __ldg(f + 4), dz = __ldg(f + 5);
    const double reach = __ldg(f + 6);
    const double tm = __dmul_rn(m, reach > 1.0 ? reach : 1.0);
    const double dn = __dsqrt_rn(dot3d(dx, dy, dz, dx, dy, dz));
    bool inside = false, ambiguous = false;
    for (int k = (int)lane; k < ntris; k += 32) {
        if (skip_id != -1 && __ldg(&ids[k]) == skip_id) continue;
        const float *p = v9 + 9 * (int64_t)k;
        const double ax = __ldg(p), ay = __ldg(p + 1), az = __ldg(p + 2);
        const double e1x = __dsub_rn(__ldg(p + 3), ax), e1y = __dsub_rn(__ldg(p + 4), ay),
                     e1z = __dsub_rn(__ldg(p + 5), az);
        const double e2x = __dsub_rn(__ldg(p + 6), ax), e2y = __dsub_rn(__ldg(p + 7), ay),
                     e2z = __dsub_rn(__ldg(p + 8), az);
        const double px = __dsub_rn(__dmul_rn(dy, e2z), __dmul_rn(dz, e2y));
        const double py = __dsub_rn(__dmul_rn(dz, e2x), __dmul_rn(dx, e2z));
        const double pz = __dsub_rn(__dmul_rn(dx, e2y), __dmul_rn(dy, e2x));
        const double det = dot3d(e1x, e1y, e1z, px, py, pz);
        const double e1n = __dsqrt_rn(dot3d(e1x, e1y, e1z, e1x, e1y, e1z));
        const double e2n = __dsqrt_rn(dot3d(e2x, e2y, e2z, e2x, e2y, e2z));
        const double scale = __dmul_rn(__dmul_rn(dn, e1n), e2n);
        if (scale == 0.0) continue;
        if (fabs(det) <= __dmul_rn(m, scale)) {
            // Grazing: ambiguous when the segment runs within the margin of
            // the triangle's plane (or crosses it).
            const double nx = __dsub_rn(__dmul_rn(e1y, e2z), __dmul_rn(e1z, e2y));
            const double ny = __dsub_rn(__dmul_rn(e1z, e2x), __dmul_rn(e1x, e2z));
            const double nz = __dsub_rn(__dmul_rn(e1x, e2y), __dmul_rn(e1y, e2x));
            const double nn = __dsqrt_rn(dot3d(nx, ny, nz, nx, ny, nz));
            if (nn == 0.0 || !(fabs(det) > 0.0)) continue;
            const double wx = __dsub_rn(ox, ax), wy = __dsub_rn(oy, ay), wz = __dsub_rn(oz, az);
            const double d0 = __ddiv_rn(dot3d(wx, wy, wz, nx, ny, nz), nn);
            const double d1 = __dadd_rn(d0, __dmul_rn(reach, __ddiv_rn(dot3d(dx, dy, dz, nx, ny, nz), nn)));
            const double el = e1n > e2n ? e1n : e2n;
            const double rl = __dmul_rn(reach, dn);
            const double lim = __dmul_rn(m, el > rl ? el : rl);
            const bool clear = (d0 > lim && d1 > lim) || (d0 < -lim && d1 < -lim);
            if (!clear) ambiguous = true;
            continue;
        }
        const double inv = __ddiv_rn(1.0, det);
        const double tx = __dsub_rn(ox, ax), ty = __dsub_rn(oy, ay), tz = __dsub_rn(oz, az);
        const double u = __dmul_rn(dot3d(tx, ty, tz, px, py, pz), inv);
        const double qx = __dsub_rn(__dmul_rn(ty, e1z), __dmul_rn(tz, e1y));
        const double qy = __dsub_rn(__dmul_rn(tz, e1x), __dmul_rn(tx, e1z));
        const double qz = __dsub_rn(__dmul_rn(tx, e1y), __dmul_rn(ty, e1x));
        const double v = __dmul_rn(dot3d(dx, dy, dz, qx, qy, qz), inv);
        const double t = __dmul_rn(dot3d(e2x, e2y, e2z, qx, qy, qz), inv);
        const double uv = __dadd_rn(u, v);
        const bool in = u > m && v > m && uv < __dsub_rn(1.0, m) && t > __dadd_rn(tmin, tm) && t < __dsub_rn(reach, tm);
        const bool out = u < -m || v < -m || uv > __dadd_rn(1.0, m) || t < __dsub_rn(tmin, tm) ||
                         t > __dadd_rn(reach, tm);
        if (in) inside = true;
        else if (!out) ambiguous = true;
    }
    const bool any_in = __any_sync(kFull, inside), any_amb = __any_sync(kFull, ambiguous);
    if (lane == 0) cls_out[w] = any_in ? 1 : (any_amb ? 2 : 0);
}

}  // namespace
}  // namespace vrad

extern "C" int32_t vrad_trace_visibility_recheck(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                                                 const vrad_trace_options *opts, const vrad_triangle *tris,
                                                 int32_t ntris, float flag_margin, double fp64_margin,
                                                 uint64_t *hit_bits, int8_t *fp64_class, vrad_recheck_stats *stats) {
    using namespace vrad;
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n < 0 || n > 0x7fffffffLL || (n && (!rays || !hit_bits || !fp64_class)) || ntris < 0 || (ntris && !tris) ||
        !(flag_margin >= 0.0f) || !(fp64_margin >= 0.0))
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid recheck arguments");
    const float tmin = opts ? opts->min_distance : 0.0f;
    const int32_t skip = opts ? opts->skip_id : -1;
    if (std::isnan(tmin) || tmin < 0.0f)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "min_distance must be a non-negative number");
    if (opts && opts->sky_does_not_block)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "the FP64 recheck covers the any-hit visibility only");
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->has_scene) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    if (ntris != ctx->scene.ntris)
        return vrad_fail(ctx, VRAD_ERR_ARG, "the scene has %d triangles, the recheck was given %d", ctx->scene.ntris,
                         ntris);
    vrad_recheck_stats st{};
    st.rays = n;
    if (n == 0) {
        if (stats) *stats = st;
        return VRAD_OK;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    std::vector<float> v9((size_t)ntris * 9);
    std::vector<int32_t> ids((size_t)ntris);
    for (int32_t k = 0; k < ntris; k++) {
        for (int c = 0; c < 3; c++) {
            v9[9 * (size_t)k + c] = tris[k].v0[c];
            v9[9 * (size_t)k + 3 + c] = tris[k].v1[c];
            v9[9 * (size_t)k + 6 + c] = tris[k].v2[c];
        }
        ids[(size_t)k] = tris[k].id;
    }
    const size_t words32 = (size_t)((n + 31) / 32), words64 = (size_t)((n + 63) / 64);
    vrad_ray *d_rays = nullptr;
    uint32_t *d_bits = nullptr;
    int32_t *d_flagged = nullptr, *d_count = nullptr, *d_ids = nullptr;
    float *d_v9 = nullptr;
    int8_t *d_cls = nullptr;
    if (e == cudaSuccess) e = dev_alloc(&d_rays, sizeof(vrad_ray) * (size_t)n);
    if (e == cudaSuccess) e = dev_alloc(&d_bits, 8 * words64);
    if (e == cudaSuccess) e = dev_alloc(&d_flagged, sizeof(int32_t) * (size_t)n);
    if (e == cudaSuccess) e = dev_alloc(&d_count, sizeof(int32_t));
    if (e == cudaSuccess) e = dev_alloc(&d_v9, sizeof(float) * (v9.size() ? v9.size() : 1));
    if (e == cudaSuccess) e = dev_alloc(&d_ids, sizeof(int32_t) * (ids.size() ? ids.size() : 1));
    if (e == cudaSuccess) e = dev_alloc(&d_cls, (size_t)n);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_rays, rays, sizeof(vrad_ray) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && ntris)
        e = cudaMemcpyAsync(d_v9, v9.data(), sizeof(float) * v9.size(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && ntris)
        e = cudaMemcpyAsync(d_ids, ids.data(), sizeof(int32_t) * ids.size(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(int32_t), ctx->stream);
    // The last 32-bit word of an odd count belongs to no warp; clear it.
    if (e == cudaSuccess && (words32 & 1)) e = cudaMemsetAsync(d_bits + words32, 0, 4, ctx->stream);
    int32_t nflagged = 0;
    if (e == cudaSuccess) {
        const DeviceScene s = ctx->scene.view();
        const size_t smem = sizeof(int) * (size_t)s.stack_depth() * kBlock;
        k_trace_flag<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, smem, ctx->stream>>>(
            s, d_rays, n, tmin, skip, flag_margin, d_bits, d_flagged, d_count, ctx->status);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nflagged, d_count, sizeof nflagged, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = wait_stream(ctx->stream);
    std::vector<int32_t> list;
    std::vector<int8_t> cls;
    if (e == cudaSuccess && nflagged > 0) {
        const int64_t threads = 32LL * nflagged;
        k_fp64_class<<<(unsigned)((threads + 32 * kClassWarps - 1) / (32 * kClassWarps)), 32 * kClassWarps, 0,
                       ctx->stream>>>(d_rays, d_flagged, nflagged, d_v9, d_ids, ntris, (double)tmin, skip,
                                      fp64_margin, d_cls);
        e = cudaGetLastError();
        list.resize((size_t)nflagged);
        cls.resize((size_t)nflagged);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(list.data(), d_flagged, sizeof(int32_t) * (size_t)nflagged, cudaMemcpyDeviceToHost,
                                ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(cls.data(), d_cls, (size_t)nflagged, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit_bits, d_bits, 8 * words64, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = wait_stream(ctx->stream);
    for (void *p : {(void *)d_rays, (void *)d_bits, (void *)d_flagged, (void *)d_count, (void *)d_v9, (void *)d_ids,
                    (void *)d_cls})
        dev_free(p);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "visibility recheck");
    uint32_t overflow = 0;
    e = cudaMemcpyAsync(&overflow, ctx->status, sizeof overflow, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = wait_stream(ctx->stream);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "reading the traversal status");
    if (overflow) {
        cudaMemsetAsync(ctx->status, 0, sizeof(uint32_t), ctx->stream);
        wait_stream(ctx->stream);
        return vrad_fail(ctx, VRAD_ERR_CUDA, "traversal stack overflow");
    }
    for (int64_t i = 0; i < n; i++) fp64_class[i] = -1;
    st.flagged = nflagged;
    for (int32_t k = 0; k < nflagged; k++) {
        const int64_t i = list[(size_t)k];
        const int8_t c = cls[(size_t)k];
        fp64_class[i] = c;
        const bool bit = (hit_bits[i >> 6] >> (i & 63)) & 1ull;
        if (c == 0) st.fp64_miss++;
        else if (c == 1) st.fp64_hit++;
        else st.fp64_ambiguous++;
        if ((c == 0 && bit) || (c == 1 && !bit)) st.disagreements++;
    }
    if (stats) *stats = st;
    return VRAD_OK;
}
