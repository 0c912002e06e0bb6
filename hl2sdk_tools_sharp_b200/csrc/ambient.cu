// ambient.cu -- the leaf ambient sample on the device: at each position the
// 162 rays into the map through the BSP surface walk, each hit's lightmap
// colour blended by the cone, projected onto the six sides of the cube.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad/Ambient):
//   AmbientSampler.ComputeRayCube (AmbientSampler.cs:211-227): ray i runs
//     from the position to position + anorm[i] x RayLength (32768 x 1.74);
//     its delta is end - start, in float; only light style 0 is kept;
//   RayAmbientLighting.Accumulate (RayAmbientLighting.cs:89-134): the cone's
//     radius at the hit, |delta| x tan(7.275 deg) x fraction, remapped from
//     [20, 40] to [0, 1] is the face average's weight (1 for a sky hit, which
//     has no luxel), the rest the luxel's;
//   AddFaceAverage (:196-226): a sky face gives the sky ambient; a lit face
//     each style-0 slot's decoded, tinted average (AmbientScene.cs:280-300);
//   AddFacePointSample (:241-291): the luxel (truncated, clamped to the
//     lightmap), each slot's RGBE decoded by the (float)(2^(e-128) / 255)
//     table (StockLightColor.cs:69-78, 262-271), tinted by reflectivity or,
//     on a sky face, replaced by the sky ambient;
//   AmbientCube.Project (AmbientCube.cs:80-103): per side, the rays whose
//     direction has a positive cosine with the side, weighted by it, summed
//     in table order, times 1 / (sum of the weights).
// Every float operation is an explicitly rounded intrinsic in the
// reference's order, so a cube is the reference's bits.
//
// Work distribution: k_ambient_rays runs one ray per thread over the
// flattened (sample, direction) list, direction fastest, so a warp's rays
// leave one point in neighbouring directions and walk much of the tree
// together; each ray writes its colour to a chunk scratch (12 B).
// k_ambient_project runs one thread per (sample, side) and sums its 162
// colours in table order (the six threads of a sample read the same 1,944
// bytes, which L1 serves).  The walk dominates: one ray visits hundreds of
// nodes; the scratch traffic is 12 B written and 72 B read per ray.

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ambient.cuh"
#include "bsp_walk.cuh"
#include "context.cuh"
#include "device_pool.h"

namespace vrad {

void AmbientBuffers::release() {
    for (void *p : {(void *)light, (void *)faces, (void *)directions, (void *)power2n, (void *)rad, (void *)flags})
        dev_free(p);
    light = nullptr;
    faces = nullptr;
    directions = power2n = rad = nullptr;
    flags = nullptr;
    rad_samples = 0;
    ready = false;
    view = AmbientView{};
}

namespace {

constexpr int kRayBlock = 128;
constexpr int kProjectBlock = 128;
constexpr int64_t kChunkSamples = 16384;  // 31.9 MB of ray colours
constexpr float kRayLength = 32768.0f * 1.74f;
constexpr uint32_t kFlagStack = 1, kFlagBadAverage = 2, kFlagOutsideLump = 4;

__device__ __forceinline__ void add_scaled(float &x, float &y, float &z, float cx, float cy, float cz, float s) {
    x = __fadd_rn(x, __fmul_rn(cx, s));
    y = __fadd_rn(y, __fmul_rn(cy, s));
    z = __fadd_rn(z, __fmul_rn(cz, s));
}

__global__ void __launch_bounds__(kRayBlock) k_ambient_rays(DeviceBsp g, AmbientView a,
                                                            const float *__restrict__ positions, int64_t nsamples,
                                                            float *__restrict__ rad, uint32_t *flags) {
    const int64_t idx = (int64_t)blockIdx.x * kRayBlock + threadIdx.x;
    if (idx >= nsamples * kAmbientDirs) return;
    const int64_t s = idx / kAmbientDirs;
    const int i = (int)(idx - s * kAmbientDirs);
    const float sx = __ldg(positions + 3 * s), sy = __ldg(positions + 3 * s + 1), sz = __ldg(positions + 3 * s + 2);
    const float ax = __ldg(a.directions + 3 * i), ay = __ldg(a.directions + 3 * i + 1),
                az = __ldg(a.directions + 3 * i + 2);
    bspwalk::Walk c;
    c.ox = sx;
    c.oy = sy;
    c.oz = sz;
    c.dx = __fsub_rn(__fadd_rn(sx, __fmul_rn(ax, kRayLength)), sx);
    c.dy = __fsub_rn(__fadd_rn(sy, __fmul_rn(ay, kRayLength)), sy);
    c.dz = __fsub_rn(__fadd_rn(sz, __fmul_rn(az, kRayLength)), sz);
    c.hit_frac = 1.0f;
    c.min_frac = 0.0f;
    c.surface = -1;
    c.has_luxel = false;
    c.luxel_s = c.luxel_t = 0.0f;
    float rx = 0.0f, ry = 0.0f, rz = 0.0f;  // light style 0
    if (!bspwalk::walk(g, c)) {
        atomicOr(flags, kFlagStack);
    } else if (c.surface >= 0) {
        const vrad_ambient_face &F = a.faces[c.surface];
        const int32_t fflags = F.flags, nstyles = F.nstyles;
        const uint32_t styles = F.styles;
        // RemapValClamped(|delta| tan(theta) fraction, 20, 40, 0, 1).
        const float len = __fsqrt_rn(bspwalk::dot3(c.dx, c.dy, c.dz, c.dx, c.dy, c.dz));
        const float dist = __fmul_rn(__fmul_rn(len, a.tan_theta), c.hit_frac);
        float cv = __fdiv_rn(__fsub_rn(dist, 20.0f), __fsub_rn(40.0f, 20.0f));
        if (cv < 0.0f) cv = 0.0f;
        else if (cv > 1.0f) cv = 1.0f;
        float scale_avg = __fadd_rn(0.0f, __fmul_rn(__fsub_rn(1.0f, 0.0f), cv));
        if (!c.has_luxel) scale_avg = 1.0f;
        const float scale_sample = __fsub_rn(1.0f, scale_avg);
        if (scale_avg != 0.0f) {
            if (fflags & VRAD_AMBIENT_SKY) {
                if (a.has_sky) add_scaled(rx, ry, rz, a.sky[0], a.sky[1], a.sky[2], scale_avg);
            } else if (fflags & VRAD_AMBIENT_BAD_AVERAGE) {
                atomicOr(flags, kFlagBadAverage);
            } else {
                for (int m = 0; m < nstyles; m++)
                    if (((styles >> (8 * m)) & 0xFF) == 0)
                        add_scaled(rx, ry, rz, F.averages[m][0], F.averages[m][1], F.averages[m][2], scale_avg);
            }
        }
        if (scale_sample != 0.0f && F.lightofs != -1) {
            if (F.smax < 1 || F.tmax < 1) {
                atomicOr(flags, kFlagOutsideLump);
            } else {
                int ds = __float2int_rz(c.luxel_s), dt = __float2int_rz(c.luxel_t);
                ds = ds < 0 ? 0 : (ds > F.smax - 1 ? F.smax - 1 : ds);
                dt = dt < 0 ? 0 : (dt > F.tmax - 1 ? F.tmax - 1 : dt);
                const int32_t index = dt * F.smax + ds;
                const uint32_t last = (uint32_t)(int32_t)(a.light_bytes - 4);
                for (int m = 0; m < nstyles; m++) {
                    // int arithmetic that wraps, as the reference's does
                    const uint32_t ofs =
                        (uint32_t)F.lightofs + ((uint32_t)index + (uint32_t)m * (uint32_t)F.stride) * 4u;
                    if (a.light_bytes < 4 || ofs > last) {
                        atomicOr(flags, kFlagOutsideLump);
                        break;
                    }
                    const uint8_t *p = a.light + ofs;
                    const float e = __ldg(a.power2n + ((int)(int8_t)__ldg(p + 3) + 128));
                    float cx = __fmul_rn((float)__ldg(p), e), cy = __fmul_rn((float)__ldg(p + 1), e),
                          cz = __fmul_rn((float)__ldg(p + 2), e);
                    if (fflags & VRAD_AMBIENT_SKY) {
                        if (a.has_sky) {
                            cx = a.sky[0];
                            cy = a.sky[1];
                            cz = a.sky[2];
                        }
                    } else {
                        cx = __fmul_rn(cx, F.reflectivity[0]);
                        cy = __fmul_rn(cy, F.reflectivity[1]);
                        cz = __fmul_rn(cz, F.reflectivity[2]);
                    }
                    if (((styles >> (8 * m)) & 0xFF) == 0) add_scaled(rx, ry, rz, cx, cy, cz, scale_sample);
                }
            }
        }
    }
    float *o = rad + 3 * idx;
    o[0] = rx;
    o[1] = ry;
    o[2] = rz;
}

// Side j's box direction: +x, -x, +y, -y, +z, -z.
__device__ __forceinline__ float box_component(int j, int axis) {
    return (j >> 1) == axis ? ((j & 1) ? -1.0f : 1.0f) : 0.0f;
}

__global__ void __launch_bounds__(kProjectBlock) k_ambient_project(const float *__restrict__ rad, int64_t nsamples,
                                                                   const float *__restrict__ dirs,
                                                                   float *__restrict__ cubes) {
    const int64_t idx = (int64_t)blockIdx.x * kProjectBlock + threadIdx.x;
    if (idx >= nsamples * kAmbientSides) return;
    const int64_t s = idx / kAmbientSides;
    const int j = (int)(idx - s * kAmbientSides);
    const float bx = box_component(j, 0), by = box_component(j, 1), bz = box_component(j, 2);
    const float *r = rad + 3 * kAmbientDirs * s;
    float t = 0.0f, x = 0.0f, y = 0.0f, z = 0.0f;
    for (int i = 0; i < kAmbientDirs; i++) {
        const float c = bspwalk::dot3(__ldg(dirs + 3 * i), __ldg(dirs + 3 * i + 1), __ldg(dirs + 3 * i + 2), bx, by, bz);
        if (c > 0.0f) {
            t = __fadd_rn(t, c);
            add_scaled(x, y, z, __ldg(r + 3 * i), __ldg(r + 3 * i + 1), __ldg(r + 3 * i + 2), c);
        }
    }
    const float inv = __fdiv_rn(1.0f, t);
    float *o = cubes + 3 * idx;
    o[0] = __fmul_rn(x, inv);
    o[1] = __fmul_rn(y, inv);
    o[2] = __fmul_rn(z, inv);
}

// Orders a caller's stream s after the context's stream (which every
// earlier call's kernels joined), so that calls on different streams take
// the chunk scratch in turn.  Not while s is being captured.
cudaError_t after_context(vrad_ctx *ctx, cudaStream_t s) {
    if (s == ctx->stream) return cudaSuccess;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess || cap != cudaStreamCaptureStatusNone) return e;
    e = cudaEventRecord(ctx->join, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->join, 0);
    return e;
}

// The cubes of n device positions into device cubes, chunk by chunk.
int32_t cubes_on(vrad_ctx *ctx, const float *d_pos, int64_t n, float *d_cubes, cudaStream_t s) {
    if (!ctx->bsp.ready) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no BSP uploaded");
    AmbientBuffers &A = ctx->ambient;
    if (!A.ready) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no ambient lighting uploaded");
    if (A.view.nfaces != ctx->bsp.nsurfaces)
        return vrad_fail(ctx, VRAD_ERR_ARG, "the ambient lighting has %d faces, the BSP %d", A.view.nfaces,
                         ctx->bsp.nsurfaces);
    const int64_t chunk = n < kChunkSamples ? n : kChunkSamples;
    cudaError_t e = after_context(ctx, s);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "ordering the caller's stream");
    if (A.rad_samples < chunk) {
        e = wait_stream(s);  // the old scratch may still be in use
        if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "ambient scratch");
        dev_free(A.rad);
        A.rad = nullptr;
        A.rad_samples = 0;
        e = dev_alloc(&A.rad, sizeof(float) * 3 * kAmbientDirs * (size_t)chunk);
        if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "ambient ray scratch");
        A.rad_samples = chunk;
    }
    for (int64_t b = 0; b < n && e == cudaSuccess; b += chunk) {
        const int64_t m = (n - b) < chunk ? (n - b) : chunk;
        const int64_t rays = m * kAmbientDirs;
        k_ambient_rays<<<(unsigned)((rays + kRayBlock - 1) / kRayBlock), kRayBlock, 0, s>>>(
            ctx->bsp.view, A.view, d_pos + 3 * b, m, A.rad, A.flags);
        const int64_t sides = m * kAmbientSides;
        k_ambient_project<<<(unsigned)((sides + kProjectBlock - 1) / kProjectBlock), kProjectBlock, 0, s>>>(
            A.rad, m, A.directions, d_cubes + 3 * kAmbientSides * b);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? VRAD_OK : vrad_cuda_fail(ctx, e, "ambient cube launch");
}

int32_t read_flags(vrad_ctx *ctx) {
    uint32_t f = 0;
    cudaError_t e = cudaMemcpyAsync(&f, ctx->ambient.flags, sizeof f, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = wait_stream(ctx->stream);
    if (e == cudaSuccess && f) e = cudaMemsetAsync(ctx->ambient.flags, 0, sizeof f, ctx->stream);
    if (e == cudaSuccess && f) e = wait_stream(ctx->stream);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "ambient status");
    if (f & kFlagStack)
        return vrad_fail(ctx, VRAD_ERR_CUDA, "the BSP walk went deeper than %d pending splits", bspwalk::kStack);
    if (f & kFlagBadAverage)
        return vrad_fail(ctx, VRAD_ERR_ARG, "a ray hit a face with light styles whose averages lie outside the lump");
    if (f & kFlagOutsideLump) return vrad_fail(ctx, VRAD_ERR_ARG, "a ray hit a luxel that lies outside the lump");
    return VRAD_OK;
}

}  // namespace
}  // namespace vrad

extern "C" int32_t vrad_ambient_upload(vrad_ctx *ctx, const vrad_ambient_lighting *L) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (!L || L->nfaces < 0 || (L->nfaces && !L->faces) || L->lighting_bytes < 0 ||
        L->lighting_bytes > 0x7fffffffLL || (L->lighting_bytes && !L->lighting) || !L->directions ||
        L->ndirections != vrad::kAmbientDirs || std::isnan(L->tan_theta))
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid ambient lighting");
    for (int32_t f = 0; f < L->nfaces; f++)
        if (L->faces[f].nstyles < 0 || L->faces[f].nstyles > 4)
            return vrad_fail(ctx, VRAD_ERR_ARG, "face %d has %d style slots", f, L->faces[f].nstyles);
    // StockLightColor's Power2N: (float)(2^(k - 128) / 255) in double, rounded once.
    float p2n[256];
    for (int k = 0; k < 256; k++) p2n[k] = (float)(std::ldexp(1.0, k - 128) / 255.0);
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = vrad::quiesce(ctx);
    vrad::AmbientBuffers &A = ctx->ambient;
    A.release();
    auto up = [&](auto **dst, const void *src, size_t bytes) {
        cudaError_t r = vrad::dev_alloc(dst, bytes ? bytes : 16);
        if (r == cudaSuccess && bytes) r = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
        return r;
    };
    if (e == cudaSuccess) e = up(&A.light, L->lighting, (size_t)L->lighting_bytes);
    if (e == cudaSuccess) e = up(&A.faces, L->faces, sizeof(vrad_ambient_face) * (size_t)L->nfaces);
    if (e == cudaSuccess) e = up(&A.directions, L->directions, sizeof(float) * 3 * vrad::kAmbientDirs);
    if (e == cudaSuccess) e = up(&A.power2n, p2n, sizeof p2n);
    if (e == cudaSuccess) e = vrad::dev_alloc(&A.flags, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(A.flags, 0, sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);  // p2n dies at return
    if (e != cudaSuccess) {
        A.release();
        return vrad_cuda_fail(ctx, e, "ambient upload");
    }
    A.view = vrad::AmbientView{A.light, L->lighting_bytes, A.faces, L->nfaces, A.directions, A.power2n,
                               L->tan_theta, L->has_sky_ambient ? 1 : 0,
                               {L->sky_ambient[0], L->sky_ambient[1], L->sky_ambient[2]}};
    A.ready = true;
    return VRAD_OK;
}

extern "C" int32_t vrad_ambient_cubes_device(vrad_ctx *ctx, const float *d_positions, int64_t n, float *d_cubes,
                                             void *stream) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n < 0 || (n && (!d_positions || !d_cubes))) return vrad_fail(ctx, VRAD_ERR_ARG, "invalid positions or cubes");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    const int32_t rc = vrad::cubes_on(ctx, d_positions, n, d_cubes, (cudaStream_t)stream);
    e = vrad::join_stream(ctx, (cudaStream_t)stream);
    return rc != VRAD_OK || e == cudaSuccess ? rc : vrad_cuda_fail(ctx, e, "joining the caller's stream");
}

extern "C" int32_t vrad_ambient_status(vrad_ctx *ctx) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->ambient.ready) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no ambient lighting uploaded");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    return vrad::read_flags(ctx);
}

extern "C" int32_t vrad_ambient_cubes(vrad_ctx *ctx, const float *positions, int64_t n, float *cubes) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (n < 0 || (n && (!positions || !cubes))) return vrad_fail(ctx, VRAD_ERR_ARG, "invalid positions or cubes");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    float *d_pos = nullptr, *d_cubes = nullptr;
    if (e == cudaSuccess) e = vrad::dev_alloc(&d_pos, sizeof(float) * 3 * (size_t)n);
    if (e == cudaSuccess) e = vrad::dev_alloc(&d_cubes, sizeof(float) * 3 * vrad::kAmbientSides * (size_t)n);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_pos, positions, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    int32_t rc = e == cudaSuccess ? vrad::cubes_on(ctx, d_pos, n, d_cubes, ctx->stream)
                                  : vrad_cuda_fail(ctx, e, "ambient set-up");
    if (rc == VRAD_OK) {
        e = cudaMemcpyAsync(cubes, d_cubes, sizeof(float) * 3 * vrad::kAmbientSides * (size_t)n,
                            cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
        rc = e == cudaSuccess ? vrad::read_flags(ctx) : vrad_cuda_fail(ctx, e, "ambient cubes");
    }
    vrad::dev_free(d_pos);
    vrad::dev_free(d_cubes);
    return rc;
}
