// gather.cuh -- the per-point light gather shared by the direct gather
// (direct.cu) and the supersampling passes (supersample.cu): every light
// of the point's cluster list in gather order, each shadow, sun and sky
// segment traced in-thread, accumulated into a LightingValue.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad/Light):
//   DirectLightGatherer.GatherPointFour (:1308-1420), GatherStandardLane
//       (:1169-1306, spotlights), EmitSkyLight / ResolveSkyLight (:536-640),
//       AmbientSky (:642-815), Resolve's dot clamp (:441-478),
//       InverseQuadratic (:1579);
//   FaceLightJob.ResolveGroup / ResolveResample (FaceLightJob.cs:400-550):
//       fxdot = (mask ? dot : 0) * falloff added with AddLight.  The group
//       resolve skips a light whose four fxdots are all zero; the resample
//       resolve adds it anyway, which adds +0 (dot and falloff are never
//       negative, and a sky light with no visible lane has a zero sun
//       amount), so one code path serves both.
// Every float operation is an explicitly rounded intrinsic in the
// reference's order.  A four-point group is four adjacent lanes; its
// "any lane" tests are shuffles within the group.  The caller guarantees
// that every lane of a warp runs the same light list (one cluster, one
// filter), so the __syncwarp()s keep the warp tracing one light, or one
// sky direction, at a time.
#pragma once

#include <cuda_runtime.h>

#include "detmath.cuh"
#include "direct.cuh"
#include "traverse.cuh"

namespace vrad {

constexpr float kMaxTraceLength = (float)(1.732050807569 * (2 * 16384));  // LightConstants.MaxTraceLength
constexpr float kEqualEpsilon = 0.001f;                                   // LightConstants.EqualEpsilon

enum : int { kSurface = 0, kPoint = 1, kSpot = 2, kSkyLight = 3, kSkyAmbient = 4 };
// LightConstants.DistEpsilon: how far a surface light's rays end off its patch.
constexpr float kDistEpsilon = 0.03125f;

// The any-hit walks' child order for the gather's segments: the farther
// child first (measured faster for these rays than nearest first).
constexpr bool kFarPoint = true;  // shadow segments to point and spot lights
constexpr bool kFarSky = true;    // the opaque walk of the sun and sky tests

__device__ __forceinline__ float maxps(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minps(float a, float b) { return a < b ? a : b; }

// True when any lane of this lane's four-lane group has v set.
__device__ __forceinline__ bool group_any(bool v, unsigned gmask) {
    unsigned x = v ? 1u : 0u;
    x |= __shfl_xor_sync(gmask, x, 1);
    x |= __shfl_xor_sync(gmask, x, 2);
    return x != 0;
}

// The segment start -> stop (LightRayLog.MakeRay: whole segment, reach 1).
// Visibility blocks on any hit; a sky test blocks only when the first hit
// is opaque.
template <int MODE, int STRIDE, bool FAR_ANY>
__device__ __forceinline__ bool segment_blocked(const DeviceScene &sc, float sx, float sy, float sz,
                                                float ex, float ey, float ez, int *stack,
                                                uint32_t *overflow) {
    const RayState r = make_ray(sx, sy, sz, __fsub_rn(ex, sx), __fsub_rn(ey, sy), __fsub_rn(ez, sz));
    bool hit;
    float t;
    int32_t orig;
    uint32_t meta;
    trace_ray<MODE, STRIDE, FAR_ANY>(sc, r, 0.0f, 1.0f, -1, stack, overflow, hit, t, orig, meta);
    return hit;
}

// QuinticInterpolatingPolynomial fade (GatherPointFour / GatherStandardLane).
__device__ __forceinline__ float fade(float dist, float start, float span) {
    float t = __fdiv_rn(__fsub_rn(dist, start), span);
    t = minps(t, 1.0f);
    t = maxps(t, 0.0f);
    t = __fsub_rn(1.0f, t);
    float mult = __fsub_rn(__fmul_rn(6.0f, t), 15.0f);
    mult = __fadd_rn(__fmul_rn(mult, t), 10.0f);
    mult = __fmul_rn(__fmul_rn(t, t), mult);
    return __fmul_rn(t, mult);
}

// InverseQuadratic: ((d*d)*q + l*d) + c, then its reciprocal.
__device__ __forceinline__ float inverse_quadratic(float d, float q, float l, float c) {
    float f = __fmul_rn(d, d);
    f = __fmul_rn(f, q);
    f = __fadd_rn(f, __fmul_rn(l, d));
    f = __fadd_rn(f, c);
    return __fdiv_rn(1.0f, f);
}

// Which lights a gather takes.
enum : int { kAllLights = 0, kAmbientOnly = 1, kDirectOnly = 2 };

// The light of one point (px, py, pz already one unit off the face, flat
// normal n): (lighting xyz, direct sun amount).  Lanes with real = false
// follow the group's decisions but trace nothing and add nothing.  With
// DUAL the same segments also light the HDR range: `second` receives its
// value from w.lights_hdr's intensities (every decision and every traced
// segment is the range-independent one, so each range gets its own pass's
// bits).
template <int BLOCK, bool DUAL = false>
__device__ __forceinline__ float4 gather_point(const DeviceScene &sc, const DeviceWorld &w, int cluster, float px,
                                               float py, float pz, float nx, float ny, float nz, bool real,
                                               unsigned gmask, int filter, int *stack, uint32_t *overflow,
                                               unsigned long long *counters, unsigned long long &vis_rays,
                                               unsigned long long &sky_rays, float4 *second = nullptr,
                                               int face = 0, unsigned long long key_group = 0) {
    float ax = 0.0f, ay = 0.0f, az = 0.0f, sun = 0.0f;
    float hx = 0.0f, hy = 0.0f, hz = 0.0f;

    const int l0 = __ldg(&w.cl_off[cluster]), l1 = __ldg(&w.cl_off[cluster + 1]);
    for (int k = l0; k < l1; k++) {
        const int li = __ldg(&w.cl_list[k]);
        const float4 *L = w.lights + kLightF4 * li;
        const float4 A = __ldg(L), B = __ldg(L + 1), C = __ldg(L + 2), D = __ldg(L + 3), E = __ldg(L + 4);
        const int type = __float_as_int(A.w);
        // Each style's lights are gathered apart (its own slot); the test
        // is warp-uniform.
        if (__float_as_int(B.w) != w.style) continue;
        // The resampling passes gather the sky ambient and the other
        // lights apart (EmitResample); the filter is warp-uniform.
        if (filter == kAmbientOnly && type != kSkyAmbient) continue;
        if (filter == kDirectOnly && type == kSkyAmbient) continue;
        float dot = 0.0f, falloff = 0.0f, sun_amount = 0.0f;

        if (type == kPoint || type == kSpot) {
            const bool hard = E.z > E.y;  // EndFadeDistance > StartFadeDistance
            float dx = __fsub_rn(A.x, px), dy = __fsub_rn(A.y, py), dz = __fsub_rn(A.z, pz);
            const float dist2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            float dist = __fsqrt_rn(dist2);
            const float rpc = __fdiv_rn(1.0f, dist);
            dx = __fmul_rn(dx, rpc);
            dy = __fmul_rn(dy, rpc);
            dz = __fmul_rn(dz, rpc);
            float d = __fadd_rn(__fadd_rn(__fmul_rn(dx, nx), __fmul_rn(dy, ny)), __fmul_rn(dz, nz));
            d = maxps(0.0f, d);
            bool live = !hard || dist <= E.z;
            if (type == kPoint) {
                // GatherPointFour.
                dist = maxps(dist, 1.0f);
                const float dd = minps(dist, E.w);
                float f = inverse_quadratic(dd, E.x, D.w, D.z);
                if (hard) f = __fmul_rn(fade(dist, E.y, __fsub_rn(E.z, E.y)), f);
                dot = live ? d : 0.0f;
                falloff = live ? f : 0.0f;
            } else if (live) {
                // GatherStandardLane, Spotlight.
                dist = maxps(dist, 1.0f);
                const float fed = minps(dist, E.w);
                const float dot2 =
                    -__fadd_rn(__fadd_rn(__fmul_rn(dx, C.x), __fmul_rn(dy, C.y)), __fmul_rn(dz, C.z));
                if (dot2 > D.y) {
                    float f = __fmul_rn(inverse_quadratic(fed, E.x, D.w, D.z), dot2);
                    const bool fringe = dot2 <= D.x;
                    float mult = __fdiv_rn(__fsub_rn(dot2, D.y), __fsub_rn(D.x, D.y));
                    mult = minps(mult, 1.0f);
                    mult = maxps(mult, 0.0f);
                    if (C.w != 0.0f && C.w != 1.0f) mult = pow_cr(mult, C.w, &counters[2]);  // DetMathF.Pow
                    mult = fringe ? mult : 1.0f;
                    f = __fmul_rn(mult, f);
                    if (hard) f = __fmul_rn(fade(dist, E.y, __fsub_rn(E.z, E.y)), f);
                    dot = d;
                    falloff = f;
                }
            }
            if (real && dot != 0.0f && falloff != 0.0f) {
                vis_rays++;
                if (segment_blocked<kModeAny, BLOCK, kFarPoint>(sc, px, py, pz, A.x, A.y, A.z, stack, overflow)) dot = 0.0f;
            }
        } else if (type == kSurface) {
            // GatherSurfaceFour (DirectLightGatherer.cs:1452-1545): the
            // patch's cosine over the squared distance, the segment to the
            // patch origin pushed off the emitter by DistEpsilon.
            const bool hard = E.z > E.y;
            float dx = __fsub_rn(A.x, px), dy = __fsub_rn(A.y, py), dz = __fsub_rn(A.z, pz);
            const float dist2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            float dist = __fsqrt_rn(dist2);
            const float rpc = __fdiv_rn(1.0f, dist);
            dx = __fmul_rn(dx, rpc);
            dy = __fmul_rn(dy, rpc);
            dz = __fmul_rn(dz, rpc);
            float d = __fadd_rn(__fadd_rn(__fmul_rn(dx, nx), __fmul_rn(dy, ny)), __fmul_rn(dz, nz));
            d = maxps(0.0f, d);
            bool live = !hard || dist <= E.z;
            dist = maxps(dist, 1.0f);
            // The negation flips the sign bit (a -0 survives maxps).
            float dot2 = -__fadd_rn(__fadd_rn(__fmul_rn(dx, C.x), __fmul_rn(dy, C.y)), __fmul_rn(dz, C.z));
            dot2 = maxps(0.0f, dot2);
            live = live && !(d == 0.0f);
            float f = __fdiv_rn(dot2, dist2);
            if (hard) f = __fmul_rn(fade(dist, E.y, __fsub_rn(E.z, E.y)), f);
            dot = live ? d : 0.0f;
            falloff = live ? f : 0.0f;
            if (real && dot != 0.0f && falloff != 0.0f) {
                vis_rays++;
                const float ex = __fadd_rn(A.x, __fmul_rn(C.x, kDistEpsilon)),
                            ey = __fadd_rn(A.y, __fmul_rn(C.y, kDistEpsilon)),
                            ez = __fadd_rn(A.z, __fmul_rn(C.z, kDistEpsilon));
                if (segment_blocked<kModeAny, BLOCK, kFarPoint>(sc, px, py, pz, ex, ey, ez, stack, overflow)) dot = 0.0f;
            }
        } else if (type == kSkyLight) {
            // EmitSkyLight / ResolveSkyLight.
            float d = -__fadd_rn(__fadd_rn(__fmul_rn(nx, C.x), __fmul_rn(ny, C.y)), __fmul_rn(nz, C.z));
            d = maxps(d, 0.0f);
            const bool need = group_any(d != 0.0f, gmask);
            if (__any_sync(kFull, need)) {
                const int ns = w.sun_samples;
                const float jitter_scale = (float)(1.732050807569 * (2 * 16384) * (double)w.sun_extent);
                float total = 0.0f;
                for (int s = 0; s < ns; s++) {
                    float ex = __fmul_rn(C.x, -kMaxTraceLength), ey = __fmul_rn(C.y, -kMaxTraceLength),
                          ez = __fmul_rn(C.z, -kMaxTraceLength);
                    if (s != 0) {
                        const float4 j = __ldg(&w.jitter[s - 1]);
                        ex = __fadd_rn(ex, __fmul_rn(j.x, jitter_scale));
                        ey = __fadd_rn(ey, __fmul_rn(j.y, jitter_scale));
                        ez = __fadd_rn(ez, __fmul_rn(j.z, jitter_scale));
                    }
                    float frac = 1.0f;
                    if (need && real) {
                        sky_rays++;
                        if (segment_blocked<kModeSkyPass, BLOCK, kFarSky>(sc, px, py, pz, __fadd_rn(ex, px),
                                                                 __fadd_rn(ey, py), __fadd_rn(ez, pz), stack,
                                                                 overflow))
                            frac = 0.0f;
                    }
                    total = __fadd_rn(total, frac);
                    __syncwarp();
                }
                if (need) {
                    const float see = __fmul_rn(total, __fdiv_rn(1.0f, (float)ns));
                    dot = __fmul_rn(d, see);
                    falloff = 1.0f;
                    sun_amount = __fmul_rn(see, 10000.0f);
                }
            }
        } else if (type == kSkyAmbient) {
            // AmbientSky: every direction in front of the face, in order.
            float sumdot = 0.0f, possible = 0.0f, ambient = 0.0f;
            for (int di = 0; di < w.ndirs; di++) {
                const float4 an = __ldg(&w.dirs[di]);
                const float dd = -__fadd_rn(__fadd_rn(__fmul_rn(nx, an.x), __fmul_rn(ny, an.y)), __fmul_rn(nz, an.z));
                const bool valid = dd > kEqualEpsilon;
                const float dv = valid ? dd : 0.0f;
                sumdot = __fadd_rn(dv, sumdot);
                possible = __fadd_rn(valid ? 1.0f : 0.0f, possible);
                float frac = 1.0f;
                if (valid && real) {
                    // surfacePos = points - anorm * -epsilon, epsilon 0;
                    // stop = anorm * -MaxTraceLength + points.
                    const float sx = __fsub_rn(px, __fmul_rn(an.x, -0.0f));
                    const float sy = __fsub_rn(py, __fmul_rn(an.y, -0.0f));
                    const float sz = __fsub_rn(pz, __fmul_rn(an.z, -0.0f));
                    const float ex = __fadd_rn(__fmul_rn(an.x, -kMaxTraceLength), px);
                    const float ey = __fadd_rn(__fmul_rn(an.y, -kMaxTraceLength), py);
                    const float ez = __fadd_rn(__fmul_rn(an.z, -kMaxTraceLength), pz);
                    sky_rays++;
                    if (segment_blocked<kModeSkyPass, BLOCK, kFarSky>(sc, sx, sy, sz, ex, ey, ez, stack, overflow)) frac = 0.0f;
                }
                ambient = __fadd_rn(ambient, __fmul_rn(frac, dv));
                __syncwarp();
            }
            const float factor = __fdiv_rn(possible, possible);
            dot = __fdiv_rn(ambient, __fmul_rn(factor, sumdot));
            falloff = 1.0f;
        }
        __syncwarp();
        // Resolve: a light behind the face lights nothing.
        dot = maxps(dot, 0.0f);
        const float fx = __fmul_rn(real ? dot : 0.0f, falloff);
        if (!group_any(fx != 0.0f, gmask)) continue;
        // ResolveGroup's FindOrAllocateStyle point: this group lights the
        // face in this style; its first lane keeps the earliest (group,
        // position in the light list) per face.
        if (w.face_key && (threadIdx.x & 3) == 0)
            atomicMin(&w.face_key[face], key_group | (unsigned long long)(k - l0));
        if (real) {
            ax = __fadd_rn(ax, __fmul_rn(fx, B.x));
            ay = __fadd_rn(ay, __fmul_rn(fx, B.y));
            az = __fadd_rn(az, __fmul_rn(fx, B.z));
            sun = __fadd_rn(sun, sun_amount);
            if (DUAL) {
                const float4 H = __ldg(w.lights_hdr + kLightF4 * li + 1);
                hx = __fadd_rn(hx, __fmul_rn(fx, H.x));
                hy = __fadd_rn(hy, __fmul_rn(fx, H.y));
                hz = __fadd_rn(hz, __fmul_rn(fx, H.z));
            }
        }
    }
    if (DUAL) *second = make_float4(hx, hy, hz, sun);
    return make_float4(ax, ay, az, sun);
}

}  // namespace vrad
