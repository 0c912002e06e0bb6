// traverse.cuh -- the per-ray BVH walk shared by the trace kernels
// (trace.cu) and the fused lighting kernels (direct.cu).
//
// Per-triangle arithmetic is the reference's KdRayTracer.IntersectTriangle
// (MapTools/Tracing/KdRayTracer.cs:1194-1267) operation for operation, each
// an explicitly rounded intrinsic, so an accepted/rejected decision and a
// hit distance are the CPU's bits.  The walk tests every triangle whose
// padded box the segment meets, which includes every triangle the
// predicate can accept.
#pragma once

#include "vrad_internal.cuh"

namespace vrad {

constexpr int kBlock = 128;       // threads per CTA of every traversal kernel
constexpr uint32_t kFull = 0xffffffffu;

struct RayState {
    float ox, oy, oz, dx, dy, dz;
    float ix, iy, iz;      // 1/d with zeros saturated to +-2^60
    float nox, noy, noz;   // -o/d, for the FMA slab test
};

__device__ inline float recip_saturate(float a) {
    // ReciprocalSaturateExact (KdRayTracer.cs:1446): a zero keeps its sign
    // and becomes 2^-60 before the divide.
    if (a == 0.0f) a = __uint_as_float(__float_as_uint(a) | 0x21800000u);
    return __frcp_rn(a);
}

__device__ inline float sel3(int axis, float x, float y, float z) {
    return axis == 0 ? x : (axis == 1 ? y : z);
}

// The FP64 recheck's flag (vrad_trace_visibility_recheck): set when a
// triangle's FP32 predicate values lie within `m` of a decision boundary --
// an edge value near 0, their sum near 1, or t near either end of the
// segment [tlo, thi] -- and no farther than `m` outside on the others.
struct NearCheck {
    float m, tlo, thi;
    bool near;
};

// The predicate.  Returns true with the exact t when the triangle accepts
// the ray (|d.n| > eps, eps < t < 1e23, both edge values >= eps, their sum
// <= 1).  With FLAG the near-boundary test runs first; the decision itself
// is the same arithmetic either way.
template <bool FLAG = false>
__device__ __forceinline__ bool kd_hit(const DeviceBvh &s, int k, const RayState &r, float &t_out,
                                       uint32_t &meta_out, int32_t &orig_out, NearCheck *nc = nullptr) {
    const float4 A = __ldg(&s.tri0[k]);
    float ddotn = __fmul_rn(r.dx, A.x);
    ddotn = __fadd_rn(__fmul_rn(r.dy, A.y), ddotn);
    ddotn = __fadd_rn(__fmul_rn(r.dz, A.z), ddotn);
    float odotn = __fmul_rn(r.ox, A.x);
    odotn = __fadd_rn(__fmul_rn(r.oy, A.y), odotn);
    odotn = __fadd_rn(__fmul_rn(r.oz, A.z), odotn);
    const float num = __fsub_rn(A.w, odotn);
    // t > eps needs num and ddotn of one sign; this rejects without the
    // divide exactly where the divide's sign would (|ddotn| > eps > 0).
    if (!(ddotn > kKdEps || ddotn < -kKdEps)) return false;
    if constexpr (FLAG) {
        const float4 B = __ldg(&s.tri1[k]);
        const float4 C = __ldg(&s.tri2[k]);
        const int drop = __float_as_uint(C.w) & 3;
        const int c0 = drop == 2 ? 0 : drop + 1;
        const int c1 = drop == 0 ? 2 : drop - 1;
        const float t = __fdiv_rn(num, ddotn);
        const float h1 = __fadd_rn(sel3(c0, r.ox, r.oy, r.oz), __fmul_rn(t, sel3(c0, r.dx, r.dy, r.dz)));
        const float h2 = __fadd_rn(sel3(c1, r.ox, r.oy, r.oz), __fmul_rn(t, sel3(c1, r.dx, r.dy, r.dz)));
        const float b0 = __fadd_rn(__fadd_rn(__fmul_rn(B.x, h1), __fmul_rn(B.y, h2)), B.z);
        const float b1 = __fadd_rn(__fadd_rn(__fmul_rn(B.w, h1), __fmul_rn(C.x, h2)), C.y);
        const float m = nc->m, tm = m * fmaxf(1.0f, fabsf(nc->thi));
        const float sum = __fadd_rn(b0, b1);
        const bool out = b0 < -m || b1 < -m || sum > 1.0f + m || t < nc->tlo - tm || t > nc->thi + tm;
        const bool in = b0 > m && b1 > m && sum < 1.0f - m && t > nc->tlo + tm && t < nc->thi - tm;
        if (!out && !in) nc->near = true;
    }
    if ((__float_as_uint(num) ^ __float_as_uint(ddotn)) & 0x80000000u) return false;
    const float t = __fdiv_rn(num, ddotn);
    if (!(t > kKdEps) || !(t < kKdHuge)) return false;
    const float4 B = __ldg(&s.tri1[k]);
    const float4 C = __ldg(&s.tri2[k]);
    const uint32_t meta = __float_as_uint(C.w);
    const int drop = meta & 3;
    const int c0 = drop == 2 ? 0 : drop + 1;
    const int c1 = drop == 0 ? 2 : drop - 1;
    const float h1 = __fadd_rn(sel3(c0, r.ox, r.oy, r.oz), __fmul_rn(t, sel3(c0, r.dx, r.dy, r.dz)));
    const float h2 = __fadd_rn(sel3(c1, r.ox, r.oy, r.oz), __fmul_rn(t, sel3(c1, r.dx, r.dy, r.dz)));
    float b0 = __fmul_rn(B.x, h1);
    b0 = __fadd_rn(b0, __fmul_rn(B.y, h2));
    b0 = __fadd_rn(b0, B.z);
    if (!(b0 >= kKdEps)) return false;
    float b1 = __fmul_rn(B.w, h1);
    b1 = __fadd_rn(b1, __fmul_rn(C.x, h2));
    b1 = __fadd_rn(b1, C.y);
    if (!(b1 >= kKdEps)) return false;
    if (!(__fadd_rn(b1, b0) <= 1.0f)) return false;
    t_out = t;
    meta_out = meta;
    orig_out = __float_as_int(C.z);
    return true;
}

__device__ __forceinline__ void slab2(const float4 &a, const float4 &b, const float4 &c,
                                      const RayState &r, float tlo, float thi, bool &h0, bool &h1,
                                      float &n0, float &n1) {
    // child 0: x (a.x, a.y), y (a.z, a.w), z (c.x, c.y); child 1: x (b.x, b.y), y (b.z, b.w), z (c.z, c.w)
    float x0 = fmaf(a.x, r.ix, r.nox), x1 = fmaf(a.y, r.ix, r.nox);
    float y0 = fmaf(a.z, r.iy, r.noy), y1 = fmaf(a.w, r.iy, r.noy);
    float z0 = fmaf(c.x, r.iz, r.noz), z1 = fmaf(c.y, r.iz, r.noz);
    float tn0 = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tlo));
    float tf0 = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), thi));
    float u0 = fmaf(b.x, r.ix, r.nox), u1 = fmaf(b.y, r.ix, r.nox);
    float v0 = fmaf(b.z, r.iy, r.noy), v1 = fmaf(b.w, r.iy, r.noy);
    float w0 = fmaf(c.z, r.iz, r.noz), w1 = fmaf(c.w, r.iz, r.noz);
    float tn1 = fmaxf(fmaxf(fminf(u0, u1), fminf(v0, v1)), fmaxf(fminf(w0, w1), tlo));
    float tf1 = fminf(fminf(fmaxf(u0, u1), fmaxf(v0, v1)), fminf(fmaxf(w0, w1), thi));
    h0 = tn0 <= tf0;
    h1 = tn1 <= tf1;
    n0 = tn0;
    n1 = tn1;
}

// One walk of one BVH.  Accepts a triangle hit (t, orig) when
// t >= tmin and (t, orig) is lexicographically below the current best
// (thi, best_orig); best_orig = -1 makes the window half-open, [tmin, thi).
// ANY stops at the first acceptance; otherwise the best is kept and the
// box window shrinks to [tmin, thi].  Returns whether anything was accepted.
// Of two children the segment meets, the nearer is entered first, or with
// FAR the farther (an any-hit walk may find its blocker sooner from the far
// end; which order pays is measured per caller).
template <bool ANY, int STRIDE = kBlock, bool FAR = false, bool FLAG = false>
__device__ __forceinline__ bool walk(const DeviceBvh &s, const int32_t *__restrict__ tri_id,
                                     const RayState &r, float tmin, int32_t skip_id, int *stack,
                                     uint32_t *overflow, float &thi, int32_t &best_orig,
                                     uint32_t &best_meta, NearCheck *nc = nullptr) {
    bool hit = false;
    int sp = 0;
    int ref = 0;
    while (true) {
        if (ref >= 0) {
            const float4 *nd = s.nodes + 4 * ref;
            const float4 a = __ldg(nd), b = __ldg(nd + 1), c = __ldg(nd + 2), d = __ldg(nd + 3);
            bool h0, h1;
            float n0, n1;
            if constexpr (FLAG) {
                // The recheck also wants the triangles just past either end.
                const float tm = nc->m * fmaxf(1.0f, fabsf(thi));
                slab2(a, b, c, r, tmin - tm, thi + tm, h0, h1, n0, n1);
            } else {
                slab2(a, b, c, r, tmin, thi, h0, h1, n0, n1);
            }
            const int r0 = __float_as_int(d.x), r1 = __float_as_int(d.y);
            if (h0 && h1) {
                int near_ref = r0, far_ref = r1;
                if (FAR ? (n1 > n0) : (n1 < n0)) {
                    near_ref = r1;
                    far_ref = r0;
                }
                if (sp < s.depth) {
                    stack[sp * STRIDE] = far_ref;
                    sp++;
                } else {
                    atomicOr(overflow, 1u);
                }
                ref = near_ref;
                continue;
            }
            if (h0) {
                ref = r0;
                continue;
            }
            if (h1) {
                ref = r1;
                continue;
            }
        } else {
            const int packed = ~ref;
            const int first = packed >> 3;
            const int count = (packed & 7) + 1;
            for (int k = first; k < first + count; k++) {
                float t;
                uint32_t meta;
                int32_t orig;
                if (!kd_hit<FLAG>(s, k, r, t, meta, orig, nc)) continue;
                if (!(t >= tmin)) continue;
                if (!(t < thi || (t == thi && orig < best_orig))) continue;
                if (skip_id != -1 && __ldg(&tri_id[orig]) == skip_id) continue;
                hit = true;
                thi = t;
                best_orig = orig;
                best_meta = meta;
                if (ANY) return true;
            }
        }
        if (sp == 0) return hit;
        sp--;
        ref = stack[sp * STRIDE];
    }
}

// One ray against the scene.  Modes:
//   kModeAny      any accepted hit in [tmin, reach), opaque or sky;
//   kModeClosest  the smallest (t, original index) in [tmin, reach);
//   kModeSkyPass  blocked iff that smallest hit exists and is opaque: the
//                 nearest sky hit (t_s, i_s) is found first, then any
//                 opaque hit below it decides, so the opaque walk stops at
//                 its first acceptance.
// FAR_ANY: the any-hit walks enter the farther child first (walk's FAR).
template <int MODE, int STRIDE = kBlock, bool FAR_ANY = false>
__device__ __forceinline__ void trace_ray(const DeviceScene &s, const RayState &r, float tmin,
                                          float reach, int32_t skip_id, int *stack,
                                          uint32_t *overflow, bool &hit, float &best_t,
                                          int32_t &best_orig, uint32_t &best_meta) {
    best_t = reach;
    best_orig = -1;
    best_meta = 0;
    hit = false;
    if (MODE == kModeAny) {
        if (s.opaque.ntris)
            hit = walk<true, STRIDE, FAR_ANY>(s.opaque, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig, best_meta);
        if (!hit && s.sky.ntris)
            hit = walk<true, STRIDE, FAR_ANY>(s.sky, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig, best_meta);
    } else if (MODE == kModeClosest) {
        if (s.opaque.ntris)
            hit = walk<false, STRIDE>(s.opaque, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig, best_meta);
        if (s.sky.ntris)
            hit |= walk<false, STRIDE>(s.sky, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig, best_meta);
    } else {
        if (s.sky.ntris)
            walk<false, STRIDE>(s.sky, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig, best_meta);
        // Blocked iff an opaque hit sorts before the nearest sky hit.
        if (s.opaque.ntris)
            hit = walk<true, STRIDE, FAR_ANY>(s.opaque, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig, best_meta);
    }
}


// kModeAny with the FP64 recheck's flag: the same walks and answer as
// trace_ray<kModeAny>, every box widened by the margin at both ends.
template <int STRIDE = kBlock>
__device__ __forceinline__ void trace_ray_flagged(const DeviceScene &s, const RayState &r, float tmin, float reach,
                                                  int32_t skip_id, int *stack, uint32_t *overflow, bool &hit,
                                                  NearCheck &nc) {
    float best_t = reach;
    int32_t best_orig = -1;
    uint32_t best_meta = 0;
    hit = false;
    if (s.opaque.ntris)
        hit = walk<true, STRIDE, false, true>(s.opaque, s.tri_id, r, tmin, skip_id, stack, overflow, best_t,
                                              best_orig, best_meta, &nc);
    if (!hit && s.sky.ntris)
        hit = walk<true, STRIDE, false, true>(s.sky, s.tri_id, r, tmin, skip_id, stack, overflow, best_t, best_orig,
                                              best_meta, &nc);
}

__device__ __forceinline__ RayState make_ray(float ox, float oy, float oz, float dx, float dy, float dz) {
    RayState r;
    r.ox = ox;
    r.oy = oy;
    r.oz = oz;
    r.dx = dx;
    r.dy = dy;
    r.dz = dz;
    r.ix = recip_saturate(dx);
    r.iy = recip_saturate(dy);
    r.iz = recip_saturate(dz);
    r.nox = -ox * r.ix;
    r.noy = -oy * r.iy;
    r.noz = -oz * r.iz;
    return r;
}

}  // namespace vrad
