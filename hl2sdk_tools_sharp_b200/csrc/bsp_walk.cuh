// bsp_walk.cuh -- the BSP surface walk as device functions: stock vrad's
// CLightSurface over EnumerateNodesAlongRay, shared by the closest-hit
// kernel (bsp_trace.cu) and the leaf ambient sample (ambient.cu).
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp,
// MapTools/Tracing/BspSurfaceTracer.cs, and its leaf-ambient twin
// MapTools/Rad/Ambient/AmbientRayTracer.cs:107-464):
//   the walk (BspSurfaceTracer.cs:233-357, AmbientRayTracer.cs:148-275):
//     front-to-back over the map's BSP tree, one plane test per node (the
//     axial shortcut reads the component), a ray straddling a node within
//     TEST_EPSILON (1/32) of it descends the near side first with the split
//     pending on a stack;
//   EnumerateLeaf (:408-464 / :330-400): the leaf's faces, backface cull,
//     the crossing fraction inside the leaf's segment and below the best so
//     far, the lightmap rectangle test, whose offsets into the rectangle are
//     the hit's luxel coordinates (m_LuxelCoord);
//   EnumerateNode (:365-406 / :279-328): a pending split's on-node faces at
//     the split point, lit faces first (the first hit ends the walk), then
//     sky faces by their windings (the last that passes ends it; a sky hit
//     has no luxel);
// Correct mode (exact normalise in the sky test), every float operation an
// explicitly rounded intrinsic in the reference's order, so a face, a
// fraction and a luxel coordinate are stock's bits.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bsp_trace.cuh"

namespace vrad {
namespace bspwalk {

constexpr float kTestEpsilon = 0.03125f;  // TEST_EPSILON
constexpr int kStack = 64;

struct Walk {
    float ox, oy, oz, dx, dy, dz;
    float hit_frac, min_frac;
    int32_t surface;
    bool has_luxel;
    float luxel_s, luxel_t;
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// TestPointAgainstSurface: inside the face's lightmap rectangle; ds and dt
// are the point's offsets from the rectangle's mins.
__device__ __forceinline__ bool in_surface(const DeviceBsp &g, int face, float px, float py, float pz, float &ds,
                                           float &dt) {
    const float4 S = __ldg(&g.surfaces[4 * face + 1]), T = __ldg(&g.surfaces[4 * face + 2]),
                 R = __ldg(&g.surfaces[4 * face + 3]);
    const float sc = __fadd_rn(dot3(px, py, pz, S.x, S.y, S.z), S.w);
    const float tc = __fadd_rn(dot3(px, py, pz, T.x, T.y, T.z), T.w);
    if (sc < R.x || tc < R.y) return false;
    ds = __fsub_rn(sc, R.x);
    dt = __fsub_rn(tc, R.y);
    return ds <= R.z && dt <= R.w;
}

__device__ __forceinline__ void normalise3(float &x, float &y, float &z) {
    const float len = __fsqrt_rn(dot3(x, y, z, x, y, z));
    if (len == 0.0f) {
        x = y = z = 0.0f;
        return;
    }
    x = __fdiv_rn(x, len);
    y = __fdiv_rn(y, len);
    z = __fdiv_rn(z, len);
}

// Cross(edge, to_pt), normalised (Vec3.Cross's operand order).
__device__ __forceinline__ void edge_normal(float ex, float ey, float ez, float tx, float ty, float tz, float &cx,
                                            float &cy, float &cz) {
    cx = __fsub_rn(__fmul_rn(ey, tz), __fmul_rn(ez, ty));
    cy = __fsub_rn(__fmul_rn(ez, tx), __fmul_rn(ex, tz));
    cz = __fsub_rn(__fmul_rn(ex, ty), __fmul_rn(ey, tx));
    normalise3(cx, cy, cz);
}

// TestPointAgainstSkySurface: every edge's normal on the first edge's side.
__device__ inline bool in_sky(const DeviceBsp &g, int face, float px, float py, float pz) {
    const int2 run = __ldg(&g.sky_run[face]);
    if (run.y < 2) return false;
    const float4 *p = g.sky_points + run.x;
    const float4 p0 = __ldg(&p[0]), p1 = __ldg(&p[1]);
    float ax, ay, az;
    edge_normal(__fsub_rn(p1.x, p0.x), __fsub_rn(p1.y, p0.y), __fsub_rn(p1.z, p0.z), __fsub_rn(px, p0.x),
                __fsub_rn(py, p0.y), __fsub_rn(pz, p0.z), ax, ay, az);
    for (int i = 1; i < run.y; i++) {
        const float4 a = __ldg(&p[i]), b = __ldg(&p[(i + 1) % run.y]);
        float cx, cy, cz;
        edge_normal(__fsub_rn(b.x, a.x), __fsub_rn(b.y, a.y), __fsub_rn(b.z, a.z), __fsub_rn(px, a.x),
                    __fsub_rn(py, a.y), __fsub_rn(pz, a.z), cx, cy, cz);
        if (dot3(cx, cy, cz, ax, ay, az) < 0.0f) return false;
    }
    return true;
}

// EnumerateNode: false ends the walk.
__device__ inline bool visit_node(const DeviceBsp &g, Walk &c, int node, float f) {
    const float4 B = __ldg(&g.nodes[2 * node + 1]);
    const int packed = __float_as_int(B.w);
    const int solid = packed & 0x7FFF, sky = (packed >> 15) & 0x7FFF;
    if ((solid | sky) == 0) return true;
    const float px = __fadd_rn(c.ox, __fmul_rn(f, c.dx)), py = __fadd_rn(c.oy, __fmul_rn(f, c.dy)),
                pz = __fadd_rn(c.oz, __fmul_rn(f, c.dz));
    const int32_t *first = g.node_faces + __float_as_int(B.z);
    for (int i = 0; i < solid; i++) {
        const int face = __ldg(&first[i]);
        float ds, dt;
        if (in_surface(g, face, px, py, pz, ds, dt)) {
            c.hit_frac = f;
            c.surface = face;
            c.has_luxel = true;
            c.luxel_s = ds;
            c.luxel_t = dt;
            return false;
        }
    }
    int sky_hit = -1;
    for (int i = 0; i < sky; i++) {
        const int face = __ldg(&first[solid + i]);
        if (in_sky(g, face, px, py, pz)) sky_hit = face;
    }
    c.surface = sky_hit;
    return sky_hit == -1;
}

// EnumerateLeaf: false ends the walk.
__device__ inline bool visit_leaf(const DeviceBsp &g, Walk &c, int leaf, float start, float end) {
    if ((unsigned)leaf >= (unsigned)g.nleaves) return true;
    const int2 run = __ldg(&g.leaf_run[leaf]);
    bool hit = false;
    for (int i = 0; i < run.y; i++) {
        const int face = __ldg(&g.leaf_faces[run.x + i]);
        const float4 P = __ldg(&g.surfaces[4 * face]);
        const float ddn = dot3(c.dx, c.dy, c.dz, P.x, P.y, P.z);
        if (ddn > 0.0f) continue;
        const float sdn = dot3(c.ox, c.oy, c.oz, P.x, P.y, P.z);
        const float front = __fsub_rn(__fadd_rn(sdn, __fmul_rn(start, ddn)), P.w);
        const float back = __fsub_rn(__fadd_rn(sdn, __fmul_rn(end, ddn)), P.w);
        const bool side = front < 0.0f;
        if ((back < 0.0f) == side) continue;
        const float f = __fdiv_rn(front, __fsub_rn(front, back));
        const float mid = __fadd_rn(__fmul_rn(start, __fsub_rn(1.0f, f)), __fmul_rn(end, f));
        if (mid >= c.hit_frac || mid < c.min_frac) continue;
        const float px = __fadd_rn(c.ox, __fmul_rn(mid, c.dx)), py = __fadd_rn(c.oy, __fmul_rn(mid, c.dy)),
                    pz = __fadd_rn(c.oz, __fmul_rn(mid, c.dz));
        float ds, dt;
        if (in_surface(g, face, px, py, pz, ds, dt)) {
            c.hit_frac = mid;
            c.surface = face;
            c.has_luxel = true;
            c.luxel_s = ds;
            c.luxel_t = dt;
            hit = true;
        }
    }
    return !hit;
}

struct Pending {
    int visit, far_child;
    float split, end;
};

// The whole walk from c's origin along c's delta.  Returns false when the
// walk needed more than kStack pending splits (c then holds no answer).
__device__ inline bool walk(const DeviceBsp &g, Walk &c) {
    Pending stack[kStack];
    int sp = 0, node = 0;
    float start = 0.0f, end = 1.0f;
    while (true) {
        while (node >= 0) {
            const float4 A = __ldg(&g.nodes[2 * node]), B = __ldg(&g.nodes[2 * node + 1]);
            const int packed = __float_as_int(B.w);
            const unsigned axis = (unsigned)packed >> 30;
            float sdn, ddn;
            if (axis == 3) {
                sdn = dot3(c.ox, c.oy, c.oz, A.x, A.y, A.z);
                ddn = dot3(c.dx, c.dy, c.dz, A.x, A.y, A.z);
            } else if (axis == 0) {
                sdn = c.ox;
                ddn = c.dx;
            } else if (axis == 1) {
                sdn = c.oy;
                ddn = c.dy;
            } else {
                sdn = c.oz;
                ddn = c.dz;
            }
            const float front = __fsub_rn(__fadd_rn(sdn, __fmul_rn(start, ddn)), A.w);
            const float back = __fsub_rn(__fadd_rn(sdn, __fmul_rn(end, ddn)), A.w);
            const int child0 = __float_as_int(B.x), child1 = __float_as_int(B.y);
            if (front <= -kTestEpsilon && back <= -kTestEpsilon) {
                node = child1;
                continue;
            }
            if (front >= kTestEpsilon && back >= kTestEpsilon) {
                node = child0;
                continue;
            }
            const bool side = front < 0.0f;
            float split;
            if (ddn == 0.0f) {
                split = 1.0f;
            } else {
                split = __fdiv_rn(__fsub_rn(A.w, sdn), ddn);
                if (split < 0.0f) split = 0.0f;
                else if (split > 1.0f) split = 1.0f;
            }
            if (sp >= kStack) return false;
            stack[sp++] = Pending{node, side ? child0 : child1, split, end};
            node = side ? child1 : child0;
            end = split;
        }
        if (!visit_leaf(g, c, -node - 1, start, end)) return true;
        if (sp == 0) return true;
        const Pending e = stack[--sp];
        if (!visit_node(g, c, e.visit, e.split)) return true;
        node = e.far_child;
        start = e.split;
        end = e.end;
    }
}

}  // namespace bspwalk
}  // namespace vrad
