// host_geom.h -- single-precision host geometry shared by the set-up files
// (world.cpp: samples, neighbours, layout; patches.cpp: the patch tree).
//
// Each helper restates a reference routine operation for operation, in
// float, in the reference's association order; the files that include this
// are compiled with -ffp-contract=off, so no multiply-add is fused and the
// results are the reference's bits.
//   Vec3 (Dot, Cross, Length, Normalise)   MapFormats/Geometry/Vec3.cs:92-189
//   WindingArena.RemoveColinearPoints / ClipEpsilon (Classify, SplitPoint) /
//   Area / AreaAndBalancePoint / Bounds / Center
//                                          MapTools/Geometry/WindingArena.cs
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace vrad {
namespace hg {

struct V3 {
    float x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(V3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }
// Vec3.Normalise: an exact length and three true divides; zero stays zero.
inline V3 normalise(V3 a) {
    float l = length(a);
    if (l == 0.0f) return {0.0f, 0.0f, 0.0f};
    return {a.x / l, a.y / l, a.z / l};
}
inline float comp(V3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

using Winding = std::vector<V3>;

constexpr double kColinearDot = 0.999;  // GeometryEpsilons.ColinearDotThreshold

// WindingArena.RemoveColinearPoints.
inline Winding remove_colinear(const Winding &w) {
    const size_t n = w.size();
    Winding kept;
    for (size_t i = 0; i < n; i++) {
        size_t j = (i + 1) % n, k = (i + n - 1) % n;
        V3 v1 = normalise(sub(w[j], w[i]));
        V3 v2 = normalise(sub(w[i], w[k]));
        if ((double)dot(v1, v2) < kColinearDot) kept.push_back(w[i]);
    }
    return kept.size() == n ? w : kept;
}

// WindingArena.ClipEpsilon of the n points at `in` against the axis plane
// p[ax] = dist (normal the unit axis).  front: the d > eps side; back:
// d < -eps; points within eps go to both.  An empty vector is the
// reference's null winding.  `in` must not alias either output.
inline void clip_axis(const V3 *in, size_t n, int ax, float dist, float eps, Winding &front, Winding &back) {
    front.clear();
    back.clear();
    // Windings here have a handful of points: local arrays, a heap
    // fallback only past 63.
    float dist_buf[64];
    int side_buf[64];
    std::vector<float> dist_big;
    std::vector<int> side_big;
    float *dists = dist_buf;
    int *sides = side_buf;  // 0 front, 1 back, 2 on
    if (n + 1 > 64) {
        dist_big.resize(n + 1);
        side_big.resize(n + 1);
        dists = dist_big.data();
        sides = side_big.data();
    }
    int counts[3] = {0, 0, 0};
    const V3 normal = {ax == 0 ? 1.0f : 0.0f, ax == 1 ? 1.0f : 0.0f, ax == 2 ? 1.0f : 0.0f};
    for (size_t i = 0; i < n; i++) {
        float d = dot(in[i], normal);
        d -= dist;
        dists[i] = d;
        sides[i] = d > eps ? 0 : (d < -eps ? 1 : 2);
        counts[sides[i]]++;
    }
    if (n == 0) return;
    sides[n] = sides[0];
    dists[n] = dists[0];
    if (counts[0] == 0) {
        back.assign(in, in + n);
        return;
    }
    if (counts[1] == 0) {
        front.assign(in, in + n);
        return;
    }
    for (size_t i = 0; i < n; i++) {
        const V3 p1 = in[i];
        if (sides[i] == 2) {
            front.push_back(p1);
            back.push_back(p1);
            continue;
        }
        if (sides[i] == 0) front.push_back(p1);
        if (sides[i] == 1) back.push_back(p1);
        if (sides[i + 1] == 2 || sides[i + 1] == sides[i]) continue;
        const V3 p2 = in[(i + 1) % n];
        const float t = dists[i] / (dists[i] - dists[i + 1]);
        auto axis = [&](float nv, float a, float b) {
            if (nv == 1.0f) return dist;
            if (nv == -1.0f) return -dist;
            return a + t * (b - a);
        };
        V3 mid = {axis(normal.x, p1.x, p2.x), axis(normal.y, p1.y, p2.y), axis(normal.z, p1.z, p2.z)};
        front.push_back(mid);
        back.push_back(mid);
    }
}

inline void clip_axis(const Winding &in, int ax, float dist, float eps, Winding &front, Winding &back) {
    clip_axis(in.data(), in.size(), ax, dist, eps, front, back);
}

// WindingArena.Area: fan from point 0, cross lengths summed, halved once.
inline float area(const Winding &p) {
    float total = 0.0f;
    for (size_t i = 2; i < p.size(); i++) total += length(cross(sub(p[i - 1], p[0]), sub(p[i], p[0])));
    return total * 0.5f;
}

// WindingArena.AreaAndBalancePoint.
inline float area_and_balance(const Winding &p, V3 &center) {
    center = {0.0f, 0.0f, 0.0f};
    float total = 0.0f;
    for (size_t i = 2; i < p.size(); i++) {
        V3 d1 = sub(p[i - 1], p[0]);
        V3 d2 = sub(p[i], p[0]);
        float a = length(cross(d1, d2));
        total += a;
        float third = (float)((double)a / 3.0);
        center = add(center, mul(p[i - 1], third));
        center = add(center, mul(p[i], third));
        center = add(center, mul(p[0], third));
    }
    if (total != 0.0f) center = mul(center, (float)(1.0 / (double)total));
    return total * 0.5f;
}

// WindingArena.Bounds: seeds +-99999.
inline void bounds(const Winding &p, V3 &mins, V3 &maxs) {
    mins = {99999.0f, 99999.0f, 99999.0f};
    maxs = {-99999.0f, -99999.0f, -99999.0f};
    for (const V3 &v : p) {
        if (v.x < mins.x) mins.x = v.x;
        if (v.x > maxs.x) maxs.x = v.x;
        if (v.y < mins.y) mins.y = v.y;
        if (v.y > maxs.y) maxs.y = v.y;
        if (v.z < mins.z) mins.z = v.z;
        if (v.z > maxs.z) maxs.z = v.z;
    }
}

// WindingArena.Center: the vertex average, scale (float)(1.0 / count).
inline V3 center(const Winding &p) {
    V3 c = {0.0f, 0.0f, 0.0f};
    for (const V3 &v : p) c = add(v, c);
    return mul(c, (float)(1.0 / (double)p.size()));
}

}  // namespace hg
}  // namespace vrad
