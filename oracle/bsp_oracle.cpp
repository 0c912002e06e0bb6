// bsp_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the reference's BSP surface
// tracer (stock vrad's CLightSurface over EnumerateNodesAlongRay), restated
// on the CPU as the checker of the device's walk.
//
// Follows muflub/hl2sdk_tools_sharp, MapTools/Tracing/BspSurfaceTracer.cs:
//   TraceOne                  :233-357  the front-to-back walk, its axial
//                                       shortcut, TEST_EPSILON, one stack
//                                       record per split
//   EnumerateNode             :365-406  on-node faces at the split point,
//                                       lit faces first, then the sky test
//   EnumerateLeaf             :408-464  the leaf's faces: backface cull,
//                                       plane crossing, fraction window
//   TestPointAgainstSurface   :466-482  the lightmap rectangle test
//   TestPointAgainstSkySurface:484-512  the sky winding's same-side test
// in the reference's Correct mode (exact normalise), every float operation
// in its order (built with -ffp-contract=off).  The arrays are the ones
// hl2sdk_tools_sharp_b200/bsp.py builds (BspTraceGeometry.Build).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr float kTestEpsilon = 0.03125f;
constexpr int kMaxStack = 256;

struct Node {
    float nx, ny, nz, dist;
    int32_t child0, child1, first_face, packed;
};
struct Surface {
    float nx, ny, nz, dist, sx, sy, sz, so, tx, ty, tz, to, min_s, min_t, size_s, size_t_;
};
struct Geometry {
    const Node *nodes;
    const Surface *surfaces;
    const int32_t *node_faces;
    const int32_t *leaf_faces;
    const int32_t *leaf_start;
    const int32_t *leaf_count;
    int32_t nleaves;
    const float *sky_points;
    const int32_t *sky_start;
    const int32_t *sky_count;
};
struct Ctx {
    float ox, oy, oz, dx, dy, dz;
    float hit_frac, min_frac;
    int32_t surface;
};
struct V {
    float x, y, z;
};
V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V cross(V a, V b) { return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)}; }
float dot(V a, V b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
V normalise(V a) {
    float len = std::sqrt((a.x * a.x) + (a.y * a.y) + (a.z * a.z));
    if (len == 0.0f) return {0, 0, 0};
    return {a.x / len, a.y / len, a.z / len};
}

bool point_in_surface(const Surface &s, float px, float py, float pz) {
    float sc = (px * s.sx) + (py * s.sy) + (pz * s.sz) + s.so;
    float tc = (px * s.tx) + (py * s.ty) + (pz * s.tz) + s.to;
    if (sc < s.min_s || tc < s.min_t) return false;
    float ds = sc - s.min_s;
    float dt = tc - s.min_t;
    return ds <= s.size_s && dt <= s.size_t_;
}

bool point_in_sky(const Geometry &g, int face, float px, float py, float pz) {
    const int start = g.sky_start[face], count = g.sky_count[face];
    if (count < 2) return false;
    auto P = [&](int i) { return V{g.sky_points[3 * (start + i)], g.sky_points[3 * (start + i) + 1], g.sky_points[3 * (start + i) + 2]}; };
    const V pt{px, py, pz};
    V to_pt = sub(pt, P(0));
    V edge = sub(P(1), P(0));
    const V test = normalise(cross(edge, to_pt));
    for (int i = 1; i < count; i++) {
        to_pt = sub(pt, P(i));
        edge = sub(P((i + 1) % count), P(i));
        const V c = normalise(cross(edge, to_pt));
        if (dot(c, test) < 0.0f) return false;
    }
    return true;
}

bool enumerate_node(const Geometry &g, Ctx &c, int node, float f) {
    const Node &n = g.nodes[node];
    const int solid = n.packed & 0x7FFF;
    const int sky = (n.packed >> 15) & 0x7FFF;
    if ((solid | sky) == 0) return true;
    const float px = c.ox + (f * c.dx), py = c.oy + (f * c.dy), pz = c.oz + (f * c.dz);
    const int32_t *first = g.node_faces + n.first_face;
    for (int i = 0; i < solid; i++) {
        const int face = first[i];
        if (point_in_surface(g.surfaces[face], px, py, pz)) {
            c.hit_frac = f;
            c.surface = face;
            return false;
        }
    }
    int sky_hit = -1;
    for (int i = 0; i < sky; i++) {
        const int face = first[solid + i];
        if (point_in_sky(g, face, px, py, pz)) sky_hit = face;
    }
    c.surface = sky_hit;
    return sky_hit == -1;
}

bool enumerate_leaf(const Geometry &g, Ctx &c, int leaf, float start, float end) {
    if ((unsigned)leaf >= (unsigned)g.nleaves) return true;
    const int count = g.leaf_count[leaf];
    if (count == 0) return true;
    const int32_t *first = g.leaf_faces + g.leaf_start[leaf];
    bool hit = false;
    for (int i = 0; i < count; i++) {
        const int face = first[i];
        const Surface &s = g.surfaces[face];
        const float delta_dot_n = (c.dx * s.nx) + (c.dy * s.ny) + (c.dz * s.nz);
        if (delta_dot_n > 0) continue;
        const float start_dot_n = (c.ox * s.nx) + (c.oy * s.ny) + (c.oz * s.nz);
        const float front = start_dot_n + (start * delta_dot_n) - s.dist;
        const float back = start_dot_n + (end * delta_dot_n) - s.dist;
        const bool side = front < 0;
        if ((back < 0) == side) continue;
        const float f = front / (front - back);
        const float mid = (start * (1.0f - f)) + (end * f);
        if (mid >= c.hit_frac || mid < c.min_frac) continue;
        const float px = c.ox + (mid * c.dx), py = c.oy + (mid * c.dy), pz = c.oz + (mid * c.dz);
        if (point_in_surface(s, px, py, pz)) {
            c.hit_frac = mid;
            c.surface = face;
            hit = true;
        }
    }
    return !hit;
}

struct Entry {
    int visit, far_child;
    float split, end;
};

// Returns 0, or -1 when the walk outgrows its stack.
int trace_one(const Geometry &g, const float *ray, float min_frac, int32_t *face_out, float *frac_out) {
    Ctx c;
    c.ox = ray[0];
    c.oy = ray[1];
    c.oz = ray[2];
    c.dx = ray[3] * ray[6];
    c.dy = ray[4] * ray[6];
    c.dz = ray[5] * ray[6];
    c.hit_frac = 1.0f;
    c.min_frac = min_frac;
    c.surface = -1;
    Entry stack[kMaxStack];
    int sp = 0, node = 0;
    float start = 0.0f, end = 1.0f;
    while (true) {
        while (node >= 0) {
            const Node &n = g.nodes[node];
            float start_dot_n, delta_dot_n;
            const int axis = (int)((uint32_t)n.packed >> 30);
            if (axis == 3) {
                start_dot_n = (c.ox * n.nx) + (c.oy * n.ny) + (c.oz * n.nz);
                delta_dot_n = (c.dx * n.nx) + (c.dy * n.ny) + (c.dz * n.nz);
            } else if (axis == 0) {
                start_dot_n = c.ox;
                delta_dot_n = c.dx;
            } else if (axis == 1) {
                start_dot_n = c.oy;
                delta_dot_n = c.dy;
            } else {
                start_dot_n = c.oz;
                delta_dot_n = c.dz;
            }
            const float front = start_dot_n + (start * delta_dot_n) - n.dist;
            const float back = start_dot_n + (end * delta_dot_n) - n.dist;
            if (front <= -kTestEpsilon && back <= -kTestEpsilon) {
                node = n.child1;
                continue;
            }
            if (front >= kTestEpsilon && back >= kTestEpsilon) {
                node = n.child0;
                continue;
            }
            const bool side = front < 0;
            float splitfrac;
            if (delta_dot_n == 0.0f) {
                splitfrac = 1.0f;
            } else {
                splitfrac = (n.dist - start_dot_n) / delta_dot_n;
                if (splitfrac < 0.0f) splitfrac = 0.0f;
                else if (splitfrac > 1.0f) splitfrac = 1.0f;
            }
            if (sp >= kMaxStack) return -1;
            stack[sp++] = Entry{node, side ? n.child0 : n.child1, splitfrac, end};
            node = side ? n.child1 : n.child0;
            end = splitfrac;
        }
        if (!enumerate_leaf(g, c, -node - 1, start, end)) break;
        if (sp == 0) break;
        const Entry e = stack[--sp];
        if (!enumerate_node(g, c, e.visit, e.split)) break;
        node = e.far_child;
        start = e.split;
        end = e.end;
    }
    *face_out = c.surface;
    *frac_out = c.surface == -1 ? 1.0f : c.hit_frac;
    return 0;
}

}  // namespace

extern "C" {

// The BSP surface tracer over n rays (7 floats: origin, direction, reach;
// the walked delta is direction x reach), all host threads: the face hit
// (-1 for none) and the fraction along the delta (1 for none).
int orc_bsp_trace(const float *nodes, const float *surfaces, const int32_t *node_faces, const int32_t *leaf_faces,
                  const int32_t *leaf_start, const int32_t *leaf_count, int32_t nleaves, const float *sky_points,
                  const int32_t *sky_start, const int32_t *sky_count, const float *rays, int64_t n, float min_frac,
                  int32_t *face_out, float *frac_out, int32_t threads) {
    const Geometry g{reinterpret_cast<const Node *>(nodes), reinterpret_cast<const Surface *>(surfaces), node_faces,
                     leaf_faces, leaf_start, leaf_count, nleaves, sky_points, sky_start, sky_count};
    std::vector<int> rc((size_t)(threads > 0 ? threads : 1), 0);
    std::vector<std::thread> pool;
    const int T = threads > 0 ? threads : 1;
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t]() {
            for (int64_t i = t; i < n; i += T)
                if (trace_one(g, rays + 7 * i, min_frac, face_out + i, frac_out + i) != 0) rc[(size_t)t] = -1;
        });
    for (auto &th : pool) th.join();
    for (int r : rc)
        if (r) return r;
    return 0;
}

}  // extern "C"
