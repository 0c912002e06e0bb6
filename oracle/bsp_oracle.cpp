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
    bool has_luxel;
    float luxel_s, luxel_t;  // m_LuxelCoord, from the lightmap rectangle test
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

bool point_in_surface(const Surface &s, float px, float py, float pz, float *ds_out = nullptr,
                      float *dt_out = nullptr) {
    float sc = (px * s.sx) + (py * s.sy) + (pz * s.sz) + s.so;
    float tc = (px * s.tx) + (py * s.ty) + (pz * s.tz) + s.to;
    if (sc < s.min_s || tc < s.min_t) return false;
    float ds = sc - s.min_s;
    float dt = tc - s.min_t;
    if (ds_out) *ds_out = ds;
    if (dt_out) *dt_out = dt;
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
        float ds, dt;
        if (point_in_surface(g.surfaces[face], px, py, pz, &ds, &dt)) {
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
        float ds, dt;
        if (point_in_surface(s, px, py, pz, &ds, &dt)) {
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

struct Entry {
    int visit, far_child;
    float split, end;
};

// The walk along c's delta; returns 0, or -1 when it outgrows its stack.
int walk(const Geometry &g, Ctx &c) {
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
    return 0;
}

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
    c.has_luxel = false;
    c.luxel_s = c.luxel_t = 0.0f;
    if (walk(g, c) != 0) return -1;
    *face_out = c.surface;
    *frac_out = c.surface == -1 ? 1.0f : c.hit_frac;
    return 0;
}

// ---- The leaf ambient sample (AmbientSampler.ComputeRayCube) ----------
//
// Follows MapTools/Rad/Ambient:
//   AmbientSampler.ComputeRayCube  AmbientSampler.cs:211-227
//   RayAmbientLighting.Accumulate  RayAmbientLighting.cs:89-134
//   AddFaceAverage                 RayAmbientLighting.cs:196-226
//   AddFacePointSample             RayAmbientLighting.cs:241-291
//   RemapValClamped                RayAmbientLighting.cs:319-330
//   AmbientCube.Project            AmbientCube.cs:80-103
//   StockLightColor.TexLightToLinear, Power2N  StockLightColor.cs:69-78, 262-271

struct AmbientFace {  // the product's vrad_ambient_face, 88 bytes
    int32_t lightofs, smax, tmax, stride, nstyles;
    uint32_t styles;
    int32_t flags;
    float refl[3];
    float avg[4][3];
};
static_assert(sizeof(AmbientFace) == 88, "face record");

struct AmbientLight {
    const AmbientFace *faces;
    const uint8_t *light;
    int64_t bytes;
    const float *dirs;
    float tan_theta;
    bool has_sky;
    float sky[3];
    float p2n[256];
};

float remap_clamped(float val, float a, float b, float c, float d) {
    if (a == b) return d;
    float cv = (val - a) / (b - a);
    cv = cv < 0.0f ? 0.0f : (cv > 1.0f ? 1.0f : cv);
    return c + ((d - c) * cv);
}

// One ray's style-0 colour; 0, or -1 (stack), -2 (bad averages), -3 (outside the lump).
int ambient_ray(const Geometry &g, const AmbientLight &A, const float *start, const float *dir, float *col) {
    const float RayLength = 32768.0f * 1.74f;
    const float end[3] = {start[0] + (dir[0] * RayLength), start[1] + (dir[1] * RayLength),
                          start[2] + (dir[2] * RayLength)};
    Ctx c;
    c.ox = start[0];
    c.oy = start[1];
    c.oz = start[2];
    c.dx = end[0] - start[0];
    c.dy = end[1] - start[1];
    c.dz = end[2] - start[2];
    c.hit_frac = 1.0f;
    c.min_frac = 0.0f;
    c.surface = -1;
    c.has_luxel = false;
    c.luxel_s = c.luxel_t = 0.0f;
    col[0] = col[1] = col[2] = 0.0f;
    if (walk(g, c) != 0) return -1;
    if (c.surface < 0) return 0;
    const AmbientFace &F = A.faces[c.surface];
    const float len = std::sqrt((c.dx * c.dx) + (c.dy * c.dy) + (c.dz * c.dz));
    const float dist = len * A.tan_theta * c.hit_frac;
    float scale_avg = remap_clamped(dist, 20.0f, 40.0f, 0.0f, 1.0f);
    if (!c.has_luxel) scale_avg = 1.0f;
    const float scale_sample = 1.0f - scale_avg;
    auto style = [&](int m) { return (int)((F.styles >> (8 * m)) & 0xFF); };
    if (scale_avg != 0) {
        if (F.flags & 1) {
            if (A.has_sky)
                for (int k = 0; k < 3; k++) col[k] += A.sky[k] * scale_avg;
        } else {
            if (F.flags & 2) return -2;
            for (int m = 0; m < F.nstyles; m++)
                if (style(m) == 0)
                    for (int k = 0; k < 3; k++) col[k] += F.avg[m][k] * scale_avg;
        }
    }
    if (scale_sample != 0 && F.lightofs != -1) {
        if (F.smax - 1 < 0 || F.tmax - 1 < 0) return -3;  // Math.Clamp's max below its min
        int ds = (int)c.luxel_s, dt = (int)c.luxel_t;
        ds = ds < 0 ? 0 : (ds > F.smax - 1 ? F.smax - 1 : ds);
        dt = dt < 0 ? 0 : (dt > F.tmax - 1 ? F.tmax - 1 : dt);
        const int32_t index = (dt * F.smax) + ds;
        for (int m = 0; m < F.nstyles; m++) {
            const int32_t offset = (int32_t)((uint32_t)F.lightofs + ((uint32_t)index + (uint32_t)m * (uint32_t)F.stride) * 4u);
            if (A.bytes < 4 || (uint32_t)offset > (uint32_t)(int32_t)(A.bytes - 4)) return -3;
            const uint8_t *p = A.light + (uint32_t)offset;
            const float e = A.p2n[(int)(int8_t)p[3] + 128];
            float v[3] = {(float)p[0] * e, (float)p[1] * e, (float)p[2] * e};
            if (F.flags & 1) {
                if (A.has_sky)
                    for (int k = 0; k < 3; k++) v[k] = A.sky[k];
            } else {
                for (int k = 0; k < 3; k++) v[k] = v[k] * F.refl[k];
            }
            if (style(m) == 0)
                for (int k = 0; k < 3; k++) col[k] += v[k] * scale_sample;
        }
    }
    return 0;
}

// AmbientCube.Project of the 162 colours onto sides +x, -x, +y, -y, +z, -z.
void project(const float *rad, const float *dirs, float *cube) {
    static const float box[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int j = 6; --j >= 0;) {
        float t = 0, sum[3] = {0, 0, 0};
        for (int i = 0; i < 162; i++) {
            const float *a = dirs + 3 * i;
            const float c = (a[0] * box[j][0]) + (a[1] * box[j][1]) + (a[2] * box[j][2]);
            if (c > 0) {
                t += c;
                for (int k = 0; k < 3; k++) sum[k] += rad[3 * i + k] * c;
            }
        }
        const float inv = 1 / t;
        for (int k = 0; k < 3; k++) cube[3 * j + k] = sum[k] * inv;
    }
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

// The ray cubes at n positions (3 floats each) into cubes (n x 6 x 3), all
// host threads: 0, or the first failure (-1 stack, -2 bad averages, -3 a
// luxel outside the lump).
int orc_ambient_cubes(const float *nodes, const float *surfaces, const int32_t *node_faces, const int32_t *leaf_faces,
                      const int32_t *leaf_start, const int32_t *leaf_count, int32_t nleaves, const float *sky_points,
                      const int32_t *sky_start, const int32_t *sky_count, const void *faces, const uint8_t *light,
                      int64_t light_bytes, const float *dirs, float tan_theta, int32_t has_sky, const float *sky,
                      const float *positions, int64_t n, float *cubes, int32_t threads) {
    const Geometry g{reinterpret_cast<const Node *>(nodes), reinterpret_cast<const Surface *>(surfaces), node_faces,
                     leaf_faces, leaf_start, leaf_count, nleaves, sky_points, sky_start, sky_count};
    AmbientLight A;
    A.faces = reinterpret_cast<const AmbientFace *>(faces);
    A.light = light;
    A.bytes = light_bytes;
    A.dirs = dirs;
    A.tan_theta = tan_theta;
    A.has_sky = has_sky != 0;
    for (int k = 0; k < 3; k++) A.sky[k] = sky[k];
    for (int k = 0; k < 256; k++) A.p2n[k] = (float)(std::ldexp(1.0, k - 128) / 255.0);
    const int T = threads > 0 ? threads : 1;
    std::vector<int> rc((size_t)T, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t]() {
            std::vector<float> rad(3 * 162);
            for (int64_t s = t; s < n; s += T) {
                for (int i = 0; i < 162; i++) {
                    const int r = ambient_ray(g, A, positions + 3 * s, dirs + 3 * i, &rad[3 * (size_t)i]);
                    if (r && !rc[(size_t)t]) rc[(size_t)t] = r;
                }
                project(rad.data(), dirs, cubes + 18 * s);
            }
        });
    for (auto &th : pool) th.join();
    for (int r : rc)
        if (r) return r;
    return 0;
}

}  // extern "C"
