// tracer_oracle.cpp -- CPU oracle: the KD tracer's triangle format, its hit
// predicate, its four-lane packet traversal, a brute-force tracer with the
// same predicate, and an FP64 geometric classifier.
//
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).  Compiled with
// -ffp-contract=off so every float operation rounds where the reference's
// does; the order of operations below is the reference's.

#include "vrad_oracle.h"
#include "oracle_internal.h"

#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr float kEps = 1.0e-10f;              // KdRayTracer "FourZeros"/epsilons (KdRayTracer.cs:1209-1230)
constexpr float kHuge = 1.0e23f;              // initial hit distance (KdRayTracer.cs:985)
constexpr float kZeroSubstitute = 8.6736174e-19f;  // 2^-60, CorrectZeroSubstitute (KdRayTracer.cs:193)

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float bitsf(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// SseLanes.Max / Min (Tracing/SseLanes.cs): maxps/minps return the SECOND
// operand unless the first compares strictly greater / less.
inline float sse_max(float a, float b) { return a > b ? a : b; }
inline float sse_min(float a, float b) { return a < b ? a : b; }

// ReciprocalSaturateExact (KdRayTracer.cs:1446): zeros (either sign) become
// +-2^-60 by OR-ing the substitute's bits in, then an IEEE divide.
inline float recip_saturate_exact(float a) {
    float safe = a;
    if (a == 0.0f) safe = bitsf(fbits(a) | fbits(kZeroSubstitute));
    return 1.0f / safe;
}

// Vec3.Normalise (MapFormats/Geometry/Vec3.cs:178-189): length by
// sqrt((x*x + y*y) + z*z), zero stays zero, three divides.
inline void normalise_exact(const float v[3], float out[3]) {
    float len = std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    if (len == 0.0f) {
        out[0] = out[1] = out[2] = 0.0f;
        return;
    }
    out[0] = v[0] / len;
    out[1] = v[1] / len;
    out[2] = v[2] / len;
}

// KdTreeBuilder.GetEdgeEquation (KdTreeBuilder.cs:1530-1552).
inline void edge_equation(const float p1[3], const float p2[3], int c1, int c2,
                          const float inside[3], float out[3]) {
    float nx = p1[c2] - p2[c2];
    float ny = p2[c1] - p1[c1];
    float d = -((nx * p1[c1]) + (ny * p1[c2]));
    float trial = ((inside[c1] * nx) + (inside[c2] * ny)) + d;
    if (trial < 0) {
        nx = -nx;
        ny = -ny;
        d = -d;
        trial = -trial;
    }
    out[0] = nx / trial;
    out[1] = ny / trial;
    out[2] = d / trial;
}

// One lane of KdRayTracer.IntersectTriangle (KdRayTracer.cs:1194-1267).
// Returns true and writes *t when the triangle is accepted against `best`.
inline bool intersect(const orc_tri &tri, const float o[3], const float dvec[3], float best,
                      float *t_out) {
    float ddotn = dvec[0] * tri.nx;
    ddotn = (dvec[1] * tri.ny) + ddotn;
    ddotn = (dvec[2] * tri.nz) + ddotn;
    bool hit = (ddotn > kEps) || (ddotn < -kEps);
    float odotn = o[0] * tri.nx;
    odotn = (o[1] * tri.ny) + odotn;
    odotn = (o[2] * tri.nz) + odotn;
    float t = (tri.d - odotn) / ddotn;
    hit = hit && (t > kEps) && (t < best);
    if (!hit) return false;
    float h1 = o[tri.cs0] + t * dvec[tri.cs0];
    float h2 = o[tri.cs1] + t * dvec[tri.cs1];
    float b0 = tri.e[0] * h1;
    b0 = b0 + tri.e[1] * h2;
    b0 = b0 + tri.e[2];
    if (!(b0 >= kEps)) return false;
    float b1 = tri.e[3] * h1;
    b1 = b1 + tri.e[4] * h2;
    b1 = b1 + tri.e[5];
    if (!(b1 >= kEps)) return false;
    float b2 = b1 + b0;
    if (!(b2 <= 1.0f)) return false;
    *t_out = t;
    return true;
}

// A four-lane packet, lanes as plain arrays.
struct Packet {
    float o[3][4];
    float d[3][4];
};

struct StackEntry {
    int node;
    float tmin[4];
    float tmax[4];
};

struct KdScene {
    const orc_kdnode *nodes;
    const int32_t *indices;
    const orc_tri *tris;
    float mn[3], mx[3];
};

// KdRayTracer.TraceSameSigns (KdRayTracer.cs:969-1182): the packet walk
// for four rays whose direction signs agree.  The mailbox is omitted: it
// only skips re-testing a triangle, which cannot change a lane's answer
// (a retest compares against a distance that has only shrunk).
void trace_same_signs(const KdScene &s, const Packet &p, const float tmin_in[4],
                      const float tmax_in[4], int sign_mask, int skip_id, int settled,
                      float out_dist[4], int out_ids[4], std::vector<StackEntry> &stack) {
    float dist[4], tmin[4], tmax[4], reach[4], inv[3][4];
    int ids[4];
    for (int l = 0; l < 4; l++) {
        dist[l] = kHuge;
        ids[l] = -1;
        tmin[l] = tmin_in[l];
        tmax[l] = tmax_in[l];
        reach[l] = tmax_in[l];
        for (int a = 0; a < 3; a++) inv[a][l] = recip_saturate_exact(p.d[a][l]);
    }
    // ClipAxis (KdRayTracer.cs:1454) on each axis of the scene bounds.
    for (int a = 0; a < 3; a++) {
        for (int l = 0; l < 4; l++) {
            float i0 = (s.mn[a] - p.o[a][l]) * inv[a][l];
            float i1 = (s.mx[a] - p.o[a][l]) * inv[a][l];
            tmin[l] = sse_max(tmin[l], sse_min(i0, i1));
            tmax[l] = sse_min(tmax[l], sse_max(i0, i1));
        }
    }
    bool any = false;
    for (int l = 0; l < 4; l++) any |= tmin[l] <= tmax[l];
    if (!any) {
        for (int l = 0; l < 4; l++) {
            out_dist[l] = dist[l];
            out_ids[l] = ids[l];
        }
        return;
    }

    stack.clear();
    int node = 0;
    while (true) {
        orc_kdnode n = s.nodes[node];
        while ((n.children & 3) != 3) {
            int axis = n.children & 3;
            int left = n.children >> 2;
            int front = (sign_mask >> axis) & 1;
            float dtp[4];
            bool hits_front = false, hits_back = false;
            for (int l = 0; l < 4; l++) {
                dtp[l] = (n.split - p.o[axis][l]) * inv[axis][l];
                bool active = tmin[l] <= tmax[l];
                hits_front |= active && (dtp[l] >= tmin[l]);
            }
            if (!hits_front) {
                node = left + (1 - front);
                for (int l = 0; l < 4; l++) tmin[l] = sse_max(tmin[l], dtp[l]);
                n = s.nodes[node];
                continue;
            }
            for (int l = 0; l < 4; l++) {
                bool active = tmin[l] <= tmax[l];
                hits_back |= active && (dtp[l] <= tmax[l]);
            }
            if (!hits_back) {
                node = left + front;
                for (int l = 0; l < 4; l++) tmax[l] = sse_min(tmax[l], dtp[l]);
                n = s.nodes[node];
                continue;
            }
            StackEntry e;
            e.node = left + (1 - front);
            for (int l = 0; l < 4; l++) {
                e.tmin[l] = sse_max(tmin[l], dtp[l]);
                e.tmax[l] = tmax[l];
            }
            stack.push_back(e);
            node = left + front;
            for (int l = 0; l < 4; l++) tmax[l] = sse_min(tmax[l], dtp[l]);
            n = s.nodes[node];
        }

        int ntris = (int)fbits(n.split);
        if (ntris != 0) {
            int start = n.children >> 2;
            for (int k = 0; k < ntris; k++) {
                int tnum = s.indices[start + k];
                const orc_tri &tri = s.tris[tnum];
                if (skip_id != -1 && tri.id == skip_id) continue;
                for (int l = 0; l < 4; l++) {
                    float o[3] = {p.o[0][l], p.o[1][l], p.o[2][l]};
                    float dv[3] = {p.d[0][l], p.d[1][l], p.d[2][l]};
                    float t;
                    if (intersect(tri, o, dv, dist[l], &t)) {
                        dist[l] = t;
                        ids[l] = tnum;
                    }
                }
            }
            bool some_beyond = false;  // movemask(tmax <= distance) != 0
            for (int l = 0; l < 4; l++) some_beyond |= tmax[l] <= dist[l];
            if (!some_beyond) break;
            if (settled >= 0) {
                int blocked = 0;
                for (int l = 0; l < 4; l++)
                    if (ids[l] > -1 && dist[l] < reach[l]) blocked |= 1 << l;
                if ((blocked | settled) == 0xF) break;
            }
        }
        if (stack.empty()) break;
        StackEntry e = stack.back();
        stack.pop_back();
        node = e.node;
        for (int l = 0; l < 4; l++) {
            tmin[l] = e.tmin[l];
            tmax[l] = e.tmax[l];
        }
    }
    for (int l = 0; l < 4; l++) {
        out_dist[l] = dist[l];
        out_ids[l] = ids[l];
    }
}

inline int sign_bit(float f) { return (int)(fbits(f) >> 31); }

// KdRayTracer.Trace4Rays (KdRayTracer.cs:868-935): uniform signs walk once;
// otherwise up to four passes, each broadcasting one lane's direction into
// the lanes that do not share its sign code.
void trace4(const KdScene &s, const Packet &p, const float tmin[4], const float tmax[4],
            int skip_id, bool settle, float out_dist[4], int out_ids[4],
            std::vector<StackEntry> &stack) {
    int code[4];
    for (int l = 0; l < 4; l++)
        code[l] = sign_bit(p.d[0][l]) | (sign_bit(p.d[1][l]) << 1) | (sign_bit(p.d[2][l]) << 2);
    bool uniform = code[0] == code[1] && code[1] == code[2] && code[2] == code[3];
    if (uniform) {
        trace_same_signs(s, p, tmin, tmax, code[0], skip_id, settle ? 0 : -1, out_dist, out_ids,
                         stack);
        return;
    }
    for (int l = 0; l < 4; l++) {
        out_dist[l] = kHuge;
        out_ids[l] = -1;
    }
    int need = 0xF;
    for (int tr = 0; tr < 4; tr++) {
        if (!(need & (1 << tr))) continue;
        int c = code[tr];
        int own = 0;
        for (int l = tr; l < 4; l++)
            if ((need & (1 << l)) && code[l] == c) own |= 1 << l;
        need &= ~own;
        Packet tmp = p;
        for (int l = 0; l < 4; l++) {
            if (own & (1 << l)) continue;
            for (int a = 0; a < 3; a++) tmp.d[a][l] = p.d[a][tr];
        }
        float sd[4];
        int si[4];
        trace_same_signs(s, tmp, tmin, tmax, c, skip_id, settle ? (~own & 0xF) : -1, sd, si,
                         stack);
        for (int l = 0; l < 4; l++) {
            if (own & (1 << l)) {
                out_dist[l] = sd[l];
                out_ids[l] = si[l];
            }
        }
    }
}

void load_packet(const orc_ray *rays, int32_t n, int32_t first, bool isolated, Packet &p,
                 float reach[4]) {
    for (int l = 0; l < 4; l++) {
        int idx = isolated ? first : (first + l < n ? first + l : n - 1);
        const orc_ray &r = rays[idx];
        p.o[0][l] = r.ox;
        p.o[1][l] = r.oy;
        p.o[2][l] = r.oz;
        p.d[0][l] = r.dx;
        p.d[1][l] = r.dy;
        p.d[2][l] = r.dz;
        reach[l] = r.reach;
    }
}

template <class F>
void parallel_for(int32_t n, int32_t threads, F &&f) {
    if (threads <= 1 || n < 1024) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    int32_t chunk = (n + threads - 1) / threads;
    chunk = (chunk + 63) & ~63;  // whole 64-ray words per worker
    for (int32_t t = 0; t < threads; t++) {
        int32_t b = t * chunk, e = std::min<int32_t>(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&f, b, e] { f(b, e); });
    }
    for (auto &th : pool) th.join();
}

}  // namespace

// One segment, traced alone (a packet of four copies, as the reference's
// TraceIsolated does, KdRayTracer.cs:609-625); true when blocked short of
// its reach (sky_pass: when its first hit is opaque).
bool orc_kd_segment_blocked(const OrcKd &kd, const orc_ray &r, bool sky_pass) {
    thread_local std::vector<StackEntry> stack;
    KdScene s{kd.nodes, kd.indices, kd.tris, {kd.bounds[0], kd.bounds[1], kd.bounds[2]},
              {kd.bounds[3], kd.bounds[4], kd.bounds[5]}};
    Packet p;
    float reach[4];
    load_packet(&r, 1, 0, true, p, reach);
    float tmin4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float dist[4];
    int ids[4];
    trace4(s, p, tmin4, reach, -1, !sky_pass, dist, ids, stack);
    bool blocked = ids[0] > -1 && dist[0] < r.reach;
    if (sky_pass && blocked && (kd.tris[ids[0]].id & ORC_TRACE_ID_SKY)) blocked = false;
    return blocked;
}

extern "C" int orc_tri_prepare(const float *v9, const int32_t *ids, const uint8_t *flags,
                               int32_t n, orc_tri *out) {
    if (n < 0 || (n > 0 && (!v9 || !out))) return -1;
    // KdTreeBuilder.ToIntersectionFormat (KdTreeBuilder.cs:1566-1610), Correct side.
    for (int32_t i = 0; i < n; i++) {
        const float *p1 = v9 + 9 * i, *p2 = p1 + 3, *p3 = p1 + 6;
        float e1[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
        float e2[3] = {p3[0] - p1[0], p3[1] - p1[1], p3[2] - p1[2]};
        // Vec3.Cross (MapFormats/Geometry/Vec3.cs): (a.y*b.z - a.z*b.y, ...).
        float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                      e1[0] * e2[1] - e1[1] * e2[0]};
        float nrm[3];
        normalise_exact(c, nrm);
        int drop = 0;
        for (int k = 1; k < 3; k++)
            if (std::fabs(nrm[k]) > std::fabs(nrm[drop])) drop = k;
        int cs0 = (drop + 1) % 3, cs1 = (drop + 2) % 3;
        float eq1[3], eq2[3];
        edge_equation(p1, p2, cs0, cs1, p3, eq1);
        edge_equation(p2, p3, cs0, cs1, p1, eq2);
        orc_tri &t = out[i];
        t.nx = nrm[0];
        t.ny = nrm[1];
        t.nz = nrm[2];
        // Vec3.Dot: (a.x*b.x + a.y*b.y) + a.z*b.z.
        t.d = (nrm[0] * p1[0] + nrm[1] * p1[1]) + nrm[2] * p1[2];
        t.id = ids ? ids[i] : i;
        t.e[0] = eq1[0];
        t.e[1] = eq1[1];
        t.e[2] = eq1[2];
        t.e[3] = eq2[0];
        t.e[4] = eq2[1];
        t.e[5] = eq2[2];
        t.cs0 = (uint8_t)cs0;
        t.cs1 = (uint8_t)cs1;
        t.flags = flags ? flags[i] : 0;
        t.unused = 0;
    }
    return 0;
}

extern "C" int orc_kd_trace(const orc_kdnode *nodes, int32_t nnodes, const int32_t *indices,
                            int32_t nindices, const orc_tri *tris, int32_t ntris,
                            const float *bounds6, const orc_ray *rays, int32_t nrays, float tmin,
                            int32_t skip_id, int32_t flags, int32_t *out_tri, float *out_dist,
                            uint64_t *out_bits, int32_t threads) {
    if (nnodes <= 0 || !nodes || !tris || !bounds6 || nrays < 0) return -1;
    (void)nindices;
    (void)ntris;
    KdScene s{nodes, indices, tris, {bounds6[0], bounds6[1], bounds6[2]},
              {bounds6[3], bounds6[4], bounds6[5]}};
    const bool closest = flags & ORC_CLOSEST;
    const bool isolated = flags & ORC_ISOLATED;
    const bool sky = flags & ORC_SKY_PASS;
    const bool full_walk = flags & ORC_FULL_WALK;
    if (out_bits)
        std::memset(out_bits, 0, sizeof(uint64_t) * (size_t)((nrays + 63) / 64));
    const int step = isolated ? 1 : 4;
    // Workers take whole 64-ray words, so packets of four never straddle
    // two workers and no bit word is shared.
    parallel_for(nrays, threads, [&](int32_t b, int32_t e) {
        std::vector<StackEntry> stack;
        stack.reserve(64);
        float tmin4[4] = {tmin, tmin, tmin, tmin};
        for (int32_t i = b; i < e; i += step) {
            Packet p;
            float reach[4];
            load_packet(rays, e, i, isolated, p, reach);
            // settle: visibility without sky pass-through stops once blocked
            // (KdRayTracer.cs:730-737, 590-596); closest never settles.
            bool settle = !closest && !full_walk && !sky;
            float dist[4];
            int ids[4];
            trace4(s, p, tmin4, reach, skip_id, settle, dist, ids, stack);
            for (int l = 0; l < step && i + l < e; l++) {
                int id = ids[l];
                if (out_tri) out_tri[i + l] = id;
                if (out_dist) out_dist[i + l] = dist[l];
                if (!closest && out_bits) {
                    bool blocked = id > -1 && dist[l] < reach[l];
                    if (sky && id >= 0 && (tris[id].id & ORC_TRACE_ID_SKY)) blocked = false;
                    if (blocked) out_bits[(i + l) >> 6] |= 1ull << ((i + l) & 63);
                }
            }
        }
    });
    return 0;
}

extern "C" int orc_brute_trace(const orc_tri *tris, int32_t ntris, const orc_ray *rays,
                               int32_t nrays, float tmin, int32_t skip_id, int32_t flags,
                               int32_t *out_tri, float *out_dist, uint64_t *out_bits,
                               int32_t threads) {
    if (nrays < 0 || ntris < 0 || (nrays > 0 && !rays)) return -1;
    const bool closest = flags & ORC_CLOSEST;
    const bool sky = flags & ORC_SKY_PASS;
    if (out_bits)
        std::memset(out_bits, 0, sizeof(uint64_t) * (size_t)((nrays + 63) / 64));
    parallel_for(nrays, threads, [&](int32_t b, int32_t e) {
        for (int32_t i = b; i < e; i++) {
            const orc_ray &r = rays[i];
            float o[3] = {r.ox, r.oy, r.oz}, d[3] = {r.dx, r.dy, r.dz};
            float best = kHuge;
            int best_id = -1;
            bool need_first = closest || sky;
            for (int32_t k = 0; k < ntris; k++) {
                const orc_tri &tri = tris[k];
                if (skip_id != -1 && tri.id == skip_id) continue;
                float t;
                // Accept against +inf so the reach / tmin window decides,
                // then keep the lexicographic minimum of (t, index).
                if (!intersect(tri, o, d, kHuge, &t)) continue;
                if (!(t >= tmin) || !(t < r.reach)) continue;
                if (t < best) {
                    best = t;
                    best_id = k;
                    if (!need_first) break;
                }
            }
            if (out_tri) out_tri[i] = best_id;
            if (out_dist) out_dist[i] = best;
            if (out_bits && !closest) {
                bool blocked = best_id >= 0;
                if (sky && blocked && (tris[best_id].id & ORC_TRACE_ID_SKY)) blocked = false;
                if (blocked) out_bits[i >> 6] |= 1ull << (i & 63);
            }
        }
    });
    return 0;
}

// FP64 ground truth for the segment test, Moller-Trumbore in double over
// the original vertices.  Used to classify rays whose FP32 answers differ
// between tracers: the reference's GPU parity gate arbitrates the same way
// (Tests/MapTools/Tracing/VulkanRayTracerFacts.cs:1215-1300).
extern "C" int orc_fp64_classify(const float *v9, int32_t ntris, const orc_ray *rays,
                                 int32_t nrays, double rel_margin, int8_t *out_class,
                                 int32_t threads) {
    if (nrays < 0 || ntris < 0 || !out_class) return -1;
    parallel_for(nrays, threads, [&](int32_t b, int32_t e) {
        for (int32_t i = b; i < e; i++) {
            const orc_ray &r = rays[i];
            double o[3] = {r.ox, r.oy, r.oz}, d[3] = {r.dx, r.dy, r.dz};
            double reach = r.reach;
            int cls = 0;
            for (int32_t k = 0; k < ntris && cls != 1; k++) {
                const float *p = v9 + 9 * k;
                double a[3] = {p[0], p[1], p[2]};
                double e1[3] = {p[3] - a[0], p[4] - a[1], p[5] - a[2]};
                double e2[3] = {p[6] - a[0], p[7] - a[1], p[8] - a[2]};
                double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2],
                                d[0] * e2[1] - d[1] * e2[0]};
                double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
                double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double e1n = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
                double e2n = std::sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
                double scale = dn * e1n * e2n;
                if (scale == 0.0) continue;
                if (std::fabs(det) <= rel_margin * scale) {
                    // Grazing: parallel within margin.  Ambiguous when the
                    // segment runs within the margin of the triangle's plane
                    // (or crosses it); a segment clear of the plane on one
                    // side misses.
                    double nv[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                    e1[0] * e2[1] - e1[1] * e2[0]};
                    double nn = std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
                    if (nn == 0.0 || !(std::fabs(det) > 0)) continue;
                    double w[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
                    double d0 = (w[0] * nv[0] + w[1] * nv[1] + w[2] * nv[2]) / nn;
                    double d1 = d0 + reach * ((d[0] * nv[0] + d[1] * nv[1] + d[2] * nv[2]) / nn);
                    double lim = e1n > e2n ? e1n : e2n;
                    double rl = reach * dn;
                    lim = rel_margin * (lim > rl ? lim : rl);
                    bool clear = (d0 > lim && d1 > lim) || (d0 < -lim && d1 < -lim);
                    if (!clear) cls = cls == 1 ? 1 : 2;
                    continue;
                }
                double inv = 1.0 / det;
                double tv[3] = {o[0] - a[0], o[1] - a[1], o[2] - a[2]};
                double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) * inv;
                double qv[3] = {tv[1] * e1[2] - tv[2] * e1[1], tv[2] * e1[0] - tv[0] * e1[2],
                                tv[0] * e1[1] - tv[1] * e1[0]};
                double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv;
                double t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv;
                double m = rel_margin;
                double tm = rel_margin * (reach > 1.0 ? reach : 1.0);
                bool inside = u > m && v > m && u + v < 1.0 - m && t > tm && t < reach - tm;
                bool outside = u < -m || v < -m || u + v > 1.0 + m || t < -tm || t > reach + tm;
                if (inside)
                    cls = 1;
                else if (!outside)
                    cls = 2;
            }
            out_class[i] = (int8_t)cls;
        }
    });
    return 0;
}
