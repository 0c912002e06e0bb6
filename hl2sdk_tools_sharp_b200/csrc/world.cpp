// world.cpp -- host-side set-up of the lighting stage: each face's luxel
// frame and its light samples, as the reference's RadWorld set-up builds
// them before any ray is traced.
//
//   FaceLightInfo.Build        MapTools/Rad/Light/FaceLightInfo.cs:79-160
//   FaceSampleBuilder          MapTools/Rad/Light/FaceSampleBuilder.cs:80-367
//   WindingArena.ClipEpsilon / AreaAndBalancePoint / Bounds /
//   RemoveColinearPoints       MapTools/Geometry/WindingArena.cs
//
// Plain single-precision host arithmetic in the reference's operation order
// (built with -ffp-contract=off: no fused multiply-add), so sample positions
// are the reference's bits.  This is set-up, not the hot path: the samples
// are the input of the device kernels.

#include <algorithm>
#include <atomic>
#include <thread>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/vrad_cuda.h"
#include "host_geom.h"
#include "world.h"

namespace {

using namespace vrad::hg;

constexpr float kLightmapOnEpsilon = 0.1f / 16.0f;  // LightConstants.LightmapOnEpsilon
constexpr double kDegenerateDet = 1.0e-20;          // FaceLightInfo.DegenerateDeterminant

struct FaceFrame {
    V3 normal;
    float dist;
    V3 w2l_s, w2l_t, l2w_s, l2w_t, origin;
    int min_s, min_t, width, height;
};

// FaceLightInfo.Build (FaceLightInfo.cs:79-160), world model (origin 0).
FaceFrame face_frame(const vrad_face &f) {
    FaceFrame fr;
    fr.normal = {f.normal[0], f.normal[1], f.normal[2]};
    fr.dist = f.dist;
    fr.w2l_s = {f.lightmap_vecs[0][0], f.lightmap_vecs[0][1], f.lightmap_vecs[0][2]};
    fr.w2l_t = {f.lightmap_vecs[1][0], f.lightmap_vecs[1][1], f.lightmap_vecs[1][2]};
    const float off_s = f.lightmap_vecs[0][3], off_t = f.lightmap_vecs[1][3];
    const V3 s = fr.w2l_s, t = fr.w2l_t, n = fr.normal;
    // The 2x2 minors, each written out as the reference pairs them.
    V3 lsc = {t.y * s.z - t.z * s.y, t.z * s.x - t.x * s.z, t.x * s.y - t.y * s.x};
    float det = -dot(n, lsc);
    V3 origin{0.0f, 0.0f, 0.0f};
    fr.l2w_s = {0.0f, 0.0f, 0.0f};
    fr.l2w_t = {0.0f, 0.0f, 0.0f};
    if (!(std::fabs((double)det) < kDegenerateDet)) {
        fr.l2w_s = {(n.z * t.y - n.y * t.z) / det, (n.x * t.z - n.z * t.x) / det,
                    (n.y * t.x - n.x * t.y) / det};
        fr.l2w_t = {(n.y * s.z - n.z * s.y) / det, (n.z * s.x - n.x * s.z) / det,
                    (n.x * s.y - n.y * s.x) / det};
        origin = {-(f.dist * lsc.x) / det, -(f.dist * lsc.y) / det, -(f.dist * lsc.z) / det};
        origin = add(origin, mul(fr.l2w_s, -off_s));
        origin = add(origin, mul(fr.l2w_t, -off_t));
    }
    origin = add(origin, V3{0.0f, 0.0f, 0.0f});  // plus the (zero) model origin
    fr.origin = origin;
    fr.min_s = f.lightmap_mins[0];
    fr.min_t = f.lightmap_mins[1];
    fr.width = f.lightmap_size[0] + 1;
    fr.height = f.lightmap_size[1] + 1;
    return fr;
}

V3 luxel_to_world(const FaceFrame &fr, float s, float t) {
    s += (float)fr.min_s;
    t += (float)fr.min_t;
    V3 pos = add(fr.origin, mul(fr.l2w_s, s));
    return add(pos, mul(fr.l2w_t, t));
}

float world_area_per_luxel(const vrad_face &f) {
    const float *a = f.lightmap_vecs[0], *b = f.lightmap_vecs[1];
    float ss = (a[0] * a[0] + a[1] * a[1]) + a[2] * a[2];
    float tt = (b[0] * b[0] + b[1] * b[1]) + b[2] * b[2];
    float product = std::sqrt(ss) * std::sqrt(tt);
    return (float)(1.0 / (double)product);
}

}  // namespace

namespace {

// LightmapCoordWinding: face f's winding, colinear points removed, in
// luxel space (z 0).  False when it lies outside the vertex array.
bool luxel_winding(const vrad_face &f, const float *vertices, int64_t nvertices, const FaceFrame &fr, Winding &w) {
    if (f.num_vertices < 3 || f.first_vertex < 0 || f.first_vertex + (int64_t)f.num_vertices > nvertices) return false;
    w.clear();
    for (int32_t k = 0; k < f.num_vertices; k++) {
        const float *v = vertices + 3 * (int64_t)(f.first_vertex + k);
        w.push_back(add(V3{v[0], v[1], v[2]}, V3{0.0f, 0.0f, 0.0f}));
    }
    w = remove_colinear(w);
    for (V3 &p : w) {
        V3 pos = sub(p, fr.origin);
        p = {dot(pos, fr.w2l_s) - (float)fr.min_s, dot(pos, fr.w2l_t) - (float)fr.min_t, 0.0f};
    }
    return true;
}

// FaceSampleBuilder.BuildFacesamples for one face (number fi): its samples
// appended to `out`.
// emit(sample) is called for each of the face's samples in order.
template <class Emit>
int32_t face_samples_to(const vrad_face &f, int32_t fi, const float *vertices, int64_t nvertices, Emit &&emit) {
    Winding cell_front, cell_back, row_front, row_back, w, row;
    const FaceFrame fr = face_frame(f);
    const float area_per_luxel = world_area_per_luxel(f);
    if (!luxel_winding(f, vertices, nvertices, fr, w)) return VRAD_ERR_ARG;
    // BuildFacesamples: rows by t, cells by s, sample offset 1.0.
    Winding lm = w;
    for (int t = 0; t < fr.height && !lm.empty(); t++) {
        clip_axis(lm, 1, (float)t + 1.0f, kLightmapOnEpsilon, row_front, row_back);
        row.swap(row_back);
        for (int s = 0; s < fr.width && !row.empty(); s++) {
            clip_axis(row, 0, (float)s + 1.0f, kLightmapOnEpsilon, cell_front, cell_back);
            if (!cell_back.empty()) {
                V3 center;
                float area = area_and_balance(cell_back, center) * area_per_luxel;
                float mn[2] = {99999.0f, 99999.0f}, mx[2] = {-99999.0f, -99999.0f};
                for (const V3 &p : cell_back) {
                    if (p.x < mn[0]) mn[0] = p.x;
                    if (p.x > mx[0]) mx[0] = p.x;
                    if (p.y < mn[1]) mn[1] = p.y;
                    if (p.y > mx[1]) mx[1] = p.y;
                }
                vrad_sample o;
                V3 pos = luxel_to_world(fr, center.x, center.y);
                o.position[0] = pos.x;
                o.position[1] = pos.y;
                o.position[2] = pos.z;
                o.area = area;
                o.coord[0] = center.x;
                o.coord[1] = center.y;
                o.mins[0] = mn[0];
                o.mins[1] = mn[1];
                o.maxs[0] = mx[0];
                o.maxs[1] = mx[1];
                o.s = s;
                o.t = t;
                o.face = fi;
                o.cluster = f.cluster;
                emit(o);
            }
            row.swap(cell_front);
        }
        lm.swap(row_front);
    }
    return VRAD_OK;
}

int32_t face_samples(const vrad_face &f, int32_t fi, const float *vertices, int64_t nvertices,
                     std::vector<vrad_sample> &out) {
    return face_samples_to(f, fi, vertices, nvertices, [&](const vrad_sample &o) { out.push_back(o); });
}

// Every face's samples, faces built in parallel (each face's samples
// depend on that face alone), one list per face.
int32_t build_all_samples(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                          std::vector<std::vector<vrad_sample>> &all) {
    if (nfaces < 0 || (nfaces > 0 && (!faces || !vertices))) return VRAD_ERR_ARG;
    all.assign((size_t)nfaces, {});
    std::atomic<int32_t> rc{VRAD_OK};
    vrad::parallel_for(nfaces, 1, [&](int64_t f) {
        const int32_t r = face_samples(faces[f], (int32_t)f, vertices, nvertices, all[(size_t)f]);
        if (r != VRAD_OK) rc = r;
    });
    return rc;
}

}  // namespace

extern "C" int32_t vrad_build_samples(const vrad_face *faces, int32_t nfaces, const float *vertices,
                                      int64_t nvertices, vrad_sample *out, int64_t capacity,
                                      int64_t *count, int64_t *face_first) {
    if (!count) return VRAD_ERR_ARG;
    if (nfaces < 0 || (nfaces > 0 && (!faces || !vertices))) return VRAD_ERR_ARG;
    // A face has at most one sample per lightmap cell.  With room for that
    // many, each face writes its samples straight into `out` at its bound's
    // offset (in parallel), and the runs are then closed up in face order
    // (no move at all when every cell has its sample).
    std::vector<int64_t> ub((size_t)nfaces + 1, 0);
    for (int32_t f = 0; f < nfaces; f++)
        ub[(size_t)f + 1] = ub[(size_t)f] + (int64_t)std::max(0, faces[f].lightmap_size[0]) *
                                                std::max(0, faces[f].lightmap_size[1]);
    if (out && capacity >= ub[(size_t)nfaces]) {
        std::vector<int64_t> n((size_t)nfaces, 0);
        std::atomic<int32_t> rc{VRAD_OK};
        std::atomic<bool> over{false};
        vrad::parallel_for(nfaces, 1, [&](int64_t f) {
            const int64_t cap = ub[(size_t)f + 1] - ub[(size_t)f];
            int64_t k = 0;
            const int32_t r = face_samples_to(faces[f], (int32_t)f, vertices, nvertices, [&](const vrad_sample &o) {
                if (k < cap) out[ub[(size_t)f] + k] = o;
                k++;
            });
            if (r != VRAD_OK) rc = r;
            if (k > cap) over = true;
            n[(size_t)f] = k;
        });
        if (rc != VRAD_OK) return rc;
        if (!over) {
            std::vector<int64_t> first((size_t)nfaces + 1, 0);
            for (int32_t f = 0; f < nfaces; f++) first[(size_t)f + 1] = first[(size_t)f] + n[(size_t)f];
            for (int32_t f = 0; f < nfaces; f++)
                if (first[(size_t)f] != ub[(size_t)f] && n[(size_t)f])
                    std::memmove(out + first[(size_t)f], out + ub[(size_t)f], sizeof(vrad_sample) * (size_t)n[(size_t)f]);
            if (face_first) std::copy(first.begin(), first.end(), face_first);
            *count = first[(size_t)nfaces];
            return VRAD_OK;
        }
    }
    std::vector<std::vector<vrad_sample>> all;
    const int32_t rc = build_all_samples(faces, nfaces, vertices, nvertices, all);
    if (rc != VRAD_OK) return rc;
    std::vector<int64_t> first((size_t)nfaces + 1, 0);
    for (int32_t f = 0; f < nfaces; f++) first[(size_t)f + 1] = first[(size_t)f] + (int64_t)all[(size_t)f].size();
    const int64_t total = first[(size_t)nfaces];
    if (face_first) std::copy(first.begin(), first.end(), face_first);
    *count = total;
    if (out) {
        if (total > capacity) return VRAD_ERR_ARG;
        vrad::parallel_for(nfaces, 16, [&](int64_t f) {
            const auto &v = all[(size_t)f];
            if (!v.empty()) std::memcpy(out + first[(size_t)f], v.data(), sizeof(vrad_sample) * v.size());
        });
    }
    return VRAD_OK;
}

namespace vrad {

bool face_row_strips(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices, RowStrips &out,
                     std::string &why) {
    struct Rows {
        std::vector<int32_t> t;
        std::vector<int32_t> n;
        std::vector<float> xy;
        bool ok = true, big = false;
    };
    std::vector<Rows> per((size_t)nfaces);
    out.apl.assign((size_t)nfaces, 0.0f);
    parallel_for(nfaces, 4, [&](int64_t fi) {
        const vrad_face &f = faces[fi];
        Rows &r = per[(size_t)fi];
        const FaceFrame fr = face_frame(f);
        out.apl[(size_t)fi] = world_area_per_luxel(f);
        Winding w, row_front, row_back;
        if (!luxel_winding(f, vertices, nvertices, fr, w)) {
            r.ok = false;
            return;
        }
        if ((int32_t)w.size() > kStripMax) {
            r.big = true;
            return;
        }
        // BuildFacesamples' rows: the winding's part between t and t + 1,
        // the rest carried to the next row.
        Winding lm = w;
        for (int t = 0; t < fr.height && !lm.empty(); t++) {
            clip_axis(lm, 1, (float)t + 1.0f, kLightmapOnEpsilon, row_front, row_back);
            if (!row_back.empty()) {
                r.t.push_back(t);
                r.n.push_back((int32_t)row_back.size());
                for (const V3 &p : row_back) {
                    r.xy.push_back(p.x);
                    r.xy.push_back(p.y);
                }
            }
            lm = row_front;
        }
    });
    size_t nrows = 0, npts = 0;
    for (const Rows &r : per) {
        if (!r.ok) {
            why = "a face's winding lies outside the vertex array";
            return false;
        }
        if (r.big) {
            why = "a face's winding has more than 56 points";
            return false;
        }
        nrows += r.t.size();
        npts += r.xy.size() / 2;
    }
    out.face.resize(nrows);
    out.t.resize(nrows);
    out.first.resize(nrows + 1);
    out.xy.resize(2 * npts);
    std::vector<size_t> row0((size_t)nfaces + 1, 0), pt0((size_t)nfaces + 1, 0);
    for (int32_t f = 0; f < nfaces; f++) {
        row0[(size_t)f + 1] = row0[(size_t)f] + per[(size_t)f].t.size();
        pt0[(size_t)f + 1] = pt0[(size_t)f] + per[(size_t)f].xy.size() / 2;
    }
    out.first[nrows] = (int64_t)npts;
    parallel_for(nfaces, 16, [&](int64_t f) {
        const Rows &r = per[(size_t)f];
        size_t k = row0[(size_t)f];
        int64_t p = (int64_t)pt0[(size_t)f];
        for (size_t i = 0; i < r.t.size(); i++, k++) {
            out.face[k] = (int32_t)f;
            out.t[k] = r.t[i];
            out.first[k] = p;
            p += r.n[i];
        }
        std::copy(r.xy.begin(), r.xy.end(), out.xy.begin() + 2 * pt0[(size_t)f]);
    });
    return true;
}

}  // namespace vrad

// ---- smoothing neighbours and the lightmap layout --------------------------

#include <map>
#include <tuple>
#include <unordered_map>

namespace {

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

}  // namespace

namespace vrad {

bool weld_faces(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                std::vector<std::vector<int32_t>> &face_verts, std::vector<std::vector<int32_t>> &vertex_face) {
    // Weld: one vertex number per distinct position, numbered in order of
    // first appearance (faces in order, each winding in order).
    struct Key {
        uint32_t x, y, z;
        bool operator==(const Key &o) const { return x == o.x && y == o.y && z == o.z; }
    };
    struct Hash {
        size_t operator()(const Key &k) const {
            uint64_t h = k.x * 0x9E3779B97F4A7C15ull;
            h ^= (h >> 29) ^ (k.y * 0xC2B2AE3D27D4EB4Full);
            h ^= (h >> 31) ^ (k.z * 0x165667B19E3779F9ull);
            return (size_t)(h ^ (h >> 32));
        }
    };
    std::unordered_map<Key, int32_t, Hash> weld;
    int64_t corners = 0;
    for (int32_t i = 0; i < nfaces; i++) corners += std::max(0, faces[i].num_vertices);
    weld.reserve((size_t)corners);
    face_verts.assign((size_t)nfaces, {});
    for (int32_t i = 0; i < nfaces; i++) {
        const vrad_face &f = faces[i];
        if (f.first_vertex < 0 || f.num_vertices < 0 || f.first_vertex + (int64_t)f.num_vertices > nvertices) return false;
        face_verts[(size_t)i].reserve((size_t)f.num_vertices);
        for (int32_t k = 0; k < f.num_vertices; k++) {
            const float *v = vertices + 3 * (int64_t)(f.first_vertex + k);
            const Key key = {fbits(v[0] + 0.0f), fbits(v[1] + 0.0f), fbits(v[2] + 0.0f)};
            const auto ins = weld.emplace(key, (int32_t)weld.size());
            face_verts[(size_t)i].push_back(ins.first->second);
        }
    }
    // vertexFace: the faces touching each vertex, in face order, once each.
    vertex_face.assign(weld.size(), {});
    for (int32_t i = 0; i < nfaces; i++)
        for (int32_t v : face_verts[(size_t)i]) {
            auto &vf = vertex_face[(size_t)v];
            if (std::find(vf.begin(), vf.end(), i) == vf.end()) vf.push_back(i);
        }
    return true;
}

bool corner_normals(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                    float smoothing_threshold, std::vector<std::vector<float>> &out) {
    std::vector<std::vector<int32_t>> face_verts, vertex_face;
    if (!weld_faces(faces, nfaces, vertices, nvertices, face_verts, vertex_face)) return false;
    out.assign((size_t)nfaces, {});
    parallel_for(nfaces, 16, [&](int64_t ii) {
        const int32_t i = (int32_t)ii;
        const V3 ni = {faces[i].normal[0], faces[i].normal[1], faces[i].normal[2]};
        std::vector<float> &o = out[(size_t)i];
        for (int32_t v : face_verts[(size_t)i]) {
            V3 sum = {0.0f, 0.0f, 0.0f};
            for (int32_t other : vertex_face[(size_t)v]) {
                if (other == i) continue;
                const V3 no = {faces[other].normal[0], faces[other].normal[1], faces[other].normal[2]};
                if ((double)dot(no, ni) < (double)smoothing_threshold) continue;
                sum = add(sum, no);
            }
            // The face's own normal last, then the exact normalise.
            const V3 n = normalise(add(sum, ni));
            o.push_back(n.x);
            o.push_back(n.y);
            o.push_back(n.z);
        }
    });
    return true;
}

}  // namespace vrad

// FaceNeighbours.Build (MapTools/Rad/Light/FaceNeighbours.cs:80-230) for
// brush faces with smoothing groups 0: faces sharing a vertex are
// neighbours when the cosine of their normals is at least the threshold
// (rule 2).  Vertices are identified by position, as a BSP's vertex lump
// welds them.  Writes offsets[nfaces + 1] and the lists, in discovery order.
namespace vrad {

int32_t face_neighbours(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                        float smoothing_threshold, std::vector<int32_t> &off, std::vector<int32_t> &list) {
    std::vector<std::vector<int32_t>> face_verts, vertex_face;
    if (!weld_faces(faces, nfaces, vertices, nvertices, face_verts, vertex_face)) return VRAD_ERR_ARG;
    std::vector<std::vector<int32_t>> found((size_t)nfaces);
    std::atomic<bool> too_many{false};
    parallel_for(nfaces, 16, [&](int64_t ii) {
        const int32_t i = (int32_t)ii;
        const V3 ni = {faces[i].normal[0], faces[i].normal[1], faces[i].normal[2]};
        std::vector<int32_t> &fo = found[(size_t)i];
        for (int32_t v : face_verts[(size_t)i]) {
            for (int32_t other : vertex_face[(size_t)v]) {
                if (other == i) continue;
                const V3 no = {faces[other].normal[0], faces[other].normal[1], faces[other].normal[2]};
                const double c = (double)dot(no, ni);
                if (c < (double)smoothing_threshold) continue;
                if (std::find(fo.begin(), fo.end(), other) == fo.end()) {
                    if (fo.size() >= 64) {  // MaxNeighbours
                        too_many = true;
                        return;
                    }
                    fo.push_back(other);
                }
            }
        }
    });
    if (too_many) return VRAD_ERR_ARG;
    off.assign((size_t)nfaces + 1, 0);
    for (int32_t i = 0; i < nfaces; i++) off[(size_t)i + 1] = off[(size_t)i] + (int32_t)found[(size_t)i].size();
    list.resize((size_t)off[(size_t)nfaces]);
    parallel_for(nfaces, 64, [&](int64_t i) {
        std::copy(found[(size_t)i].begin(), found[(size_t)i].end(), list.begin() + off[(size_t)i]);
    });
    return VRAD_OK;
}

}  // namespace vrad

extern "C" int32_t vrad_build_neighbours(const vrad_face *faces, int32_t nfaces, const float *vertices,
                                         int64_t nvertices, float smoothing_threshold, int32_t *offsets,
                                         int32_t *list, int64_t capacity, int64_t *count) {
    if (nfaces < 0 || (nfaces && (!faces || !vertices)) || !offsets || !count) return VRAD_ERR_ARG;
    std::vector<int32_t> off, lst;
    const int32_t rc = vrad::face_neighbours(faces, nfaces, vertices, nvertices, smoothing_threshold, off, lst);
    if (rc != VRAD_OK) return rc;
    std::copy(off.begin(), off.end(), offsets);
    *count = (int64_t)lst.size();
    if (list) {
        if ((int64_t)lst.size() > capacity) return VRAD_ERR_ARG;
        std::copy(lst.begin(), lst.end(), list);
    }
    return VRAD_OK;
}

// LightmapOffsets.Compute (MapTools/Rad/Light/LightmapOffsets.cs:54-126):
// per face its styles' four-byte medians before its lightofs, then each
// style's (w + 1) * (h + 1) luxels.  styles (nullable): four bytes per face,
// 255 ending the list; without it every face has style 0 alone.
extern "C" int32_t vrad_lightmap_layout_styles(const vrad_face *faces, int32_t nfaces, const uint8_t *styles,
                                               int32_t *lightofs, int64_t *total) {
    if (nfaces < 0 || (nfaces && !faces) || !lightofs || !total) return VRAD_ERR_ARG;
    int64_t size = 0;
    for (int32_t f = 0; f < nfaces; f++) {
        int lightstyles = 1;
        if (styles)
            for (lightstyles = 0; lightstyles < 4 && styles[4 * (int64_t)f + lightstyles] != 255; lightstyles++) {
            }
        if (lightstyles == 0) {
            lightofs[f] = -1;  // a face without styles gets no lightmap
            continue;
        }
        size += lightstyles * 4;
        lightofs[f] = (int32_t)size;
        const int64_t luxels = (int64_t)(faces[f].lightmap_size[0] + 1) * (faces[f].lightmap_size[1] + 1);
        size += luxels * 4 * lightstyles;
    }
    *total = size;
    return VRAD_OK;
}

extern "C" int32_t vrad_lightmap_layout(const vrad_face *faces, int32_t nfaces, int32_t *lightofs,
                                        int64_t *total) {
    return vrad_lightmap_layout_styles(faces, nfaces, nullptr, lightofs, total);
}

// ---- frames for the other translation units --------------------------------

namespace vrad {

void face_frame_of(const vrad_face &f, FaceFrameOut &out) {
    const FaceFrame fr = face_frame(f);
    const V3 *src[5] = {&fr.origin, &fr.w2l_s, &fr.w2l_t, &fr.l2w_s, &fr.l2w_t};
    float *dst[5] = {out.origin, out.w2l_s, out.w2l_t, out.l2w_s, out.l2w_t};
    for (int k = 0; k < 5; k++) {
        dst[k][0] = src[k]->x;
        dst[k][1] = src[k]->y;
        dst[k][2] = src[k]->z;
    }
    out.min_s = fr.min_s;
    out.min_t = fr.min_t;
    out.width = fr.width;
    out.height = fr.height;
}

void frame_luxel_to_world(const FaceFrameOut &fr, float s, float t, float out[3]) {
    s += (float)fr.min_s;
    t += (float)fr.min_t;
    V3 pos = add(V3{fr.origin[0], fr.origin[1], fr.origin[2]}, mul(V3{fr.l2w_s[0], fr.l2w_s[1], fr.l2w_s[2]}, s));
    pos = add(pos, mul(V3{fr.l2w_t[0], fr.l2w_t[1], fr.l2w_t[2]}, t));
    out[0] = pos.x;
    out[1] = pos.y;
    out[2] = pos.z;
}

void frame_world_to_luxel(const FaceFrameOut &fr, const float p[3], float &s, float &t) {
    const V3 pos = sub(V3{p[0], p[1], p[2]}, V3{fr.origin[0], fr.origin[1], fr.origin[2]});
    s = dot(pos, V3{fr.w2l_s[0], fr.w2l_s[1], fr.w2l_s[2]}) - (float)fr.min_s;
    t = dot(pos, V3{fr.w2l_t[0], fr.w2l_t[1], fr.w2l_t[2]}) - (float)fr.min_t;
}

}  // namespace vrad
