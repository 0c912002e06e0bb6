// bounce_oracle.cpp -- CPU oracle for the lighting stage's bounce.
//
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).  A restatement, in the
// reference's own structure (linked patch lists, recursion, scalar loops),
// of:
//   FaceNeighbours.Build (corner normals)  MapTools/Rad/Light/FaceNeighbours.cs:183-340
//   PhongNormals.Compute                   MapTools/Rad/Light/PhongNormals.cs:60-140
//   PatchBuilder.Build / MakePatchForFace  MapTools/Rad/Light/PatchBuilder.cs:90-300
//   PatchSubdivider.Subdivide / SubdividePatch / CreateChildPatch /
//     RebuildFaceLists / ResolveClusters   MapTools/Rad/Light/PatchSubdivider.cs:101-480
//   PatchLighting.BuildPatchLights / AddSampleToPatch
//                                          MapTools/Rad/Light/PatchLighting.cs:65-249
//   VisMatrix.ReceiverOrder / FacesInRow / Enumerator / MakeRays /
//     TransferRay / MakeTransfers / MakeTransfer / MakeScales
//                                          MapTools/Rad/Bounce/VisMatrix.cs:180-1004
//   FormFactors.DiffToDiff / PolyToDiff    MapTools/Rad/Bounce/FormFactors.cs:58-140
//   Radiosity.BounceAsync / MoveDirectLightToEmission / GatherLight /
//     CollectLight                         MapTools/Rad/Bounce/Radiosity.cs:132-316
// The sky and PVS model of the synthetic worlds: one BSP leaf per cluster,
// holding the faces that lie in it; a patch's cluster is its face's.
// DetMathF.Asin is restated as the x87 extended-precision arcsine rounded
// once to float.  Rays are traced with the restated KD walk.
// Built with -ffp-contract=off.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>
#include <tuple>
#include <vector>

#include "oracle_internal.h"
#include "vrad_oracle.h"

namespace {

struct V {
    float x, y, z;
};
V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V operator*(V a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float Dot(V a, V b) { return (a.x * b.x) + (a.y * b.y) + (a.z * b.z); }
V Cross(V a, V b) { return {(a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x)}; }
float Length(V a) { return std::sqrt((a.x * a.x) + (a.y * a.y) + (a.z * a.z)); }
V Normalise(V a, float &len) {
    len = Length(a);
    if (len == 0.0f) return {0, 0, 0};
    return {a.x / len, a.y / len, a.z / len};
}
V Normalise(V a) {
    float l;
    return Normalise(a, l);
}
float At(V v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

typedef std::vector<V> Winding;

// ---- WindingArena ------------------------------------------------------------

Winding RemoveColinearPoints(const Winding &w) {
    Winding out;
    const int n = (int)w.size();
    for (int i = 0; i < n; i++) {
        V v1 = Normalise(w[(i + 1) % n] - w[i]);
        V v2 = Normalise(w[i] - w[(i + n - 1) % n]);
        if ((double)Dot(v1, v2) < 0.999) out.push_back(w[i]);
    }
    return (int)out.size() == n ? w : out;
}

float Area(const Winding &p) {
    float total = 0.0f;
    for (size_t i = 2; i < p.size(); i++) total += Length(Cross(p[i - 1] - p[0], p[i] - p[0]));
    return total * 0.5f;
}

float AreaAndBalancePoint(const Winding &p, V &center) {
    center = {0, 0, 0};
    float total = 0.0f;
    for (size_t i = 2; i < p.size(); i++) {
        float area = Length(Cross(p[i - 1] - p[0], p[i] - p[0]));
        total += area;
        float third = (float)(area / 3.0);
        center = center + p[i - 1] * third;
        center = center + p[i] * third;
        center = center + p[0] * third;
    }
    if (total != 0.0f) center = center * (float)(1.0 / total);
    return total * 0.5f;
}

void Bounds(const Winding &p, V &mins, V &maxs) {
    float a = 99999.0f, b = 99999.0f, c = 99999.0f, d = -99999.0f, e = -99999.0f, f = -99999.0f;
    for (V v : p) {
        if (v.x < a) a = v.x;
        if (v.x > d) d = v.x;
        if (v.y < b) b = v.y;
        if (v.y > e) e = v.y;
        if (v.z < c) c = v.z;
        if (v.z > f) f = v.z;
    }
    mins = {a, b, c};
    maxs = {d, e, f};
}

V Center(const Winding &p) {
    V c = {0, 0, 0};
    for (V v : p) c = v + c;
    return c * (float)(1.0 / (double)p.size());
}

// ClipEpsilon against a unit-axis plane: o1 = front, o2 = back.
void ClipEpsilon(const Winding &in, V normal, float dist, float eps, Winding &front, Winding &back) {
    const int n = (int)in.size();
    std::vector<float> dists(n + 1);
    std::vector<int> sides(n + 1);
    int counts[3] = {0, 0, 0};  // front, back, on
    for (int i = 0; i < n; i++) {
        float dot = Dot(in[i], normal);
        dot -= dist;
        dists[i] = dot;
        sides[i] = dot > eps ? 0 : (dot < -eps ? 1 : 2);
        counts[sides[i]]++;
    }
    front.clear();
    back.clear();
    if (n == 0) return;
    sides[n] = sides[0];
    dists[n] = dists[0];
    if (counts[0] == 0) {
        back = in;
        return;
    }
    if (counts[1] == 0) {
        front = in;
        return;
    }
    for (int i = 0; i < n; i++) {
        V p1 = in[i];
        if (sides[i] == 2) {
            front.push_back(p1);
            back.push_back(p1);
            continue;
        }
        if (sides[i] == 0) front.push_back(p1);
        if (sides[i] == 1) back.push_back(p1);
        if (sides[i + 1] == 2 || sides[i + 1] == sides[i]) continue;
        V p2 = in[(i + 1) % n];
        float dot = dists[i] / (dists[i] - dists[i + 1]);
        auto axis = [&](float nv, float a, float b) {
            if (nv == 1.0f) return dist;
            if (nv == -1.0f) return -dist;
            return a + dot * (b - a);
        };
        V mid = {axis(normal.x, p1.x, p2.x), axis(normal.y, p1.y, p2.y), axis(normal.z, p1.z, p2.z)};
        front.push_back(mid);
        back.push_back(mid);
    }
}

// DetMathF.Asin: the correctly rounded float arcsine, here the x87
// extended arcsine rounded once.
float AsinCR(float x) {
    if (x == 0.0f || std::isnan(x)) return x;
    if (!(std::fabs(x) <= 1.0f)) return std::nanf("");
    return (float)asinl((long double)x);
}

// ---- the patch set ----------------------------------------------------------

constexpr int Invalid = -1;

struct Patch {
    Winding winding;
    V mins, maxs, face_mins, face_maxs, origin, plane_normal;
    float plane_dist, cached_plane_dist;
    V normal;
    bool sky;
    float chop, lux_scale, area;
    V reflectivity, direct_light, sample_light;
    float sample_area;
    V total_light;
    int face, cluster, parent, child1, child2, next, next_parent, next_cluster_child;
};

struct World {
    std::vector<orc_face> faces;
    std::vector<float> verts;
    std::vector<orc_sample> samples;
    std::vector<int64_t> face_first;
    std::vector<float> refl;
    std::vector<int32_t> pvs_off, pvs_list;
    int nclusters;
    float max_chop, min_chop;
    int bounces;
    float threshold;
    OrcKd kd;
    int threads;

    std::vector<Patch> patches;
    std::vector<int> face_patches, face_parents, cluster_children;
    std::vector<V> centroids;
    std::vector<std::vector<V>> corner_normals;
    // Transfers per patch, (source, weight), once built.
    std::vector<std::vector<std::pair<int, float>>> transfers;
    std::vector<char> computed;  // per patch: its transfer list is built
    bool have_transfers = false;
    int64_t rays = 0, blocked = 0;
    int bounces_run = 0;
    float added[3] = {0, 0, 0};

    V vertex(int f, int j) const {
        const orc_face &fc = faces[(size_t)f];
        j %= fc.num_vertices;
        const float *p = &verts[3 * (size_t)(fc.first_vertex + j)];
        return {p[0], p[1], p[2]};
    }
    V face_normal(int f) const { return {faces[(size_t)f].normal[0], faces[(size_t)f].normal[1], faces[(size_t)f].normal[2]}; }
};

// FaceNeighbours.Build's corner normals, rule 2 (every face a brush face in
// smoothing group 0); vertices welded by position.
void BuildCornerNormals(World &w) {
    const int nf = (int)w.faces.size();
    std::map<std::tuple<float, float, float>, int> ids;
    std::vector<std::vector<int>> fv((size_t)nf);
    for (int i = 0; i < nf; i++)
        for (int k = 0; k < w.faces[(size_t)i].num_vertices; k++) {
            V p = w.vertex(i, k);
            auto key = std::make_tuple(p.x + 0.0f, p.y + 0.0f, p.z + 0.0f);
            auto it = ids.find(key);
            int id = it == ids.end() ? (int)ids.size() : it->second;
            if (it == ids.end()) ids.emplace(key, id);
            fv[(size_t)i].push_back(id);
        }
    std::vector<std::vector<int>> vertex_face(ids.size());
    for (int i = 0; i < nf; i++)
        for (int n : fv[(size_t)i]) {
            auto &l = vertex_face[(size_t)n];
            if (std::find(l.begin(), l.end(), i) == l.end()) l.push_back(i);
        }
    w.corner_normals.assign((size_t)nf, {});
    for (int i = 0; i < nf; i++) {
        std::vector<V> normals(fv[(size_t)i].size(), V{0, 0, 0});
        for (size_t j = 0; j < fv[(size_t)i].size(); j++)
            for (int other : vertex_face[(size_t)fv[(size_t)i][j]]) {
                if (other == i) continue;
                V nn = w.face_normal(other);
                double cosv = Dot(nn, w.face_normal(i));
                if (cosv < (double)0.7071067f) continue;
                normals[j] = normals[j] + nn;
            }
        for (V &n : normals) n = Normalise(n + w.face_normal(i));
        w.corner_normals[(size_t)i] = normals;
    }
}

V PhongCompute(const World &w, int face, V spot) {
    V fn = w.face_normal(face);
    const std::vector<V> &corners = w.corner_normals[(size_t)face];
    V centroid = w.centroids[(size_t)face];
    int numEdges = w.faces[(size_t)face].num_vertices;
    for (int j = 0; j < numEdges; j++) {
        V n1 = corners[(size_t)j], n2 = corners[(size_t)((j + 1) % numEdges)];
        V v1 = w.vertex(face, j) - centroid;
        V v2 = w.vertex(face, j + 1) - centroid;
        V vspot = spot - centroid;
        float aa = Dot(v1, v1), bb = Dot(v2, v2), ab = Dot(v1, v2);
        float a1 = ((bb * Dot(v1, vspot)) - (ab * Dot(vspot, v2))) / ((aa * bb) - (ab * ab));
        float a2 = (Dot(vspot, v2) - (a1 * ab)) / bb;
        if (a1 >= 0.0f && a2 >= 0.0f) {
            float scale = (float)(1.0 - a1 - a2);
            V blended = (fn * scale) + (n1 * a1) + (n2 * a2);
            return Normalise(blended);
        }
    }
    return fn;
}

float AxisLength(const float *row) { return std::sqrt((row[0] * row[0]) + (row[1] * row[1]) + (row[2] * row[2])); }

void MakePatchForFace(World &w, int faceNum) {
    const orc_face &face = w.faces[(size_t)faceNum];
    Winding winding;
    for (int i = 0; i < face.num_vertices; i++) winding.push_back(w.vertex(faceNum, i) + V{0, 0, 0});
    winding = RemoveColinearPoints(winding);
    float area = Area(winding);
    if (area <= 0) return;
    Patch patch{};
    patch.next = patch.next_parent = patch.next_cluster_child = Invalid;
    patch.child1 = patch.child2 = patch.parent = Invalid;
    float chopS = AxisLength(face.vecs[0]), chopT = AxisLength(face.vecs[1]);
    patch.area = area;
    patch.sky = (face.flags & 0x0004) != 0;
    patch.lux_scale = (chopS + chopT) / 2.0f;
    patch.chop = w.max_chop;
    patch.winding = winding;
    patch.plane_normal = w.face_normal(faceNum);
    patch.plane_dist = face.dist;
    patch.face = faceNum;
    patch.origin = Center(winding);
    w.centroids[(size_t)faceNum] = patch.origin;
    patch.normal = patch.plane_normal;
    V mins, maxs;
    Bounds(winding, mins, maxs);
    patch.face_mins = patch.mins = mins;
    patch.face_maxs = patch.maxs = maxs;
    const float *r = &w.refl[3 * (size_t)faceNum];
    patch.reflectivity = {std::min(r[0] * 1.0f, 0.99f), std::min(r[1] * 1.0f, 0.99f), std::min(r[2] * 1.0f, 0.99f)};
    patch.next = w.face_patches[(size_t)faceNum];
    w.patches.push_back(patch);
    w.face_patches[(size_t)faceNum] = (int)w.patches.size() - 1;
}

int CreateChildPatch(World &w, int parentIndex, const Winding &winding, float area, V center) {
    Patch child = w.patches[(size_t)parentIndex];
    child.next = child.next_parent = child.next_cluster_child = Invalid;
    child.child1 = child.child2 = Invalid;
    child.parent = parentIndex;
    child.winding = winding;
    child.area = area;
    child.origin = center;
    child.normal = PhongCompute(w, child.face, child.origin);
    child.cached_plane_dist = child.plane_dist;
    V mins, maxs;
    Bounds(winding, mins, maxs);
    child.mins = mins;
    child.maxs = maxs;
    // A surface light's patches skip the face-edge rule ("don't check
    // edges on surf lights", PatchSubdivider.cs:375-380): a face whose
    // texture emits carries the library's emitting-face bit.
    if (w.faces[(size_t)child.face].flags & 0x40000000) {
        w.patches.push_back(child);
        return (int)w.patches.size() - 1;
    }
    V total = (maxs - mins) * child.lux_scale;
    if (child.chop > w.min_chop && total.x < child.chop && total.y < child.chop && total.z < child.chop) {
        for (int i = 0; i < 3; i++) {
            bool touches = At(child.face_maxs, i) == At(maxs, i) || At(child.face_mins, i) == At(mins, i);
            if (touches && At(total, i) > w.min_chop) {
                child.chop = std::max(w.min_chop, child.chop / 2.0f);
                break;
            }
        }
    }
    w.patches.push_back(child);
    return (int)w.patches.size() - 1;
}

void SubdividePatch(World &w, int patchIndex) {
    if (w.patches[(size_t)patchIndex].sky) return;
    V total = (w.patches[(size_t)patchIndex].maxs - w.patches[(size_t)patchIndex].mins) * w.patches[(size_t)patchIndex].lux_scale;
    float chop = w.patches[(size_t)patchIndex].chop;
    int widestAxis = -1;
    float widest = -1.0f;
    bool subdivide = false;
    for (int i = 0; i < 3; i++) {
        float t = At(total, i);
        if (t > widest) {
            widestAxis = i;
            widest = t;
        }
        if (t >= chop && t >= w.min_chop) subdivide = true;
    }
    if (!subdivide && widestAxis != -1) {
        float wd = At(total, widestAxis);
        if (wd > At(total, (widestAxis + 1) % 3) * 2.0f && wd > At(total, (widestAxis + 2) % 3) * 2.0f && chop > w.min_chop) {
            subdivide = true;
            chop = std::max(w.min_chop, chop / 2.0f);
            w.patches[(size_t)patchIndex].chop = chop;
        }
    }
    if (!subdivide) return;
    V split = widestAxis == 0 ? V{1, 0, 0} : (widestAxis == 1 ? V{0, 1, 0} : V{0, 0, 1});
    const Patch &p = w.patches[(size_t)patchIndex];
    float dist = (At(p.mins, widestAxis) + At(p.maxs, widestAxis)) * 0.5f;
    Winding o1, o2;
    ClipEpsilon(p.winding, split, dist, 0.1f, o1, o2);
    V c1, c2;
    float area1 = AreaAndBalancePoint(o1, c1);
    float area2 = AreaAndBalancePoint(o2, c2);
    if (area1 == 0.0f || area2 == 0.0f) return;
    int child1 = CreateChildPatch(w, patchIndex, o1, area1, c1);
    int child2 = CreateChildPatch(w, patchIndex, o2, area2, c2);
    w.patches[(size_t)patchIndex].child1 = child1;
    w.patches[(size_t)patchIndex].child2 = child2;
    SubdividePatch(w, child1);
    SubdividePatch(w, child2);
}

void BuildPatches(World &w) {
    const int nf = (int)w.faces.size();
    w.face_patches.assign((size_t)nf, Invalid);
    w.face_parents.assign((size_t)nf, Invalid);
    w.cluster_children.assign((size_t)w.nclusters, Invalid);
    w.centroids.assign((size_t)nf, V{0, 0, 0});
    BuildCornerNormals(w);
    for (int f = 0; f < nf; f++) MakePatchForFace(w, f);
    // PatchSubdivider.Subdivide (bounces > 0, not -fast).
    const int before = (int)w.patches.size();
    for (int i = 0; i < before; i++) {
        Patch &p = w.patches[(size_t)i];
        p.cached_plane_dist = p.plane_dist;
        p.next_parent = w.face_parents[(size_t)p.face];
        w.face_parents[(size_t)p.face] = i;
    }
    for (int i = 0; i < before; i++) {
        w.patches[(size_t)i].parent = Invalid;
        const int flags = w.faces[(size_t)w.patches[(size_t)i].face].flags;
        const bool prevent = (flags & 0x4000) || ((flags & 0x0400) && !(flags & 0x0001));
        if (prevent) continue;
        SubdividePatch(w, i);
    }
    // RebuildFaceLists.
    std::fill(w.face_patches.begin(), w.face_patches.end(), Invalid);
    for (int i = 0; i < (int)w.patches.size(); i++) {
        Patch &p = w.patches[(size_t)i];
        p.next = w.face_patches[(size_t)p.face];
        w.face_patches[(size_t)p.face] = i;
    }
    // ResolveClusters: a patch lies on its face, in its face's cluster.
    for (Patch &p : w.patches) p.cluster = w.faces[(size_t)p.face].cluster;
    for (int num = 0; num < (int)w.patches.size(); num++) {
        int i = (int)w.patches.size() - num - 1;
        Patch &p = w.patches[(size_t)i];
        if (p.child1 != Invalid || p.cluster == -1) continue;
        p.next_cluster_child = w.cluster_children[(size_t)p.cluster];
        w.cluster_children[(size_t)p.cluster] = i;
    }
}

// ---- PatchLighting ----------------------------------------------------------

void AddSampleToPatch(World &w, const orc_sample &sample, V light, int faceNum) {
    if ((light.x + light.y + light.z) / 3 < 1) return;
    int head = w.face_patches[(size_t)faceNum];
    if (head == Invalid) return;
    float radius = (float)(std::sqrt(sample.area) / 2.0);
    for (int p = head; p != Invalid; p = w.patches[(size_t)p].next) {
        Patch &patch = w.patches[(size_t)p];
        if (patch.sky || patch.child1 != Invalid) continue;
        V mins, maxs;
        Bounds(patch.winding, mins, maxs);
        bool inside = true;
        for (int i = 0; i < 3 && inside; i++)
            if (At(mins, i) > sample.position[i] + radius || At(maxs, i) < sample.position[i] - radius) inside = false;
        if (!inside) continue;
        patch.sample_area += sample.area;
        patch.sample_light = {patch.sample_light.x + (sample.area * light.x), patch.sample_light.y + (sample.area * light.y),
                              patch.sample_light.z + (sample.area * light.z)};
    }
}

void BuildPatchLights(World &w, int faceNum, const float *sample_light) {
    for (int64_t i = w.face_first[(size_t)faceNum]; i < w.face_first[(size_t)faceNum + 1]; i++) {
        const float *l = sample_light + 4 * i;
        AddSampleToPatch(w, w.samples[(size_t)i], V{l[0], l[1], l[2]}, faceNum);
    }
    int head = w.face_patches[(size_t)faceNum];
    if (head == Invalid) return;
    for (int p = head; p != Invalid; p = w.patches[(size_t)p].next) {
        Patch &patch = w.patches[(size_t)p];
        if (patch.parent == Invalid) continue;
        Patch &parent = w.patches[(size_t)patch.parent];
        parent.sample_area += patch.sample_area;
        parent.sample_light = parent.sample_light + patch.sample_light;
    }
    for (int p = head; p != Invalid; p = w.patches[(size_t)p].next) {
        Patch &patch = w.patches[(size_t)p];
        if (patch.sample_area != 0.0f) {
            float scale = (float)(1.0 / patch.sample_area);
            V v = patch.sample_light * scale;
            patch.total_light = patch.total_light + v;
            patch.direct_light = patch.direct_light + v;
        }
    }
    for (int p = head; p != Invalid; p = w.patches[(size_t)p].next) {
        Patch &patch = w.patches[(size_t)p];
        if (patch.child1 == Invalid) continue;
        const Patch &c1 = w.patches[(size_t)patch.child1], &c2 = w.patches[(size_t)patch.child2];
        float s1 = c1.area / (c1.area + c2.area);
        float s2 = c2.area / (c1.area + c2.area);
        V total = c1.total_light * s1;
        total = total + c2.total_light * s2;
        patch.total_light = total;
        patch.direct_light = total;
    }
}

// ---- VisMatrix --------------------------------------------------------------

std::vector<int> ReceiverOrder(const World &w) {
    std::vector<int> order;
    for (int c = 0; c < w.nclusters; c++)
        for (int p = w.cluster_children[(size_t)c]; p != Invalid; p = w.patches[(size_t)p].next_cluster_child) order.push_back(p);
    return order;
}

std::vector<int> FacesInRow(const World &w, int cluster) {
    std::vector<int> faces;
    std::vector<char> stamp(w.faces.size(), 0);
    for (int32_t k = w.pvs_off[(size_t)cluster]; k < w.pvs_off[(size_t)cluster + 1]; k++) {
        const int j = w.pvs_list[(size_t)k];
        for (int l = 0; l < (int)w.faces.size(); l++) {  // leaf j's faces
            if (w.faces[(size_t)l].cluster != j || stamp[(size_t)l]) continue;
            stamp[(size_t)l] = 1;
            faces.push_back(l);
        }
    }
    return faces;
}

void TestPatchToPatch(const World &w, V me_origin, V me_normal, float me_dist, int source, std::vector<int> &sink) {
    const Patch &patch2 = w.patches[(size_t)source];
    if (patch2.child1 != Invalid) {
        V tmp = me_origin - patch2.origin;
        if (Dot(tmp, tmp) * 0.0625 < patch2.area) {
            TestPatchToPatch(w, me_origin, me_normal, me_dist, patch2.child1, sink);
            TestPatchToPatch(w, me_origin, me_normal, me_dist, patch2.child2, sink);
            return;
        }
    }
    if (Dot(patch2.origin, me_normal) > me_dist + 0.01) sink.push_back(source);
}

std::vector<int> Candidates(const World &w, int receiver, const std::vector<int> &row) {
    const Patch &patch = w.patches[(size_t)receiver];
    std::vector<int> sink;
    for (int face : row) {
        if (face == patch.face) continue;
        int head = w.face_parents[(size_t)face];
        if (head == Invalid) continue;
        const Patch &first = w.patches[(size_t)head];
        if (!(Dot(patch.origin, first.normal) > first.cached_plane_dist + 0.01)) continue;
        for (int p = head; p != Invalid; p = w.patches[(size_t)p].next_parent)
            TestPatchToPatch(w, patch.origin, patch.plane_normal, patch.cached_plane_dist, p, sink);
    }
    return sink;
}

float DiffToDiff(V o1, V n1, V o2, V n2) {
    float length;
    V delta = Normalise(o1 - o2, length);
    return -Dot(delta, n1) * Dot(delta, n2) / (length * length);
}

float PolyToDiff(const Winding &polygon, float area, V origin, V normal) {
    float ff = 0.0f;
    const int n = (int)polygon.size();
    for (int point = 0; point < n; point++) {
        int next = point < n - 1 ? point + 1 : 0;
        V v1 = Normalise(polygon[(size_t)point] - origin);
        V v2 = Normalise(polygon[(size_t)next] - origin);
        float sinAlpha;
        V gamma = Normalise(Cross(v1, v2), sinAlpha);
        if (sinAlpha < -1.0f || sinAlpha > 1.0f) sinAlpha = sinAlpha > 1.0f ? 1.0f : -1.0f;
        gamma = gamma * AsinCR(sinAlpha);
        ff += Dot(gamma, normal);
    }
    ff *= 0.5f / area;
    return ff;
}

bool MakeTransfer(const World &w, int receiver, int source, float &trans) {
    trans = 0.0f;
    const Patch &patch1 = w.patches[(size_t)receiver], &patch2 = w.patches[(size_t)source];
    if (w.faces[(size_t)patch2.face].flags & 0x0004) return false;
    if (patch2.area <= 0) return false;
    float scale = DiffToDiff(patch2.origin, patch2.normal, patch1.origin, patch1.normal);
    if (scale <= 0) return false;
    V delta = patch1.origin - patch2.origin;
    float threshold = (float)((M_PI * 0.04) * Dot(delta, delta));
    if (threshold < patch2.area) {
        scale = PolyToDiff(patch2.winding, patch2.area, patch1.origin, patch1.normal);
        if (scale <= 0.0) return false;
    }
    trans = patch2.area * scale;
    return trans > 0.0000001;
}

void MakeScales(std::vector<std::pair<int, float>> &t) {
    if (t.empty()) return;
    float total = 0;
    for (auto &x : t) total += x.second;
    total = total > M_PI ? 1.0f / total : (float)(1.0f / M_PI);
    for (auto &x : t) x.second = x.second * total;
}

// The transfers of one receiver: its candidates' rays traced (StockExact),
// then MakeTransfers on the open ones, capped at MaxPatches.
void ReceiverTransfers(const World &w, int receiver, const std::vector<int> &row,
                       std::vector<std::pair<int, float>> &out, int64_t &rays, int64_t &blocked) {
    out.clear();
    std::vector<int> cand = Candidates(w, receiver, row);
    const Patch &patch = w.patches[(size_t)receiver];
    V p1 = patch.origin + patch.normal;
    for (int s : cand) {
        const Patch &patch2 = w.patches[(size_t)s];
        V end = patch2.origin + patch2.normal;
        V delta = end - p1;
        float len = Length(delta);
        float safe = len == 0.0f ? 1.1920929E-07f : len;
        orc_ray ray{p1.x, p1.y, p1.z, delta.x / safe, delta.y / safe, delta.z / safe, len};
        rays++;
        if (orc_kd_segment_blocked(w.kd, ray, false)) {
            blocked++;
            continue;
        }
        if ((int64_t)out.size() >= 4 * 65536) continue;
        float trans;
        if (MakeTransfer(w, receiver, s, trans)) out.push_back({s, trans});
    }
    MakeScales(out);
}

void BuildTransfers(World &w, const std::vector<int> &all) {
    w.transfers.resize(w.patches.size());
    w.computed.resize(w.patches.size(), 0);
    std::vector<int> receivers;
    for (int r : all)
        if (!w.computed[(size_t)r]) receivers.push_back(r);
    std::atomic<size_t> next{0};
    std::atomic<int64_t> rays{0}, blocked{0};
    auto work = [&]() {
        std::vector<std::pair<int, float>> tmp;
        int last_cluster = -1;
        std::vector<int> row;
        for (;;) {
            size_t k = next.fetch_add(1);
            if (k >= receivers.size()) break;
            int r = receivers[k];
            int c = w.patches[(size_t)r].cluster;
            if (c != last_cluster) {
                row = FacesInRow(w, c);
                last_cluster = c;
            }
            int64_t nr = 0, nb = 0;
            ReceiverTransfers(w, r, row, tmp, nr, nb);
            w.transfers[(size_t)r] = tmp;
            w.computed[(size_t)r] = 1;
            rays += nr;
            blocked += nb;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, w.threads); t++) pool.emplace_back(work);
    for (auto &t : pool) t.join();
    w.rays += rays;
    w.blocked += blocked;
}

// ---- Radiosity --------------------------------------------------------------

void Bounce(World &w) {
    const size_t P = w.patches.size();
    std::vector<V> emit(P), shoot(P), add(P);
    auto Shoot = [](V e, V r) { return V{e.x * r.x, e.y * r.y, e.z * r.z}; };
    for (size_t i = 0; i < P; i++) {
        Patch &patch = w.patches[i];
        emit[i] = patch.total_light;
        shoot[i] = Shoot(emit[i], patch.reflectivity);
        patch.total_light = {0, 0, 0};
    }
    w.bounces_run = 0;
    for (int i = 0;; i++) {
        // GatherLight over every patch.
        std::atomic<size_t> next{0};
        auto gather = [&]() {
            for (;;) {
                size_t j = next.fetch_add(256);
                if (j >= P) break;
                for (size_t q = j; q < std::min(P, j + 256); q++) {
                    V sum = {0, 0, 0};
                    for (auto &t : w.transfers[q]) {
                        V v = shoot[(size_t)t.first];
                        v = v * t.second;
                        sum = sum + v;
                    }
                    add[q] = sum;
                }
            }
        };
        std::vector<std::thread> pool;
        for (int t = 0; t < std::max(1, w.threads); t++) pool.emplace_back(gather);
        for (auto &t : pool) t.join();
        // CollectLight, descending index order.
        V total = {0, 0, 0};
        for (int q = (int)P - 1; q >= 0; q--) {
            Patch &patch = w.patches[(size_t)q];
            if (patch.sky) {
                emit[(size_t)q] = {0, 0, 0};
                shoot[(size_t)q] = Shoot(emit[(size_t)q], patch.reflectivity);
            } else if (patch.child1 == Invalid) {
                patch.total_light = patch.total_light + add[(size_t)q];
                emit[(size_t)q] = add[(size_t)q];
                shoot[(size_t)q] = Shoot(emit[(size_t)q], patch.reflectivity);
                total = total + emit[(size_t)q];
            } else {
                const Patch &c1 = w.patches[(size_t)patch.child1], &c2 = w.patches[(size_t)patch.child2];
                float s1 = c1.area / (c1.area + c2.area);
                float s2 = c2.area / (c1.area + c2.area);
                V light = c1.total_light * s1;
                patch.total_light = light + (c2.total_light * s2);
                emit[(size_t)q] = (emit[(size_t)patch.child1] * s1) + (emit[(size_t)patch.child2] * s2);
                shoot[(size_t)q] = Shoot(emit[(size_t)q], patch.reflectivity);
            }
            add[(size_t)q] = {0, 0, 0};
        }
        w.bounces_run = i + 1;
        w.added[0] = total.x, w.added[1] = total.y, w.added[2] = total.z;
        if (i + 1 == w.bounces || ((double)total.x < (double)w.threshold && (double)total.y < (double)w.threshold &&
                                   (double)total.z < (double)w.threshold))
            break;
    }
}

}  // namespace

extern "C" {

void *orc_bounce_new(const orc_bounce_in *in) {
    World *w = new World();
    w->faces.assign(in->faces, in->faces + in->nfaces);
    int64_t nv = 0;
    for (int f = 0; f < in->nfaces; f++) nv = std::max<int64_t>(nv, in->faces[f].first_vertex + in->faces[f].num_vertices);
    w->verts.assign(in->verts, in->verts + 3 * nv);
    w->samples.assign(in->samples, in->samples + in->face_first[in->nfaces]);
    w->face_first.assign(in->face_first, in->face_first + in->nfaces + 1);
    w->refl.assign(in->reflectivity, in->reflectivity + 3 * (size_t)in->nfaces);
    w->pvs_off.assign(in->pvs_off, in->pvs_off + in->nclusters + 1);
    w->pvs_list.assign(in->pvs_list, in->pvs_list + in->pvs_off[in->nclusters]);
    w->nclusters = in->nclusters;
    w->max_chop = in->max_chop;
    w->min_chop = in->min_chop;
    w->bounces = in->bounces;
    w->threshold = in->threshold;
    w->kd = OrcKd{in->nodes, in->indices, in->tris,
                  {in->bounds6[0], in->bounds6[1], in->bounds6[2], in->bounds6[3], in->bounds6[4], in->bounds6[5]}};
    w->threads = in->threads;
    BuildPatches(*w);
    return w;
}

void orc_bounce_free(void *h) { delete static_cast<World *>(h); }

int orc_bounce_patches(void *h, orc_patch *out, int64_t capacity, int64_t *count, float *points, int64_t point_capacity,
                       int64_t *point_count) {
    World &w = *static_cast<World *>(h);
    *count = (int64_t)w.patches.size();
    int64_t np = 0;
    for (const Patch &p : w.patches) np += (int64_t)p.winding.size();
    *point_count = np;
    if (!out && !points) return 0;
    if ((out && capacity < *count) || (points && point_capacity < np)) return -1;
    int64_t at = 0;
    for (size_t i = 0; i < w.patches.size(); i++) {
        const Patch &p = w.patches[i];
        if (out) {
            orc_patch &o = out[i];
            std::memset(&o, 0, sizeof o);
            o.origin[0] = p.origin.x, o.origin[1] = p.origin.y, o.origin[2] = p.origin.z;
            o.area = p.area;
            o.normal[0] = p.normal.x, o.normal[1] = p.normal.y, o.normal[2] = p.normal.z;
            o.plane_dist = p.plane_dist;
            o.mins[0] = p.mins.x, o.mins[1] = p.mins.y, o.mins[2] = p.mins.z;
            o.chop = p.chop;
            o.maxs[0] = p.maxs.x, o.maxs[1] = p.maxs.y, o.maxs[2] = p.maxs.z;
            o.lux_scale = p.lux_scale;
            o.face_mins[0] = p.face_mins.x, o.face_mins[1] = p.face_mins.y, o.face_mins[2] = p.face_mins.z;
            o.face = p.face;
            o.face_maxs[0] = p.face_maxs.x, o.face_maxs[1] = p.face_maxs.y, o.face_maxs[2] = p.face_maxs.z;
            o.cluster = p.cluster;
            o.reflectivity[0] = p.reflectivity.x, o.reflectivity[1] = p.reflectivity.y, o.reflectivity[2] = p.reflectivity.z;
            o.sky = p.sky ? 1 : 0;
            o.parent = p.parent;
            o.child1 = p.child1;
            o.child2 = p.child2;
            o.first_point = (int32_t)at;
            o.num_points = (int32_t)p.winding.size();
        }
        for (V v : p.winding) {
            if (points) {
                points[3 * at] = v.x;
                points[3 * at + 1] = v.y;
                points[3 * at + 2] = v.z;
            }
            at++;
        }
    }
    return 0;
}

int orc_bounce_transfers(void *h, const int32_t *receivers, int32_t nreceivers, int64_t *offsets, int32_t *src,
                         float *weight, int64_t capacity, int64_t *count, int64_t *rays) {
    World &w = *static_cast<World *>(h);
    std::vector<int> recv;
    if (receivers) recv.assign(receivers, receivers + nreceivers);
    else recv = ReceiverOrder(w);
    const int64_t before = w.rays;
    BuildTransfers(w, recv);
    if (!receivers) w.have_transfers = true;
    if (rays) *rays = w.rays - before;
    // Lists by patch index, for the receivers asked for (all: every patch).
    std::vector<char> asked(w.patches.size(), receivers ? 0 : 1);
    for (int r : recv) asked[(size_t)r] = 1;
    int64_t k = 0;
    for (size_t p = 0; p < w.patches.size(); p++) {
        offsets[p] = k;
        if (!asked[p]) continue;
        for (auto &t : w.transfers[p]) {
            if (src) {
                if (k >= capacity) return -1;
                src[k] = t.first;
                weight[k] = t.second;
            }
            k++;
        }
    }
    offsets[w.patches.size()] = k;
    *count = k;
    return 0;
}

int orc_bounce_set_transfers(void *h, const int64_t *offsets, const int32_t *src, const float *weight) {
    World &w = *static_cast<World *>(h);
    w.transfers.assign(w.patches.size(), {});
    w.computed.assign(w.patches.size(), 1);
    for (size_t p = 0; p < w.patches.size(); p++)
        for (int64_t k = offsets[p]; k < offsets[p + 1]; k++) w.transfers[p].push_back({src[k], weight[k]});
    w.have_transfers = true;
    return 0;
}

int orc_bounce_run(void *h, const float *sample_light, float *total_light, float *direct_light, int32_t *bounces_run,
                   float *added) {
    World &w = *static_cast<World *>(h);
    for (Patch &p : w.patches) {
        p.sample_light = p.direct_light = p.total_light = {0, 0, 0};
        p.sample_area = 0.0f;
    }
    for (int f = 0; f < (int)w.faces.size(); f++) BuildPatchLights(w, f, sample_light);
    if (direct_light)
        for (size_t p = 0; p < w.patches.size(); p++) {
            direct_light[3 * p] = w.patches[p].direct_light.x;
            direct_light[3 * p + 1] = w.patches[p].direct_light.y;
            direct_light[3 * p + 2] = w.patches[p].direct_light.z;
        }
    if (w.bounces <= 0) return 0;
    if (!w.have_transfers) {
        BuildTransfers(w, ReceiverOrder(w));
        w.have_transfers = true;
    }
    Bounce(w);
    if (total_light)
        for (size_t p = 0; p < w.patches.size(); p++) {
            total_light[3 * p] = w.patches[p].total_light.x;
            total_light[3 * p + 1] = w.patches[p].total_light.y;
            total_light[3 * p + 2] = w.patches[p].total_light.z;
        }
    if (bounces_run) *bounces_run = w.bounces_run;
    if (added)
        for (int c = 0; c < 3; c++) added[c] = w.added[c];
    return 0;
}

int orc_bounce_final(void *h, const float *sample_light, uint8_t *lighting, int64_t capacity, int32_t *lightofs,
                     int64_t *total) {
    return orc_bounce_final_styles(h, sample_light, nullptr, nullptr, lighting, capacity, lightofs, total);
}

int orc_bounce_final_styles(void *h, const float *sample_light, const float *slots_light, const uint8_t *face_styles,
                            uint8_t *lighting, int64_t capacity, int32_t *lightofs, int64_t *total) {
    World &w = *static_cast<World *>(h);
    OrcBounced b;
    b.face_leaves.assign(w.faces.size(), {});
    for (size_t f = 0; f < w.faces.size(); f++)
        for (int p = w.face_patches[f]; p != Invalid; p = w.patches[(size_t)p].next) {
            const Patch &patch = w.patches[(size_t)p];
            if (patch.child1 != Invalid) continue;
            OrcBouncedPatch bp;
            for (V v : patch.winding) {
                bp.winding.push_back(v.x);
                bp.winding.push_back(v.y);
                bp.winding.push_back(v.z);
            }
            bp.origin[0] = patch.origin.x, bp.origin[1] = patch.origin.y, bp.origin[2] = patch.origin.z;
            bp.light[0] = patch.total_light.x, bp.light[1] = patch.total_light.y, bp.light[2] = patch.total_light.z;
            b.face_leaves[f].push_back(bp);
        }
    return orc_final_impl(w.faces.data(), (int32_t)w.faces.size(), w.verts.data(), w.samples.data(), w.face_first.data(),
                          sample_light, lighting, capacity, lightofs, total, w.bounces > 0 ? &b : nullptr,
                          slots_light, face_styles);
}

int64_t orc_bounce_stats(void *h, int64_t *blocked) {
    World &w = *static_cast<World *>(h);
    if (blocked) *blocked = w.blocked;
    return w.rays;
}

float orc_asin(float x) { return AsinCR(x); }

// FormFactors.DiffToDiff(o1, n1, o2, n2); q = 12 floats.
float orc_diff_to_diff(const float *q) {
    return DiffToDiff(V{q[0], q[1], q[2]}, V{q[3], q[4], q[5]}, V{q[6], q[7], q[8]}, V{q[9], q[10], q[11]});
}

// FormFactors.PolyToDiff of a winding of `count` xyz points.
float orc_poly_to_diff(const float *points, int32_t count, float area, const float *origin, const float *normal) {
    Winding w;
    for (int32_t k = 0; k < count; k++) w.push_back(V{points[3 * k], points[3 * k + 1], points[3 * k + 2]});
    return PolyToDiff(w, area, V{origin[0], origin[1], origin[2]}, V{normal[0], normal[1], normal[2]});
}

// Drops every built transfer list, so the next build traces again.
void orc_bounce_forget_transfers(void *h) {
    World &w = *static_cast<World *>(h);
    w.transfers.assign(w.patches.size(), {});
    w.computed.assign(w.patches.size(), 0);
    w.have_transfers = false;
}

// The candidate pairs of every receiver (the transfer rays one full build
// traces), counted by the enumerator alone.
int64_t orc_bounce_count_candidates(void *h) {
    World &w = *static_cast<World *>(h);
    std::vector<int> recv = ReceiverOrder(w);
    std::atomic<size_t> next{0};
    std::atomic<int64_t> total{0};
    auto work = [&]() {
        int last = -1;
        std::vector<int> row;
        int64_t n = 0;
        for (;;) {
            size_t k = next.fetch_add(1);
            if (k >= recv.size()) break;
            int c = w.patches[(size_t)recv[k]].cluster;
            if (c != last) {
                row = FacesInRow(w, c);
                last = c;
            }
            n += (int64_t)Candidates(w, recv[k], row).size();
        }
        total += n;
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, w.threads); t++) pool.emplace_back(work);
    for (auto &t : pool) t.join();
    return total;
}

}  // extern "C"
