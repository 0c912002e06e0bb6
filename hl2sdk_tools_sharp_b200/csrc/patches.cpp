// patches.cpp -- host-side set-up of the bounce: the patch tree every face
// is cut into before the transfers are built.
//
//   PatchBuilder.Build / MakePatchForFace     MapTools/Rad/Light/PatchBuilder.cs:90-300
//   PatchSubdivider.Subdivide / SubdividePatch / CreateChildPatch /
//     RebuildFaceLists / ResolveClusters      MapTools/Rad/Light/PatchSubdivider.cs:101-480
//   PhongNormals.Compute                      MapTools/Rad/Light/PhongNormals.cs:60-140
//
// Patch indices are the reference's: one root per face with a non-zero
// area, in face order, then each root's descendants in the order
// SubdividePatch creates them (child1, child2, then child1's subtree, then
// child2's).  So a face's descendants occupy one contiguous index range,
// which is how the device kernels walk a face's patch list: the
// reference's FacePatches list is that range in descending order followed
// by the root.  Single precision in the reference's operation order
// (-ffp-contract=off), so origins, normals and areas are its bits.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/vrad_cuda.h"
#include "host_geom.h"
#include "patches.h"
#include "setup_clock.h"
#include "world.h"

namespace vrad {

namespace {

using namespace hg;

constexpr float kOnEpsilon = 0.1f;          // LightConstants.OnEpsilon
constexpr float kMaxReflectivity = 0.99f;   // PatchBuilder.MaxReflectivity
constexpr float kSmoothing = 0.7071067f;    // LightConstants.DefaultSmoothingThreshold

// One root's subtree under construction: local indices, the root at 0.
struct Builder {
    const vrad_face *faces;
    const float *vertices;
    float min_chop;
    const std::vector<std::vector<float>> *corner_normals;  // per face, xyz per winding vertex
    const std::vector<V3> *centroids;                       // PatchSet.Centroids
    std::vector<vrad_patch> patches;
    // The patches' windings, one flat array: patch k's points are
    // pts[wfirst[k] .. wfirst[k] + wcount[k]).
    std::vector<V3> pts;
    std::vector<int32_t> wfirst, wcount;
    Winding o1, o2;  // SubdividePatch's halves (scratch)

    V3 vertex(int32_t f, int32_t k) const {
        const vrad_face &fc = faces[f];
        k %= fc.num_vertices;
        const float *v = vertices + 3 * (int64_t)(fc.first_vertex + k);
        return {v[0], v[1], v[2]};
    }

    // PhongNormals.Compute at `spot` on face f (no model offset).
    V3 phong(int32_t f, V3 spot) const {
        const vrad_face &fc = faces[f];
        const V3 fn = {fc.normal[0], fc.normal[1], fc.normal[2]};
        const std::vector<float> &cn = (*corner_normals)[(size_t)f];
        const V3 c = (*centroids)[(size_t)f];
        const int n = fc.num_vertices;
        for (int j = 0; j < n; j++) {
            const int j2 = (j + 1) % n;
            const V3 n1 = {cn[3 * j], cn[3 * j + 1], cn[3 * j + 2]};
            const V3 n2 = {cn[3 * j2], cn[3 * j2 + 1], cn[3 * j2 + 2]};
            const V3 v1 = sub(vertex(f, j), c);
            const V3 v2 = sub(vertex(f, j + 1), c);
            const V3 vs = sub(spot, c);
            const float aa = dot(v1, v1), bb = dot(v2, v2), ab = dot(v1, v2);
            const float a1 = ((bb * dot(v1, vs)) - (ab * dot(vs, v2))) / ((aa * bb) - (ab * ab));
            const float a2 = (dot(vs, v2) - (a1 * ab)) / bb;
            if (a1 >= 0.0f && a2 >= 0.0f) {
                const float scale = (float)(1.0 - (double)a1 - (double)a2);
                const V3 blended = add(add(mul(fn, scale), mul(n1, a1)), mul(n2, a2));
                return normalise(blended);
            }
        }
        return fn;
    }

    int32_t add_patch(const vrad_patch &p, const Winding &w) {
        patches.push_back(p);
        wfirst.push_back((int32_t)pts.size());
        wcount.push_back((int32_t)w.size());
        pts.insert(pts.end(), w.begin(), w.end());
        return (int32_t)patches.size() - 1;
    }

    // CreateChildPatch: the parent copied, then the child's own fields.
    int32_t child(int32_t parent, const Winding &w, float area, V3 c) {
        vrad_patch ch = patches[(size_t)parent];
        ch.child1 = ch.child2 = -1;
        ch.parent = parent;
        ch.area = area;
        ch.origin[0] = c.x;
        ch.origin[1] = c.y;
        ch.origin[2] = c.z;
        const V3 n = phong(ch.face, c);
        ch.normal[0] = n.x;
        ch.normal[1] = n.y;
        ch.normal[2] = n.z;
        V3 mn, mx;
        bounds(w, mn, mx);
        ch.mins[0] = mn.x, ch.mins[1] = mn.y, ch.mins[2] = mn.z;
        ch.maxs[0] = mx.x, ch.maxs[1] = mx.y, ch.maxs[2] = mx.z;
        // A surface light's patches are never refined by the face-edge
        // rule (PatchSubdivider.cs:375-380).  Otherwise a child already
        // under chop on every axis that touches the face's bounds has its
        // chop halved once.
        if (faces[ch.face].flags & VRAD_FACE_EMITS) return add_patch(ch, w);
        const V3 total = mul(sub(mx, mn), ch.lux_scale);
        if (ch.chop > min_chop && total.x < ch.chop && total.y < ch.chop && total.z < ch.chop) {
            for (int i = 0; i < 3; i++) {
                const bool edge = ch.face_maxs[i] == comp(mx, i) || ch.face_mins[i] == comp(mn, i);
                if (edge && comp(total, i) > min_chop) {
                    ch.chop = std::max(min_chop, ch.chop / 2.0f);
                    break;
                }
            }
        }
        return add_patch(ch, w);
    }

    // SubdividePatch.
    void subdivide(int32_t i) {
        if (patches[(size_t)i].sky) return;
        V3 total, mn, mx;
        float chop;
        {
            const vrad_patch &p = patches[(size_t)i];
            mn = {p.mins[0], p.mins[1], p.mins[2]};
            mx = {p.maxs[0], p.maxs[1], p.maxs[2]};
            total = mul(sub(mx, mn), p.lux_scale);
            chop = p.chop;
        }
        int widest_axis = -1;
        float widest = -1.0f;
        bool split = false;
        for (int a = 0; a < 3; a++) {
            const float t = comp(total, a);
            if (t > widest) {
                widest_axis = a;
                widest = t;
            }
            if (t >= chop && t >= min_chop) split = true;
        }
        if (!split && widest_axis != -1) {
            const float w = comp(total, widest_axis);
            if (w > comp(total, (widest_axis + 1) % 3) * 2.0f && w > comp(total, (widest_axis + 2) % 3) * 2.0f &&
                chop > min_chop) {
                split = true;
                chop = std::max(min_chop, chop / 2.0f);
                patches[(size_t)i].chop = chop;
            }
        }
        if (!split) return;
        const float dist = (comp(mn, widest_axis) + comp(mx, widest_axis)) * 0.5f;
        clip_axis(pts.data() + wfirst[(size_t)i], (size_t)wcount[(size_t)i], widest_axis, dist, kOnEpsilon, o1, o2);
        V3 c1, c2;
        const float a1 = area_and_balance(o1, c1);
        const float a2 = area_and_balance(o2, c2);
        if (a1 == 0.0f || a2 == 0.0f) return;
        const int32_t k1 = child(i, o1, a1, c1);
        const int32_t k2 = child(i, o2, a2, c2);
        patches[(size_t)i].child1 = k1;
        patches[(size_t)i].child2 = k2;
        subdivide(k1);
        subdivide(k2);
    }
};

float axis_length(const float *row) { return std::sqrt((row[0] * row[0] + row[1] * row[1]) + row[2] * row[2]); }

bool prevent_subdivision(int32_t flags) {
    if (flags & VRAD_SURF_NOCHOP) return true;
    return (flags & VRAD_SURF_NOLIGHT) && !(flags & VRAD_SURF_LIGHT);
}

}  // namespace

struct PatchForest::Impl {
    const vrad_face *faces = nullptr;
    int32_t nfaces = 0;
    float max_chop = 0.0f, min_chop = 0.0f;
    std::vector<std::vector<float>> corners;
    std::vector<V3> centroid;
    std::vector<Builder> subtree;
};

PatchForest::PatchForest() = default;
PatchForest::~PatchForest() = default;
PatchForest::PatchForest(PatchForest &&) noexcept = default;
PatchForest &PatchForest::operator=(PatchForest &&) noexcept = default;

bool PatchForest::grown() const { return impl_ != nullptr; }
float PatchForest::max_chop() const { return impl_ ? impl_->max_chop : 0.0f; }
float PatchForest::min_chop() const { return impl_ ? impl_->min_chop : 0.0f; }

bool PatchForest::grow(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                       float max_chop, float min_chop, std::string &why) {
    impl_.reset();
    SetupClock clock("patch_tree");
    std::unique_ptr<Impl> f(new Impl);
    f->faces = faces;
    f->nfaces = nfaces;
    f->max_chop = max_chop;
    f->min_chop = min_chop;
    if (!corner_normals(faces, nfaces, vertices, nvertices, kSmoothing, f->corners)) {
        why = "a face's winding lies outside the vertex array";
        return false;
    }
    clock.mark("corner normals");
    f->centroid.assign((size_t)nfaces, V3{0.0f, 0.0f, 0.0f});
    // MakePatchForFace, face by face: the roots, in face order.  The
    // reflectivity is filled in when the forest is numbered (every patch
    // of a face carries the face's).
    std::vector<Builder> &subtree = f->subtree;
    for (int32_t fi = 0; fi < nfaces; fi++) {
        const vrad_face &fc = faces[fi];
        if (fc.num_vertices < 3) {
            why = "a face has fewer than three vertices";
            return false;
        }
        Winding w;
        for (int32_t k = 0; k < fc.num_vertices; k++) {
            const float *v = vertices + 3 * (int64_t)(fc.first_vertex + k);
            w.push_back(add(V3{v[0], v[1], v[2]}, V3{0.0f, 0.0f, 0.0f}));
        }
        w = remove_colinear(w);
        const float ar = area(w);
        if (ar <= 0.0f) continue;  // a degenerate face gets no patch
        vrad_patch p;
        std::memset(&p, 0, sizeof p);
        p.child1 = p.child2 = p.parent = -1;
        p.area = ar;
        p.lux_scale = (axis_length(fc.lightmap_vecs[0]) + axis_length(fc.lightmap_vecs[1])) / 2.0f;
        p.chop = max_chop;
        p.plane_dist = fc.dist;
        p.face = fi;
        // ResolveClusters: the cluster of the patch's origin, which lies on
        // the face, is the cluster the face's samples lie in.
        p.cluster = fc.cluster;
        p.sky = (fc.flags & VRAD_SURF_SKY) ? 1 : 0;
        const V3 c = center(w);
        f->centroid[(size_t)fi] = c;
        p.origin[0] = c.x, p.origin[1] = c.y, p.origin[2] = c.z;
        for (int a = 0; a < 3; a++) p.normal[a] = fc.normal[a];
        V3 mn, mx;
        bounds(w, mn, mx);
        p.mins[0] = p.face_mins[0] = mn.x;
        p.mins[1] = p.face_mins[1] = mn.y;
        p.mins[2] = p.face_mins[2] = mn.z;
        p.maxs[0] = p.face_maxs[0] = mx.x;
        p.maxs[1] = p.face_maxs[1] = mx.y;
        p.maxs[2] = p.face_maxs[2] = mx.z;
        Builder b;
        b.faces = faces;
        b.vertices = vertices;
        b.min_chop = min_chop;
        b.corner_normals = &f->corners;
        b.centroids = &f->centroid;
        b.add_patch(p, w);
        subtree.push_back(std::move(b));
    }
    const int32_t roots = (int32_t)subtree.size();
    clock.mark("roots");
    // PatchSubdivider.Subdivide with bounces > 0, not -fast.  Each root's
    // subtree depends on nothing outside its face, so the roots are split
    // on worker threads, each into its own arrays; the largest faces (by
    // luxel count, which the patch count follows) are handed out first so
    // that no large face starts last.
    std::vector<int32_t> by_size((size_t)roots);
    std::vector<int64_t> luxels((size_t)roots);
    for (int32_t i = 0; i < roots; i++) {
        const vrad_face &fc = faces[subtree[(size_t)i].patches[0].face];
        luxels[(size_t)i] = (int64_t)(fc.lightmap_size[0] + 1) * (fc.lightmap_size[1] + 1);
        by_size[(size_t)i] = i;
    }
    std::stable_sort(by_size.begin(), by_size.end(),
                     [&](int32_t a, int32_t b) { return luxels[(size_t)a] > luxels[(size_t)b]; });
    parallel_for(roots, 1, [&](int64_t k) {
        Builder &b = subtree[(size_t)by_size[(size_t)k]];
        if (!prevent_subdivision(faces[b.patches[0].face].flags)) b.subdivide(0);
    });
    clock.mark("subdivide");
    impl_ = std::move(f);
    return true;
}

bool PatchForest::merge(const float *reflectivity, PatchTree &out, PatchSink &sink, std::string &why) {
    if (!impl_) {
        why = "no patch forest grown";
        return false;
    }
    SetupClock clock("patch_tree");
    std::vector<Builder> &subtree = impl_->subtree;
    const int32_t nfaces = impl_->nfaces;
    const int32_t roots = (int32_t)subtree.size();
    // Global indices: the roots 0..roots-1 in face order, then each root's
    // descendants in creation order (the order SubdividePatch adds them);
    // the windings' points in the same order.
    std::vector<int32_t> base((size_t)roots);
    std::vector<int64_t> root_pt((size_t)roots + 1, 0), desc_pt((size_t)roots + 1, 0);
    int32_t total = roots;
    for (int32_t i = 0; i < roots; i++) {
        const Builder &b = subtree[(size_t)i];
        base[(size_t)i] = total;
        total += (int32_t)b.patches.size() - 1;
        root_pt[(size_t)i + 1] = root_pt[(size_t)i] + b.wcount[0];
        desc_pt[(size_t)i + 1] = desc_pt[(size_t)i] + (int64_t)b.pts.size() - b.wcount[0];
    }
    const int64_t npoints = root_pt[(size_t)roots] + desc_pt[(size_t)roots];
    if (!sink.prepare(total, npoints)) {
        why = "patch tables";
        return false;
    }
    out.face_root.assign((size_t)nfaces, -1);
    out.face_first.assign((size_t)nfaces, 0);
    out.face_end.assign((size_t)nfaces, 0);
    // Each root's block of patches, renumbered, given the face's
    // reflectivity (PatchBuilder clamps it to MaxReflectivity) and handed
    // to the sink, in parallel.
    parallel_for(roots, 8, [&](int64_t ii) {
        const int32_t i = (int32_t)ii;
        Builder &b = subtree[(size_t)i];
        auto global = [&](int32_t local) { return local < 0 ? -1 : (local == 0 ? i : base[(size_t)i] + local - 1); };
        const int64_t desc0 = root_pt[(size_t)roots] + desc_pt[(size_t)i] - b.wcount[0];
        float refl[3];
        for (int a = 0; a < 3; a++) {
            const float r = reflectivity[3 * (int64_t)b.patches[0].face + a];
            refl[a] = r < kMaxReflectivity ? r : kMaxReflectivity;
        }
        for (size_t k = 0; k < b.patches.size(); k++) {
            vrad_patch p = b.patches[k];
            p.parent = global(p.parent);
            p.child1 = global(p.child1);
            p.child2 = global(p.child2);
            p.first_point = (int32_t)(k == 0 ? root_pt[(size_t)i] : desc0 + b.wfirst[k]);
            p.num_points = b.wcount[k];
            for (int a = 0; a < 3; a++) p.reflectivity[a] = refl[a];
            sink.put(global((int32_t)k), p, &b.pts[(size_t)b.wfirst[k]].x);
        }
    });
    for (int32_t i = 0; i < roots; i++) {
        const Builder &b = subtree[(size_t)i];
        const int32_t f = b.patches[0].face;
        out.face_first[(size_t)f] = base[(size_t)i];
        out.face_end[(size_t)f] = base[(size_t)i] + (int32_t)b.patches.size() - 1;
        out.face_root[(size_t)f] = i;
    }
    out.npatches = total;
    out.npoints = npoints;
    out.roots = roots;
    clock.mark("merge");
    return true;
}

bool build_patch_tree(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                      const float *reflectivity, float max_chop, float min_chop, PatchTree &out, PatchSink &sink,
                      std::string &why) {
    PatchForest forest;
    return forest.grow(faces, nfaces, vertices, nvertices, max_chop, min_chop, why) &&
           forest.merge(reflectivity, out, sink, why);
}

}  // namespace vrad

extern "C" int32_t vrad_build_patches(const vrad_face *faces, int32_t nfaces, const float *vertices,
                                      int64_t nvertices, const float *reflectivity, float max_chop, float min_chop,
                                      vrad_patch *out, int64_t capacity, int64_t *count, float *points,
                                      int64_t point_capacity, int64_t *point_count) {
    if (nfaces < 0 || (nfaces > 0 && (!faces || !vertices || !reflectivity)) || !count || !point_count)
        return VRAD_ERR_ARG;
    if (!(max_chop > 0.0f) || !(min_chop > 0.0f)) return VRAD_ERR_ARG;
    vrad::PatchTree tree;
    vrad::PatchArrays arrays;
    std::string why;
    if (!vrad::build_patch_tree(faces, nfaces, vertices, nvertices, reflectivity, max_chop, min_chop, tree, arrays, why))
        return VRAD_ERR_ARG;
    *count = (int64_t)arrays.patches.size();
    *point_count = (int64_t)arrays.points.size() / 3;
    if (!out && !points) return VRAD_OK;  // a counting pass
    if ((out && capacity < *count) || (points && point_capacity < *point_count)) return VRAD_ERR_ARG;
    if (out) std::memcpy(out, arrays.patches.data(), sizeof(vrad_patch) * arrays.patches.size());
    if (points) std::memcpy(points, arrays.points.data(), sizeof(float) * arrays.points.size());
    return VRAD_OK;
}
