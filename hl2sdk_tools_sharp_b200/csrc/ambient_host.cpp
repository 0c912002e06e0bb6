// ambient_host.cpp -- the leaf ambient stage's sample positions, on the host.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad/Ambient):
//   StockRandomStream (StockRandomStream.cs:13-234): stock's
//     CUniformRandomStream, the Park-Miller minimal standard generator with
//     a 32-entry Bays-Durham shuffle (Numerical Recipes' ran1), seeded 0;
//     RandomFloat scales (float)(AM * draw), clamped to RNMX, into [lo, hi];
//   BspParents (BspParents.cs:31-96): every node's and leaf's parent, from a
//     depth-first walk of the tree (a leaf no node names keeps parent 0);
//   LeafBoundaryPlanes.Gather (LeafBoundaryPlanes.cs:32-70): the planes from
//     the leaf up to the root, each facing the leaf's side;
//   LeafBrushTrace (LeafBrushTrace.cs:43-265): the segment against the
//     leaf's opaque brushes in leaf-brush order, the first brush that clips
//     it (or holds its start) answering; bevel sides skipped; the clip's
//     DIST_EPSILON arithmetic in double as stock's;
//   LeafSampler.Generate (LeafSampler.cs:38-148): up to 1000 draws of a
//     point in the leaf's box, kept when it is 1/32 inside every boundary
//     plane and the six axis segments to the box's faces neither start in
//     a brush nor leave through a brush's back; otherwise the box's centre;
//   LeafAmbientBuilder.CandidateSampleCount (LeafAmbientBuilder.cs:420-454):
//     (size x / 32) cubed, clamped to 1..128 (stock's quirk sizes all three
//     axes by x).
// Every float operation is the reference's, in its order (this file is built
// with -ffp-contract=off); each leaf's stream starts from seed 0, so leaves
// are independent and run on the host pool.

#include <cstdint>
#include <cstring>
#include <vector>

#include "host_parallel.h"
#include "vrad_cuda.h"

int32_t vrad_fail(struct vrad_ctx *ctx, int32_t code, const char *fmt, ...);

namespace {

constexpr int kMaxTries = 1000;
constexpr int kMaxSamples = 128;
constexpr int kContentsSolid = 0x1;
constexpr int kMaskOpaque = 0x1 | 0x4000 | 0x80;
constexpr float kDistEpsilonSingle = 0.03125f;
constexpr double kDistEpsilon = 0.03125;
constexpr float kNeverUpdated = -9999.0f;

class Ran1 {
public:
    Ran1() { seed(0); }
    void seed(int32_t s) {
        idum_ = s < 0 ? s : -s;
        iy_ = 0;
    }
    int32_t next() {
        int32_t k;
        if (idum_ <= 0 || iy_ == 0) {
            idum_ = (-idum_ < 1) ? 1 : -idum_;
            for (int j = kNtab + 7; j >= 0; j--) {
                k = idum_ / kIq;
                idum_ = kIa * (idum_ - k * kIq) - kIr * k;
                if (idum_ < 0) idum_ += kIm;
                if (j < kNtab) iv_[j] = idum_;
            }
            iy_ = iv_[0];
        }
        k = idum_ / kIq;
        idum_ = kIa * (idum_ - k * kIq) - kIr * k;
        if (idum_ < 0) idum_ += kIm;
        const int slot = iy_ / kNdiv;
        iy_ = iv_[slot];
        iv_[slot] = idum_;
        return iy_;
    }
    float uniform(float lo, float hi) {
        float fl = (float)(kAm * (double)next());
        if ((double)fl > kRnmx) fl = (float)kRnmx;
        return fl * (hi - lo) + lo;
    }

private:
    static constexpr int32_t kNtab = 32, kIa = 16807, kIm = 2147483647, kIq = 127773, kIr = 2836;
    static constexpr int32_t kNdiv = 1 + (kIm - 1) / kNtab;
    static constexpr double kAm = 1.0 / kIm;
    static constexpr double kRnmx = 1.0 - 1.2e-7;
    int32_t idum_ = 0, iy_ = 0;
    int32_t iv_[kNtab] = {};
};

struct V3 {
    float x, y, z;
};

inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct Plane {
    V3 n;
    float d;
};

struct Tree {
    const vrad_ambient_tree *t;
    std::vector<int32_t> node_parent, leaf_parent;

    V3 plane_normal(int p) const { return {t->planes[4 * p], t->planes[4 * p + 1], t->planes[4 * p + 2]}; }
    float plane_dist(int p) const { return t->planes[4 * p + 3]; }
    const int32_t *leaf(int l) const { return t->leaves + 9 * l; }
};

// LeafBrushTrace.ClipToBrush.
struct BrushHit {
    float frac;
    V3 normal;
    bool start_solid;
};

BrushHit clip_to_brush(const Tree &T, int brush, V3 p1, V3 p2) {
    const int32_t *b = T.t->brushes + 3 * brush;
    const int first = b[0], count = b[1];
    if (count == 0) return {1.0f, {0, 0, 0}, false};
    float enter = kNeverUpdated, leave = 1.0f;
    int clip_plane = -1;
    bool start_out = false;
    for (int i = 0; i < count; i++) {
        const int32_t *side = T.t->brush_sides + 2 * (first + i);
        if (side[1] == 1) continue;  // bevel
        const int p = side[0];
        const V3 n = T.plane_normal(p);
        const float dist = T.plane_dist(p);
        const float d1 = dot(p1, n) - dist;
        const float d2 = dot(p2, n) - dist;
        if (d1 > 0 && d2 > 0) return {1.0f, {0, 0, 0}, false};
        if (d1 > 0) start_out = true;
        if (d1 <= 0 && d2 <= 0) continue;
        if (d1 > d2) {
            const float f = (float)(((double)d1 - kDistEpsilon) / (double)(d1 - d2));
            if (f > enter) {
                enter = f;
                clip_plane = p;
            }
        } else {
            const float f = (float)(((double)d1 + kDistEpsilon) / (double)(d1 - d2));
            if (f < leave) leave = f;
        }
    }
    if (!start_out) return {1.0f, {0, 0, 0}, true};
    if (enter < leave && enter > kNeverUpdated && enter < 1.0f) {
        if (enter < 0) enter = 0;
        return {enter, T.plane_normal(clip_plane), false};
    }
    return {1.0f, {0, 0, 0}, false};
}

// LeafBrushTrace.Trace: the first opaque brush, in leaf-brush order, that
// clips the segment or holds its start.
BrushHit trace_leaf_brushes(const Tree &T, int leaf, V3 start, V3 end) {
    const int32_t *L = T.leaf(leaf);
    for (int i = 0; i < L[8]; i++) {
        const int brush = T.t->leaf_brushes[L[7] + i];
        if ((T.t->brushes[3 * brush + 2] & kMaskOpaque) == 0) continue;
        BrushHit h = clip_to_brush(T, brush, start, end);
        if (h.frac != 1.0f || h.start_solid) {
            if (h.start_solid) h.frac = 0.0f;
            return h;
        }
    }
    return {1.0f, {0, 0, 0}, false};
}

// LeafBoundaryPlanes.Gather.
void boundary_planes(const Tree &T, int leaf, std::vector<Plane> &out) {
    out.clear();
    int node = T.leaf_parent[(size_t)leaf];
    int child = -(leaf + 1);
    while (node >= 0) {
        const int32_t *N = T.t->nodes + 3 * node;
        const int p = N[0];
        const V3 n = T.plane_normal(p);
        const float d = T.plane_dist(p);
        if (N[1] == child)
            out.push_back({n, d});
        else
            out.push_back({{-n.x, -n.y, -n.z}, -d});
        child = node;
        node = T.node_parent[(size_t)child];
    }
}

int candidate_count(const int32_t *L) {
    int x = (L[4] - L[1]) / 32;
    x = x < 1 ? 1 : x;
    const int y = x, z = x;  // stock sizes all three axes by x
    // int arithmetic that wraps, as the reference's unchecked product does
    const int32_t v = (int32_t)((uint32_t)x * (uint32_t)y * (uint32_t)z);
    return v < 1 ? 1 : (v > kMaxSamples ? kMaxSamples : v);
}

// LeafSampler.Generate for one draw sequence.
V3 generate(const Tree &T, int leaf, const std::vector<Plane> &planes, Ran1 &rng) {
    const int32_t *L = T.leaf(leaf);
    const float mn[3] = {(float)L[1], (float)L[2], (float)L[3]};
    const float mx[3] = {(float)L[4], (float)L[5], (float)L[6]};
    const float dx = (float)(L[4] - L[1]), dy = (float)(L[5] - L[2]), dz = (float)(L[6] - L[3]);
    V3 pos{0, 0, 0};
    bool valid = false;
    for (int i = 0; i < kMaxTries && !valid; i++) {
        const float a = rng.uniform(0.0f, dx);
        const float b = rng.uniform(0.0f, dy);
        const float c = rng.uniform(0.0f, dz);
        pos = {mn[0] + a, mn[1] + b, mn[2] + c};
        valid = true;
        for (int j = (int)planes.size(); --j >= 0 && valid;) {
            const float d = dot(planes[(size_t)j].n, pos) - planes[(size_t)j].d;
            if (d < kDistEpsilonSingle) valid = false;
        }
        if (!valid) continue;
        for (int j = 0; j < 6; j++) {
            const int axis = j % 3;
            const float bound = j < 3 ? mn[axis] : mx[axis];
            V3 start = pos;
            (axis == 0 ? start.x : axis == 1 ? start.y : start.z) = bound;
            const BrushHit h = trace_leaf_brushes(T, leaf, pos, start);
            float t = h.frac;
            V3 normal = h.normal;
            if (!(h.frac != 1.0f || h.start_solid)) {
                t = 1.0f;
                normal = {0, 0, 0};
            }
            if (t == 0.0f) {
                valid = false;  // inside a detail brush
                break;
            }
            if (t != 1.0f) {
                const V3 delta{start.x - pos.x, start.y - pos.y, start.z - pos.z};
                if (dot(delta, normal) > 0) {
                    valid = false;
                    break;
                }
            }
        }
    }
    if (!valid) {
        pos = {(mn[0] + mx[0]) * 0.5f, (mn[1] + mx[1]) * 0.5f, (mn[2] + mx[2]) * 0.5f};
    }
    return pos;
}

bool parents(const vrad_ambient_tree *t, Tree &T) {
    T.node_parent.assign((size_t)t->nnodes, 0);
    T.leaf_parent.assign((size_t)t->nleaves, 0);
    if (t->nnodes == 0) return true;
    T.node_parent[0] = -1;
    std::vector<int> pending{0};
    std::vector<char> seen((size_t)t->nnodes, 0);
    seen[0] = 1;
    while (!pending.empty()) {
        const int n = pending.back();
        pending.pop_back();
        for (int i = 0; i < 2; i++) {
            const int child = t->nodes[3 * n + 1 + i];
            if (child < 0) {
                const int leaf = -child - 1;
                if (leaf >= t->nleaves) return false;
                T.leaf_parent[(size_t)leaf] = n;
            } else {
                if (child >= t->nnodes || seen[(size_t)child]) return false;  // not a tree
                seen[(size_t)child] = 1;
                T.node_parent[(size_t)child] = n;
                pending.push_back(child);
            }
        }
    }
    return true;
}

}  // namespace

extern "C" int32_t vrad_leaf_ambient_positions(const vrad_ambient_tree *t, int32_t *counts, float *positions,
                                               int64_t capacity, int64_t *total, int32_t threads) {
    if (!t || !counts || !total || t->nplanes < 0 || t->nnodes < 0 || t->nleaves < 0 || t->nleaf_brushes < 0 ||
        t->nbrushes < 0 || t->nbrush_sides < 0 || (t->nplanes && !t->planes) || (t->nnodes && !t->nodes) ||
        (t->nleaves && !t->leaves) || (t->nleaf_brushes && !t->leaf_brushes) || (t->nbrushes && !t->brushes) ||
        (t->nbrush_sides && !t->brush_sides))
        return vrad_fail(nullptr, VRAD_ERR_ARG, "invalid leaf ambient tree");
    // Every index the sampler follows is checked once, here.
    for (int32_t n = 0; n < t->nnodes; n++)
        if (t->nodes[3 * n] < 0 || t->nodes[3 * n] >= t->nplanes)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "node %d names plane %d", n, t->nodes[3 * n]);
    for (int32_t b = 0; b < t->nbrushes; b++) {
        const int32_t first = t->brushes[3 * b], count = t->brushes[3 * b + 1];
        if (first < 0 || count < 0 || (int64_t)first + count > t->nbrush_sides)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "brush %d's sides lie outside the side list", b);
    }
    for (int32_t s = 0; s < t->nbrush_sides; s++)
        if (t->brush_sides[2 * s] < 0 || t->brush_sides[2 * s] >= t->nplanes)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "brush side %d names plane %d", s, t->brush_sides[2 * s]);
    for (int32_t k = 0; k < t->nleaf_brushes; k++)
        if (t->leaf_brushes[k] < 0 || t->leaf_brushes[k] >= t->nbrushes)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "leaf brush %d names brush %d", k, t->leaf_brushes[k]);
    int64_t sum = 0;
    std::vector<int64_t> first((size_t)t->nleaves + 1, 0);
    for (int32_t l = 0; l < t->nleaves; l++) {
        const int32_t *L = t->leaves + 9 * l;
        if (L[7] < 0 || L[8] < 0 || (int64_t)L[7] + L[8] > t->nleaf_brushes)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "leaf %d's brushes lie outside the leaf brush list", l);
        counts[l] = (L[0] & kContentsSolid) ? 0 : candidate_count(L);
        first[(size_t)l] = sum;
        sum += counts[l];
    }
    first[(size_t)t->nleaves] = sum;
    *total = sum;
    if (!positions) return VRAD_OK;
    if (capacity < sum) return vrad_fail(nullptr, VRAD_ERR_ARG, "%lld positions, room for %lld", (long long)sum,
                                         (long long)capacity);
    Tree T{t, {}, {}};
    if (!parents(t, T)) return vrad_fail(nullptr, VRAD_ERR_ARG, "the nodes do not form a tree");
    auto one = [&](int64_t l) {
        const int n = counts[l];
        if (n == 0) return;
        std::vector<Plane> planes;
        boundary_planes(T, (int)l, planes);
        Ran1 rng;  // each leaf's own stream, seeded 0
        float *out = positions + 3 * first[(size_t)l];
        for (int i = 0; i < n; i++) {
            const V3 p = generate(T, (int)l, planes, rng);
            out[3 * i] = p.x;
            out[3 * i + 1] = p.y;
            out[3 * i + 2] = p.z;
        }
    };
    if (threads == 1) {
        for (int64_t l = 0; l < t->nleaves; l++) one(l);
    } else {
        vrad::parallel_for(t->nleaves, 4, one);
    }
    return VRAD_OK;
}
