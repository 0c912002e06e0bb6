// kd_build_oracle.cpp -- restatement of the reference's SAH KD-tree build
// (MapTools/Tracing/KdTreeBuilder.cs), so the oracle can run the
// reference's own CPU traversal on scenes the reference never recorded.
//
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).  The sequential recursion
// (KdTreeBuilder.Build / RefineNode, KdTreeBuilder.cs:130-150, 828-866)
// defines the tree; the reference's parallel build is required to produce
// the same nodes.  Pinned node for node against the reference's recorded
// stock trees (tests/test_oracle_fixtures.py).

#include "vrad_oracle.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

constexpr float kCostTraversal = 75.0f;     // KdTreeBuilder.cs:40
constexpr float kCostIntersection = 167.0f; // KdTreeBuilder.cs:43
constexpr int kMaxDepth = 21;               // KdTreeBuilder.cs:46
constexpr float kHuge = 1.0e23f;
constexpr int kMaxTrials = 34;

// .NET MathF.Min / MathF.Max: NaN propagates; -0 orders below +0.
inline float net_min(float a, float b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a < b) return a;
    if (b < a) return b;
    return std::signbit(a) ? a : b;
}
inline float net_max(float a, float b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a > b) return a;
    if (b > a) return b;
    return std::signbit(a) ? b : a;
}

struct V3 {
    float v[3];
};

// BoxSurfaceArea (KdTreeBuilder.cs:567-580): float products and sums, a
// double doubling, rounded back to float.
inline float box_area(const V3 &mn, const V3 &mx) {
    float dx = mx.v[0] - mn.v[0], dy = mx.v[1] - mn.v[1], dz = mx.v[2] - mn.v[2];
    float s = ((dx * dz) + (dx * dy)) + (dy * dz);
    return (float)(2.0 * (double)s);
}

// ClassifyAgainstAxisSplit (KdTreeBuilder.cs:650-667): 1 right, -1 left, 0 both.
inline int classify(float minc, float maxc, float split) {
    if (minc >= split) return 1;
    if (maxc <= split) return -1;
    if (minc == maxc) return 1;
    return 0;
}

struct Builder {
    const float *v9;
    std::vector<orc_kdnode> nodes;
    std::vector<int32_t> indices;

    float coord(int tri, int vert, int axis) const { return v9[9 * tri + 3 * vert + axis]; }

    struct Best {
        float cost = kHuge;
        int axis = 0;
        float trial = 0, value = 0;
        int nl = 0, nr = 0, nb = 0;
    };

    void make_leaf(int node, const std::vector<int> &list, int off, int count) {
        orc_kdnode &n = nodes[node];
        n.children = 3 + ((int32_t)indices.size() << 2);
        int32_t c = count;
        std::memcpy(&n.split, &c, 4);
        for (int t = 0; t < count; t++) indices.push_back(list[off + t]);
    }

    // RefineNode + ChooseSplit + Finalise (KdTreeBuilder.cs:828-1030).
    void refine(int node, const std::vector<int> &list, int off, int count, V3 mn, V3 mx,
                int depth) {
        if (count < 3 || depth > kMaxDepth) {
            make_leaf(node, list, off, count);
            return;
        }
        Best best;
        std::vector<float> mins[3], maxs[3];
        for (int axis = 0; axis < 3; axis++) {
            mins[axis].resize(count);
            maxs[axis].resize(count);
            // AxisExtents (KdTreeBuilder.cs:582-603).
            float minc = kHuge, maxc = -kHuge;
            for (int t = 0; t < count; t++) {
                int tri = list[off + t];
                float a = coord(tri, 0, axis), b = coord(tri, 1, axis), c = coord(tri, 2, axis);
                minc = net_min(net_min(net_min(minc, a), b), c);
                maxc = net_max(net_max(net_max(maxc, a), b), c);
                mins[axis][t] = net_min(net_min(a, b), c);
                maxs[axis][t] = net_max(net_max(a, b), c);
            }
            // CollectTrialSplits (KdTreeBuilder.cs:605-642).
            float splits[kMaxTrials];
            int ns = 0;
            int skip = 1 + count / 10;
            for (int ts = -1; ts < count; ts += skip) {
                for (int tv = 0; tv < 3; tv++) {
                    float trial;
                    if (ts == -1) {
                        trial = 0.5f * (mn.v[axis] + mx.v[axis]);
                    } else {
                        trial = coord(list[off + ts], tv, axis);
                        if (trial > mx.v[axis] || trial < mn.v[axis]) continue;
                    }
                    splits[ns++] = trial;
                    if (ts == -1) break;
                }
            }
            // CalculateCostsOfSplit (KdTreeBuilder.cs:720-760) per trial.
            float isa = (float)(1.0 / (double)box_area(mn, mx));
            for (int k = 0; k < ns; k++) {
                float value = splits[k];
                int nl = 0, nr = 0;
                for (int t = 0; t < count; t++) {
                    int c = classify(mins[axis][t], maxs[axis][t], value);
                    if (c < 0) nl++;
                    else if (c > 0) nr++;
                }
                int nb = count - nl - nr;
                if (nl != 0 && nb == 0 && nr == 0) value = maxc;
                if (nr != 0 && nb == 0 && nl == 0) value = minc;
                V3 lmax = mx, rmin = mn;
                lmax.v[axis] = value;
                rmin.v[axis] = value;
                float sal = box_area(mn, lmax), sar = box_area(rmin, mx);
                float inner = ((float)nb + (sal * isa) * (float)nl) + (sar * isa) * (float)nr;
                float cost = kCostTraversal + kCostIntersection * inner;
                if (cost < best.cost) {
                    best.cost = cost;
                    best.axis = axis;
                    best.trial = splits[k];
                    best.value = value;
                    best.nl = nl;
                    best.nr = nr;
                    best.nb = nb;
                }
            }
        }
        // Finalise (KdTreeBuilder.cs:934-1004).
        float no_split = kCostIntersection * (float)count;
        if (no_split <= best.cost || depth > kMaxDepth) {
            make_leaf(node, list, off, count);
            return;
        }
        std::vector<int> part(count);
        int nlo = 0, nbo = 0, nro = 0;
        for (int t = 0; t < count; t++) {
            int idx = list[off + t];
            switch (classify(mins[best.axis][t], maxs[best.axis][t], best.trial)) {
                case -1: part[nlo++] = idx; break;
                case 1: nro++; part[count - nro] = idx; break;
                default: part[best.nl + nbo] = idx; nbo++; break;
            }
        }
        if (count < 20 && (best.nl == 0 || best.nr == 0)) depth += 100;
        int child_depth = depth + 1;
        V3 lmax = mx, rmin = mn;
        lmax.v[best.axis] = best.value;
        rmin.v[best.axis] = best.value;

        int left = (int)nodes.size();
        nodes[node].children = best.axis + (left << 2);
        nodes[node].split = best.value;
        nodes.push_back(orc_kdnode{0, 0.0f});
        nodes.push_back(orc_kdnode{0, 0.0f});
        refine(left, part, 0, best.nl + best.nb, mn, lmax, child_depth);
        refine(left + 1, part, best.nl, best.nr + best.nb, rmin, mx, child_depth);
    }
};

}  // namespace

extern "C" int orc_kd_build(const float *v9, const int32_t *ids, const uint8_t *flags, int32_t n,
                            orc_kdtree *out) {
    if (!v9 || !out || n <= 0) return -1;  // RefuseEmpty (KdTreeBuilder.cs:520-529)
    std::memset(out, 0, sizeof(*out));
    // SceneExtent (KdTreeBuilder.cs:551-565).
    V3 mn, mx;
    for (int a = 0; a < 3; a++) {
        float lo = kHuge, hi = -kHuge;
        for (int32_t i = 0; i < n; i++) {
            float p = v9[9 * i + a], q = v9[9 * i + 3 + a], r = v9[9 * i + 6 + a];
            lo = net_min(net_min(net_min(lo, p), q), r);
            hi = net_max(net_max(net_max(hi, p), q), r);
        }
        mn.v[a] = lo;
        mx.v[a] = hi;
    }
    Builder b;
    b.v9 = v9;
    b.nodes.push_back(orc_kdnode{0, 0.0f});
    std::vector<int> root(n);
    for (int32_t i = 0; i < n; i++) root[i] = i;
    b.refine(0, root, 0, n, mn, mx, 0);

    out->nnodes = (int32_t)b.nodes.size();
    out->nodes = (orc_kdnode *)std::malloc(sizeof(orc_kdnode) * b.nodes.size());
    std::memcpy(out->nodes, b.nodes.data(), sizeof(orc_kdnode) * b.nodes.size());
    out->nindices = (int32_t)b.indices.size();
    out->indices = (int32_t *)std::malloc(sizeof(int32_t) * (b.indices.size() + 1));
    if (!b.indices.empty())
        std::memcpy(out->indices, b.indices.data(), sizeof(int32_t) * b.indices.size());
    out->ntris = n;
    out->tris = (orc_tri *)std::malloc(sizeof(orc_tri) * n);
    orc_tri_prepare(v9, ids, flags, n, out->tris);
    for (int a = 0; a < 3; a++) {
        out->bounds[a] = mn.v[a];
        out->bounds[3 + a] = mx.v[a];
    }
    return 0;
}

extern "C" void orc_kd_free(orc_kdtree *t) {
    if (!t) return;
    std::free(t->nodes);
    std::free(t->indices);
    std::free(t->tris);
    std::memset(t, 0, sizeof(*t));
}
