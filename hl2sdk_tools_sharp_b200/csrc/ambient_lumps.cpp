// ambient_lumps.cpp -- the leaf ambient stage's last steps on the host: each
// leaf's samples into the 16-sample list, compressed, and the two lumps
// (LEAF_AMBIENT_INDEX, LEAF_AMBIENT_LIGHTING) with empty leaves pointed at
// their nearest lit neighbour.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad/Ambient):
//   AmbientSampleList.Add (AmbientSampleList.cs:40-130): past 16 samples,
//     evict the sample whose nearest neighbour is closest, the distance
//     scaled by 0.1 + 0.9 x the pair's largest colour difference (below
//     1e-4 counts as 0, above 1 as 1); stock's tie-break never fires
//     (StockQuirk.AmbientSampleTieBreakNeverFires), the Correct mode breaks
//     a distance tie on the summed colour differences; the last sample
//     fills the hole;
//   AmbientSampleList.Compress (:132-160): a sample whose cube the others'
//     inverse-square weighted mean reproduces within 3 steps of the screen
//     gamma table is dropped (ColorAtPosition :162-196,
//     CubeDeltaGammaSpace :198-222);
//   LeafAmbientBuilder.Encode (LeafAmbientBuilder.cs:503-560): per leaf its
//     count and first record; each record the 8-bit position fractions of
//     the leaf's box (Fixed8Fraction :660-670) and six RGBE colours
//     (StockLightColor.Encode, StockLightColor.cs:110-150);
//   NearestNeighborWithLight (:562-640): an empty leaf's first record is the
//     leaf, among those a box three times its size touches
//     (ToolBspTree.EnumerateLeavesInBox, ToolBspTree.cs:20-90), with samples
//     and the nearest box (AabbDistance).
// Every float operation is the reference's, in its order (this file is built
// with -ffp-contract=off).  Leaves are independent until the neighbour
// search, so the lists run on the host pool.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "host_parallel.h"
#include "vrad_cuda.h"

int32_t vrad_fail(struct vrad_ctx *ctx, int32_t code, const char *fmt, ...);

namespace {

constexpr int kMaxSamples = 16;
constexpr int kContentsSolid = 0x1;
constexpr float kTestEpsilon = 0.03125f;

struct V3 {
    float x, y, z;
};

inline float length(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
inline float length_sq(V3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }

struct Sample {
    V3 pos;
    V3 cube[6];
};

inline float max_of(float a, float b) { return a > b ? a : b; }

// AmbientSampleList.Add.
void add_sample(std::vector<Sample> &list, const Sample &s, bool dead_tiebreak) {
    list.push_back(s);
    if ((int)list.size() <= kMaxSamples) return;
    const int n = (int)list.size();
    int nearest = 0;
    float nearest_dist = 3.402823466e38f, nearest_total = 0.0f;
    for (int i = 0; i < n; i++) {
        const Sample &a = list[(size_t)i];
        float closest = 3.402823466e38f, total = 0.0f;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            const Sample &b = list[(size_t)j];
            float dist = length(sub(a.pos, b.pos));
            float max_dc = 0.0f;
            for (int k = 0; k < 6; k++) {
                max_dc = max_of(max_dc, std::fabs(a.cube[k].x - b.cube[k].x));
                max_dc = max_of(max_dc, std::fabs(a.cube[k].y - b.cube[k].y));
                max_dc = max_of(max_dc, std::fabs(a.cube[k].z - b.cube[k].z));
                total += max_dc;
            }
            if (max_dc < 1e-4f) max_dc = 0.0f;
            else if (max_dc > 1.0f) max_dc = 1.0f;
            const float factor = 0.1f + (max_dc * 0.9f);
            dist *= factor;
            if (dist < closest) closest = dist;
        }
        const bool better = closest < nearest_dist || (!dead_tiebreak && closest == nearest_dist && total < nearest_total);
        if (better) {
            nearest_dist = closest;
            nearest = i;
            if (!dead_tiebreak) nearest_total = total;
        }
    }
    list[(size_t)nearest] = list.back();
    list.pop_back();
}

// StockLightColor.LinearToScreenGamma over the caller's 1,024-entry table.
inline int screen_gamma(float f, const int32_t *table) {
    int i = (int)(f * 1023);
    if (i < 0) i = 0;
    if (i > 1023) i = 1023;
    return table[i];
}

// AmbientSampleList.Compress.
void compress(std::vector<Sample> &list, const int32_t *gamma) {
    for (int i = 0; i < (int)list.size(); i++) {
        if (list.size() <= 1) continue;
        V3 test[6];
        for (auto &t : test) t = {0.0f, 0.0f, 0.0f};
        float total = 0.0f;
        for (int k = 0; k < (int)list.size(); k++) {
            if (k == i) continue;
            const float dist = length_sq(sub(list[(size_t)k].pos, list[(size_t)i].pos));
            const float factor = 1.0f / (dist + 1.0f);
            total += factor;
            for (int j = 0; j < 6; j++) {
                const V3 c = list[(size_t)k].cube[j];
                test[j] = {test[j].x + c.x * factor, test[j].y + c.y * factor, test[j].z + c.z * factor};
            }
        }
        const float inv = 1.0f / total;
        int delta = 0;
        for (int j = 0; j < 6; j++) {
            const V3 t = {test[j].x * inv, test[j].y * inv, test[j].z * inv};
            const float a[3] = {t.x, t.y, t.z};
            const float b[3] = {list[(size_t)i].cube[j].x, list[(size_t)i].cube[j].y, list[(size_t)i].cube[j].z};
            for (int c = 0; c < 3; c++) {
                const int d = std::abs(screen_gamma(a[c], gamma) - screen_gamma(b[c], gamma));
                if (d > delta) delta = d;
            }
        }
        if (delta < 3) {
            list[(size_t)i] = list.back();
            list.pop_back();
            i--;
        }
    }
}

// StockLightColor.Encode: RGBE with the exponent from the largest channel.
void encode_rgbe(V3 v, uint8_t *out) {
    float mx;
    if (v.x > v.y) mx = v.x > v.z ? v.x : v.z;
    else mx = v.y > v.z ? v.y : v.z;
    int e = 0;
    if (mx != 0.0f) {
        uint32_t bits;
        std::memcpy(&bits, &mx, 4);
        e = (int)((bits & 0x7F800000u) >> 23) - (7 + 127);
    }
    const uint32_t sbits = (uint32_t)(127 - e) << 23;
    float scalar;
    std::memcpy(&scalar, &sbits, 4);
    // (byte)(int)(c * scalar): truncation toward zero, then the low byte.
    auto chan = [&](float c) -> uint8_t {
        const float p = c * scalar;
        const int iv = std::isnan(p) ? 0 : (p >= 2147483648.0f ? 2147483647 : (p < -2147483648.0f ? (int)0x80000000 : (int)p));
        return (uint8_t)(iv & 0xFF);
    };
    out[0] = chan(v.x);
    out[1] = chan(v.y);
    out[2] = chan(v.z);
    out[3] = (uint8_t)(int8_t)e;
}

// LeafAmbientBuilder.Fixed8Fraction.
uint8_t fixed8(float t, float lo, float hi) {
    if (hi <= lo) return 0;
    float cv = (t - lo) / (hi - lo);
    cv = cv < 0.0f ? 0.0f : (cv > 1.0f ? 1.0f : cv);
    const float frac = 0.0f + ((255.0f - 0.0f) * cv);
    return (uint8_t)((int)(frac + 0.5f) & 0xFF);
}

struct Tree {
    const vrad_ambient_tree *t;
    V3 mins(int l) const {
        const int32_t *L = t->leaves + 9 * l;
        return {(float)L[1], (float)L[2], (float)L[3]};
    }
    V3 maxs(int l) const {
        const int32_t *L = t->leaves + 9 * l;
        return {(float)L[4], (float)L[5], (float)L[6]};
    }
};

// ToolBspTree.EnumerateLeavesInBox: front child first and completely.
bool leaves_in_box(const Tree &T, V3 mn, V3 mx, std::vector<int> &into) {
    into.clear();
    int pending[256];
    int sp = 0;
    pending[sp++] = 0;
    const float bmin[3] = {mn.x, mn.y, mn.z}, bmax[3] = {mx.x, mx.y, mx.z};
    while (sp > 0) {
        int node = pending[--sp];
        while (node >= 0) {
            const int32_t *N = T.t->nodes + 3 * node;
            const float *P = T.t->planes + 4 * N[0];
            float cmin[3], cmax[3];
            for (int i = 0; i < 3; i++) {
                if (P[i] >= 0) {
                    cmin[i] = bmin[i];
                    cmax[i] = bmax[i];
                } else {
                    cmin[i] = bmax[i];
                    cmax[i] = bmin[i];
                }
            }
            const float dot_max = (P[0] * cmax[0]) + (P[1] * cmax[1]) + (P[2] * cmax[2]);
            const float dot_min = (P[0] * cmin[0]) + (P[1] * cmin[1]) + (P[2] * cmin[2]);
            if (dot_max - P[3] <= -kTestEpsilon) {
                node = N[2];
            } else if (dot_min - P[3] >= kTestEpsilon) {
                node = N[1];
            } else {
                if (sp >= 256) return false;
                pending[sp++] = N[2];
                node = N[1];
            }
        }
        into.push_back(-node - 1);
    }
    return true;
}

// LeafAmbientBuilder.AabbDistance.
float aabb_distance(V3 mn0, V3 mx0, V3 mn1, V3 mx1) {
    const float a0[3] = {mn0.x, mn0.y, mn0.z}, b0[3] = {mx0.x, mx0.y, mx0.z};
    const float a1[3] = {mn1.x, mn1.y, mn1.z}, b1[3] = {mx1.x, mx1.y, mx1.z};
    float d[3];
    for (int i = 0; i < 3; i++) {
        const float gmin = std::fmax(a0[i], a1[i]);
        const float lmax = std::fmin(b0[i], b1[i]);
        d[i] = gmin < lmax ? 0.0f : lmax - gmin;
    }
    return length({d[0], d[1], d[2]});
}

}  // namespace

extern "C" int32_t vrad_leaf_ambient_lumps(const vrad_ambient_tree *t, const int32_t *counts, const float *positions,
                                           const float *cubes, const int32_t *gamma_table, int32_t correct_tiebreak,
                                           uint8_t *index_out, uint8_t *lighting_out, int64_t capacity,
                                           int64_t *records, int32_t *bad_leaves) {
    if (!t || !counts || !gamma_table || !index_out || !records || t->nleaves < 0 || (t->nleaves && !t->leaves) ||
        t->nnodes < 1 || !t->nodes || !t->planes)
        return vrad_fail(nullptr, VRAD_ERR_ARG, "invalid leaf ambient lump arguments");
    for (int32_t n = 0; n < t->nnodes; n++) {
        const int32_t *N = t->nodes + 3 * n;
        if (N[0] < 0 || N[0] >= t->nplanes || N[1] >= t->nnodes || N[2] >= t->nnodes || -N[1] - 1 >= t->nleaves ||
            -N[2] - 1 >= t->nleaves)
            return vrad_fail(nullptr, VRAD_ERR_ARG, "node %d names a plane, node or leaf the map does not have", n);
    }
    const int L = t->nleaves;
    std::vector<int64_t> first((size_t)L + 1, 0);
    for (int l = 0; l < L; l++) {
        if (counts[l] < 0) return vrad_fail(nullptr, VRAD_ERR_ARG, "leaf %d has %d samples", l, counts[l]);
        first[(size_t)l + 1] = first[(size_t)l] + counts[l];
    }
    if (first[(size_t)L] && (!positions || !cubes)) return vrad_fail(nullptr, VRAD_ERR_ARG, "null samples");
    // Each leaf's list, added in sample order and compressed.
    std::vector<std::vector<Sample>> lists((size_t)L);
    vrad::parallel_for(L, 4, [&](int64_t l) {
        std::vector<Sample> &list = lists[(size_t)l];
        for (int64_t k = first[(size_t)l]; k < first[(size_t)l + 1]; k++) {
            Sample s;
            s.pos = {positions[3 * k], positions[3 * k + 1], positions[3 * k + 2]};
            for (int j = 0; j < 6; j++)
                s.cube[j] = {cubes[18 * k + 3 * j], cubes[18 * k + 3 * j + 1], cubes[18 * k + 3 * j + 2]};
            add_sample(list, s, correct_tiebreak == 0);
        }
        compress(list, gamma_table);
    });
    int64_t total = 0;
    for (auto &l : lists) total += (int64_t)l.size();
    *records = total;
    if (total > 0xFFFF) return vrad_fail(nullptr, VRAD_ERR_ARG, "%lld samples do not fit the 16-bit index", (long long)total);
    if (!lighting_out) return VRAD_OK;
    if (capacity < total) return vrad_fail(nullptr, VRAD_ERR_ARG, "%lld records, room for %lld", (long long)total,
                                           (long long)capacity);
    const Tree T{t};
    std::vector<uint16_t> count((size_t)L), firstrec((size_t)L);
    int64_t at = 0;
    for (int l = 0; l < L; l++) {
        const std::vector<Sample> &list = lists[(size_t)l];
        count[(size_t)l] = (uint16_t)list.size();
        firstrec[(size_t)l] = list.empty() ? 0 : (uint16_t)at;
        const V3 mn = T.mins(l), mx = T.maxs(l);
        for (const Sample &s : list) {
            uint8_t *r = lighting_out + 28 * at;
            for (int j = 0; j < 6; j++) encode_rgbe(s.cube[j], r + 4 * j);
            r[24] = fixed8(s.pos.x, mn.x, mx.x);
            r[25] = fixed8(s.pos.y, mn.y, mx.y);
            r[26] = fixed8(s.pos.z, mn.z, mx.z);
            r[27] = 0;
            at++;
        }
    }
    // Empty leaves point at their nearest neighbour with samples.
    int bad = 0;
    std::vector<int> near;
    for (int l = 0; l < L; l++) {
        if (count[(size_t)l] != 0) continue;
        if ((t->leaves[9 * l] & kContentsSolid) == 0) bad++;
        const V3 mn = T.mins(l), mx = T.maxs(l);
        const V3 size = sub(mx, mn);
        if (!leaves_in_box(T, sub(mn, size), {mx.x + size.x, mx.y + size.y, mx.z + size.z}, near))
            return vrad_fail(nullptr, VRAD_ERR_ARG, "the leaf box walk went deeper than 256 pending splits");
        float best = 3.402823466e38f;
        int best_leaf = l;
        for (int other : near) {
            if (other < 0 || other >= L || count[(size_t)other] == 0) continue;
            const float d = aabb_distance(mn, mx, T.mins(other), T.maxs(other));
            if (d < best) {
                best = d;
                best_leaf = other;
            }
        }
        firstrec[(size_t)l] = (uint16_t)best_leaf;
    }
    for (int l = 0; l < L; l++) {
        std::memcpy(index_out + 4 * l, &count[(size_t)l], 2);
        std::memcpy(index_out + 4 * l + 2, &firstrec[(size_t)l], 2);
    }
    if (bad_leaves) *bad_leaves = bad;
    return VRAD_OK;
}
