// final_oracle.cpp -- CPU oracle for the lighting stage's final pass.
//
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).  A restatement, in the
// reference's own structure (scatter each sample into the radial arrays,
// then read each luxel back), of:
//   FaceNeighbours.Build        MapTools/Rad/Light/FaceNeighbours.cs:80-230
//   LightmapOffsets.Compute     MapTools/Rad/Light/LightmapOffsets.cs:54-126
//   FinalLightFace.Run / BuildLuxelRadial / Median
//                               MapTools/Rad/Final/FinalLightFace.cs:93-360
//   LuxelRadial.Reset / AddDirect / Sample
//                               MapTools/Rad/Final/LuxelRadial.cs:60-331
//   StockLightColor.Encode      MapTools/Rad/Ambient/StockLightColor.cs:136-185
// Style 0, bounce 0, minlight 0, no macro textures.  -ffp-contract=off.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "oracle_internal.h"
#include "vrad_oracle.h"

namespace {

struct P3 {
    float x, y, z;
};
float dot3(P3 a, P3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// FaceLightInfo's frame (same formulas as direct_oracle.cpp's face_info).
struct Frame {
    P3 ws, wt, ls, lt, o;
    int mins, mint, w, h;
};

Frame frame(const orc_face &f) {
    Frame fr;
    P3 n = {f.normal[0], f.normal[1], f.normal[2]};
    fr.ws = {f.vecs[0][0], f.vecs[0][1], f.vecs[0][2]};
    fr.wt = {f.vecs[1][0], f.vecs[1][1], f.vecs[1][2]};
    P3 s = fr.ws, t = fr.wt;
    P3 c = {t.y * s.z - t.z * s.y, t.z * s.x - t.x * s.z, t.x * s.y - t.y * s.x};
    float det = -dot3(n, c);
    fr.ls = fr.lt = {0, 0, 0};
    P3 o = {0, 0, 0};
    if (!(std::fabs((double)det) < 1.0e-20)) {
        fr.ls = {(n.z * t.y - n.y * t.z) / det, (n.x * t.z - n.z * t.x) / det, (n.y * t.x - n.x * t.y) / det};
        fr.lt = {(n.y * s.z - n.z * s.y) / det, (n.z * s.x - n.x * s.z) / det, (n.x * s.y - n.y * s.x) / det};
        o = {-(f.dist * c.x) / det, -(f.dist * c.y) / det, -(f.dist * c.z) / det};
        float os = -f.vecs[0][3], ot = -f.vecs[1][3];
        o = {o.x + fr.ls.x * os, o.y + fr.ls.y * os, o.z + fr.ls.z * os};
        o = {o.x + fr.lt.x * ot, o.y + fr.lt.y * ot, o.z + fr.lt.z * ot};
    }
    fr.o = {o.x + 0.0f, o.y + 0.0f, o.z + 0.0f};
    fr.mins = f.mins[0];
    fr.mint = f.mins[1];
    fr.w = f.size[0] + 1;
    fr.h = f.size[1] + 1;
    return fr;
}

P3 l2w(const Frame &fr, float s, float t) {
    s += (float)fr.mins;
    t += (float)fr.mint;
    P3 p = {fr.o.x + fr.ls.x * s, fr.o.y + fr.ls.y * s, fr.o.z + fr.ls.z * s};
    return {p.x + fr.lt.x * t, p.y + fr.lt.y * t, p.z + fr.lt.z * t};
}

void w2l(const Frame &fr, P3 p, float &s, float &t) {
    P3 q = {p.x - fr.o.x, p.y - fr.o.y, p.z - fr.o.z};
    s = dot3(q, fr.ws) - (float)fr.mins;
    t = dot3(q, fr.wt) - (float)fr.mint;
}

uint32_t encode(float x, float y, float z) {
    float m = x > y ? (x > z ? x : z) : (y > z ? y : z);
    int e = 0;
    if (m != 0.0f) {
        uint32_t b;
        std::memcpy(&b, &m, 4);
        e = (int)((b & 0x7F800000u) >> 23) - (7 + 127);
    }
    uint32_t sb = (uint32_t)(127 - e) << 23;
    float sc;
    std::memcpy(&sc, &sb, 4);
    uint8_t r = (uint8_t)(int)(x * sc), g = (uint8_t)(int)(y * sc), bb = (uint8_t)(int)(z * sc);
    return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)bb << 16) | ((uint32_t)(uint8_t)(int8_t)e << 24);
}

struct Radial {
    Frame fr;
    std::vector<float> weight;
    std::vector<float> light;  // 4 per cell: lighting xyz, sun

    void reset(const Frame &f) {
        fr = f;
        weight.assign((size_t)f.w * f.h, 0.0f);
        light.assign((size_t)f.w * f.h * 4, 0.0f);
    }

    void add_direct(P3 point, float minS, float minT, float maxS, float maxT, const float *lv) {
        float cs, ct;
        w2l(fr, point, cs, ct);
        int sMin = (int)minS, tMin = (int)minT;
        int sMax = (int)(maxS + 0.9999f) + 1, tMax = (int)(maxT + 0.9999f) + 1;
        sMin = std::max(sMin, 0);
        tMin = std::max(tMin, 0);
        sMax = std::min(sMax, fr.w);
        tMax = std::min(tMax, fr.h);
        for (int s = sMin; s < sMax; s++) {
            for (int t = tMin; t < tMax; t++) {
                double a = (double)(minS - (float)s), b = (double)(minT - (float)t);
                double c = (double)(maxS - (float)s), d = (double)(maxT - (float)t);
                float s0 = (float)(a > -1.0 ? a : -1.0);
                float t0 = (float)(b > -1.0 ? b : -1.0);
                float s1 = (float)(c < 1.0 ? c : 1.0);
                float t1 = (float)(d < 1.0 ? d : 1.0);
                float area = (s1 - s0) * (t1 - t0);
                if ((double)area > 0.001) {
                    float ds = std::fabs(cs - (float)s), dt = std::fabs(ct - (float)t);
                    float r = ds > dt ? ds : dt;
                    r = (double)r < 0.1 ? (float)((double)area / 0.1) : area / r;
                    size_t i = (size_t)(s + t * fr.w);
                    light[4 * i + 0] = light[4 * i + 0] + r * lv[0];
                    light[4 * i + 1] = light[4 * i + 1] + r * lv[1];
                    light[4 * i + 2] = light[4 * i + 2] + r * lv[2];
                    light[4 * i + 3] += r * lv[3];
                    weight[i] += r;
                }
            }
        }
    }

    // LuxelRadial.AddBounced (LuxelRadial.cs:238-307), unbumped.
    void add_bounced(P3 point, float minS, float minT, float maxS, float maxT, const float *lv) {
        float cs, ct;
        w2l(fr, point, cs, ct);
        float distS = maxS - minS, distT = maxT - minT;
        distS = (float)(1.0 > (double)distS ? 1.0 : (double)distS);
        distT = (float)(1.0 > (double)distT ? 1.0 : (double)distT);
        int sMin = (int)((double)cs - (double)distS * 1.42);
        int tMin = (int)((double)ct - (double)distT * 1.42);
        int sMax = (int)((double)cs + (double)distS * 1.42 + 1.0f);
        int tMax = (int)((double)ct + (double)distT * 1.42 + 1.0f);
        sMin = std::max(sMin, 0);
        tMin = std::max(tMin, 0);
        sMax = std::min(sMax, fr.w);
        tMax = std::min(tMax, fr.h);
        for (int s = sMin; s < sMax; s++) {
            for (int t = tMin; t < tMax; t++) {
                float ds = (cs - (float)s) / distS;
                float dt = (ct - (float)t) / distT;
                float r = 2.0f - (ds * ds + dt * dt);
                size_t i = (size_t)(s + t * fr.w);
                if (r > 0) {
                    light[4 * i + 0] = light[4 * i + 0] + r * lv[0];
                    light[4 * i + 1] = light[4 * i + 1] + r * lv[1];
                    light[4 * i + 2] = light[4 * i + 2] + r * lv[2];
                    weight[i] += r;
                }
            }
        }
    }

    bool sample(P3 point, float out[3]) const {
        float cs, ct;
        w2l(fr, point, cs, ct);
        int u = (int)(cs + 0.5f), v = (int)(ct + 0.5f);
        if (u < 0 || u >= fr.w || v < 0 || v >= fr.h) {
            out[0] = 2550.0f;
            out[1] = out[2] = 0.0f;
            return false;
        }
        size_t i = (size_t)(u + v * fr.w);
        float wgt = weight[i];
        if (wgt > 0.00001f) {
            float sc = (float)(1.0 / (double)wgt);
            out[0] = light[4 * i] * sc;
            out[1] = light[4 * i + 1] * sc;
            out[2] = light[4 * i + 2] * sc;
            return true;
        }
        out[0] = out[1] = out[2] = 0.0f;
        return false;
    }
};

}  // namespace

extern "C" int orc_neighbours(const orc_face *faces, int32_t nfaces, const float *verts, float threshold,
                              int32_t *offsets, int32_t *list, int64_t capacity, int64_t *count) {
    std::map<std::tuple<float, float, float>, int> ids;  // position -> vertex number (+0 == -0)
    std::vector<std::vector<int>> fv((size_t)nfaces);
    for (int i = 0; i < nfaces; i++)
        for (int k = 0; k < faces[i].num_vertices; k++) {
            const float *p = verts + 3 * (faces[i].first_vertex + k);
            auto key = std::make_tuple(p[0] + 0.0f, p[1] + 0.0f, p[2] + 0.0f);
            auto it = ids.find(key);
            int id = it == ids.end() ? (int)ids.size() : it->second;
            if (it == ids.end()) ids.emplace(key, id);
            fv[(size_t)i].push_back(id);
        }
    // vertexFace, filled in face order with a linear dedup.
    std::vector<std::vector<int>> vface(ids.size());
    for (int i = 0; i < nfaces; i++)
        for (int n : fv[(size_t)i]) {
            bool seen = false;
            for (int x : vface[(size_t)n]) seen |= x == i;
            if (!seen) vface[(size_t)n].push_back(i);
        }
    int64_t k = 0;
    for (int i = 0; i < nfaces; i++) {
        offsets[i] = (int32_t)k;
        P3 ni = {faces[i].normal[0], faces[i].normal[1], faces[i].normal[2]};
        std::vector<int> scratch;
        for (int n : fv[(size_t)i])
            for (int other : vface[(size_t)n]) {
                if (other == i) continue;
                P3 no = {faces[other].normal[0], faces[other].normal[1], faces[other].normal[2]};
                double cosn = dot3(no, ni);
                if (cosn < (double)threshold) continue;
                if (std::find(scratch.begin(), scratch.end(), other) == scratch.end()) scratch.push_back(other);
            }
        for (int o : scratch) {
            if (list) {
                if (k >= capacity) return -1;
                list[k] = o;
            }
            k++;
        }
    }
    offsets[nfaces] = (int32_t)k;
    *count = k;
    return 0;
}

int orc_final_impl(const orc_face *faces, int32_t nfaces, const float *verts, const orc_sample *samples,
                   const int64_t *face_first, const float *sample_light, uint8_t *lighting, int64_t capacity,
                   int32_t *lightofs, int64_t *total, const OrcBounced *bounced, const float *slots_light,
                   const uint8_t *face_styles) {
    // Each face's styles (FaceLight.Styles; style 0 alone without a table)
    // and a sample's light in one slot (slot 0 in sample_light, slots 1..3
    // in slots_light).
    const int64_t nsamples = face_first[nfaces];
    static const uint8_t kStyle0[4] = {0, 255, 255, 255};
    auto styles_of = [&](int f) { return face_styles ? face_styles + 4 * (int64_t)f : kStyle0; };
    auto light_of = [&](int k, int64_t i) {
        return k == 0 ? sample_light + 4 * i : slots_light + 4 * ((k - 1) * nsamples + i);
    };
    auto nstyles = [&](int f) {
        int n = 0;
        while (n < 4 && styles_of(f)[n] != 255) n++;
        return n;
    };
    // LightmapOffsets.Compute (LightmapOffsets.cs:84-123): per lit face its
    // styles' four-byte averages, then each style's luxels.
    int64_t size = 0;
    std::vector<int32_t> ofs((size_t)nfaces);
    for (int f = 0; f < nfaces; f++) {
        const int ls = nstyles(f);
        size += 4 * ls;
        ofs[(size_t)f] = (int32_t)size;
        size += (int64_t)(faces[f].size[0] + 1) * (faces[f].size[1] + 1) * 4 * ls;
    }
    *total = size;
    if (lightofs) std::memcpy(lightofs, ofs.data(), sizeof(int32_t) * (size_t)nfaces);
    if (!lighting) return 0;
    if (capacity < size) return -1;
    std::memset(lighting, 0, (size_t)size);
    std::vector<int32_t> noff((size_t)nfaces + 1);
    int64_t nn = 0;
    orc_neighbours(faces, nfaces, verts, 0.7071067f, noff.data(), nullptr, 0, &nn);
    std::vector<int32_t> nlist((size_t)(nn ? nn : 1));
    orc_neighbours(faces, nfaces, verts, 0.7071067f, noff.data(), nlist.data(), nn, &nn);
    std::vector<Frame> frames((size_t)nfaces);
    for (int f = 0; f < nfaces; f++) frames[(size_t)f] = frame(faces[f]);
    Radial rad, prad;
    std::vector<float> red, green, blue;
    for (int f = 0; f < nfaces; f++)
    for (int slot = 0; slot < nstyles(f); slot++) {
        const Frame &fr = frames[(size_t)f];
        rad.reset(fr);
        // BuildLuxelRadial: own samples of this slot, then each neighbour's
        // samples of the same style NUMBER, in order; a neighbour without
        // that style adds nothing (FinalLightFace.cs:339-380).
        for (int64_t k = face_first[f]; k < face_first[f + 1]; k++) {
            const orc_sample &sm = samples[k];
            rad.add_direct({sm.position[0], sm.position[1], sm.position[2]}, sm.mins[0], sm.mins[1], sm.maxs[0],
                           sm.maxs[1], light_of(slot, k));
        }
        const uint8_t wanted = styles_of(f)[slot];
        for (int q = noff[(size_t)f]; q < noff[(size_t)f + 1]; q++) {
            const int g = nlist[(size_t)q];
            int ns = 0;
            while (ns < 4 && styles_of(g)[ns] != wanted) ns++;
            if (ns >= 4) continue;
            const Frame &l = frames[(size_t)g];
            for (int64_t k = face_first[g]; k < face_first[g + 1]; k++) {
                const orc_sample &sm = samples[k];
                float mins, mint, maxs, maxt;
                w2l(fr, l2w(l, sm.mins[0], sm.mins[1]), mins, mint);
                w2l(fr, l2w(l, sm.maxs[0], sm.maxs[1]), maxs, maxt);
                rad.add_direct({sm.position[0], sm.position[1], sm.position[2]}, mins, mint, maxs, maxt,
                               light_of(ns, k));
            }
        }
        // BuildPatchRadial (style 0 only): the leaf patches of the face,
        // then of each neighbour (AddFacePatches), splatted with their
        // bounced light.
        const bool bounce_here = bounced && slot == 0;
        if (bounce_here) {
            prad.reset(fr);
            std::vector<int> order = {f};
            for (int q = noff[(size_t)f]; q < noff[(size_t)f + 1]; q++) order.push_back(nlist[(size_t)q]);
            for (int g : order)
                for (const OrcBouncedPatch &bp : bounced->face_leaves[(size_t)g]) {
                    // PatchLightmapCoordRange in this face's luxel space.
                    float minS = 1e30f, minT = 1e30f, maxS = -1e30f, maxT = -1e30f;
                    for (size_t k = 0; k + 2 < bp.winding.size(); k += 3) {
                        float ps, pt;
                        w2l(fr, {bp.winding[k], bp.winding[k + 1], bp.winding[k + 2]}, ps, pt);
                        minS = minS < ps ? minS : ps;
                        maxS = maxS > ps ? maxS : ps;
                        minT = minT < pt ? minT : pt;
                        maxT = maxT > pt ? maxT : pt;
                    }
                    prad.add_bounced({bp.origin[0], bp.origin[1], bp.origin[2]}, minS, minT, maxS, maxT, bp.light);
                }
        }
        // Each luxel: Sample at its own position, minlight 0, encode.
        red.clear();
        green.clear();
        blue.clear();
        const bool no_samples = face_first[f + 1] == face_first[f];
        const int n = fr.w * fr.h;
        for (int j = 0; j < n; j++) {
            const int s = j % fr.w, t = j / fr.w;
            float lb[3];
            bool ok = rad.sample(l2w(fr, (float)s, (float)t), lb);
            if (bounce_here) {
                float v[3];
                (void)prad.sample(l2w(fr, (float)s, (float)t), v);
                for (int c = 0; c < 3; c++) lb[c] = lb[c] + v[c];
            }
            if (no_samples) {
                lb[0] = 255.0f;
                lb[1] = lb[2] = 0.0f;
                ok = false;
            }
            for (int c = 0; c < 3; c++) lb[c] = lb[c] > 0.0f ? lb[c] : 0.0f;
            if (ok) {
                red.push_back(lb[0]);
                green.push_back(lb[1]);
                blue.push_back(lb[2]);
            }
            uint32_t w = encode(lb[0], lb[1], lb[2]);
            std::memcpy(lighting + ofs[(size_t)f] + 4 * ((int64_t)slot * n + j), &w, 4);
        }
        float med[3] = {0.0f, 0.0f, 0.0f};
        if (!red.empty()) {
            std::sort(red.begin(), red.end());
            std::sort(green.begin(), green.end());
            std::sort(blue.begin(), blue.end());
            med[0] = red[red.size() >> 1];
            med[1] = green[green.size() >> 1];
            med[2] = blue[blue.size() >> 1];
        }
        // Before lightofs, in reverse style order.
        uint32_t w = encode(med[0], med[1], med[2]);
        std::memcpy(lighting + ofs[(size_t)f] - 4 * (slot + 1), &w, 4);
    }
    return 0;
}

// The final pass of a map with light styles: slots_light holds slots 1..3
// (nsamples x 4 floats each), face_styles 4 bytes per face.
extern "C" int orc_final_styles(const orc_face *faces, int32_t nfaces, const float *verts, const orc_sample *samples,
                                const int64_t *face_first, const float *sample_light, const float *slots_light,
                                const uint8_t *face_styles, uint8_t *lighting, int64_t capacity, int32_t *lightofs,
                                int64_t *total) {
    return orc_final_impl(faces, nfaces, verts, samples, face_first, sample_light, lighting, capacity, lightofs,
                          total, nullptr, slots_light, face_styles);
}

extern "C" int orc_final(const orc_face *faces, int32_t nfaces, const float *verts, const orc_sample *samples,
                         const int64_t *face_first, const float *sample_light, uint8_t *lighting,
                         int64_t capacity, int32_t *lightofs, int64_t *total) {
    return orc_final_impl(faces, nfaces, verts, samples, face_first, sample_light, lighting, capacity, lightofs,
                          total, nullptr);
}
