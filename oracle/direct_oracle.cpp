// direct_oracle.cpp -- CPU oracle for the lighting stage's direct gather.
//
// TEST INFRASTRUCTURE ONLY (see vrad_oracle.h).  A restatement, in the
// reference's own structure, of:
//   FaceLightInfo.Build             MapTools/Rad/Light/FaceLightInfo.cs:79-160
//   FaceSampleBuilder.BuildFacesamples  FaceSampleBuilder.cs:121-206, 293-330
//   WindingArena.ClipEpsilon / AreaAndBalancePoint / Bounds / RemoveColinearPoints
//   FaceLightJob.EmitGroup / ResolveGroup (four-sample groups, padding by
//                                          repeating the last sample)
//   DirectLightGatherer.GatherPointFour / GatherStandardLane / EmitSkyLight /
//                       ResolveSkyLight / AmbientSky / Resolve
// Rays are traced with the restated KD walk (oracle_internal.h), one
// segment at a time.  Built with -ffp-contract=off.

#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_internal.h"
#include "vrad_oracle.h"

namespace {

struct F3 {
    float x, y, z;
};
F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float Dot(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
F3 Cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float Len(F3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }
F3 Normalise(F3 a) {
    float l = Len(a);
    if (l == 0.0f) return {0, 0, 0};
    return {a.x / l, a.y / l, a.z / l};
}
float MaxPs(float a, float b) { return a > b ? a : b; }
float MinPs(float a, float b) { return a < b ? a : b; }

// ---- samples ---------------------------------------------------------------

struct Info {
    F3 n;
    float dist;
    F3 ws, wt, ls, lt, origin;
    int mins, mint, width, height;
};

Info face_info(const orc_face &f) {
    Info in;
    in.n = {f.normal[0], f.normal[1], f.normal[2]};
    in.dist = f.dist;
    in.ws = {f.vecs[0][0], f.vecs[0][1], f.vecs[0][2]};
    in.wt = {f.vecs[1][0], f.vecs[1][1], f.vecs[1][2]};
    F3 S = in.ws, Tt = in.wt, N = in.n;
    F3 cr = {Tt.y * S.z - Tt.z * S.y, Tt.z * S.x - Tt.x * S.z, Tt.x * S.y - Tt.y * S.x};
    float det = -Dot(N, cr);
    in.ls = in.lt = {0, 0, 0};
    F3 o = {0, 0, 0};
    if (!(std::fabs((double)det) < 1.0e-20)) {
        in.ls = {(N.z * Tt.y - N.y * Tt.z) / det, (N.x * Tt.z - N.z * Tt.x) / det, (N.y * Tt.x - N.x * Tt.y) / det};
        in.lt = {(N.y * S.z - N.z * S.y) / det, (N.z * S.x - N.x * S.z) / det, (N.x * S.y - N.y * S.x) / det};
        o = {-(f.dist * cr.x) / det, -(f.dist * cr.y) / det, -(f.dist * cr.z) / det};
        o = o + in.ls * -f.vecs[0][3];
        o = o + in.lt * -f.vecs[1][3];
    }
    in.origin = o + F3{0, 0, 0};
    in.mins = f.mins[0];
    in.mint = f.mins[1];
    in.width = f.size[0] + 1;
    in.height = f.size[1] + 1;
    return in;
}

typedef std::vector<F3> W;

// ClipEpsilon against the axis plane p[axis] = d; the face's luxel-space
// windings are planar in z = 0.
void clip(const W &w, int axis, float d, float eps, W &front, W &back) {
    front.clear();
    back.clear();
    int n = (int)w.size();
    F3 nrm = {axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, 0.0f};
    std::vector<float> dd(n + 1);
    std::vector<int> side(n + 1);
    int cf = 0, cb = 0;
    for (int i = 0; i < n; i++) {
        float v = Dot(w[i], nrm);
        v -= d;
        dd[i] = v;
        side[i] = v > eps ? 1 : (v < -eps ? -1 : 0);
        if (side[i] == 1) cf++;
        if (side[i] == -1) cb++;
    }
    dd[n] = dd[0];
    side[n] = side[0];
    if (cf == 0) {
        back = w;
        return;
    }
    if (cb == 0) {
        front = w;
        return;
    }
    for (int i = 0; i < n; i++) {
        F3 p1 = w[i];
        if (side[i] == 0) {
            front.push_back(p1);
            back.push_back(p1);
            continue;
        }
        (side[i] == 1 ? front : back).push_back(p1);
        if (side[i + 1] == 0 || side[i + 1] == side[i]) continue;
        F3 p2 = w[(i + 1) % n];
        float f = dd[i] / (dd[i] - dd[i + 1]);
        float c[3];
        const float a[3] = {p1.x, p1.y, p1.z}, b[3] = {p2.x, p2.y, p2.z}, nn[3] = {nrm.x, nrm.y, nrm.z};
        for (int k = 0; k < 3; k++) c[k] = nn[k] == 1.0f ? d : (nn[k] == -1.0f ? -d : a[k] + f * (b[k] - a[k]));
        front.push_back({c[0], c[1], c[2]});
        back.push_back({c[0], c[1], c[2]});
    }
}

}  // namespace

namespace {

// FaceSampleBuilder.BuildFacesamples for one face, appending its samples;
// with wind set, each partial sample's cell winding in world space
// (MakeSample keeps it when area < worldAreaPerLuxel - EQUAL_EPSILON, in
// double), an empty one for a whole cell.
void face_samples(const orc_face &f, int32_t fi, const float *verts, std::vector<orc_sample> &out,
                  std::vector<W> *wind) {
    const float eps = 0.1f / 16.0f;
    Info in = face_info(f);
    float ss = (f.vecs[0][0] * f.vecs[0][0] + f.vecs[0][1] * f.vecs[0][1]) + f.vecs[0][2] * f.vecs[0][2];
    float tt = (f.vecs[1][0] * f.vecs[1][0] + f.vecs[1][1] * f.vecs[1][1]) + f.vecs[1][2] * f.vecs[1][2];
    float apl = (float)(1.0 / (double)(std::sqrt(ss) * std::sqrt(tt)));
    W w;
    for (int v = 0; v < f.num_vertices; v++) {
        const float *p = verts + 3 * (f.first_vertex + v);
        w.push_back(F3{p[0], p[1], p[2]} + F3{0, 0, 0});
    }
    // RemoveColinearPoints.
    {
        W kept;
        int n = (int)w.size();
        for (int i = 0; i < n; i++) {
            F3 v1 = Normalise(w[(i + 1) % n] - w[i]);
            F3 v2 = Normalise(w[i] - w[(i + n - 1) % n]);
            if ((double)Dot(v1, v2) < 0.999) kept.push_back(w[i]);
        }
        if ((int)kept.size() != n) w = kept;
    }
    for (F3 &p : w) {
        F3 q = p - in.origin;
        p = {Dot(q, in.ws) - (float)in.mins, Dot(q, in.wt) - (float)in.mint, 0.0f};
    }
    auto l2w = [&](float s, float t) {
        float su = s + (float)in.mins, tv = t + (float)in.mint;
        F3 pos = in.origin + in.ls * su;
        return pos + in.lt * tv;
    };
    W rest = w, rowf, rowb, cf, cb;
    for (int t = 0; t < in.height && !rest.empty(); t++) {
        clip(rest, 1, (float)t + 1.0f, eps, rowf, rowb);
        W row = rowb;
        for (int s = 0; s < in.width && !row.empty(); s++) {
            clip(row, 0, (float)s + 1.0f, eps, cf, cb);
            if (!cb.empty()) {
                // AreaAndBalancePoint.
                F3 c = {0, 0, 0};
                float total = 0.0f;
                for (size_t i = 2; i < cb.size(); i++) {
                    float a = Len(Cross(cb[i - 1] - cb[0], cb[i] - cb[0]));
                    total += a;
                    float third = (float)((double)a / 3.0);
                    c = c + cb[i - 1] * third;
                    c = c + cb[i] * third;
                    c = c + cb[0] * third;
                }
                if (total != 0.0f) c = c * (float)(1.0 / (double)total);
                float area = total * 0.5f * apl;
                orc_sample o;
                o.area = area;
                o.coord[0] = c.x;
                o.coord[1] = c.y;
                float mn[2] = {99999.0f, 99999.0f}, mx[2] = {-99999.0f, -99999.0f};
                for (const F3 &p : cb) {
                    if (p.x < mn[0]) mn[0] = p.x;
                    if (p.x > mx[0]) mx[0] = p.x;
                    if (p.y < mn[1]) mn[1] = p.y;
                    if (p.y > mx[1]) mx[1] = p.y;
                }
                o.mins[0] = mn[0];
                o.mins[1] = mn[1];
                o.maxs[0] = mx[0];
                o.maxs[1] = mx[1];
                F3 pos = l2w(c.x, c.y);
                o.position[0] = pos.x;
                o.position[1] = pos.y;
                o.position[2] = pos.z;
                o.s = s;
                o.t = t;
                o.face = fi;
                o.cluster = f.cluster;
                out.push_back(o);
                if (wind) {
                    W cell;
                    if ((double)area < (double)apl - 0.001)
                        for (const F3 &p : cb) cell.push_back(l2w(p.x, p.y));
                    wind->push_back(cell);
                }
            }
            row = cf;
        }
        rest = rowf;
    }
}

}  // namespace

extern "C" int orc_build_samples(const orc_face *faces, int32_t nfaces, const float *verts,
                                 orc_sample *out, int64_t capacity, int64_t *count, int64_t *first) {
    int64_t k = 0;
    std::vector<orc_sample> tmp;
    for (int32_t fi = 0; fi < nfaces; fi++) {
        if (first) first[fi] = k;
        tmp.clear();
        face_samples(faces[fi], fi, verts, tmp, nullptr);
        for (const orc_sample &o : tmp) {
            if (out) {
                if (k >= capacity) return -1;
                out[k] = o;
            }
            k++;
        }
    }
    if (first) first[nfaces] = k;
    *count = k;
    return 0;
}

// ---- the gather --------------------------------------------------------------

namespace {

constexpr float kMaxTrace = (float)(1.732050807569 * (2 * 16384));
constexpr int kLanes = 4;

struct Out4 {
    float dot[4], falloff[4], sun[4];
};

struct Ctx {
    OrcKd kd;
    const orc_light *lights;
    const float *dirs;
    int ndirs;
    const float *jitter;
    float extent;
    int nsun;
};

thread_local int64_t t_rays = 0;

bool visible(const Ctx &c, F3 a, F3 b, bool sky) {
    // LightRayLog.MakeRay: the whole segment, reach 1.
    t_rays++;
    F3 d = b - a;
    orc_ray r{a.x, a.y, a.z, d.x, d.y, d.z, 1.0f};
    return !orc_kd_segment_blocked(c.kd, r, sky);
}

// DetMathF.Pow: the correctly rounded float power, here the x87 extended
// power rounded once.
float PowF(float x, float y) { return (float)powl((long double)x, (long double)y); }

// DetMath.PowToSingle: x^y rounded to double, then to float.
float PowToSingle(double x, double y) { return (float)(double)powl((long double)x, (long double)y); }

float inv_quadratic(const orc_light &L, float d) {
    float f = d * d;
    f *= L.quadratic;
    f += L.linear * d;
    f += L.constant;
    return 1.0f / f;
}

float quintic(float dist, const orc_light &L) {
    float t = (dist - L.start_fade) / (L.end_fade - L.start_fade);
    t = MinPs(t, 1.0f);
    t = MaxPs(t, 0.0f);
    t = 1.0f - t;
    float mult = (6.0f * t) - 15.0f;
    mult = (mult * t) + 10.0f;
    mult = (t * t) * mult;
    return t * mult;
}

// One light over one group: the reference's emit + trace + resolve.
void gather(const Ctx &c, const orc_light &L, const F3 pts[4], const F3 nrm[4], int count, Out4 &o) {
    std::memset(&o, 0, sizeof o);
    const bool hard = L.end_fade > L.start_fade;
    const F3 src = {L.origin[0], L.origin[1], L.origin[2]};
    const F3 ln = {L.normal[0], L.normal[1], L.normal[2]};
    if (L.type == 1) {
        // GatherPointFour, then the visibility multiply of the resolve.
        for (int l = 0; l < kLanes; l++) {
            float dx = src.x - pts[l].x, dy = src.y - pts[l].y, dz = src.z - pts[l].z;
            float d2 = ((dx * dx) + (dy * dy)) + (dz * dz);
            float dist = std::sqrt(d2);
            float r = 1.0f / dist;
            dx *= r;
            dy *= r;
            dz *= r;
            float dot = ((dx * nrm[l].x) + (dy * nrm[l].y)) + (dz * nrm[l].z);
            dot = MaxPs(0.0f, dot);
            bool live = !hard || dist <= L.end_fade;
            dist = MaxPs(dist, 1.0f);
            float d = MinPs(dist, L.cap_dist);
            float fall = inv_quadratic(L, d);
            if (hard) fall = quintic(dist, L) * fall;
            o.dot[l] = live ? dot : 0.0f;
            o.falloff[l] = live ? fall : 0.0f;
            if (l < count && o.dot[l] != 0.0f && o.falloff[l] != 0.0f)
                o.dot[l] = (visible(c, pts[l], src, false) ? 1.0f : 0.0f) * o.dot[l];
        }
    } else if (L.type == 0) {
        // GatherSurfaceFour (DirectLightGatherer.cs:1452-1545): the
        // emitter's cosine over the squared distance; the segment ends
        // DistEpsilon off the emitting patch.
        const F3 end = src + ln * 0.03125f;
        for (int l = 0; l < kLanes; l++) {
            float dx = src.x - pts[l].x, dy = src.y - pts[l].y, dz = src.z - pts[l].z;
            float d2 = ((dx * dx) + (dy * dy)) + (dz * dz);
            float dist = std::sqrt(d2);
            float r = 1.0f / dist;
            dx *= r;
            dy *= r;
            dz *= r;
            float dot = ((dx * nrm[l].x) + (dy * nrm[l].y)) + (dz * nrm[l].z);
            dot = MaxPs(0.0f, dot);
            bool live = !hard || dist <= L.end_fade;
            dist = MaxPs(dist, 1.0f);
            float dot2 = -(((dx * ln.x) + (dy * ln.y)) + (dz * ln.z));
            dot2 = MaxPs(0.0f, dot2);
            live = live && !(dot == 0.0f);
            float fall = dot2 / d2;
            if (hard) fall = quintic(dist, L) * fall;
            o.dot[l] = live ? dot : 0.0f;
            o.falloff[l] = live ? fall : 0.0f;
            if (l < count && o.dot[l] != 0.0f && o.falloff[l] != 0.0f)
                o.dot[l] = (visible(c, pts[l], end, false) ? 1.0f : 0.0f) * o.dot[l];
        }
    } else if (L.type == 2) {
        // GatherStandardLane (Spotlight) for the real lanes; the resolve
        // copies the last real lane into the padding.
        for (int l = 0; l < count; l++) {
            F3 delta = src - pts[l];
            float d2 = (delta.x * delta.x + delta.y * delta.y) + delta.z * delta.z;
            float r = 1.0f / std::sqrt(d2);
            delta = delta * r;
            float dist = std::sqrt(d2);
            float dot = Dot(delta, nrm[l]);
            dot = MaxPs(0.0f, dot);
            if (hard && !(dist <= L.end_fade)) continue;
            dist = MaxPs(dist, 1.0f);
            float fed = MinPs(dist, L.cap_dist);
            float dot2 = -Dot(delta, ln);
            if (!(dot2 > L.stop_dot2)) continue;
            float fall = inv_quadratic(L, fed) * dot2;
            bool fringe = dot2 <= L.stop_dot;
            float mult = (dot2 - L.stop_dot2) / (L.stop_dot - L.stop_dot2);
            mult = MinPs(mult, 1.0f);
            mult = MaxPs(mult, 0.0f);
            if (L.exponent != 0.0f && L.exponent != 1.0f) mult = PowF(mult, L.exponent);
            mult = fringe ? mult : 1.0f;
            fall = mult * fall;
            if (hard) fall = quintic(dist, L) * fall;
            bool trace = dot != 0.0f && fall != 0.0f;
            o.dot[l] = dot;
            o.falloff[l] = fall;
            if (trace) o.dot[l] = (visible(c, pts[l], src, false) ? 1.0f : 0.0f) * o.dot[l];
        }
        for (int l = count; l < kLanes; l++) {
            o.dot[l] = o.dot[count - 1];
            o.falloff[l] = o.falloff[count - 1];
        }
    } else if (L.type == 3) {
        // EmitSkyLight / ResolveSkyLight.
        float dot[4];
        bool all_zero = true;
        for (int l = 0; l < kLanes; l++) {
            dot[l] = MaxPs(-Dot(nrm[l], ln), 0.0f);
            all_zero &= dot[l] == 0.0f;
        }
        if (!all_zero) {
            float total[4] = {0, 0, 0, 0};
            float js = (float)(1.732050807569 * (2 * 16384) * (double)c.extent);
            for (int d = 0; d < c.nsun; d++) {
                F3 delta = ln * -kMaxTrace;
                if (d != 0) {
                    const float *j = c.jitter + 3 * (d - 1);
                    delta = delta + F3{j[0], j[1], j[2]} * js;
                }
                for (int l = 0; l < count; l++) {
                    F3 stop = delta + pts[l];
                    total[l] += visible(c, pts[l], stop, true) ? 1.0f : 0.0f;
                }
            }
            float inv = 1.0f / (float)c.nsun;
            for (int l = 0; l < kLanes; l++) {
                float see = total[l] * inv;
                o.dot[l] = dot[l] * see;
                o.falloff[l] = 1.0f;
                o.sun[l] = see * 10000.0f;
            }
        }
    } else if (L.type == 4) {
        // AmbientSky (flat normals, no skybox recursion, epsilon 0).
        float sumdot[4] = {0, 0, 0, 0}, possible[4] = {0, 0, 0, 0}, amb[4] = {0, 0, 0, 0};
        for (int di = 0; di < c.ndirs; di++) {
            F3 an = {c.dirs[3 * di], c.dirs[3 * di + 1], c.dirs[3 * di + 2]};
            bool valid[4], any = false;
            float dots[4];
            for (int l = 0; l < kLanes; l++) {
                float d = -Dot(nrm[l], an);
                valid[l] = d > 0.001f;
                any |= valid[l];
                dots[l] = valid[l] ? d : 0.0f;
            }
            if (!any) continue;
            for (int l = 0; l < kLanes; l++) {
                sumdot[l] = dots[l] + sumdot[l];
                possible[l] = (valid[l] ? 1.0f : 0.0f) + possible[l];
                float frac = 1.0f;
                if (valid[l] && l < count) {
                    F3 stop = (an * -kMaxTrace) + pts[l];
                    F3 start = pts[l] - (an * -0.0f);
                    frac = visible(c, start, stop, true) ? 1.0f : 0.0f;
                }
                amb[l] = amb[l] + (frac * dots[l]);
            }
        }
        for (int l = 0; l < kLanes; l++) {
            o.falloff[l] = 1.0f;
            float factor = possible[l] / possible[l];
            o.dot[l] = amb[l] / (factor * sumdot[l]);
        }
    }
    // Resolve: clamp the dot.
    for (int l = 0; l < kLanes; l++) o.dot[l] = MaxPs(o.dot[l], 0.0f);
}

}  // namespace

namespace {

// PointsInWinding (FaceLightJob.cs:902-940).
bool PointsInWinding(const F3 pts[4], const W &winding, int &invalidBits) {
    invalidBits = 0;
    const int n = (int)winding.size();
    F3 test[4];
    bool invalid[4] = {false, false, false, false};
    for (int l = 0; l < 4; l++) test[l] = Normalise(Cross(winding[1 % n] - winding[0], pts[l] - winding[0]));
    for (int k = 1; k < n; k++) {
        F3 p0 = winding[k], p1 = winding[(k + 1) % n];
        F3 edge = p1 - p0;
        invalidBits = 0;
        for (int l = 0; l < 4; l++) {
            F3 cr = Normalise(Cross(edge, pts[l] - p0));
            float dot = Dot(cr, test[l]);
            invalid[l] |= dot < 0.0f;
            invalidBits |= invalid[l] ? 1 << l : 0;
        }
        if (invalidBits == 0xF) return false;
    }
    return true;
}

// EmitResample + ResolveResample for one row of four points: the ambient
// light alone or every other light, of one style (FaceLightJob.cs:465-550),
// each added with AddLight (no skip).
void Resample(const Ctx &c, const F3 pts[4], F3 n, int cl, const int32_t *cl_off, const int32_t *cl_list,
              bool ambientOnly, int style, float result[4][4]) {
    std::memset(result, 0, sizeof(float) * 16);
    F3 nrm[4] = {n, n, n, n};
    for (int k = cl_off[cl]; k < cl_off[cl + 1]; k++) {
        const orc_light &L = c.lights[cl_list[k]];
        if (ambientOnly && L.type != 4) continue;
        if (!ambientOnly && L.type == 4) continue;
        if (L.style != style) continue;
        Out4 o;
        gather(c, L, pts, nrm, 4, o);
        for (int l = 0; l < 4; l++) {
            float f = o.falloff[l] * o.dot[l];
            result[l][0] = result[l][0] + (f * L.intensity[0]);
            result[l][1] = result[l][1] + (f * L.intensity[1]);
            result[l][2] = result[l][2] + (f * L.intensity[2]);
            result[l][3] += o.sun[l];
        }
    }
}

// The supersampling passes of one style slot of one face
// (FaceLightJob.AdvanceAfterRound and StyleSupersample), over its samples'
// light in that slot (4 floats each).
int64_t Supersample(const Ctx &c, const orc_face &f, const orc_sample *samples, int64_t nsamp, const std::vector<W> &wind,
                    const int32_t *cl_off, const int32_t *cl_list, int extra_passes, int style, float *light) {
    const Info in = face_info(f);
    const int w = in.width, h = in.height, size = w * h;
    std::vector<float> inten((size_t)size, 0.0f);
    std::vector<char> has((size_t)size, 0), processed((size_t)nsamp, 0);
    std::vector<float> grad((size_t)nsamp, 0.0f);
    auto intensity = [&](int64_t i) {
        const float *v = light + 4 * i;
        float sum = v[0] + v[1] + v[2];
        inten[(size_t)(samples[i].s + samples[i].t * w)] = PowToSingle(sum / 256.0, 1.0 / 2.2);
    };
    for (int64_t i = 0; i < nsamp; i++) has[(size_t)(samples[i].s + samples[i].t * w)] = 1;
    for (int64_t i = 0; i < nsamp; i++) intensity(i);
    const F3 n = {f.normal[0], f.normal[1], f.normal[2]};
    auto w2l = [&](F3 p, float &s, float &t) {
        F3 q = p - in.origin;
        s = Dot(q, in.ws) - (float)in.mins;
        t = Dot(q, in.wt) - (float)in.mint;
    };
    auto l2w = [&](float s, float t) {
        float su = s + (float)in.mins, tv = t + (float)in.mint;
        F3 pos = in.origin + in.ls * su;
        return pos + in.lt * tv;
    };
    int64_t done = 0;
    int pass = 1;
    bool another = true;
    std::vector<int64_t> selected;
    for (;;) {
        if (!another || pass > extra_passes) break;
        // ComputeGradients, then the selection.
        for (int64_t i = 0; i < nsamp; i++) {
            if (processed[(size_t)i]) continue;
            float g = 0.0f;
            const int j = samples[i].s + samples[i].t * w;
            const float cv = inten[(size_t)j];
            auto step = [&](int idx) {
                if (!has[(size_t)idx]) return;
                float d = std::fabs(cv - inten[(size_t)idx]);
                g = g > d ? g : d;
            };
            const int S = samples[i].s, T = samples[i].t;
            if (T > 0) {
                if (S > 0) step(j - 1 - w);
                step(j - w);
                if (S < w - 1) step(j + 1 - w);
            }
            if (T < h - 1) {
                if (S > 0) step(j - 1 + w);
                step(j + w);
                if (S < w - 1) step(j + 1 + w);
            }
            if (S > 0) step(j - 1);
            if (S < w - 1) step(j + 1);
            grad[(size_t)i] = g;
        }
        selected.clear();
        for (int64_t i = 0; i < nsamp; i++) {
            if (processed[(size_t)i]) continue;
            if (grad[(size_t)i] < 0.0625f) continue;
            processed[(size_t)i] = 1;
            selected.push_back(i);
        }
        another = !selected.empty();
        if (!another) break;
        for (int64_t i : selected) {
            const orc_sample &sm = samples[i];
            float os, ot;
            w2l(F3{sm.position[0], sm.position[1], sm.position[2]}, os, ot);
            const W &wd = wind[(size_t)i];
            float amb[4] = {0, 0, 0, 0}, dir[4] = {0, 0, 0, 0};
            int ac = 0, dc = 0;
            for (int pt = 0; pt < 2; pt++) {
                const bool ambientOnly = pt == 0;
                const float width = ambientOnly ? 2.0f : 4.0f;
                const float cscale = 1.0f / width;
                const float csshift = (float)(-((width - 1) * cscale) / 2.0);
                float aRow[4];
                for (int k = 0; k < 4; k++) aRow[k] = csshift + (k * cscale);
                const int rows = ambientOnly ? 1 : 4;
                for (int r = 0; r < rows; r++) {
                    F3 pos[4];
                    for (int l = 0; l < 4; l++) {
                        float cs, ct;
                        if (ambientOnly) {
                            cs = os + (l < 2 ? csshift : csshift + cscale);
                            ct = ot + ((l & 1) == 0 ? csshift : csshift + cscale);
                        } else {
                            cs = os + aRow[r];
                            ct = ot + aRow[l];
                        }
                        pos[l] = l2w(cs, ct);
                    }
                    int bits = 0;
                    if (!wd.empty() && !PointsInWinding(pos, wd, bits)) {
                        if (ambientOnly) break;
                        continue;
                    }
                    F3 pts[4];
                    for (int l = 0; l < 4; l++) pts[l] = pos[l] + n;
                    float res[4][4];
                    Resample(c, pts, n, f.cluster, cl_off, cl_list, ambientOnly, style, res);
                    float *acc = ambientOnly ? amb : dir;
                    int &cnt = ambientOnly ? ac : dc;
                    for (int l = 0; l < 4; l++) {
                        if ((bits >> l) & 1) continue;
                        acc[0] = acc[0] + res[l][0];
                        acc[1] = acc[1] + res[l][1];
                        acc[2] = acc[2] + res[l][2];
                        acc[3] += res[l][3];
                        cnt++;
                    }
                }
            }
            if (ac > 0 && dc > 0) {
                float *v = light + 4 * i;
                float wdir = 1.0f / dc, wamb = 1.0f / ac;
                v[0] = 0.0f + wdir * dir[0];
                v[1] = 0.0f + wdir * dir[1];
                v[2] = 0.0f + wdir * dir[2];
                v[3] = 0.0f + wdir * dir[3];
                v[0] = v[0] + wamb * amb[0];
                v[1] = v[1] + wamb * amb[1];
                v[2] = v[2] + wamb * amb[2];
                v[3] += wamb * amb[3];
                intensity(i);
            }
        }
        done += (int64_t)selected.size();
        pass++;
    }
    return done;
}

// FaceLight.FindOrAllocateStyle (FaceLight.cs:200-223): the slot holding
// `style`, a free slot taken for it, or -1 when all four are taken.
int FindOrAllocateStyle(uint8_t styles[4], int style) {
    for (int k = 0; k < 4; k++) {
        if (styles[k] == style) return k;
        if (styles[k] == 255) {
            styles[k] = (uint8_t)style;
            return k;
        }
    }
    return -1;
}

}  // namespace

// The direct gather with light styles: per face, style 0 in slot 0 from the
// start (FaceLightJob.cs:184-186), every other style given the next free
// slot by the first four-sample group it lights (ResolveGroup,
// FaceLightJob.cs:399-455; a fifth style is warned and dropped), then the
// supersampling passes of each slot with that style's lights alone.
// out: slot 0 (4 floats per sample); out_slots (nullable): slots 1..3, each
// nsamples x 4 floats, zero where the slot is not the face's;
// face_styles (nullable): 4 bytes per face (255: no style); dropped
// (nullable): faces warned of a fifth style.
extern "C" int orc_direct_styles(const orc_kdnode *nodes, const int32_t *indices, const orc_tri *tris,
                                 const float *bounds6, const orc_face *faces, int32_t nfaces, const float *verts,
                                 const orc_sample *samples, const int64_t *face_first, const orc_light *lights,
                                 const int32_t *cl_off, const int32_t *cl_list, const float *dirs, int32_t ndirs,
                                 const float *jitter, int32_t sun_samples, float sun_extent, int32_t extra_passes,
                                 float *out, float *out_slots, uint8_t *face_styles, int64_t *dropped,
                                 int32_t threads, int64_t *rays_out, int64_t *supersampled_out) {
    std::atomic<int64_t> rays(0), supersampled(0), warned(0);
    const int64_t nsamples = face_first[nfaces];
    std::atomic<bool> mismatch(false);
    Ctx c;
    c.kd = OrcKd{nodes, indices, tris, {bounds6[0], bounds6[1], bounds6[2], bounds6[3], bounds6[4], bounds6[5]}};
    c.lights = lights;
    c.dirs = dirs;
    c.ndirs = ndirs;
    c.jitter = jitter;
    c.extent = sun_extent;
    c.nsun = sun_samples;
    auto work = [&](int32_t f0, int32_t f1) {
        t_rays = 0;
        for (int32_t fi = f0; fi < f1; fi++) {
            const int64_t a = face_first[fi], b = face_first[fi + 1];
            const F3 n = {faces[fi].normal[0], faces[fi].normal[1], faces[fi].normal[2]};
            const int cl = faces[fi].cluster;
            uint8_t st[4] = {0, 255, 255, 255};
            bool warn = false;
            // The face's light per slot (slot 0 in out); zero until a slot is taken.
            std::vector<float> mine_slots((size_t)(3 * 4 * (b - a)), 0.0f);
            auto slot_light = [&](int k, int64_t i) {
                return k == 0 ? out + 4 * i : mine_slots.data() + 4 * ((k - 1) * (b - a) + (i - a));
            };
            for (int64_t g = a; g < b; g += 4) {
                int count = (int)((b - g) < 4 ? (b - g) : 4);
                F3 pts[4], nrm[4];
                for (int l = 0; l < 4; l++) {
                    const orc_sample &s = samples[g + (l < count ? l : count - 1)];
                    pts[l] = F3{s.position[0], s.position[1], s.position[2]} + n;
                    nrm[l] = n;
                }
                float acc[4][4][4];
                std::memset(acc, 0, sizeof acc);
                for (int k = cl_off[cl]; k < cl_off[cl + 1]; k++) {
                    const orc_light &L = lights[cl_list[k]];
                    Out4 o;
                    gather(c, L, pts, nrm, count, o);
                    float fx[4];
                    bool skip = true;
                    for (int l = 0; l < 4; l++) {
                        float masked = l < count ? o.dot[l] : 0.0f;
                        fx[l] = masked * o.falloff[l];
                        skip &= fx[l] == 0.0f;
                    }
                    if (skip) continue;
                    const int slot = FindOrAllocateStyle(st, L.style);
                    if (slot < 0) {
                        warn = true;
                        continue;
                    }
                    for (int l = 0; l < count; l++) {
                        acc[slot][l][0] = acc[slot][l][0] + (fx[l] * L.intensity[0]);
                        acc[slot][l][1] = acc[slot][l][1] + (fx[l] * L.intensity[1]);
                        acc[slot][l][2] = acc[slot][l][2] + (fx[l] * L.intensity[2]);
                        acc[slot][l][3] += o.sun[l];
                    }
                }
                for (int k = 0; k < 4; k++)
                    for (int l = 0; l < count; l++) std::memcpy(slot_light(k, g + l), acc[k][l], 16);
            }
            if (warn) warned++;
            if (face_styles) std::memcpy(face_styles + 4 * (int64_t)fi, st, 4);
            auto keep_slots = [&]() {
                if (!out_slots) return;
                for (int k = 1; k < 4; k++)
                    std::memcpy(out_slots + 4 * ((k - 1) * nsamples + a), slot_light(k, a), sizeof(float) * 4 * (b - a));
            };
            if (extra_passes > 0 && b > a) {
                // The face's own samples and their windings (the caller's
                // samples must be the builder's: checked, not assumed).
                std::vector<orc_sample> mine;
                std::vector<W> wind;
                face_samples(faces[fi], fi, verts, mine, &wind);
                bool same = (int64_t)mine.size() == b - a;
                for (int64_t k = 0; same && k < b - a; k++) {
                    orc_sample x = mine[(size_t)k];
                    x.face = samples[a + k].face;
                    same = std::memcmp(&x, &samples[a + k], sizeof x) == 0;
                }
                if (!same) {
                    mismatch = true;
                    keep_slots();
                    continue;
                }
                for (int k = 0; k < 4 && st[k] != 255; k++)
                    supersampled += Supersample(c, faces[fi], samples + a, b - a, wind, cl_off, cl_list, extra_passes,
                                                st[k], slot_light(k, a));
            }
            keep_slots();
        }
        rays += t_rays;
    };
    if (threads <= 1) {
        work(0, nfaces);
    } else {
        std::vector<std::thread> pool;
        int32_t per = (nfaces + threads * 8 - 1) / (threads * 8);
        std::atomic<int32_t> cursor(0);
        for (int t = 0; t < threads; t++)
            pool.emplace_back([&] {
                for (;;) {
                    int32_t f0 = cursor.fetch_add(per);
                    if (f0 >= nfaces) break;
                    work(f0, f0 + per < nfaces ? f0 + per : nfaces);
                }
            });
        for (auto &th : pool) th.join();
    }
    if (rays_out) *rays_out = rays.load();
    if (supersampled_out) *supersampled_out = supersampled.load();
    if (dropped) *dropped = warned.load();
    return mismatch ? -2 : 0;
}

// The gather's slot 0 alone (every light of the maps this was first written
// for is style 0).
extern "C" int orc_direct(const orc_kdnode *nodes, const int32_t *indices, const orc_tri *tris,
                          const float *bounds6, const orc_face *faces, int32_t nfaces, const float *verts,
                          const orc_sample *samples, const int64_t *face_first, const orc_light *lights,
                          const int32_t *cl_off, const int32_t *cl_list, const float *dirs, int32_t ndirs,
                          const float *jitter, int32_t sun_samples, float sun_extent, int32_t extra_passes,
                          float *out, int32_t threads, int64_t *rays_out, int64_t *supersampled_out) {
    return orc_direct_styles(nodes, indices, tris, bounds6, faces, nfaces, verts, samples, face_first, lights,
                             cl_off, cl_list, dirs, ndirs, jitter, sun_samples, sun_extent, extra_passes, out,
                             nullptr, nullptr, nullptr, threads, rays_out, supersampled_out);
}

// DetMathF.Pow as the oracle computes it (the spotlight cone's power).
extern "C" float orc_powf(float x, float y) { return PowF(x, y); }
