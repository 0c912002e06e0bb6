// windings.cu -- the supersampling tables rebuilt on the device: the
// partial cells' windings (FaceSampleBuilder.MakeSample with do_extra,
// FaceSampleBuilder.cs:325-367), each sample's luxel origin and cell, and
// the check that the world's samples are the builder's own.
//
// The host cuts each face's luxel-space winding into its row strips
// (world.cpp:face_row_strips, the builder's row clips).  Here one thread
// per strip clips it into cells at s + 1 (WindingArena.ClipEpsilon) and,
// per non-empty cell, restates AreaAndBalancePoint, the bounds, the
// partial-cell test and LuxelToWorld with explicitly rounded operations in
// the host builder's order, so every rebuilt sample is the builder's bit
// for bit.  A first launch counts each strip's samples and partial-cell
// points; after a scan, the second writes them at their offsets and
// compares each sample with the uploaded one: position and face (the
// world's sample positions), bounds (the final pass's sample boxes), area
// and coord (a table uploaded for the check), s and t (the final pass's
// cell table must name the sample at its cell).

#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <string>

#include "setup_clock.h"
#include "supersample.cuh"
#include "world.h"
#include "sync_wait.h"

namespace vrad {

namespace {

constexpr int kPolyMax = 64;                // a cell of a kStripMax-point strip holds at most kStripMax + 4
constexpr float kOnEpsilon = 0.1f / 16.0f;  // LightConstants.LightmapOnEpsilon
constexpr int kWindBlock = 128;

static_assert(kStripMax + 8 <= kPolyMax, "strip capacity");

struct Pt {
    float x, y;
};

__device__ __forceinline__ int side_of(float d) { return d > kOnEpsilon ? 0 : (d < -kOnEpsilon ? 1 : 2); }

// WindingArena.ClipEpsilon against the plane x = dist (points in luxel
// space, z 0): front d > eps, back d < -eps, points within eps go to both;
// an empty output is the reference's null winding.  d = x - dist is the
// host's dot-with-axis minus dist exactly (dist >= 1, so no signed zero
// reaches a split).  False when an output would exceed kPolyMax.
__device__ bool clip_x(const Pt *in, int n, float dist, Pt *front, int &nf, Pt *back, int &nb) {
    nf = nb = 0;
    if (n == 0) return true;
    int c0 = 0, c1 = 0;
    for (int i = 0; i < n; i++) {
        const int sd = side_of(__fsub_rn(in[i].x, dist));
        c0 += sd == 0;
        c1 += sd == 1;
    }
    if (c0 == 0) {
        for (int i = 0; i < n; i++) back[i] = in[i];
        nb = n;
        return true;
    }
    if (c1 == 0) {
        for (int i = 0; i < n; i++) front[i] = in[i];
        nf = n;
        return true;
    }
    for (int i = 0; i < n; i++) {
        const Pt p1 = in[i];
        const float d1 = __fsub_rn(p1.x, dist);
        const int s1 = side_of(d1);
        if (nf + 2 > kPolyMax || nb + 2 > kPolyMax) return false;
        if (s1 == 2) {
            front[nf++] = p1;
            back[nb++] = p1;
            continue;
        }
        if (s1 == 0) front[nf++] = p1;
        else back[nb++] = p1;
        const Pt p2 = in[i + 1 == n ? 0 : i + 1];
        const float d2 = __fsub_rn(p2.x, dist);
        const int s2 = side_of(d2);
        if (s2 == 2 || s2 == s1) continue;
        const float t = __fdiv_rn(d1, __fsub_rn(d1, d2));
        const Pt mid = {dist, __fadd_rn(p1.y, __fmul_rn(t, __fsub_rn(p2.y, p1.y)))};
        front[nf++] = mid;
        back[nb++] = mid;
    }
    return true;
}

struct Frame {
    float ox, oy, oz;
    float sx, sy, sz;  // world to luxel s
    float tx, ty, tz;  // world to luxel t
    float ls[3], lt[3];  // luxel to world
    int width, min_s, min_t;
};

__device__ __forceinline__ Frame frame_of(const float4 *frames, int f) {
    const float4 a = __ldg(&frames[5 * f]), b = __ldg(&frames[5 * f + 1]), c = __ldg(&frames[5 * f + 2]),
                 d = __ldg(&frames[5 * f + 3]), e = __ldg(&frames[5 * f + 4]);
    Frame fr;
    fr.ox = a.x, fr.oy = a.y, fr.oz = a.z;
    fr.width = __float_as_int(a.w);
    fr.sx = b.x, fr.sy = b.y, fr.sz = b.z;
    fr.tx = c.x, fr.ty = c.y, fr.tz = c.z;
    fr.min_s = __float_as_int(c.w);
    fr.ls[0] = d.x, fr.ls[1] = d.y, fr.ls[2] = d.z;
    fr.min_t = __float_as_int(d.w);
    fr.lt[0] = e.x, fr.lt[1] = e.y, fr.lt[2] = e.z;
    return fr;
}

// LuxelToWorld: origin + l2w_s (s + min_s), then + l2w_t (t + min_t).
__device__ __forceinline__ void luxel_to_world(const Frame &fr, float s, float t, float out[3]) {
    s = __fadd_rn(s, (float)fr.min_s);
    t = __fadd_rn(t, (float)fr.min_t);
    const float o[3] = {fr.ox, fr.oy, fr.oz};
    for (int a = 0; a < 3; a++) out[a] = __fadd_rn(__fadd_rn(o[a], __fmul_rn(fr.ls[a], s)), __fmul_rn(fr.lt[a], t));
}

// One strip's cells.  COUNT: its samples and partial-cell points into
// ns[k], np[k].  Otherwise: the samples at s_off[k].., their windings'
// points at p_off[k].., each compared with the world's sample.
template <bool COUNT>
__global__ void __launch_bounds__(kWindBlock) k_wind_strips(
    int32_t nrows, const int32_t *__restrict__ row_face, const int32_t *__restrict__ row_t,
    const int64_t *__restrict__ row_first, const float2 *__restrict__ row_xy, const float *__restrict__ apl,
    FinalView fv, const float4 *__restrict__ check, int64_t nsamples, int32_t *__restrict__ ns,
    int32_t *__restrict__ np, const int64_t *__restrict__ s_off, const int64_t *__restrict__ p_off,
    int2 *__restrict__ wind, float4 *__restrict__ points, int32_t *__restrict__ cell, float2 *__restrict__ origin_st,
    uint32_t *__restrict__ flags) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nrows) return;
    const int f = __ldg(&row_face[k]), t = __ldg(&row_t[k]);
    const int64_t p0 = __ldg(&row_first[k]);
    int n = (int)(__ldg(&row_first[k + 1]) - p0);
    Pt buf[3][kPolyMax];
    Pt *row = buf[0], *rest = buf[1], *cellp = buf[2];
    for (int i = 0; i < n; i++) {
        const float2 q = __ldg(&row_xy[p0 + i]);
        row[i] = {q.x, q.y};
    }
    const Frame fr = frame_of(fv.frames, f);
    const float area_per_luxel = __ldg(&apl[f]);
    const double partial_below = __dsub_rn((double)area_per_luxel, 0.001);
    int64_t si = COUNT ? 0 : __ldg(&s_off[k]);
    int64_t pi = COUNT ? 0 : __ldg(&p_off[k]);
    int cnt_s = 0, cnt_p = 0;
    bool bad = false;
    for (int s = 0; s < fr.width && n > 0; s++) {
        int nf, nb;
        if (!clip_x(row, n, (float)s + 1.0f, rest, nf, cellp, nb)) {
            atomicOr(&flags[1], 1u);
            return;
        }
        if (nb > 0) {
            // AreaAndBalancePoint (z 0: the cross product's length is |z|
            // computed as sqrt(z * z), the host's (x x + y y) + z z with x, y 0).
            float cx = 0.0f, cy = 0.0f, total = 0.0f;
            for (int i = 2; i < nb; i++) {
                const float d1x = __fsub_rn(cellp[i - 1].x, cellp[0].x), d1y = __fsub_rn(cellp[i - 1].y, cellp[0].y);
                const float d2x = __fsub_rn(cellp[i].x, cellp[0].x), d2y = __fsub_rn(cellp[i].y, cellp[0].y);
                const float c = __fsub_rn(__fmul_rn(d1x, d2y), __fmul_rn(d1y, d2x));
                const float a = __fsqrt_rn(__fmul_rn(c, c));
                total = __fadd_rn(total, a);
                const float third = __double2float_rn(__ddiv_rn((double)a, 3.0));
                cx = __fadd_rn(cx, __fmul_rn(cellp[i - 1].x, third));
                cy = __fadd_rn(cy, __fmul_rn(cellp[i - 1].y, third));
                cx = __fadd_rn(cx, __fmul_rn(cellp[i].x, third));
                cy = __fadd_rn(cy, __fmul_rn(cellp[i].y, third));
                cx = __fadd_rn(cx, __fmul_rn(cellp[0].x, third));
                cy = __fadd_rn(cy, __fmul_rn(cellp[0].y, third));
            }
            if (total != 0.0f) {
                const float inv = __double2float_rn(__ddiv_rn(1.0, (double)total));
                cx = __fmul_rn(cx, inv);
                cy = __fmul_rn(cy, inv);
            }
            const float area = __fmul_rn(__fmul_rn(total, 0.5f), area_per_luxel);
            const bool partial = (double)area < partial_below;
            cnt_s++;
            if (partial) cnt_p += nb;
            if (!COUNT) {
                float mn0 = 99999.0f, mn1 = 99999.0f, mx0 = -99999.0f, mx1 = -99999.0f;
                for (int i = 0; i < nb; i++) {
                    if (cellp[i].x < mn0) mn0 = cellp[i].x;
                    if (cellp[i].x > mx0) mx0 = cellp[i].x;
                    if (cellp[i].y < mn1) mn1 = cellp[i].y;
                    if (cellp[i].y > mx1) mx1 = cellp[i].y;
                }
                float pos[3];
                luxel_to_world(fr, cx, cy, pos);
                // The world's sample at this index must be this one.
                if (si >= nsamples) {
                    bad = true;
                } else {
                    const float4 P = __ldg(&fv.sample_pos[si]), B = __ldg(&fv.sample_box[si]), C = __ldg(&check[si]);
                    const int cidx = __ldg(&fv.face_cells[f]) + s + t * fr.width;
                    bad |= __float_as_uint(P.x) != __float_as_uint(pos[0]) ||
                           __float_as_uint(P.y) != __float_as_uint(pos[1]) ||
                           __float_as_uint(P.z) != __float_as_uint(pos[2]) || __float_as_int(P.w) != f;
                    bad |= __float_as_uint(B.x) != __float_as_uint(mn0) || __float_as_uint(B.y) != __float_as_uint(mn1) ||
                           __float_as_uint(B.z) != __float_as_uint(mx0) || __float_as_uint(B.w) != __float_as_uint(mx1);
                    bad |= __float_as_uint(C.x) != __float_as_uint(area) || __float_as_uint(C.y) != __float_as_uint(cx) ||
                           __float_as_uint(C.z) != __float_as_uint(cy);
                    bad |= __ldg(&fv.cell_sample[cidx]) != (int32_t)si;
                    // The cell's winding in world space when partial.
                    wind[si] = partial ? make_int2((int)pi, nb) : make_int2(0, 0);
                    if (partial)
                        for (int i = 0; i < nb; i++) {
                            float w[3];
                            luxel_to_world(fr, cellp[i].x, cellp[i].y, w);
                            points[pi + i] = make_float4(w[0], w[1], w[2], 0.0f);
                        }
                    cell[si] = cidx;
                    // WorldToLuxel of the sample's position.
                    const float dx = __fsub_rn(pos[0], fr.ox), dy = __fsub_rn(pos[1], fr.oy), dz = __fsub_rn(pos[2], fr.oz);
                    const float os = __fsub_rn(
                        __fadd_rn(__fadd_rn(__fmul_rn(dx, fr.sx), __fmul_rn(dy, fr.sy)), __fmul_rn(dz, fr.sz)),
                        (float)fr.min_s);
                    const float ot = __fsub_rn(
                        __fadd_rn(__fadd_rn(__fmul_rn(dx, fr.tx), __fmul_rn(dy, fr.ty)), __fmul_rn(dz, fr.tz)),
                        (float)fr.min_t);
                    origin_st[si] = make_float2(os, ot);
                }
                if (partial) pi += nb;
                si++;
            }
        }
        Pt *tmp = row;
        row = rest;
        rest = tmp;
        n = nf;
    }
    if (COUNT) {
        ns[k] = cnt_s;
        np[k] = cnt_p;
    } else if (bad) {
        atomicOr(&flags[0], 1u);
    }
}

unsigned blocks_of(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

cudaError_t device_windings(SupersampleBuffers &ss, const RowStrips &rs, const FinalView &fv,
                            const float4 *check, int64_t nsamples, Stager &stager, cudaStream_t stream, bool &match,
                            std::string &why) {
    match = false;
    const int32_t nrows = (int32_t)rs.face.size();
    const int64_t S = nsamples;
    int32_t *d_face = nullptr, *d_t = nullptr, *d_ns = nullptr, *d_np = nullptr;
    int64_t *d_first = nullptr, *d_soff = nullptr, *d_poff = nullptr;
    float *d_xy = nullptr;  // (x, y) pairs
    float *d_apl = nullptr;
    float4 *d_check = nullptr;
    uint32_t *d_flags = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int64_t totals[2] = {0, 0};
    uint32_t flags[2] = {0, 0};
    const size_t R1 = (size_t)(nrows ? nrows : 1);
    cudaError_t e = stage_table(stager, stream, &d_face, rs.face);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_t, rs.t);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_first, rs.first);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_xy, rs.xy);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_apl, rs.apl);
    if (e == cudaSuccess) e = dma_table(&d_check, check, (size_t)S, stream);
    if (e == cudaSuccess) e = dev_alloc(&d_ns, sizeof(int32_t) * R1);
    if (e == cudaSuccess) e = dev_alloc(&d_np, sizeof(int32_t) * R1);
    if (e == cudaSuccess) e = dev_alloc(&d_soff, sizeof(int64_t) * (R1 + 1));
    if (e == cudaSuccess) e = dev_alloc(&d_poff, sizeof(int64_t) * (R1 + 1));
    if (e == cudaSuccess) e = dev_alloc(&d_flags, sizeof(uint32_t) * 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flags, 0, sizeof(uint32_t) * 2, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_soff, 0, sizeof(int64_t), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_poff, 0, sizeof(int64_t), stream);
    if (e == cudaSuccess && nrows > 0) {
        k_wind_strips<true><<<blocks_of(nrows, kWindBlock), kWindBlock, 0, stream>>>(
            nrows, d_face, d_t, d_first, reinterpret_cast<const float2 *>(d_xy), d_apl, fv, d_check, S, d_ns, d_np, nullptr, nullptr, nullptr, nullptr,
            nullptr, nullptr, d_flags);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, d_ns, d_soff + 1, nrows, stream);
        if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes ? tmp_bytes : 1);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, d_ns, d_soff + 1, nrows, stream);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, d_np, d_poff + 1, nrows, stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&totals[0], d_soff + nrows, sizeof(int64_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&totals[1], d_poff + nrows, sizeof(int64_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, d_flags, sizeof flags, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = stager.finish(stream);
    if (e == cudaSuccess && !flags[1] && totals[0] == S) {
        const size_t S1 = (size_t)(S ? S : 1);
        e = dev_alloc(&ss.wind, sizeof(int2) * S1);
        if (e == cudaSuccess) e = dev_alloc(&ss.points, sizeof(float4) * (size_t)(totals[1] ? totals[1] : 1));
        if (e == cudaSuccess) e = dev_alloc(&ss.cell, sizeof(int32_t) * S1);
        if (e == cudaSuccess) e = dev_alloc(&ss.origin_st, sizeof(float2) * S1);
        if (e == cudaSuccess && nrows > 0) {
            k_wind_strips<false><<<blocks_of(nrows, kWindBlock), kWindBlock, 0, stream>>>(
                nrows, d_face, d_t, d_first, reinterpret_cast<const float2 *>(d_xy), d_apl, fv, d_check, S, nullptr, nullptr, d_soff, d_poff, ss.wind,
                ss.points, ss.cell, ss.origin_st, d_flags);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(flags, d_flags, sizeof flags, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = vrad::wait_stream(stream);
        match = e == cudaSuccess && !flags[0] && !flags[1];
    }
    if (e == cudaSuccess && !match)
        why = flags[1] ? "a cell winding exceeds the rebuild's point capacity"
                       : "the samples are not the face sample builder's own, so their cell windings are unknown";
    for (void *q : {(void *)d_face, (void *)d_t, (void *)d_ns, (void *)d_np, (void *)d_first, (void *)d_soff,
                    (void *)d_poff, (void *)d_xy, (void *)d_apl, (void *)d_check, (void *)d_flags, tmp})
        dev_free(q);
    return e;
}

}  // namespace vrad
