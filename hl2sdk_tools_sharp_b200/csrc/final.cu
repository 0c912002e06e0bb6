// final.cu -- the lighting stage's final pass: each face's luxels from its
// own and its smoothing neighbours' light samples, minlight, the RGBE
// encode and the per-face median, written straight into the LIGHTING
// lump's byte image at the faces' lightofs.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad):
//   FinalLightFace.Run / BuildLuxelRadial (Final/FinalLightFace.cs:93-360),
//       style 0, no bounce (-bounce 0), no macro textures, minlight 0;
//   LuxelRadial.AddDirect / Sample (Final/LuxelRadial.cs:140-331);
//   StockLightColor.Encode (Ambient/StockLightColor.cs:136-185);
//   FinalLightFace.Median: sort, take element count >> 1;
//   LightmapOffsets.Compute (Light/LightmapOffsets.cs:54-126).
//
// Kernels (one launch each per pass):
//   k_radial  one thread per radial cell: the weighted sum of every sample
//             whose box covers the cell, in the reference's sample order
//             (the face's own samples, then each neighbour's)
//   k_luxel   one thread per luxel: LuxelRadial.Sample at the luxel's own
//             position, minlight, Encode, store
//   k_median  one CTA per face: bitonic sort of the sampled luxels per
//             channel, the median, Encode, store before lightofs

#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cstring>
#include <vector>

#include <string>
#include <type_traits>

#include "bounce_host.h"
#include "context.cuh"
#include "device_pool.h"
#include "final.cuh"
#include "host_parallel.h"
#include "setup_clock.h"
#include "world.h"
#include "sync_wait.h"

namespace vrad {

namespace {

constexpr int kMedianThreads = 1024;
constexpr int kMedianMax = 2048;  // luxels per face the median sorts in shared memory

__device__ __forceinline__ void world_to_luxel(const float4 &o, const float4 &ws, const float4 &wt, int mins,
                                               int mint, float px, float py, float pz, float &s, float &t) {
    const float x = __fsub_rn(px, o.x), y = __fsub_rn(py, o.y), z = __fsub_rn(pz, o.z);
    s = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, ws.x), __fmul_rn(y, ws.y)), __fmul_rn(z, ws.z)), (float)mins);
    t = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(x, wt.x), __fmul_rn(y, wt.y)), __fmul_rn(z, wt.z)), (float)mint);
}

struct Frame {
    float4 o, ws, wt, ls, lt;
    int w, h, mins, mint, lightofs;
};

__device__ __forceinline__ Frame load_frame(const float4 *__restrict__ frames, int f) {
    Frame fr;
    fr.o = __ldg(&frames[5 * f + 0]);
    fr.ws = __ldg(&frames[5 * f + 1]);
    fr.wt = __ldg(&frames[5 * f + 2]);
    fr.ls = __ldg(&frames[5 * f + 3]);
    fr.lt = __ldg(&frames[5 * f + 4]);
    fr.w = __float_as_int(fr.o.w);
    fr.h = __float_as_int(fr.ws.w);
    fr.mins = __float_as_int(fr.wt.w);
    fr.mint = __float_as_int(fr.ls.w);
    fr.lightofs = __float_as_int(fr.lt.w);
    return fr;
}

// One sample's contribution to cell (s, t): LuxelRadial.AddDirect.
__device__ __forceinline__ void add_direct(const Frame &fr, int s, int t, const float4 &pos, const float4 &box,
                                           const float4 &light, float &lx, float &ly, float &lz, float &lsun,
                                           float &weight) {
    float cs, ct;
    world_to_luxel(fr.o, fr.ws, fr.wt, fr.mins, fr.mint, pos.x, pos.y, pos.z, cs, ct);
    int smin = __float2int_rz(box.x), tmin = __float2int_rz(box.y);
    int smax = __float2int_rz(__fadd_rn(box.z, 0.9999f)) + 1, tmax = __float2int_rz(__fadd_rn(box.w, 0.9999f)) + 1;
    smin = max(smin, 0);
    tmin = max(tmin, 0);
    smax = min(smax, fr.w);
    tmax = min(tmax, fr.h);
    if (s < smin || s >= smax || t < tmin || t >= tmax) return;
    // max / min against -1 and 1 (compared in double, which changes nothing).
    const float ds0 = __fsub_rn(box.x, (float)s);
    const float s0 = ds0 > -1.0f ? ds0 : -1.0f;
    const float dt0 = __fsub_rn(box.y, (float)t);
    const float t0 = dt0 > -1.0f ? dt0 : -1.0f;
    const float ds1 = __fsub_rn(box.z, (float)s);
    const float s1 = ds1 < 1.0f ? ds1 : 1.0f;
    const float dt1 = __fsub_rn(box.w, (float)t);
    const float t1 = dt1 < 1.0f ? dt1 : 1.0f;
    const float area = __fmul_rn(__fsub_rn(s1, s0), __fsub_rn(t1, t0));
    if (!((double)area > 0.001)) return;
    const float ds = fabsf(__fsub_rn(cs, (float)s)), dt = fabsf(__fsub_rn(ct, (float)t));
    float r = ds > dt ? ds : dt;
    r = ((double)r < 0.1) ? (float)__ddiv_rn((double)area, 0.1) : __fdiv_rn(area, r);
    lx = __fadd_rn(lx, __fmul_rn(r, light.x));
    ly = __fadd_rn(ly, __fmul_rn(r, light.y));
    lz = __fadd_rn(lz, __fmul_rn(r, light.z));
    lsun = __fadd_rn(lsun, __fmul_rn(r, light.w));
    weight = __fadd_rn(weight, r);
}

__global__ void k_radial(FinalView v, const float4 *__restrict__ sample_light, float4 *__restrict__ rad_light,
                         float *__restrict__ rad_weight) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= v.ncells) return;
    const int f = __ldg(&v.cell_face[c]);
    if (v.style_slot && __ldg(&v.style_slot[f]) < 0) return;
    const Frame fr = load_frame(v.frames, f);
    const int base = __ldg(&v.face_cells[f]);
    const int local = (int)(c - base);
    const int s = local % fr.w, t = local / fr.w;
    float lx = 0.0f, ly = 0.0f, lz = 0.0f, lsun = 0.0f, weight = 0.0f;
    // The face's own samples: only cells within two of this one can cover
    // it, visited in sample order (rows, then columns).
    for (int tc = t - 2; tc <= t + 1; tc++) {
        if (tc < 0 || tc >= fr.h) continue;
        for (int sc = s - 2; sc <= s + 1; sc++) {
            if (sc < 0 || sc >= fr.w) continue;
            const int k = __ldg(&v.cell_sample[base + sc + tc * fr.w]);
            if (k < 0) continue;
            add_direct(fr, s, t, __ldg(&v.sample_pos[k]), __ldg(&v.sample_box[k]), __ldg(&sample_light[k]), lx, ly,
                       lz, lsun, weight);
        }
    }
    // Then every neighbour's samples that can reach this face, in order
    // (of a neighbour that has this light style: BuildLuxelRadial matches
    // the style number, FinalLightFace.cs:339-360).
    const int c0 = __ldg(&v.cand_off[f]), c1 = __ldg(&v.cand_off[f + 1]);
    for (int q = c0; q < c1; q++) {
        const int k = __ldg(&v.cand_sample[q]);
        const float4 pos = __ldg(&v.sample_pos[k]);
        if (v.style_slot && __ldg(&v.style_slot[__float_as_int(pos.w)]) < 0) continue;
        add_direct(fr, s, t, pos, __ldg(&v.cand_box[q]), __ldg(&sample_light[k]), lx, ly, lz, lsun, weight);
    }
    rad_light[c] = make_float4(lx, ly, lz, lsun);
    rad_weight[c] = weight;
}

// The bounced light's radial grid: LuxelRadial.AddBounced for every leaf
// patch in the face's list whose box holds this cell, in list order.
__global__ void k_patch_radial(FinalView v, PatchRadialView p) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= v.ncells) return;
    const int f = __ldg(&v.cell_face[c]);
    const int base = __ldg(&v.face_cells[f]);
    const int w = __float_as_int(__ldg(&v.frames[5 * f].w));
    const int local = (int)(c - base);
    const int s = local % w, t = local / w;
    float lx = 0.0f, ly = 0.0f, lz = 0.0f, weight = 0.0f;
    const int q0 = __ldg(&p.off[f]), q1 = __ldg(&p.off[f + 1]);
    for (int q = q0; q < q1; q++) {
        const int4 b = __ldg(&p.box[q]);
        if (s < b.x || s >= b.z || t < b.y || t >= b.w) continue;
        const float4 k = __ldg(&p.coord[q]);
        const float ds = __fdiv_rn(__fsub_rn(k.x, (float)s), k.z);
        const float dt = __fdiv_rn(__fsub_rn(k.y, (float)t), k.w);
        const float r = __fsub_rn(2.0f, __fadd_rn(__fmul_rn(ds, ds), __fmul_rn(dt, dt)));
        if (r > 0.0f) {
            const float4 L = __ldg(&p.light[__ldg(&p.patch[q])]);
            lx = __fadd_rn(lx, __fmul_rn(r, L.x));
            ly = __fadd_rn(ly, __fmul_rn(r, L.y));
            lz = __fadd_rn(lz, __fmul_rn(r, L.z));
            weight = __fadd_rn(weight, r);
        }
    }
    p.rad_light[c] = make_float4(lx, ly, lz, 0.0f);
    p.rad_weight[c] = weight;
}

// StockLightColor.Encode: ColorRGBExp32 as a little-endian word.
__device__ __forceinline__ uint32_t encode(float x, float y, float z) {
    float m;
    if (x > y)
        m = x > z ? x : z;
    else
        m = y > z ? y : z;
    int e = 0;
    if (m != 0.0f) e = (int)((__float_as_uint(m) & 0x7F800000u) >> 23) - (7 + 127);
    const float scalar = __uint_as_float((uint32_t)(127 - e) << 23);
    const uint32_t r = (uint8_t)__float2int_rz(__fmul_rn(x, scalar));
    const uint32_t g = (uint8_t)__float2int_rz(__fmul_rn(y, scalar));
    const uint32_t b = (uint8_t)__float2int_rz(__fmul_rn(z, scalar));
    return r | (g << 8) | (b << 16) | ((uint32_t)(uint8_t)(int8_t)e << 24);
}

__global__ void k_luxel(FinalView v, const float4 *__restrict__ rad_light, const float *__restrict__ rad_weight,
                        const float4 *__restrict__ prad_light, const float *__restrict__ prad_weight,
                        uint32_t *__restrict__ lighting, float4 *__restrict__ flat) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= v.ncells) return;
    const int f = __ldg(&v.cell_face[c]);
    const int slot = v.style_slot ? __ldg(&v.style_slot[f]) : 0;
    if (slot < 0) return;
    const Frame fr = load_frame(v.frames, f);
    const int base = __ldg(&v.face_cells[f]);
    const int j = (int)(c - base);
    const float s = (float)(j % fr.w), t = (float)(j / fr.w);
    // The luxel's world position (BuildFaceLuxels), back into luxel space.
    const float ss = __fadd_rn(s, (float)fr.mins), tt = __fadd_rn(t, (float)fr.mint);
    const float px = __fadd_rn(__fadd_rn(fr.o.x, __fmul_rn(fr.ls.x, ss)), __fmul_rn(fr.lt.x, tt));
    const float py = __fadd_rn(__fadd_rn(fr.o.y, __fmul_rn(fr.ls.y, ss)), __fmul_rn(fr.lt.y, tt));
    const float pz = __fadd_rn(__fadd_rn(fr.o.z, __fmul_rn(fr.ls.z, ss)), __fmul_rn(fr.lt.z, tt));
    float cs, ct;
    world_to_luxel(fr.o, fr.ws, fr.wt, fr.mins, fr.mint, px, py, pz, cs, ct);
    const int u = __float2int_rz(__fadd_rn(cs, 0.5f)), w = __float2int_rz(__fadd_rn(ct, 0.5f));
    float lx = 0.0f, ly = 0.0f, lz = 0.0f;
    bool ok = true;
    if (u < 0 || u >= fr.w || w < 0 || w >= fr.h) {
        lx = 2550.0f;  // LuxelRadial.ErrorRed
        ok = false;
    } else {
        const int i = base + u + w * fr.w;
        const float wt = rad_weight[i];
        if (wt > 0.00001f) {
            const float4 L = rad_light[i];
            const float scale = (float)__drcp_rn((double)wt);
            lx = __fmul_rn(L.x, scale);
            ly = __fmul_rn(L.y, scale);
            lz = __fmul_rn(L.z, scale);
        } else {
            ok = false;
        }
    }
    if (prad_light) {
        // The bounced light, style 0: the patch grid sampled the same way
        // (its own off-grid red and weight test), added before minlight.
        float bx = 0.0f, by = 0.0f, bz = 0.0f;
        if (u < 0 || u >= fr.w || w < 0 || w >= fr.h) {
            bx = 2550.0f;
        } else {
            const int i = base + u + w * fr.w;
            const float wt = prad_weight[i];
            if (wt > 0.00001f) {
                const float4 L = prad_light[i];
                const float scale = (float)__drcp_rn((double)wt);
                bx = __fmul_rn(L.x, scale);
                by = __fmul_rn(L.y, scale);
                bz = __fmul_rn(L.z, scale);
            }
        }
        lx = __fadd_rn(lx, bx);
        ly = __fadd_rn(ly, by);
        lz = __fadd_rn(lz, bz);
    }
    if (__ldg(&v.face_nsamples[f]) == 0) {
        lx = 255.0f;
        ly = 0.0f;
        lz = 0.0f;
        ok = false;
    }
    // max(value, minlight) with minlight 0.
    lx = lx > 0.0f ? lx : 0.0f;
    ly = ly > 0.0f ? ly : 0.0f;
    lz = lz > 0.0f ? lz : 0.0f;
    // Slot k's luxels follow slot k - 1's.
    lighting[fr.lightofs / 4 + slot * fr.w * fr.h + j] = encode(lx, ly, lz);
    flat[c] = make_float4(lx, ly, lz, ok ? 1.0f : 0.0f);
}

__device__ void bitonic(float *a, int n) {
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const float x = a[i], y = a[l];
                    if ((x > y) == up) {
                        a[i] = y;
                        a[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kMedianThreads) k_median(FinalView v, const float4 *__restrict__ flat,
                                                           uint32_t *__restrict__ lighting) {
    __shared__ float ch[3][kMedianMax];
    __shared__ int count;
    const int f = blockIdx.x;
    const int style_slot = v.style_slot ? __ldg(&v.style_slot[f]) : 0;
    if (style_slot < 0) return;  // the whole block
    const Frame fr = load_frame(v.frames, f);
    const int base = __ldg(&v.face_cells[f]);
    const int n = fr.w * fr.h;
    if (threadIdx.x == 0) count = 0;
    for (int i = threadIdx.x; i < kMedianMax; i += blockDim.x) ch[0][i] = ch[1][i] = ch[2][i] = FLT_MAX;
    __syncthreads();
    // Compact the sampled luxels, in luxel order (their order is irrelevant
    // to a sort, but the count is what the median index uses).
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 q = flat[base + i];
        if (q.w != 0.0f) {
            const int slot = atomicAdd(&count, 1);
            ch[0][slot] = q.x;
            ch[1][slot] = q.y;
            ch[2][slot] = q.z;
        }
    }
    __syncthreads();
    bitonic(ch[0], kMedianMax);
    bitonic(ch[1], kMedianMax);
    bitonic(ch[2], kMedianMax);
    if (threadIdx.x == 0) {
        const int m = count >> 1;
        const float x = count ? ch[0][m] : 0.0f, y = count ? ch[1][m] : 0.0f, z = count ? ch[2][m] : 0.0f;
        // Before lightofs, in reverse style order.
        lighting[fr.lightofs / 4 - 1 - style_slot] = encode(x, y, z);
    }
}

}  // namespace

void FinalBuffers::release() {
    dev_free(frames);
    dev_free(face_cells);
    dev_free(face_nsamples);
    dev_free(cell_face);
    dev_free(cell_sample);
    dev_free(sample_box);
    dev_free(cand_off);
    dev_free(cand_sample);
    dev_free(cand_box);
    dev_free(rad_light);
    dev_free(rad_weight);
    dev_free(flat);
    *this = FinalBuffers();
}

cudaError_t launch_final(const FinalView &v, const float4 *sample_light, float4 *rad_light, float *rad_weight,
                         float4 *flat, uint8_t *lighting, int nfaces, const PatchRadialView *prad,
                         cudaStream_t stream) {
    if (v.ncells == 0) return cudaSuccess;
    const unsigned grid = (unsigned)((v.ncells + 255) / 256);
    k_radial<<<grid, 256, 0, stream>>>(v, sample_light, rad_light, rad_weight);
    if (prad) k_patch_radial<<<grid, 256, 0, stream>>>(v, *prad);
    k_luxel<<<grid, 256, 0, stream>>>(v, rad_light, rad_weight, prad ? prad->rad_light : nullptr,
                                      prad ? prad->rad_weight : nullptr, reinterpret_cast<uint32_t *>(lighting), flat);
    k_median<<<nfaces, kMedianThreads, 0, stream>>>(v, flat, reinterpret_cast<uint32_t *>(lighting));
    return cudaGetLastError();
}

namespace {

// x86's truncating float-to-int conversion, which the host set-up's
// (int) casts compile to: out of range and NaN give INT_MIN.
__device__ __forceinline__ int trunc_x86(float x) {
    return (x > -2147483648.0f && x < 2147483648.0f) ? __float2int_rz(x) : INT_MIN;
}

// LuxelToWorld / WorldToLuxel of the luxel frames (frames[5 f ..]: origin
// and width, world-to-luxel s and height, world-to-luxel t and min_s,
// luxel-to-world s and min_t, luxel-to-world t), each operation rounded
// on its own in the host's order.
__device__ __forceinline__ void frame_l2w(const float4 *fr, float s, float t, float out[3]) {
    const float4 o = __ldg(&fr[0]), ls = __ldg(&fr[3]), lt = __ldg(&fr[4]);
    s = __fadd_rn(s, (float)__float_as_int(__ldg(&fr[2].w)));
    t = __fadd_rn(t, (float)__float_as_int(ls.w));
    out[0] = __fadd_rn(__fadd_rn(o.x, __fmul_rn(ls.x, s)), __fmul_rn(lt.x, t));
    out[1] = __fadd_rn(__fadd_rn(o.y, __fmul_rn(ls.y, s)), __fmul_rn(lt.y, t));
    out[2] = __fadd_rn(__fadd_rn(o.z, __fmul_rn(ls.z, s)), __fmul_rn(lt.z, t));
}

__device__ __forceinline__ void frame_w2l(const float4 *fr, const float p[3], float &s, float &t) {
    const float4 o = __ldg(&fr[0]), ws = __ldg(&fr[1]), wt = __ldg(&fr[2]), ls = __ldg(&fr[3]);
    const float dx = __fsub_rn(p[0], o.x), dy = __fsub_rn(p[1], o.y), dz = __fsub_rn(p[2], o.z);
    s = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, ws.x), __fmul_rn(dy, ws.y)), __fmul_rn(dz, ws.z)),
                  (float)__float_as_int(wt.w));
    t = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, wt.x), __fmul_rn(dy, wt.y)), __fmul_rn(dz, wt.z)),
                  (float)__float_as_int(ls.w));
}

// One (face, neighbour) pair: the neighbour's samples whose box, moved
// into the face's luxel space, covers a cell.  COUNT: their number into
// counts[q]; else their indices and moved boxes at off[q]...
template <bool COUNT>
__global__ void k_final_cands(int32_t npairs, const int32_t *__restrict__ pair_face, const int32_t *__restrict__ nlist,
                              const float4 *__restrict__ frames, const int64_t *__restrict__ srun,
                              const float4 *__restrict__ sbox, int32_t *__restrict__ counts,
                              const int64_t *__restrict__ off, int32_t *__restrict__ cand_sample,
                              float4 *__restrict__ cand_box) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npairs) return;
    const int f = __ldg(&pair_face[q]), g = __ldg(&nlist[q]);
    const float4 *me = frames + 5 * (int64_t)f, *nb = frames + 5 * (int64_t)g;
    const int width = __float_as_int(__ldg(&me[0].w)), height = __float_as_int(__ldg(&me[1].w));
    int64_t at = COUNT ? 0 : __ldg(&off[q]);
    int n = 0;
    for (int64_t k = __ldg(&srun[2 * g]); k < __ldg(&srun[2 * g + 1]); k++) {
        const float4 b = __ldg(&sbox[k]);
        float tmp[3], mins, mint, maxs, maxt;
        frame_l2w(nb, b.x, b.y, tmp);
        frame_w2l(me, tmp, mins, mint);
        frame_l2w(nb, b.z, b.w, tmp);
        frame_w2l(me, tmp, maxs, maxt);
        int smin = trunc_x86(mins), tmin = trunc_x86(mint);
        int smax = trunc_x86(__fadd_rn(maxs, 0.9999f)) + 1, tmax = trunc_x86(__fadd_rn(maxt, 0.9999f)) + 1;
        smin = smin > 0 ? smin : 0;
        tmin = tmin > 0 ? tmin : 0;
        smax = smax < width ? smax : width;
        tmax = tmax < height ? tmax : height;
        if (smin >= smax || tmin >= tmax) continue;
        if (!COUNT) {
            cand_sample[at] = (int32_t)k;
            cand_box[at] = make_float4(mins, mint, maxs, maxt);
            at++;
        }
        n++;
    }
    if (COUNT) counts[q] = n;
}

// cand_off[f] = off[noff[f]].
__global__ void k_final_cand_off(int32_t nfaces, const int32_t *__restrict__ noff, const int64_t *__restrict__ off,
                                 int32_t *__restrict__ cand_off) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f <= nfaces) cand_off[f] = (int32_t)off[noff[f]];
}

unsigned blocks_of(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

// The final pass's neighbour candidate tables on the device (fb.frames and
// fb.sample_box already uploaded on `stream`): fb.cand_off, cand_sample,
// cand_box.  Synchronises the stream once, for the total's size.
cudaError_t neighbour_candidates(FinalBuffers &fb, int32_t nfaces, const std::vector<int32_t> &noff,
                                 const std::vector<int32_t> &nlist, const std::vector<int64_t> &sfirst,
                                 const std::vector<int64_t> &send, Stager &stager, cudaStream_t stream) {
    const int32_t npairs = noff[(size_t)nfaces];
    std::vector<int32_t> pair_face((size_t)(npairs ? npairs : 1), 0);
    for (int32_t f = 0; f < nfaces; f++)
        for (int32_t q = noff[(size_t)f]; q < noff[(size_t)f + 1]; q++) pair_face[(size_t)q] = f;
    std::vector<int64_t> srun(2 * (size_t)(nfaces ? nfaces : 1), 0);
    for (int32_t f = 0; f < nfaces; f++) {
        srun[2 * (size_t)f] = sfirst[(size_t)f];
        srun[2 * (size_t)f + 1] = send[(size_t)f];
    }
    int32_t *d_pf = nullptr, *d_nlist = nullptr, *d_noff = nullptr, *d_counts = nullptr;
    int64_t *d_srun = nullptr, *d_off = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int64_t total = 0;
    const size_t P1 = (size_t)(npairs ? npairs : 1);
    cudaError_t e = stage_table(stager, stream, &d_pf, pair_face);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_nlist, nlist);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_noff, noff);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_srun, srun);
    if (e == cudaSuccess) e = dev_alloc(&d_counts, sizeof(int32_t) * P1);
    if (e == cudaSuccess) e = dev_alloc(&d_off, sizeof(int64_t) * (P1 + 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_off, 0, sizeof(int64_t), stream);
    if (e == cudaSuccess && npairs > 0) {
        k_final_cands<true><<<blocks_of(npairs, 128), 128, 0, stream>>>(npairs, d_pf, d_nlist, fb.frames, d_srun,
                                                                       fb.sample_box, d_counts, nullptr, nullptr,
                                                                       nullptr);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, d_counts, d_off + 1, npairs, stream);
        if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes ? tmp_bytes : 1);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, d_counts, d_off + 1, npairs, stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, d_off + npairs, sizeof total, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = stager.finish(stream);
    if (e == cudaSuccess) e = dev_alloc(&fb.cand_off, sizeof(int32_t) * ((size_t)nfaces + 1));
    if (e == cudaSuccess) e = dev_alloc(&fb.cand_sample, sizeof(int32_t) * (size_t)(total ? total : 1));
    if (e == cudaSuccess) e = dev_alloc(&fb.cand_box, sizeof(float4) * (size_t)(total ? total : 1));
    if (e == cudaSuccess && npairs > 0) {
        k_final_cands<false><<<blocks_of(npairs, 128), 128, 0, stream>>>(npairs, d_pf, d_nlist, fb.frames, d_srun,
                                                                        fb.sample_box, nullptr, d_off, fb.cand_sample,
                                                                        fb.cand_box);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_final_cand_off<<<blocks_of((int64_t)nfaces + 1, 256), 256, 0, stream>>>(nfaces, d_noff, d_off, fb.cand_off);
        e = cudaGetLastError();
    }
    // The temporaries go back to the pool once the kernels are done.
    if (e == cudaSuccess) e = vrad::wait_stream(stream);
    for (void *q : {(void *)d_pf, (void *)d_nlist, (void *)d_noff, (void *)d_counts, (void *)d_srun, (void *)d_off, tmp})
        dev_free(q);
    return e;
}

}  // namespace

// Host-side set-up of the final pass from the uploaded world.
cudaError_t build_final(FinalBuffers &fb, const vrad_face *faces, int32_t nfaces, const vrad_sample *samples,
                        int64_t nsamples, const float *vertices, int64_t nvertices, std::vector<int32_t> &noff,
                        std::vector<int32_t> &nlist, Stager &stager, cudaStream_t stream, std::string &why,
                        const int64_t *run_first, const int64_t *run_end) {
    fb.release();
    SetupClock clock("final_tables");
    std::vector<FaceFrameOut> fr((size_t)nfaces);
    for (int32_t f = 0; f < nfaces; f++) face_frame_of(faces[f], fr[(size_t)f]);
    // Neighbours (FaceNeighbours.Build, DefaultSmoothingThreshold), kept
    // for the bounce's set-up.
    if (face_neighbours(faces, nfaces, vertices, nvertices, 0.7071067f, noff, nlist) != VRAD_OK) {
        why = "invalid face windings";
        return cudaErrorInvalidValue;
    }
    if (nlist.empty()) nlist.push_back(0);
    clock.mark("neighbours");
    std::vector<int32_t> lightofs((size_t)nfaces);
    int64_t total = 0;
    vrad_lightmap_layout(faces, nfaces, lightofs.data(), &total);
    // Each face's sample run [sfirst, send) (the world upload checked
    // that a face's samples are contiguous; runs need not be in face order).
    std::vector<int64_t> sfirst((size_t)nfaces, 0), send((size_t)nfaces, 0), scount((size_t)nfaces, 0);
    if (run_first && run_end) {
        for (int32_t f = 0; f < nfaces; f++)
            if (run_first[f] >= 0) {
                sfirst[(size_t)f] = run_first[f];
                send[(size_t)f] = run_end[f];
            }
    } else {
        parallel_for(nsamples, 1 << 16, [&](int64_t k) {
            const int32_t f = samples[k].face;
            if (k == 0 || samples[k - 1].face != f) sfirst[(size_t)f] = k;
            if (k + 1 == nsamples || samples[k + 1].face != f) send[(size_t)f] = k + 1;
        });
    }
    for (int32_t f = 0; f < nfaces; f++) scount[(size_t)f] = send[(size_t)f] - sfirst[(size_t)f];
    // Frames, cells, own-sample cell table.
    std::vector<float4> frames((size_t)nfaces * 5);
    std::vector<int32_t> face_cells((size_t)nfaces + 1, 0), face_ns((size_t)nfaces);
    for (int32_t f = 0; f < nfaces; f++) {
        const FaceFrameOut &q = fr[(size_t)f];
        if ((int64_t)q.width * q.height > kMedianMax) {
            why = "a face's lightmap exceeds the 2048 luxels the median sorts on chip";
            return cudaErrorInvalidValue;
        }
        auto bitsf = [](int32_t x) {
            float y;
            memcpy(&y, &x, 4);
            return y;
        };
        frames[5 * (size_t)f + 0] = make_float4(q.origin[0], q.origin[1], q.origin[2], bitsf(q.width));
        frames[5 * (size_t)f + 1] = make_float4(q.w2l_s[0], q.w2l_s[1], q.w2l_s[2], bitsf(q.height));
        frames[5 * (size_t)f + 2] = make_float4(q.w2l_t[0], q.w2l_t[1], q.w2l_t[2], bitsf(q.min_s));
        frames[5 * (size_t)f + 3] = make_float4(q.l2w_s[0], q.l2w_s[1], q.l2w_s[2], bitsf(q.min_t));
        frames[5 * (size_t)f + 4] = make_float4(q.l2w_t[0], q.l2w_t[1], q.l2w_t[2], bitsf(lightofs[(size_t)f]));
        face_cells[(size_t)f + 1] = face_cells[(size_t)f] + q.width * q.height;
        face_ns[(size_t)f] = (int32_t)scount[(size_t)f];
    }
    const int64_t ncells = face_cells[(size_t)nfaces];
    uvector<int32_t> cell_face((size_t)ncells), cell_sample((size_t)ncells);
    parallel_for(nfaces, 16, [&](int64_t f) {
        for (int32_t c = face_cells[(size_t)f]; c < face_cells[(size_t)f + 1]; c++) {
            cell_face[(size_t)c] = (int32_t)f;
            cell_sample[(size_t)c] = -1;
        }
    });
    uvector<float4> sbox((size_t)nsamples);
    std::atomic<bool> outside{false};
    parallel_for(nsamples, 1 << 15, [&](int64_t i) {
        const vrad_sample &sm = samples[i];
        const FaceFrameOut &q = fr[(size_t)sm.face];
        if (sm.s < 0 || sm.s >= q.width || sm.t < 0 || sm.t >= q.height) {
            outside = true;
            return;
        }
        cell_sample[(size_t)(face_cells[(size_t)sm.face] + sm.s + sm.t * q.width)] = (int32_t)i;
        sbox[(size_t)i] = make_float4(sm.mins[0], sm.mins[1], sm.maxs[0], sm.maxs[1]);
    });
    if (outside) {
        why = "a sample's cell lies outside its face's lightmap";
        return cudaErrorInvalidValue;
    }
    clock.mark("frames and cells");
    auto up = [&](auto **dst, const auto &v) { return stage_table(stager, stream, dst, v); };
    cudaError_t e = up(&fb.frames, frames);
    if (e == cudaSuccess) e = up(&fb.face_cells, face_cells);
    if (e == cudaSuccess) e = up(&fb.face_nsamples, face_ns);
    if (e == cudaSuccess) e = up(&fb.cell_face, cell_face);
    if (e == cudaSuccess) e = up(&fb.cell_sample, cell_sample);
    if (e == cudaSuccess) e = up(&fb.sample_box, sbox);
    // Neighbour candidates on the device: each neighbour's samples whose
    // box, moved into this face's luxel space as BuildLuxelRadial moves
    // it, can cover a cell; one thread per (face, neighbour) pair, counted,
    // scanned, then written in face, neighbour and sample order.
    if (e == cudaSuccess) e = neighbour_candidates(fb, nfaces, noff, nlist, sfirst, send, stager, stream);
    clock.mark("candidates");
    if (e == cudaSuccess) e = vrad::dev_alloc(&fb.rad_light, sizeof(float4) * (size_t)(ncells ? ncells : 1));
    if (e == cudaSuccess) e = vrad::dev_alloc(&fb.rad_weight, sizeof(float) * (size_t)(ncells ? ncells : 1));
    if (e == cudaSuccess) e = vrad::dev_alloc(&fb.flat, sizeof(float4) * (size_t)(ncells ? ncells : 1));
    if (e != cudaSuccess) {
        fb.release();
        why = "final-pass buffers";
        return e;
    }
    clock.mark("upload");
    fb.lighting_bytes = total;
    fb.nfaces = nfaces;
    fb.lightofs = lightofs;
    fb.h_frames = frames;
    fb.view = FinalView{fb.frames, fb.face_cells, fb.face_nsamples, fb.cell_face, fb.cell_sample, nullptr,
                        fb.sample_box, fb.cand_off, fb.cand_sample, fb.cand_box, ncells};
    fb.ready = true;
    return cudaSuccess;
}

}  // namespace vrad

namespace {

// One light pass's events: its start, the end of the direct gather, and
// per range the end of its bounce and of its final pass.
struct PassEvents {
    cudaEvent_t start = nullptr, direct = nullptr, bounce[2] = {nullptr, nullptr}, final_[2] = {nullptr, nullptr};
    cudaError_t create() {
        cudaError_t e = cudaSuccess;
        for (cudaEvent_t *x : {&start, &direct, &bounce[0], &bounce[1], &final_[0], &final_[1]})
            if (e == cudaSuccess) e = cudaEventCreate(x);
        return e;
    }
    ~PassEvents() {
        for (cudaEvent_t x : {start, direct, bounce[0], bounce[1], final_[0], final_[1]})
            if (x) cudaEventDestroy(x);
    }
};

// The style slots and the lightmap layout of a world with light styles
// above 0, made once per world on stream s: each style's lights gathered
// (LDR) with the first-lit keys, then per face style 0 in slot 0 and the
// styles its groups light, in key order, three at most (FaceLightJob's
// FindOrAllocateStyle; a fifth style is dropped and counted), then the
// layout (LightmapOffsets.Compute) and the frames' lightofs words.
int32_t ensure_style_layout(vrad_ctx *ctx, cudaStream_t s) {
    vrad::StyleState &st = ctx->styles;
    if (st.styles.empty() || st.ready) return VRAD_OK;
    vrad::FinalBuffers &fb = ctx->final_pass;
    if (!fb.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without face windings");
    const int32_t nf = fb.nfaces, S = (int32_t)st.styles.size();
    const int64_t ns = ctx->world.view.nsamples;
    cudaError_t e = cudaSuccess;
    for (int r = 0; r < 2 && e == cudaSuccess; r++) {
        if (r == 1 && !ctx->world.view.lights_hdr) break;
        st.light[r].assign((size_t)S, nullptr);
        for (int32_t i = 0; i < S && e == cudaSuccess; i++)
            e = vrad::dev_alloc(&st.light[r][(size_t)i], sizeof(float4) * (size_t)(ns ? ns : 1));
    }
    if (e == cudaSuccess) e = vrad::dev_alloc(&st.keys, sizeof(unsigned long long) * (size_t)S * (size_t)(nf ? nf : 1));
    if (e == cudaSuccess) e = vrad::dev_alloc(&st.slots, (size_t)S * (size_t)(nf ? nf : 1));
    // The ray counts of these gathers go to a scratch counter: a light
    // pass's statistics count its own rays.
    unsigned long long *scratch = nullptr;
    if (e == cudaSuccess) e = vrad::dev_alloc(&scratch, 3 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(st.keys, 0xFF, sizeof(unsigned long long) * (size_t)S * nf, s);
    for (int32_t i = 0; i < S && e == cudaSuccess; i++) {
        vrad::DeviceWorld v = vrad::range_view(ctx->world.view, false);
        v.style = st.styles[(size_t)i];
        v.face_key = st.keys + (size_t)i * nf;
        e = vrad::launch_direct(ctx->scene.view(), v, st.light[0][(size_t)i], nullptr, scratch, ctx->status, s,
                                ctx->world.block);
    }
    std::vector<unsigned long long> keys((size_t)S * nf);
    if (e == cudaSuccess && nf)
        e = cudaMemcpyAsync(keys.data(), st.keys, sizeof(unsigned long long) * keys.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = vrad::wait_stream(s);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "light style slots");  // (scratch kept: kernels may run)
    vrad::dev_free(scratch);
    std::vector<int8_t> slots((size_t)S * nf, -1);
    st.face_styles.assign((size_t)nf * 4, 255);
    st.dropped = 0;
    for (int32_t f = 0; f < nf; f++) {
        std::vector<std::pair<unsigned long long, int32_t>> lit;
        for (int32_t i = 0; i < S; i++)
            if (keys[(size_t)i * nf + f] != ~0ull) lit.push_back({keys[(size_t)i * nf + f], i});
        std::sort(lit.begin(), lit.end());
        st.face_styles[(size_t)f * 4] = 0;
        for (size_t k = 0; k < lit.size(); k++) {
            if (k >= 3) {
                st.dropped++;
                break;
            }
            st.face_styles[(size_t)f * 4 + 1 + k] = (uint8_t)st.styles[(size_t)lit[k].second];
            slots[(size_t)lit[k].second * nf + f] = (int8_t)(1 + k);
        }
    }
    int64_t total = 0;
    std::vector<int32_t> ofs((size_t)nf);
    vrad_lightmap_layout_styles(ctx->h_faces.data(), nf, st.face_styles.data(), ofs.data(), &total);
    for (int32_t f = 0; f < nf; f++) std::memcpy(&fb.h_frames[(size_t)f * 5 + 4].w, &ofs[(size_t)f], 4);
    if (e == cudaSuccess && nf)
        e = cudaMemcpyAsync(st.slots, slots.data(), slots.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && nf)
        e = cudaMemcpyAsync(fb.frames, fb.h_frames.data(), sizeof(float4) * fb.h_frames.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = vrad::wait_stream(s);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "light style layout");
    fb.lightofs = ofs;
    fb.lighting_bytes = total;
    st.ready = true;
    return VRAD_OK;
}

// A world with light styles above 0 first makes its style slots (they
// decide the layout): the call then gathers each such style once.
int32_t style_layout_now(vrad_ctx *ctx) {
    if (ctx->styles.styles.empty() || ctx->styles.ready) return VRAD_OK;
    if (!ctx->has_scene) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    if (!ctx->world.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no lighting world uploaded");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    return ensure_style_layout(ctx, ctx->stream);
}

// The light pass for `ranges` (VRAD_RANGE_*) on stream s: the direct
// gather (or, with ahead, the one queued at the world upload, its end
// marked by ctx->ahead_done), then per range, LDR first, its bounce (the
// first range builds the transfers, the second reuses them) and its final
// pass into d_out[range].  ev (nullable) marks the steps; bstats
// (nullable, two records) receives each range's bounce statistics.
int32_t pass_on(vrad_ctx *ctx, int32_t ranges, uint8_t *d_ldr, uint8_t *d_hdr, cudaStream_t s, PassEvents *ev,
                vrad_bounce_stats *bstats, bool ahead = false) {
    if (!ctx->has_scene) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    if (!ctx->world.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no lighting world uploaded");
    if (!ctx->final_pass.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without face windings");
    if ((ranges & VRAD_RANGE_HDR) && !ctx->sample_light_hdr)
        return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without an HDR light list");
    vrad::FinalBuffers &fb = ctx->final_pass;
    cudaError_t e = cudaSuccess;
    if (ev) e = cudaEventRecord(ev->start, s);
    if (e == cudaSuccess && ahead) {
        e = cudaStreamWaitEvent(s, ctx->ahead_done, 0);
        if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "joining the direct gather");
    } else if (e == cudaSuccess) {
        const int32_t rc = vrad::direct_pass(ctx, (ranges & VRAD_RANGE_LDR) ? ctx->sample_light : nullptr,
                                             (ranges & VRAD_RANGE_HDR) ? ctx->sample_light_hdr : nullptr, s);
        if (rc != VRAD_OK) return rc;
    }
    // Light styles above 0: each style's gather (both ranges in one
    // traversal) and its supersampling passes on the faces that hold it.
    vrad::StyleState &st = ctx->styles;
    if (!st.styles.empty() && !st.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "light style slots not made");
    for (size_t i = 0; i < st.styles.size() && e == cudaSuccess; i++) {
        vrad::DeviceWorld v = ctx->world.view;
        v.style = st.styles[i];
        v.face_slot = st.slots + i * (size_t)fb.nfaces;
        float4 *lo = (ranges & VRAD_RANGE_LDR) ? st.light[0][i] : nullptr;
        float4 *hi = (ranges & VRAD_RANGE_HDR) ? st.light[1][i] : nullptr;
        if (lo && hi)
            e = vrad::launch_direct(ctx->scene.view(), v, lo, hi, ctx->world.counters, ctx->status, s, ctx->world.block);
        else
            e = vrad::launch_direct(ctx->scene.view(), vrad::range_view(v, hi != nullptr), lo ? lo : hi, nullptr,
                                    ctx->world.counters, ctx->status, s, ctx->world.block);
        for (int r = 0; r < 2 && e == cudaSuccess; r++) {
            float4 *out = r == 0 ? lo : hi;
            if (!out) continue;
            vrad::SupersampleBuffers &ss = ctx->supersample;
            e = vrad::run_supersample(ss, ctx->scene.view(), vrad::range_view(v, r == 1), fb.view, out,
                                      ctx->world.counters, ctx->status, s);
            ctx->range_ss[r].supersampled += ss.supersampled;
            ctx->range_ss[r].ms += ss.ms;
        }
    }
    if (e == cudaSuccess && ev) e = cudaEventRecord(ev->direct, s);
    const bool bounce = vrad::bounce_active(ctx);
    bool built = false;
    for (int r = 0; r < 2; r++) std::memset(&ctx->range_bounce[r], 0, sizeof ctx->range_bounce[r]);
    for (int r = 0; r < 2 && e == cudaSuccess; r++) {
        if (bstats) std::memset(&bstats[r], 0, sizeof bstats[r]);
        if (!(ranges & (1 << r))) continue;
        const float4 *light = r == 0 ? ctx->sample_light : ctx->sample_light_hdr;
        uint8_t *out = r == 0 ? d_ldr : d_hdr;
        // The bounce (patch light, transfers, bounces), when one is uploaded.
        vrad::PatchRadialView prad{};
        if (bounce) {
            std::string why;
            e = vrad::run_bounce(ctx, s, light, !built && !ctx->bounce.installed, why);
            if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, why.c_str());
            built = true;
            prad = vrad::patch_radial_view(ctx);
            vrad::fill_bounce_stats(ctx, &ctx->range_bounce[r]);
            if (bstats) bstats[r] = ctx->range_bounce[r];
        }
        if (e == cudaSuccess && ev) e = cudaEventRecord(ev->bounce[r], s);
        if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, (size_t)fb.lighting_bytes, s);
        if (e == cudaSuccess)
            e = vrad::launch_final(fb.view, light, fb.rad_light, fb.rad_weight, fb.flat, out, fb.nfaces,
                                   bounce ? &prad : nullptr, s);
        // Each further style into its slots (the bounce goes into style 0's
        // alone).
        for (size_t i = 0; i < st.styles.size() && e == cudaSuccess; i++) {
            vrad::FinalView v = fb.view;
            v.style_slot = st.slots + i * (size_t)fb.nfaces;
            e = vrad::launch_final(v, st.light[r][i], fb.rad_light, fb.rad_weight, fb.flat, out, fb.nfaces, nullptr, s);
        }
        if (e == cudaSuccess && ev) e = cudaEventRecord(ev->final_[r], s);
    }
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "light pass launch");
    return VRAD_OK;
}

// The device-buffer pass: always gathers (the gather queued ahead is
// dropped).
int32_t pass_device(vrad_ctx *ctx, int32_t ranges, uint8_t *d_ldr, uint8_t *d_hdr, void *stream) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (ranges < 1 || ranges > 3) return vrad_fail(ctx, VRAD_ERR_ARG, "ranges %d is not LDR, HDR or both", ranges);
    for (int r = 0; r < 2; r++) {
        uint8_t *d = r == 0 ? d_ldr : d_hdr;
        if ((ranges & (1 << r)) && (!d || ((uintptr_t)d & 3)))
            return vrad_fail(ctx, VRAD_ERR_ARG, "lighting buffer null or not 4-byte aligned");
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    int32_t rc = style_layout_now(ctx);
    if (rc != VRAD_OK) return rc;
    rc = pass_on(ctx, ranges, d_ldr, d_hdr, (cudaStream_t)stream, nullptr, nullptr);
    e = vrad::join_stream(ctx, (cudaStream_t)stream);
    return rc != VRAD_OK || e == cudaSuccess ? rc : vrad_cuda_fail(ctx, e, "joining the caller's stream");
}

// The host-buffer pass: takes the gather queued ahead when it lit every
// range asked for.
int32_t pass_host(vrad_ctx *ctx, int32_t ranges, uint8_t *ldr, int64_t ldr_capacity, uint8_t *hdr,
                  int64_t hdr_capacity, int32_t *lightofs, vrad_pass_stats *stats, vrad_bounce_stats *bstats) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (ranges < 1 || ranges > 3) return vrad_fail(ctx, VRAD_ERR_ARG, "ranges %d is not LDR, HDR or both", ranges);
    std::lock_guard<std::mutex> g(ctx->mu);
    // The direct gather the world upload queued ahead, when there is one.
    const bool ahead = vrad::settle_direct(ctx) && (ctx->ahead_ranges & ranges) == ranges;
    vrad::FinalBuffers &fb = ctx->final_pass;
    if (!fb.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without face windings");
    const int32_t lrc = style_layout_now(ctx);
    if (lrc != VRAD_OK) return lrc;
    for (int r = 0; r < 2; r++) {
        if (!(ranges & (1 << r))) continue;
        const uint8_t *h = r == 0 ? ldr : hdr;
        const int64_t cap = r == 0 ? ldr_capacity : hdr_capacity;
        if (!h || cap < fb.lighting_bytes)
            return vrad_fail(ctx, VRAD_ERR_ARG, "the %s lump needs %lld bytes, %lld given",
                             r == 0 ? "LIGHTING" : "LIGHTING_HDR", (long long)fb.lighting_bytes, (long long)cap);
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->pass_stream ? ctx->pass_stream : ctx->stream;
    uint8_t *d_out[2] = {nullptr, nullptr};
    PassEvents ev;
    for (int r = 0; r < 2 && e == cudaSuccess; r++)
        if (ranges & (1 << r)) e = vrad::dev_alloc(&d_out[r], (size_t)(fb.lighting_bytes ? fb.lighting_bytes : 4));
    if (e == cudaSuccess) e = ev.create();
    int32_t rc = e == cudaSuccess ? pass_on(ctx, ranges, d_out[0], d_out[1], s, &ev, bstats, ahead)
                                  : vrad_cuda_fail(ctx, e, "light pass set-up");
    unsigned long long counts[2] = {0, 0};
    uint32_t overflow = 0;
    if (rc == VRAD_OK) {
        for (int r = 0; r < 2 && e == cudaSuccess; r++)
            if (ranges & (1 << r))
                e = cudaMemcpyAsync(r == 0 ? ldr : hdr, d_out[r], (size_t)fb.lighting_bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(counts, ctx->world.counters, sizeof counts, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&overflow, ctx->status, sizeof overflow, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = vrad::wait_stream(s);
        if (e != cudaSuccess) rc = vrad_cuda_fail(ctx, e, "light pass");
    }
    if (rc == VRAD_OK && overflow) {
        cudaMemsetAsync(ctx->status, 0, sizeof(uint32_t), s);
        rc = vrad_fail(ctx, VRAD_ERR_CUDA, "traversal stack overflow (BVH deeper than %d)", vrad::kStackDepth);
    }
    if (rc == VRAD_OK) {
        float final_ms[2] = {0.0f, 0.0f};
        for (int r = 0; r < 2; r++)
            if (ranges & (1 << r)) cudaEventElapsedTime(&final_ms[r], ev.bounce[r], ev.final_[r]);
        ctx->bounce.final_ms = (ranges & VRAD_RANGE_HDR) ? final_ms[1] : final_ms[0];
        for (int r = 0; r < 2; r++) {
            ctx->range_bounce[r].final_ms = final_ms[r];
            if (bstats) bstats[r].final_ms = final_ms[r];
        }
        if (lightofs)
            for (int32_t f = 0; f < fb.nfaces; f++) lightofs[f] = fb.lightofs[(size_t)f];
        if (stats) {
            float d_ms = 0.0f;
            // The gather's own device time, also when it ran ahead.
            if (ahead) cudaEventElapsedTime(&d_ms, ctx->ahead_start, ctx->ahead_done);
            else cudaEventElapsedTime(&d_ms, ev.start, ev.direct);
            std::memset(stats, 0, sizeof *stats);
            stats->samples = ctx->world.view.nsamples;
            stats->luxels = fb.view.ncells;
            stats->visibility_rays = (int64_t)counts[0];
            stats->sky_rays = (int64_t)counts[1];
            stats->lighting_bytes = fb.lighting_bytes;
            stats->direct_ms = d_ms;
            stats->final_ms = final_ms[0] + final_ms[1];
            for (int r = 0; r < 2; r++) {
                if (!(ranges & (1 << r))) continue;
                stats->extra_passes_run = std::max(stats->extra_passes_run, ctx->range_ss[r].passes_run);
                stats->supersampled += ctx->range_ss[r].supersampled;
                stats->supersample_ms += ctx->range_ss[r].ms;
            }
        }
    }
    if (rc != VRAD_OK) vrad::wait_stream(s);  // no kernel still writes the lumps
    if (s != ctx->stream) vrad::join_stream(ctx, s);
    vrad::dev_free(d_out[0]);
    vrad::dev_free(d_out[1]);
    return rc;
}

}  // namespace

extern "C" int32_t vrad_lighting_size(vrad_ctx *ctx, int64_t *bytes) {
    if (!ctx || !bytes) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->final_pass.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without face windings");
    const int32_t rc = style_layout_now(ctx);
    if (rc != VRAD_OK) return rc;
    *bytes = ctx->final_pass.lighting_bytes;
    return VRAD_OK;
}

extern "C" int32_t vrad_face_styles(vrad_ctx *ctx, uint8_t *styles, int32_t nfaces, int64_t *dropped) {
    if (!ctx || !styles) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::FinalBuffers &fb = ctx->final_pass;
    if (!fb.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without face windings");
    if (nfaces != fb.nfaces) return vrad_fail(ctx, VRAD_ERR_ARG, "%d faces, %d asked", fb.nfaces, nfaces);
    const int32_t rc = style_layout_now(ctx);
    if (rc != VRAD_OK) return rc;
    const vrad::StyleState &st = ctx->styles;
    for (int32_t f = 0; f < nfaces; f++)
        for (int k = 0; k < 4; k++)
            styles[4 * (int64_t)f + k] = st.styles.empty() ? (k == 0 ? 0 : 255) : st.face_styles[(size_t)f * 4 + k];
    if (dropped) *dropped = st.dropped;
    return VRAD_OK;
}

extern "C" int32_t vrad_light_pass_device(vrad_ctx *ctx, uint8_t *d_lighting, void *stream) {
    return pass_device(ctx, VRAD_RANGE_LDR, d_lighting, nullptr, stream);
}

extern "C" int32_t vrad_light_pass(vrad_ctx *ctx, uint8_t *lighting, int64_t capacity, int32_t *lightofs,
                                   vrad_pass_stats *stats) {
    return pass_host(ctx, VRAD_RANGE_LDR, lighting, capacity, nullptr, 0, lightofs, stats, nullptr);
}

extern "C" int32_t vrad_light_pass_ranges(vrad_ctx *ctx, int32_t ranges, uint8_t *ldr, int64_t ldr_capacity,
                                          uint8_t *hdr, int64_t hdr_capacity, int32_t *lightofs,
                                          vrad_pass_stats *stats, vrad_bounce_stats *bounce_stats) {
    return pass_host(ctx, ranges, ldr, ldr_capacity, hdr, hdr_capacity, lightofs, stats, bounce_stats);
}

extern "C" int32_t vrad_light_pass_ranges_device(vrad_ctx *ctx, int32_t ranges, uint8_t *d_ldr, uint8_t *d_hdr,
                                                 void *stream) {
    return pass_device(ctx, ranges, d_ldr, d_hdr, stream);
}

extern "C" int32_t vrad_pass_sample_light(vrad_ctx *ctx, int32_t range, vrad_lighting_value *out, int64_t n) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (range != VRAD_RANGE_LDR && range != VRAD_RANGE_HDR) return vrad_fail(ctx, VRAD_ERR_ARG, "range %d", range);
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    const float4 *src = range == VRAD_RANGE_LDR ? ctx->sample_light : ctx->sample_light_hdr;
    if (!ctx->world.ready || !src) return vrad_fail(ctx, VRAD_ERR_ARG, "no light pass of that range");
    if (!out || n != ctx->world.view.nsamples)
        return vrad_fail(ctx, VRAD_ERR_ARG, "%lld samples, %lld asked", (long long)ctx->world.view.nsamples, (long long)n);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = vrad::quiesce(ctx);
    if (e == cudaSuccess && n) e = cudaMemcpy(out, src, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? VRAD_OK : vrad_cuda_fail(ctx, e, "sample light");
}

extern "C" int32_t vrad_bounce_stats_ranges(vrad_ctx *ctx, vrad_bounce_stats *stats) {
    if (!ctx || !stats) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    stats[0] = ctx->range_bounce[0];
    stats[1] = ctx->range_bounce[1];
    return VRAD_OK;
}
