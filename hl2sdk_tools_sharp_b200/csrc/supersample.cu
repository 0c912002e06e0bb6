// supersample.cu -- the direct gather's supersampling passes: luxels whose
// light differs sharply from a neighbour's are gathered again at 4x4 points
// (the lights) and 2x2 points (the sky ambient) across their cell, and the
// averages replace their light.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad/Light):
//   FaceLightJob.AdvanceAfterRound / StartRound (FaceLightJob.cs:553-740):
//       passes 1 .. ExtraPasses (4) while a pass selects anything;
//   StyleSupersample.ComputeLuxelIntensity / SelectForPass / ComputeGradients
//       (FaceLightJob.cs:1062-1180): intensity = PowToSingle(I / 256, 1 / 2.2),
//       gradient = max |difference| to the 8 neighbouring cells that have a
//       sample, selected when not below 0.0625 and not selected before;
//   FaceLightJob.EmitSupersamplePoint / ResolveSupersampleItem /
//       ResolveSupersamplePoint / PointsInWinding (FaceLightJob.cs:741-930):
//       the point grids, the partial cell's winding test per row of four,
//       the sky ambient and the other lights gathered apart, the valid
//       lanes summed in order and averaged with AddWeighted;
//   FaceSampleBuilder.MakeSample (FaceSampleBuilder.cs:325-367): which
//       samples keep a winding.
// with the reference's defaults (style 0, flat faces, no -debugextra, the
// zero-initialised gradient scratch).  A selected sample's light depends
// on nothing else selected in its pass, so the pass runs every selected
// sample at once; passes run in order.
//
// Kernels of one pass: k_ss_select (the gradients and the selection),
// k_ss_place (each selected sample's five rows into its cluster's runs),
// k_resample (one thread per point, the shared gather), k_ss_resolve (the
// averages and the new intensities).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "device_pool.h"
#include "gather.cuh"
#include "host_parallel.h"
#include "setup_clock.h"
#include "supersample.cuh"
#include "world.h"
#include "sync_wait.h"

namespace vrad {

namespace {

constexpr int kSsBlock = 128;
constexpr float kSupersampleGradient = 0.0625f;  // LightConstants.SupersampleGradient

// DetMath.PowToSingle: x^y rounded to double, then to float.  CUDA's pow
// is within a few units of the last double place, so its double rounds to
// the reference's float unless it lies next to a midpoint between two
// floats; such a case keeps the plain rounding and is counted in *open.
__device__ __forceinline__ float pow_to_single(double x, double y, unsigned long long *open) {
    const double r = pow(x, y);
    const float f = __double2float_rn(r);
    if (!isfinite(r) || r == 0.0 || (double)f == r) return f;
    const double ar = fabs(r);
    const float af = fabsf(f);
    const float g = ar > (double)af ? nextafterf(af, INFINITY) : nextafterf(af, 0.0f);
    const double mid = __dmul_rn(__dadd_rn((double)af, (double)g), 0.5);
    if (fabs(__dsub_rn(ar, mid)) > 8.0 * ldexp(1.0, ilogb(ar) - 52)) return f;
    atomicAdd(open, 1ull);
    return f;
}

// ComputeLuxelIntensity: the light's sum, over 256, to the power 1/2.2.
__device__ __forceinline__ float luxel_intensity(const float4 &v, unsigned long long *open) {
    const float i = __fadd_rn(__fadd_rn(v.x, v.y), v.z);
    return pow_to_single(__ddiv_rn((double)i, 256.0), 1.0 / 2.2, open);
}

__global__ void k_ss_intensity(int64_t n, const float4 *__restrict__ light, float *__restrict__ intensity,
                               uint8_t *__restrict__ processed, unsigned long long *open) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    intensity[i] = luxel_intensity(light[i], open);
    processed[i] = 0;
}

// SelectForPass: each sample not yet supersampled whose gradient over its
// eight neighbouring cells reaches the threshold.
__global__ void k_ss_select(int64_t n, FinalView fv, DeviceWorld w, const int32_t *__restrict__ cell,
                            const float *__restrict__ intensity, uint8_t *__restrict__ processed,
                            int32_t *__restrict__ selected, int32_t *__restrict__ counts) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || processed[i]) return;
    const int c = __ldg(&cell[i]);
    const int f = __ldg(&fv.cell_face[c]);
    // A style that is not this face's has no supersampling state here.
    if (w.face_slot && __ldg(&w.face_slot[f]) < 0) return;
    const int base = __ldg(&fv.face_cells[f]);
    const int wd = __float_as_int(__ldg(&fv.frames[5 * f].w)), ht = __float_as_int(__ldg(&fv.frames[5 * f + 1].w));
    const int s = (c - base) % wd, t = (c - base) / wd;
    const float cv = intensity[i];
    float g = 0.0f;
    // Step: a neighbour cell without a sample is passed over.
    auto step = [&](int cc) {
        const int k = __ldg(&fv.cell_sample[cc]);
        if (k < 0) return;
        const float d = fabsf(__fsub_rn(cv, intensity[k]));
        g = g > d ? g : d;
    };
    if (t > 0) {
        if (s > 0) step(c - 1 - wd);
        step(c - wd);
        if (s < wd - 1) step(c + 1 - wd);
    }
    if (t < ht - 1) {
        if (s > 0) step(c - 1 + wd);
        step(c + wd);
        if (s < wd - 1) step(c + 1 + wd);
    }
    if (s > 0) step(c - 1);
    if (s < wd - 1) step(c + 1);
    if (g < kSupersampleGradient) return;
    processed[i] = 1;
    const int k = atomicAdd(&counts[0], 1);
    selected[k] = (int32_t)i;
    const int face = __float_as_int(__ldg(&w.sample_pos[i].w));
    atomicAdd(&counts[1 + __float_as_int(__ldg(&w.face_normal[face].w))], 1);
}

// Each selected sample's ambient row and four direct rows into its
// cluster's runs (base[2c] ambient, base[2c + 1] direct).  The slot order
// inside a run is immaterial: every row writes its own output.
__global__ void k_ss_place(int32_t nsel, DeviceWorld w, const int32_t *__restrict__ selected,
                           const int32_t *__restrict__ base, int32_t *__restrict__ cursor, int32_t *__restrict__ rows) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsel) return;
    const int i = selected[k];
    const int face = __float_as_int(__ldg(&w.sample_pos[i].w));
    const int c = __float_as_int(__ldg(&w.face_normal[face].w));
    const int pos = atomicAdd(&cursor[c], 1);
    rows[base[2 * c] + pos] = 5 * k;
    for (int r = 0; r < 4; r++) rows[base[2 * c + 1] + 4 * pos + r] = 5 * k + 1 + r;
}

// PointsInWinding for one point: whether an edge of the cell winding has it
// on the other side from the first edge.
__device__ bool point_outside(float x, float y, float z, const float4 *__restrict__ pts, int n) {
    auto sub = [](float4 a, float4 b, float &dx, float &dy, float &dz) {
        dx = __fsub_rn(a.x, b.x);
        dy = __fsub_rn(a.y, b.y);
        dz = __fsub_rn(a.z, b.z);
    };
    auto unit_cross = [](float ax, float ay, float az, float bx, float by, float bz, float &cx, float &cy, float &cz) {
        cx = __fsub_rn(__fmul_rn(ay, bz), __fmul_rn(az, by));
        cy = __fsub_rn(__fmul_rn(az, bx), __fmul_rn(ax, bz));
        cz = __fsub_rn(__fmul_rn(ax, by), __fmul_rn(ay, bx));
        const float l = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz)));
        if (l == 0.0f) {
            cx = cy = cz = 0.0f;
        } else {
            cx = __fdiv_rn(cx, l);
            cy = __fdiv_rn(cy, l);
            cz = __fdiv_rn(cz, l);
        }
    };
    const float4 p = make_float4(x, y, z, 0.0f);
    const float4 w0 = __ldg(&pts[0]), w1 = __ldg(&pts[1 % n]);
    float ex, ey, ez, tx, ty, tz, ux, uy, uz;
    sub(w1, w0, ex, ey, ez);
    sub(p, w0, tx, ty, tz);
    unit_cross(ex, ey, ez, tx, ty, tz, ux, uy, uz);
    bool invalid = false;
    for (int k = 1; k < n; k++) {
        const float4 p0 = __ldg(&pts[k]), p1 = __ldg(&pts[(k + 1) % n]);
        float cx, cy, cz;
        sub(p1, p0, ex, ey, ez);
        sub(p, p0, tx, ty, tz);
        unit_cross(ex, ey, ez, tx, ty, tz, cx, cy, cz);
        const float d = __fadd_rn(__fadd_rn(__fmul_rn(cx, ux), __fmul_rn(cy, uy)), __fmul_rn(cz, uz));
        invalid |= d < 0.0f;
    }
    return invalid;
}

// One point of a supersampled row: its position in the cell, the winding
// test of its row of four, the gather (the sky ambient for row 0, the other
// lights for rows 1-4) and its LightingValue.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_resample(DeviceScene sc, DeviceWorld w, FinalView fv, int32_t ngroups,
                                                    int32_t nruns, const int32_t *__restrict__ base,
                                                    const int32_t *__restrict__ rows,
                                                    const int32_t *__restrict__ selected,
                                                    const float2 *__restrict__ origin_st, const int2 *__restrict__ wind,
                                                    const float4 *__restrict__ points, float4 *__restrict__ row_out,
                                                    int32_t *__restrict__ row_bits, unsigned long long *counters,
                                                    uint32_t *overflow) {
    extern __shared__ int stack_mem[];  // sc.stack_depth() entries per thread
    int *stack = stack_mem + threadIdx.x;
    const int64_t tid = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
    const int g = (int)(tid >> 2), l4 = (int)(tid & 3);
    // Runs hold whole warps, so a warp returns whole.
    if (g >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const unsigned gmask = 0xFu << (lane & ~3);
    int run = 0;
    {
        int lo = 0, hi = nruns;  // largest run with base[run] <= g
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(&base[mid]) <= g) lo = mid;
            else hi = mid;
        }
        run = lo;
    }
    const int cluster = run >> 1;
    const bool ambient = (run & 1) == 0;
    const int code = __ldg(&rows[g]);
    float px = 0.0f, py = 0.0f, pz = 0.0f, nx = 0.0f, ny = 0.0f, nz = 1.0f;
    bool real = false, invalid = true;
    if (code >= 0) {
        const int k = code / 5, row = code % 5;
        const int i = __ldg(&selected[k]);
        const int face = __float_as_int(__ldg(&w.sample_pos[i].w));
        const float4 fn = __ldg(&w.face_normal[face]);
        nx = fn.x, ny = fn.y, nz = fn.z;
        const float4 o = __ldg(&fv.frames[5 * face]), ls = __ldg(&fv.frames[5 * face + 3]),
                     lt = __ldg(&fv.frames[5 * face + 4]);
        const int mins = __float_as_int(__ldg(&fv.frames[5 * face + 2].w)), mint = __float_as_int(ls.w);
        const float2 st = __ldg(&origin_st[i]);
        // EmitSupersamplePoint's grids: 2x2 at +-1/4 (ambient), 4x4 at
        // -3/8, -1/8, 1/8, 3/8 (direct), rows along s.
        float cs, ct;
        if (row == 0) {
            cs = __fadd_rn(st.x, l4 < 2 ? -0.25f : 0.25f);
            ct = __fadd_rn(st.y, (l4 & 1) == 0 ? -0.25f : 0.25f);
        } else {
            const float a[4] = {-0.375f, -0.125f, 0.125f, 0.375f};
            cs = __fadd_rn(st.x, a[row - 1]);
            ct = __fadd_rn(st.y, a[l4]);
        }
        // LuxelToWorld.
        const float ss = __fadd_rn(cs, (float)mins), tt = __fadd_rn(ct, (float)mint);
        const float x = __fadd_rn(__fadd_rn(o.x, __fmul_rn(ls.x, ss)), __fmul_rn(lt.x, tt));
        const float y = __fadd_rn(__fadd_rn(o.y, __fmul_rn(ls.y, ss)), __fmul_rn(lt.y, tt));
        const float z = __fadd_rn(__fadd_rn(o.z, __fmul_rn(ls.z, ss)), __fmul_rn(lt.z, tt));
        const int2 wn = __ldg(&wind[i]);
        invalid = wn.y > 0 ? point_outside(x, y, z, points + wn.x, wn.y) : false;
        // One unit off the face.
        px = __fadd_rn(x, nx);
        py = __fadd_rn(y, ny);
        pz = __fadd_rn(z, nz);
    }
    unsigned bits = invalid ? 1u << l4 : 0u;
    bits |= __shfl_xor_sync(gmask, bits, 1);
    bits |= __shfl_xor_sync(gmask, bits, 2);
    // A row whose four points all lie outside is not gathered.
    real = code >= 0 && bits != 0xFu;
    unsigned long long vis_rays = 0, sky_rays = 0;
    const float4 r = gather_point<BLOCK>(sc, w, cluster, px, py, pz, nx, ny, nz, real, gmask,
                                         ambient ? kAmbientOnly : kDirectOnly, stack, overflow, counters, vis_rays,
                                         sky_rays);
    if (code >= 0) {
        row_out[4 * (int64_t)code + l4] = r;
        if (l4 == 0) row_bits[code] = real ? (int32_t)bits : -1;
    }
    __syncwarp();
    for (int o = 16; o > 0; o >>= 1) {
        vis_rays += __shfl_xor_sync(kFull, vis_rays, o);
        sky_rays += __shfl_xor_sync(kFull, sky_rays, o);
    }
    if (lane == 0) {
        atomicAdd(&counters[0], vis_rays);
        atomicAdd(&counters[1], sky_rays);
    }
}

// ResolveSupersampleItem: the valid points of each grid summed in order,
// and, when both grids have one, the sample's light replaced by the direct
// average plus the ambient average; then its intensity.
__global__ void k_ss_resolve(int32_t nsel, const int32_t *__restrict__ selected, const float4 *__restrict__ row_out,
                             const int32_t *__restrict__ row_bits, float4 *__restrict__ light,
                             float *__restrict__ intensity, unsigned long long *open) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsel) return;
    float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), d = a;
    int ac = 0, dc = 0;
    for (int r = 0; r < 5; r++) {
        const int bits = row_bits[5 * k + r];
        if (bits == -1) continue;
        for (int l = 0; l < 4; l++) {
            if ((bits >> l) & 1) continue;
            const float4 v = row_out[4 * (5 * (int64_t)k + r) + l];
            float4 &acc = r == 0 ? a : d;
            acc = make_float4(__fadd_rn(acc.x, v.x), __fadd_rn(acc.y, v.y), __fadd_rn(acc.z, v.z),
                              __fadd_rn(acc.w, v.w));
            (r == 0 ? ac : dc)++;
        }
    }
    if (ac == 0 || dc == 0) return;
    const int i = selected[k];
    const float wd = __fdiv_rn(1.0f, (float)dc), wa = __fdiv_rn(1.0f, (float)ac);
    float4 v;
    v.x = __fadd_rn(0.0f, __fmul_rn(wd, d.x));
    v.y = __fadd_rn(0.0f, __fmul_rn(wd, d.y));
    v.z = __fadd_rn(0.0f, __fmul_rn(wd, d.z));
    v.w = __fadd_rn(0.0f, __fmul_rn(wd, d.w));
    v.x = __fadd_rn(v.x, __fmul_rn(wa, a.x));
    v.y = __fadd_rn(v.y, __fmul_rn(wa, a.y));
    v.z = __fadd_rn(v.z, __fmul_rn(wa, a.z));
    v.w = __fadd_rn(v.w, __fmul_rn(wa, a.w));
    light[i] = v;
    intensity[i] = luxel_intensity(v, open);
}

unsigned grid_of(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

void SupersampleBuffers::release() {
    void *ptrs[] = {origin_st, cell, wind, points, intensity, processed, selected, counts, base, rows, row_out, row_bits};
    for (void *p : ptrs) dev_free(p);
    // The pinned counts stay for the next upload (freeing pinned memory
    // can stall for a good part of a second); free_pinned() frees them.
    const int32_t keep = extra_passes;
    int32_t *pinned = h_counts;
    const size_t cap = h_counts_cap;
    *this = SupersampleBuffers();
    extra_passes = keep;
    h_counts = pinned;
    h_counts_cap = cap;
}

void SupersampleBuffers::free_pinned() {
    cudaFreeHost(h_counts);
    h_counts = nullptr;
    h_counts_cap = 0;
}

cudaError_t build_supersample(SupersampleBuffers &ss, const std::vector<vrad_face> &faces,
                              const std::vector<float> &vertices, const float4 *area_coord, int64_t nsamples,
                              const FinalBuffers &fb, int32_t nclusters, Stager &stager, cudaStream_t stream,
                              bool &have, std::string &why) {
    ss.release();
    have = false;
    SetupClock clock("supersample_tables");
    // The faces' row strips on the host, their cells on the device, which
    // checks that the world's samples are the builder's own.
    RowStrips rs;
    if (!face_row_strips(faces.data(), (int32_t)faces.size(), vertices.data(), (int64_t)vertices.size() / 3, rs, why))
        return cudaSuccess;
    clock.mark("row strips");
    bool match = false;
    cudaError_t e = device_windings(ss, rs, fb.view, area_coord, nsamples, stager, stream, match, why);
    if (e != cudaSuccess || !match) {
        ss.release();
        if (e != cudaSuccess) why = "supersampling windings";
        return e;
    }
    clock.mark("windings");
    const size_t S = (size_t)nsamples;
    const size_t S1 = S ? S : 1;
    const size_t groups = 5 * S1 + 16 * (size_t)(nclusters + 1);
    e = dev_alloc(&ss.intensity, sizeof(float) * S1);
    if (e == cudaSuccess) e = dev_alloc(&ss.processed, S1);
    if (e == cudaSuccess) e = dev_alloc(&ss.selected, sizeof(int32_t) * S1);
    if (e == cudaSuccess) e = dev_alloc(&ss.counts, sizeof(int32_t) * (1 + 2 * (size_t)nclusters));
    if (e == cudaSuccess) e = dev_alloc(&ss.base, sizeof(int32_t) * (2 * (size_t)nclusters + 1));
    if (e == cudaSuccess) e = dev_alloc(&ss.rows, sizeof(int32_t) * groups);
    if (e == cudaSuccess) e = dev_alloc(&ss.row_out, sizeof(float4) * 20 * S1);
    if (e == cudaSuccess) e = dev_alloc(&ss.row_bits, sizeof(int32_t) * 5 * S1);
    if (e == cudaSuccess && ss.h_counts_cap < 1 + (size_t)nclusters) {
        ss.free_pinned();
        e = cudaMallocHost(&ss.h_counts, sizeof(int32_t) * (1 + (size_t)nclusters));
        if (e == cudaSuccess) ss.h_counts_cap = 1 + (size_t)nclusters;
    }
    if (e != cudaSuccess) {
        ss.release();
        why = "supersampling buffers";
        return e;
    }
    clock.mark("buffers");
    ss.nsamples = (int64_t)S;
    ss.nclusters = nclusters;
    ss.ready = true;
    have = true;
    return cudaSuccess;
}

cudaError_t run_supersample(SupersampleBuffers &ss, const DeviceScene &scene, const DeviceWorld &world,
                            const FinalView &fv, float4 *light, unsigned long long *counters, uint32_t *overflow,
                            cudaStream_t s) {
    ss.supersampled = 0;
    ss.passes_run = 0;
    ss.ms = 0.0f;
    if (!ss.ready || ss.extra_passes <= 0 || ss.nsamples == 0) return cudaSuccess;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaEventRecord(a, s);
    const int64_t S = ss.nsamples;
    const int32_t C = ss.nclusters;
    if (e == cudaSuccess) k_ss_intensity<<<grid_of(S, 256), 256, 0, s>>>(S, light, ss.intensity, ss.processed, &counters[2]);
    std::vector<int32_t> base((size_t)2 * C + 1);
    for (int pass = 1; e == cudaSuccess && pass <= ss.extra_passes; pass++) {
        e = cudaMemsetAsync(ss.counts, 0, sizeof(int32_t) * (1 + 2 * (size_t)C), s);
        if (e == cudaSuccess)
            k_ss_select<<<grid_of(S, 256), 256, 0, s>>>(S, fv, world, ss.cell, ss.intensity, ss.processed,
                                                       ss.selected, ss.counts);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ss.h_counts, ss.counts, sizeof(int32_t) * (1 + (size_t)C), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = vrad::wait_stream(s);
        if (e != cudaSuccess) break;
        const int32_t nsel = ss.h_counts[0];
        if (nsel == 0) break;
        // Each cluster's ambient run, then its direct run, each padded to
        // whole warps (eight groups of four).
        int32_t g = 0;
        for (int32_t c = 0; c < C; c++) {
            const int32_t n = ss.h_counts[1 + c];
            base[(size_t)2 * c] = g;
            g += (n + 7) / 8 * 8;
            base[(size_t)2 * c + 1] = g;
            g += (4 * n + 7) / 8 * 8;
        }
        base[(size_t)2 * C] = g;
        e = cudaMemcpyAsync(ss.base, base.data(), sizeof(int32_t) * base.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(ss.rows, 0xFF, sizeof(int32_t) * (size_t)g, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(ss.counts + 1 + C, 0, sizeof(int32_t) * (size_t)C, s);
        if (e == cudaSuccess)
            k_ss_place<<<grid_of(nsel, 256), 256, 0, s>>>(nsel, world, ss.selected, ss.base, ss.counts + 1 + C, ss.rows);
        if (e == cudaSuccess && g > 0)
            k_resample<kSsBlock><<<grid_of(4 * (int64_t)g, kSsBlock), kSsBlock,
                                  sizeof(int) * scene.stack_depth() * kSsBlock, s>>>(
                scene, world, fv, g, 2 * C + 1, ss.base, ss.rows, ss.selected, ss.origin_st, ss.wind, ss.points,
                ss.row_out, ss.row_bits, counters, overflow);
        if (e == cudaSuccess)
            k_ss_resolve<<<grid_of(nsel, 256), 256, 0, s>>>(nsel, ss.selected, ss.row_out, ss.row_bits, light,
                                                           ss.intensity, &counters[2]);
        if (e == cudaSuccess) e = cudaGetLastError();
        // The base table is read by this pass's kernels before the next
        // pass rewrites it.
        if (e == cudaSuccess) e = vrad::wait_stream(s);
        ss.supersampled += nsel;
        ss.passes_run = pass;
    }
    if (e == cudaSuccess) e = cudaEventRecord(b, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e == cudaSuccess) cudaEventElapsedTime(&ss.ms, a, b);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    return e;
}

}  // namespace vrad
