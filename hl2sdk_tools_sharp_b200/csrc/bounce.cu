// bounce.cu -- the radiosity bounce: the patches' direct light, the
// transfers (candidate pairs, their rays and form factors), the bounces,
// and the tables the final pass reads the bounced light through.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad):
//   PatchLighting.BuildPatchLights / AddSampleToPatch  Light/PatchLighting.cs:65-249
//   Radiosity.MoveDirectLightToEmission / GatherLight /
//             CollectLight / BounceAsync               Bounce/Radiosity.cs:132-316
//   VisMatrix.ReceiverOrder / FacesInRow / Enumerator.Run /
//             TestPatchToFace / TestPatchToPatch /
//             TransferRay / MakeTransfers / MakeTransfer /
//             MakeScales                               Bounce/VisMatrix.cs:180-1004
//   FormFactors.DiffToDiff / PolyToDiff                Bounce/FormFactors.cs:58-140
//   DetMathF.Asin (correctly rounded)                  MapFormats/Numerics/DetMathF.cs:141-164
//   FinalLightFace.BuildPatchRadial / AddFacePatches /
//             PatchLightmapCoordRange                  Final/FinalLightFace.cs:393-540
// with the reference's default settings: no compliance quirks (the
// receiver's plane normal in the plane test, true divides in the transfer
// rays, sines above one clamped), the exact normalise, bounces > 0.
//
// Every float operation of those routines is an explicitly rounded
// intrinsic, in the reference's association order, and every sum runs in
// the reference's order, so the transfers, the patch light and the stop
// decision are the reference's bits.
//
// Kernels of one light pass (after the direct gather):
//   k_patch_samples   one thread per patch: the face's samples that overlap
//                     it, in sample order (AddSampleToPatch)
//   k_patch_tree      one thread per face: pushes, averages and area blends
//                     over the face's patch list, then the move to emission
//   k_candidates      one thread per receiver: the candidate sources in the
//                     enumerator's order (a counting and a writing launch)
//   k_transfer        one thread per candidate: the transfer ray, traced
//                     in-thread, and MakeTransfer for an open pair
//   k_transfer_count / k_transfer_write  one warp per receiver: the
//                     accepted pairs compacted in order, capped at
//                     MaxPatches, and MakeScales' ordered sum
//   k_sell_*          the transfer lists copied into slices of 32 receivers
//                     sorted by count (SELL-32), once per pass
//   k_gather          one thread per receiver (in count order): GatherLight's
//                     ordered sum from its slice lane, then CollectLight's
//                     leaf update
//   k_collect_level   one thread per parent of one tree level: CollectLight's
//                     parents, one launch per level, bottom up
//   k_totals          fp64 sums of the light a bounce added, with absolute
//                     sums that bound the reference's float sum
//   k_exact_total     one block: the reference's sequential float sum, run
//                     only when the bound cannot settle the stop rule

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bounce.cuh"
#include "device_pool.h"
#include "context.cuh"
#include "detmath.cuh"
#include "mlp.cuh"
#include "patches.h"
#include "traverse.cuh"
#include "world.h"

namespace vrad {

namespace {

constexpr int kBounceBlock = 128;
constexpr int kEnumStack = 64;  // patch tree depth the candidate walk holds

// ---- float and double-double helpers ----------------------------------------

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(const float4 &a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ F3 add3(F3 a, F3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 mul3(F3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
// Vec3.Normalise: exact length, three true divides, zero for zero.
__device__ __forceinline__ F3 normalise3(F3 a, float &len) {
    len = __fsqrt_rn(dot3(a, a));
    if (len == 0.0f) return {0.0f, 0.0f, 0.0f};
    return {__fdiv_rn(a.x, len), __fdiv_rn(a.y, len), __fdiv_rn(a.z, len)};
}

// ---- the patches' direct light ----------------------------------------------

// AddSampleToPatch for one patch over its face's samples, in sample order:
// acc = (sample light * area summed, sample area summed).
__global__ void k_patch_samples(BounceView v, const float4 *__restrict__ sample_light, float4 *__restrict__ acc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= v.npatches) return;
    const int4 tr = __ldg(&v.tree[p]);
    float lx = 0.0f, ly = 0.0f, lz = 0.0f, area = 0.0f;
    if (tr.y == -1 && tr.w == 0) {
        const float4 mn = __ldg(&v.mins[p]), mx = __ldg(&v.maxs[p]);
        const int f = __float_as_int(mn.w);
        const int2 fs = __ldg(&v.face_samples[f]);
        for (int k = fs.x; k < fs.x + fs.y; k++) {
            const float4 L = __ldg(&sample_light[k]);
            // VectorAvg: a float divide by 3.
            if (__fdiv_rn(__fadd_rn(__fadd_rn(L.x, L.y), L.z), 3.0f) < 1.0f) continue;
            const float a = __ldg(&v.sample_area[k]);
            const float4 P = __ldg(&v.sample_pos[k]);
            const float radius = (float)__ddiv_rn((double)__fsqrt_rn(a), 2.0);
            if (mn.x > __fadd_rn(P.x, radius) || mx.x < __fsub_rn(P.x, radius)) continue;
            if (mn.y > __fadd_rn(P.y, radius) || mx.y < __fsub_rn(P.y, radius)) continue;
            if (mn.z > __fadd_rn(P.z, radius) || mx.z < __fsub_rn(P.z, radius)) continue;
            area = __fadd_rn(area, a);
            lx = __fadd_rn(lx, __fmul_rn(a, L.x));
            ly = __fadd_rn(ly, __fmul_rn(a, L.y));
            lz = __fadd_rn(lz, __fmul_rn(a, L.z));
        }
    }
    acc[p] = make_float4(lx, ly, lz, area);
}

// The face's patch list (FacePatches after RebuildFaceLists): its
// descendants in descending index order, then its root.
struct FaceList {
    int root, first, end;
    __device__ __forceinline__ int count() const { return root < 0 ? 0 : end - first + 1; }
    __device__ __forceinline__ int at(int k) const { return k < end - first ? end - 1 - k : root; }
};

// BuildPatchLights after the samples (pushes to parents, averages, area
// blends), then MoveDirectLightToEmission for the face's patches.
__global__ void k_patch_tree(BounceView v, float4 *__restrict__ acc, float4 *__restrict__ direct,
                             float4 *__restrict__ total, float4 *__restrict__ emit, float4 *__restrict__ shoot) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= v.nfaces) return;
    const int4 fr = __ldg(&v.face_range[f]);
    const FaceList L{fr.x, fr.y, fr.z};
    const int n = L.count();
    for (int k = 0; k < n; k++) {
        const int p = L.at(k);
        const int parent = __ldg(&v.tree[p].x);
        if (parent == -1) continue;
        const float4 a = acc[p], b = acc[parent];
        acc[parent] = make_float4(__fadd_rn(b.x, a.x), __fadd_rn(b.y, a.y), __fadd_rn(b.z, a.z), __fadd_rn(b.w, a.w));
    }
    for (int k = 0; k < n; k++) {
        const int p = L.at(k);
        const float4 a = acc[p];
        float4 t = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (a.w != 0.0f) {
            const float scale = (float)__drcp_rn((double)a.w);
            t = make_float4(__fadd_rn(0.0f, __fmul_rn(a.x, scale)), __fadd_rn(0.0f, __fmul_rn(a.y, scale)),
                            __fadd_rn(0.0f, __fmul_rn(a.z, scale)), 0.0f);
        }
        total[p] = t;
        direct[p] = t;
    }
    for (int k = 0; k < n; k++) {
        const int p = L.at(k);
        const int4 tr = __ldg(&v.tree[p]);
        if (tr.y == -1) continue;
        const float a1 = __ldg(&v.origin[tr.y].w), a2 = __ldg(&v.origin[tr.z].w);
        const float s1 = __fdiv_rn(a1, __fadd_rn(a1, a2)), s2 = __fdiv_rn(a2, __fadd_rn(a1, a2));
        const float4 c1 = total[tr.y], c2 = total[tr.z];
        const float4 t = make_float4(__fadd_rn(__fmul_rn(c1.x, s1), __fmul_rn(c2.x, s2)),
                                     __fadd_rn(__fmul_rn(c1.y, s1), __fmul_rn(c2.y, s2)),
                                     __fadd_rn(__fmul_rn(c1.z, s1), __fmul_rn(c2.z, s2)), 0.0f);
        total[p] = t;
        direct[p] = t;
    }
    for (int k = 0; k < n; k++) {
        const int p = L.at(k);
        const float4 e = total[p], r = __ldg(&v.refl[p]);
        emit[p] = e;
        shoot[p] = make_float4(__fmul_rn(e.x, r.x), __fmul_rn(e.y, r.y), __fmul_rn(e.z, r.z), 0.0f);
        total[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// ---- transfers ---------------------------------------------------------------

// Enumerator.Run for one receiver: the faces of its cluster's PVS row
// other than its own, each tested with TestPatchToFace, then its patch
// tree walked as TestPatchToPatch recurses (child1's subtree before
// child2's).  Counts (out == nullptr) or writes the candidates.
__global__ void k_candidates(BounceView v, const int64_t *__restrict__ cand_off, int64_t *__restrict__ counts,
                             int32_t *__restrict__ out, uint32_t *__restrict__ overflow) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= v.nreceivers) return;
    const int p = __ldg(&v.recv[r]);
    const F3 o = f3(__ldg(&v.origin[p]));
    const float4 mn = __ldg(&v.mins[p]), mx = __ldg(&v.maxs[p]);
    const int face = __float_as_int(mn.w), cluster = __float_as_int(mx.w);
    const float4 pl = __ldg(&v.face_plane[face]);
    const F3 me_n = {pl.x, pl.y, pl.z};
    const double me_d = (double)__ldg(&v.normal[p].w) + 0.01;
    int64_t n = 0;
    int64_t at = out ? cand_off[r] : 0;
    int stack[kEnumStack];
    const int q0 = __ldg(&v.row_off[cluster]), q1 = __ldg(&v.row_off[cluster + 1]);
    for (int q = q0; q < q1; q++) {
        const int g = __ldg(&v.row_faces[q]);
        if (g == face) continue;
        const int root = __ldg(&v.face_range[g].x);
        if (root < 0) continue;
        const float4 rn = __ldg(&v.normal[root]);
        if (!((double)dot3(o, f3(rn)) > (double)rn.w + 0.01)) continue;
        int sp = 0;
        stack[sp++] = root;
        while (sp > 0) {
            const int s = stack[--sp];
            const int4 tr = __ldg(&v.tree[s]);
            const float4 so = __ldg(&v.origin[s]);
            if (tr.y != -1) {
                const F3 d = sub3(o, f3(so));
                if ((double)dot3(d, d) * 0.0625 < (double)so.w) {
                    if (sp + 2 > kEnumStack) {
                        atomicOr(overflow, 2u);
                        continue;
                    }
                    stack[sp++] = tr.z;
                    stack[sp++] = tr.y;
                    continue;
                }
            }
            if ((double)dot3(f3(so), me_n) > me_d) {
                if (out) out[at] = s;
                at++;
                n++;
            }
        }
    }
    if (!out) counts[r] = n;
}

// FormFactors.DiffToDiff(o1, n1, o2, n2): delta = normalise(o1 - o2), then
// -(delta . n1) * (delta . n2) / (len * len).
__device__ __forceinline__ float diff_to_diff(F3 o1, F3 n1, F3 o2, F3 n2) {
    float dl;
    const F3 d = normalise3(sub3(o1, o2), dl);
    return __fdiv_rn(__fmul_rn(-dot3(d, n1), dot3(d, n2)), __fmul_rn(dl, dl));
}

// FormFactors.PolyToDiff of a winding of `count` points seen from (o, n).
__device__ float poly_to_diff_pts(const float4 *__restrict__ pts, int count, float area, F3 o, F3 n,
                                  unsigned long long *open) {
    float ff = 0.0f;
    for (int k = 0; k < count; k++) {
        const int k2 = k < count - 1 ? k + 1 : 0;
        float l;
        const F3 v1 = normalise3(sub3(f3(__ldg(&pts[k])), o), l);
        const F3 v2 = normalise3(sub3(f3(__ldg(&pts[k2])), o), l);
        float sin_alpha;
        F3 gamma = normalise3(cross3(v1, v2), sin_alpha);
        if (sin_alpha < -1.0f || sin_alpha > 1.0f) sin_alpha = sin_alpha > 1.0f ? 1.0f : -1.0f;
        gamma = mul3(gamma, asin_cr(sin_alpha, open));
        ff = __fadd_rn(ff, dot3(gamma, n));
    }
    return __fmul_rn(ff, __fdiv_rn(0.5f, area));
}

// PolyToDiff of source s's winding seen from (o, n).
__device__ __forceinline__ float poly_to_diff(const BounceView &v, int s, float area, F3 o, F3 n,
                                              unsigned long long *open) {
    const int2 w = __ldg(&v.wind[s]);
    return poly_to_diff_pts(v.points + w.x, w.y, area, o, n, open);
}

// One candidate pair: VisMatrix.TransferRay traced (StockExact: every
// triangle blocks, t in (0, len)), then MakeTransfer.  cand_w = the
// transfer, 0 for none.  Twelve CTAs per SM (40 registers, a few spilled
// to L1): the walk is latency-bound, and the extra resident warps hide
// more of it than the spills cost (measured 66 against 72 ms at 64
// registers and 8 CTAs on the 8x8 map).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 12) k_transfer(BounceView v, DeviceScene sc, const int64_t *__restrict__ cand_off,
                                                    const int32_t *__restrict__ cand_src, float *__restrict__ cand_w,
                                                    int64_t ncand, unsigned long long *counters, uint32_t *overflow) {
    extern __shared__ int stack_mem[];  // sc.stack_depth() entries per thread
    int *stack = stack_mem + threadIdx.x;
    const int64_t q = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
    const bool live = q < ncand;
    float w = 0.0f;
    bool blocked = false;
    // The receiver whose run holds q: one binary search per warp, for its
    // first candidate, then each lane steps forward (a warp's 32
    // candidates seldom span more than one or two receivers).
    const int64_t q0 = (int64_t)blockIdx.x * BLOCK + (threadIdx.x & ~31);
    int r0 = 0;
    if ((threadIdx.x & 31) == 0 && q0 < ncand) {
        int lo = 0, hi = v.nreceivers;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(&cand_off[mid]) <= q0) lo = mid;
            else hi = mid;
        }
        r0 = lo;
    }
    r0 = __shfl_sync(kFull, r0, 0);
    if (live) {
        int lo = r0;
        while (__ldg(&cand_off[lo + 1]) <= q) lo++;
        const int p = __ldg(&v.recv[lo]);
        const int s = __ldg(&cand_src[q]);
        const float4 po = __ldg(&v.origin[p]), pn = __ldg(&v.normal[p]);
        const float4 so = __ldg(&v.origin[s]), sn = __ldg(&v.normal[s]);
        const F3 start = add3(f3(po), f3(pn)), end = add3(f3(so), f3(sn));
        const F3 delta = sub3(end, start);
        const float len = __fsqrt_rn(dot3(delta, delta));
        const float safe = len == 0.0f ? 1.1920929e-07f : len;
        const RayState ray = make_ray(start.x, start.y, start.z, __fdiv_rn(delta.x, safe), __fdiv_rn(delta.y, safe),
                                      __fdiv_rn(delta.z, safe));
        float t;
        int32_t orig;
        uint32_t meta;
        trace_ray<kModeAny, BLOCK>(sc, ray, 0.0f, len, -1, stack, overflow, blocked, t, orig, meta);
        if (!blocked && __ldg(&v.tree[s].w) == 0 && so.w > 0.0f) {
            // MakeTransfer: DiffToDiff(source, receiver), the polygon form
            // factor for a near source, trans = area * scale > 1e-7.
            float scale = diff_to_diff(f3(so), f3(sn), f3(po), f3(pn));
            if (!(scale <= 0.0f)) {
                const F3 dd = sub3(f3(po), f3(so));
                const float threshold = (float)__dmul_rn(3.141592653589793 * 0.04, (double)dot3(dd, dd));
                bool ok = true;
                if (threshold < so.w) {
                    scale = poly_to_diff(v, s, so.w, f3(po), f3(pn), &counters[2]);
                    ok = !(scale <= 0.0f);
                }
                if (ok) {
                    const float trans = __fmul_rn(so.w, scale);
                    if ((double)trans > 0.0000001) w = trans;
                }
            }
        }
        cand_w[q] = w;
    }
    // Ray counts: one warp add each.
    const unsigned lane = threadIdx.x & 31;
    const int nlive = __popc(__ballot_sync(kFull, live));
    const int nblocked = __popc(__ballot_sync(kFull, live && blocked));
    if (lane == 0) {
        if (nlive) atomicAdd(&counters[0], (unsigned long long)nlive);
        if (nblocked) atomicAdd(&counters[1], (unsigned long long)nblocked);
    }
}

// MakeTransfers' count per receiver: accepted pairs, at most MaxPatches.
__global__ void k_transfer_count(int nrecv, const int64_t *__restrict__ cand_off, const float *__restrict__ cand_w,
                                 int64_t *__restrict__ counts) {
    const int r = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const unsigned lane = threadIdx.x & 31;
    if (r >= nrecv) return;
    const int64_t a = cand_off[r], b = cand_off[r + 1];
    int64_t n = 0;
    for (int64_t base = a; base < b; base += 32) {
        const int64_t q = base + lane;
        n += __popc(__ballot_sync(kFull, q < b && cand_w[q] > 0.0f));
    }
    if (lane == 0) counts[r] = n < kMaxTransfersPerReceiver ? n : kMaxTransfersPerReceiver;
}

// MakeTransfers' writes in candidate order (the first MaxPatches), then
// MakeScales: the float sum in order, total > pi ? 1/total : 1/pi, and the
// weights scaled.
__global__ void k_transfer_write(int nrecv, const int64_t *__restrict__ cand_off, const int32_t *__restrict__ cand_src,
                                 const float *__restrict__ cand_w, const int64_t *__restrict__ tr_off,
                                 int2 *__restrict__ tr) {
    const int r = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const unsigned lane = threadIdx.x & 31;
    if (r >= nrecv) return;
    const int64_t a = cand_off[r], b = cand_off[r + 1];
    const int64_t o0 = tr_off[r], o1 = tr_off[r + 1];
    int64_t made = 0;
    for (int64_t base = a; base < b && o0 + made < o1; base += 32) {
        const int64_t q = base + lane;
        const float w = q < b ? cand_w[q] : 0.0f;
        const unsigned ok = __ballot_sync(kFull, w > 0.0f);
        const int64_t at = o0 + made + __popc(ok & ((1u << lane) - 1u));
        if (w > 0.0f && at < o1) tr[at] = make_int2(cand_src[q], __float_as_int(w));
        made += __popc(ok);
    }
    __syncwarp();
    float scale = 0.0f;
    if (lane == 0 && o1 > o0) {
        float total = 0.0f;
        for (int64_t j = o0; j < o1; j++) total = __fadd_rn(total, __int_as_float(tr[j].y));
        scale = (double)total > 3.141592653589793 ? __fdiv_rn(1.0f, total) : (float)(1.0 / 3.141592653589793);
    }
    scale = __shfl_sync(kFull, scale, 0);
    __syncwarp();
    for (int64_t j = o0 + lane; j < o1; j += 32) {
        const int2 t = tr[j];
        tr[j] = make_int2(t.x, __float_as_int(__fmul_rn(__int_as_float(t.y), scale)));
    }
}

// ---- bounces ---------------------------------------------------------------

// The gather's slices (SELL-32) of the transfer lists: each receiver's
// count and index for the sort by count.
__global__ void k_sell_keys(int nrecv, const int64_t *__restrict__ tr_off, int32_t *__restrict__ key,
                            int32_t *__restrict__ idx) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrecv) return;
    key[r] = (int32_t)(tr_off[r + 1] - tr_off[r]);
    idx[r] = r;
}

// Slice s's size: 32 times its first (largest) count.
__global__ void k_sell_width(int nrecv, int nslices, const int32_t *__restrict__ count, int64_t *__restrict__ width) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslices) return;
    width[s] = 32 * (int64_t)count[32 * s];
}

// Copies each receiver's transfers into its lane of its slice.
__global__ void k_sell_pack(int nrecv, const int32_t *__restrict__ order, const int32_t *__restrict__ count,
                            const int64_t *__restrict__ sell_off, const int64_t *__restrict__ tr_off,
                            const int2 *__restrict__ tr, int2 *__restrict__ sell) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrecv) return;
    const int r = order[i], n = count[i];
    const int2 *src = tr + tr_off[r];
    int2 *dst = sell + sell_off[i >> 5] + (i & 31);
    for (int j = 0; j < n; j++) dst[32 * (int64_t)j] = __ldg(&src[j]);
}

// GatherLight for one receiver (the ordered sum over its transfers of the
// sources' shoot times the weight), then CollectLight's update of that
// leaf: the light added, emitted and shot on.  Thread i takes the i-th
// receiver of the count order, its transfers from its lane of its slice.
__global__ void k_gather(BounceView v, const int32_t *__restrict__ order, const int32_t *__restrict__ count,
                         const int64_t *__restrict__ sell_off, const int2 *__restrict__ sell,
                         const float4 *__restrict__ shoot_in, float4 *__restrict__ total,
                         float4 *__restrict__ emit_out, float4 *__restrict__ shoot_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.nreceivers) return;
    const int p = __ldg(&v.recv[__ldg(&order[i])]);
    const int n = __ldg(&count[i]);
    const int2 *src = sell + __ldg(&sell_off[i >> 5]) + (i & 31);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int j = 0; j < n; j++) {
        const int2 t = __ldg(&src[32 * (int64_t)j]);
        const float w = __int_as_float(t.y);
        const float4 s = __ldg(&shoot_in[t.x]);
        sx = __fadd_rn(sx, __fmul_rn(s.x, w));
        sy = __fadd_rn(sy, __fmul_rn(s.y, w));
        sz = __fadd_rn(sz, __fmul_rn(s.z, w));
    }
    if (__ldg(&v.tree[p].w)) {
        emit_out[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        shoot_out[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float4 t = total[p];
    total[p] = make_float4(__fadd_rn(t.x, sx), __fadd_rn(t.y, sy), __fadd_rn(t.z, sz), 0.0f);
    emit_out[p] = make_float4(sx, sy, sz, 0.0f);
    const float4 rf = __ldg(&v.refl[p]);
    shoot_out[p] = make_float4(__fmul_rn(sx, rf.x), __fmul_rn(sy, rf.y), __fmul_rn(sz, rf.z), 0.0f);
}

// CollectLight's parents for one level of the patch trees: every parent
// whose subtree is `level` deep, each the area blend of its children's
// light and emission (the children, one level lower, are final).  Run for
// levels 1, 2, ... this is CollectLight's bottom-up order within each face.
__global__ void k_collect_level(BounceView v, const int32_t *__restrict__ parents, int n, float4 *__restrict__ total,
                                float4 *__restrict__ emit_out, float4 *__restrict__ shoot_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = __ldg(&parents[i]);
    const int4 tr = __ldg(&v.tree[p]);
    if (tr.w) {
        emit_out[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        shoot_out[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float a1 = __ldg(&v.origin[tr.y].w), a2 = __ldg(&v.origin[tr.z].w);
    const float s1 = __fdiv_rn(a1, __fadd_rn(a1, a2)), s2 = __fdiv_rn(a2, __fadd_rn(a1, a2));
    const float4 c1 = total[tr.y], c2 = total[tr.z];
    total[p] = make_float4(__fadd_rn(__fmul_rn(c1.x, s1), __fmul_rn(c2.x, s2)),
                           __fadd_rn(__fmul_rn(c1.y, s1), __fmul_rn(c2.y, s2)),
                           __fadd_rn(__fmul_rn(c1.z, s1), __fmul_rn(c2.z, s2)), 0.0f);
    const float4 e1 = emit_out[tr.y], e2 = emit_out[tr.z];
    const float4 e = make_float4(__fadd_rn(__fmul_rn(e1.x, s1), __fmul_rn(e2.x, s2)),
                                 __fadd_rn(__fmul_rn(e1.y, s1), __fmul_rn(e2.y, s2)),
                                 __fadd_rn(__fmul_rn(e1.z, s1), __fmul_rn(e2.z, s2)), 0.0f);
    emit_out[p] = e;
    const float4 rf = __ldg(&v.refl[p]);
    shoot_out[p] = make_float4(__fmul_rn(e.x, rf.x), __fmul_rn(e.y, rf.y), __fmul_rn(e.z, rf.z), 0.0f);
}

// The light a bounce added (the leaves' emission), in fp64, with two sums
// that bound how far the reference's float sum (CollectLight's, in
// leaf_desc order) can lie from it: the absolute values, and the absolute
// values each weighted by the number of terms from it to the end of that
// order (n - rank).  Recursive summation's error is at most
// u * sum_k |partial sum k| <= u * sum_i |x_i| (n - rank_i), over 1 - n u.
__global__ void k_totals(BounceView v, const float4 *__restrict__ emit, const int32_t *__restrict__ leaf_rank,
                         int32_t nleaves, double *__restrict__ sums) {
    __shared__ double part[kSums][kBounceBlock / 32];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double s[kSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (p < v.npatches) {
        const int4 tr = __ldg(&v.tree[p]);
        if (tr.y == -1 && tr.w == 0) {
            const float4 e = emit[p];
            const double w = (double)(nleaves - __ldg(&leaf_rank[p]));
            s[0] = e.x, s[1] = e.y, s[2] = e.z;
            s[3] = fabs((double)e.x), s[4] = fabs((double)e.y), s[5] = fabs((double)e.z);
            s[6] = s[3] * w, s[7] = s[4] * w, s[8] = s[5] * w;
        }
    }
    for (int k = 0; k < kSums; k++)
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_down_sync(kFull, s[k], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < kSums; k++) part[k][warp] = s[k];
    __syncthreads();
    if (threadIdx.x < kSums) {
        double t = 0.0;
        for (int w = 0; w < kBounceBlock / 32; w++) t += part[threadIdx.x][w];
        atomicAdd(&sums[threadIdx.x], t);
    }
}

// CollectLight's own total: the leaves' emission summed in float, in
// descending index order (leaf_desc lists the sky-free leaves that way).
// The sum is one chain of dependent adds; one block keeps it fed: all of
// its threads stage the next tile of values in shared memory while warp 0
// adds up the current one, every lane of it the same chain.
constexpr int kExactThreads = 1024;
constexpr int kExactTile = 1024;  // two tiles of float4: 32 KB of shared memory

__global__ void __launch_bounds__(kExactThreads) k_exact_total(const int32_t *__restrict__ leaf_desc, int32_t n,
                                                               const float4 *__restrict__ emit, float *__restrict__ out) {
    __shared__ float4 tile[2][kExactTile];
    float x = 0.0f, y = 0.0f, z = 0.0f;
    // Stages tile `buf` with threads [first, kExactThreads).
    auto stage = [&](int buf, int base, int first) {
        for (int k = (int)threadIdx.x - first; k < kExactTile; k += kExactThreads - first) {
            const int i = base + k;
            tile[buf][k] = i < n ? __ldg(&emit[__ldg(&leaf_desc[i])]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    };
    stage(0, 0, 0);
    __syncthreads();
    for (int base = 0, buf = 0; base < n; base += kExactTile, buf ^= 1) {
        if (threadIdx.x >= 32) {
            stage(buf ^ 1, base + kExactTile, 32);
        } else {
            // The three chains of dependent adds; unrolled so the tile's
            // loads run ahead of them.
            const int m = min(kExactTile, n - base);
            const float4 *t = tile[buf];
#pragma unroll 16
            for (int k = 0; k < m; k++) {
                const float4 v = t[k];
                x = __fadd_rn(x, v.x);
                y = __fadd_rn(y, v.y);
                z = __fadd_rn(z, v.z);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = x;
        out[1] = y;
        out[2] = z;
    }
}

// ---- the learned warm start --------------------------------------------------

// Per receiver, the network's 32 inputs (BF16): the shading normal, log2 of
// the area over 16, the reflectivity, log1p of the direct and of the
// first-bounce light over 8, log2(1 + d) over 16 of the distances d to the
// eight nearest point and spot lights (1 when there are fewer), zeros.
__global__ void k_features(BounceView v, const float4 *__restrict__ direct, const float4 *__restrict__ first,
                           const float4 *__restrict__ lights, int32_t nlights, uint16_t *__restrict__ x) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= v.nreceivers) return;
    const int p = __ldg(&v.recv[r]);
    const float4 o = __ldg(&v.origin[p]), nrm = __ldg(&v.normal[p]), rf = __ldg(&v.refl[p]);
    const float4 d = direct[p], b1 = first[p];
    float f[kFeatures];
    f[0] = nrm.x, f[1] = nrm.y, f[2] = nrm.z;
    f[3] = log2f(fmaxf(o.w, 1e-6f)) / 16.0f;
    f[4] = rf.x, f[5] = rf.y, f[6] = rf.z;
    f[7] = log1pf(fmaxf(d.x, 0.0f)) / 8.0f, f[8] = log1pf(fmaxf(d.y, 0.0f)) / 8.0f, f[9] = log1pf(fmaxf(d.z, 0.0f)) / 8.0f;
    f[10] = log1pf(fmaxf(b1.x, 0.0f)) / 8.0f, f[11] = log1pf(fmaxf(b1.y, 0.0f)) / 8.0f;
    f[12] = log1pf(fmaxf(b1.z, 0.0f)) / 8.0f;
    float best[8];
    for (int k = 0; k < 8; k++) best[k] = INFINITY;
    for (int l = 0; l < nlights; l++) {
        const float4 a = __ldg(&lights[5 * l]);
        const int type = __float_as_int(a.w);
        if (type != 1 && type != 2) continue;
        const float dx = a.x - o.x, dy = a.y - o.y, dz = a.z - o.z;
        float q = dx * dx + dy * dy + dz * dz;
        for (int k = 0; k < 8; k++) {
            if (q < best[k]) {
                const float tmp = best[k];
                best[k] = q;
                q = tmp;
            }
        }
    }
    for (int k = 0; k < 8; k++) f[13 + k] = isinf(best[k]) ? 1.0f : log2f(1.0f + sqrtf(best[k])) / 16.0f;
    for (int k = 21; k < kFeatures; k++) f[k] = 0.0f;
    for (int k = 0; k < kFeatures; k++) x[(int64_t)r * kFeatures + k] = __bfloat16_as_ushort(__float2bfloat16_rn(f[k]));
}

// The network's guess as light per patch: expm1 of its output, at least
// zero, on the non-sky receivers (everything else zero).
__global__ void k_guess(BounceView v, const float *__restrict__ y, float4 *__restrict__ guess) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= v.nreceivers) return;
    const int p = __ldg(&v.recv[r]);
    float4 gv = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!__ldg(&v.tree[p].w)) {
        gv.x = fmaxf(expm1f(y[3 * (int64_t)r]), 0.0f);
        gv.y = fmaxf(expm1f(y[3 * (int64_t)r + 1]), 0.0f);
        gv.z = fmaxf(expm1f(y[3 * (int64_t)r + 2]), 0.0f);
    }
    guess[p] = gv;
}

// A per-patch quantity of one level's parents as the area blend of their
// children (as CollectLight blends the light); run level by level.
__global__ void k_blend_level(BounceView v, const int32_t *__restrict__ parents, int n, float4 *__restrict__ a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = __ldg(&parents[i]);
    const int4 tr = __ldg(&v.tree[p]);
    const float a1 = __ldg(&v.origin[tr.y].w), a2 = __ldg(&v.origin[tr.z].w);
    const float s1 = a1 / (a1 + a2), s2 = a2 / (a1 + a2);
    const float4 c1 = a[tr.y], c2 = a[tr.z];
    a[p] = make_float4(c1.x * s1 + c2.x * s2, c1.y * s1 + c2.y * s2, c1.z * s1 + c2.z * s2, 0.0f);
}

// The first warm step for each receiver (in count order, its transfers
// from its slice lane): A = the transfers' gather of the guess's shot
// light, then light = B1 + A (the Jacobi step from the guess), emission =
// light - guess (the change, which later bounces carry on).
__global__ void k_warm_combine(BounceView v, const int32_t *__restrict__ order, const int32_t *__restrict__ count,
                               const int64_t *__restrict__ sell_off, const int2 *__restrict__ sell,
                               const float4 *__restrict__ guess, const float4 *__restrict__ first,
                               float4 *__restrict__ total, float4 *__restrict__ emit_out, float4 *__restrict__ shoot_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.nreceivers) return;
    const int p = __ldg(&v.recv[__ldg(&order[i])]);
    const int n = __ldg(&count[i]);
    const int2 *src = sell + __ldg(&sell_off[i >> 5]) + (i & 31);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int j = 0; j < n; j++) {
        const int2 t = __ldg(&src[32 * (int64_t)j]);
        const float w = __int_as_float(t.y);
        const float4 gs = guess[t.x], rf = __ldg(&v.refl[t.x]);
        sx += gs.x * rf.x * w;
        sy += gs.y * rf.y * w;
        sz += gs.z * rf.z * w;
    }
    if (__ldg(&v.tree[p].w)) {
        emit_out[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        shoot_out[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float4 b1 = first[p], gv = guess[p];
    const float4 t = make_float4(b1.x + sx, b1.y + sy, b1.z + sz, 0.0f);
    total[p] = t;
    const float4 d = make_float4(t.x - gv.x, t.y - gv.y, t.z - gv.z, 0.0f);
    emit_out[p] = d;
    const float4 rf = __ldg(&v.refl[p]);
    shoot_out[p] = make_float4(d.x * rf.x, d.y * rf.y, d.z * rf.z, 0.0f);
}

unsigned blocks(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

void BounceBuffers::release() {
    void *ptrs[] = {origin, normal, mins, maxs, refl, tree, wind, points, face_range, face_samples, face_plane,
                    recv, row_off, row_faces, sample_area, cand_off, cand_src, cand_w, tr_off, tr, scan_tmp,
                    acc, direct, total, emit[0], emit[1], shoot[0], shoot[1], sums, exact, counters, leaf_desc,
                    level_patch, leaf_rank, sell_key, sell_idx, sell_count, sell_order, sell_off, sell, sort_tmp,
                    first, guess, feat, pred,
                    pr_off, pr_patch, pr_box, pr_coord, prad_light, prad_weight};
    for (void *q : ptrs) dev_free(q);
    for (cudaGraphExec_t &g : bounce_graph)
        if (g) cudaGraphExecDestroy(g);
    // The pinned stop-rule sums stay for the next upload (freeing pinned
    // memory can stall); free_pinned() frees them.
    double *sums_h = h_sums;
    float *exact_h = h_exact;
    *this = BounceBuffers();
    h_sums = sums_h;
    h_exact = exact_h;
}

void BounceBuffers::free_pinned() {
    cudaFreeHost(h_sums);
    cudaFreeHost(h_exact);
    h_sums = nullptr;
    h_exact = nullptr;
}

cudaError_t launch_patch_light(const BounceBuffers &b, const float4 *sample_light, cudaStream_t stream) {
    if (b.npatches == 0) return cudaSuccess;
    k_patch_samples<<<blocks(b.npatches, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, sample_light, b.acc);
    k_patch_tree<<<blocks(b.nfaces, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.acc, b.direct, b.total,
                                                                              b.emit[0], b.shoot[0]);
    return cudaGetLastError();
}

// The transfer build.  count_only: the candidate counts and offsets alone
// (at upload: they size the buffers, and they depend only on the patch
// tree and the PVS rows, so they stay valid until the next upload).
// Otherwise, with those offsets, the candidates written, their rays and
// form factors, and the transfer lists; counters[0..1] are added to.
cudaError_t launch_transfers(BounceBuffers &b, const DeviceScene &scene, uint32_t *overflow, cudaStream_t stream,
                             bool count_only) {
    const int R = b.nreceivers;
    if (R == 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    size_t tmp = 0;
    if (count_only) {
        // Candidate counts into cand_off[1..R], then the exclusive scan.
        k_candidates<<<blocks(R, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, nullptr, b.cand_off + 1, nullptr,
                                                                           overflow);
        e = cudaMemsetAsync(b.cand_off, 0, sizeof(int64_t), stream);
        if (e != cudaSuccess) return e;
        tmp = b.scan_tmp_bytes;
        e = cub::DeviceScan::InclusiveSum(b.scan_tmp, tmp, b.cand_off + 1, b.cand_off + 1, R, stream);
        return e != cudaSuccess ? e : cudaGetLastError();
    }
    k_candidates<<<blocks(R, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.cand_off, nullptr, b.cand_src,
                                                                       overflow);
    if (b.ncand > 0)
        k_transfer<kBlock><<<blocks(b.ncand, kBlock), kBlock, sizeof(int) * scene.stack_depth() * kBlock, stream>>>(b.view, scene, b.cand_off, b.cand_src,
                                                                           b.cand_w, b.ncand, b.counters, overflow);
    k_transfer_count<<<blocks((int64_t)R * 32, kBounceBlock), kBounceBlock, 0, stream>>>(R, b.cand_off, b.cand_w,
                                                                                         b.tr_off + 1);
    e = cudaMemsetAsync(b.tr_off, 0, sizeof(int64_t), stream);
    if (e != cudaSuccess) return e;
    tmp = b.scan_tmp_bytes;
    e = cub::DeviceScan::InclusiveSum(b.scan_tmp, tmp, b.tr_off + 1, b.tr_off + 1, R, stream);
    if (e != cudaSuccess) return e;
    if (!b.tr) return cudaGetLastError();
    k_transfer_write<<<blocks((int64_t)R * 32, kBounceBlock), kBounceBlock, 0, stream>>>(
        R, b.cand_off, b.cand_src, b.cand_w, b.tr_off, b.tr);
    e = cudaGetLastError();
    return e != cudaSuccess ? e : launch_sell(b, stream);
}

// The gather's slices (SELL-32) from the transfer lists tr_off / tr.
cudaError_t launch_sell(BounceBuffers &b, cudaStream_t stream) {
    const int R = b.nreceivers;
    if (R == 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    size_t tmp = 0;
    const int nslices = (R + 31) / 32;
    k_sell_keys<<<blocks(R, kBounceBlock), kBounceBlock, 0, stream>>>(R, b.tr_off, b.sell_key, b.sell_idx);
    tmp = b.sort_tmp_bytes;
    e = cub::DeviceRadixSort::SortPairsDescending(b.sort_tmp, tmp, b.sell_key, b.sell_count, b.sell_idx, b.sell_order,
                                                  R, 0, 20, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.sell_off, 0, sizeof(int64_t), stream);
    if (e != cudaSuccess) return e;
    k_sell_width<<<blocks(nslices, kBounceBlock), kBounceBlock, 0, stream>>>(R, nslices, b.sell_count, b.sell_off + 1);
    tmp = b.scan_tmp_bytes;
    e = cub::DeviceScan::InclusiveSum(b.scan_tmp, tmp, b.sell_off + 1, b.sell_off + 1, nslices, stream);
    if (e != cudaSuccess) return e;
    k_sell_pack<<<blocks(R, kBounceBlock), kBounceBlock, 0, stream>>>(R, b.sell_order, b.sell_count, b.sell_off,
                                                                      b.tr_off, b.tr, b.sell);
    return cudaGetLastError();
}

// CollectLight's parents, level by level.
cudaError_t launch_collect(const BounceBuffers &b, float4 *emit_out, float4 *shoot_out, cudaStream_t stream) {
    for (size_t h = 1; h + 1 < b.h_level_off.size(); h++) {
        const int32_t a = b.h_level_off[h], n = b.h_level_off[h + 1] - a;
        if (n > 0)
            k_collect_level<<<blocks(n, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.level_patch + a, n, b.total,
                                                                                  emit_out, shoot_out);
    }
    return cudaGetLastError();
}

// Bounce number `bounce` (0-based): reads shoot[bounce & 1], writes the
// other half, then the fp64 totals.
cudaError_t launch_gather(BounceBuffers &b, int bounce, cudaStream_t stream) {
    const int in = bounce & 1, out = in ^ 1;
    if (b.nreceivers)
        k_gather<<<blocks(b.nreceivers, kBounceBlock), kBounceBlock, 0, stream>>>(
            b.view, b.sell_order, b.sell_count, b.sell_off, b.sell, b.shoot[in], b.total, b.emit[out], b.shoot[out]);
    cudaError_t e = launch_collect(b, b.emit[out], b.shoot[out], stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.sums, 0, kSums * sizeof(double), stream);
    if (e != cudaSuccess) return e;
    if (b.npatches)
        k_totals<<<blocks(b.npatches, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.emit[out], b.leaf_rank,
                                                                                b.nleaves, b.sums);
    b.last_buffer = out;
    return cudaGetLastError();
}

cudaError_t launch_features(BounceBuffers &b, const DeviceWorld &w, cudaStream_t stream) {
    if (!b.nreceivers) return cudaSuccess;
    k_features<<<blocks(b.nreceivers, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.direct, b.first, w.lights,
                                                                                w.nlights, b.feat);
    return cudaGetLastError();
}

// The warm start after bounce 0 (which left B1 in b.first): the guess from
// the network, blended to the parents, the first warm step into the other
// emit/shoot half, the parents' light and emission, and the totals.
cudaError_t launch_warm_start(BounceBuffers &b, const DeviceWorld &w, const vrad_mlp &m, cudaStream_t stream) {
    if (!b.nreceivers) return cudaSuccess;
    cudaError_t e = launch_features(b, w, stream);
    if (e == cudaSuccess) e = mlp_forward(m, b.feat, b.nreceivers, b.pred, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.guess, 0, sizeof(float4) * (size_t)b.npatches, stream);
    if (e != cudaSuccess) return e;
    k_guess<<<blocks(b.nreceivers, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.pred, b.guess);
    for (size_t h = 1; h + 1 < b.h_level_off.size(); h++) {
        const int32_t a = b.h_level_off[h], n = b.h_level_off[h + 1] - a;
        if (n > 0)
            k_blend_level<<<blocks(n, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.level_patch + a, n, b.guess);
    }
    // Bounce 0 wrote half 1; the warm step writes half 0, as bounce 1 would.
    k_warm_combine<<<blocks(b.nreceivers, kBounceBlock), kBounceBlock, 0, stream>>>(
        b.view, b.sell_order, b.sell_count, b.sell_off, b.sell, b.guess, b.first, b.total, b.emit[0], b.shoot[0]);
    e = launch_collect(b, b.emit[0], b.shoot[0], stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.sums, 0, kSums * sizeof(double), stream);
    if (e != cudaSuccess) return e;
    k_totals<<<blocks(b.npatches, kBounceBlock), kBounceBlock, 0, stream>>>(b.view, b.emit[0], b.leaf_rank, b.nleaves,
                                                                            b.sums);
    b.last_buffer = 0;
    return cudaGetLastError();
}

cudaError_t launch_bounce_graph(BounceBuffers &b, int bounce, cudaStream_t capture, cudaStream_t stream) {
    const int k = bounce & 1;
    if (!b.bounce_graph[k]) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(capture, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        cudaError_t inside = launch_gather(b, bounce, capture);
        if (inside == cudaSuccess)
            inside = cudaMemcpyAsync(b.h_sums, b.sums, kSums * sizeof(double), cudaMemcpyDeviceToHost, capture);
        e = cudaStreamEndCapture(capture, &g);
        if (e == cudaSuccess) e = inside;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b.bounce_graph[k], g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b.bounce_graph[k] = nullptr;
            return e;
        }
    }
    b.last_buffer = k ^ 1;
    return cudaGraphLaunch(b.bounce_graph[k], stream);
}

cudaError_t launch_exact_total(BounceBuffers &b, int bounce, cudaStream_t stream) {
    k_exact_total<<<1, kExactThreads, 0, stream>>>(b.leaf_desc, b.nleaves, b.emit[(bounce & 1) ^ 1], b.exact);
    return cudaGetLastError();
}

}  // namespace vrad

// ---- form factors on their own (inspection) ----------------------------------
//
// The transfer build's DiffToDiff and PolyToDiff, evaluated for caller-given
// cases by the same device functions k_transfer calls, so the reference's
// known-answer cases (Tests/MapTools/Rad/Bounce/FormFactorsTests.cs) run on
// the device's own arithmetic.

namespace {

__global__ void k_ff_diff(const float *__restrict__ c, int64_t n, float *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *q = c + 12 * i;
    out[i] = vrad::diff_to_diff({q[0], q[1], q[2]}, {q[3], q[4], q[5]}, {q[6], q[7], q[8]}, {q[9], q[10], q[11]});
}

__global__ void k_ff_poly(const float4 *__restrict__ pts, const int32_t *__restrict__ first,
                          const float *__restrict__ c, int64_t n, float *__restrict__ out,
                          unsigned long long *open) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *q = c + 7 * i;
    out[i] = vrad::poly_to_diff_pts(pts + first[i], first[i + 1] - first[i], q[0], {q[1], q[2], q[3]},
                                    {q[4], q[5], q[6]}, open);
}

// Copies `bytes` from host to a fresh device block (the inspection calls'
// own small temporaries).
cudaError_t upload_tmp(void **d, const void *h, size_t bytes, cudaStream_t s) {
    cudaError_t e = cudaMalloc(d, bytes ? bytes : 16);
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(*d, h, bytes, cudaMemcpyHostToDevice, s);
    return e;
}

}  // namespace

extern "C" int32_t vrad_form_factor_diff(vrad_ctx *ctx, const float *cases, int64_t n, float *out) {
    if (!ctx || n < 0 || (n && (!cases || !out))) return vrad_fail(ctx, VRAD_ERR_ARG, "invalid form factor cases");
    if (n == 0) return VRAD_OK;
    std::lock_guard<std::mutex> g(ctx->mu);
    void *dc = nullptr, *dout = nullptr;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = upload_tmp(&dc, cases, sizeof(float) * 12 * (size_t)n, ctx->stream);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(float) * (size_t)n);
    if (e == cudaSuccess) {
        k_ff_diff<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(static_cast<const float *>(dc), n,
                                                                      static_cast<float *>(dout));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    cudaFree(dc);
    cudaFree(dout);
    return e == cudaSuccess ? VRAD_OK : vrad_cuda_fail(ctx, e, "form factors");
}

extern "C" int32_t vrad_form_factor_poly(vrad_ctx *ctx, const float *points, const int32_t *first,
                                         const float *cases, int64_t n, float *out) {
    if (!ctx || n < 0 || (n && (!points || !first || !cases || !out)))
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid form factor cases");
    if (n == 0) return VRAD_OK;
    for (int64_t i = 0; i < n; i++)
        if (first[i] < 0 || first[i + 1] < first[i] + 3)
            return vrad_fail(ctx, VRAD_ERR_ARG, "winding %lld has fewer than three points", (long long)i);
    const int64_t np = first[n];
    std::vector<float4> pts((size_t)np);
    for (int64_t k = 0; k < np; k++) pts[(size_t)k] = make_float4(points[3 * k], points[3 * k + 1], points[3 * k + 2], 0.0f);
    std::lock_guard<std::mutex> g(ctx->mu);
    void *dp = nullptr, *df = nullptr, *dc = nullptr, *dout = nullptr, *dopen = nullptr;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = upload_tmp(&dp, pts.data(), sizeof(float4) * (size_t)np, ctx->stream);
    if (e == cudaSuccess) e = upload_tmp(&df, first, sizeof(int32_t) * (size_t)(n + 1), ctx->stream);
    if (e == cudaSuccess) e = upload_tmp(&dc, cases, sizeof(float) * 7 * (size_t)n, ctx->stream);
    if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(float) * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dopen, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(dopen, 0, sizeof(unsigned long long), ctx->stream);
    if (e == cudaSuccess) {
        k_ff_poly<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
            static_cast<const float4 *>(dp), static_cast<const int32_t *>(df), static_cast<const float *>(dc), n,
            static_cast<float *>(dout), static_cast<unsigned long long *>(dopen));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    for (void *q : {dp, df, dc, dout, dopen}) cudaFree(q);
    return e == cudaSuccess ? VRAD_OK : vrad_cuda_fail(ctx, e, "form factors");
}
