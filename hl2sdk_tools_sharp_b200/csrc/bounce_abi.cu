// bounce_abi.cu -- host side of the bounce: vrad_bounce_upload (the patch
// tree, receiver order, PVS rows and the final pass's patch tables, and
// the buffers sized by a candidate count), the bounce loop of a light
// pass with the reference's stop rule, and the inspection entry points.

#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bounce.cuh"
#include "bounce_host.h"
#include "context.cuh"
#include "device_pool.h"
#include "host_parallel.h"
#include "patches.h"
#include "setup_clock.h"
#include "world.h"
#include "sync_wait.h"

namespace vrad {

namespace {

inline float bits_f(int32_t x) {
    float y;
    std::memcpy(&y, &x, 4);
    return y;
}

// x86's truncating double-to-int conversion, which the host set-up's
// (int) casts compile to: out of range and NaN give INT_MIN.
__device__ __forceinline__ int dtrunc_x86(double x) {
    return (x > -2147483649.0 && x < 2147483648.0) ? __double2int_rz(x) : INT_MIN;
}

// WorldToLuxel of the final pass's frame fr (5 float4: origin and width,
// world-to-luxel s and height, world-to-luxel t and min_s, luxel-to-world
// s and min_t, luxel-to-world t), each operation rounded on its own.
__device__ __forceinline__ void radial_w2l(const float4 *fr, float px, float py, float pz, float &s, float &t) {
    const float4 o = __ldg(&fr[0]), ws = __ldg(&fr[1]), wt = __ldg(&fr[2]), ls = __ldg(&fr[3]);
    const float dx = __fsub_rn(px, o.x), dy = __fsub_rn(py, o.y), dz = __fsub_rn(pz, o.z);
    s = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, ws.x), __fmul_rn(dy, ws.y)), __fmul_rn(dz, ws.z)),
                  (float)__float_as_int(wt.w));
    t = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, wt.x), __fmul_rn(dy, wt.y)), __fmul_rn(dz, wt.z)),
                  (float)__float_as_int(ls.w));
}

// The per-face candidate list of the bounced light's radial grid
// (BuildPatchRadial): the face's own leaf patches, then each smoothing
// neighbour's, each list in FacePatches order (descendants by descending
// index, then the root); each kept with its box in this face's cells when
// that box holds at least one cell.  One thread per (face, source face)
// pair, pairs in that order: COUNT counts into counts[q]; otherwise the
// entries are written at off[q]...
template <bool COUNT>
__global__ void k_radial_pairs(int32_t npairs, const int32_t *__restrict__ pair_face,
                               const int32_t *__restrict__ pair_src, BounceView v, const float4 *__restrict__ frames,
                               int32_t *__restrict__ counts, const int64_t *__restrict__ off,
                               int32_t *__restrict__ out_patch, int4 *__restrict__ out_box,
                               float4 *__restrict__ out_coord) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npairs) return;
    const int f = __ldg(&pair_face[q]), g = __ldg(&pair_src[q]);
    const float4 *me = frames + 5 * (int64_t)f;
    const int width = __float_as_int(__ldg(&me[0].w)), height = __float_as_int(__ldg(&me[1].w));
    const int4 fr = __ldg(&v.face_range[g]);  // root, first descendant, end
    int64_t at = COUNT ? 0 : __ldg(&off[q]);
    int n = 0;
    if (fr.x >= 0) {
        for (int k = 0; k <= fr.z - fr.y; k++) {
            const int p = k < fr.z - fr.y ? fr.z - 1 - k : fr.x;
            if (__ldg(&v.tree[p].y) != -1) continue;
            // PatchLightmapCoordRange.
            const int2 w = __ldg(&v.wind[p]);
            float min_s = 1e30f, min_t = 1e30f, max_s = -1e30f, max_t = -1e30f;
            for (int i = 0; i < w.y; i++) {
                const float4 pt = __ldg(&v.points[w.x + i]);
                float s, t;
                radial_w2l(me, pt.x, pt.y, pt.z, s, t);
                min_s = min_s < s ? min_s : s;
                max_s = max_s > s ? max_s : s;
                min_t = min_t < t ? min_t : t;
                max_t = max_t > t ? max_t : t;
            }
            // LuxelRadial.AddBounced's extent and box.
            const float4 o = __ldg(&v.origin[p]);
            float cs, ct;
            radial_w2l(me, o.x, o.y, o.z, cs, ct);
            float ds = __fsub_rn(max_s, min_s), dt = __fsub_rn(max_t, min_t);
            ds = 1.0 > (double)ds ? 1.0f : ds;
            dt = 1.0 > (double)dt ? 1.0f : dt;
            const double es = __dmul_rn((double)ds, 1.42), et = __dmul_rn((double)dt, 1.42);
            int smin = dtrunc_x86(__dsub_rn((double)cs, es));
            int tmin = dtrunc_x86(__dsub_rn((double)ct, et));
            int smax = dtrunc_x86(__dadd_rn(__dadd_rn((double)cs, es), 1.0));
            int tmax = dtrunc_x86(__dadd_rn(__dadd_rn((double)ct, et), 1.0));
            smin = smin > 0 ? smin : 0;
            tmin = tmin > 0 ? tmin : 0;
            smax = smax < width ? smax : width;
            tmax = tmax < height ? tmax : height;
            if (smin >= smax || tmin >= tmax) continue;
            if (!COUNT) {
                out_patch[at] = p;
                out_box[at] = make_int4(smin, tmin, smax, tmax);
                out_coord[at] = make_float4(cs, ct, ds, dt);
                at++;
            }
            n++;
        }
    }
    if (COUNT) counts[q] = n;
}

// pr_off[f] = off[first pair of face f].
__global__ void k_radial_off(int32_t nfaces, const int32_t *__restrict__ face_pair0, const int64_t *__restrict__ off,
                             int32_t *__restrict__ pr_off) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f <= nfaces) pr_off[f] = (int32_t)off[face_pair0[f]];
}

unsigned grid_for(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

// The radial tables on the device, from the uploaded patches (b.view) and
// the final pass's frames, into b.pr_off, pr_patch, pr_box, pr_coord.
// Synchronises the stream once, for the total's size.
cudaError_t radial_tables(BounceBuffers &b, const float4 *frames, int32_t nf, const std::vector<int32_t> &noff,
                          const std::vector<int32_t> &nlist, Stager &stager, cudaStream_t stream) {
    const int32_t npairs = nf + noff[(size_t)nf];
    std::vector<int32_t> pair_face((size_t)(npairs ? npairs : 1)), pair_src((size_t)(npairs ? npairs : 1)),
        face_pair0((size_t)nf + 1);
    int32_t q = 0;
    for (int32_t f = 0; f < nf; f++) {
        face_pair0[(size_t)f] = q;
        pair_face[(size_t)q] = f;
        pair_src[(size_t)q++] = f;
        for (int32_t k = noff[(size_t)f]; k < noff[(size_t)f + 1]; k++) {
            pair_face[(size_t)q] = f;
            pair_src[(size_t)q++] = nlist[(size_t)k];
        }
    }
    face_pair0[(size_t)nf] = q;
    int32_t *d_pf = nullptr, *d_ps = nullptr, *d_p0 = nullptr, *d_counts = nullptr;
    int64_t *d_off = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    int64_t total = 0;
    const size_t Q1 = (size_t)(npairs ? npairs : 1);
    cudaError_t e = stage_table(stager, stream, &d_pf, pair_face);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_ps, pair_src);
    if (e == cudaSuccess) e = stage_table(stager, stream, &d_p0, face_pair0);
    if (e == cudaSuccess) e = dev_alloc(&d_counts, sizeof(int32_t) * Q1);
    if (e == cudaSuccess) e = dev_alloc(&d_off, sizeof(int64_t) * (Q1 + 1));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_off, 0, sizeof(int64_t), stream);
    if (e == cudaSuccess && npairs > 0) {
        k_radial_pairs<true><<<grid_for(npairs, 128), 128, 0, stream>>>(npairs, d_pf, d_ps, b.view, frames, d_counts,
                                                                       nullptr, nullptr, nullptr, nullptr);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, d_counts, d_off + 1, npairs, stream);
        if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes ? tmp_bytes : 1);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, d_counts, d_off + 1, npairs, stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, d_off + npairs, sizeof total, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = vrad::wait_stream(stream);
    const size_t T1 = (size_t)(total ? total : 1);
    if (e == cudaSuccess) e = dev_alloc(&b.pr_off, sizeof(int32_t) * ((size_t)nf + 1));
    if (e == cudaSuccess) e = dev_alloc(&b.pr_patch, sizeof(int32_t) * T1);
    if (e == cudaSuccess) e = dev_alloc(&b.pr_box, sizeof(int4) * T1);
    if (e == cudaSuccess) e = dev_alloc(&b.pr_coord, sizeof(float4) * T1);
    if (e == cudaSuccess && npairs > 0) {
        k_radial_pairs<false><<<grid_for(npairs, 128), 128, 0, stream>>>(npairs, d_pf, d_ps, b.view, frames, nullptr,
                                                                        d_off, b.pr_patch, b.pr_box, b.pr_coord);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_radial_off<<<grid_for((int64_t)nf + 1, 256), 256, 0, stream>>>(nf, d_p0, d_off, b.pr_off);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = vrad::wait_stream(stream);
    for (void *x : {(void *)d_pf, (void *)d_ps, (void *)d_p0, (void *)d_counts, (void *)d_off, tmp}) dev_free(x);
    return e;
}

}  // namespace

// The bounce of one light pass, after the direct gather wrote
// sample_light: patch light, transfers (unless the pass's previous range
// built them), bounces to the stop rule.  Leaves the bounced light in
// b.total.  Blocks on the stream once per bounce (the stop rule is decided
// on the host).
cudaError_t run_bounce(vrad_ctx *ctx, cudaStream_t s, const float4 *sample_light, bool build_transfers,
                       std::string &why) {
    BounceBuffers &b = ctx->bounce;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 4 && e == cudaSuccess; k++) e = cudaEventCreate(&ev[k]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], s);
    if (e == cudaSuccess) e = launch_patch_light(b, sample_light, s);
    if (e == cudaSuccess) e = cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.counters, 0, 3 * sizeof(unsigned long long), s);
    if (e == cudaSuccess && build_transfers) e = launch_transfers(b, ctx->scene.view(), ctx->status, s, false);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], s);
    b.bounces_run = 0;
    b.exact_totals = 0;
    // The float sum's error bound: u / (1 - n u) times the rank-weighted
    // absolute sum (k_totals).
    const double u = std::ldexp(1.0, -24);
    const double nu = (double)b.nleaves * u;
    const double scale = nu < 0.5 ? u / (1.0 - nu) : INFINITY;
    const vrad_mlp *model = ctx->bounce_model;
    for (int i = 0; e == cudaSuccess && i < b.max_bounces; i++) {
        // With a network attached, the second step starts from its guess
        // (launch_warm_start) instead of bouncing the first bounce's light.
        // The later plain bounces are one captured graph each.
        const bool graph = i > 0 && !(model && i == 1);
        if (graph) e = launch_bounce_graph(b, i, ctx->stream, s);
        else e = (model && i == 1) ? launch_warm_start(b, ctx->world.view, *model, s) : launch_gather(b, i, s);
        if (e == cudaSuccess && i == 0)
            e = cudaMemcpyAsync(b.first, b.total, sizeof(float4) * (size_t)b.npatches, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess && !graph)
            e = cudaMemcpyAsync(b.h_sums, b.sums, kSums * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = vrad::wait_stream(s);
        if (e != cudaSuccess) break;
        b.bounces_run = i + 1;
        if (model) {
            // The warm iteration's changes can be negative: it stops on the
            // sum of their magnitudes.
            for (int c = 0; c < 3; c++) b.added[c] = b.h_sums[3 + c];
            if (b.added[0] < (double)b.threshold && b.added[1] < (double)b.threshold && b.added[2] < (double)b.threshold)
                break;
            continue;
        }
        // Radiosity.BounceAsync's stop rule on CollectLight's float total:
        // settled by the fp64 total when the float sum's error bound keeps
        // it on one side of the threshold, else by the sequential sum.  The
        // 1.0001 covers the fp64 sums' own rounding.
        bool below[3], settled = true;
        for (int c = 0; c < 3; c++) {
            const double S = b.h_sums[c], bound = scale * b.h_sums[6 + c] * 1.0001;
            b.added[c] = S;
            if (S + bound < (double)b.threshold) below[c] = true;
            else if (S - bound >= (double)b.threshold) below[c] = false;
            else settled = false;
        }
        if (!settled) {
            b.exact_totals++;
            e = launch_exact_total(b, i, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(b.h_exact, b.exact, 3 * sizeof(float), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = vrad::wait_stream(s);
            if (e != cudaSuccess) break;
            for (int c = 0; c < 3; c++) {
                b.added[c] = b.h_exact[c];
                below[c] = (double)b.h_exact[c] < (double)b.threshold;
            }
        }
        if (below[0] && below[1] && below[2]) break;
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev[3], s);
    unsigned long long counts[3] = {0, 0, 0};
    int64_t ntr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts, b.counters, sizeof counts, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && b.nreceivers)
        e = cudaMemcpyAsync(&ntr, b.tr_off + b.nreceivers, sizeof ntr, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = vrad::wait_stream(s);
    if (e == cudaSuccess) {
        b.ntransfers = ntr;
        b.lists_ready = true;
    }
    if (e == cudaSuccess) {
        cudaEventElapsedTime(&b.patch_light_ms, ev[0], ev[1]);
        cudaEventElapsedTime(&b.transfer_ms, ev[1], ev[2]);
        cudaEventElapsedTime(&b.bounce_ms, ev[2], ev[3]);
        b.rays = counts[0];
        b.blocked = counts[1];
        b.open_ties = counts[2];
    } else {
        why = "bounce";
    }
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    return e;
}

bool bounce_active(const vrad_ctx *ctx) { return ctx->bounce.ready && ctx->bounce.max_bounces > 0; }

PatchRadialView patch_radial_view(vrad_ctx *ctx) {
    BounceBuffers &b = ctx->bounce;
    return PatchRadialView{b.pr_off, b.pr_patch, b.pr_box, b.pr_coord, b.total, b.prad_light, b.prad_weight};
}

}  // namespace vrad

extern "C" int32_t vrad_bounce_upload(vrad_ctx *ctx, const vrad_bounce_desc *d) {
    using namespace vrad;
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->has_scene) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    if (!ctx->world.ready || !ctx->final_pass.ready || ctx->h_vertices.empty())
        return vrad_fail(ctx, VRAD_ERR_ARG, "upload the world, with face windings, before the bounce");
    const int32_t nf = (int32_t)ctx->h_faces.size();
    if (!d || (nf && !d->reflectivity) || !d->pvs_offsets || d->nclusters != ctx->nclusters || d->bounces < 0 ||
        !(d->max_chop > 0.0f) || !(d->min_chop > 0.0f) || !(d->threshold >= 0.0f))
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid bounce description");
    const int32_t C = d->nclusters;
    for (int32_t c = 0; c < C; c++) {
        if (d->pvs_offsets[c] > d->pvs_offsets[c + 1]) return vrad_fail(ctx, VRAD_ERR_ARG, "PVS offsets decrease at %d", c);
        for (int32_t k = d->pvs_offsets[c]; k < d->pvs_offsets[c + 1]; k++) {
            const int32_t j = d->pvs_clusters[k];
            if (j < 0 || j >= C || (k > d->pvs_offsets[c] && j <= d->pvs_clusters[k - 1]))
                return vrad_fail(ctx, VRAD_ERR_ARG, "PVS row %d is not ascending clusters", c);
        }
    }
    for (int32_t f = 0; f < nf; f++)
        if (ctx->h_faces[(size_t)f].flags & VRAD_SURF_BUMPLIGHT)
            return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "face %d is bump-mapped", f);

    SetupClock clock("bounce_upload");
    cudaError_t e = cudaSetDevice(ctx->device);
    // The old bounce's blocks go back to the device pool: no kernel of
    // this context may still read them.  Light passes leave none running
    // (one on a caller's stream joined the context's stream), and the
    // direct gather queued ahead, which this upload overlaps, reads no
    // bounce table.
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    BounceBuffers &b = ctx->bounce;
    b.release();
    clock.mark("release");
    // The patch tree, its patches written straight into the device's SoA
    // rows (and each leaf's cluster, for the receiver order) as the merge
    // numbers them.
    // The rows go into the context's pinned shelf, from which each reaches
    // the device by one DMA.
    struct SoaRows : PatchSink {
        int32_t C = 0;
        PinnedShelf *shelf = nullptr;
        int32_t n = 0;
        int64_t npoints = 0;
        float4 *origin = nullptr, *normal = nullptr, *mins = nullptr, *maxs = nullptr, *refl = nullptr,
               *points = nullptr;
        int4 *tr = nullptr;
        int2 *wind = nullptr;
        uvector<int32_t> leaf_cluster;
        std::atomic<int32_t> bad{INT32_MAX};
        bool prepare(int32_t np, int64_t npts) override {
            n = np;
            npoints = npts;
            float4 **rows[] = {&origin, &normal, &mins, &maxs, &refl};
            for (int k = 0; k < 5; k++)
                if (shelf->get(k, (size_t)n, rows[k]) != cudaSuccess) return false;
            if (shelf->get(5, (size_t)npoints, &points) != cudaSuccess || shelf->get(6, (size_t)n, &tr) != cudaSuccess ||
                shelf->get(7, (size_t)n, &wind) != cudaSuccess)
                return false;
            leaf_cluster.resize((size_t)n);
            return true;
        }
        void put(int32_t i, const vrad_patch &p, const float *xyz) override {
            if (p.cluster < 0 || p.cluster >= C) {
                int32_t cur = bad.load();
                while (i < cur && !bad.compare_exchange_weak(cur, i)) {
                }
            }
            origin[(size_t)i] = make_float4(p.origin[0], p.origin[1], p.origin[2], p.area);
            normal[(size_t)i] = make_float4(p.normal[0], p.normal[1], p.normal[2], p.plane_dist);
            mins[(size_t)i] = make_float4(p.mins[0], p.mins[1], p.mins[2], bits_f(p.face));
            maxs[(size_t)i] = make_float4(p.maxs[0], p.maxs[1], p.maxs[2], bits_f(p.cluster));
            refl[(size_t)i] = make_float4(p.reflectivity[0], p.reflectivity[1], p.reflectivity[2], 0.0f);
            tr[(size_t)i] = make_int4(p.parent, p.child1, p.child2, p.sky);
            wind[(size_t)i] = make_int2(p.first_point, p.num_points);
            leaf_cluster[(size_t)i] = p.child1 == -1 ? p.cluster : -1;
            for (int32_t k = 0; k < p.num_points; k++)
                points[(size_t)p.first_point + (size_t)k] = make_float4(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], 0.0f);
        }
    };
    PatchTree tree;
    SoaRows rows;
    rows.C = C;
    rows.shelf = &ctx->shelf;
    std::string why;
    const int64_t nvert = (int64_t)ctx->h_vertices.size() / 3;
    // The forest the world upload grew ahead, when its chop sizes are this
    // upload's; otherwise grown here.
    vrad::join_ahead(ctx);
    PatchForest forest = std::move(ctx->ahead);
    const bool ahead = ctx->ahead_ok && forest.grown() && forest.max_chop() == d->max_chop &&
                       forest.min_chop() == d->min_chop;
    ctx->ahead = PatchForest();
    ctx->ahead_ok = false;
    if (!(ahead || forest.grow(ctx->h_faces.data(), nf, ctx->h_vertices.data(), nvert, d->max_chop, d->min_chop,
                               why)) ||
        !forest.merge(d->reflectivity, tree, rows, why))
        return vrad_fail(ctx, VRAD_ERR_ARG, "patches: %s", why.c_str());
    forest = PatchForest();
    const int32_t P = tree.npatches;
    clock.mark("patch tree");
    if (rows.bad.load() != INT32_MAX)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "patch %d lies outside every cluster", rows.bad.load());
    const int4 *tr = rows.tr;
    const uvector<int32_t> &leaf_cluster = rows.leaf_cluster;
    // The rows' DMAs start now and run under the host work that follows.
    const cudaStream_t rs = ctx->stream;
    cudaError_t e_rows = dma_table(&b.origin, rows.origin, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.normal, rows.normal, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.mins, rows.mins, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.maxs, rows.maxs, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.refl, rows.refl, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.tree, rows.tr, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.wind, rows.wind, (size_t)P, rs);
    if (e_rows == cudaSuccess) e_rows = dma_table(&b.points, rows.points, (size_t)rows.npoints, rs);
    // Per face.
    std::vector<int4> face_range((size_t)nf);
    std::vector<int2> face_samples((size_t)nf, make_int2(0, 0));
    std::vector<float4> face_plane((size_t)nf);
    for (int32_t f = 0; f < nf; f++) {
        face_range[(size_t)f] = make_int4(tree.face_root[(size_t)f], tree.face_first[(size_t)f], tree.face_end[(size_t)f], 0);
        const vrad_face &fc = ctx->h_faces[(size_t)f];
        face_plane[(size_t)f] = make_float4(fc.normal[0], fc.normal[1], fc.normal[2], fc.dist);
    }
    // Each face's sample run (first sample, count) and the samples' areas,
    // as the world upload recorded them.
    face_samples = ctx->h_face_samples;
    const uvector<float> &sample_area = ctx->h_sample_area;
    clock.mark("patch tables");
    // VisMatrix.ReceiverOrder: cluster by cluster, leaf patches in index
    // order (a stable counting sort on the leaves' clusters), and the
    // sky-free leaves in descending index order; both in chunks of patches
    // on worker threads, each chunk's place found from the counts of the
    // chunks before it.
    constexpr int32_t kChunk = 1 << 16;
    const int32_t nchunks = (P + kChunk - 1) / kChunk;
    std::vector<int32_t> ccount((size_t)nchunks * (size_t)(C + 1), 0);  // per chunk: C cluster counts, sky-free leaves
    parallel_for(nchunks, 1, [&](int64_t k) {
        int32_t *cc = &ccount[(size_t)k * (size_t)(C + 1)];
        for (int32_t i = (int32_t)k * kChunk; i < std::min(P, (int32_t)(k + 1) * kChunk); i++) {
            if (leaf_cluster[(size_t)i] >= 0) cc[leaf_cluster[(size_t)i]]++;
            if (tr[(size_t)i].y == -1 && !tr[(size_t)i].w) cc[C]++;
        }
    });
    std::vector<int32_t> cstart((size_t)C + 1, 0);
    std::vector<int32_t> chunk_at((size_t)nchunks * (size_t)(C + 1));
    for (int32_t c = 0; c < C; c++) {
        int32_t at = cstart[(size_t)c];
        for (int32_t k = 0; k < nchunks; k++) {
            chunk_at[(size_t)k * (size_t)(C + 1) + c] = at;
            at += ccount[(size_t)k * (size_t)(C + 1) + c];
        }
        cstart[(size_t)c + 1] = at;
    }
    int32_t nleaves = 0;
    for (int32_t k = nchunks - 1; k >= 0; k--) {
        chunk_at[(size_t)k * (size_t)(C + 1) + C] = nleaves;
        nleaves += ccount[(size_t)k * (size_t)(C + 1) + C];
    }
    uvector<int32_t> recv((size_t)cstart[(size_t)C]), leaf_desc((size_t)nleaves), leaf_rank((size_t)P, -1);
    parallel_for(nchunks, 1, [&](int64_t k) {
        int32_t *at = &chunk_at[(size_t)k * (size_t)(C + 1)];
        const int32_t lo = (int32_t)k * kChunk, hi = std::min(P, (int32_t)(k + 1) * kChunk);
        for (int32_t i = lo; i < hi; i++)
            if (leaf_cluster[(size_t)i] >= 0) recv[(size_t)at[leaf_cluster[(size_t)i]]++] = i;
        for (int32_t i = hi - 1; i >= lo; i--)
            if (tr[(size_t)i].y == -1 && !tr[(size_t)i].w) {
                leaf_rank[(size_t)i] = at[C];
                leaf_desc[(size_t)at[C]++] = i;
            }
    });
    // Each parent's level (1 + its deeper child's; leaves 0): a face's
    // tree is its root and its descendants, children numbered above their
    // parent, so one descending pass per face, faces in parallel; then the
    // parents grouped by level, index order within a level.
    uvector<uint8_t> level((size_t)P, 0);
    std::vector<int32_t> face_top((size_t)nf, 0);
    parallel_for(nf, 16, [&](int64_t f) {
        const int32_t root = tree.face_root[(size_t)f];
        if (root < 0) return;
        int32_t top_f = 0;
        auto visit = [&](int32_t i) {
            const int4 t = tr[(size_t)i];
            if (t.y == -1) return;
            const int h = 1 + std::max(level[(size_t)t.y], level[(size_t)t.z]);
            level[(size_t)i] = (uint8_t)std::min(h, 255);
            top_f = std::max(top_f, h);
        };
        for (int32_t i = tree.face_end[(size_t)f] - 1; i >= tree.face_first[(size_t)f]; i--) visit(i);
        visit(root);
        face_top[(size_t)f] = top_f;
    });
    int32_t top = 0;
    for (int32_t f = 0; f < nf; f++) top = std::max(top, face_top[(size_t)f]);
    if (top > 255) {
        vrad::wait_stream(rs);  // no DMA still reads the shelf or writes a released block
        b.release();
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "a patch's subtree is deeper than 255 levels");
    }
    std::vector<int32_t> level_off((size_t)top + 2, 0);
    for (int32_t i = 0; i < P; i++)
        if (level[(size_t)i]) level_off[(size_t)level[(size_t)i] + 1]++;
    for (int32_t h = 0; h <= top; h++) level_off[(size_t)h + 1] += level_off[(size_t)h];
    uvector<int32_t> level_patch((size_t)level_off[(size_t)top + 1]);
    {
        std::vector<int32_t> at(level_off.begin(), level_off.end() - 1);
        for (int32_t i = 0; i < P; i++)
            if (level[(size_t)i]) level_patch[(size_t)at[level[(size_t)i]]++] = i;
    }
    // FacesInRow: each visible cluster's faces, in face order (one leaf per
    // cluster, whose faces are the faces that lie in it).
    std::vector<std::vector<int32_t>> cluster_faces((size_t)C);
    for (int32_t f = 0; f < nf; f++) cluster_faces[(size_t)ctx->h_faces[(size_t)f].cluster].push_back(f);
    std::vector<int32_t> row_off((size_t)C + 1, 0), row_faces;
    for (int32_t c = 0; c < C; c++) {
        for (int32_t k = d->pvs_offsets[c]; k < d->pvs_offsets[c + 1]; k++) {
            const auto &fl = cluster_faces[(size_t)d->pvs_clusters[k]];
            row_faces.insert(row_faces.end(), fl.begin(), fl.end());
        }
        row_off[(size_t)c + 1] = (int32_t)row_faces.size();
    }
    clock.mark("receivers and rows");
    // The final pass's patch tables over the smoothing neighbours (the
    // world upload's).
    if (ctx->h_noff.size() != (size_t)nf + 1) {
        vrad::wait_stream(rs);  // no DMA still reads the shelf or writes a released block
        b.release();
        return vrad_fail(ctx, VRAD_ERR_ARG, "the world has no smoothing neighbours");
    }
    const std::vector<int32_t> &noff = ctx->h_noff, &nlist = ctx->h_nlist;
    clock.mark("neighbours");

    const int32_t R = (int32_t)recv.size();
    const int64_t ncells = ctx->final_pass.view.ncells;
    if (e == cudaSuccess) e = e_rows;
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.face_range, face_range);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.face_samples, face_samples);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.face_plane, face_plane);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.recv, recv);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.leaf_desc, leaf_desc);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.leaf_rank, leaf_rank);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.level_patch, level_patch);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.row_off, row_off);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.row_faces, row_faces);
    if (e == cudaSuccess) e = stage_table(ctx->stager, ctx->stream, &b.sample_area, sample_area);
    clock.mark("tables copied");
    const size_t P1 = (size_t)(P ? P : 1), R1 = (size_t)R + 1, N1 = (size_t)(ncells ? ncells : 1);
    if (e == cudaSuccess) e = dev_alloc(&b.cand_off, sizeof(int64_t) * R1);
    if (e == cudaSuccess) e = dev_alloc(&b.tr_off, sizeof(int64_t) * R1);
    for (float4 **q : {&b.acc, &b.direct, &b.total, &b.emit[0], &b.emit[1], &b.shoot[0], &b.shoot[1]})
        if (e == cudaSuccess) e = dev_alloc(q, sizeof(float4) * P1);
    if (e == cudaSuccess) e = dev_alloc(&b.sums, kSums * sizeof(double));
    if (e == cudaSuccess) e = dev_alloc(&b.exact, 3 * sizeof(float));
    if (e == cudaSuccess) e = dev_alloc(&b.counters, 3 * sizeof(unsigned long long));
    if (e == cudaSuccess && !b.h_sums) e = cudaMallocHost(&b.h_sums, kSums * sizeof(double));
    if (e == cudaSuccess && !b.h_exact) e = cudaMallocHost(&b.h_exact, 3 * sizeof(float));
    if (e == cudaSuccess) e = dev_alloc(&b.first, sizeof(float4) * P1);
    if (e == cudaSuccess) e = dev_alloc(&b.guess, sizeof(float4) * P1);
    if (e == cudaSuccess) e = dev_alloc(&b.feat, sizeof(uint16_t) * kFeatures * (size_t)(R ? R : 1));
    if (e == cudaSuccess) e = dev_alloc(&b.pred, sizeof(float) * 3 * (size_t)(R ? R : 1));
    if (e == cudaSuccess) e = dev_alloc(&b.prad_light, sizeof(float4) * N1);
    if (e == cudaSuccess) e = dev_alloc(&b.prad_weight, sizeof(float) * N1);
    const int32_t nslices = (R + 31) / 32;
    if (e == cudaSuccess && R > 0) {
        // One scan buffer for the receiver scans and the slice scan; one
        // sort buffer for the slices' count order.
        size_t need = 0, need2 = 0;
        e = cub::DeviceScan::InclusiveSum(nullptr, need, b.cand_off + 1, b.cand_off + 1, R);
        if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, need2, b.cand_off + 1, b.cand_off + 1, nslices);
        need = std::max(need, need2);
        if (e == cudaSuccess) e = dev_alloc(&b.scan_tmp, need ? need : 1);
        b.scan_tmp_bytes = need;
        size_t sort = 0;
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairsDescending(nullptr, sort, (const int32_t *)nullptr, (int32_t *)nullptr,
                                                          (const int32_t *)nullptr, (int32_t *)nullptr, R, 0, 20);
        if (e == cudaSuccess) e = dev_alloc(&b.sort_tmp, sort ? sort : 1);
        b.sort_tmp_bytes = sort;
    }
    for (int32_t **q : {&b.sell_key, &b.sell_idx, &b.sell_count, &b.sell_order})
        if (e == cudaSuccess) e = dev_alloc(q, sizeof(int32_t) * (size_t)(R ? R : 1));
    if (e == cudaSuccess) e = dev_alloc(&b.sell_off, sizeof(int64_t) * ((size_t)nslices + 1));
    if (e != cudaSuccess) {
        ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        b.release();
        return vrad_cuda_fail(ctx, e, "bounce upload");
    }
    clock.mark("device buffers");
    b.npatches = P;
    b.nfaces = nf;
    b.nreceivers = R;
    b.nleaves = nleaves;
    b.max_bounces = d->bounces;
    b.threshold = d->threshold;
    b.h_recv = recv;
    b.h_level_off = level_off;
    b.view = BounceView{P, nf, R, b.origin, b.normal, b.mins, b.maxs, b.tree, b.refl, b.wind, b.points,
                        b.face_range, b.face_samples, b.face_plane, b.recv, b.row_off, b.row_faces, b.sample_area,
                        ctx->world.sample_pos};
    cudaStream_t s = ctx->stream;
    // The final pass's patch tables over the smoothing neighbours, on the
    // device from the uploaded patches.
    e = radial_tables(b, ctx->final_pass.frames, nf, noff, nlist, ctx->stager, s);
    if (e != cudaSuccess) {
        ctx->stager.finish(s);
        b.release();
        return vrad_cuda_fail(ctx, e, "patch radial tables");
    }
    clock.mark("patch radial tables");
    // Size the candidate and transfer arrays by one build.  The walk's
    // overflow flag is a status word of its own (status[1]): a direct
    // gather queued ahead may be running beside this upload.
    uint32_t *walk_flag = ctx->status + 1;
    if (e == cudaSuccess) e = cudaMemsetAsync(walk_flag, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) e = launch_transfers(b, ctx->scene.view(), walk_flag, s, true);
    int64_t ncand = 0;
    if (e == cudaSuccess && R > 0) e = cudaMemcpyAsync(&ncand, b.cand_off + R, sizeof ncand, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = vrad::wait_stream(s);
    b.ncand = ncand;
    clock.mark("candidate count");
    if (e == cudaSuccess) e = dev_alloc(&b.cand_src, sizeof(int32_t) * (size_t)(ncand ? ncand : 1));
    if (e == cudaSuccess) e = dev_alloc(&b.cand_w, sizeof(float) * (size_t)(ncand ? ncand : 1));
    // Transfers are at most the candidates: the list array takes that
    // bound, so sizing needs no trace.
    uint32_t overflow = 0;
    if (e == cudaSuccess) e = dev_alloc(&b.tr, sizeof(int2) * (size_t)(ncand ? ncand : 1));
    // The slices hold the transfers and at most 32 times the largest count
    // of padding.
    const int64_t sell_cap = ncand + 32 * std::min<int64_t>(kMaxTransfersPerReceiver, ncand);
    if (e == cudaSuccess) e = dev_alloc(&b.sell, sizeof(int2) * (size_t)(sell_cap ? sell_cap : 1));
    if (e == cudaSuccess) e = cudaMemcpyAsync(&overflow, walk_flag, sizeof overflow, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = vrad::wait_stream(s);
    if (e != cudaSuccess) {
        ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        b.release();
        return vrad_cuda_fail(ctx, e, "transfer sizing");
    }
    if (overflow) {
        cudaMemsetAsync(walk_flag, 0, sizeof(uint32_t), ctx->stream);
        ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        b.release();
        return vrad_fail(ctx, VRAD_ERR_CUDA, "stack overflow in the candidate walk (flags %u)", overflow);
    }
    e = ctx->stager.finish(s);
    if (e != cudaSuccess) {
        b.release();
        return vrad_cuda_fail(ctx, e, "bounce upload");
    }
    clock.mark("candidate sizing");
    const int64_t ntr = 0;
    b.ntransfers = ntr;
    b.ready = true;
    ctx->bounced = true;
    ctx->last_max_chop = d->max_chop;
    ctx->last_min_chop = d->min_chop;
    return VRAD_OK;
}

namespace vrad {
void fill_bounce_stats(const vrad_ctx *ctx, vrad_bounce_stats *st) {
    const vrad::BounceBuffers &b = ctx->bounce;
    std::memset(st, 0, sizeof *st);
    st->patches = b.npatches;
    st->receivers = b.nreceivers;
    st->transfer_rays = (int64_t)b.rays;
    st->blocked = (int64_t)b.blocked;
    st->transfers = b.ntransfers;
    st->bounces = b.bounces_run;
    st->exact_totals = b.exact_totals;
    for (int c = 0; c < 3; c++) st->added[c] = b.added[c];
    st->patch_light_ms = b.patch_light_ms;
    st->transfer_ms = b.transfer_ms;
    st->bounce_ms = b.bounce_ms;
    st->final_ms = b.final_ms;
    st->unsettled_asin = (int64_t)b.open_ties;
    st->transfers_cached = b.installed ? 1 : 0;
}
}  // namespace vrad

extern "C" int32_t vrad_bounce_stats_get(vrad_ctx *ctx, vrad_bounce_stats *st) {
    if (!ctx || !st) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    if (!ctx->bounce.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce uploaded");
    vrad::fill_bounce_stats(ctx, st);
    return VRAD_OK;
}

extern "C" int32_t vrad_bounce_patch_light(vrad_ctx *ctx, float *total_light, float *direct_light, int64_t npatches) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::BounceBuffers &b = ctx->bounce;
    if (!b.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce uploaded");
    if (npatches != b.npatches) return vrad_fail(ctx, VRAD_ERR_ARG, "%d patches, %lld asked", b.npatches, (long long)npatches);
    std::vector<float4> tmp((size_t)(npatches ? npatches : 1));
    cudaError_t e = cudaSetDevice(ctx->device);
    for (int k = 0; k < 2 && e == cudaSuccess; k++) {
        float *dst = k == 0 ? total_light : direct_light;
        if (!dst || npatches == 0) continue;
        e = cudaMemcpy(tmp.data(), k == 0 ? b.total : b.direct, sizeof(float4) * (size_t)npatches, cudaMemcpyDeviceToHost);
        for (int64_t i = 0; e == cudaSuccess && i < npatches; i++) {
            dst[3 * i] = tmp[(size_t)i].x;
            dst[3 * i + 1] = tmp[(size_t)i].y;
            dst[3 * i + 2] = tmp[(size_t)i].z;
        }
    }
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "patch light download");
    return VRAD_OK;
}

extern "C" int32_t vrad_bounce_transfers(vrad_ctx *ctx, int64_t *offsets, int64_t npatches, vrad_transfer *transfers,
                                         int64_t capacity, int64_t *count) {
    if (!ctx || !offsets || !count) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::BounceBuffers &b = ctx->bounce;
    if (!b.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce uploaded");
    if (npatches != b.npatches) return vrad_fail(ctx, VRAD_ERR_ARG, "%d patches, %lld asked", b.npatches, (long long)npatches);
    const int32_t R = b.nreceivers;
    std::vector<int64_t> off((size_t)R + 1, 0);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess && R) e = cudaMemcpy(off.data(), b.tr_off, sizeof(int64_t) * ((size_t)R + 1), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "transfer download");
    std::vector<int64_t> len((size_t)npatches, 0), from((size_t)npatches, 0);
    for (int32_t r = 0; r < R; r++) {
        len[(size_t)b.h_recv[(size_t)r]] = off[(size_t)r + 1] - off[(size_t)r];
        from[(size_t)b.h_recv[(size_t)r]] = off[(size_t)r];
    }
    offsets[0] = 0;
    for (int64_t p = 0; p < npatches; p++) offsets[p + 1] = offsets[p] + len[(size_t)p];
    *count = offsets[npatches];
    if (!transfers) return VRAD_OK;
    if (capacity < *count) return vrad_fail(ctx, VRAD_ERR_ARG, "%lld transfers, room for %lld", (long long)*count, (long long)capacity);
    std::vector<int2> all((size_t)(off[(size_t)R] ? off[(size_t)R] : 1));
    if (off[(size_t)R]) e = cudaMemcpy(all.data(), b.tr, sizeof(int2) * (size_t)off[(size_t)R], cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "transfer download");
    for (int64_t p = 0; p < npatches; p++)
        for (int64_t k = 0; k < len[(size_t)p]; k++) {
            const int2 t = all[(size_t)(from[(size_t)p] + k)];
            transfers[offsets[p] + k].patch = t.x;
            std::memcpy(&transfers[offsets[p] + k].weight, &t.y, 4);
        }
    return VRAD_OK;
}

extern "C" int32_t vrad_bounce_last_total(vrad_ctx *ctx, float *total) {
    if (!ctx || !total) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::BounceBuffers &b = ctx->bounce;
    if (!b.ready || b.bounces_run == 0) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce has run");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = vrad::launch_exact_total(b, b.bounces_run - 1, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.h_exact, b.exact, 3 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "bounce total");
    for (int c = 0; c < 3; c++) total[c] = b.h_exact[c];
    return VRAD_OK;
}

namespace {

__global__ void k_targets(vrad::BounceView v, const float4 *__restrict__ total, float *__restrict__ t) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= v.nreceivers) return;
    const float4 x = total[__ldg(&v.recv[r])];
    t[3 * (int64_t)r] = log1pf(fmaxf(x.x, 0.0f));
    t[3 * (int64_t)r + 1] = log1pf(fmaxf(x.y, 0.0f));
    t[3 * (int64_t)r + 2] = log1pf(fmaxf(x.z, 0.0f));
}

}  // namespace

extern "C" int32_t vrad_bounce_set_model(vrad_ctx *ctx, const vrad_mlp *model) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->bounce_model = model;
    return VRAD_OK;
}

extern "C" int32_t vrad_bounce_features_device(vrad_ctx *ctx, uint16_t *x, float *target, int64_t capacity,
                                               int64_t *count, void *stream) {
    if (!ctx || !count) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::BounceBuffers &b = ctx->bounce;
    if (!b.ready || b.bounces_run == 0) return vrad_fail(ctx, VRAD_ERR_ARG, "no bounce has run");
    *count = b.nreceivers;
    if (!x && !target) return VRAD_OK;
    if (capacity < b.nreceivers) return vrad_fail(ctx, VRAD_ERR_ARG, "%d receivers, room for %lld", b.nreceivers, (long long)capacity);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess && x) e = vrad::launch_features(b, ctx->world.view, s);
    if (e == cudaSuccess && x)
        e = cudaMemcpyAsync(x, b.feat, sizeof(uint16_t) * vrad::kFeatures * (size_t)b.nreceivers, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && target && b.nreceivers) {
        k_targets<<<(b.nreceivers + 127) / 128, 128, 0, s>>>(b.view, b.total, target);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "bounce features");
    return VRAD_OK;
}
