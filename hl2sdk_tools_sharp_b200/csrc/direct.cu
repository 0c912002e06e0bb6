// direct.cu -- the fused direct-lighting gather: per luxel sample, every
// light of its cluster's list in gather order, each shadow, sun and sky
// segment traced in-thread, accumulated into the sample's LightingValue.
//
// Reference behaviour restated (muflub/hl2sdk_tools_sharp, MapTools/Rad/Light):
//   FaceLightJob.ComputeIlluminationPointAndNormals (FaceLightJob.cs:237-320):
//       the point is the sample position plus the face normal;
//   FaceLightJob.EmitGroup / ResolveGroup (FaceLightJob.cs:329-460): lights in
//       list order, fxdot = (mask ? dot : 0) * falloff, a light skipped when
//       every lane of the four-sample group has fxdot 0, AddLight otherwise;
//   DirectLightGatherer.GatherPointFour (:1308-1420), GatherStandardLane
//       (:1169-1306, spotlights), EmitSkyLight / ResolveSkyLight (:536-640),
//       AmbientSky (:642-815), Resolve's dot clamp (:441-478),
//       InverseQuadratic (:1579).
// Every float operation is an explicitly rounded intrinsic in the
// reference's order, so a sample's result is the CPU's bits whenever the
// rays answer as the CPU's do.  The four-sample group is four adjacent
// lanes; its "every lane zero" tests are shuffles within the group.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "context.cuh"
#include "device_pool.h"
#include "gather.cuh"
#include "host_parallel.h"
#include "setup_clock.h"
#include "supersample.cuh"
#include "sync_wait.h"

namespace vrad {

namespace {

// BLOCK threads per CTA (32, 64 or 128, chosen by vrad_direct_autotune):
// every thread traces its samples' whole light list, so a small CTA frees
// its SM slot as soon as its own warps are done.
// DUAL: one traversal lights both ranges (out from w.lights, out_hdr from
// w.lights_hdr).
template <int BLOCK, bool DUAL>
__global__ void __launch_bounds__(BLOCK) k_direct(DeviceScene sc, DeviceWorld w, float4 *__restrict__ out,
                                                  float4 *__restrict__ out_hdr,
                                                  unsigned long long *__restrict__ counters,
                                                  uint32_t *__restrict__ overflow) {
    extern __shared__ int stack_mem[];  // sc.stack_depth() entries per thread
    int *stack = stack_mem + threadIdx.x;
    const int64_t slot = (int64_t)blockIdx.x * BLOCK + threadIdx.x;
    // nslots is a multiple of 32 and every warp's slots share one cluster
    // (vrad_world_upload lays them out so), so the light loop is
    // warp-uniform and the __syncwarp()s below keep the lanes in step: a
    // warp traces one light (or one sky direction) at a time, coherently.
    if (slot >= w.nslots) return;
    const int32_t code = __ldg(&w.slots[slot]);
    const int lane = threadIdx.x & 31;
    const unsigned gmask = 0xFu << (lane & ~3);
    const bool real = (code & 0x80000000) == 0;
    const int32_t si = code & 0x7fffffff;

    const float4 sp = __ldg(&w.sample_pos[si]);
    const int face = __float_as_int(sp.w);
    const float4 fn = __ldg(&w.face_normal[face]);
    const int cluster = __float_as_int(fn.w);
    const float nx = fn.x, ny = fn.y, nz = fn.z;
    // One unit off the face (ComputeIlluminationPointAndNormals).
    const float px = __fadd_rn(sp.x, nx), py = __fadd_rn(sp.y, ny), pz = __fadd_rn(sp.z, nz);

    unsigned long long vis_rays = 0, sky_rays = 0;
    float4 h;
    // The group's first sample (a face's groups start on lanes 0, 4, ...):
    // groups in sample order are ResolveGroup's order.
    const unsigned long long key_group = (unsigned long long)(uint32_t)__shfl_sync(kFull, si, lane & ~3) << 32;
    const float4 r = gather_point<BLOCK, DUAL>(sc, w, cluster, px, py, pz, nx, ny, nz, real, gmask, kAllLights,
                                               stack, overflow, counters, vis_rays, sky_rays, &h, face, key_group);
    if (real) {
        out[si] = r;
        if (DUAL) out_hdr[si] = h;
    }

    // Ray counts: one atomic per warp.
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

}  // namespace

void StyleState::release() {
    for (int r = 0; r < 2; r++) {
        for (float4 *p : light[r]) dev_free(p);
        light[r].clear();
    }
    dev_free(keys);
    dev_free(slots);
    keys = nullptr;
    slots = nullptr;
    styles.clear();
    face_styles.clear();
    dropped = 0;
    ready = false;
}

void WorldBuffers::release() {
    dev_free(slots);
    dev_free(sample_pos);
    dev_free(face_normal);
    dev_free(lights);
    dev_free(lights_hdr);
    dev_free(cl_off);
    dev_free(cl_list);
    dev_free(dirs);
    dev_free(jitter);
    dev_free(counters);
    slots = nullptr;
    sample_pos = face_normal = lights = lights_hdr = dirs = jitter = nullptr;
    cl_off = cl_list = nullptr;
    counters = nullptr;
    view = DeviceWorld{};
    ready = false;
}

cudaError_t launch_direct(const DeviceScene &scene, const DeviceWorld &world, float4 *out, float4 *out_hdr,
                          unsigned long long *counters, uint32_t *overflow, cudaStream_t stream,
                          int block) {
    if (world.nslots == 0) return cudaSuccess;
    if (out_hdr && !world.lights_hdr) return cudaErrorInvalidValue;
    const size_t smem = sizeof(int) * (size_t)scene.stack_depth();  // per thread
    const unsigned g32 = (unsigned)((world.nslots + 31) / 32), g64 = (unsigned)((world.nslots + 63) / 64),
                   g128 = (unsigned)((world.nslots + 127) / 128);
    if (out_hdr) {
        switch (block) {
            case 32: k_direct<32, true><<<g32, 32, smem * 32, stream>>>(scene, world, out, out_hdr, counters, overflow); break;
            case 64: k_direct<64, true><<<g64, 64, smem * 64, stream>>>(scene, world, out, out_hdr, counters, overflow); break;
            default: k_direct<128, true><<<g128, 128, smem * 128, stream>>>(scene, world, out, out_hdr, counters, overflow); break;
        }
    } else {
        switch (block) {
            case 32: k_direct<32, false><<<g32, 32, smem * 32, stream>>>(scene, world, out, nullptr, counters, overflow); break;
            case 64: k_direct<64, false><<<g64, 64, smem * 64, stream>>>(scene, world, out, nullptr, counters, overflow); break;
            default: k_direct<128, false><<<g128, 128, smem * 128, stream>>>(scene, world, out, nullptr, counters, overflow); break;
        }
    }
    return cudaGetLastError();
}

}  // namespace vrad

extern "C" int32_t vrad_world_upload(vrad_ctx *ctx, const vrad_world_desc *w) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (!w || w->nfaces < 0 || w->nsamples < 0 || w->nlights < 0 || w->nclusters < 0 ||
        (w->nfaces && !w->faces) || (w->nsamples && !w->samples) || (w->nlights && !w->lights) ||
        !w->cluster_light_offsets || (w->nsky_directions && !w->sky_directions) ||
        (w->nsun_jitter && !w->sun_jitter) || w->sun_samples < 1 || w->sun_samples - 1 > w->nsun_jitter)
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid world description");
    vrad::SetupClock clock("world_upload");
    const int32_t nl = w->nlights;
    for (int32_t l = 0; l < nl; l++) {
        const int t = w->lights[l].type;
        if (t < 0 || t > 4) return vrad_fail(ctx, VRAD_ERR_ARG, "light %d has type %d", l, t);
        // A face's style slots are bytes, 255 meaning none.
        if (w->lights[l].style < 0 || w->lights[l].style > 254)
            return vrad_fail(ctx, VRAD_ERR_ARG, "light %d has style %d (0 to 254)", l, w->lights[l].style);
    }
    const int32_t total = w->cluster_light_offsets[w->nclusters];
    for (int32_t c = 0; c < w->nclusters; c++)
        if (w->cluster_light_offsets[c] > w->cluster_light_offsets[c + 1])
            return vrad_fail(ctx, VRAD_ERR_ARG, "cluster light offsets decrease at %d", c);
    for (int32_t k = 0; k < total; k++)
        if (w->cluster_lights[k] < 0 || w->cluster_lights[k] >= nl)
            return vrad_fail(ctx, VRAD_ERR_ARG, "cluster light list names light %d", w->cluster_lights[k]);

    // Samples: the runs of one face (marked in parallel, walked in one
    // scan), then the runs' cluster checks and positions in parallel.
    const int64_t ns = w->nsamples;
    vrad::uvector<uint8_t> run_start((size_t)ns + 1);
    vrad::parallel_for(ns, 1 << 16, [&](int64_t k) {
        run_start[(size_t)k] = k == 0 || w->samples[k - 1].face != w->samples[k].face;
    });
    run_start[(size_t)ns] = 1;
    std::vector<int64_t> fstart((size_t)w->nfaces, -1), fend((size_t)w->nfaces, -1);
    std::vector<int32_t> run_face;
    int64_t i = 0;
    while (i < ns) {
        const int32_t face = w->samples[i].face;
        if (face < 0 || face >= w->nfaces) return vrad_fail(ctx, VRAD_ERR_ARG, "sample %lld names face %d", (long long)i, face);
        if (fstart[(size_t)face] != -1)
            return vrad_fail(ctx, VRAD_ERR_ARG, "face %d's samples are not contiguous", face);
        const uint8_t *next = static_cast<const uint8_t *>(memchr(&run_start[(size_t)i + 1], 1, (size_t)(ns - i)));
        const int64_t j = next - run_start.data();
        const int32_t cl = w->faces[face].cluster;
        if (cl < 0 || cl >= w->nclusters)
            return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "face %d has cluster %d outside the light lists", face, cl);
        fstart[(size_t)face] = i;
        fend[(size_t)face] = j;
        run_face.push_back(face);
        i = j;
    }
    // One pass over the samples: positions (with the face), the areas and
    // coords the supersampling rebuild is checked against, the areas the
    // bounce's patch light reads.
    // Positions and the check table go straight into the context's pinned
    // shelf, from which one DMA each sends them (the shelf is the
    // context's: the lock is taken here).
    std::unique_lock<std::mutex> g(ctx->mu);
    float4 *pos = nullptr, *area_coord = nullptr;
    if (ctx->shelf.get(8, (size_t)w->nsamples, &pos) != cudaSuccess ||
        ctx->shelf.get(9, (size_t)w->nsamples, &area_coord) != cudaSuccess)
        return vrad_fail(ctx, VRAD_ERR_OOM, "pinned sample tables");
    vrad::uvector<float> area((size_t)w->nsamples);
    std::atomic<int64_t> mixed{INT64_MAX};
    vrad::parallel_for((int64_t)run_face.size(), 16, [&](int64_t r) {
        const int32_t face = run_face[(size_t)r];
        const int32_t cl = w->faces[face].cluster;
        for (int64_t s = fstart[(size_t)face]; s < fend[(size_t)face]; s++) {
            const vrad_sample &sm = w->samples[s];
            if (sm.cluster != cl) {
                int64_t cur = mixed.load();
                while (s < cur && !mixed.compare_exchange_weak(cur, s)) {
                }
            }
            float4 p;
            p.x = sm.position[0];
            p.y = sm.position[1];
            p.z = sm.position[2];
            int32_t f = face;
            memcpy(&p.w, &f, 4);
            pos[(size_t)s] = p;
            area_coord[(size_t)s] = make_float4(sm.area, sm.coord[0], sm.coord[1], 0.0f);
            area[(size_t)s] = sm.area;
        }
    });
    if (mixed.load() != INT64_MAX) {
        const int64_t s = mixed.load();
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED,
                         "sample %lld is in cluster %d, its face in %d: mixed-cluster groups are not supported",
                         (long long)s, w->samples[s].cluster, w->faces[w->samples[s].face].cluster);
    }
    clock.mark("samples");
    // Slots, cluster by cluster: each face's samples in whole groups of
    // four (the last group repeating its last sample as padding), each
    // cluster's run padded to whole warps with more padding lanes, so no
    // warp mixes two light lists.
    // Laid out face by face first (each face's first slot, each cluster's
    // padding run), then written in parallel.
    std::vector<std::vector<int32_t>> by_cluster((size_t)w->nclusters);
    for (int32_t f = 0; f < w->nfaces; f++)
        if (fstart[(size_t)f] >= 0) by_cluster[(size_t)w->faces[f].cluster].push_back(f);
    std::vector<int64_t> face_slot((size_t)w->nfaces, -1), pad_from((size_t)w->nclusters), pad_to((size_t)w->nclusters);
    std::vector<int32_t> pad_sample((size_t)w->nclusters, -1);
    int64_t nslots = 0;
    for (int32_t c = 0; c < w->nclusters; c++) {
        int32_t last = -1;
        for (int32_t f : by_cluster[(size_t)c]) {
            face_slot[(size_t)f] = nslots;
            nslots += (fend[(size_t)f] - fstart[(size_t)f] + 3) / 4 * 4;
            last = (int32_t)(fend[(size_t)f] - 1);
        }
        pad_from[(size_t)c] = nslots;
        if (last >= 0) nslots = (nslots + 31) / 32 * 32;
        pad_to[(size_t)c] = nslots;
        pad_sample[(size_t)c] = last;
    }
    vrad::uvector<int32_t> slots((size_t)nslots);
    vrad::parallel_for(w->nfaces, 64, [&](int64_t f) {
        if (face_slot[(size_t)f] < 0) return;
        const int64_t a = fstart[(size_t)f], b = fend[(size_t)f];
        int32_t *o = slots.data() + face_slot[(size_t)f];
        for (int64_t s = a; s < (b - a + 3) / 4 * 4 + a; s++)
            *o++ = s < b ? (int32_t)s : (int32_t)((b - 1) | 0x80000000LL);
    });
    for (int32_t c = 0; c < w->nclusters; c++)
        for (int64_t k = pad_from[(size_t)c]; k < pad_to[(size_t)c]; k++)
            slots[(size_t)k] = (int32_t)(pad_sample[(size_t)c] | 0x80000000LL);
    std::vector<float4> fnorm((size_t)w->nfaces);
    for (int32_t f = 0; f < w->nfaces; f++) {
        float4 v;
        v.x = w->faces[f].normal[0];
        v.y = w->faces[f].normal[1];
        v.z = w->faces[f].normal[2];
        int32_t c = w->faces[f].cluster;
        memcpy(&v.w, &c, 4);
        fnorm[(size_t)f] = v;
    }
    auto pack = [nl](const vrad_light *src) {
        std::vector<float4> lights((size_t)nl * vrad::kLightF4);
        for (int32_t l = 0; l < nl; l++) {
            const vrad_light &s = src[l];
            float4 *o = &lights[(size_t)l * vrad::kLightF4];
            int32_t type = s.type, style = s.style;
            o[0] = make_float4(s.origin[0], s.origin[1], s.origin[2], 0.0f);
            memcpy(&o[0].w, &type, 4);
            o[1] = make_float4(s.intensity[0], s.intensity[1], s.intensity[2], 0.0f);
            memcpy(&o[1].w, &style, 4);
            o[2] = make_float4(s.normal[0], s.normal[1], s.normal[2], s.exponent);
            o[3] = make_float4(s.stop_dot, s.stop_dot2, s.constant_attn, s.linear_attn);
            o[4] = make_float4(s.quadratic_attn, s.start_fade_distance, s.end_fade_distance, s.cap_dist);
        }
        return lights;
    };
    const std::vector<float4> lights = pack(w->lights);
    // The HDR list differs from the LDR one in intensity alone (both come
    // from the same entities): every other word must match.
    std::vector<float4> lights_hdr;
    if (w->lights_hdr) {
        lights_hdr = pack(w->lights_hdr);
        for (int32_t l = 0; l < nl; l++)
            for (int k = 0; k < vrad::kLightF4; k++) {
                const float4 &a = lights[(size_t)l * vrad::kLightF4 + k], &b = lights_hdr[(size_t)l * vrad::kLightF4 + k];
                const bool intensity = k == 1;
                if ((!intensity && memcmp(&a, &b, sizeof a) != 0) || (intensity && memcmp(&a.w, &b.w, 4) != 0))
                    return vrad_fail(ctx, VRAD_ERR_ARG, "HDR light %d differs from the LDR light in more than intensity", l);
            }
    }
    std::vector<int32_t> cl_off(w->cluster_light_offsets, w->cluster_light_offsets + w->nclusters + 1);
    std::vector<int32_t> cl_list(w->cluster_lights, w->cluster_lights + total);
    std::vector<float4> dirs((size_t)w->nsky_directions), jit((size_t)w->nsun_jitter);
    for (int32_t d = 0; d < w->nsky_directions; d++)
        dirs[(size_t)d] = make_float4(w->sky_directions[3 * d], w->sky_directions[3 * d + 1], w->sky_directions[3 * d + 2], 0.0f);
    for (int32_t d = 0; d < w->nsun_jitter; d++)
        jit[(size_t)d] = make_float4(w->sun_jitter[3 * d], w->sun_jitter[3 * d + 1], w->sun_jitter[3 * d + 2], 0.0f);

    clock.mark("slots and lights");
    vrad::settle_direct(ctx);
    cudaError_t e = cudaSetDevice(ctx->device);
    // The old world's blocks go back to the device pool: no kernel of this
    // context, on any stream, may still read them.
    if (e == cudaSuccess) e = vrad::quiesce(ctx);
    vrad::WorldBuffers &wb = ctx->world;
    wb.release();
    ctx->styles.release();
    for (int32_t l = 0; l < nl; l++)
        if (w->lights[l].style != 0) ctx->styles.styles.push_back(w->lights[l].style);
    std::sort(ctx->styles.styles.begin(), ctx->styles.styles.end());
    ctx->styles.styles.erase(std::unique(ctx->styles.styles.begin(), ctx->styles.styles.end()),
                             ctx->styles.styles.end());
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.slots, slots);
    if (e == cudaSuccess) e = vrad::dma_table(&wb.sample_pos, pos, (size_t)w->nsamples, ctx->stream);
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.face_normal, fnorm);
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.lights, lights);
    if (e == cudaSuccess && !lights_hdr.empty())
        e = vrad::stage_table(ctx->stager, ctx->stream, &wb.lights_hdr, lights_hdr);
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.cl_off, cl_off);
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.cl_list, cl_list);
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.dirs, dirs);
    if (e == cudaSuccess) e = vrad::stage_table(ctx->stager, ctx->stream, &wb.jitter, jit);
    if (e == cudaSuccess) e = vrad::dev_alloc(&wb.counters, 3 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        wb.release();
        return vrad_cuda_fail(ctx, e, "world upload");
    }
    wb.view = vrad::DeviceWorld{wb.slots, (int64_t)slots.size(), wb.sample_pos, wb.face_normal, wb.lights, nl,
                                wb.cl_off, wb.cl_list, w->nclusters, wb.dirs, w->nsky_directions, wb.jitter,
                                w->nsun_jitter, w->sun_angular_extent, w->sun_samples, w->nsamples,
                                wb.lights_hdr};
    clock.mark("world buffers");
    // The final pass's tables, and the direct gather's output buffer.  A
    // new world drops the old bounce.
    ctx->bounce.release();
    clock.mark("bounce released");
    // The forest grown ahead for the previous world reads the host copies.
    vrad::join_ahead(ctx);
    ctx->ahead = vrad::PatchForest();
    ctx->ahead_ok = false;
    ctx->h_faces.assign(w->faces, w->faces + w->nfaces);
    ctx->h_sample_area.swap(area);
    ctx->h_face_samples.assign((size_t)w->nfaces, make_int2(0, 0));
    for (int32_t f = 0; f < w->nfaces; f++)
        if (fstart[(size_t)f] >= 0)
            ctx->h_face_samples[(size_t)f] =
                make_int2((int32_t)fstart[(size_t)f], (int32_t)(fend[(size_t)f] - fstart[(size_t)f]));
    ctx->h_noff.clear();
    ctx->h_nlist.clear();
    if (w->vertices && w->nvertices > 0) ctx->h_vertices.assign(w->vertices, w->vertices + 3 * w->nvertices);
    else ctx->h_vertices.clear();
    ctx->nclusters = w->nclusters;
    if (ctx->bounced && !ctx->h_vertices.empty()) {
        // PatchBuilder and PatchSubdivider need only the faces and their
        // windings: grow the forest while the final-pass and supersampling
        // tables are built (their parallel loops and the forest's share the
        // host pool).
        const float mx = ctx->last_max_chop, mn = ctx->last_min_chop;
        ctx->ahead_thread = std::thread([ctx, mx, mn]() {
            ctx->ahead_ok = ctx->ahead.grow(ctx->h_faces.data(), (int32_t)ctx->h_faces.size(), ctx->h_vertices.data(),
                                            (int64_t)ctx->h_vertices.size() / 3, mx, mn, ctx->ahead_why);
        });
    }
    ctx->final_pass.release();
    vrad::dev_free(ctx->sample_light);
    ctx->sample_light = nullptr;
    vrad::dev_free(ctx->sample_light_hdr);
    ctx->sample_light_hdr = nullptr;
    clock.mark("host copies");
    if (w->vertices && w->nvertices > 0) {
        std::string why;
        e = vrad::build_final(ctx->final_pass, w->faces, w->nfaces, w->samples, w->nsamples, w->vertices,
                              w->nvertices, ctx->h_noff, ctx->h_nlist, ctx->stager, ctx->stream, why, fstart.data(),
                              fend.data());
        if (e != cudaSuccess) {
            ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        wb.release();
            if (e == cudaErrorInvalidValue) return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "final pass: %s", why.c_str());
            return vrad_cuda_fail(ctx, e, why.c_str());
        }
        clock.mark("final pass tables");
        ctx->final_pass.view.sample_pos = wb.sample_pos;
        bool have = false;
        e = vrad::build_supersample(ctx->supersample, ctx->h_faces, ctx->h_vertices, area_coord, w->nsamples,
                                    ctx->final_pass,
                                    w->nclusters, ctx->stager, ctx->stream, have, why);
        if (e != cudaSuccess) {
            ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        wb.release();
            ctx->final_pass.release();
            return vrad_cuda_fail(ctx, e, why.c_str());
        }
        ctx->supersample_why = have ? std::string() : why;
        clock.mark("supersample tables");
    } else {
        ctx->supersample.release();
        ctx->supersample_why = "the world was uploaded without face windings";
    }
    e = vrad::dev_alloc(&ctx->sample_light, sizeof(float4) * (size_t)(w->nsamples ? w->nsamples : 1));
    if (e == cudaSuccess && wb.lights_hdr)
        e = vrad::dev_alloc(&ctx->sample_light_hdr, sizeof(float4) * (size_t)(w->nsamples ? w->nsamples : 1));
    if (e != cudaSuccess) {
        ctx->stager.finish(ctx->stream);  // no copy in flight into a released block
        wb.release();
        ctx->final_pass.release();
        return vrad_cuda_fail(ctx, e, "sample light buffer");
    }
    e = ctx->stager.finish(ctx->stream);
    if (e != cudaSuccess) {
        wb.release();
        ctx->final_pass.release();
        return vrad_cuda_fail(ctx, e, "world upload");
    }
    wb.ready = true;
    vrad::start_direct_ahead(ctx);
    return VRAD_OK;
}

namespace {

// The direct gather with its supersampling passes: LDR into ldr_out, HDR
// into hdr_out (either may be null, not both).  With both, the first round
// is one traversal for the two ranges; each range then has its own
// supersampling passes (their selections follow each range's gradients).
int32_t direct_on(vrad_ctx *ctx, float4 *ldr_out, float4 *hdr_out, cudaStream_t s) {
    if (!ctx->has_scene) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    if (!ctx->world.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no lighting world uploaded");
    if (hdr_out && !ctx->world.view.lights_hdr)
        return vrad_fail(ctx, VRAD_ERR_ARG, "the world was uploaded without an HDR light list");
    if (ctx->supersample.extra_passes > 0 && !ctx->supersample.ready && ctx->world.view.nsamples)
        return vrad_fail(ctx, VRAD_ERR_UNSUPPORTED, "supersampling: %s (vrad_set_extra_passes 0 turns it off)",
                         ctx->supersample_why.c_str());
    const vrad::DeviceWorld ldr = vrad::range_view(ctx->world.view, false);
    const vrad::DeviceWorld hdr = hdr_out ? vrad::range_view(ctx->world.view, true) : ldr;
    cudaError_t e = cudaMemsetAsync(ctx->world.counters, 0, 3 * sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
        if (ldr_out && hdr_out)
            e = vrad::launch_direct(ctx->scene.view(), ctx->world.view, ldr_out, hdr_out, ctx->world.counters,
                                    ctx->status, s, ctx->world.block);
        else
            e = vrad::launch_direct(ctx->scene.view(), ldr_out ? ldr : hdr, ldr_out ? ldr_out : hdr_out, nullptr,
                                    ctx->world.counters, ctx->status, s, ctx->world.block);
    }
    // The supersampling passes (FaceLightJob's rounds after the first),
    // per range.
    for (int r = 0; r < 2; r++) {
        float4 *out = r == 0 ? ldr_out : hdr_out;
        vrad::SupersampleBuffers &ss = ctx->supersample;
        ctx->range_ss[r] = vrad::RangeSupersample{};
        if (!out || e != cudaSuccess) continue;
        e = vrad::run_supersample(ss, ctx->scene.view(), r == 0 ? ldr : hdr, ctx->final_pass.view, out,
                                  ctx->world.counters, ctx->status, s);
        ctx->range_ss[r] = vrad::RangeSupersample{ss.passes_run, ss.supersampled, ss.ms};
    }
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "direct lighting launch");
    return VRAD_OK;
}

}  // namespace

namespace vrad {
void start_direct_ahead(vrad_ctx *ctx) {
    if (!ctx->has_scene || !ctx->world.ready || !ctx->final_pass.ready || !ctx->sample_light || !ctx->ahead_stream)
        return;
    const cudaStream_t s = ctx->pass_stream ? ctx->pass_stream : ctx->ahead_stream;
    ctx->direct_ahead = true;
    ctx->direct_ahead_rc = VRAD_ERR_CUDA;
    // Every range the world has: a world with an HDR list is lit in both.
    ctx->ahead_ranges = VRAD_RANGE_LDR | (ctx->sample_light_hdr ? VRAD_RANGE_HDR : 0);
    ctx->direct_thread = std::thread([ctx, s]() {
        // The thread sleeps in its waits: its core goes to the bounce
        // upload's host work meanwhile.
        set_sleeping_waits(true);
        int32_t rc = cudaSetDevice(ctx->device) == cudaSuccess && cudaEventRecord(ctx->ahead_start, s) == cudaSuccess
                         ? direct_on(ctx, ctx->sample_light, ctx->sample_light_hdr, s)
                         : VRAD_ERR_CUDA;
        if (rc == VRAD_OK && cudaEventRecord(ctx->ahead_done, s) != cudaSuccess) rc = VRAD_ERR_CUDA;
        ctx->direct_ahead_rc = rc;
        set_sleeping_waits(false);
    });
}
}  // namespace vrad

namespace vrad {
// The direct gather with its supersampling passes (the light pass's first
// step), for the ranges whose outputs are given.
int32_t direct_pass(vrad_ctx *ctx, float4 *ldr_out, float4 *hdr_out, cudaStream_t s) {
    return direct_on(ctx, ldr_out, hdr_out, s);
}
}  // namespace vrad

extern "C" int32_t vrad_direct_lighting_device(vrad_ctx *ctx, vrad_lighting_value *d_out, void *stream) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (!d_out && ctx->world.view.nsamples) return vrad_fail(ctx, VRAD_ERR_ARG, "null output");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "cudaSetDevice");
    const int32_t rc = direct_on(ctx, reinterpret_cast<float4 *>(d_out), nullptr, (cudaStream_t)stream);
    e = vrad::join_stream(ctx, (cudaStream_t)stream);
    return rc != VRAD_OK || e == cudaSuccess ? rc : vrad_cuda_fail(ctx, e, "joining the caller's stream");
}

extern "C" int32_t vrad_direct_lighting(vrad_ctx *ctx, vrad_lighting_value *out, vrad_direct_stats *stats) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    const int64_t n = ctx->world.view.nsamples;
    if (n && !out) return vrad_fail(ctx, VRAD_ERR_ARG, "null output");
    cudaError_t e = cudaSetDevice(ctx->device);
    float4 *d_out = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    if (e == cudaSuccess) e = vrad::dev_alloc(&d_out, sizeof(float4) * (size_t)(n ? n : 1));
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) e = cudaEventRecord(a, ctx->stream);
    if (e != cudaSuccess) {
        vrad::dev_free(d_out);
        if (a) cudaEventDestroy(a);
        return vrad_cuda_fail(ctx, e, "direct lighting set-up");
    }
    int32_t rc = direct_on(ctx, d_out, nullptr, ctx->stream);
    unsigned long long counts[2] = {0, 0};
    uint32_t overflow = 0;
    if (rc == VRAD_OK) {
        e = cudaEventRecord(b, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out, d_out, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(counts, ctx->world.counters, sizeof counts, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&overflow, ctx->status, sizeof overflow, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = vrad::wait_stream(ctx->stream);
        if (e != cudaSuccess) rc = vrad_cuda_fail(ctx, e, "direct lighting");
    }
    if (rc == VRAD_OK && overflow) {
        cudaMemsetAsync(ctx->status, 0, sizeof(uint32_t), ctx->stream);
        rc = vrad_fail(ctx, VRAD_ERR_CUDA, "traversal stack overflow (BVH deeper than %d)", vrad::kStackDepth);
    }
    if (rc == VRAD_OK && stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        stats->samples = n;
        stats->visibility_rays = (int64_t)counts[0];
        stats->sky_rays = (int64_t)counts[1];
        stats->kernel_ms = ms;
        stats->extra_passes_run = ctx->supersample.passes_run;
        stats->supersampled = ctx->supersample.supersampled;
    }
    vrad::dev_free(d_out);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

extern "C" int32_t vrad_direct_autotune(vrad_ctx *ctx, int32_t *chosen_block, float *times_ms) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    if (!ctx->has_scene) return vrad_fail(ctx, VRAD_ERR_NO_SCENE, "no scene uploaded");
    if (!ctx->world.ready) return vrad_fail(ctx, VRAD_ERR_ARG, "no lighting world uploaded");
    cudaError_t e = cudaSetDevice(ctx->device);
    const int64_t n = ctx->world.view.nsamples;
    float4 *d_out = nullptr, *d_hdr = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    // A world with an HDR list is gathered for both ranges at once: the
    // shape is tuned on that kernel.
    const bool dual = ctx->world.view.lights_hdr != nullptr;
    if (e == cudaSuccess) e = vrad::dev_alloc(&d_out, sizeof(float4) * (size_t)(n ? n : 1));
    if (e == cudaSuccess && dual) e = vrad::dev_alloc(&d_hdr, sizeof(float4) * (size_t)(n ? n : 1));
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    const int candidates[3] = {32, 64, 128};
    float best = 1e30f;
    int best_block = 128;
    for (int k = 0; k < 3 && e == cudaSuccess; k++) {
        e = cudaEventRecord(a, ctx->stream);
        if (e == cudaSuccess)
            e = vrad::launch_direct(ctx->scene.view(), dual ? ctx->world.view : vrad::range_view(ctx->world.view, false),
                                    d_out, d_hdr, ctx->world.counters, ctx->status, ctx->stream, candidates[k]);
        if (e == cudaSuccess) e = cudaEventRecord(b, ctx->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
        if (times_ms) times_ms[k] = ms;
        if (e == cudaSuccess && ms < best) {
            best = ms;
            best_block = candidates[k];
        }
    }
    vrad::dev_free(d_out);
    vrad::dev_free(d_hdr);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "direct autotune");
    ctx->world.block = best_block;
    if (chosen_block) *chosen_block = best_block;
    return VRAD_OK;
}

extern "C" int32_t vrad_set_extra_passes(vrad_ctx *ctx, int32_t passes) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if (passes < 0) return vrad_fail(ctx, VRAD_ERR_ARG, "extra passes %d < 0", passes);
    std::lock_guard<std::mutex> g(ctx->mu);
    vrad::settle_direct(ctx);
    ctx->supersample.extra_passes = passes;
    return VRAD_OK;
}
