// direct.cuh -- the lighting world resident on one device, and the fused
// direct-gather launch.
//
// Layout in HBM:
//   slots[k]        int32: sample index of thread k; bit 31 marks a padding
//                   lane, which repeats a sample, traces nothing and writes
//                   nothing (a face's last group of four repeats its last
//                   sample, as FaceLightJob.EmitGroup pads).  Slots run
//                   cluster by cluster, each face's samples starting on a
//                   multiple of four (a reference sample group is four
//                   adjacent lanes) and each cluster padded to whole warps,
//                   so a warp's lanes share one light list.
//   sample_pos[i]   float4 (position xyz, face index bits)
//   face_normal[f]  float4 (plane normal xyz, cluster bits)
//   lights[l]       5 x float4, the DirectLight fields:
//                   (origin, type) (intensity, style) (normal, exponent)
//                   (stop_dot, stop_dot2, constant, linear)
//                   (quadratic, start_fade, end_fade, cap_dist)
//   lights_hdr[l]   the same 5 x float4 for the HDR range (intensity the
//                   only difference), or null for a world without one
//   cl_off, cl_list per-cluster light lists in gather order (CSR)
//   dirs[d]         float4 sky-ambient directions; jitter[d] sun jitter
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "vrad_internal.cuh"

namespace vrad {

constexpr int kLightF4 = 5;

struct DeviceWorld {
    const int32_t *slots;
    int64_t nslots;
    const float4 *sample_pos;
    const float4 *face_normal;
    const float4 *lights;
    int32_t nlights;
    const int32_t *cl_off;
    const int32_t *cl_list;
    int32_t nclusters;
    const float4 *dirs;
    int32_t ndirs;
    const float4 *jitter;
    int32_t njitter;
    float sun_extent;
    int32_t sun_samples;
    int64_t nsamples;
    const float4 *lights_hdr;  // null: the world has one range
    // Light styles (FaceLight.Styles): a launch gathers the lights of one
    // style alone.  With face_key set, the gather also records, per face,
    // the first (sample group, light) that the style lights: the key that
    // orders the face's style slots (FaceLight.FindOrAllocateStyle).  With
    // face_slot set, the supersampling passes skip the faces whose slot for
    // this style is negative (the style is not the face's).
    int32_t style;
    unsigned long long *face_key;
    const int8_t *face_slot;
};

struct WorldBuffers {
    int32_t *slots = nullptr;
    float4 *sample_pos = nullptr;
    float4 *face_normal = nullptr;
    float4 *lights = nullptr;
    float4 *lights_hdr = nullptr;
    int32_t *cl_off = nullptr;
    int32_t *cl_list = nullptr;
    float4 *dirs = nullptr;
    float4 *jitter = nullptr;
    unsigned long long *counters = nullptr;  // [0] visibility rays, [1] sky rays
    DeviceWorld view{};
    bool ready = false;
    int block = 64;  // threads per CTA of the gather; vrad_direct_autotune picks it

    void release();
};

// Light styles above 0 (FaceLight.Styles, MapTools/Rad/Light/FaceLight.cs):
// each style's lights are gathered apart into a sample light of their own;
// a face keeps style 0 in slot 0 and takes up to three more styles in the
// order its sample groups first light them (FaceLightJob.ResolveGroup), a
// fifth being warned and dropped.  The slots decide the lightmap layout, so
// they are made once per world, before the first light pass.
struct StyleState {
    std::vector<int32_t> styles;         // the world's light styles above 0, ascending
    std::vector<float4 *> light[2];      // per style, its sample light (LDR, HDR)
    unsigned long long *keys = nullptr;  // styles x faces: (first group's sample, light position)
    int8_t *slots = nullptr;             // styles x faces: the style's slot on the face, -1 none
    std::vector<uint8_t> face_styles;    // faces x 4 (FaceLight.Styles; 255: empty)
    int64_t dropped = 0;                 // faces warned of a fifth style
    bool ready = false;                  // slots and layout made for the uploaded world

    void release();
};

// Launches the fused gather: out[i] = (lighting xyz, direct sun amount).
// With out_hdr (and world.lights_hdr) one traversal lights both ranges:
// out from world.lights, out_hdr from world.lights_hdr.
cudaError_t launch_direct(const DeviceScene &scene, const DeviceWorld &world, float4 *out, float4 *out_hdr,
                          unsigned long long *counters, uint32_t *overflow, cudaStream_t stream,
                          int block);

// The world as one range sees it: lights = that range's table, no second.
inline DeviceWorld range_view(const DeviceWorld &w, bool hdr) {
    DeviceWorld v = w;
    if (hdr) v.lights = w.lights_hdr;
    v.lights_hdr = nullptr;
    return v;
}

}  // namespace vrad
