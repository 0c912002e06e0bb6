// bounce.cuh -- the radiosity bounce resident on one device.
//
// Layout in HBM (P patches in the reference's index order, R receivers,
// F faces, Q candidate pairs, T transfers):
//   origin[P]    float4 (origin xyz, area)
//   normal[P]    float4 (shading normal xyz, plane dist)
//   mins[P]      float4 (winding bounds min xyz, face bits)
//   maxs[P]      float4 (winding bounds max xyz, cluster bits)
//   tree[P]      int4   (parent, child1, child2, sky)
//   refl[P]      float4 (reflectivity xyz, -)
//   wind[P]      int2   (first point, count) into points[] float4
//   face_range[F] int4  (root patch, first descendant, end of descendants, -)
//   face_samples[F] int2 (first sample, count)
//   face_plane[F] float4 (plane normal xyz, dist)
//   recv[R]      int32  receiver order (VisMatrix.ReceiverOrder): cluster by
//                       cluster, each cluster's leaf patches in index order
//   row_off / row_faces  per cluster, the faces its PVS row reaches, in
//                       VisMatrix.FacesInRow order
//   cand_off[R+1] int64, cand_src[Q] int32, cand_w[Q] float: each receiver's
//                       candidate sources in enumeration order and the
//                       transfer each earns (0 when blocked or none)
//   tr_off[R+1] int64, tr[T] int2 (source, weight bits): the transfer lists
//                       (TransferSet), by receiver
//   acc[P] float4 (sample light xyz, sample area); direct[P], total[P],
//   emit[2][P], shoot[2][P] float4: PatchLighting and Radiosity state
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "direct.cuh"
#include "host_parallel.h"
#include "scene.cuh"
#include "vrad_internal.cuh"

struct vrad_mlp;

namespace vrad {

constexpr int64_t kMaxTransfersPerReceiver = 4 * 65536;  // VisMatrix.MaxPatches
constexpr int kSums = 9;  // doubles in BounceBuffers::sums
constexpr int kFeatures = 32;                            // the warm start network's inputs

struct BounceView {
    int32_t npatches, nfaces, nreceivers;
    const float4 *origin;
    const float4 *normal;
    const float4 *mins;
    const float4 *maxs;
    const int4 *tree;
    const float4 *refl;
    const int2 *wind;
    const float4 *points;
    const int4 *face_range;
    const int2 *face_samples;
    const float4 *face_plane;
    const int32_t *recv;
    const int32_t *row_off;
    const int32_t *row_faces;
    const float *sample_area;
    const float4 *sample_pos;  // the world's (xyz, face bits)
};

struct BounceBuffers {
    // Geometry and tables, built once by vrad_bounce_upload.
    float4 *origin = nullptr, *normal = nullptr, *mins = nullptr, *maxs = nullptr, *refl = nullptr;
    int4 *tree = nullptr;
    int2 *wind = nullptr;
    float4 *points = nullptr;
    int4 *face_range = nullptr;
    int2 *face_samples = nullptr;
    float4 *face_plane = nullptr;
    int32_t *recv = nullptr, *row_off = nullptr, *row_faces = nullptr;
    float *sample_area = nullptr;
    // Transfer build.
    int64_t *cand_off = nullptr;   // R + 1
    int32_t *cand_src = nullptr;   // Q
    float *cand_w = nullptr;       // Q
    int64_t *tr_off = nullptr;     // R + 1
    int2 *tr = nullptr;            // T
    void *scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    // The transfers again, in slices for the gather (SELL-32): receivers
    // sorted by transfer count, descending (stable), 32 to a slice; entry j
    // of lane l of slice s at sell[sell_off[s] + 32 j + l], so a warp's
    // loads of step j are one contiguous 256 B row.
    int32_t *sell_key = nullptr, *sell_idx = nullptr;      // R: counts and receivers before the sort
    int32_t *sell_count = nullptr, *sell_order = nullptr;  // R: after it
    int64_t *sell_off = nullptr;   // slices + 1
    int2 *sell = nullptr;          // at most T + 32 * (the largest count) entries
    void *sort_tmp = nullptr;
    size_t sort_tmp_bytes = 0;
    int64_t ncand = 0, ntransfers = 0;
    // Light state.
    float4 *acc = nullptr, *direct = nullptr, *total = nullptr;
    float4 *emit[2] = {nullptr, nullptr}, *shoot[2] = {nullptr, nullptr};
    double *sums = nullptr;        // fp64 totals of a bounce (kSums): 3 sums, 3 absolute sums,
                                   // 3 absolute sums weighted by the terms left in CollectLight's order
    float *exact = nullptr;        // the sequential float total, when needed
    int32_t *leaf_desc = nullptr;  // the sky-free leaves, descending index (CollectLight's total order)
    int32_t *leaf_rank = nullptr;  // per patch: its position in leaf_desc, -1 off it
    // CollectLight's parents by level (the depth of the subtree below):
    // level h's are level_patch[h_level_off[h] .. h_level_off[h + 1]).
    int32_t *level_patch = nullptr;
    std::vector<int32_t> h_level_off;
    // Learned warm start.
    float4 *first = nullptr;       // the first bounce's light per patch (bounce 0's total)
    float4 *guess = nullptr;       // the network's guess per patch
    uint16_t *feat = nullptr;      // R x 32 BF16 inputs
    float *pred = nullptr;         // R x 3 outputs
    const vrad_mlp *model = nullptr;
    unsigned long long *counters = nullptr;  // [0] transfer rays, [1] blocked, [2] asin ties left open
    double *h_sums = nullptr;      // pinned host copies
    float *h_exact = nullptr;
    // Final pass: each face's leaf patches whose radial box reaches it.
    int32_t *pr_off = nullptr;     // F + 1
    int32_t *pr_patch = nullptr;
    int4 *pr_box = nullptr;        // sMin, tMin, sMax, tMax
    float4 *pr_coord = nullptr;    // coordS, coordT, distS, distT
    float4 *prad_light = nullptr;  // per cell
    float *prad_weight = nullptr;

    BounceView view{};
    uvector<int32_t> h_recv;         // host copy of the receiver order
    int32_t npatches = 0, nfaces = 0, nreceivers = 0, nleaves = 0;
    int32_t max_bounces = 0;
    float threshold = 1.0f;
    int32_t last_buffer = 0;         // which emit/shoot half the last bounce wrote
    // One bounce of each parity captured as a graph (gather, CollectLight's
    // levels, the totals, their copy to h_sums), made on first use.
    cudaGraphExec_t bounce_graph[2] = {nullptr, nullptr};
    bool ready = false;
    // The transfer lists came from vrad_transfer_install: every light pass
    // bounces with them instead of building, until the next upload.
    bool installed = false;
    // tr_off / tr hold a set (a light pass bounced, or one was installed).
    bool lists_ready = false;
    // Statistics of the last pass.
    int32_t bounces_run = 0, exact_totals = 0;
    double added[3] = {0, 0, 0};
    float patch_light_ms = 0, transfer_ms = 0, bounce_ms = 0, final_ms = 0;
    unsigned long long rays = 0, blocked = 0, open_ties = 0;

    void release();      // the device tables; the pinned sums stay
    void free_pinned();  // the pinned sums
};

// Device phases of one bounce pass, all on `stream`.
cudaError_t launch_patch_light(const BounceBuffers &b, const float4 *sample_light, cudaStream_t stream);
cudaError_t launch_transfers(BounceBuffers &b, const DeviceScene &scene, uint32_t *overflow, cudaStream_t stream,
                             bool count_only);
// The gather's slices from the transfer lists (the transfer build's last
// step; also after the lists are installed from a cache).
cudaError_t launch_sell(BounceBuffers &b, cudaStream_t stream);
cudaError_t launch_gather(BounceBuffers &b, int bounce, cudaStream_t stream);
cudaError_t launch_exact_total(BounceBuffers &b, int bounce, cudaStream_t stream);
// Bounce number `bounce` and the copy of its totals to h_sums as one graph
// launch on `stream`; the graph of its parity is captured on `capture` (a
// stream of the library's own) the first time.
cudaError_t launch_bounce_graph(BounceBuffers &b, int bounce, cudaStream_t capture, cudaStream_t stream);
cudaError_t launch_features(BounceBuffers &b, const DeviceWorld &w, cudaStream_t stream);
cudaError_t launch_warm_start(BounceBuffers &b, const DeviceWorld &w, const vrad_mlp &m, cudaStream_t stream);

}  // namespace vrad
