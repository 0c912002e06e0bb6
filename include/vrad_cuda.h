/*
 * vrad_cuda.h -- C ABI of libvrad_cuda.so, the B200 (sm_100a) implementation
 * of the ray-tracing seam of vrad's lighting stage.
 *
 * Plain pointers and sizes only.  Every call returns an int32 status
 * (VRAD_OK or a negative VRAD_ERR_*); vrad_last_error() gives the message.
 * The caller owns every buffer it passes; the library owns the device state
 * behind the opaque context.  Calls on one context are serialised inside the
 * library, so a host may call from many threads.
 *
 * Reference interfaces replaced (paths inside muflub/hl2sdk_tools_sharp):
 *   IRayTracer                 src/SourceSharp.MapTools/Tracing/IRayTracer.cs:128-230
 *   Ray (28-byte record)       src/SourceSharp.MapTools/Tracing/IRayTracer.cs:32-42
 *   HitId (8-byte record)      src/SourceSharp.MapTools/Tracing/HitId.cs:70
 *   RayTraceOptions            src/SourceSharp.MapTools/Tracing/RayTraceOptions.cs:65-145
 *   TracedTriangle             src/SourceSharp.MapTools/Tracing/KdTree.cs:30-38
 *   KdTriangle (48-byte form)  src/SourceSharp.MapTools/Tracing/KdTree.cs:120-167
 *   IGpuTracerFactory offer    src/SourceSharp.MapTools/Rad/GpuTracing.cs:28-75
 */
#ifndef VRAD_CUDA_H
#define VRAD_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VRAD_ABI_VERSION 1

/* Status codes. */
#define VRAD_OK 0
#define VRAD_ERR_ARG (-1)          /* bad argument (ArgumentException in the reference) */
#define VRAD_ERR_CUDA (-2)         /* a CUDA runtime call failed                         */
#define VRAD_ERR_OOM (-3)          /* device allocation failed                           */
#define VRAD_ERR_TIMEOUT (-4)      /* a bounded device wait ran out                      */
#define VRAD_ERR_NO_SCENE (-5)     /* trace before vrad_scene_upload                     */
#define VRAD_ERR_UNSUPPORTED (-6)  /* option this tracer cannot honour (NotSupported)    */
#define VRAD_ERR_NO_DEVICE (-7)    /* no CUDA device / wrong architecture                */
#define VRAD_ERR_FORMAT (-8)       /* bytes that do not decode (the codec's null result) */

/* Ray: origin, direction (need not be unit length), reach in units of the
 * direction's length.  28 bytes, the reference's wire format. */
typedef struct vrad_ray {
    float origin[3];
    float direction[3];
    float max_distance;
} vrad_ray;

/* HitId: the caller's triangle id (-1 = miss) and the hit's position along
 * the ray in units of max_distance (t when max_distance is 1, else
 * t / max_distance).  A miss is (-1, 1.0f). */
typedef struct vrad_hit {
    int32_t surface;
    float fraction;
} vrad_hit;

/* TracedTriangle: caller id (several triangles may share one), three
 * vertices, FCACHETRI flags.  The id's 0x01000000 bit is TraceId.Sky. */
typedef struct vrad_triangle {
    int32_t id;
    float v0[3];
    float v1[3];
    float v2[3];
    uint8_t flags;
    uint8_t pad[3];
} vrad_triangle;

/* KdTriangle: the intersection form (plane, two pre-scaled edge equations,
 * projection axes).  Only needed to trace with coefficients computed by a
 * normalise other than the library's (e.g. stock's reciprocal estimate). */
typedef struct vrad_kd_triangle {
    float n[3];
    float d;
    int32_t id;
    float e[6];
    uint8_t cs0, cs1, flags, unused;
} vrad_kd_triangle;

/* RayTraceOptions.  min_distance: hits with t < min_distance are ignored
 * (StockExact = 0, SelfIntersectionSafe = 1e-3).  skip_id: triangles with
 * this id are ignored (-1 = none).  sky_does_not_block: visibility only; a
 * ray whose first hit is a sky triangle is not blocked.  isolated_rays: the
 * GPU traces every ray alone, so it is accepted and changes nothing. */
typedef struct vrad_trace_options {
    float min_distance;
    int32_t skip_id;
    int32_t sky_does_not_block;
    int32_t isolated_rays;
} vrad_trace_options;

typedef struct vrad_scene_info {
    int32_t triangles;
    int32_t bvh_nodes;
    int32_t bvh_leaves;
    int32_t max_leaf;
    float bounds_min[3];
    float bounds_max[3];
    float box_pad;
    float build_ms;
    int64_t device_bytes;
    int32_t bvh_depth;      /* inner nodes on the deepest path: the traversal stack's size */
} vrad_scene_info;

typedef struct vrad_ctx vrad_ctx;

/* Context on one CUDA device.  Fails with VRAD_ERR_NO_DEVICE when the device
 * is absent or is not compute capability 10.0 (the library holds sm_100a
 * code only).  Replaces IGpuTracerFactory.TryCreateAsync's device probe. */
int32_t vrad_create(int32_t device, vrad_ctx **out);
int32_t vrad_destroy(vrad_ctx *ctx);

/* Builds the scene on the device: intersection form (Correct-mode
 * normalise, bit-identical to KdTreeBuilder.ToIntersectionFormat) and
 * padded boxes on the GPU, the BVH's topology by the surface area
 * heuristic on the host.  Replaces ShadowCasterSet.BuildTracerAsync
 * (src/SourceSharp.MapTools/Rad/ShadowCasterSet.cs) for the device tracer. */
int32_t vrad_scene_upload(vrad_ctx *ctx, const vrad_triangle *tris, int32_t n);

/* As vrad_scene_upload, but the intersection form is given (one per
 * triangle, same order); the vertices still define the boxes. */
int32_t vrad_scene_upload_prepared(vrad_ctx *ctx, const vrad_triangle *tris,
                                   const vrad_kd_triangle *prepared, int32_t n);

int32_t vrad_scene_get_info(vrad_ctx *ctx, vrad_scene_info *out);

/* IRayTracer.Supports: 1 when the options are honoured (all are, except a
 * NaN or negative min_distance), else 0. */
int32_t vrad_supports(const vrad_trace_options *opts);

/* IRayTracer.TraceVisibilityAsync with HOST buffers: one bit per ray,
 * least-significant first, set when an accepted hit lies in
 * [min_distance, max_distance).  hit_bits must hold (n + 63) / 64 words;
 * every word is overwritten.  Blocks until the bits are written. */
int32_t vrad_trace_visibility(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                              const vrad_trace_options *opts, uint64_t *hit_bits);

/* IRayTracer.TraceClosestAsync with HOST buffers: the nearest accepted hit
 * in [min_distance, max_distance), ties to the lower triangle index. */
int32_t vrad_trace_closest(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                           const vrad_trace_options *opts, vrad_hit *hits);

/* The same two operations on DEVICE buffers, enqueued on `stream`
 * (a cudaStream_t; NULL is the CUDA default stream, as everywhere in CUDA).
 * Asynchronous: the results are ready when the stream reaches this point.
 * d_hit_bits must be 4-byte aligned and hold (n + 63) / 64 words.  Launches
 * on different streams may overlap; they share no device scratch. */
int32_t vrad_trace_visibility_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n,
                                     const vrad_trace_options *opts, uint64_t *d_hit_bits,
                                     void *stream);
int32_t vrad_trace_closest_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n,
                                  const vrad_trace_options *opts, vrad_hit *d_hits,
                                  void *stream);

/* ---- FP64 recheck ---------------------------------------------------------
 *
 * The check the reference's own GPU tracer is held to
 * (Tests/MapTools/Tracing/VulkanRayTracerFacts.cs:1215-1300), on the device.
 * The visibility bits are vrad_trace_visibility's (the reference's FP32
 * answer, opts as there; the sky pass-through mode is VRAD_ERR_UNSUPPORTED).
 * A ray is flagged when some triangle's FP32 edge values, their sum or t lie
 * within flag_margin of a boundary (an edge, 1, either end of the segment);
 * each flagged ray is re-tested in FP64 against every triangle of `tris` (the
 * array given to vrad_scene_upload, for the original vertices):
 * fp64_class[i] = 0 miss, 1 hit, 2 within fp64_margin of a boundary
 * (ambiguous), -1 not flagged.  A flagged ray whose clear FP64 class differs
 * from its FP32 bit is a disagreement.  Host buffers; blocks. */
typedef struct vrad_recheck_stats {
    int64_t rays;
    int64_t flagged;
    int64_t fp64_hit;
    int64_t fp64_miss;
    int64_t fp64_ambiguous;
    int64_t disagreements;
} vrad_recheck_stats;

int32_t vrad_trace_visibility_recheck(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                                      const vrad_trace_options *opts, const vrad_triangle *tris, int32_t ntris,
                                      float flag_margin, double fp64_margin, uint64_t *hit_bits,
                                      int8_t *fp64_class, vrad_recheck_stats *stats);

/* ---- Lighting stage ------------------------------------------------------
 *
 * The direct-lighting gather of vrad's lighting stage (the reference's
 * RadWorld.LightFacesAsync, MapTools/Rad/Light/RadWorld.Facelights.cs:194,
 * FaceLightJob.EmitGroup / ResolveGroup, FaceLightJob.cs:329-460, and
 * DirectLightGatherer, DirectLightGatherer.cs:405-1634), fused with its
 * rays: one kernel computes every sample's light from every light in its
 * cluster's list, tracing each shadow, sun and sky segment in-thread. */

/* One lit face: the inputs of FaceLightInfo.Build (FaceLightInfo.cs:79-160).
 * lightmap_vecs are the texinfo's lightmapVecsLuxelsPerWorldUnits rows (s,
 * t), lightmap_mins / lightmap_size the face's LightmapTextureMinsInLuxels /
 * LightmapTextureSizeInLuxels.  The winding is num_vertices points starting
 * at first_vertex of a shared xyz array.  cluster is the cluster of the
 * face's samples. */
typedef struct vrad_face {
    float normal[3];
    float dist;
    float lightmap_vecs[2][4];
    int32_t lightmap_mins[2];
    int32_t lightmap_size[2];
    int32_t first_vertex;
    int32_t num_vertices;
    int32_t cluster;
    int32_t flags;
} vrad_face;

/* LightSample (MapTools/Rad/Light/FaceLight.cs:30-70): one per lightmap cell
 * the face covers; coord is the cell's balance point in luxel space. */
typedef struct vrad_sample {
    float position[3];
    float area;
    float coord[2];
    float mins[2];
    float maxs[2];
    int32_t s, t;
    int32_t face;
    int32_t cluster;
} vrad_sample;

/* DirectLight (MapTools/Rad/Light/DirectLight.cs), EmitType numbering:
 * 0 surface, 1 point, 2 spotlight, 3 sky light (sun), 4 sky ambient. */
typedef struct vrad_light {
    int32_t type;
    int32_t style;
    float origin[3];
    float intensity[3];
    float normal[3];
    float stop_dot;
    float stop_dot2;
    float exponent;
    float constant_attn;
    float linear_attn;
    float quadratic_attn;
    float start_fade_distance;
    float end_fade_distance;
    float cap_dist;
} vrad_light;

/* LightingValue (MapTools/Rad/Light/LightingValue.cs). */
typedef struct vrad_lighting_value {
    float lighting[3];
    float direct_sun_amount;
} vrad_lighting_value;

/* What the lighting stage reads.  samples are face-major, each face's in
 * the order vrad_build_samples writes them.  lights are the active list in
 * gather order; cluster_lights lists, per cluster, the lights whose PVS
 * reaches it, in list order (DirectLightGatherer's per-cluster lists).
 * sky_directions are the DirectionalSampler prefix (xyz each) the sky
 * ambient uses; sun_jitter the prefix the sun's jittered rays use (entry
 * d-1 for ray d); sun_samples is 1 with no angular extent. */
typedef struct vrad_world_desc {
    const vrad_face *faces;
    int32_t nfaces;
    const vrad_sample *samples;
    int64_t nsamples;
    const vrad_light *lights;
    int32_t nlights;
    const int32_t *cluster_light_offsets;  /* nclusters + 1 */
    const int32_t *cluster_lights;
    int32_t nclusters;
    const float *sky_directions;
    int32_t nsky_directions;
    const float *sun_jitter;
    int32_t nsun_jitter;
    float sun_angular_extent;
    int32_t sun_samples;
    const float *vertices;                 /* face windings, xyz each (vrad_face.first_vertex) */
    int64_t nvertices;
    /* The HDR pass's light list (nullable): the same nlights lights in the
     * same order, parsed for the HDR range (DirectLightBuilder.ParseGeneric
     * with the HDR flag, MapTools/Rad/Light/DirectLightBuilder.cs:198-278:
     * _lightHDR, _lightscaleHDR, _ambientHDR), which differs from the LDR
     * list in intensity alone; any other difference is VRAD_ERR_ARG.  With
     * it the world can be lit in both ranges (vrad_light_pass_ranges). */
    const vrad_light *lights_hdr;
} vrad_world_desc;

typedef struct vrad_direct_stats {
    int64_t samples;
    int64_t visibility_rays;   /* shadow segments to point and spot lights */
    int64_t sky_rays;          /* sun and sky-ambient sky tests */
    float kernel_ms;
    int32_t extra_passes_run;  /* supersampling passes that selected samples */
    int64_t supersampled;      /* samples supersampled, over all passes */
} vrad_direct_stats;

/* FaceSampleBuilder.CalcPoints without -fast (FaceSampleBuilder.cs:80-367):
 * host-side set-up, no device needed.  Writes each face's samples into out
 * (capacity entries) and face_first[f] (nfaces + 1 entries) = index of face
 * f's first sample.  With out = NULL it only counts. */
int32_t vrad_build_samples(const vrad_face *faces, int32_t nfaces, const float *vertices,
                           int64_t nvertices, vrad_sample *out, int64_t capacity, int64_t *count,
                           int64_t *face_first);

/* FaceNeighbours.Build (MapTools/Rad/Light/FaceNeighbours.cs:80-230) for
 * brush faces with smoothing groups 0: faces sharing a vertex position are
 * neighbours when the cosine of their normals is at least
 * smoothing_threshold (the reference's default is 0.7071067).  offsets has
 * nfaces + 1 entries; with list = NULL it only counts.  Host-side set-up. */
int32_t vrad_build_neighbours(const vrad_face *faces, int32_t nfaces, const float *vertices,
                              int64_t nvertices, float smoothing_threshold, int32_t *offsets,
                              int32_t *list, int64_t capacity, int64_t *count);

/* LightmapOffsets.Compute (MapTools/Rad/Light/LightmapOffsets.cs:54-126)
 * for faces lit in style 0: each face's lightofs (its median's four bytes
 * sit just before it) and the LIGHTING lump's total size.  Host-side. */
int32_t vrad_lightmap_layout(const vrad_face *faces, int32_t nfaces, int32_t *lightofs, int64_t *total);
/* The layout with light styles: styles holds four bytes per face (its
 * FaceLight.Styles, 255 ending the list; vrad_face_styles gives a lit
 * world's); each face's style medians precede its lightofs, in reverse
 * style order, and its styles' luxels follow it, style after style. */
int32_t vrad_lightmap_layout_styles(const vrad_face *faces, int32_t nfaces, const uint8_t *styles,
                                    int32_t *lightofs, int64_t *total);

/* Uploads the lighting world to the context's device (kept until the next
 * upload or vrad_destroy).  The scene (vrad_scene_upload) is the shadow
 * casters.  Lights of every type (0 surface, 1 point, 2 spot, 3 sun, 4 sky
 * ambient) and style (0 to 254) are lit; VRAD_ERR_UNSUPPORTED for a group
 * of four samples that spans two clusters.  With the scene and the
 * face windings present, the upload also queues the next light pass's
 * direct gather (with its supersampling passes) on the device from a host
 * thread, so that it runs while the caller's bounce upload builds its
 * tables; the next vrad_light_pass takes it.  Calls that change what the
 * gather reads (vrad_scene_upload, vrad_world_upload,
 * vrad_set_extra_passes) or that gather themselves wait for it and drop
 * it. */
int32_t vrad_world_upload(vrad_ctx *ctx, const vrad_world_desc *world);

/* The direct gather of every sample, style 0, flat normals: out[i] is
 * sample i's LightingValue (host buffer, nsamples entries), after the
 * supersampling passes (FaceLightJob's rounds after the first,
 * FaceLightJob.cs:553-930: samples whose perceptual light differs from a
 * neighbour's by 1/16 or more are gathered again on 4x4 and 2x2 grids
 * across their cell, up to vrad_set_extra_passes passes).  Supersampling
 * needs the world uploaded with face windings and samples exactly as
 * vrad_build_samples makes them (their partial cells' windings are rebuilt
 * from the faces); otherwise, with extra passes above 0, the call fails
 * with VRAD_ERR_UNSUPPORTED.  Blocks. */
int32_t vrad_direct_lighting(vrad_ctx *ctx, vrad_lighting_value *out, vrad_direct_stats *stats);

/* The same into a device buffer on `stream` (NULL = default stream). */
int32_t vrad_direct_lighting_device(vrad_ctx *ctx, vrad_lighting_value *d_out, void *stream);

typedef struct vrad_pass_stats {
    int64_t samples;
    int64_t luxels;
    int64_t visibility_rays;
    int64_t sky_rays;
    int64_t lighting_bytes;
    float direct_ms;
    float final_ms;
    int32_t extra_passes_run;
    int64_t supersampled;
    float supersample_ms;     /* of direct_ms */
} vrad_pass_stats;

/* Size in bytes of the LIGHTING lump the uploaded world produces
 * (LightmapOffsets.Compute's LightDataSize). */
int32_t vrad_lighting_size(vrad_ctx *ctx, int64_t *bytes);

/* Light styles (FaceLight.Styles): lights of a style other than 0 light
 * their own lightmap of the face.  A face holds style 0 in its first slot
 * and up to three more styles, in the order its first sample groups light
 * them (FaceLightJob.ResolveGroup's FindOrAllocateStyle); a fifth style is
 * dropped from the face ("Too many light styles on a face").  The slots
 * decide the layout: for a world with styled lights, vrad_lighting_size and
 * the first light pass make them (each such style gathered once).
 * vrad_face_styles gives each face's four style bytes (FACES' styles, 255 an
 * empty slot; nfaces x 4) and the number of faces that dropped a style. */
int32_t vrad_face_styles(vrad_ctx *ctx, uint8_t *styles, int32_t nfaces, int64_t *dropped);

/* The lighting stage with -bounce 0 (the reference's Vrad.RunPassAsync
 * without the bounce, MapTools/Rad/Vrad.cs:392-530): the direct gather, then
 * FinalLightFace for every face (LuxelRadial filter over the face's own and
 * its smoothing neighbours' samples, minlight, StockLightColor.Encode, the
 * per-face median), written as the LIGHTING lump's bytes.  lighting must
 * hold vrad_lighting_size bytes (bytes no face owns are zero); lightofs
 * (nfaces entries, nullable) receives each face's FACES lightofs; styles
 * are 0 then 255 for every lit face.  Host buffers; blocks. */
int32_t vrad_light_pass(vrad_ctx *ctx, uint8_t *lighting, int64_t capacity, int32_t *lightofs,
                        vrad_pass_stats *stats);

/* The same into a device buffer on `stream` (NULL = default stream). */
int32_t vrad_light_pass_device(vrad_ctx *ctx, uint8_t *d_lighting, void *stream);

/* DirectLightingSettings.ExtraPasses: how many supersampling passes the
 * direct gather may run (the reference's default, and this library's, is
 * 4; 0 is -noextra, no supersampling). */
int32_t vrad_set_extra_passes(vrad_ctx *ctx, int32_t passes);

/* Times the gather once per launch shape (32, 64 and 128 threads per CTA)
 * on the uploaded world and keeps the fastest for later calls; times_ms
 * (nullable, 3 entries) receives each shape's time.  No counterpart in the
 * reference (its CPU work queue has no launch shape). */
int32_t vrad_direct_autotune(vrad_ctx *ctx, int32_t *chosen_block, float *times_ms);

/* ---- Bounce ---------------------------------------------------------------
 *
 * The radiosity bounce of the lighting stage (the reference's
 * RadWorld.BounceAsync, MapTools/Rad/Light/RadWorld.Bounce.cs:240-290):
 * the patch tree (PatchBuilder, PatchSubdivider), the patches' direct light
 * (PatchLighting.BuildPatchLights), the transfers (VisMatrix.BuildAsync
 * with FormFactors), the bounces (Radiosity.BounceAsync) and the bounced
 * light's radial filter in the final pass (FinalLightFace.BuildPatchRadial).
 * The replaced stage boundary is IVradBounceStage.BounceAsync
 * (MapTools/Rad/VradStages.cs:112-183), whose contract is that the
 * patches' TotalLight holds the bounced light only. */

/* Texinfo surface flags (SurfaceFlags) read from vrad_face.flags. */
#define VRAD_SURF_LIGHT 0x0001
#define VRAD_SURF_SKY 0x0004
#define VRAD_SURF_NOLIGHT 0x0400
#define VRAD_SURF_BUMPLIGHT 0x0800
#define VRAD_SURF_NOCHOP 0x4000
/* Not a SurfaceFlags bit: the face's texture emits (PatchBuilder's
 * BaseLightForFace is nonzero), so its patches are surface lights' and skip
 * the face-edge refinement (PatchSubdivider.cs:375-380).  The caller makes
 * the surface lights themselves (DirectLightBuilder.AddSurfaceLights) from
 * the leaf patches, as type 0 lights. */
#define VRAD_FACE_EMITS 0x40000000

/* Patch (MapTools/Rad/Light/Patch.cs:44-234), the fields the bounce reads.
 * normal is the shading normal (the plane normal for a root, the phong
 * normal at the origin for a child); plane_dist is the face plane's.
 * cluster is the cluster of the patch's face; the winding is num_points
 * points from first_point of the point array vrad_build_patches fills. */
typedef struct vrad_patch {
    float origin[3];
    float area;
    float normal[3];
    float plane_dist;
    float mins[3];
    float chop;
    float maxs[3];
    float lux_scale;
    float face_mins[3];
    int32_t face;
    float face_maxs[3];
    int32_t cluster;
    float reflectivity[3];
    int32_t sky;
    int32_t parent;
    int32_t child1;
    int32_t child2;
    int32_t first_point;
    int32_t num_points;
    int32_t pad[3];
} vrad_patch;

/* PatchBuilder.Build + PatchSubdivider.Subdivide (bounces > 0, not -fast)
 * on the host: one root patch per face in face order, then each root's
 * subtree in creation order, the reference's patch indices.  reflectivity
 * is nfaces x 3 (the faces' texdata reflectivity, clamped to 0.99 here);
 * max_chop / min_chop in luxels (the reference's defaults are 4 and 4).
 * With out and points NULL it only counts. */
int32_t vrad_build_patches(const vrad_face *faces, int32_t nfaces, const float *vertices, int64_t nvertices,
                           const float *reflectivity, float max_chop, float min_chop, vrad_patch *out,
                           int64_t capacity, int64_t *count, float *points, int64_t point_capacity,
                           int64_t *point_count);

/* What the bounce reads beyond the world: per-face reflectivity, the PVS
 * (per cluster, the clusters its row sets, ascending), the chop sizes and
 * the stop rule.  Radiosity.BounceAsync stops after `bounces` bounces or
 * once a bounce adds less than `threshold` in every channel (the
 * reference's threshold is 1.0). */
typedef struct vrad_bounce_desc {
    const float *reflectivity;     /* nfaces x 3 */
    const int32_t *pvs_offsets;    /* nclusters + 1 */
    const int32_t *pvs_clusters;
    int32_t nclusters;
    float max_chop;
    float min_chop;
    int32_t bounces;               /* 0: the light pass does not bounce */
    float threshold;
} vrad_bounce_desc;

/* Builds the patch tree for the uploaded world (vrad_world_upload first,
 * with face windings) and keeps it, with the transfer and final-pass
 * tables, on the device: every later vrad_light_pass then bounces.
 * VRAD_ERR_UNSUPPORTED for bumped faces. */
int32_t vrad_bounce_upload(vrad_ctx *ctx, const vrad_bounce_desc *desc);

typedef struct vrad_bounce_stats {
    int64_t patches;
    int64_t receivers;        /* leaf patches in a cluster (VisMatrix.ReceiverOrder) */
    int64_t transfer_rays;    /* candidate pairs traced (VisMatrixStatistics.Rays) */
    int64_t blocked;          /* of them, blocked */
    int64_t transfers;
    int32_t bounces;          /* bounces run */
    int32_t exact_totals;     /* stop decisions the bounded fp64 total could not settle */
    double added[3];          /* light the last bounce added, over leaf patches */
    float patch_light_ms;
    float transfer_ms;
    float bounce_ms;
    float final_ms;
    int64_t unsettled_asin;   /* form-factor arcsines left at the plain rounding (expected 0) */
    int32_t transfers_cached; /* 1: the pass bounced with transfers from vrad_transfer_install
                                 (RadWorld.TransfersWereCached); transfer_rays and blocked are 0 */
} vrad_bounce_stats;

/* The statistics of the last light pass's bounce. */
int32_t vrad_bounce_stats_get(vrad_ctx *ctx, vrad_bounce_stats *stats);

/* The ranges a compile lights (Vrad.Passes, MapTools/Rad/Vrad.cs:150-158):
 * LDR, HDR, or both (-both: LDR first). */
#define VRAD_RANGE_LDR 1
#define VRAD_RANGE_HDR 2

/* The lighting stage for one or both ranges, as the reference runs its
 * passes (Vrad.LightTakenAsync / RunPassAsync, MapTools/Rad/Vrad.cs:262-285,
 * 392-590): each range's direct gather, supersampling, bounce and final
 * pass, writing LIGHTING (ldr) and LIGHTING_HDR (hdr), each
 * vrad_lighting_size bytes.  The second range reuses the first's transfers
 * (they are geometry; Rad/Vrad.cs:261-263, RadWorld.BounceAsync), so one
 * transfer build serves both.  With both ranges the first round of the
 * direct gather is one traversal: every shadow, sun and sky segment is
 * traced once and lights both ranges (the ranges differ in intensity
 * only), so each range's sample light is the bits its own pass would give.
 * FACES and FACES_HDR share the layout: lightofs (nullable) is written
 * once.  bounce_stats (nullable) receives two records, LDR then HDR (a
 * range not lit is zeroed); afterwards vrad_bounce_patch_light and the
 * other bounce inspections report the last range lit.  HDR needs a world
 * uploaded with lights_hdr.  Host buffers; blocks. */
int32_t vrad_light_pass_ranges(vrad_ctx *ctx, int32_t ranges, uint8_t *ldr, int64_t ldr_capacity, uint8_t *hdr,
                               int64_t hdr_capacity, int32_t *lightofs, vrad_pass_stats *stats,
                               vrad_bounce_stats *bounce_stats);

/* vrad_light_pass_ranges into device buffers (4-byte aligned, each
 * vrad_lighting_size bytes; the one of a range not lit may be NULL),
 * queued on `stream` (NULL: the default stream). */
int32_t vrad_light_pass_ranges_device(vrad_ctx *ctx, int32_t ranges, uint8_t *d_ldr, uint8_t *d_hdr, void *stream);

/* After a light pass: one range's per-sample direct light (LightingValue,
 * FaceLight's sample values after the supersampling rounds) as that pass's
 * patch light and final pass read it; n = the world's sample count.  The
 * reference keeps it per range in RadPass.LightData (FaceLight). */
int32_t vrad_pass_sample_light(vrad_ctx *ctx, int32_t range, vrad_lighting_value *out, int64_t n);

/* The last light pass's bounce statistics per range: two records, LDR then
 * HDR (zeroed for a range the pass did not light; final_ms is kept only by
 * the host-buffer passes).  Device-buffer passes report here too. */
int32_t vrad_bounce_stats_ranges(vrad_ctx *ctx, vrad_bounce_stats *stats);

/* After a light pass: each patch's bounced light (TotalLight.Flat) and
 * direct light (DirectLight), npatches x 3 each; either may be NULL. */
int32_t vrad_bounce_patch_light(vrad_ctx *ctx, float *total_light, float *direct_light, int64_t npatches);

/* After a light pass: the light the last bounce added, summed as
 * Radiosity.CollectLight sums it (float, descending patch index; the
 * value its stop rule compares), xyz. */
int32_t vrad_bounce_last_total(vrad_ctx *ctx, float *total);

/* The transfer build's form factors on their own, evaluated on the device by
 * the functions the transfer kernel calls; they replace
 * FormFactors.DiffToDiff and FormFactors.PolyToDiff
 * (MapTools/Rad/Bounce/FormFactors.cs:58-140, Correct mode) for inspection.
 *   vrad_form_factor_diff: cases are n x 12 floats (o1, n1, o2, n2); out[i]
 *     = -(d . n1)(d . n2) / len^2 with d, len = normalise(o1 - o2).
 *   vrad_form_factor_poly: winding i is points[first[i] .. first[i+1]) (xyz
 *     triples, at least three); cases are n x 7 floats (the winding's area,
 *     the receiving point, its normal); out[i] the polygon form factor
 *     (Sum gamma_k asin|v_k x v_k+1| . n) * 0.5 / area, with the correctly
 *     rounded arcsine.
 * Both block and allocate their own small device temporaries. */
int32_t vrad_form_factor_diff(vrad_ctx *ctx, const float *cases, int64_t n, float *out);
int32_t vrad_form_factor_poly(vrad_ctx *ctx, const float *points, const int32_t *first, const float *cases,
                              int64_t n, float *out);

/* Transfer (MapTools/Rad/Bounce/TransferSet.cs:26): source patch, weight. */
typedef struct vrad_transfer {
    int32_t patch;
    float weight;
} vrad_transfer;

/* After a light pass: the transfer lists by receiving patch,
 * offsets[npatches + 1] (TransferSet.For(patch) = transfers[offsets[p] ..
 * offsets[p + 1])).  With transfers NULL it only fills offsets and count. */
int32_t vrad_bounce_transfers(vrad_ctx *ctx, int64_t *offsets, int64_t npatches, vrad_transfer *transfers,
                              int64_t capacity, int64_t *count);

/* ---- Transfer cache: a transfer set as bytes ------------------------------
 *
 * TransferSetCodec (MapTools/Rad/Bounce/TransferSetCodec.cs:23-447), the
 * format the reference's cross-compile transfer cache stores
 * (Compile/Cache/StoreTransferCache.cs:241-262, 360-378):
 *   index: "TRF1" (u32 0x31465254), the patch count (i32), the longest list
 *     (i32), the total (i64), then every patch's count (i32), little-endian;
 *   chunks: the transfers patch after patch as (patch i32, weight's f32
 *     bits), cut every max(1, max_chunk_bytes / 8) transfers (a list may
 *     straddle two chunks; an empty set has no chunk);
 *   packed chunk: the chunk's transfer count n (i32), then a zlib stream
 *     (RFC 1950, deflate level 1) of 8n bytes: byte b of every patch delta
 *     (the patch minus the one before it in the chunk, the first minus 0,
 *     wrapping) as plane b, then byte b of every weight as plane 4 + b.
 * The planes are the reference's byte for byte; the deflate stream is
 * zlib's own, so the packed bytes are not necessarily those of another
 * deflater, and any zlib stream of the right bytes reads back. */
#define VRAD_TRANSFER_MAGIC 0x31465254u

/* Index(set) from the lists' offsets (offsets[npatches + 1], as
 * vrad_bounce_transfers fills them) into out (20 + 4 npatches bytes).
 * VRAD_ERR_ARG when a list is longer than an int or the offsets fall. */
int32_t vrad_transfer_index(const int64_t *offsets, int32_t npatches, uint8_t *out, int64_t capacity);

/* Pack(chunk) on host bytes: len a multiple of 8.  *written = the packed
 * size; vrad_transfer_pack_bound(len) bytes always suffice. */
int64_t vrad_transfer_pack_bound(int64_t len);
int32_t vrad_transfer_pack(const uint8_t *chunk, int64_t len, uint8_t *out, int64_t capacity, int64_t *written);

/* Unpack(packed) on host bytes.  VRAD_ERR_FORMAT (the reference's null)
 * when the bytes are not a packed chunk: shorter than 4, a count out of
 * range, a stream that does not inflate to exactly 8n bytes. */
int32_t vrad_transfer_unpack(const uint8_t *packed, int64_t len, uint8_t *out, int64_t capacity, int64_t *written);

/* The context's transfer set (after a light pass that bounced, or an
 * install) as the index and its packed chunks, for a store: the set is put
 * in patch order and shuffled into planes on the device, then each chunk is
 * deflated on the host's threads.  vrad_transfer_export_size reports the
 * index size, the chunk count and a packed size that always suffices;
 * vrad_transfer_export writes the index, the packed chunks back to back
 * into packed, their sizes into chunk_sizes[nchunks], and the bytes used
 * into *packed_len.  Blocks. */
int32_t vrad_transfer_export_size(vrad_ctx *ctx, int64_t max_chunk_bytes, int64_t *index_len, int64_t *nchunks,
                                  int64_t *packed_bound);
int32_t vrad_transfer_export(vrad_ctx *ctx, int64_t max_chunk_bytes, uint8_t *index, int64_t index_capacity,
                             uint8_t *packed, int64_t packed_capacity, int64_t *chunk_sizes, int64_t chunk_capacity,
                             int64_t *packed_len);

/* ReadPacked(index, chunks, patch_count) into host arrays: chunk k is
 * packed[at_k .. at_k + chunk_sizes[k]) with at_k the sum of the sizes
 * before it.  The chunks inflate on the host's threads and their planes are
 * turned back into transfers on ctx's device; offsets[patch_count + 1] and
 * *total are filled, transfers (nullable: offsets only) needs room for the
 * total.  VRAD_ERR_FORMAT (the reference's null) when they do not fit
 * together: the index's magic, patch count, size, counts, total and
 * longest list; the chunks' counts adding up to the total; every chunk
 * inflating to exactly its count; every patch in range.  Blocks. */
int32_t vrad_transfer_read_packed(vrad_ctx *ctx, const uint8_t *index, int64_t index_len, const uint8_t *packed,
                                  const int64_t *chunk_sizes, int64_t nchunks, int32_t patch_count,
                                  int64_t *offsets, vrad_transfer *transfers, int64_t capacity, int64_t *total);

/* A cache hit (RadWorld.BounceAsync's TryGetAsync branch,
 * MapTools/Rad/Light/RadWorld.Bounce.cs:364-374): ReadPacked with the
 * uploaded bounce's patch count, straight into the bounce's transfer
 * lists; every later light pass bounces with them instead of building its
 * own (vrad_bounce_stats.transfers_cached), until the next
 * vrad_bounce_upload.  VRAD_ERR_FORMAT as vrad_transfer_read_packed, and
 * when the set cannot be this bounce's: a list on a patch that receives
 * none here, or more transfers than the bounce's candidate pairs.  A
 * refused set leaves the context's transfers as they were.  Blocks. */
int32_t vrad_transfer_install(vrad_ctx *ctx, const uint8_t *index, int64_t index_len, const uint8_t *packed,
                              const int64_t *chunk_sizes, int64_t nchunks);

/* ---- Learned warm start ---------------------------------------------------
 *
 * A small network (32 -> 128 -> 128 -> 3, ReLU, BF16 weights and
 * activations, FP32 accumulation) that predicts a patch's converged bounced
 * light from per-patch features; the bounce can start from its guess
 * (vrad_bounce_set_model).  No counterpart in the reference: its bounce
 * always starts from zero, and that plain bounce stays the default here.
 * Training and inference run on the context's device, on tensor cores.
 * A network is not safe to use from two threads at once. */

#define VRAD_MLP_INPUTS 32
#define VRAD_MLP_HIDDEN 128
#define VRAD_MLP_OUTPUTS 3
/* Parameters in order: w1 [32][128], b1 [128], w2 [128][128], b2 [128],
 * w3 [128][3], b3 [3]; w[k][n] maps input k to output n. */
#define VRAD_MLP_PARAMS (32 * 128 + 128 + 128 * 128 + 128 + 128 * 3 + 3)

typedef struct vrad_mlp vrad_mlp;

/* A new network on ctx's device, He-initialised from `seed`. */
int32_t vrad_mlp_create(vrad_ctx *ctx, uint64_t seed, vrad_mlp **out);
int32_t vrad_mlp_destroy(vrad_mlp *m);

/* Reads (get) and/or replaces (set) the FP32 parameters, host arrays of
 * VRAD_MLP_PARAMS floats. */
int32_t vrad_mlp_params(vrad_mlp *m, float *get, const float *set);

/* y[n][3] = the network on x[n][32] (BF16 bit patterns), device buffers,
 * on `stream` (NULL = default stream). */
int32_t vrad_mlp_forward_device(vrad_mlp *m, const uint16_t *x, int64_t n, float *y, void *stream);

/* The gradient of the mean squared error against target[n][3] (device
 * buffers): grad (host, VRAD_MLP_PARAMS floats, nullable) and the loss
 * (host, nullable).  Blocks. */
int32_t vrad_mlp_gradient_device(vrad_mlp *m, const uint16_t *x, const float *target, int64_t n, float *grad,
                                 float *loss, void *stream);

/* One Adam step (beta1 0.9, beta2 0.999) on that gradient, learning rate
 * lr, on `stream`; vrad_mlp_loss reads the step's loss. */
int32_t vrad_mlp_train_step_device(vrad_mlp *m, const uint16_t *x, const float *target, int64_t n, float lr,
                                   void *stream);
int32_t vrad_mlp_loss(vrad_mlp *m, float *loss);

/* The forward runs on the fifth-generation tensor cores (tcgen05.mma, TMEM
 * accumulators); each of its MMA waits is bounded, and a wait that runs out
 * is recorded on the device.  This call reads and clears that record:
 * VRAD_ERR_TIMEOUT when a forward since the last call gave up. */
int32_t vrad_mlp_status(vrad_mlp *m);

/* Attaches a network to the bounce (NULL detaches it: the plain bounce).
 * With one attached, a light pass bounces once from the direct light (B1),
 * asks the network for each patch's converged bounced light G from its
 * features, and then iterates T <- B1 + gather(G) and T_next = T + the
 * bounced change from there, stopping when the summed magnitude of a
 * step's change is below the threshold.  The network must outlive its
 * use; the context does not own it. */
int32_t vrad_bounce_set_model(vrad_ctx *ctx, const vrad_mlp *model);

/* After a light pass: per receiver (VisMatrix.ReceiverOrder), the network's
 * 32 BF16 inputs (x, nullable) and log1p of the bounced light the pass
 * converged to (target, 3 floats, nullable), device buffers of `capacity`
 * rows; *count = the receivers.  The training set of the warm start. */
int32_t vrad_bounce_features_device(vrad_ctx *ctx, uint16_t *x, float *target, int64_t capacity, int64_t *count,
                                    void *stream);

/* Largest batch vrad_trace_visibility_static accepts: four of the
 * reference's 16,384-ray batches. */
#define VRAD_STATIC_MAX_RAYS 65536

/* vrad_trace_visibility for callers that must not allocate device memory
 * during a run: processes that reserve all their device memory at
 * start-up, or hosts that must not stall on the device-wide synchronisation
 * that freeing device memory can bring.  No counterpart in the
 * reference.  Same arguments, answers and errors as vrad_trace_visibility,
 * but rays and bits are staged through one fixed array inside the library
 * (1,843,456 bytes: sizeof(vrad_ray) x VRAD_STATIC_MAX_RAYS for the rays,
 * 8 KiB for the bits, 256 B for a status word), held on every GPU that
 * loads the library until the process exits, instead of buffers grown with
 * cudaMalloc, so the call makes no allocation.
 * n above VRAD_STATIC_MAX_RAYS is refused with VRAD_ERR_ARG.
 *
 * vrad_create places the array and the trace kernels on its device and
 * looks up the array's address there, at set-up; later calls only use
 * them.  (With lazy module loading that placement would otherwise happen
 * at the first call, and it takes device memory.)  All calls on one
 * device share the array: calls that overlap on the GPU (two contexts on
 * one device, driven from two threads) race and must be serialised by the
 * caller.  The call blocks until the bits are written.  The library does
 * not survive a cudaDeviceReset of that device. */
int32_t vrad_trace_visibility_static(vrad_ctx *ctx, const vrad_ray *rays, int64_t n,
                                     const vrad_trace_options *opts, uint64_t *hit_bits);

/* ---- The BSP surface walk -------------------------------------------------
 *
 * Stock vrad's other tracer: CLightSurface over EnumerateNodesAlongRay, a
 * front-to-back walk of the map's own BSP tree that tests lit faces in
 * lightmap space and sky faces by their windings, stopping at the first hit.
 * Leaf ambient traces with it.  Replaces BspSurfaceTracer.TraceClosest
 * (MapTools/Tracing/BspSurfaceTracer.cs:166-199, 233-357) over the arrays
 * BspTraceGeometry.Build makes (MapTools/Tracing/BspTraceGeometry.cs:291-
 * 899; hl2sdk_tools_sharp_b200/bsp.py builds them from a BSP file):
 *   nodes       8 words per node: plane normal xyz, dist, then as int32
 *               child0, child1 (a leaf is -1 - index), first node face,
 *               packed (lit face count | sky face count << 15 | axis << 30,
 *               axis 3 for a plane that is not axial);
 *   surfaces    16 floats per face: plane normal xyz, dist, lightmap s
 *               (xyz, offset), t (xyz, offset), lightmap mins s, t and
 *               sizes s, t (sizes -1 for a face with no lightmap);
 *   node_faces  every node's on-node candidates, lit then sky;
 *   leaf_faces  every leaf's candidates; leaf_start / leaf_count per leaf;
 *   sky_points  the sky faces' windings (xyz), sky_start / sky_count per face.
 * Every index is checked at upload; the context keeps the tree until the
 * next upload or vrad_destroy. */
typedef struct vrad_bsp_geometry {
    const float *nodes;
    int32_t nnodes;
    const float *surfaces;
    int32_t nsurfaces;
    const int32_t *node_faces;
    int32_t nnode_faces;
    const int32_t *leaf_faces;
    int32_t nleaf_faces;
    const int32_t *leaf_start;
    const int32_t *leaf_count;
    int32_t nleaves;
    const float *sky_points;
    int32_t nsky_points;
    const int32_t *sky_start;
    const int32_t *sky_count;
} vrad_bsp_geometry;

int32_t vrad_bsp_upload(vrad_ctx *ctx, const vrad_bsp_geometry *bsp);

/* The walk for n rays: the segment from origin along direction x reach
 * (stock's start + delta over the fraction 0..1).  hits[i] = the face hit
 * and the fraction along the segment, or -1 and 1 for none.  min_distance
 * is the smallest fraction a leaf face may be hit at (RayTraceOptions'
 * MinDistance); a skip id is VRAD_ERR_UNSUPPORTED.  A walk deeper than 64
 * pending splits fails the call with VRAD_ERR_CUDA, as the reference's
 * throws.  Host buffers; blocks.  The _device form takes device buffers and
 * queues on `stream`. */
int32_t vrad_bsp_trace_closest(vrad_ctx *ctx, const vrad_ray *rays, int64_t n, const vrad_trace_options *opts,
                               vrad_hit *hits);
int32_t vrad_bsp_trace_closest_device(vrad_ctx *ctx, const vrad_ray *d_rays, int64_t n, float min_distance,
                                      vrad_hit *d_hits, void *stream);

/* ---- Leaf ambient ---------------------------------------------------------
 *
 * Stock vrad's per-leaf ambient cubes (ComputePerLeafAmbientLighting,
 * MapTools/Rad/Ambient/LeafAmbientBuilder.cs:22-688), the stage that is
 * 51.6 % of stock vrad's wall clock.  Two parts live here:
 *   vrad_leaf_ambient_positions  each leaf's candidate sample positions
 *     (host code: LeafAmbientBuilder.PlanSamples, :252-276, over
 *     LeafSampler.Generate, LeafSampler.cs:38-148);
 *   vrad_ambient_cubes  at each position the 162 rays into the map through
 *     the BSP surface walk, each hit's lightmap colour blended by the cone
 *     (RayAmbientLighting.Accumulate, RayAmbientLighting.cs:89-134), and
 *     the colours projected onto the six cube sides (AmbientCube.Project,
 *     AmbientCube.cs:80-103): AmbientSampler.ComputeRayCube
 *     (AmbientSampler.cs:211-227), on the device.
 * The baked surface lights (AmbientSampler.AddSurfaceLights), the 16-sample
 * list and the lump encoding are not part of these calls, and neither are
 * displacements: a map with displacement faces is the caller's to refuse. */

/* The BSP pieces the sampler reads, one int32 array per lump, widened:
 *   planes        nplanes x 4 floats: normal xyz, dist
 *   nodes         nnodes x 3: plane, child 0, child 1 (a leaf is -1 - leaf)
 *   leaves        nleaves x 9: contents, mins xyz, maxs xyz, first leaf
 *                 brush, leaf brush count
 *   leaf_brushes  nleaf_brushes brush numbers
 *   brushes       nbrushes x 3: first side, side count, contents
 *   brush_sides   nbrush_sides x 2: plane, bevel */
typedef struct vrad_ambient_tree {
    const float *planes;
    int32_t nplanes;
    const int32_t *nodes;
    int32_t nnodes;
    const int32_t *leaves;
    int32_t nleaves;
    const int32_t *leaf_brushes;
    int32_t nleaf_brushes;
    const int32_t *brushes;
    int32_t nbrushes;
    const int32_t *brush_sides;
    int32_t nbrush_sides;
} vrad_ambient_tree;

/* Every leaf's candidate sample positions in leaf order: counts[l] = the
 * leaf's candidate count (stock's, with the sample-count quirk that sizes
 * all three axes by x: LeafAmbientBuilder.CandidateSampleCount, :420-454;
 * 0 for a solid leaf), positions = the positions, 3 floats each, leaf after
 * leaf.  Each leaf draws from its own stream seeded 0, as stock's
 * per-leaf CLeafSampler does.  With positions NULL only counts and *total
 * are filled; otherwise capacity (in positions) must hold *total.  Host
 * code on `threads` threads (0: all); needs no device. */
int32_t vrad_leaf_ambient_positions(const vrad_ambient_tree *tree, int32_t *counts, float *positions,
                                    int64_t capacity, int64_t *total, int32_t threads);

/* The stage's last steps (host code): every leaf's samples, in order, into
 * the 16-sample list (AmbientSampleList.Add; stock's tie-break, which never
 * fires, unless correct_tiebreak), compressed (AmbientSampleList.Compress,
 * over gamma_table: StockLightColor's 1,024-entry linear-to-screen table),
 * and encoded (LeafAmbientBuilder.Encode): index_out = nleaves records of
 * (uint16 count, uint16 first), an empty leaf's first naming its nearest
 * neighbour with samples; lighting_out = *records records of 28 bytes (six
 * RGBE colours, the 8-bit position fractions, a zero pad).  counts and
 * positions are vrad_leaf_ambient_positions', cubes the samples' cubes (18
 * floats each: with the baked surface lights added, when the caller has
 * them).  With lighting_out NULL only *records is filled. */
int32_t vrad_leaf_ambient_lumps(const vrad_ambient_tree *tree, const int32_t *counts, const float *positions,
                                const float *cubes, const int32_t *gamma_table, int32_t correct_tiebreak,
                                uint8_t *index_out, uint8_t *lighting_out, int64_t capacity, int64_t *records,
                                int32_t *bad_leaves);

/* One BSP face's lightmap lookups (AmbientScene's FaceShade,
 * AmbientScene.cs:247-318).  styles packs the four style bytes, slot 0 in
 * the low byte; averages[k] is slot k's average colour (the four bytes
 * before the lightmap, counting back) decoded and tinted by reflectivity. */
#define VRAD_AMBIENT_SKY 1          /* SURF_SKY: a hit reads the sky ambient  */
#define VRAD_AMBIENT_BAD_AVERAGE 2  /* a slot's average lies outside the lump */
typedef struct vrad_ambient_face {
    int32_t lightofs;    /* byte offset of the face's lightmap; -1: none */
    int32_t smax, tmax;  /* luxels a row, rows */
    int32_t stride;      /* luxels between style slots (x4 when bumped) */
    int32_t nstyles;     /* slots in use, up to 4 */
    uint32_t styles;
    int32_t flags;       /* VRAD_AMBIENT_* */
    float reflectivity[3];
    float averages[4][3];
} vrad_ambient_face;

/* The lighting the cubes read: one range's lighting lump (LDR or HDR), the
 * faces' records (the range's face lump), the 162 sample directions
 * (VertexNormals; 3 floats each), tan of the cone's inner half-angle, and
 * the sky ambient (the range's first emit_skyambient world light's
 * intensity) when the map has one.  Needs vrad_bsp_upload of the same map;
 * nfaces must equal its surface count. */
typedef struct vrad_ambient_lighting {
    const uint8_t *lighting;
    int64_t lighting_bytes;
    const vrad_ambient_face *faces;
    int32_t nfaces;
    const float *directions;
    int32_t ndirections;  /* 162 */
    float tan_theta;
    int32_t has_sky_ambient;
    float sky_ambient[3];
} vrad_ambient_lighting;

int32_t vrad_ambient_upload(vrad_ctx *ctx, const vrad_ambient_lighting *lighting);

/* The ray cubes at n positions (3 floats each): cubes[6 n] colours (3
 * floats each), sides +x, -x, +y, -y, +z, -z.  Fails with VRAD_ERR_ARG
 * when a ray hits a face whose lightmap or averages lie outside the lump
 * (the reference's InvalidOperationException) and with VRAD_ERR_CUDA when a
 * walk goes deeper than 64 pending splits.  Host buffers; blocks.  The
 * _device form takes device buffers and queues on `stream`; its faults
 * are reported by the next vrad_ambient_status. */
int32_t vrad_ambient_cubes(vrad_ctx *ctx, const float *positions, int64_t n, float *cubes);
int32_t vrad_ambient_cubes_device(vrad_ctx *ctx, const float *d_positions, int64_t n, float *d_cubes, void *stream);
int32_t vrad_ambient_status(vrad_ctx *ctx);

/* ---- Batches of maps ------------------------------------------------------
 *
 * Many maps lit on one device.  No counterpart in the reference, which
 * lights one map per call (Vrad.RunAsync, MapTools/Rad/Vrad.cs:160-390).
 * A batch owns `workers` persistent host threads, each with its own context
 * (stream, device tables, pinned staging).  The threads take maps from one
 * shared queue, largest first.  Each map goes through the whole lighting
 * stage: vrad_scene_upload, vrad_world_upload, vrad_set_extra_passes,
 * vrad_bounce_upload when the map has a bounce, then vrad_light_pass.  One
 * map's host set-up (BVH, sample slots, patch tree) therefore overlaps other
 * maps' passes on the device, and small maps' kernels share the SMs.  Each
 * lump is byte-identical to the one the single-map calls write. */

#define VRAD_BATCH_MAX_WORKERS 8

typedef struct vrad_batch vrad_batch;

/* One map of a batch.  The inputs are what the single-map calls take.
 * The run fills in the outputs. */
typedef struct vrad_batch_map {
    const vrad_triangle *triangles;  /* the shadow casters (vrad_scene_upload) */
    const vrad_world_desc *world;
    const vrad_bounce_desc *bounce;  /* NULL: the map is not bounced */
    uint8_t *lighting;               /* host, capacity bytes: the LIGHTING lump */
    int32_t *lightofs;               /* nfaces entries, nullable */
    int64_t capacity;
    int32_t ntriangles;
    int32_t extra_passes;            /* supersampling passes; negative: the default 4 */
    /* written by the run */
    int32_t status;                  /* VRAD_OK, or the code of the call that failed */
    int32_t worker;                  /* the worker that lit the map */
    int64_t lighting_bytes;
    double seconds;                  /* the map's time on its worker, uploads included */
    double scene_s;                  /* of it: vrad_scene_upload */
    double world_s;                  /* vrad_world_upload and vrad_set_extra_passes */
    double bounce_s;                 /* vrad_bounce_upload */
    double pass_s;                   /* vrad_light_pass, the lump read back */
    vrad_pass_stats pass;
    vrad_bounce_stats bounce_stats;  /* zero when the map is not bounced */
    char error[256];                 /* the failing call's message */
} vrad_batch_map;

typedef struct vrad_batch_stats {
    int32_t workers;        /* workers that took maps */
    int32_t maps;
    int32_t failed;
    int32_t block;          /* the gather's threads per CTA; 0: each context's default */
    double seconds;         /* wall time of the whole batch */
    double busy_seconds;    /* sum of the maps' times */
    int64_t rays;           /* visibility, sky and transfer rays of every map */
    int64_t luxels;
    int64_t lighting_bytes;
    int64_t device_mallocs;      /* cudaMalloc calls of the library's device pool during the run */
    int64_t device_malloc_bytes;
    int64_t device_trims;        /* out-of-memory retries that emptied the pool's cache */
} vrad_batch_stats;

/* A batch runner on `device` with `workers` threads and contexts
 * (1..VRAD_BATCH_MAX_WORKERS). */
int32_t vrad_batch_create(int32_t device, int32_t workers, vrad_batch **out);
int32_t vrad_batch_destroy(vrad_batch *batch);

/* Lights every map; blocks until all are done.  workers: how many of the
 * batch's workers take maps (0: the count the autotuner chose, else all).
 * A worker hands its map's device tables back as soon as the map's lump is
 * read, and a map that ran out of device memory beside the others is lit
 * again at the end, alone.  Returns VRAD_OK when every map's status is
 * VRAD_OK; otherwise the first failing map's code, after all maps have
 * run. */
int32_t vrad_batch_run(vrad_batch *batch, vrad_batch_map *maps, int32_t nmaps, int32_t workers,
                       vrad_batch_stats *stats);

/* The batch's autotuner.  It first uploads the largest map on one context
 * and picks the gather's launch shape there (vrad_direct_autotune).  It then
 * lights all of `maps` once untimed on every worker (so that no count is
 * timed with its first allocations), then once per worker count
 * 1..created, and keeps the fastest count.  seconds (nullable, `created` entries) receives each count's wall
 * time.  The maps' outputs hold the last sweep's results. */
int32_t vrad_batch_autotune(vrad_batch *batch, vrad_batch_map *maps, int32_t nmaps, int32_t *chosen_workers,
                            int32_t *chosen_block, double *seconds);

/* DetMathF.Asin / DetMathF.Pow (MapFormats/Numerics/DetMathF.cs:141-164,
 * 265-292) as the device computes them inside the transfer build and the
 * spotlight falloff: the float nearest the exact value.  out[i] = asin a[i]
 * or a[i]^b[i] (b unused for the arcsine).  open (nullable) receives how
 * many results sat so near a rounding midpoint that the device could not
 * settle them (expected 0).  Host buffers; blocks. */
#define VRAD_DETMATH_ASIN 0
#define VRAD_DETMATH_POW 1
int32_t vrad_detmath(vrad_ctx *ctx, int32_t fn, const float *a, const float *b, float *out, int64_t n,
                     int64_t *open);

/* IRayTracer.TracerIdentity: backend, device and build, one token. */
int32_t vrad_tracer_identity(vrad_ctx *ctx, char *buf, int32_t cap);

/* The last error message on this context (or the last context-less error
 * when ctx is NULL).  Returns the message length. */
int32_t vrad_last_error(vrad_ctx *ctx, char *buf, int32_t cap);

/* Library version, for a loader's sanity check. */
int32_t vrad_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* VRAD_CUDA_H */
