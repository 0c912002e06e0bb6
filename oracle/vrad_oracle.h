/*
 * vrad_oracle.h -- CPU oracle for the vrad lighting path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, its
 * C ABI, the Python host layer) links, loads or calls anything declared here.
 * Only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * use it, and only as the checker.
 *
 * This is a plain C++17 restatement of the reference's CPU arithmetic
 * (SourceSharp.MapTools, Correct compliance).  Each function names the
 * reference file and lines it follows.  Parity is pinned against the
 * reference's own stock-tracer fixtures (kd-scene / kd-boxes answers), see
 * tests/test_oracle_fixtures.py.
 */
#ifndef VRAD_ORACLE_H
#define VRAD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* KdTriangle (MapTools/Tracing/KdTree.cs:120-167): 48 bytes. */
typedef struct orc_tri {
    float nx, ny, nz, d;
    int32_t id;
    float e[6];
    uint8_t cs0, cs1, flags, unused;
} orc_tri;

/* Ray (MapTools/Tracing/IRayTracer.cs:32): 28 bytes. */
typedef struct orc_ray {
    float ox, oy, oz, dx, dy, dz, reach;
} orc_ray;

/* KdNode (MapTools/Tracing/KdTree.cs:60-100): 8 bytes. */
typedef struct orc_kdnode {
    int32_t children;
    float split;
} orc_kdnode;

enum {
    ORC_CLOSEST = 1,    /* closest hit (else visibility)            */
    ORC_ISOLATED = 2,   /* RayTraceOptions.IsolatedRays             */
    ORC_SKY_PASS = 4,   /* RayTraceOptions.SkyDoesNotBlock          */
    ORC_FULL_WALK = 8,  /* KdRayTracer.WithFullVisibilityWalk       */
};

/* TraceId.Sky (MapTools/Rad/TraceId.cs). */
#define ORC_TRACE_ID_SKY 0x01000000

/* Correct-mode KdTreeBuilder.ToIntersectionFormat for n triangles given as
 * nine floats each (v0, v1, v2). */
int orc_tri_prepare(const float *verts9, const int32_t *ids, const uint8_t *flags,
                    int32_t n, orc_tri *out);

/* KdRayTracer.TraceVisibility / TraceClosest over an already-built tree.
 * out_tri receives the tree's triangle INDEX (-1 on a miss), out_dist the
 * raw hit distance, out_bits (visibility only) one bit per ray. */
int orc_kd_trace(const orc_kdnode *nodes, int32_t nnodes, const int32_t *indices,
                 int32_t nindices, const orc_tri *tris, int32_t ntris,
                 const float *bounds6, const orc_ray *rays, int32_t nrays,
                 float tmin, int32_t skip_id, int32_t flags, int32_t *out_tri,
                 float *out_dist, uint64_t *out_bits, int32_t threads);

/* The semantic the CUDA tracer implements, by brute force over every
 * triangle with the same FP32 predicate: visibility = any accepted hit with
 * tmin <= t < reach; closest = lexicographic minimum of (t, triangle index)
 * over accepted hits with tmin <= t < reach.  out_tri = triangle index or -1,
 * out_dist = t. */
int orc_brute_trace(const orc_tri *tris, int32_t ntris, const orc_ray *rays,
                    int32_t nrays, float tmin, int32_t skip_id, int32_t flags,
                    int32_t *out_tri, float *out_dist, uint64_t *out_bits,
                    int32_t threads);

/* KdTreeBuilder (MapTools/Tracing/KdTreeBuilder.cs): SAH KD build.
 * Returns the node / index counts through the pointers; the arrays are
 * owned by the oracle until orc_kd_free. */
typedef struct orc_kdtree {
    orc_kdnode *nodes;
    int32_t nnodes;
    int32_t *indices;
    int32_t nindices;
    orc_tri *tris;
    int32_t ntris;
    float bounds[6];
} orc_kdtree;

int orc_kd_build(const float *verts9, const int32_t *ids, const uint8_t *flags, int32_t n,
                 orc_kdtree *out);
void orc_kd_free(orc_kdtree *tree);

/* FP64 classification of each ray against the triangles' true geometry:
 * 1 = blocked by a margin, 0 = clear by a margin, 2 = within margin (ambiguous). */
int orc_fp64_classify(const float *verts9, int32_t ntris, const orc_ray *rays, int32_t nrays,
                      double rel_margin, int8_t *out_class, int32_t threads);

/* ---- lighting stage ---------------------------------------------------- */

/* A lit face (the inputs of FaceLightInfo.Build).  Same layout as the
 * library's vrad_face so a test can hand one buffer to both. */
typedef struct orc_face {
    float normal[3];
    float dist;
    float vecs[2][4];
    int32_t mins[2];
    int32_t size[2];
    int32_t first_vertex;
    int32_t num_vertices;
    int32_t cluster;
    int32_t flags;
} orc_face;

/* LightSample (FaceLight.cs:30-70).  Same layout as vrad_sample. */
typedef struct orc_sample {
    float position[3];
    float area;
    float coord[2];
    float mins[2];
    float maxs[2];
    int32_t s, t;
    int32_t face;
    int32_t cluster;
} orc_sample;

/* DirectLight fields (DirectLight.cs).  Same layout as vrad_light. */
typedef struct orc_light {
    int32_t type;
    int32_t style;
    float origin[3];
    float intensity[3];
    float normal[3];
    float stop_dot, stop_dot2, exponent;
    float constant, linear, quadratic;
    float start_fade, end_fade, cap_dist;
} orc_light;

/* FaceSampleBuilder.BuildFacesamples over every face. */
int orc_build_samples(const orc_face *faces, int32_t nfaces, const float *verts, orc_sample *out,
                      int64_t capacity, int64_t *count, int64_t *first);

/* The direct gather (style 0, flat faces) over every sample, in four-sample
 * groups per face, then up to extra_passes supersampling passes per face
 * (the samples must be the builder's own for the faces and verts given:
 * -2 otherwise); out is 4 floats per sample (lighting xyz, sun amount). */
int orc_direct(const orc_kdnode *nodes, const int32_t *indices, const orc_tri *tris,
               const float *bounds6, const orc_face *faces, int32_t nfaces, const float *verts,
               const orc_sample *samples, const int64_t *face_first, const orc_light *lights,
               const int32_t *cl_off, const int32_t *cl_list, const float *dirs, int32_t ndirs,
               const float *jitter, int32_t sun_samples, float sun_extent, int32_t extra_passes,
               float *out, int32_t threads, int64_t *rays_out, int64_t *supersampled_out);

/* orc_direct with light styles: out is slot 0; out_slots (nullable) slots
 * 1..3 (each nsamples x 4 floats, zero where the face has no such slot);
 * face_styles (nullable) 4 bytes per face, 255 for an empty slot; dropped
 * (nullable) the faces warned of a fifth style. */
int orc_direct_styles(const orc_kdnode *nodes, const int32_t *indices, const orc_tri *tris,
                      const float *bounds6, const orc_face *faces, int32_t nfaces, const float *verts,
                      const orc_sample *samples, const int64_t *face_first, const orc_light *lights,
                      const int32_t *cl_off, const int32_t *cl_list, const float *dirs, int32_t ndirs,
                      const float *jitter, int32_t sun_samples, float sun_extent, int32_t extra_passes,
                      float *out, float *out_slots, uint8_t *face_styles, int64_t *dropped, int32_t threads,
                      int64_t *rays_out, int64_t *supersampled_out);

/* FaceNeighbours.Build for smoothing groups 0 (vertices welded by position). */
int orc_neighbours(const orc_face *faces, int32_t nfaces, const float *verts, float threshold,
                   int32_t *offsets, int32_t *list, int64_t capacity, int64_t *count);

/* FinalLightFace for every face, bounce 0: the LIGHTING lump bytes (total
 * size in *total; lighting may be NULL to size it) and each face's lightofs.
 * sample_light is the direct gather's output, 4 floats per sample. */
int orc_final(const orc_face *faces, int32_t nfaces, const float *verts, const orc_sample *samples,
              const int64_t *face_first, const float *sample_light, uint8_t *lighting,
              int64_t capacity, int32_t *lightofs, int64_t *total);

/* ---- bounce ------------------------------------------------------------- */

/* Patch (Patch.cs), the fields compared with the library's vrad_patch;
 * same layout. */
typedef struct orc_patch {
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
} orc_patch;

/* A world for the bounce: faces and windings, samples (face-major, with
 * face_first), per-face reflectivity, the PVS (per cluster, ascending
 * clusters), chop sizes, the stop rule, the KD scene for the transfer rays
 * and a thread count. */
typedef struct orc_bounce_in {
    const orc_face *faces;
    int32_t nfaces;
    const float *verts;
    const orc_sample *samples;
    const int64_t *face_first;
    const float *reflectivity;
    const int32_t *pvs_off;
    const int32_t *pvs_list;
    int32_t nclusters;
    float max_chop;
    float min_chop;
    int32_t bounces;
    float threshold;
    const orc_kdnode *nodes;
    const int32_t *indices;
    const orc_tri *tris;
    const float *bounds6;
    int32_t threads;
} orc_bounce_in;

/* PatchBuilder + PatchSubdivider; returns a handle. */
void *orc_bounce_new(const orc_bounce_in *in);
void orc_bounce_free(void *h);
/* The patches and their windings (counts only with out and points NULL). */
int orc_bounce_patches(void *h, orc_patch *out, int64_t capacity, int64_t *count, float *points,
                       int64_t point_capacity, int64_t *point_count);
/* VisMatrix for the given receivers (patch indices; NULL = every receiver
 * in ReceiverOrder), lists by patch index in offsets[npatches + 1]; rays =
 * candidate rays traced.  src / weight NULL: counts only. */
int orc_bounce_transfers(void *h, const int32_t *receivers, int32_t nreceivers, int64_t *offsets, int32_t *src,
                         float *weight, int64_t capacity, int64_t *count, int64_t *rays);
/* Replaces the transfers (lists by patch index). */
int orc_bounce_set_transfers(void *h, const int64_t *offsets, const int32_t *src, const float *weight);
/* BuildPatchLights from the direct sample light (4 floats per sample), then
 * (building every transfer first unless set) Radiosity.BounceAsync.
 * Outputs per patch xyz: TotalLight.Flat and DirectLight. */
int orc_bounce_run(void *h, const float *sample_light, float *total_light, float *direct_light,
                   int32_t *bounces_run, float *added);
/* FinalLightFace for every face with the bounced light of the last run. */
int orc_bounce_final(void *h, const float *sample_light, uint8_t *lighting, int64_t capacity, int32_t *lightofs,
                     int64_t *total);
/* orc_bounce_final with light styles (slots 1..3 and 4 style bytes per
 * face, as orc_direct_styles gives them); the bounce goes into slot 0. */
int orc_bounce_final_styles(void *h, const float *sample_light, const float *slots_light, const uint8_t *face_styles,
                            uint8_t *lighting, int64_t capacity, int32_t *lightofs, int64_t *total);
/* orc_final with light styles. */
int orc_final_styles(const orc_face *faces, int32_t nfaces, const float *verts, const orc_sample *samples,
                     const int64_t *face_first, const float *sample_light, const float *slots_light,
                     const uint8_t *face_styles, uint8_t *lighting, int64_t capacity, int32_t *lightofs,
                     int64_t *total);
/* Rays traced so far; *blocked of them blocked. */
int64_t orc_bounce_stats(void *h, int64_t *blocked);
/* Drops the built transfer lists (the next build traces again). */
void orc_bounce_forget_transfers(void *h);
/* Every receiver's candidate pairs, counted without tracing. */
int64_t orc_bounce_count_candidates(void *h);
/* DetMathF.Pow as the oracle computes it. */
float orc_powf(float x, float y);
/* DetMathF.Asin as the oracle computes it. */
float orc_asin(float x);
/* FormFactors.DiffToDiff (o1, n1, o2, n2 as 12 floats) and PolyToDiff
 * (MapTools/Rad/Bounce/FormFactors.cs:58-140). */
float orc_diff_to_diff(const float *q);
float orc_poly_to_diff(const float *points, int32_t count, float area, const float *origin, const float *normal);

#ifdef __cplusplus
}
#endif

#endif
