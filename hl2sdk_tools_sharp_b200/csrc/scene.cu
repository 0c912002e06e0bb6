// scene.cu -- scene build: the reference's triangle intersection form and
// padded boxes on the device, the BVH's topology by the surface area
// heuristic on the host (bvh_sah.cu), the triangles gathered into leaf
// order on the device.
//
// Build pipeline:
//   k_prepare      KdTreeBuilder.ToIntersectionFormat per triangle (Correct
//                  compliance: exact sqrt and divides, no FMA contraction),
//                  unpadded box per triangle
//   k_bounds       scene bounds (one block, fixed-order reduction)
//   host           boxes padded, SAH tree (two-child nodes of 64 B, leaf
//                  references), uploaded
//   k_gather       triangles into leaf order
//
// The tree's shape is free: no answer depends on it (the traversal tests
// every triangle whose padded box the segment meets, and ties go to the
// lower original index), so only the boxes' conservativeness matters.

#include <cfloat>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "bvh_sah.h"
#include "device_pool.h"
#include "scene.cuh"
#include "sync_wait.h"

namespace vrad {

namespace {

__device__ inline float dmin(float a, float b) { return a < b ? a : b; }
__device__ inline float dmax(float a, float b) { return a > b ? a : b; }

// Vec3.Normalise (MapFormats/Geometry/Vec3.cs:178-189) and
// KdTreeBuilder.GetEdgeEquation / ToIntersectionFormat
// (MapTools/Tracing/KdTreeBuilder.cs:1530-1610), every operation an
// explicitly rounded intrinsic so none is contracted into an FMA.
__device__ inline void edge_equation(const float p1[3], const float p2[3], int c1, int c2,
                                     const float in[3], float out[3]) {
    float nx = __fsub_rn(p1[c2], p2[c2]);
    float ny = __fsub_rn(p2[c1], p1[c1]);
    float d = -__fadd_rn(__fmul_rn(nx, p1[c1]), __fmul_rn(ny, p1[c2]));
    float trial = __fadd_rn(__fadd_rn(__fmul_rn(in[c1], nx), __fmul_rn(in[c2], ny)), d);
    if (trial < 0.0f) {
        nx = -nx;
        ny = -ny;
        d = -d;
        trial = -trial;
    }
    out[0] = __fdiv_rn(nx, trial);
    out[1] = __fdiv_rn(ny, trial);
    out[2] = __fdiv_rn(d, trial);
}

__global__ void k_prepare(const vrad_triangle *__restrict__ in,
                          const vrad_kd_triangle *__restrict__ prepared,
                          const int32_t *__restrict__ orig, int n, float4 *__restrict__ t0,
                          float4 *__restrict__ t1, float4 *__restrict__ t2,
                          float *__restrict__ box) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const vrad_triangle &src = in[i];
    float p1[3] = {src.v0[0], src.v0[1], src.v0[2]};
    float p2[3] = {src.v1[0], src.v1[1], src.v1[2]};
    float p3[3] = {src.v2[0], src.v2[1], src.v2[2]};
    float nrm[3], eq1[3], eq2[3], d;
    int cs0, cs1, drop;
    int32_t id = src.id;
    uint32_t flags = src.flags;
    if (prepared) {
        const vrad_kd_triangle &p = prepared[i];
        nrm[0] = p.n[0];
        nrm[1] = p.n[1];
        nrm[2] = p.n[2];
        d = p.d;
        eq1[0] = p.e[0];
        eq1[1] = p.e[1];
        eq1[2] = p.e[2];
        eq2[0] = p.e[3];
        eq2[1] = p.e[4];
        eq2[2] = p.e[5];
        cs0 = p.cs0;
        cs1 = p.cs1;
        drop = 3 - cs0 - cs1;
        id = p.id;
        flags = p.flags;
    } else {
        float e1[3] = {__fsub_rn(p2[0], p1[0]), __fsub_rn(p2[1], p1[1]), __fsub_rn(p2[2], p1[2])};
        float e2[3] = {__fsub_rn(p3[0], p1[0]), __fsub_rn(p3[1], p1[1]), __fsub_rn(p3[2], p1[2])};
        float c[3] = {__fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1])),
                      __fsub_rn(__fmul_rn(e1[2], e2[0]), __fmul_rn(e1[0], e2[2])),
                      __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]))};
        float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(c[0], c[0]), __fmul_rn(c[1], c[1])),
                                         __fmul_rn(c[2], c[2])));
        if (len == 0.0f) {
            nrm[0] = nrm[1] = nrm[2] = 0.0f;
        } else {
            nrm[0] = __fdiv_rn(c[0], len);
            nrm[1] = __fdiv_rn(c[1], len);
            nrm[2] = __fdiv_rn(c[2], len);
        }
        drop = 0;
        for (int k = 1; k < 3; k++)
            if (fabsf(nrm[k]) > fabsf(nrm[drop])) drop = k;
        cs0 = (drop + 1) % 3;
        cs1 = (drop + 2) % 3;
        edge_equation(p1, p2, cs0, cs1, p3, eq1);
        edge_equation(p2, p3, cs0, cs1, p1, eq2);
        d = __fadd_rn(__fadd_rn(__fmul_rn(nrm[0], p1[0]), __fmul_rn(nrm[1], p1[1])),
                      __fmul_rn(nrm[2], p1[2]));
    }
    // The traversal reads the two projection axes as "the drop axis's
    // successors"; a caller-supplied form must follow the same rule.
    if (cs0 != (drop + 1) % 3 || cs1 != (drop + 2) % 3) drop = 3;  // flagged below
    uint32_t meta = (uint32_t)(drop & 3) | (((uint32_t)id & kTraceIdSky) ? 4u : 0u) | (flags << 8);
    t0[i] = make_float4(nrm[0], nrm[1], nrm[2], d);
    t1[i] = make_float4(eq1[0], eq1[1], eq1[2], eq2[0]);
    t2[i] = make_float4(eq2[1], eq2[2], __int_as_float(orig[i]), __uint_as_float(meta));
    for (int a = 0; a < 3; a++) {
        box[6 * i + a] = dmin(dmin(p1[a], p2[a]), p3[a]);
        box[6 * i + 3 + a] = dmax(dmax(p1[a], p2[a]), p3[a]);
    }
}

// Scene bounds by one block: fixed-order strided scan, then a tree
// reduction in shared memory.  bounds[0..2] = min, [3..5] = max,
// bounds[6] = largest absolute coordinate.
__global__ void k_bounds(const float *__restrict__ box, int n, float *__restrict__ bounds) {
    __shared__ float s[7][256];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        for (int a = 0; a < 3; a++) {
            lo[a] = dmin(lo[a], box[6 * i + a]);
            hi[a] = dmax(hi[a], box[6 * i + 3 + a]);
        }
    }
    for (int a = 0; a < 3; a++) {
        s[a][threadIdx.x] = lo[a];
        s[3 + a][threadIdx.x] = hi[a];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            for (int a = 0; a < 3; a++) {
                s[a][threadIdx.x] = dmin(s[a][threadIdx.x], s[a][threadIdx.x + w]);
                s[3 + a][threadIdx.x] = dmax(s[3 + a][threadIdx.x], s[3 + a][threadIdx.x + w]);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        float m = 0.0f;
        for (int a = 0; a < 6; a++) {
            bounds[a] = s[a][0];
            m = dmax(m, fabsf(s[a][0]));
        }
        bounds[6] = m;
    }
}

// A one-triangle scene: a root whose second child is an empty box.
__global__ void k_emit_single(const float *__restrict__ leaf_box, float4 *__restrict__ nodes) {
    const float *b = leaf_box;
    nodes[0] = make_float4(b[0], b[3], b[1], b[4]);
    nodes[1] = make_float4(FLT_MAX, -FLT_MAX, FLT_MAX, -FLT_MAX);
    nodes[2] = make_float4(b[2], b[5], FLT_MAX, -FLT_MAX);
    nodes[3] = make_float4(__int_as_float(leaf_ref(0, 1)), __int_as_float(leaf_ref(0, 1)), 0.0f, 0.0f);
}

__global__ void k_pad_single(const float *__restrict__ tri_box, const float *__restrict__ bounds,
                             float *__restrict__ leaf_box) {
    const float pad = ldexpf(bounds[6], -16) + 1e-6f;
    for (int a = 0; a < 3; a++) {
        leaf_box[a] = tri_box[a] - pad;
        leaf_box[3 + a] = tri_box[3 + a] + pad;
    }
}

__global__ void k_gather(const int32_t *__restrict__ order, int n, const float4 *__restrict__ s0,
                         const float4 *__restrict__ s1, const float4 *__restrict__ s2,
                         float4 *__restrict__ d0, float4 *__restrict__ d1, float4 *__restrict__ d2) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int src = order[k];
    d0[k] = s0[src];
    d1[k] = s1[src];
    d2[k] = s2[src];
}

__global__ void k_check_axes(const float4 *__restrict__ t2, int n, int *__restrict__ stats) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if ((__float_as_uint(t2[i].w) & 3u) == 3u) atomicAdd(&stats[3], 1);
}

inline int blocks(int n, int b) { return (n + b - 1) / b; }

}  // namespace

#define VRAD_TRY(expr)                                   \
    do {                                                 \
        cudaError_t e__ = (expr);                        \
        if (e__ != cudaSuccess) {                        \
            err = e__;                                   \
            goto fail;                                   \
        }                                                \
    } while (0)

cudaError_t build_bvh(BvhBuffers &sb, const vrad_triangle *h_tris,
                      const vrad_kd_triangle *h_prepared, const int32_t *h_orig, int n,
                      cudaStream_t stream, SceneBuildReport *report) {
    cudaError_t err = cudaSuccess;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Scratch (freed at the end of the build).
    vrad_triangle *d_in = nullptr;
    vrad_kd_triangle *d_prep = nullptr;
    int32_t *d_orig = nullptr;
    float4 *u0 = nullptr, *u1 = nullptr, *u2 = nullptr;
    float *tri_box = nullptr, *d_bounds = nullptr, *leaf_box = nullptr;
    int32_t *order = nullptr;
    int *d_stats = nullptr;
    int stats[4] = {0, 0, 0, 0};
    float bounds[7];
    const int inner = n > 1 ? n - 1 : 1;
    SahTree tree;

    sb.release();
    if (n <= 0) return cudaSuccess;  // an empty subset: no BVH, never traversed
    VRAD_TRY(cudaEventCreate(&ev0));
    VRAD_TRY(cudaEventCreate(&ev1));
    VRAD_TRY(cudaEventRecord(ev0, stream));

    VRAD_TRY(dev_alloc(&d_in, sizeof(vrad_triangle) * n));
    VRAD_TRY(cudaMemcpyAsync(d_in, h_tris, sizeof(vrad_triangle) * n, cudaMemcpyHostToDevice, stream));
    if (h_prepared) {
        VRAD_TRY(dev_alloc(&d_prep, sizeof(vrad_kd_triangle) * n));
        VRAD_TRY(cudaMemcpyAsync(d_prep, h_prepared, sizeof(vrad_kd_triangle) * n,
                                 cudaMemcpyHostToDevice, stream));
    }
    VRAD_TRY(dev_alloc(&d_orig, sizeof(int32_t) * n));
    VRAD_TRY(cudaMemcpyAsync(d_orig, h_orig, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
    VRAD_TRY(dev_alloc(&u0, sizeof(float4) * n));
    VRAD_TRY(dev_alloc(&u1, sizeof(float4) * n));
    VRAD_TRY(dev_alloc(&u2, sizeof(float4) * n));
    VRAD_TRY(dev_alloc(&tri_box, sizeof(float) * 6 * n));
    VRAD_TRY(dev_alloc(&d_bounds, sizeof(float) * 8));
    VRAD_TRY(dev_alloc(&sb.tri0, sizeof(float4) * n));
    VRAD_TRY(dev_alloc(&sb.tri1, sizeof(float4) * n));
    VRAD_TRY(dev_alloc(&sb.tri2, sizeof(float4) * n));
    VRAD_TRY(dev_alloc(&sb.nodes, sizeof(float4) * 4 * inner));
    VRAD_TRY(dev_alloc(&leaf_box, sizeof(float) * 6 * n));
    VRAD_TRY(dev_alloc(&d_stats, sizeof(int) * 4));
    VRAD_TRY(cudaMemsetAsync(d_stats, 0, sizeof(int) * 4, stream));

    k_prepare<<<blocks(n, 128), 128, 0, stream>>>(d_in, d_prep, d_orig, n, u0, u1, u2, tri_box);
    VRAD_TRY(cudaGetLastError());
    k_bounds<<<1, 256, 0, stream>>>(tri_box, n, d_bounds);
    VRAD_TRY(cudaGetLastError());
    k_check_axes<<<blocks(n, 256), 256, 0, stream>>>(u2, n, d_stats);
    VRAD_TRY(cudaGetLastError());

    if (n == 1) {
        int32_t zero = 0;
        VRAD_TRY(dev_alloc(&order, sizeof(int32_t)));
        VRAD_TRY(cudaMemcpyAsync(order, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        k_pad_single<<<1, 1, 0, stream>>>(tri_box, d_bounds, leaf_box);
        k_emit_single<<<1, 1, 0, stream>>>(leaf_box, sb.nodes);
        k_gather<<<1, 32, 0, stream>>>(order, 1, u0, u1, u2, sb.tri0, sb.tri1, sb.tri2);
        VRAD_TRY(cudaGetLastError());
        stats[0] = 1;
        stats[1] = 1;
        stats[2] = 1;
        sb.depth = 1;
    } else {
        // The boxes to the host, padded there as the walk's slab test needs
        // (a scene-relative margin), the SAH tree built, its nodes and leaf
        // order back.
        std::vector<float> box((size_t)6 * n);
        VRAD_TRY(cudaMemcpyAsync(box.data(), tri_box, sizeof(float) * box.size(), cudaMemcpyDeviceToHost, stream));
        VRAD_TRY(cudaMemcpyAsync(bounds, d_bounds, sizeof(float) * 7, cudaMemcpyDeviceToHost, stream));
        VRAD_TRY(vrad::wait_stream(stream));
        const float pad = ldexpf(bounds[6], -16) + 1e-6f;
        for (int i = 0; i < n; i++)
            for (int a = 0; a < 3; a++) {
                box[6 * (size_t)i + a] -= pad;
                box[6 * (size_t)i + 3 + a] += pad;
            }
        build_sah(box.data(), n, tree);
        VRAD_TRY(dev_alloc(&order, sizeof(int32_t) * n));
        VRAD_TRY(cudaMemcpyAsync(order, tree.order.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
        VRAD_TRY(cudaMemcpyAsync(sb.nodes, tree.nodes.data(), sizeof(float4) * tree.nodes.size(),
                                 cudaMemcpyHostToDevice, stream));
        k_gather<<<blocks(n, 256), 256, 0, stream>>>(order, n, u0, u1, u2, sb.tri0, sb.tri1, sb.tri2);
        VRAD_TRY(cudaGetLastError());
        stats[0] = tree.inner;
        stats[1] = tree.leaves;
        stats[2] = tree.max_leaf;
        sb.depth = tree.depth > kStackDepth ? kStackDepth : tree.depth;  // deeper: walks report an overflow
    }
    {
        int dstats[4];
        VRAD_TRY(cudaMemcpyAsync(dstats, d_stats, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream));
        VRAD_TRY(cudaMemcpyAsync(bounds, d_bounds, sizeof(float) * 7, cudaMemcpyDeviceToHost, stream));
        VRAD_TRY(cudaEventRecord(ev1, stream));
        VRAD_TRY(vrad::wait_stream(stream));
        stats[3] = dstats[3];
    }
    if (stats[3] != 0) {
        err = cudaErrorInvalidValue;  // a supplied form whose axes are not the drop axis's successors
        goto fail;
    }
    sb.ntris = n;
    if (report) {
        report->max_depth = sb.depth > report->max_depth ? sb.depth : report->max_depth;
        const bool first = report->nodes == 0 && report->leaves == 0;
        report->nodes += stats[0];
        report->leaves += stats[1];
        report->max_leaf = stats[2] > report->max_leaf ? stats[2] : report->max_leaf;
        report->sah_cost += tree.sah_cost;
        for (int a = 0; a < 3; a++) {
            report->bounds[a] = first ? bounds[a] : fminf(report->bounds[a], bounds[a]);
            report->bounds[3 + a] = first ? bounds[3 + a] : fmaxf(report->bounds[3 + a], bounds[3 + a]);
        }
        report->pad = fmaxf(report->pad, ldexpf(bounds[6], -16) + 1e-6f);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        report->build_ms += ms;
        report->device_bytes += (int64_t)n * 48 + (int64_t)inner * 64;
    }

fail:
    // The scratch goes back to the device pool once the stream is done with it.
    if (err != cudaSuccess) vrad::wait_stream(stream);
    dev_free(d_in);
    dev_free(d_prep);
    dev_free(d_orig);
    dev_free(u0);
    dev_free(u1);
    dev_free(u2);
    dev_free(tri_box);
    dev_free(d_bounds);
    dev_free(leaf_box);
    dev_free(order);
    dev_free(d_stats);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (err != cudaSuccess) sb.release();
    return err;
}

void BvhBuffers::release() {
    dev_free(tri0);
    dev_free(tri1);
    dev_free(tri2);
    dev_free(nodes);
    tri0 = tri1 = tri2 = nullptr;
    nodes = nullptr;
    ntris = 0;
    depth = 0;
}

void SceneBuffers::release() {
    opaque.release();
    sky.release();
    dev_free(tri_id);
    tri_id = nullptr;
    ntris = 0;
}

}  // namespace vrad
