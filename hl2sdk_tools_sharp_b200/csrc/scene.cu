// scene.cu -- scene build on the device: the reference's triangle
// intersection form, padded boxes, and a BVH built entirely on the GPU.
//
// Build pipeline (one stream, no host round trips between kernels):
//   k_prepare      KdTreeBuilder.ToIntersectionFormat per triangle (Correct
//                  compliance: exact sqrt and divides, no FMA contraction),
//                  unpadded box per triangle
//   k_bounds       scene bounds (one block, fixed-order reduction)
//   k_morton       63-bit Morton code of each box centre
//   radix sort     (code, index) pairs
//   k_radix_tree   Karras' binary radix tree over the sorted codes
//   k_refit        bottom-up padded boxes + SAH collapse decision
//   k_emit         two-child nodes (64 B) and leaf references
//   k_gather       triangles into leaf order
//
// The tree's shape is free: no answer depends on it (the traversal tests
// every triangle whose padded box the segment meets, and ties go to the
// lower original index), so only the boxes' conservativeness matters.

#include <cub/device/device_radix_sort.cuh>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "scene.cuh"

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

__device__ inline uint64_t spread21(uint32_t x) {
    uint64_t v = x & 0x1fffffu;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(const float *__restrict__ box, int n, const float *__restrict__ bounds,
                         uint64_t *__restrict__ codes, int32_t *__restrict__ order) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t q[3];
    for (int a = 0; a < 3; a++) {
        float c = 0.5f * (box[6 * i + a] + box[6 * i + 3 + a]);
        float ext = bounds[3 + a] - bounds[a];
        float u = ext > 0.0f ? (c - bounds[a]) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        q[a] = (uint32_t)fminf(u * 2097152.0f, 2097151.0f);
    }
    codes[i] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
    order[i] = i;
}

// Common-prefix length of sorted keys i and j, index-extended for equal
// codes (Karras 2012); -1 outside [0, n).
__device__ inline int delta(const uint64_t *codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = codes[i], b = codes[j];
    if (a != b) return __clzll((long long)(a ^ b));
    return 64 + __clz(i ^ j);
}

// Inner node i of the radix tree over n sorted leaves.  child refs use
// c >= 0 for inner nodes and c = ~leaf for leaves.
__global__ void k_radix_tree(const uint64_t *__restrict__ codes, int n, int2 *__restrict__ child,
                             int2 *__restrict__ range, int32_t *__restrict__ parent_inner,
                             int32_t *__restrict__ parent_leaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin_ = delta(codes, n, i, i - d);
    int lmax = 2;
    while (delta(codes, n, i, i + lmax * d) > dmin_) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(codes, n, i, i + (l + t) * d) > dmin_) l += t;
    int j = i + l * d;
    int dnode = delta(codes, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + (d < 0 ? -1 : 0);
    int lo = i < j ? i : j, hi = i < j ? j : i;
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    child[i] = make_int2(left, right);
    range[i] = make_int2(lo, hi);
    if (left < 0) parent_leaf[~left] = i; else parent_inner[left] = i;
    if (right < 0) parent_leaf[~right] = i; else parent_inner[right] = i;
}

__device__ inline float half_area(const float *b) {
    float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return dx * dy + dy * dz + dz * dx;
}

// Bottom-up: padded boxes of every inner node and its SAH cost; a subtree
// of at most kMaxLeaf triangles becomes one leaf when that is no dearer.
__global__ void k_refit(const float *__restrict__ tri_box, const int32_t *__restrict__ order,
                        int n, const int2 *__restrict__ child, const int32_t *__restrict__ parent_inner,
                        const int32_t *__restrict__ parent_leaf, const float *__restrict__ bounds,
                        float *node_box, float *node_cost, int32_t *collapse,
                        uint32_t *__restrict__ arrivals, float *__restrict__ leaf_box) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float pad = ldexpf(bounds[6], -16) + 1e-6f;
    int src = order[k];
    for (int a = 0; a < 3; a++) {
        leaf_box[6 * k + a] = tri_box[6 * src + a] - pad;
        leaf_box[6 * k + 3 + a] = tri_box[6 * src + 3 + a] + pad;
    }
    __threadfence();
    const float ct = 1.0f, ci = 1.0f;
    int node = parent_leaf[k];
    while (node >= 0) {
        if (atomicAdd(&arrivals[node], 1u) == 0u) return;  // first arrival: sibling not ready
        __threadfence();
        int2 c = child[node];
        float b[6], bl[6], br[6], costl, costr;
        int cntl, cntr;
        const float *pl = c.x < 0 ? &leaf_box[6 * (~c.x)] : &node_box[6 * c.x];
        const float *pr = c.y < 0 ? &leaf_box[6 * (~c.y)] : &node_box[6 * c.y];
        for (int a = 0; a < 6; a++) {
            bl[a] = __ldcg(pl + a);
            br[a] = __ldcg(pr + a);
        }
        costl = c.x < 0 ? ci : __ldcg(&node_cost[c.x]);
        costr = c.y < 0 ? ci : __ldcg(&node_cost[c.y]);
        cntl = c.x < 0 ? 1 : __ldcg(&collapse[c.x]) >> 1;
        cntr = c.y < 0 ? 1 : __ldcg(&collapse[c.y]) >> 1;
        for (int a = 0; a < 3; a++) {
            b[a] = dmin(bl[a], br[a]);
            b[3 + a] = dmax(bl[3 + a], br[3 + a]);
        }
        float sa = fmaxf(half_area(b), 1e-30f);
        float split = ct + (half_area(bl) * costl + half_area(br) * costr) / sa;
        int cnt = cntl + cntr;
        float leaf = ci * (float)cnt;
        bool as_leaf = cnt <= kMaxLeaf && leaf <= split;
        for (int a = 0; a < 6; a++) node_box[6 * node + a] = b[a];
        node_cost[node] = as_leaf ? leaf : split;
        collapse[node] = (cnt << 1) | (as_leaf ? 1 : 0);
        __threadfence();
        node = parent_inner[node];
    }
}

__device__ inline int32_t ref_of(int c, const int2 *range, const int32_t *collapse) {
    if (c < 0) return leaf_ref(~c, 1);
    if (collapse[c] & 1) {
        int2 r = range[c];
        return leaf_ref(r.x, r.y - r.x + 1);
    }
    return c;
}

__global__ void k_emit(int n, const int2 *__restrict__ child, const int2 *__restrict__ range,
                       const int32_t *__restrict__ collapse, const float *__restrict__ node_box,
                       const float *__restrict__ leaf_box, float4 *__restrict__ nodes) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int2 c = child[i];
    const float *b0 = c.x < 0 ? &leaf_box[6 * (~c.x)] : &node_box[6 * c.x];
    const float *b1 = c.y < 0 ? &leaf_box[6 * (~c.y)] : &node_box[6 * c.y];
    nodes[4 * i + 0] = make_float4(b0[0], b0[3], b0[1], b0[4]);
    nodes[4 * i + 1] = make_float4(b1[0], b1[3], b1[1], b1[4]);
    nodes[4 * i + 2] = make_float4(b0[2], b0[5], b1[2], b1[5]);
    nodes[4 * i + 3] = make_float4(__int_as_float(ref_of(c.x, range, collapse)),
                                   __int_as_float(ref_of(c.y, range, collapse)), 0.0f, 0.0f);
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

__global__ void k_count_leaves(int n, const int2 *__restrict__ child, const int2 *__restrict__ range,
                               const int32_t *__restrict__ collapse, const int32_t *__restrict__ parent_inner,
                               int *__restrict__ stats) {
    // stats[0] = reachable inner nodes, stats[1] = leaves, stats[2] = largest leaf,
    // stats[3] = bad projection axes in a supplied form.
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    // Reachable iff no ancestor (including itself) is collapsed.
    bool reachable = !(collapse[i] & 1);
    for (int p = parent_inner[i]; reachable && p >= 0; p = parent_inner[p]) reachable = !(collapse[p] & 1);
    if (!reachable) return;
    atomicAdd(&stats[0], 1);
    int2 c = child[i];
    for (int s = 0; s < 2; s++) {
        int ch = s ? c.y : c.x;
        int cnt = 0;
        if (ch < 0) cnt = 1;
        else if (collapse[ch] & 1) cnt = range[ch].y - range[ch].x + 1;
        if (cnt) {
            atomicAdd(&stats[1], 1);
            atomicMax(&stats[2], cnt);
        }
    }
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
    float *tri_box = nullptr, *d_bounds = nullptr, *node_box = nullptr, *node_cost = nullptr,
          *leaf_box = nullptr;
    uint64_t *codes = nullptr, *codes_sorted = nullptr;
    int32_t *order = nullptr, *order_sorted = nullptr, *parent_inner = nullptr,
            *parent_leaf = nullptr, *collapse = nullptr;
    int2 *child = nullptr, *range = nullptr;
    uint32_t *arrivals = nullptr;
    int *d_stats = nullptr;
    void *sort_tmp = nullptr;
    size_t sort_bytes = 0;
    int stats[4] = {0, 0, 0, 0};
    float bounds[7];
    const int inner = n > 1 ? n - 1 : 1;

    sb.release();
    if (n <= 0) return cudaSuccess;  // an empty subset: no BVH, never traversed
    VRAD_TRY(cudaEventCreate(&ev0));
    VRAD_TRY(cudaEventCreate(&ev1));
    VRAD_TRY(cudaEventRecord(ev0, stream));

    VRAD_TRY(cudaMalloc(&d_in, sizeof(vrad_triangle) * n));
    VRAD_TRY(cudaMemcpyAsync(d_in, h_tris, sizeof(vrad_triangle) * n, cudaMemcpyHostToDevice, stream));
    if (h_prepared) {
        VRAD_TRY(cudaMalloc(&d_prep, sizeof(vrad_kd_triangle) * n));
        VRAD_TRY(cudaMemcpyAsync(d_prep, h_prepared, sizeof(vrad_kd_triangle) * n,
                                 cudaMemcpyHostToDevice, stream));
    }
    VRAD_TRY(cudaMalloc(&d_orig, sizeof(int32_t) * n));
    VRAD_TRY(cudaMemcpyAsync(d_orig, h_orig, sizeof(int32_t) * n, cudaMemcpyHostToDevice, stream));
    VRAD_TRY(cudaMalloc(&u0, sizeof(float4) * n));
    VRAD_TRY(cudaMalloc(&u1, sizeof(float4) * n));
    VRAD_TRY(cudaMalloc(&u2, sizeof(float4) * n));
    VRAD_TRY(cudaMalloc(&tri_box, sizeof(float) * 6 * n));
    VRAD_TRY(cudaMalloc(&d_bounds, sizeof(float) * 8));
    VRAD_TRY(cudaMalloc(&sb.tri0, sizeof(float4) * n));
    VRAD_TRY(cudaMalloc(&sb.tri1, sizeof(float4) * n));
    VRAD_TRY(cudaMalloc(&sb.tri2, sizeof(float4) * n));
    VRAD_TRY(cudaMalloc(&sb.nodes, sizeof(float4) * 4 * inner));
    VRAD_TRY(cudaMalloc(&leaf_box, sizeof(float) * 6 * n));
    VRAD_TRY(cudaMalloc(&d_stats, sizeof(int) * 4));
    VRAD_TRY(cudaMemsetAsync(d_stats, 0, sizeof(int) * 4, stream));

    k_prepare<<<blocks(n, 128), 128, 0, stream>>>(d_in, d_prep, d_orig, n, u0, u1, u2, tri_box);
    VRAD_TRY(cudaGetLastError());
    k_bounds<<<1, 256, 0, stream>>>(tri_box, n, d_bounds);
    VRAD_TRY(cudaGetLastError());
    k_check_axes<<<blocks(n, 256), 256, 0, stream>>>(u2, n, d_stats);
    VRAD_TRY(cudaGetLastError());

    if (n == 1) {
        int32_t zero = 0;
        VRAD_TRY(cudaMalloc(&order, sizeof(int32_t)));
        VRAD_TRY(cudaMemcpyAsync(order, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        k_pad_single<<<1, 1, 0, stream>>>(tri_box, d_bounds, leaf_box);
        k_emit_single<<<1, 1, 0, stream>>>(leaf_box, sb.nodes);
        k_gather<<<1, 32, 0, stream>>>(order, 1, u0, u1, u2, sb.tri0, sb.tri1, sb.tri2);
        VRAD_TRY(cudaGetLastError());
        stats[0] = 1;
        stats[1] = 1;
        stats[2] = 1;
    } else {
        VRAD_TRY(cudaMalloc(&codes, sizeof(uint64_t) * n));
        VRAD_TRY(cudaMalloc(&codes_sorted, sizeof(uint64_t) * n));
        VRAD_TRY(cudaMalloc(&order, sizeof(int32_t) * n));
        VRAD_TRY(cudaMalloc(&order_sorted, sizeof(int32_t) * n));
        k_morton<<<blocks(n, 256), 256, 0, stream>>>(tri_box, n, d_bounds, codes, order);
        VRAD_TRY(cudaGetLastError());
        VRAD_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, codes, codes_sorted, order,
                                                 order_sorted, n, 0, 63, stream));
        VRAD_TRY(cudaMalloc(&sort_tmp, sort_bytes));
        VRAD_TRY(cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, codes, codes_sorted, order,
                                                 order_sorted, n, 0, 63, stream));

        VRAD_TRY(cudaMalloc(&child, sizeof(int2) * inner));
        VRAD_TRY(cudaMalloc(&range, sizeof(int2) * inner));
        VRAD_TRY(cudaMalloc(&parent_inner, sizeof(int32_t) * inner));
        VRAD_TRY(cudaMalloc(&parent_leaf, sizeof(int32_t) * n));
        VRAD_TRY(cudaMalloc(&node_box, sizeof(float) * 6 * inner));
        VRAD_TRY(cudaMalloc(&node_cost, sizeof(float) * inner));
        VRAD_TRY(cudaMalloc(&collapse, sizeof(int32_t) * inner));
        VRAD_TRY(cudaMalloc(&arrivals, sizeof(uint32_t) * inner));
        VRAD_TRY(cudaMemsetAsync(parent_inner, 0xff, sizeof(int32_t) * inner, stream));  // root: -1
        VRAD_TRY(cudaMemsetAsync(arrivals, 0, sizeof(uint32_t) * inner, stream));
        k_radix_tree<<<blocks(n - 1, 256), 256, 0, stream>>>(codes_sorted, n, child, range,
                                                             parent_inner, parent_leaf);
        VRAD_TRY(cudaGetLastError());
        k_refit<<<blocks(n, 256), 256, 0, stream>>>(tri_box, order_sorted, n, child, parent_inner,
                                                    parent_leaf, d_bounds, node_box, node_cost,
                                                    collapse, arrivals, leaf_box);
        VRAD_TRY(cudaGetLastError());
        // The root stays an inner node so traversal always starts at node 0.
        {
            int32_t root_cnt = 0;
            VRAD_TRY(cudaMemcpyAsync(&root_cnt, collapse, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
            VRAD_TRY(cudaStreamSynchronize(stream));
            root_cnt &= ~1;
            VRAD_TRY(cudaMemcpyAsync(collapse, &root_cnt, sizeof(int32_t), cudaMemcpyHostToDevice, stream));
        }
        k_emit<<<blocks(n - 1, 256), 256, 0, stream>>>(n, child, range, collapse, node_box, leaf_box,
                                                       sb.nodes);
        VRAD_TRY(cudaGetLastError());
        k_gather<<<blocks(n, 256), 256, 0, stream>>>(order_sorted, n, u0, u1, u2, sb.tri0, sb.tri1,
                                                     sb.tri2);
        VRAD_TRY(cudaGetLastError());
        k_count_leaves<<<blocks(n - 1, 256), 256, 0, stream>>>(n, child, range, collapse,
                                                               parent_inner, d_stats);
        VRAD_TRY(cudaGetLastError());
    }
    {
        int dstats[4];
        VRAD_TRY(cudaMemcpyAsync(dstats, d_stats, sizeof(int) * 4, cudaMemcpyDeviceToHost, stream));
        VRAD_TRY(cudaMemcpyAsync(bounds, d_bounds, sizeof(float) * 7, cudaMemcpyDeviceToHost, stream));
        VRAD_TRY(cudaEventRecord(ev1, stream));
        VRAD_TRY(cudaStreamSynchronize(stream));
        if (n > 1) {
            stats[0] = dstats[0];
            stats[1] = dstats[1];
            stats[2] = dstats[2];
        }
        stats[3] = dstats[3];
    }
    if (stats[3] != 0) {
        err = cudaErrorInvalidValue;  // a supplied form whose axes are not the drop axis's successors
        goto fail;
    }
    sb.ntris = n;
    // The tree's depth in inner nodes, from the emitted nodes: the deepest
    // stack a walk can build (each inner node pushes at most one entry).
    // Nodes sit at their inner-node numbers (0 .. n-2, the root at 0); the
    // collapsed subtrees' nodes stay in the array, unreachable.
    if (n > 1 && stats[0] > 0) {
        std::vector<float4> nodes((size_t)inner * 4);
        VRAD_TRY(cudaMemcpy(nodes.data(), sb.nodes, sizeof(float4) * nodes.size(), cudaMemcpyDeviceToHost));
        std::vector<std::pair<int32_t, int32_t>> todo = {{0, 1}};
        int32_t depth = 0;
        while (!todo.empty()) {
            const auto [node, d] = todo.back();
            todo.pop_back();
            depth = d > depth ? d : depth;
            if (d > kStackDepth) break;  // the walk's limit: deeper is an error either way
            int32_t refs[2];
            std::memcpy(refs, &nodes[(size_t)node * 4 + 3], sizeof refs);
            for (int32_t r : refs)
                if (r >= 0 && r < inner) todo.push_back({r, d + 1});
        }
        sb.depth = depth > kStackDepth ? kStackDepth : depth;  // deeper: walks report an overflow
    } else {
        sb.depth = n > 0 ? 1 : 0;
    }
    if (report) {
        report->max_depth = sb.depth > report->max_depth ? sb.depth : report->max_depth;
        const bool first = report->nodes == 0 && report->leaves == 0;
        report->nodes += stats[0];
        report->leaves += stats[1];
        report->max_leaf = stats[2] > report->max_leaf ? stats[2] : report->max_leaf;
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
    cudaFree(d_in);
    cudaFree(d_prep);
    cudaFree(d_orig);
    cudaFree(u0);
    cudaFree(u1);
    cudaFree(u2);
    cudaFree(tri_box);
    cudaFree(d_bounds);
    cudaFree(node_box);
    cudaFree(node_cost);
    cudaFree(leaf_box);
    cudaFree(codes);
    cudaFree(codes_sorted);
    cudaFree(order);
    cudaFree(order_sorted);
    cudaFree(parent_inner);
    cudaFree(parent_leaf);
    cudaFree(collapse);
    cudaFree(child);
    cudaFree(range);
    cudaFree(arrivals);
    cudaFree(d_stats);
    cudaFree(sort_tmp);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (err != cudaSuccess) sb.release();
    return err;
}

void BvhBuffers::release() {
    cudaFree(tri0);
    cudaFree(tri1);
    cudaFree(tri2);
    cudaFree(nodes);
    tri0 = tri1 = tri2 = nullptr;
    nodes = nullptr;
    ntris = 0;
    depth = 0;
}

void SceneBuffers::release() {
    opaque.release();
    sky.release();
    cudaFree(tri_id);
    tri_id = nullptr;
    ntris = 0;
}

}  // namespace vrad
