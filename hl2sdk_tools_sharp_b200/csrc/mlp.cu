// mlp.cu -- the learned warm start's network on the tensor cores: forward,
// backward and Adam, each a kernel of this library.
//
// Every matrix product is mma.sync.m16n8k16 with BF16 operands and FP32
// accumulators.  The forward keeps a warp's 16 rows in registers through
// all three layers: the accumulator fragments of one layer are, packed to
// BF16, the A fragments of the next (the m16n8 C layout of two adjacent
// n-tiles is the m16k16 A layout).  The backward does the same for the
// activation gradients; the weight gradients are P^T Q reductions over the
// rows, staged transposed in shared memory per 128-row tile, accumulated
// in registers across tiles and added once per CTA.  Master weights and
// Adam's moments are FP32; the BF16 operand copies are refreshed after
// every step.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "context.cuh"
#include "mlp.cuh"

namespace vrad {

namespace {

constexpr int kMlpWarps = 8;
constexpr int kMlpThreads = 32 * kMlpWarps;
constexpr int kTileRows = 16 * kMlpWarps;  // rows per CTA iteration

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ float bf_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf_hi(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }

__device__ __forceinline__ uint32_t ld32(const uint16_t *p) { return *reinterpret_cast<const uint32_t *>(p); }

// The forward's weights in shared memory.
struct FwdSmem {
    uint16_t w1t[kMlpHidden * kMlpIn];
    uint16_t w2t[kMlpHidden * kMlpHidden];
    uint16_t w3t[kMlpOutPad * kMlpHidden];
    float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpOutPad];
};

__device__ void load_fwd(FwdSmem &s, const vrad_mlp &m) {
    for (int i = threadIdx.x; i < kMlpHidden * kMlpIn / 2; i += blockDim.x)
        reinterpret_cast<uint32_t *>(s.w1t)[i] = reinterpret_cast<const uint32_t *>(m.w1t)[i];
    for (int i = threadIdx.x; i < kMlpHidden * kMlpHidden / 2; i += blockDim.x)
        reinterpret_cast<uint32_t *>(s.w2t)[i] = reinterpret_cast<const uint32_t *>(m.w2t)[i];
    for (int i = threadIdx.x; i < kMlpOutPad * kMlpHidden / 2; i += blockDim.x)
        reinterpret_cast<uint32_t *>(s.w3t)[i] = reinterpret_cast<const uint32_t *>(m.w3t)[i];
    for (int i = threadIdx.x; i < kMlpHidden; i += blockDim.x) {
        s.b1[i] = m.master[kOffB1 + i];
        s.b2[i] = m.master[kOffB2 + i];
    }
    if (threadIdx.x < kMlpOutPad) s.b3[threadIdx.x] = threadIdx.x < kMlpOut ? m.master[kOffB3 + threadIdx.x] : 0.0f;
}

// One hidden layer: acc[16 n-tiles] = bias + A (16 x 16*KT) B, B from
// output-major bf16 wt[n][k] with row stride K.
template <int KT>
__device__ __forceinline__ void layer(float acc[16][4], const uint32_t a[][4], const uint16_t *wt, const float *bias,
                                      int g, int t) {
    constexpr int K = 16 * KT;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const float b0 = bias[8 * j + 2 * t], b1 = bias[8 * j + 2 * t + 1];
        acc[j][0] = b0;
        acc[j][1] = b1;
        acc[j][2] = b0;
        acc[j][3] = b1;
#pragma unroll
        for (int kt = 0; kt < KT; kt++) {
            const uint16_t *row = wt + (8 * j + g) * K + 16 * kt + 2 * t;
            const uint32_t b[2] = {ld32(row), ld32(row + 8)};
            mma16816(acc[j], a[kt], b);
        }
    }
}

// ReLU, then the accumulators as the next layer's A fragments.
__device__ __forceinline__ void relu_pack(float acc[16][4], uint32_t a[8][4]) {
#pragma unroll
    for (int j = 0; j < 16; j++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[j][q] = acc[j][q] > 0.0f ? acc[j][q] : 0.0f;
#pragma unroll
    for (int kt = 0; kt < 8; kt++) {
        a[kt][0] = pack2(acc[2 * kt][0], acc[2 * kt][1]);
        a[kt][1] = pack2(acc[2 * kt][2], acc[2 * kt][3]);
        a[kt][2] = pack2(acc[2 * kt + 1][0], acc[2 * kt + 1][1]);
        a[kt][3] = pack2(acc[2 * kt + 1][2], acc[2 * kt + 1][3]);
    }
}

// Stores a warp's 16 x 128 bf16 activations from its A fragments.
__device__ __forceinline__ void store_act(uint16_t *dst, const uint32_t a[8][4], int64_t r0, int64_t n, int g, int t) {
    const int64_t ra = r0 + g, rb = r0 + g + 8;
#pragma unroll
    for (int kt = 0; kt < 8; kt++) {
        if (ra < n) {
            *reinterpret_cast<uint32_t *>(dst + ra * kMlpHidden + 16 * kt + 2 * t) = a[kt][0];
            *reinterpret_cast<uint32_t *>(dst + ra * kMlpHidden + 16 * kt + 8 + 2 * t) = a[kt][2];
        }
        if (rb < n) {
            *reinterpret_cast<uint32_t *>(dst + rb * kMlpHidden + 16 * kt + 2 * t) = a[kt][1];
            *reinterpret_cast<uint32_t *>(dst + rb * kMlpHidden + 16 * kt + 8 + 2 * t) = a[kt][3];
        }
    }
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_forward(vrad_mlp m, const uint16_t *__restrict__ x, int64_t n,
                                                             float *__restrict__ y, uint16_t *__restrict__ h1,
                                                             uint16_t *__restrict__ h2) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FwdSmem &s = *reinterpret_cast<FwdSmem *>(smem_raw);
    load_fwd(s, m);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int64_t tile = blockIdx.x; tile * kTileRows < n; tile += gridDim.x) {
        const int64_t r0 = tile * kTileRows + 16 * warp;
        if (r0 >= n) continue;
        const int64_t ra = r0 + g, rb = r0 + g + 8;
        uint32_t ax[2][4];
#pragma unroll
        for (int kt = 0; kt < 2; kt++) {
            ax[kt][0] = ra < n ? ld32(x + ra * kMlpIn + 16 * kt + 2 * t) : 0u;
            ax[kt][1] = rb < n ? ld32(x + rb * kMlpIn + 16 * kt + 2 * t) : 0u;
            ax[kt][2] = ra < n ? ld32(x + ra * kMlpIn + 16 * kt + 8 + 2 * t) : 0u;
            ax[kt][3] = rb < n ? ld32(x + rb * kMlpIn + 16 * kt + 8 + 2 * t) : 0u;
        }
        float acc[16][4];
        uint32_t ah[8][4];
        layer<2>(acc, ax, s.w1t, s.b1, g, t);
        relu_pack(acc, ah);
        if (h1) store_act(h1, ah, r0, n, g, t);
        layer<8>(acc, ah, s.w2t, s.b2, g, t);
        relu_pack(acc, ah);
        if (h2) store_act(h2, ah, r0, n, g, t);
        float out[4] = {s.b3[2 * t], s.b3[2 * t + 1], s.b3[2 * t], s.b3[2 * t + 1]};
#pragma unroll
        for (int kt = 0; kt < 8; kt++) {
            const uint16_t *row = s.w3t + g * kMlpHidden + 16 * kt + 2 * t;
            const uint32_t b[2] = {ld32(row), ld32(row + 8)};
            mma16816(out, ah[kt], b);
        }
        // Output columns 2t, 2t + 1: the first three are the network's.
        for (int q = 0; q < 2; q++) {
            const int c = 2 * t + q;
            if (c >= kMlpOut) continue;
            if (ra < n) y[ra * kMlpOut + c] = out[q];
            if (rb < n) y[rb * kMlpOut + c] = out[2 + q];
        }
    }
}

// The activation gradients of the mean squared error over n rows and three
// outputs: dy = 2 (y - target) / 3n, dz2 = (dy W3^T) * [h2 > 0],
// dz1 = (dz2 W2^T) * [h1 > 0], each stored as the bf16 the weight
// gradients read; the loss summed into *loss.
struct BwdSmem {
    uint16_t w2[kMlpHidden * kMlpHidden];  // input-major
    uint16_t w3[kMlpHidden * kMlpOutPad];  // input-major
};

__global__ void __launch_bounds__(kMlpThreads) k_mlp_backward(vrad_mlp m, const float *__restrict__ target, int64_t n,
                                                              float inv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BwdSmem &s = *reinterpret_cast<BwdSmem *>(smem_raw);
    for (int i = threadIdx.x; i < kMlpHidden * kMlpHidden / 2; i += blockDim.x)
        reinterpret_cast<uint32_t *>(s.w2)[i] = reinterpret_cast<const uint32_t *>(m.w2)[i];
    for (int i = threadIdx.x; i < kMlpHidden * kMlpOutPad / 2; i += blockDim.x)
        reinterpret_cast<uint32_t *>(s.w3)[i] = reinterpret_cast<const uint32_t *>(m.w3)[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float loss = 0.0f;
    for (int64_t tile = blockIdx.x; tile * kTileRows < n; tile += gridDim.x) {
        const int64_t r0 = tile * kTileRows + 16 * warp;
        if (r0 >= n) continue;
        const int64_t ra = r0 + g, rb = r0 + g + 8;
        // dy for columns 2t, 2t + 1 of rows ra, rb.
        float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int q = 0; q < 2; q++) {
            const int c = 2 * t + q;
            if (c >= kMlpOut) continue;
            if (ra < n) {
                const float e = m.y[ra * kMlpOut + c] - target[ra * kMlpOut + c];
                loss += e * e;
                d[q] = 2.0f * e * inv;
            }
            if (rb < n) {
                const float e = m.y[rb * kMlpOut + c] - target[rb * kMlpOut + c];
                loss += e * e;
                d[2 + q] = 2.0f * e * inv;
            }
        }
        const uint32_t dya = pack2(d[0], d[1]), dyb = pack2(d[2], d[3]);
        if (ra < n) *reinterpret_cast<uint32_t *>(m.dy + ra * kMlpOutPad + 2 * t) = dya;
        if (rb < n) *reinterpret_cast<uint32_t *>(m.dy + rb * kMlpOutPad + 2 * t) = dyb;
        // dh2 = dy (16 x 8, k padded to 16 with zeros) W3^T.
        const uint32_t ady[4] = {dya, dyb, 0u, 0u};
        float acc[16][4];
        uint32_t az[8][4];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
            const uint32_t b[2] = {ld32(s.w3 + (8 * j + g) * kMlpOutPad + 2 * t), 0u};
            mma16816(acc[j], ady, b);
        }
        // Mask by h2 > 0, pack, store dz2.
        auto mask_pack = [&](const uint16_t *h, uint16_t *dz) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const uint32_t ha = ra < n ? ld32(h + ra * kMlpHidden + 8 * j + 2 * t) : 0u;
                const uint32_t hb = rb < n ? ld32(h + rb * kMlpHidden + 8 * j + 2 * t) : 0u;
                if (!(bf_lo(ha) > 0.0f)) acc[j][0] = 0.0f;
                if (!(bf_hi(ha) > 0.0f)) acc[j][1] = 0.0f;
                if (!(bf_lo(hb) > 0.0f)) acc[j][2] = 0.0f;
                if (!(bf_hi(hb) > 0.0f)) acc[j][3] = 0.0f;
            }
#pragma unroll
            for (int kt = 0; kt < 8; kt++) {
                az[kt][0] = pack2(acc[2 * kt][0], acc[2 * kt][1]);
                az[kt][1] = pack2(acc[2 * kt][2], acc[2 * kt][3]);
                az[kt][2] = pack2(acc[2 * kt + 1][0], acc[2 * kt + 1][1]);
                az[kt][3] = pack2(acc[2 * kt + 1][2], acc[2 * kt + 1][3]);
            }
            store_act(dz, az, r0, n, g, t);
        };
        mask_pack(m.h2, m.dz2);
        // dh1 = dz2 W2^T.
#pragma unroll
        for (int j = 0; j < 16; j++) {
            acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
            for (int kt = 0; kt < 8; kt++) {
                const uint16_t *row = s.w2 + (8 * j + g) * kMlpHidden + 16 * kt + 2 * t;
                const uint32_t b[2] = {ld32(row), ld32(row + 8)};
                mma16816(acc[j], az[kt], b);
            }
        }
        mask_pack(m.h1, m.dz1);
    }
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) atomicAdd(m.loss, loss * inv);
}

// grad[M][N] += P^T Q over n rows (P [n][M], Q [n][N], bf16), and
// bias[N] += the column sums of Q, for one weight matrix.
template <int M, int N>
__global__ void __launch_bounds__(kMlpThreads) k_mlp_wgrad(const uint16_t *__restrict__ p, const uint16_t *__restrict__ q,
                                                           int64_t n, int qstride, int ncols, float *__restrict__ grad,
                                                           int gstride, float *__restrict__ bias) {
    constexpr int R = kTileRows;       // rows per tile (the k extent)
    constexpr int RS = R + 8;          // padded row of the transposed tiles
    constexpr int TILES = (M / 16) * (N / 8);
    constexpr int PER = (TILES + kMlpWarps - 1) / kMlpWarps;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint16_t *pt = reinterpret_cast<uint16_t *>(smem_raw);  // [M][RS]
    uint16_t *qt = pt + M * RS;                             // [N][RS]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[PER][4];
#pragma unroll
    for (int i = 0; i < PER; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0f;
    float colsum = 0.0f;  // thread c < N: column c's sum
    for (int64_t tile = blockIdx.x; tile * R < n; tile += gridDim.x) {
        const int64_t r0 = tile * R;
        __syncthreads();
        for (int i = threadIdx.x; i < R * M; i += blockDim.x) {
            const int r = i / M, c = i % M;
            pt[c * RS + r] = r0 + r < n ? p[(r0 + r) * M + c] : (uint16_t)0;
        }
        for (int i = threadIdx.x; i < R * N; i += blockDim.x) {
            const int r = i / N, c = i % N;
            qt[c * RS + r] = (r0 + r < n && c < ncols) ? q[(r0 + r) * qstride + c] : (uint16_t)0;
        }
        __syncthreads();
        if (bias && threadIdx.x < N)
            for (int r = 0; r < R; r++) colsum += __uint_as_float((uint32_t)qt[threadIdx.x * RS + r] << 16);
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int tileid = warp + kMlpWarps * i;
            if (tileid >= TILES) break;
            const int mt = tileid / (N / 8), nt = tileid % (N / 8);
#pragma unroll
            for (int kt = 0; kt < R / 16; kt++) {
                const uint16_t *a0 = pt + (16 * mt + g) * RS + 16 * kt + 2 * t;
                const uint16_t *a1 = pt + (16 * mt + g + 8) * RS + 16 * kt + 2 * t;
                const uint32_t a[4] = {ld32(a0), ld32(a1), ld32(a0 + 8), ld32(a1 + 8)};
                const uint16_t *bq = qt + (8 * nt + g) * RS + 16 * kt + 2 * t;
                const uint32_t b[2] = {ld32(bq), ld32(bq + 8)};
                mma16816(acc[i], a, b);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < PER; i++) {
        const int tileid = warp + kMlpWarps * i;
        if (tileid >= TILES) break;
        const int mt = tileid / (N / 8), nt = tileid % (N / 8);
        const int m0 = 16 * mt + g, n0 = 8 * nt + 2 * t;
        if (n0 < ncols) {
            atomicAdd(&grad[m0 * gstride + n0], acc[i][0]);
            atomicAdd(&grad[(m0 + 8) * gstride + n0], acc[i][2]);
        }
        if (n0 + 1 < ncols) {
            atomicAdd(&grad[m0 * gstride + n0 + 1], acc[i][1]);
            atomicAdd(&grad[(m0 + 8) * gstride + n0 + 1], acc[i][3]);
        }
    }
    if (bias && threadIdx.x < ncols) atomicAdd(&bias[threadIdx.x], colsum);
}

// The BF16 operand copies of the master weights.
__global__ void k_mlp_refresh(vrad_mlp m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kW1) {
        const int k = i / kMlpHidden, c = i % kMlpHidden;
        m.w1t[c * kMlpIn + k] = __bfloat16_as_ushort(__float2bfloat16_rn(m.master[i]));
    }
    if (i < kW2) {
        const int k = i / kMlpHidden, c = i % kMlpHidden;
        const uint16_t v = __bfloat16_as_ushort(__float2bfloat16_rn(m.master[kOffW2 + i]));
        m.w2t[c * kMlpHidden + k] = v;
        m.w2[k * kMlpHidden + c] = v;
    }
    if (i < kMlpHidden * kMlpOutPad) {
        const int k = i / kMlpOutPad, c = i % kMlpOutPad;
        const uint16_t v = c < kMlpOut ? __bfloat16_as_ushort(__float2bfloat16_rn(m.master[kOffW3 + k * kMlpOut + c]))
                                       : (uint16_t)0;
        m.w3t[c * kMlpHidden + k] = v;
        m.w3[k * kMlpOutPad + c] = v;
    }
}

// Adam (beta1 0.9, beta2 0.999, epsilon 1e-8) on the master weights.
__global__ void k_mlp_adam(vrad_mlp m, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMlpParams) return;
    const float gr = m.grad[i];
    const float mm = 0.9f * m.adam_m[i] + 0.1f * gr;
    const float vv = 0.999f * m.adam_v[i] + 0.001f * gr * gr;
    m.adam_m[i] = mm;
    m.adam_v[i] = vv;
    m.master[i] -= lr * (mm / c1) / (sqrtf(vv / c2) + 1e-8f);
}

unsigned blocks_for(int64_t n) {
    const int64_t tiles = (n + kTileRows - 1) / kTileRows;
    return (unsigned)(tiles < 4 * 148 ? (tiles > 0 ? tiles : 1) : 4 * 148);
}

cudaError_t grow(vrad_mlp &m, int64_t n) {
    if (n <= m.scratch_rows) return cudaSuccess;
    for (void *p : {(void *)m.h1, (void *)m.h2, (void *)m.dz1, (void *)m.dz2, (void *)m.dy, (void *)m.y}) cudaFree(p);
    m.h1 = m.h2 = m.dz1 = m.dz2 = m.dy = nullptr;
    m.y = nullptr;
    m.scratch_rows = 0;
    cudaError_t e = cudaMalloc(&m.h1, sizeof(uint16_t) * kMlpHidden * n);
    if (e == cudaSuccess) e = cudaMalloc(&m.h2, sizeof(uint16_t) * kMlpHidden * n);
    if (e == cudaSuccess) e = cudaMalloc(&m.dz1, sizeof(uint16_t) * kMlpHidden * n);
    if (e == cudaSuccess) e = cudaMalloc(&m.dz2, sizeof(uint16_t) * kMlpHidden * n);
    if (e == cudaSuccess) e = cudaMalloc(&m.dy, sizeof(uint16_t) * kMlpOutPad * n);
    if (e == cudaSuccess) e = cudaMalloc(&m.y, sizeof(float) * kMlpOut * n);
    if (e == cudaSuccess) m.scratch_rows = n;
    return e;
}

// The MSE gradient into m.grad (and the loss into m.loss), on `s`.
cudaError_t gradient(vrad_mlp &m, const uint16_t *x, const float *target, int64_t n, cudaStream_t s) {
    cudaError_t e = grow(m, n);
    if (e == cudaSuccess) e = cudaMemsetAsync(m.grad, 0, sizeof(float) * kMlpParams, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(m.loss, 0, sizeof(float), s);
    if (e != cudaSuccess || n == 0) return e;
    const unsigned nb = blocks_for(n);
    k_mlp_forward<<<nb, kMlpThreads, sizeof(FwdSmem), s>>>(m, x, n, m.y, m.h1, m.h2);
    k_mlp_backward<<<nb, kMlpThreads, sizeof(BwdSmem), s>>>(m, target, n, 1.0f / (3.0f * (float)n));
    constexpr int RS = kTileRows + 8;
    // dW3 = h2^T dy (+ db3), dW2 = h1^T dz2 (+ db2), dW1 = x^T dz1 (+ db1).
    k_mlp_wgrad<kMlpHidden, kMlpOutPad><<<nb, kMlpThreads, sizeof(uint16_t) * RS * (kMlpHidden + kMlpOutPad), s>>>(
        m.h2, m.dy, n, kMlpOutPad, kMlpOut, m.grad + kOffW3, kMlpOut, m.grad + kOffB3);
    k_mlp_wgrad<kMlpHidden, kMlpHidden><<<nb, kMlpThreads, sizeof(uint16_t) * RS * (2 * kMlpHidden), s>>>(
        m.h1, m.dz2, n, kMlpHidden, kMlpHidden, m.grad + kOffW2, kMlpHidden, m.grad + kOffB2);
    k_mlp_wgrad<kMlpIn, kMlpHidden><<<nb, kMlpThreads, sizeof(uint16_t) * RS * (kMlpIn + kMlpHidden), s>>>(
        x, m.dz1, n, kMlpHidden, kMlpHidden, m.grad, kMlpHidden, m.grad + kOffB1);
    return cudaGetLastError();
}

bool smem_ready[64];
std::mutex smem_mu;

cudaError_t allow_smem(int device) {
    std::lock_guard<std::mutex> g(smem_mu);
    if (device >= 0 && device < 64 && smem_ready[device]) return cudaSuccess;
    constexpr int RS = kTileRows + 8;
    cudaError_t e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FwdSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(BwdSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_wgrad<kMlpHidden, kMlpHidden>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(uint16_t) * RS * 2 * kMlpHidden));
    if (e == cudaSuccess && device >= 0 && device < 64) smem_ready[device] = true;
    return e;
}

}  // namespace

cudaError_t mlp_forward(const vrad_mlp &m, const uint16_t *x, int64_t n, float *y, cudaStream_t s) {
    return mlp_forward_tc(m, x, n, y, s);
}

}  // namespace vrad

namespace {

void release_mlp(vrad_mlp *m) {
    for (void *p : {(void *)m->master, (void *)m->adam_m, (void *)m->adam_v, (void *)m->grad, (void *)m->w1t,
                    (void *)m->w2t, (void *)m->w3t, (void *)m->w2, (void *)m->w3, (void *)m->loss, (void *)m->flags,
                    (void *)m->h1,
                    (void *)m->h2, (void *)m->dz1, (void *)m->dz2, (void *)m->dy, (void *)m->y})
        cudaFree(p);
    delete m;
}

cudaError_t refresh(vrad_mlp *m, cudaStream_t s) {
    vrad::k_mlp_refresh<<<(vrad::kW2 + 255) / 256, 256, 0, s>>>(*m);
    return cudaGetLastError();
}

}  // namespace

extern "C" int32_t vrad_mlp_create(vrad_ctx *ctx, uint64_t seed, vrad_mlp **out) {
    using namespace vrad;
    if (!ctx || !out) return vrad_fail(ctx, VRAD_ERR_ARG, "null argument");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(ctx->device);
    vrad_mlp *m = new vrad_mlp();
    m->device = ctx->device;
    for (float **p : {&m->master, &m->adam_m, &m->adam_v, &m->grad})
        if (e == cudaSuccess) e = cudaMalloc(p, sizeof(float) * kMlpParams);
    for (uint16_t **p : {&m->w1t, &m->w2t, &m->w3t, &m->w2, &m->w3})
        if (e == cudaSuccess) e = cudaMalloc(p, sizeof(uint16_t) * kW2);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->flags, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(m->flags, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = allow_smem(ctx->device);
    // He initialisation from a seeded generator; biases zero.
    std::vector<float> w((size_t)kMlpParams, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int count) {
        std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / fan_in));
        for (int i = 0; i < count; i++) w[(size_t)(off + i)] = (float)nd(rng);
    };
    fill(0, kMlpIn, kW1);
    fill(kOffW2, kMlpHidden, kW2);
    fill(kOffW3, kMlpHidden, kW3);
    if (e == cudaSuccess) e = cudaMemcpy(m->master, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->adam_m, 0, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMemset(m->adam_v, 0, sizeof(float) * kMlpParams);
    if (e == cudaSuccess) e = cudaMemset(m->w3t, 0, sizeof(uint16_t) * kW2);
    if (e == cudaSuccess) e = refresh(m, nullptr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        release_mlp(m);
        return vrad_cuda_fail(ctx, e, "network creation");
    }
    *out = m;
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_destroy(vrad_mlp *m) {
    if (!m) return VRAD_OK;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    release_mlp(m);
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_params(vrad_mlp *m, float *get, const float *set) {
    if (!m) return vrad_fail(nullptr, VRAD_ERR_ARG, "null network");
    cudaError_t e = cudaSetDevice(m->device);
    if (e == cudaSuccess && set) e = cudaMemcpy(m->master, set, sizeof(float) * vrad::kMlpParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && set) e = refresh(m, nullptr);
    if (e == cudaSuccess && get) e = cudaMemcpy(get, m->master, sizeof(float) * vrad::kMlpParams, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return vrad_cuda_fail(nullptr, e, "network parameters");
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_forward_device(vrad_mlp *m, const uint16_t *x, int64_t n, float *y, void *stream) {
    if (!m || n < 0 || (n && (!x || !y))) return vrad_fail(nullptr, VRAD_ERR_ARG, "invalid network forward");
    if (((uintptr_t)x & 3) || ((uintptr_t)y & 3)) return vrad_fail(nullptr, VRAD_ERR_ARG, "x and y must be 4-byte aligned");
    cudaError_t e = cudaSetDevice(m->device);
    if (e == cudaSuccess) e = vrad::mlp_forward(*m, x, n, y, (cudaStream_t)stream);
    if (e != cudaSuccess) return vrad_cuda_fail(nullptr, e, "network forward");
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_gradient_device(vrad_mlp *m, const uint16_t *x, const float *target, int64_t n,
                                            float *grad, float *loss, void *stream) {
    if (!m || n < 0 || (n && (!x || !target))) return vrad_fail(nullptr, VRAD_ERR_ARG, "invalid network gradient");
    cudaError_t e = cudaSetDevice(m->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (e == cudaSuccess) e = vrad::gradient(*m, x, target, n, s);
    if (e == cudaSuccess && grad)
        e = cudaMemcpyAsync(grad, m->grad, sizeof(float) * vrad::kMlpParams, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return vrad_cuda_fail(nullptr, e, "network gradient");
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_train_step_device(vrad_mlp *m, const uint16_t *x, const float *target, int64_t n, float lr,
                                              void *stream) {
    if (!m || n <= 0 || !x || !target || !(lr > 0.0f)) return vrad_fail(nullptr, VRAD_ERR_ARG, "invalid training step");
    cudaError_t e = cudaSetDevice(m->device);
    cudaStream_t s = (cudaStream_t)stream;
    if (e == cudaSuccess) e = vrad::gradient(*m, x, target, n, s);
    if (e == cudaSuccess) {
        m->step++;
        const float c1 = 1.0f - (float)std::pow(0.9, (double)m->step), c2 = 1.0f - (float)std::pow(0.999, (double)m->step);
        vrad::k_mlp_adam<<<(vrad::kMlpParams + 255) / 256, 256, 0, s>>>(*m, lr, c1, c2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = refresh(m, s);
    if (e != cudaSuccess) return vrad_cuda_fail(nullptr, e, "training step");
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_loss(vrad_mlp *m, float *loss) {
    if (!m || !loss) return vrad_fail(nullptr, VRAD_ERR_ARG, "null argument");
    cudaError_t e = cudaSetDevice(m->device);
    if (e == cudaSuccess) e = cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return vrad_cuda_fail(nullptr, e, "network loss");
    return VRAD_OK;
}

extern "C" int32_t vrad_mlp_status(vrad_mlp *m) {
    if (!m) return vrad_fail(nullptr, VRAD_ERR_ARG, "null network");
    uint32_t f = 0;
    cudaError_t e = cudaSetDevice(m->device);
    if (e == cudaSuccess) e = cudaMemcpy(&f, m->flags, sizeof f, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && f) e = cudaMemset(m->flags, 0, sizeof f);
    if (e != cudaSuccess) return vrad_cuda_fail(nullptr, e, "network status");
    if (f) return vrad_fail(nullptr, VRAD_ERR_TIMEOUT, "a network forward's tensor-core wait ran out");
    return VRAD_OK;
}
