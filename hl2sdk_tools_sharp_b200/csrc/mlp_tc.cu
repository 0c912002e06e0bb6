// mlp_tc.cu -- the learned warm start's forward on Blackwell's fifth-
// generation tensor cores: tcgen05.mma with the accumulators in TMEM.
//
// The network is 32 -> 128 -> 128 -> 3 (ReLU, BF16 weights and activations,
// FP32 accumulation; mlp.cuh).  One CTA of 8 warps works on 128 rows at a
// time and keeps the whole network in shared memory:
//   w1 (N 128, K 32), w2 (N 128, K 128), w3 (N 16, K 128; rows 3..15 zero)
//   as the MMAs' B operands and the row tile's x (K 32) and hidden layer h
//   (K 128) as their A operands, all in the canonical K-major layout
//   without swizzle: 8-row x 16-byte core matrices, each 128 contiguous
//   bytes, core (row group g, K chunk k) at (k x row groups + g) x 128 B;
// and 128 TMEM columns (128 lanes x 128 FP32) that each layer's
// accumulator reuses.  Per tile:
//   x -> shared memory (each thread 32 bytes of a row, loaded from global
//     memory while the previous tile ran)
//   layer 1: 2 x tcgen05.mma M128 N128 K16 -> TMEM, commit -> mbarrier
//   epilogue: tcgen05.ld (warp w reads lanes 32 (w % 4) .., columns
//     64 (w / 4) ..), + bias, ReLU, BF16 -> h in shared memory
//   layer 2: 8 x M128 N128 K16 over h; the same epilogue into h
//   layer 3: 8 x M128 N16 K16 over h; warps 0-3 add the bias and write
//     the three outputs.
// Thread 0 issues every MMA and the commit; everyone waits on the
// mbarrier, each wait bounded by a clock limit after which the kernel
// records the fault in the network's flags and every thread of the CTA
// leaves together (the TMEM is freed on the way out).  Two CTAs share an
// SM (87 KB of shared memory, 128 TMEM columns each), so one CTA's
// epilogue overlaps the other's MMAs.
//
// The sums are the mma.sync forward's (mlp.cu) up to FP32 rounding: the
// bias is added after the products here rather than before.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <mutex>

#include "mlp.cuh"

namespace vrad {
namespace {

constexpr int kTcWarps = 8;
constexpr int kTcThreads = 32 * kTcWarps;
constexpr int kTcRows = 128;
constexpr uint32_t kTmemCols = 128;
constexpr int kN3 = 16;                                 // layer 3's N, padded
constexpr long long kWaitCycles = 2000000000LL;         // about a second at the B200's clocks
constexpr uint32_t kFlagTimeout = 1;

struct __align__(1024) TcSmem {
    uint16_t w1[kMlpHidden * kMlpIn];
    uint16_t w2[kMlpHidden * kMlpHidden];
    uint16_t w3[kN3 * kMlpHidden];
    uint16_t x[kTcRows * kMlpIn];
    uint16_t h[kTcRows * kMlpHidden];
    float b1[kMlpHidden], b2[kMlpHidden], b3[kN3];
    unsigned long long bar;
    uint32_t tmem;
    int abort;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// The element offset of (row r, column c) in a canonical K-major
// no-swizzle operand with `groups` row groups of 8.
__device__ __forceinline__ int canon(int r, int c, int groups) {
    return ((c >> 3) * groups + (r >> 3)) * 64 + (r & 7) * 8 + (c & 7);
}

// Shared memory descriptor: start, leading (K) and stride (row group)
// byte offsets in 16-byte units, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// both K-major, M 128.
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, bool acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"((uint32_t)acc)
        : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for phase `parity` of the mbarrier, at most kWaitCycles.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kWaitCycles) return false;
    }
}

// 32 consecutive FP32 columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld4(uint32_t addr, float v[4]) {
    uint32_t r[4];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
#pragma unroll
    for (int i = 0; i < 4; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// Bias, ReLU and BF16 of this thread's 64 accumulator columns of row r into h.
// Both 32-column loads are in flight before the one wait.
__device__ __forceinline__ void hidden_epilogue(TcSmem &s, uint32_t taddr, const float *bias, int r, int c0) {
    float v[64];
    tmem_ld32(taddr + (uint32_t)c0, v);
    tmem_ld32(taddr + (uint32_t)(c0 + 32), v + 32);
    tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const int c = c0 + 8 * q;
        uint4 w;
        uint32_t *pw = reinterpret_cast<uint32_t *>(&w);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const float a = fmaxf(__fadd_rn(v[8 * q + 2 * e], bias[c + 2 * e]), 0.0f);
            const float b = fmaxf(__fadd_rn(v[8 * q + 2 * e + 1], bias[c + 2 * e + 1]), 0.0f);
            pw[e] = pack2(a, b);
        }
        *reinterpret_cast<uint4 *>(s.h + canon(r, c, kTcRows / 8)) = w;
    }
}

__global__ void __launch_bounds__(kTcThreads) k_mlp_forward_tc(vrad_mlp m, const uint16_t *__restrict__ x, int64_t n,
                                                               float *__restrict__ y) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TcSmem &s = *reinterpret_cast<TcSmem *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // The network into shared memory, as B operands.
    for (int i = tid; i < kMlpHidden * kMlpIn / 8; i += kTcThreads) {
        const int nn = i / (kMlpIn / 8), kc = i % (kMlpIn / 8);
        *reinterpret_cast<uint4 *>(s.w1 + canon(nn, 8 * kc, kMlpHidden / 8)) =
            *reinterpret_cast<const uint4 *>(m.w1t + nn * kMlpIn + 8 * kc);
    }
    for (int i = tid; i < kMlpHidden * kMlpHidden / 8; i += kTcThreads) {
        const int nn = i / (kMlpHidden / 8), kc = i % (kMlpHidden / 8);
        *reinterpret_cast<uint4 *>(s.w2 + canon(nn, 8 * kc, kMlpHidden / 8)) =
            *reinterpret_cast<const uint4 *>(m.w2t + nn * kMlpHidden + 8 * kc);
    }
    for (int i = tid; i < kN3 * kMlpHidden / 8; i += kTcThreads) {
        const int nn = i / (kMlpHidden / 8), kc = i % (kMlpHidden / 8);
        uint4 w = make_uint4(0, 0, 0, 0);
        if (nn < kMlpOutPad) w = *reinterpret_cast<const uint4 *>(m.w3t + nn * kMlpHidden + 8 * kc);
        *reinterpret_cast<uint4 *>(s.w3 + canon(nn, 8 * kc, kN3 / 8)) = w;
    }
    for (int i = tid; i < kMlpHidden; i += kTcThreads) {
        s.b1[i] = m.master[kOffB1 + i];
        s.b2[i] = m.master[kOffB2 + i];
    }
    if (tid < kN3) s.b3[tid] = tid < kMlpOut ? m.master[kOffB3 + tid] : 0.0f;
    const uint32_t bar = smem_u32(&s.bar);
    if (tid == 0) {
        s.abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = s.tmem;
    // This warp's TMEM lanes and accumulator columns.
    const int row = 32 * (warp & 3) + lane;
    const int c0 = 64 * (warp >> 2);
    const uint32_t taddr = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const uint32_t ax = smem_u32(s.x), ah = smem_u32(s.h), bw1 = smem_u32(s.w1), bw2 = smem_u32(s.w2),
                   bw3 = smem_u32(s.w3);
    constexpr uint32_t kLboWide = 16 * 128, kLboW3 = 2 * 128, kSbo = 128;
    const bool x16 = ((uintptr_t)x & 15) == 0;
    uint32_t parity = 0;
    bool ok = true;

    // Waits for the MMAs just committed; every thread of the CTA returns
    // the same answer.
    auto wait_all = [&]() -> bool {
        const bool mine = wait_bar(bar, parity);
        parity ^= 1;
        if (!mine) atomicOr(&s.abort, 1);
        __syncthreads();
        fence_after();
        return s.abort == 0;
    };

    // x: thread t holds half of row t / 2 (two 16-byte chunks) of a tile;
    // the next tile's are loaded while this tile's layers run.
    const int xr_row = tid >> 1, xr_kc = 2 * (tid & 1);
    uint4 xr[2];
    auto load_x = [&](int64_t tile) {
        const int64_t gr = tile * kTcRows + xr_row;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            xr[q] = make_uint4(0, 0, 0, 0);
            if (gr < n) {
                const uint16_t *src = x + gr * kMlpIn + 8 * (xr_kc + q);
                if (x16) {
                    xr[q] = *reinterpret_cast<const uint4 *>(src);
                } else {
                    const uint32_t *s32 = reinterpret_cast<const uint32_t *>(src);
                    xr[q] = make_uint4(s32[0], s32[1], s32[2], s32[3]);
                }
            }
        }
    };
    load_x(blockIdx.x);

    for (int64_t tile = blockIdx.x; ok && tile * kTcRows < n; tile += gridDim.x) {
        const int64_t r0 = tile * kTcRows;
#pragma unroll
        for (int q = 0; q < 2; q++) *reinterpret_cast<uint4 *>(s.x + canon(xr_row, 8 * (xr_kc + q), kTcRows / 8)) = xr[q];
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int k = 0; k < kMlpIn / 16; k++)
                mma(tmem, sdesc(ax + 2 * k * kLboWide, kLboWide, kSbo), sdesc(bw1 + 2 * k * kLboWide, kLboWide, kSbo),
                    idesc(kMlpHidden), k > 0);
            commit(bar);
        }
        load_x(tile + gridDim.x);
        if (!(ok = wait_all())) break;
        hidden_epilogue(s, taddr, s.b1, row, c0);
        fence_before();
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int k = 0; k < kMlpHidden / 16; k++)
                mma(tmem, sdesc(ah + 2 * k * kLboWide, kLboWide, kSbo), sdesc(bw2 + 2 * k * kLboWide, kLboWide, kSbo),
                    idesc(kMlpHidden), k > 0);
            commit(bar);
        }
        if (!(ok = wait_all())) break;
        hidden_epilogue(s, taddr, s.b2, row, c0);
        fence_before();
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            fence_after();
#pragma unroll
            for (int k = 0; k < kMlpHidden / 16; k++)
                mma(tmem, sdesc(ah + 2 * k * kLboWide, kLboWide, kSbo), sdesc(bw3 + 2 * k * kLboW3, kLboW3, kSbo),
                    idesc(kN3), k > 0);
            commit(bar);
        }
        if (!(ok = wait_all())) break;
        if (warp < 4) {
            float v[4];
            tmem_ld4(taddr, v);
            tmem_wait_ld();
            const int64_t gr = r0 + row;
            if (gr < n) {
#pragma unroll
                for (int c = 0; c < kMlpOut; c++) y[gr * kMlpOut + c] = __fadd_rn(v[c], s.b3[c]);
            }
        }
        fence_before();
        __syncthreads();
        fence_after();
    }
    // After a timeout: record it, and leave with no MMA in flight (the last
    // commit's phase waited for once more, bounded again), then free the
    // TMEM.
    if (!ok && tid == 0) {
        atomicOr(m.flags, kFlagTimeout);
        wait_bar(bar, parity ^ 1);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

std::mutex tc_mu;
bool tc_ready[64];
int tc_sms[64];

}  // namespace

cudaError_t mlp_forward_tc(const vrad_mlp &m, const uint16_t *x, int64_t n, float *y, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const int dev = m.device;
    int sms = 148;
    {
        std::lock_guard<std::mutex> g(tc_mu);
        if (dev >= 0 && dev < 64 && tc_ready[dev]) {
            sms = tc_sms[dev];
        } else {
            cudaError_t e = cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)sizeof(TcSmem));
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) {
                tc_sms[dev] = sms;
                tc_ready[dev] = true;
            }
        }
    }
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    const int64_t grid = tiles < 2LL * sms ? tiles : 2LL * sms;
    k_mlp_forward_tc<<<(unsigned)grid, kTcThreads, sizeof(TcSmem), s>>>(m, x, n, y);
    return cudaGetLastError();
}

}  // namespace vrad
