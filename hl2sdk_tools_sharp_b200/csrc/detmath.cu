// detmath.cu -- vrad_detmath: the device's correctly rounded arcsine and
// power (detmath.cuh) over a batch, the functions the transfer build and
// the spotlight falloff call, so they can be checked against known answers.

#include <cuda_runtime.h>

#include <mutex>

#include "context.cuh"
#include "detmath.cuh"

namespace {

__global__ void k_detmath(int fn, const float *__restrict__ a, const float *__restrict__ b, float *__restrict__ out,
                          int64_t n, unsigned long long *open) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = fn == VRAD_DETMATH_ASIN ? vrad::asin_cr(a[i], open) : vrad::pow_cr(a[i], b[i], open);
}

}  // namespace

extern "C" int32_t vrad_detmath(vrad_ctx *ctx, int32_t fn, const float *a, const float *b, float *out, int64_t n,
                                int64_t *open) {
    if (!ctx) return vrad_fail(nullptr, VRAD_ERR_ARG, "null context");
    if ((fn != VRAD_DETMATH_ASIN && fn != VRAD_DETMATH_POW) || n < 0 || (n && (!a || !out)) ||
        (fn == VRAD_DETMATH_POW && n && !b))
        return vrad_fail(ctx, VRAD_ERR_ARG, "invalid detmath call");
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    float *d = nullptr;
    unsigned long long *d_open = nullptr, h_open = 0;
    const size_t bytes = sizeof(float) * (size_t)(n ? n : 1);
    if (e == cudaSuccess) e = cudaMalloc(&d, 3 * bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d_open, sizeof h_open);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_open, 0, sizeof h_open, ctx->stream);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(d, a, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && n && b)
        e = cudaMemcpyAsync(d + n, b, sizeof(float) * n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && n)
        k_detmath<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(fn, d, d + n, d + 2 * n, n, d_open);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(out, d + 2 * n, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_open, d_open, sizeof h_open, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    cudaFree(d_open);
    if (e != cudaSuccess) return vrad_cuda_fail(ctx, e, "detmath");
    if (open) *open = (int64_t)h_open;
    return VRAD_OK;
}
