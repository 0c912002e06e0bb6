// mlp.cuh -- the learned warm start's network: 32 -> 128 -> 128 -> 3 with
// ReLU, BF16 weights and activations, FP32 accumulation (mlp.cu: training
// on mma.sync; mlp_tc.cu: the forward on tcgen05 with TMEM accumulators).
//
// Device layout of one network (struct vrad_mlp):
//   master  float  FP32 parameters, the order of kMlpParams (w1 [32][128],
//                  b1 [128], w2 [128][128], b2 [128], w3 [128][3], b3 [3]);
//                  w[k][n] maps input k to output n
//   adam_m, adam_v float  Adam's moments, same order
//   grad   float   the gradient of the last step, same order
//   w1t [128][32], w2t [128][128], w3t [8][128] bf16: the forward's B
//                  operands, output-major (rows 3..7 of w3t zero)
//   w2 [128][128], w3 [128][8] bf16: the backward's B operands, input-major
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace vrad {

constexpr int kMlpIn = 32;
constexpr int kMlpHidden = 128;
constexpr int kMlpOut = 3;
constexpr int kMlpOutPad = 8;
constexpr int kW1 = kMlpIn * kMlpHidden;
constexpr int kW2 = kMlpHidden * kMlpHidden;
constexpr int kW3 = kMlpHidden * kMlpOut;
constexpr int kOffB1 = kW1;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kW2;
constexpr int kOffW3 = kOffB2 + kMlpHidden;
constexpr int kOffB3 = kOffW3 + kW3;
constexpr int kMlpParams = kOffB3 + kMlpOut;

}  // namespace vrad

struct vrad_mlp {
    int device = 0;
    float *master = nullptr, *adam_m = nullptr, *adam_v = nullptr, *grad = nullptr;
    uint16_t *w1t = nullptr, *w2t = nullptr, *w3t = nullptr, *w2 = nullptr, *w3 = nullptr;
    float *loss = nullptr;        // device scalar of the last step
    uint32_t *flags = nullptr;    // device word: bit 0, a forward's MMA wait ran out (sticky)
    // Training scratch, grown on demand: activations and their gradients.
    uint16_t *h1 = nullptr, *h2 = nullptr, *dz1 = nullptr, *dz2 = nullptr, *dy = nullptr;
    float *y = nullptr;
    int64_t scratch_rows = 0;
    int64_t step = 0;
};

namespace vrad {

// y[n][3] = the network on x[n][32] (bf16 bits), on `stream`: the
// tcgen05 forward (mlp_tc.cu).
cudaError_t mlp_forward(const vrad_mlp &m, const uint16_t *x, int64_t n, float *y, cudaStream_t stream);
cudaError_t mlp_forward_tc(const vrad_mlp &m, const uint16_t *x, int64_t n, float *y, cudaStream_t stream);

}  // namespace vrad
