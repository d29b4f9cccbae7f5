// cnn.cuh -- the flux-correction network of the learned coarse shallow-water solver: three 5x5
// convolutions (3 -> 32 -> 32 -> 6 channels, ReLU between), bf16 weights and activations, fp32
// accumulation on the tensor cores (tcgen05 for the 32-channel inputs, mma.sync m16n8k16 for the 8-channel ones
// and as an alternative), trained with Adam on fp32 master weights.
// No counterpart in the reference; its error is measured against the plain fine solver (ShallowWater.kernel).
//
// Layouts (per sample, row-major cells, channels innermost):
//   x0   bf16 [H][W][8]   features (h - 1) * 4, hu * 4, hv * 4, then zeros
//   a1   bf16 [H][W][32]  relu(conv1), a2 likewise; y3 fp32 [H][W][8]: conv3 (six used: the east face's mass,
//                         x- and y-momentum corrections, then the north face's)
//   weights, forward      bf16 [cout][taps * cin] tap-major (tap = ky * 5 + kx), cin = 8 (layer 1: 26 taps,
//                         the last zero, so that a 16-wide k step covers two taps) or 32
//   weights, backward     the same shape with cin and cout swapped and the taps mirrored (tap 24 - t)
//   master parameters     fp32, in this order: w1 [32][25][3], b1 [32], w2 [32][25][32], b2 [32],
//                         w3 [6][25][32], b3 [6]
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace vf {

constexpr int CNN_HID = 32;      // hidden channels
constexpr int CNN_IN = 8;        // input channels as stored (3 used)
constexpr int CNN_OUT = 8;       // output channels as stored (6 used)
constexpr int CNN_TAPS = 25;
constexpr int CNN_FEATURES = 3, CNN_FLUXES = 6;
constexpr int CNN_PARAMS = CNN_HID * CNN_TAPS * CNN_FEATURES + CNN_HID + CNN_HID * CNN_TAPS * CNN_HID + CNN_HID +
                           CNN_FLUXES * CNN_TAPS * CNN_HID + CNN_FLUXES;   // 32870
constexpr float CNN_SCALE_H = 4.0f, CNN_SCALE_Q = 4.0f;                     // feature scales

// Offsets of the master parameters.
constexpr int P_W1 = 0, P_B1 = P_W1 + CNN_HID * CNN_TAPS * CNN_FEATURES, P_W2 = P_B1 + CNN_HID,
              P_B2 = P_W2 + CNN_HID * CNN_TAPS * CNN_HID, P_W3 = P_B2 + CNN_HID,
              P_B3 = P_W3 + CNN_FLUXES * CNN_TAPS * CNN_HID;

// Row length (k extent) of a bf16 weight matrix whose inputs have cin channels.
__host__ __device__ constexpr int conv_k(int cin) { return cin == 8 ? 26 * 8 : CNN_TAPS * cin; }

enum ConvMode { CONV_RELU = 0, CONV_LINEAR = 1, CONV_GRAD_MASK = 2 };

struct ConvArgs {
    const __nv_bfloat16* in;     // [B][H][W][cin]
    const __nv_bfloat16* w;      // [cout][conv_k(cin)]
    const float* bias;           // [cout real] or null
    int bias_n;                  // real output channels with a bias
    __nv_bfloat16* out_b;        // CONV_RELU / CONV_GRAD_MASK: [B][H][W][cout]
    float* out_f;                // CONV_LINEAR: [B][H][W][cout]
    const __nv_bfloat16* mask;   // CONV_GRAD_MASK: [B][H][W][cout], the gradient passes where mask > 0
    int H, W, B;
};

struct WgradArgs {
    const __nv_bfloat16* in;     // [B][H][W][cin], the layer's input
    const __nv_bfloat16* dy;     // [B][H][W][cout], the gradient at the layer's output
    float* dw;                   // master layout [cout real][25][cin real], accumulated
    float* db;                   // [cout real], accumulated
    int cin_real, cout_real;
    int H, W, B;
};

// The convolution kernels (cin, cout, mode) = (8, 32, RELU), (32, 32, RELU), (32, 8, LINEAR), (8, 32, GRAD_MASK),
// (32, 32, GRAD_MASK), and the weight gradients (cin, cout) = (8, 32), (32, 32), (32, 8): 256 threads, the
// dynamic shared memory below, a persistent grid of any size. rows: the row-blocked kernels for 32 input
// channels (a warp computes several output rows from each loaded A fragment); false: one output row per warp.
const void* conv_kernel(int cin, int cout, int mode, bool rows);
const void* wgrad_kernel(int cin, int cout);
cudaError_t launch_conv(int cin, int cout, int mode, bool rows, int grid, const ConvArgs& a, cudaStream_t s);
cudaError_t launch_wgrad(int cin, int cout, int grid, const WgradArgs& a, cudaStream_t s);
size_t conv_smem(int cin, int cout, bool rows);
size_t wgrad_smem(int cin, int cout);

// The convolutions on tcgen05 with warp-specialised roles (cnn_tc.cu): TMA into a ring of input rows, one
// MMA-issuing thread, eight epilogue warps; (cin, cout, mode) as conv_kernel's; 320 threads, one CTA per SM
// (conv_tc_smem bytes); the launch builds the input's tensor map.
const void* conv_tc_kernel(int cin, int cout, int mode);
size_t conv_tc_smem(int cin, int cout);
cudaError_t launch_conv_tc(int cin, int cout, int mode, const ConvArgs& a, uint32_t* status, cudaStream_t s);

}  // namespace vf
