// lprec.cuh -- the learned pressure preconditioner: a 4-layer 3^3
// convolution network (3 -> 16 -> 16 -> 16 -> 1 channels, ReLU after the
// first three layers, no biases), BF16 weights and activations with FP32
// accumulation, applied on the tile-blocked grid.  No reference counterpart.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "native.cuh"

namespace flip {

constexpr int kLpLayers = 4;
constexpr int kLpCh = 16;
constexpr int kLpCin[kLpLayers] = {3, kLpCh, kLpCh, kLpCh};
constexpr int kLpCout[kLpLayers] = {kLpCh, kLpCh, kLpCh, 1};
// weights of layer l: [27 taps][Cin][Cout], taps ordered dz, dy, dx in -1..1
constexpr int kLpW[kLpLayers] = {27 * 3 * kLpCh, 27 * kLpCh * kLpCh, 27 * kLpCh * kLpCh, 27 * kLpCh};
constexpr int kLpWOff[kLpLayers + 1] = {0, kLpW[0], kLpW[0] + kLpW[1], kLpW[0] + kLpW[1] + kLpW[2],
                                        kLpW[0] + kLpW[1] + kLpW[2] + kLpW[3]};
constexpr int kLpNumW = kLpWOff[kLpLayers];

struct LpNet {
    int dil[kLpLayers];   // dilation of each layer
    float* w;             // FP32 master weights [kLpNumW]
    float* g;             // gradient [kLpNumW]
    float* m;             // Adam first moment
    float* v;             // Adam second moment
    __nv_bfloat16* wb;    // BF16 copy used by the kernels
    __nv_bfloat16* act[3];  // activations after layers 0..2: [slot][16]
    __nv_bfloat16* actz[3]; // the same for the zero-residual pass f(0)
    float* gact;          // gradient of one activation layer: [slot][16]
    float* gact2;         // second gradient buffer: [slot][16]
    int adam_t;
    int tensor_cores;     // 1: the 16 -> 16 layers run on tcgen05 (forward and backward)
    int sms;              // SM count (persistent grid of the tensor-core kernels)
    int* err;             // device error word of the tensor-core kernels (bit 0: a wait timed out)
};

// Inputs the network reads: residual r (FP32, read only at fluid cells),
// cell types (0 air, 1 fluid, 2 solid), the per-tile active flags and the
// tile lists (the layers 0..2 run on the dilated list, layer 3 on the fluid
// tile list).
struct LpGrid {
    const float* r;
    const uint8_t* type;
    const uint8_t* tile_active;  // [tiles] nonzero where activations are valid
    const uint32_t* act_tiles;   // tiles where activations are computed
    const uint32_t* d_nact;
    const uint32_t* out_tiles;   // tiles with fluid cells (outputs)
    const uint32_t* d_nout;
    const int* halt;             // optional: nonzero stops the kernels (a converged FPCG)
    const uint8_t* cell;         // PCG cell codes: fluid bit, Jacobi diagonal in bits 0-2
    NatDims D;
};

// one 16 -> 16 layer (ReLU) on the tensor cores: out = relu(conv(in)) on the
// active tiles (lprec_tc.cu); dil in {1, 2, 4}
int lp_mid_forward_tc(const LpGrid& G, const __nv_bfloat16* wb, int dil, const __nv_bfloat16* in, __nv_bfloat16* out,
                      int* err, int sms, cudaStream_t st);
// The network: N(r) = s (f(r/s) - f(0)) on fluid cells, 0 elsewhere, with
// f = the convolutions on the channels [r/s, fluid, solid], s = 1/(*d_inv_s)
// = rms(r) over the fluid cells.  f(0) depends on the geometry only; without
// it the network can answer every residual with the same geometry-shaped
// field (the hydrostatic part of the training solutions), which gives
// flexible CG nothing new after its first step.
// f0 = f(0) (once per problem; uses the actz buffers)
int lp_bias_dev(const LpNet& net, const LpGrid& G, const float* d_inv_s, float* f0, int grid, cudaStream_t st);
// z = N(r) given f0
int lp_forward_dev(const LpNet& net, const LpGrid& G, const float* d_inv_s, const float* f0, float* z, int grid,
                   cudaStream_t st);
// one 16 -> 16 layer on a small grid whose every tile is active, on the
// tensor cores: a CTA per 128 voxels (lprec_tc.cu)
int lp_small_mid_forward_tc(const LpGrid& G, const __nv_bfloat16* wb, int dil, const __nv_bfloat16* in, __nv_bfloat16* out,
                            int* err, uint32_t ntiles, cudaStream_t st);
// the same two passes on a small grid whose every tile is in G's tile lists
// (ntiles tiles, the coarsest level of the multilevel preconditioner): a CTA
// per 16 voxels
int lp_small_bias(const LpNet& net, const LpGrid& G, uint32_t ntiles, const float* d_inv_s, float* f0, cudaStream_t st);
int lp_small_forward(const LpNet& net, const LpGrid& G, uint32_t ntiles, const float* d_inv_s, const float* f0, float* z,
                     cudaStream_t st);
// gradient of the loss with respect to the weights given dL/dz (gz, FP32 on
// the slots of the active tiles, zero off fluid cells), through both the
// f(r/s) and the f(0) activations; accumulates into net.g (caller zeroes it)
int lp_backward_dev(LpNet& net, const LpGrid& G, const float* d_inv_s, const float* gz, int grid, cudaStream_t st);
// the backward pass of one 16 -> 16 layer on the tensor cores (lprec_tc.cu),
// over the voxels of the active list: gin = relu'(ain) * (the gradient of the
// layer's input from gout), and dw += the weight gradient (FP32 atomics)
int lp_mid_dgrad_tc(const LpGrid& G, const __nv_bfloat16* wb, int dil, const float* gout, const __nv_bfloat16* ain,
                    float* gin, int* err, int sms, cudaStream_t st);
int lp_mid_wgrad_tc(const LpGrid& G, int dil, const float* gout, const __nv_bfloat16* ain, float* dw, int* err, int sms,
                    cudaStream_t st);
// the weight gradients of the input layer (3 -> 16; its input channels from
// G.r, G.type and the scale) and of the output layer (16 -> 1; dL/dout =
// sign * s * gz on the output tiles) on the tensor cores
int lp_in_wgrad_tc(const LpGrid& G, int dil, const float* gout, const float* d_inv_s, float* dw, int* err, int sms,
                   cudaStream_t st);
int lp_out_wgrad_tc(const LpGrid& G, int dil, const float* gz, const __nv_bfloat16* ain, const float* d_inv_s, float sign,
                    float* dw, int* err, int sms, cudaStream_t st);
// training loss of the preconditioner M(r) = N(r) + D^-1 r for a sample
// (r, e) with A e = r: L = |M(r) - e|_A^2 / |e|_A^2 = (m.Am - 2 m.r)/e.r + 1.
// Accumulates m.Am, m.r, e.r into d_sums[0..2] (caller zeroes them), keeps
// A m - r in wbuf and writes gz = dL/dN = 2 (A m - r) / e.r on the fluid
// cells of the active tiles (0 elsewhere)
int lp_loss_grad(const LpGrid& G, const float* z, const float* ev, float* wbuf, float* gz, double* d_sums, int grid,
                 cudaStream_t st);
// white-noise error sample: e ~ N(0,1) on fluid cells (hash of seed and slot), r = A e
int lp_noise_sample(const LpGrid& G, uint64_t seed, float* ev, float* r, int grid, cudaStream_t st);
// xs = x + xg (the reference solution) and e = xs - (x + xg) on the fluid cells
int lp_store_solution(const LpGrid& G, const double* x, const float* xg, float* xs, int grid, cudaStream_t st);
int lp_error_from_solution(const LpGrid& G, const double* x, const float* xg, const float* xs, float* ev, int grid,
                           cudaStream_t st);
// *d_inv_s = 1 / rms(r) over the fluid cells of the output tiles
int lp_input_scale(const LpGrid& G, double* d_acc, const double* d_nfluid, float* d_inv_s, int grid, cudaStream_t st);
// Adam step on the FP32 master weights, then the BF16 copy
int lp_adam(LpNet& net, float lr, cudaStream_t st);
int lp_sync_bf16(LpNet& net, cudaStream_t st);

}  // namespace flip
