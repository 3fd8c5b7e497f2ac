// fcgnet.cuh — the learned preconditioner of the 3D flexible CG: a linear
// 4-level convolutional encoder-decoder on the cell grid.
//
// Layers (3x3x3 kernels, zero padding, no bias, no activation):
//   a1 = c1(r)                     level 1 (n),    1 -> 16
//   a2 = c2(pool(a1))              level 2 (n/2), 16 -> 32
//   a3 = c3(pool(a2))              level 3 (n/4), 32 -> 64
//   a4 = c4(pool(a3))              level 4 (n/8), 64 -> 64
//   b3 = c5(up(a4) + a3)           level 3,       64 -> 32
//   b2 = c6(up(b3) + a2)           level 2,       32 -> 16
//   z  = c7(up(b2) + a1)           level 1,       16 -> 1
// pool = 2x2x2 mean, up = nearest-neighbour (each coarse cell to its 8
// children). Activations are BF16, channels innermost (x fastest, then y, z);
// accumulation is FP32. The network is linear, so it is applied to r / rms(r)
// and its output scaled back, with the grid spacing factor h^2 of A^-1.
//
// Parameters: one FP32 array, layer after layer, each W[co][tap][ci] with
// tap = 9 (dz+1) + 3 (dy+1) + (dx+1).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace flursys {

constexpr int kNetLayers = 7;
constexpr int kNetCin[kNetLayers] = {1, 16, 32, 64, 64, 32, 16};
constexpr int kNetCout[kNetLayers] = {16, 32, 64, 64, 32, 16, 1};

long long net_param_offset(int layer);
long long net_param_count();

// Device buffers of one network on one grid size (grown on demand).
struct NetWorkspace {
    int nx = 0, ny = 0, nz = 0;
    bool training = false;
    size_t bytes = 0;
    void *base = nullptr;
    // activations (bf16) and their gradients
    uint16_t *a1 = nullptr, *x2 = nullptr, *a2 = nullptr, *x3 = nullptr, *a3 = nullptr, *x4 = nullptr, *a4 = nullptr;
    uint16_t *x5 = nullptr, *b3 = nullptr, *x6 = nullptr, *b2 = nullptr, *x7 = nullptr;
    uint16_t *g7 = nullptr, *g6 = nullptr, *g5 = nullptr, *g4 = nullptr, *g3 = nullptr, *g2 = nullptr;
    uint16_t *gb2 = nullptr, *gb3 = nullptr, *ga4 = nullptr, *ga3 = nullptr, *ga2 = nullptr, *ga1 = nullptr;
    float *out32 = nullptr;  // training: network output
    float *gout = nullptr;   // training: dL/d(output)
    float *lq = nullptr;     // training: L e of the residual-norm loss
    double *scalars = nullptr;  // [0] input scale, [1] loss sum, [2..] partials
    double *partials = nullptr;
    int npartials = 0;
    cudaError_t ensure(int nx, int ny, int nz, bool training);
    void release();
};

// BF16 copies of the parameters: forward layout and the transposed, flipped
// layout that turns the data gradient into a forward convolution.
// Interior composite 5x5x5 stencil of the fused output layer, passed to its
// kernel by value (constant-bank operands).
struct NetOutParams {
    float k[125];         // (dz * 5 + dy) * 5 + dx, offsets -2..2
};

struct NetWeights {
    uint16_t *fwd = nullptr;   // W[co][tap][ci]
    uint16_t *bwd = nullptr;   // W'[ci][26 - tap][co]
    float *fwd_f32 = nullptr;  // FP32 copies of c1, c7 (CUDA-core layers) and their transposes
    float *fused = nullptr;    // FP32 composite stencils of the fused full-resolution layers
    uint32_t *upfrag = nullptr;  // the output layer's up-path weights as tensor-core B fragments
    uint32_t *infrag = nullptr;  // the input layer's composite stencil as tensor-core B fragments
    // host copy of the output layer's interior stencil, refreshed from `fused` on the
    // first application after a repack
    mutable NetOutParams out_params{};
    mutable bool host_params_valid = false;
    cudaError_t allocate();
    void release();
};

// Packs FP32 master parameters (device) into the BF16 copies.
cudaError_t net_pack_weights(const float *master, NetWeights &w, cudaStream_t st);

// z = N(r): scale = 1/rms(r) is computed on the device, the output is
// multiplied by h2 / scale. r and z are FP32 cell vectors.
cudaError_t net_apply(const NetWeights &w, NetWorkspace &ws, int nx, int ny, int nz, double h2, const float *r,
                      float *z, cudaStream_t st);

// Training losses of e = net(b_hat) - p_hat on the unit-spacing pure-Neumann
// operator L (L p_hat = b_hat, sum b_hat = 0); constants are free:
//   energy    e.L e / norm          (norm = p_hat . b_hat)
//   residual  |L e|^2 / norm        (norm = b_hat . b_hat), i.e. |L net(b) - b|^2
enum NetLoss : int { kNetLossEnergy = 0, kNetLossResidual = 1 };

// One training sample: forward on b_hat (already normalised), loss,
// backward; accumulates dL/dW into grad (FP32, net_param_count()) and the
// loss into *loss (device).
cudaError_t net_train_sample(const NetWeights &w, NetWorkspace &ws, int nx, int ny, int nz, const float *b_hat,
                             const float *p_hat, double norm, int loss_kind, float *grad, double *loss,
                             cudaStream_t st);

// Adam on FP32 master weights (bias-corrected, step t >= 1), gradient
// multiplied by grad_scale first.
cudaError_t net_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float beta1, float beta2,
                     float eps, long long t, float grad_scale, cudaStream_t st);

}  // namespace flursys
