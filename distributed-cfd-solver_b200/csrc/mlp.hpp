// Learned initial guess for the Newton linear solve: a per-cell MLP
// (48 features -> 64 -> 64 -> 16 outputs, ReLU, BF16 weights and
// activations, FP32 accumulation in tensor memory) run by hand-written
// tcgen05 kernels for inference and training.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace cfdg {

constexpr int kMlpIn = 48;    // features per cell (7 groups of nvars + log CFL, zero padded)
constexpr int kMlpHid = 64;   // hidden width
constexpr int kMlpOut = 16;   // outputs (nvars used, zero padded)
constexpr int kMlpTile = 128; // cells per tensor-core tile (MMA M)
// fp32 parameter vector: W1[64x48] b1[64] W2[64x64] b2[64] W3[16x64] b3[16]
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpHid * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHid;
constexpr int kOffB2 = kOffW2 + kMlpHid * kMlpHid;
constexpr int kOffW3 = kOffB2 + kMlpHid;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpHid;
constexpr int kMlpParams = kOffB3 + kMlpOut;  // 8336

// Device views of the network used by the kernels.
struct MlpDev {
    const uint16_t* w1;  // bf16 bits, row-major out x in
    const uint16_t* w2;
    const uint16_t* w3;
    const float* params;  // fp32 master (biases are read from here)
    int nout;             // outputs that carry a loss (nvars)
};

// D[128 x N] = A[128 x K] * B[N x K]^T with bf16 inputs (row-major) on one
// CTA; N in {16, 32, 48, 64}, K a multiple of 16 up to 128.  Returns a
// device error flag value (0 = ok).
void launch_tc_selftest(const uint16_t* A, const uint16_t* B, float* D, int N, int K, int* err, cudaStream_t s);

// out[r * nv + v] = scale[v] * y_v(features row r) for v < nv.
void launch_mlp_forward(const MlpDev& net, const uint16_t* feat, int64_t rows, const double* scale, int nv,
                        double* out, int* err, int grid, cudaStream_t s);

// Loss and gradient partials of mean squared error over `rows` samples:
// partials[cta * (kMlpParams + 1) + p], last entry the CTA's loss sum.
void launch_mlp_grad(const MlpDev& net, const uint16_t* feat, const float* target, int64_t rows, float* partials,
                     int* err, int grid, cudaStream_t s);

// Sums the CTA partials in fixed order, scales by 1/(rows * nout), and
// applies one Adam step (or only writes the gradient when adam == false).
void launch_mlp_adam(float* params, float* m, float* v, uint16_t* w1, uint16_t* w2, uint16_t* w3,
                     const float* partials, int nparts, double inv_count, float lr, float beta1, float beta2,
                     float eps, int step, bool adam, float* grad_out, float* loss_out, cudaStream_t s);

// Rounds the fp32 master weights to the bf16 copies.
void launch_mlp_sync_bf16(const float* params, uint16_t* w1, uint16_t* w2, uint16_t* w3, cudaStream_t s);

}  // namespace cfdg
