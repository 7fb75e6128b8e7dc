// Learned CG warm start: per-vertex MLP 13 -> 64 -> 64 -> 64 -> 3 (GELU,
// BF16 weights and layer inputs on the tensor cores, FP32 accumulation) that
// predicts the solution of the first CG solve of an outer iteration from
// kinematic features.  No counterpart in the reference.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace silkb {

constexpr int kMlpIn = 13;    // features per vertex
constexpr int kMlpK = 16;     // padded input width
constexpr int kMlpH = 64;     // hidden width
constexpr int kMlpOut = 3;    // outputs per vertex
constexpr int kMlpKOut = 8;   // padded output width
// FP32 parameter vector layout: weights are row-major (input, output).
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpK * kMlpH;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpH * kMlpH;
constexpr int kOffW4 = kOffB3 + kMlpH;
constexpr int kOffB4 = kOffW4 + kMlpH * kMlpKOut;
constexpr int kOffMean = kOffB4 + kMlpKOut;     // feature mean (16)
constexpr int kOffStd = kOffMean + kMlpK;       // feature std (16)
constexpr int kOffOutScale = kOffStd + kMlpK;   // output scale (8)
constexpr int kMlpParams = kOffOutScale + kMlpKOut;
constexpr int kMlpTrainParams = kOffMean;       // learned part

// BF16 elements of the weight image (the four layers' B operands as the
// forward holds them in shared memory: 64x16, 64x64, 64x64, 16x64).
constexpr int kMlpWeightImage = kMlpH * kMlpK + 2 * kMlpH * kMlpH + 16 * kMlpH;

// Device model: FP32 parameters and their BF16 weight image.
struct MlpDev {
  const float* params = nullptr;    // kMlpParams
  const uint16_t* image = nullptr;  // kMlpWeightImage BF16 (mlp_image of params)
  int* fail = nullptr;              // kFailMlpWait is set here when a tensor-core wait gives up
};

// Build the weight image of a parameter vector (device pointers).
void mlp_image(const float* params, uint16_t* image, cudaStream_t st);

// Bit of the solver's failure word: a tensor-core product of the forward did
// not complete within its bounded wait.
constexpr int kFailMlpWait = 8;

// Output o (n x 3, normalised units) of raw features (n x 16: displacement
// features divided by the step scale, pin flag, zero padding).
void mlp_forward(const MlpDev& m, const float* feat, int n, float* out, cudaStream_t st);

// Loss (mean squared error against t_hat, n x 4 with 3 used) and its gradient
// over the trainable parameters (grad: kMlpParams, statistics zero).  work
// must hold mlp_work_floats(n) floats; loss is written to loss_out (device).
size_t mlp_work_floats(int n);
void mlp_loss_grad(const MlpDev& m, const float* feat, const float* t_hat, int n,
                   const int* index, float* work, float* grad, double* loss_out,
                   cudaStream_t st);

// One Adam step on the trainable part (FP32 state m, v).
void mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr,
              cudaStream_t st);

// Per-vertex warm-start features of the vertices [0, n): start x0, previous
// step starts x1, x2, inertial prediction y, pin flags, 1-ring CSR.
void warm_features(int n, const float4* x0, const float4* x1, const float4* x2,
                   const float4* y, const uint8_t* pin, const int* ring_off,
                   const int* ring, float inv_sigma, float* feat, cudaStream_t st);
// x_pred = y + sigma * out_scale * MLP(feat).
void warm_predict(const MlpDev& m, int n, const float* feat, const float4* y, float sigma,
                  float* out_tmp, float4* x_pred, cudaStream_t st);
// Training target of the first CG solve: (x - y) / sigma.
void warm_target(int n, const float4* x, const float4* y, float inv_sigma, float* t,
                 cudaStream_t st);

// Learned iterate start: sigma (device scalar) = RMS of x - h1; features of
// (x, h1 = x_(k-1), h2 = x_(k-2)) into feat (n x 16); with a model (m.params
// not null) x_pred = x + sigma * out_scale * MLP(feat).
void iterate_predict(const MlpDev& m, int n, const float4* x, const float4* h1, const float4* h2,
                     const uint8_t* pin, const int* ring_off, const int* ring, float* sigma,
                     float* feat, float* out_tmp, float4* x_pred, cudaStream_t st);
// Append m samples (features from feat, target (x_new - x_old) / sigma) to
// out_feat / out_tgt at the counter's position while below cap.
void iterate_samples(int m, int n, unsigned salt, const float* feat, const float4* x_new,
                     const float4* x_old, const float* sigma, float* out_feat, float* out_tgt,
                     int* counter, int cap, const int* skip, cudaStream_t st);
constexpr int kIterSamplesPerSolve = 256;   // vertices recorded per ADMM iteration
constexpr int kIterSampleCap = 1 << 19;     // samples per step

// Standalone entry points on host buffers (the trainer and the gradient
// checks): forward outputs (n x 3), loss and gradient, Adam training.
void mlp_forward_host(const float* params, const float* feat, int64_t n, float* out);
void mlp_loss_grad_host(const float* params, const float* feat, const float* tgt, int64_t n,
                        float* grad, double* loss);
void mlp_train_host(float* params, const float* feat, const float* tgt, int64_t n, int steps,
                    int batch, float lr, uint64_t seed, float* loss_hist);

}  // namespace silkb
