// Host side of the standalone MLP entry points (forward, loss gradient and
// the Adam training loop on the GPU) used by the warm-start trainer and the
// gradient checks.
#include <cstring>
#include <vector>

#include "learned.cuh"
#include "world.hpp"

namespace silkb {

namespace {

__global__ void sample_index_kernel(int* idx, int batch, int n, unsigned long long seed,
                                    int step) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= batch) return;
  unsigned long long z = seed ^ ((unsigned long long)step << 32) ^ (unsigned long long)i;
  z += 0x9e3779b97f4a7c15ULL;  // splitmix64
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  idx[i] = (int)(z % (unsigned long long)n);
}

struct MlpBuffers {
  DevBuf<float> params, feat, tgt, out, grad, work, m, v;
  DevBuf<uint16_t> image;
  DevBuf<double> loss;
  DevBuf<int> idx, fail;
  void load(const float* p, const float* f, const float* t, int n, cudaStream_t st) {
    params.alloc(kMlpParams);
    image.alloc(kMlpWeightImage);
    fail.alloc(1);
    fail.zero(st);
    CUDA_CHECK(cudaMemcpyAsync(params.p, p, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, st));
    if (f) {
      feat.alloc((size_t)kMlpK * n);
      CUDA_CHECK(cudaMemcpyAsync(feat.p, f, (size_t)kMlpK * n * sizeof(float),
                                 cudaMemcpyHostToDevice, st));
    }
    if (t) {
      tgt.alloc((size_t)4 * n);
      CUDA_CHECK(cudaMemcpyAsync(tgt.p, t, (size_t)4 * n * sizeof(float),
                                 cudaMemcpyHostToDevice, st));
    }
  }
  MlpDev dev() const { return MlpDev{params.p, image.p, fail.p}; }
  // A tensor-core wait of the forward gave up (after the work on `st`).
  void check(cudaStream_t st) const {
    int f = 0;
    CUDA_CHECK(cudaMemcpyAsync(&f, fail.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_CHECK(cudaStreamSynchronize(st));
    if (f) throw CudaError("tensor-core wait gave up");
  }
};

}  // namespace

void mlp_forward_host(const float* params, const float* feat, int64_t n, float* out) {
  cudaStream_t st = nullptr;
  MlpBuffers b;
  b.load(params, feat, nullptr, (int)n, st);
  b.out.alloc((size_t)kMlpOut * n);
  mlp_image(b.params.p, b.image.p, st);
  mlp_forward(b.dev(), b.feat.p, (int)n, b.out.p, st);
  b.check(st);
  CUDA_CHECK(cudaMemcpy(out, b.out.p, (size_t)kMlpOut * n * sizeof(float), cudaMemcpyDeviceToHost));
}

void mlp_loss_grad_host(const float* params, const float* feat, const float* tgt, int64_t n,
                        float* grad, double* loss) {
  cudaStream_t st = nullptr;
  MlpBuffers b;
  b.load(params, feat, tgt, (int)n, st);
  b.grad.alloc(kMlpParams);
  b.work.alloc(mlp_work_floats((int)n));
  b.loss.alloc(1);
  mlp_image(b.params.p, b.image.p, st);
  mlp_loss_grad(b.dev(), b.feat.p, b.tgt.p, (int)n, nullptr, b.work.p, b.grad.p, b.loss.p, st);
  b.check(st);
  CUDA_CHECK(cudaMemcpy(grad, b.grad.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
  CUDA_CHECK(cudaMemcpy(loss, b.loss.p, sizeof(double), cudaMemcpyDeviceToHost));
}

void mlp_train_host(float* params, const float* feat, const float* tgt, int64_t n, int steps,
                    int batch, float lr, uint64_t seed, float* loss_hist) {
  cudaStream_t st = nullptr;
  MlpBuffers b;
  b.load(params, feat, tgt, (int)n, st);
  const bool full = batch <= 0 || batch >= n;
  const int nb = full ? (int)n : batch;
  b.grad.alloc(kMlpParams);
  b.work.alloc(mlp_work_floats(nb));
  b.m.alloc(kMlpParams);
  b.v.alloc(kMlpParams);
  b.m.zero(st);
  b.v.zero(st);
  b.loss.alloc(steps > 0 ? steps : 1);
  if (!full) b.idx.alloc(nb);
  for (int step = 1; step <= steps; ++step) {
    if (!full) {
      sample_index_kernel<<<div_up(nb, 256), 256, 0, st>>>(b.idx.p, nb, (int)n, seed, step);
      SILK_LAUNCHED();
    }
    mlp_image(b.params.p, b.image.p, st);
    mlp_loss_grad(b.dev(), b.feat.p, b.tgt.p, nb, full ? nullptr : b.idx.p, b.work.p, b.grad.p,
                  b.loss.p + (step - 1), st);
    mlp_adam(b.params.p, b.grad.p, b.m.p, b.v.p, step, lr, st);
  }
  b.check(st);
  CUDA_CHECK(cudaMemcpy(params, b.params.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss_hist && steps > 0) {
    std::vector<double> h(steps);
    CUDA_CHECK(cudaMemcpy(h.data(), b.loss.p, steps * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < steps; ++i) loss_hist[i] = (float)h[i];
  }
}

}  // namespace silkb
