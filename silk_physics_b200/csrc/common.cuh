// Shared device/host helpers for the B200 cloth solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

namespace silkb {

#define SILK_HD __host__ __device__ __forceinline__

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define CUDA_CHECK(x) ::silkb::check_cuda((x), #x)

// Counts every kernel launch issued by this library (reported in the per-step
// statistics so callers can see how many native kernels a step took).
extern thread_local long long g_launch_count;
#define SILK_LAUNCHED() (++::silkb::g_launch_count)

constexpr int BANK = 32;           // MAS bank size (vertices per partition)
constexpr int MAX_COARSE = 4;      // coarse MAS levels
constexpr int THREADS = 256;

SILK_HD int div_up(int a, int b) { return (a + b - 1) / b; }

SILK_HD float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
SILK_HD float3 f3(const float4& v) { return make_float3(v.x, v.y, v.z); }
SILK_HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
SILK_HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
SILK_HD float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
SILK_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Packed upper-triangular index of a symmetric n x n matrix (row-major).
SILK_HD int upper_index(int n, int i, int j) {
  if (i > j) {
    int t = i;
    i = j;
    j = t;
  }
  return i * n - (i * (i + 1)) / 2 + j;
}

}  // namespace silkb
