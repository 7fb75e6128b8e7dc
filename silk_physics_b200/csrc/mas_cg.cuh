// Multilevel additive Schwarz (MAS) preconditioner and the persistent
// preconditioned conjugate-gradient kernel.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace silkb {

constexpr int kPacked = BANK * (BANK + 1) / 2;  // 528 packed upper entries

struct MasLevelDev {
  int nbank = 0;
  int nnode = 0;                    // real nodes at this level (coarse)
  const int* fill_src = nullptr;    // 528 per bank
  const signed char* slot_cco = nullptr;
  const int* cco_base = nullptr;
  const int* ncco = nullptr;
  float* M = nullptr;               // packed inverse, FP32
  __nv_bfloat16* Mb = nullptr;      // packed inverse, BF16
  float4* rin = nullptr;            // coarse: input per node (restriction)
  float4* zout = nullptr;           // coarse: output per node
  float4* rout = nullptr;           // restriction to the next coarse space
};

struct GalerkinDev {
  int n_entries = 0;
  const int* src_off = nullptr;
  const int* src = nullptr;
  const int* diag_off = nullptr;
  const int* diag = nullptr;
  double* vals = nullptr;
};

// Everything the CG kernel of one cloth needs.
struct CgArgs {
  int nv = 0;
  // Off-diagonal part of L in sliced ELL (32 rows per slice).
  int nslices = 0;
  const int* sl_ptr = nullptr;
  const int* sl_w = nullptr;
  const int2* ent = nullptr;  // (column, float bits)
  const float* Ldiag = nullptr;
  const float* dyn = nullptr;  // dynamic diagonal (mass/dt^2 + pins + contacts)
  const float4* b = nullptr;
  float4* x = nullptr;
  float4* r = nullptr;
  float4* z0 = nullptr;
  float4* p = nullptr;
  float4* Ap = nullptr;
  const int4* cmap = nullptr;
  // Fine level (banks = parts).
  int nbank0 = 0;
  const int* part_off = nullptr;
  MasLevelDev fine;
  int levels = 0;
  MasLevelDev coarse[4];
  int bf16 = 0;
  // Scratch.
  double* partials = nullptr;  // gridDim.x * 4
  double* coarse_partial = nullptr;
  unsigned* barrier = nullptr;  // [count, err, gen]
  float rel_tol = 1e-3f, abs_tol = 1e-7f;
  int max_iter = 1000;
  int* result = nullptr;  // [iterations, status]
  int* stats = nullptr;   // accumulated [iterations, solves]
  float* result_rr = nullptr;
};

enum CgStatus {
  kCgAbsTol = 0,
  kCgRelTol = 1,
  kCgMaxIter = 2,
  kCgInvalidInitialResidual = 3,
  kCgBarrierTimeout = 4
};

void launch_galerkin_fill(const GalerkinDev& g, const double* src_vals,
                          const float* dyn, cudaStream_t st);
// mode 0: fine level (fill from L, add dynamic diagonal via part offsets).
void launch_bank_invert(const MasLevelDev& lv, bool fine, const int* part_off,
                        const double* src_vals, const float* dyn,
                        cudaStream_t st);
int cg_grid_size(int nslices, int nbank0);
void launch_cg(const CgArgs& a, int grid, cudaStream_t st);

}  // namespace silkb
