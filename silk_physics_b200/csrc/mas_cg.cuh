// Multilevel additive Schwarz (MAS) preconditioner and the persistent
// preconditioned conjugate-gradient kernel.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace silkb {

// Bits of the solver failure word (World::cg_fail), read by the ADMM
// convergence test and reported as IterativeSolveFail.
constexpr int kFailBarrier = 1;   // a grid-barrier wait of a CG kernel gave up
constexpr int kFailMasPivot = 2;  // a MAS bank had a zero or non-finite pivot
constexpr int kFailContactWait = 4;  // a contact Gauss-Seidel copy did not land in time

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
  // Coarse levels above the first: the nodes of the level below that sum
  // into each node (CSR over this level's nodes, members in slot order).
  const int* member_off = nullptr;
  const int* member = nullptr;
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
  int* stats = nullptr;   // accumulated [iterations, solves, first-solve iterations,
                          // learned starts taken, extrapolated starts taken, -]
  // Alternative start (learned warm start or ADMM extrapolation; null =
  // none): the CG starts from x + w (x_alt - x) with the residual-minimising
  // w >= 0 (w = 0: the plain start), while the stopping rule keeps the
  // residual of x as rr0 (the plain start judges the alternative).
  const float4* x_alt = nullptr;
  int alt_stat = 3;       // stats slot counting the alternative starts taken
  int first_solve = 0;    // count this solve's iterations in stats[2]
  float* result_rr = nullptr;
  // Resident form: one block of kResThreads per first-level coarse bank (32
  // fine banks), see cg_resident_kernel.  res_blocks == 0: not available.
  int res_blocks = 0;
  const int* rb_ptr = nullptr;  // per fine bank: first entry of its ELL slice
  const int* rb_w = nullptr;    // per fine bank: slice width
  const int2* rent = nullptr;   // (column, value bits); column < 0: slot -1-c of the block
                                // (slots >= kResThreads: the block's halo)
  const int* halo_off = nullptr;  // per block: first entry of its halo in halo_col
  const int* halo_col = nullptr;  // halo vertices (outside the block, read by its rows)
  int halo_full = 0;  // every off-block column of the resident rows is in its block's halo
  int* fail = nullptr;          // kFail* bits: a barrier wait gave up
  // Device-decided ADMM iterations: the kernel returns at entry when *skip is
  // set (the ADMM solve already ended) and takes its relative tolerance from
  // *rel_tol_dev (the next tolerance set by the ADMM convergence test) when
  // not null.
  const int* skip = nullptr;
  const float* rel_tol_dev = nullptr;
  long long barrier_spin_limit = 0;  // > 0: grid-barrier polls before giving up
  int withhold_block = -1;      // >= 0: that block skips its barrier arrivals (tests)
  // Cluster form with redundant coarse levels (cg_dsm_cluster_kernel): fine
  // banks per CTA (8 or 16; 0 = not this form).  It uses the rb_ptr / rb_w /
  // rent / halo_off / halo_col layout built for blocks of dsm_f fine banks.
  int dsm_f = 0;
  // Its matrix rows in tensor memory: columns allocated per CTA (a power of
  // two, 32..512; 0 = rows read from rent in global memory every SpMV) and
  // row entries held per bank slot (a multiple of 8, at least every rb_w).
  int tm_cols = 0;
  int tm_rw = 0;
  // Its pushes of fine-level z to the halos of other CTAs: per CTA (CSR)
  // entries own slot | consumer CTA << 10 | consumer halo index << 15.
  const int* push_off = nullptr;
  const int* push = nullptr;
  // Optional phase trace of block 0 (null = off): [0] globaltimer and [1]
  // clock64 at entry, [2] and [3] at exit, [4] traced iterations, [5] kernel
  // form (0 streaming, 1 resident), then for each of the first kCgTraceIters
  // iterations kCgTraceSlots clock64 stamps (unused slots repeat the last).
  long long* trace = nullptr;
};

// Per-cloth CG statistics words (CgArgs::stats).
constexpr int kCgStats = 6;
// Halo slots per block of the resident CG kernel (shared memory after the
// block's own kResThreads slots).
constexpr int kResHalo = 1024;
constexpr int kCgTraceIters = 64;
constexpr int kCgTraceSlots = 16;
constexpr int kCgTraceLen = 8 + kCgTraceIters * kCgTraceSlots;

enum CgStatus {
  kCgAbsTol = 0,
  kCgRelTol = 1,
  kCgMaxIter = 2,
  kCgInvalidInitialResidual = 3,
  kCgBarrierTimeout = 4
};

constexpr int kResThreads = 1024;     // one thread per fine-bank slot
constexpr int kResCoarseBanks = 16;   // banks of the coarse levels held by every block
// Resident launch form for a system with res_blocks blocks: 0 = not possible
// on this device, > 0 = cooperative grid of that many blocks, < 0 = one
// thread-block cluster of -value blocks.
int cg_resident_grid(int res_blocks);

void launch_galerkin_fill(const GalerkinDev& g, const double* src_vals,
                          const float* dyn, cudaStream_t st);
// mode 0: fine level (fill from L, add dynamic diagonal via part offsets).
void launch_bank_invert(const MasLevelDev& lv, bool fine, const int* part_off,
                        const double* src_vals, const float* dyn, int* fail,
                        cudaStream_t st);
int cg_grid_size(int nslices, int nbank0);
void launch_cg(const CgArgs& a, int grid, cudaStream_t st);
void launch_cg_resident(const CgArgs& a, int grid, cudaStream_t st);
// Cluster form with redundant coarse levels: CTAs of f fine banks (8 or 16)
// for nbank0 fine banks if they form one launchable cluster (at most 16
// CTAs), else 0.
constexpr int kDsmCoarseBankLimit = 16;  // banks of all coarse levels together
// Pushes of fine-level z per CTA of the cluster form: at most 2 per thread.
constexpr int kDsmPushPerThread = 2;
int cg_dsm_ctas(int nbank0, int f);
void launch_cg_dsm(const CgArgs& a, int nctas, cudaStream_t st);

}  // namespace silkb
