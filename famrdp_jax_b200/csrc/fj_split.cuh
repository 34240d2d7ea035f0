// fj_split.cuh -- the three-kernel stage pipeline over a table of blocks
// (fj_stage_split.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fj_common.cuh"

namespace fj {

constexpr int kMaxSplitBlocks = 32;  // blocks per launch (more are chunked)

struct SplitBlock {
  const double* q;       // stage input (5, ni, nj, nk)
  const double* q0;      // step start state (stages 2, 3)
  double* out;           // RHS (stage 0) or stage result; may alias q0, never q
  const double* kxyz;    // (3, 3, ni, nj, nk)
  const float* kxyz32;   // optional FP32 copy (FP32-flux path) or nullptr
  const double* vol;     // (ni, nj, nk)
  void* prim;            // scratch: 6 x N flux-type values
  void* F;               // scratch: 15 x N (face c | c+e_a, axis-major)
  void* G;               // scratch: 9 x N viscous flux components
  int ni, nj, nk;
  int cta_begin;         // filled by the launcher
};

// Scratch bytes of the intermediates of `cells` padded cells in total.
size_t split_scratch_bytes(int precision, int64_t cells);
// Points prim/F/G of every block into one scratch region of
// split_scratch_bytes(precision, sum of the blocks' cells) bytes.
void split_assign_scratch(int precision, SplitBlock* blocks, int nblocks, void* scratch);
// One RHS (stage 0) or TVD-RK3 stage (1..3) of all blocks: three launches.
int split_stage(fj_ctx* ctx, const SplitBlock* blocks, int nblocks, const Phys& ph, int flags,
                int stage, double dt, int precision, cudaStream_t st);

}  // namespace fj
