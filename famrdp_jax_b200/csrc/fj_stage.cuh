// fj_stage.cuh -- arguments of the fused stage kernel (fj_stage_fused.cu).
#pragma once

#include <cuda_runtime.h>

#include "fj_common.cuh"

namespace fj {

struct StageArgs {
  const double* q;       // stage input (5, ni, nj, nk)
  const double* q0;      // step start state (stages 2, 3), else unused
  const double* kxyz;    // (3, 3, ni, nj, nk) FP64
  const float* kxyz32;   // optional FP32 copy of kxyz (FP32-flux path), or nullptr
  const double* vol;     // (ni, nj, nk)
  double* out;           // RHS (stage 0) or stage result; may alias q0, never q
  int ni, nj, nk;
  int ntj, ntk, seg;     // filled by the launcher
  int flags;             // kRhsInvscd | kRhsViscous
  int stage;             // 0 = RHS only, 1..3 = TVD-RK3 stage
  double dt;
  Phys ph;
};

// One fused launch for one block.  `seg` = planes per CTA along i (0 =
// automatic); `tile` selects the (TJ, TK) tile shape: 0 = 8x32, 1 = 4x32,
// 2 = 6x32, 3 = 8x16.
int fused_stage(fj_ctx* ctx, const StageArgs& a, int seg, int precision, int tile, cudaStream_t st);

}  // namespace fj
