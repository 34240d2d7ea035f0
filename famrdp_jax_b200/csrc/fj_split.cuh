// fj_split.cuh -- the three-kernel stage pipeline over a table of blocks
// (fj_stage_split.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fj_common.cuh"

namespace fj {

constexpr int kMaxSplitBlocks = 64;  // blocks per launch (more are chunked)

// Values per cell of the metric record copy in flux type T: kxyz[l][m]
// l-major (9 values), padded to a multiple of 16 bytes.
template <typename T>
constexpr int kRecK = sizeof(T) == 4 ? 12 : 10;

struct SplitBlock {
  const double* q;       // stage input (5, ni, nj, nk)
  const double* q0;      // step start state (stages 2, 3)
  double* out;           // RHS (stage 0) or stage result; may alias q0, never q
  const double* kxyz;    // (3, 3, ni, nj, nk)
  const void* kaos;      // FP32-flux only: optional FP32 metric records (kRecK per cell), or nullptr
  const double* vol;     // (ni, nj, nk)
  void* prim;            // scratch: the primitives of the stage input (records in FP32)
  void* prim_next;       // where the assembly writes the next stage's primitives: a
                         // second buffer (the assembly also reads prim: its k faces)
  void* F;               // scratch: FP64 10 x N (face c | c+e_a for a = i, j, axis-major); FP32 records of
                         // the i face and the first three j-face components (8 per cell)
  void* Fz;              // FP32 only: the last two j-face components, two per cell
  void* G;               // scratch: viscous flux components (records: 8 per cell)
  void* Gz;              // records only: the ninth component, one per cell
  void* Fk;              // FP32 only: the k face c | c+1 of each cell, 5 per cell (written and read only
                         // by the kernels of tables too small to fill the GPU; zero where no face exists)
  double mu0;            // viscosity scale of this block (per-instance ensembles)
  double dt;             // time step of this block (stages 1..3)
  int ni, nj, nk;
  int cta_begin;         // filled by the launcher
  int cta_begin_asm;     // the same for the FP32 assembly's 248-cell CTAs
};

// Metric records (kRecK values of the flux type per cell) from the caller's
// field-major FP64 kxyz (3, 3, ni, nj, nk): the nine kxyz[l][m] and, in FP32
// records, the three face-normal difference sums the pressure offset uses.
int split_metric_records(const double* kxyz, void* out, int ni, int nj, int nk, int precision, cudaStream_t st);
// Mean pressure over all padded cells of the blocks, on stream st with
// mean_pressure_scratch_bytes(nblocks) bytes of device scratch; waits for st.
size_t mean_pressure_scratch_bytes(int nblocks);
int mean_pressure(const fj_block* blocks, int nblocks, double gm1, double* scratch, cudaStream_t st, double* out);
// Bytes of one block's metric records.
size_t split_metric_record_bytes(int precision, int64_t N);
// Scratch bytes of the intermediates of `cells` padded cells in total.
size_t split_scratch_bytes(int precision, int64_t cells);
// Points prim/F/G of every block into one scratch region of
// split_scratch_bytes(precision, sum of the blocks' cells) bytes.
void split_assign_scratch(int precision, SplitBlock* blocks, int nblocks, void* scratch);
// One RHS (stage 0) or TVD-RK3 stage (1..3) of all blocks: three launches
// (per chunk of kMaxSplitBlocks blocks).  ph supplies everything but mu0,
// which comes per block like dt.
// prims_ready: the blocks' primitives were already written (by the previous
// stage's assembly with next_prims), so the primitive launch is skipped;
// next_prims (stages 1, 2): the assembly also writes the primitives of its
// result for the next stage.
// variant: launch shape of the FP32 record kernels (0 .. FJ_NUM_SPLIT_VARIANTS-1);
// after_fluxes (optional): recorded on st right after the (first) flux launch.
int split_stage(fj_ctx* ctx, const SplitBlock* blocks, int nblocks, const Phys& ph, int flags,
                int stage, int precision, cudaStream_t st, bool prims_ready = false, bool next_prims = false,
                int variant = 0, cudaEvent_t after_fluxes = nullptr);

}  // namespace fj
